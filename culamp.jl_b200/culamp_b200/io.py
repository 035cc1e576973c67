"""File formats of the kernelized solvers.

* Potentials: one value per line in `<prefix>.row`, `<prefix>.col` and (LAMP)
  `<prefix>.spp_col` (SinkhornKernel.jl:581-593, MirrorProxKernel.jl:1152-1170).
  Values are written with 17 significant digits so they read back bit-exactly
  (Julia's `println` prints the shortest round-trip form of the same double).
* Convergence log: the CSV rows the reference prints,
  `time(s),iter,infeas,ot_objective,[primal,]dual,solver` (SinkhornKernel.jl:533,
  MirrorProxKernel.jl:1097), so existing log parsers keep working.
"""
from __future__ import annotations

import math

import numpy as np


def write_potentials(prefix: str, row=None, col=None, spp_col=None) -> None:
    for ext, v in ((".spp_col", spp_col), (".row", row), (".col", col)):
        if v is None:
            continue
        with open(prefix + ext, "w") as f:
            for x in np.asarray(v, dtype=np.float64).ravel():
                f.write(f"{float(x)!r}\n")


def read_potentials(prefix: str, ext: str) -> np.ndarray:
    with open(prefix + ext) as f:
        return np.array([float(line) for line in f if line.strip()], dtype=np.float64)


def write_assignments(path: str, img) -> None:
    """Barycentric image, one point per line (the reference writes the whole
    array per index, SinkhornKernel.jl:594-607; one row per point is the
    readable equivalent)."""
    a = np.asarray(img, dtype=np.float64)
    with open(path, "w") as f:
        for i, pt in enumerate(a.reshape(a.shape[0], -1)):
            f.write(",".join(repr(float(v)) for v in pt) + f",{i + 1}\n")


def format_row(row, solver: str, eta_col: bool = False) -> str:
    t, it, infeas, obj, primal, dual = row
    if eta_col:   # annealed Sinkhorn: time,iter,infeas,ot_objective,eta,solver
        return f"{t:.6e},{it},{infeas:.14e},{obj:.14e},{dual:.14e},{solver}"
    if solver == "sinkhorn_kernel":
        return f"{t:.6e},{it},{infeas:.14e},{obj:.14e},{dual:.14e},{solver}"
    return f"{t:.6e},{it},{infeas:.14e},{obj:.14e},{primal:.14e},{dual:.14e},{solver}"


def print_log(rows, solver: str, header: str | None = None, eta_col: bool = False) -> None:
    if header:
        print(header)
    for r in rows:
        print(format_row(r, solver, eta_col))


def parse_log(text: str):
    """Parse CSV log rows (either layout) back into dicts."""
    out = []
    for line in text.strip().splitlines():
        parts = line.split(",")
        if not parts or not parts[0] or parts[0].startswith("time"):
            continue
        vals = [float(p) if p not in ("", "nan") else math.nan for p in parts[:-1]]
        out.append({"time": vals[0], "iter": int(vals[1]), "infeas": vals[2],
                    "ot_objective": vals[3], "rest": vals[4:], "solver": parts[-1]})
    return out
