"""EOTArgs and read_args_json (src/Utilities.jl:18-31, 88-92).

Parsing goes through the C ABI (culamp_args_from_json), the same reader a Julia
caller of the library uses, so both hosts see identical settings.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import asdict, dataclass, fields

from . import _lib


@dataclass
class EOTArgs:
    """Solver settings with the reference's field names and defaults."""
    eta_p: float = 0.0
    eta_mu: float = 0.0
    tau_p: float = 1.0
    tau_mu: float = 1.0
    alpha: float = 0.01
    B: float = 1.0
    epsilon: float = 1e-4
    anneal_mult: float = 0.95
    itermax: int = 10_000
    inner_iter: int = 10
    tmax: float = math.inf
    verbose: bool = True

    def to_c(self) -> _lib.CArgs:
        return _lib.CArgs(float(self.eta_p), float(self.eta_mu), float(self.tau_p),
                          float(self.tau_mu), float(self.alpha), float(self.B),
                          float(self.epsilon), float(self.anneal_mult), int(self.itermax),
                          int(self.inner_iter), float(self.tmax), int(bool(self.verbose)), 0)

    @classmethod
    def from_c(cls, a: _lib.CArgs) -> "EOTArgs":
        return cls(eta_p=a.eta_p, eta_mu=a.eta_mu, tau_p=a.tau_p, tau_mu=a.tau_mu, alpha=a.alpha,
                   B=a.B, epsilon=a.epsilon, anneal_mult=a.anneal_mult, itermax=int(a.itermax),
                   inner_iter=int(a.inner_iter), tmax=a.tmax, verbose=bool(a.verbose))

    def copy(self, **kw) -> "EOTArgs":
        d = asdict(self)
        d.update(kw)
        return EOTArgs(**d)


def default_args() -> EOTArgs:
    a = _lib.CArgs()
    st = _lib.load().culamp_args_default(C.byref(a))
    if st:
        raise _lib.CulampError(st, "culamp_args_default")
    return EOTArgs.from_c(a)


def read_args_json(fpath: str, dtype=float) -> EOTArgs:
    """read_args_json (Utilities.jl:88-92): missing keys keep their defaults."""
    a = _lib.CArgs()
    st = _lib.load().culamp_args_from_json(fpath.encode(), C.byref(a))
    if st:
        raise _lib.CulampError(st, f"cannot read settings {fpath!r}")
    return EOTArgs.from_c(a)


def args_from_json_string(text: str) -> EOTArgs:
    a = _lib.CArgs()
    st = _lib.load().culamp_args_from_json_string(text.encode(), C.byref(a))
    if st:
        raise _lib.CulampError(st, "invalid settings JSON")
    return EOTArgs.from_c(a)


ARG_FIELDS = tuple(f.name for f in fields(EOTArgs))
