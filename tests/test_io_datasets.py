"""File formats and seeded generators (CPU)."""
import math

import numpy as np

from culamp_b200 import datasets as D
from culamp_b200 import io as cio


def test_potential_files_round_trip(tmp_path):
    v = np.array([0.1, -3.25e-17, 1e300, -math.pi])
    prefix = str(tmp_path / "pot")
    cio.write_potentials(prefix, row=v, col=v[::-1], spp_col=v * 2)
    for ext, want in ((".row", v), (".col", v[::-1]), (".spp_col", v * 2)):
        assert np.array_equal(cio.read_potentials(prefix, ext), want)


def test_log_rows_format_and_parse():
    rows = [(0.5, 1, 1e-3, 2.0, math.nan, 3.0), (1.0, 101, 1e-7, 2.5, math.nan, 3.5)]
    text = "\n".join(cio.format_row(r, "sinkhorn_kernel") for r in rows)
    back = cio.parse_log(text)
    assert [b["iter"] for b in back] == [1, 101]
    assert back[1]["infeas"] == 1e-7 and back[0]["solver"] == "sinkhorn_kernel"
    lamp = cio.format_row((0.1, 1, 0.5, 0.2, 0.3, 0.1), "lamp_kernel")
    assert lamp.count(",") == 6


def test_generators_are_seeded_and_shaped():
    x, y, r, c = D.grid_instance(64, 64, "mixture")
    assert x.shape == (4096, 3) and np.all(x[:, 2] == 0)
    assert abs(r.sum() - 1) < 1e-12 and r.min() > 0
    x2, _, r2, _ = D.grid_instance(64, 64, "mixture")
    assert np.array_equal(r, r2)
    g = D.grid_coords(32, 32, scaled=True)
    assert g.max() == 1.0 and g.min() == 0.0
    xf, yf, rf, cf = D.feature_instance(64, 48, 16)
    assert np.allclose(np.linalg.norm(xf, axis=1), 1.0)
    assert (xf >= 0).all() and abs(rf.sum() - 1) < 1e-12
    xr, yr, _, _ = D.rgb_instance(1000, 900)
    assert xr.shape == (1000, 3) and yr.min() >= 0 and yr.max() <= 1
    inst = D.batched_instances(5)
    assert len(inst) == 5 and all(256 <= a[0].shape[0] <= 8192 for a in inst)


def test_dotmark_smoothing():
    v = np.array([0.0, 1.0, 3.0])
    s = D.dotmark_smoothing(v)
    assert abs(s.sum() - 1) < 1e-15 and s[0] > 0
