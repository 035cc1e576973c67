"""PNG codec and KDE marginals of the colour-transfer inputs (ImgUtilities.jl:30-59).

CPU tests: the PNG reader against images written with every row filter, and
the binned-FFT Gaussian KDE against a direct kernel sum at the data points.
"""
import math

import numpy as np
import pytest

from culamp_b200 import imageio as I


def _img(h, w, seed):
    g = np.random.Generator(np.random.PCG64(seed))
    return np.rint(g.uniform(0, 255, size=(h, w, 3))) / 255.0


@pytest.mark.parametrize("filters", [None, [1], [2], [3], [4], [0, 1, 2, 3, 4]])
def test_png_round_trip_every_filter(tmp_path, filters):
    img = _img(13, 17, 1)
    path = str(tmp_path / "x.png")
    I.write_png(path, img, filters=filters)
    back = I.read_png(path)
    assert back.shape == (13, 17, 3)
    assert np.array_equal(np.rint(back * 255), np.rint(img * 255))


def test_png_rejects_bad_crc(tmp_path):
    path = str(tmp_path / "x.png")
    I.write_png(path, _img(4, 4, 2))
    data = bytearray(open(path, "rb").read())
    data[-20] ^= 0xFF                       # inside the IDAT body
    open(path, "wb").write(bytes(data))
    with pytest.raises(ValueError):
        I.read_png(path)


def test_load_and_save_keep_pixel_order(tmp_path):
    img = _img(6, 9, 3)
    path = str(tmp_path / "a.png")
    I.write_png(path, img)
    pts, shape, marg = I.load_rgb(path, uniform_marginal=True)
    assert shape == (3, 6, 9) and pts.shape == (54, 3)
    # column-major pixel order of the (channels, height, width) view: i = y + h x
    assert np.allclose(pts[2 + 6 * 4], img[2, 4])
    assert np.allclose(marg, 1.0 / 54)
    out = str(tmp_path / "b.png")
    I.save_image(out, pts, shape)
    assert np.array_equal(np.rint(I.read_png(out) * 255), np.rint(img * 255))


def test_resize_bilinear_identity_and_shape():
    img = _img(8, 8, 4)
    assert np.array_equal(I.resize_bilinear(img, 8, 8), img)
    r = I.resize_bilinear(img, 4, 5)
    assert r.shape == (4, 5, 3) and r.min() >= img.min() - 1e-12 and r.max() <= img.max() + 1e-12


def test_kde_matches_direct_gaussian_sum():
    g = np.random.Generator(np.random.PCG64(5))
    x = np.concatenate([g.normal(0.3, 0.05, 3000), g.normal(0.7, 0.1, 1000)])
    grid, dens = I.kde_grid(x, 4096)
    h = I.kde_bandwidth(x)
    assert np.sum(dens) * (grid[1] - grid[0]) == pytest.approx(1.0, rel=1e-6)
    pts = np.linspace(0.2, 0.9, 50)
    direct = np.exp(-0.5 * ((pts[:, None] - x[None, :]) / h) ** 2).sum(1) / (x.size * h * math.sqrt(2 * math.pi))
    np.testing.assert_allclose(I.kde_pdf(grid, dens, pts), direct, rtol=2e-3, atol=1e-3)


def test_kde_marginal_sums_to_one_and_favours_dense_colours():
    g = np.random.Generator(np.random.PCG64(6))
    pts = np.clip(np.concatenate([g.normal(0.2, 0.02, (900, 3)), g.uniform(0, 1, (100, 3))]), 0, 1)
    m = I.kde_marginal(pts)
    assert m.shape == (1000,) and np.all(m > 0)
    assert m.sum() == pytest.approx(1.0, rel=1e-12)
    assert m[:900].mean() > 3 * m[900:].mean()
