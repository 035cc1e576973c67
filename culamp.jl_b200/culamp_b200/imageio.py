"""Image inputs of the colour-transfer path: PNG load / save and KDE marginals.

load_rgb (ImgUtilities.jl:30-52) reads an RGB image, flattens it to a point
cloud (one point per pixel, coordinates = the channels in [0, 1]) and, unless
uniform marginals are asked for, weights every pixel by a kernel density
estimate of its colour: per channel a Gaussian KDE on a grid of the next
power of two above the pixel count (KernelDensity.jl `kde(x, npoints=...)`),
the grid density divided by its 2-norm (`normalize!`), evaluated at the
pixel's value (`pdf`), the three channel densities summed and the result
normalised to sum 1. save_image (:56-59) writes a flattened cloud back as an
RGB image.

KernelDensity.jl is not vendored with the reference (a Project.toml
dependency, unpinned). Its published algorithm is restated here: Silverman's
bandwidth 0.9 * min(std, IQR / 1.34) * n^(-1/5); a grid from min - 4 h to
max + 4 h; linear binning of the data onto the grid; circular convolution
with the Gaussian kernel through the FFT (the kernel's characteristic
function); quadratic spline interpolation of the grid density at the data.
No reference output pins these numbers (parity unpinned at this boundary).

Images are decoded and encoded by a small PNG codec (zlib + the five PNG row
filters), 8- and 16-bit grey / grey-alpha / RGB / RGBA / palette, without
interlacing; alpha is dropped and grey is replicated to three channels.
Pixel order of the flattened cloud follows Julia's column-major
reshape of the (channels, height, width) channel view: point i = y + height * x.
"""
from __future__ import annotations

import math
import struct
import zlib

import numpy as np

_SIG = b"\x89PNG\r\n\x1a\n"


# ------------------------------------------------------------------ PNG codec

def _chunks(data: bytes):
    if data[:8] != _SIG:
        raise ValueError("not a PNG file")
    k = 8
    while k < len(data):
        (length,) = struct.unpack(">I", data[k:k + 4])
        kind = data[k + 4:k + 8]
        body = data[k + 8:k + 8 + length]
        (crc,) = struct.unpack(">I", data[k + 8 + length:k + 12 + length])
        if zlib.crc32(kind + body) & 0xFFFFFFFF != crc:
            raise ValueError(f"PNG chunk {kind!r}: CRC mismatch")
        yield kind, body
        k += 12 + length


def _unfilter(raw: bytes, h: int, stride: int, bpp: int) -> np.ndarray:
    """Undo the per-row PNG filters (None, Sub, Up, Average, Paeth)."""
    rows = np.frombuffer(raw, dtype=np.uint8).reshape(h, stride + 1)
    out = np.zeros((h, stride), dtype=np.uint8)
    prev = np.zeros(stride, dtype=np.int32)
    for y in range(h):
        f = int(rows[y, 0])
        cur = rows[y, 1:].astype(np.int32)
        if f == 0:
            rec = cur
        elif f == 1:      # Sub: cumulative sum along each byte lane of the pixel
            rec = np.cumsum(cur.reshape(-1, bpp), axis=0).reshape(-1) & 0xFF
        elif f == 2:      # Up
            rec = (cur + prev) & 0xFF
        elif f in (3, 4):  # Average / Paeth: sequential in the left neighbour
            rec = np.zeros(stride, dtype=np.int32)
            for x in range(0, stride, bpp):
                a = rec[x - bpp:x] if x >= bpp else np.zeros(bpp, dtype=np.int32)
                b = prev[x:x + bpp]
                if f == 3:
                    pred = (a + b) >> 1
                else:
                    c = prev[x - bpp:x] if x >= bpp else np.zeros(bpp, dtype=np.int32)
                    p = a + b - c
                    pa, pb, pc = np.abs(p - a), np.abs(p - b), np.abs(p - c)
                    pred = np.where((pa <= pb) & (pa <= pc), a, np.where(pb <= pc, b, c))
                rec[x:x + bpp] = (cur[x:x + bpp] + pred) & 0xFF
        else:
            raise ValueError(f"PNG row filter {f} unknown")
        out[y] = rec
        prev = rec
    return out


def read_png(path: str) -> np.ndarray:
    """PNG file -> float64 array (height, width, 3) in [0, 1]."""
    with open(path, "rb") as f:
        data = f.read()
    hdr, idat, palette = None, [], None
    for kind, body in _chunks(data):
        if kind == b"IHDR":
            hdr = struct.unpack(">IIBBBBB", body)
        elif kind == b"PLTE":
            palette = np.frombuffer(body, dtype=np.uint8).reshape(-1, 3)
        elif kind == b"IDAT":
            idat.append(body)
    if hdr is None:
        raise ValueError("PNG without IHDR")
    w, h, depth, ctype, _, _, interlace = hdr
    if interlace:
        raise ValueError("interlaced PNG is not supported")
    channels = {0: 1, 2: 3, 3: 1, 4: 2, 6: 4}[ctype]
    if depth not in (8, 16) or (ctype == 3 and depth != 8):
        raise ValueError(f"PNG bit depth {depth} (colour type {ctype}) is not supported")
    bpp = channels * depth // 8
    pix = _unfilter(zlib.decompress(b"".join(idat)), h, w * bpp, bpp)
    if depth == 16:
        v = pix.reshape(h, w, channels, 2).astype(np.uint32)
        img = ((v[..., 0] << 8) | v[..., 1]).astype(np.float64) / 65535.0
    else:
        img = pix.reshape(h, w, channels).astype(np.float64) / 255.0
    if ctype == 3:
        if palette is None:
            raise ValueError("palette PNG without PLTE")
        img = palette[pix.reshape(h, w)].astype(np.float64) / 255.0
    elif ctype in (0, 4):
        img = np.repeat(img[..., :1], 3, axis=2)
    else:
        img = img[..., :3]
    return img


def _chunk(kind: bytes, body: bytes) -> bytes:
    return struct.pack(">I", len(body)) + kind + body + struct.pack(">I", zlib.crc32(kind + body) & 0xFFFFFFFF)


def write_png(path: str, img, filters=None) -> None:
    """float array (height, width, 3) in [0, 1] -> 8-bit RGB PNG. `filters`
    (one PNG filter type per row, default all 0) exists for codec tests."""
    a = np.clip(np.rint(np.asarray(img, dtype=np.float64) * 255.0), 0, 255).astype(np.uint8)
    h, w, _ = a.shape
    rows = a.reshape(h, w * 3).astype(np.int32)
    out = bytearray()
    prev = np.zeros(w * 3, dtype=np.int32)
    for y in range(h):
        f = 0 if filters is None else int(filters[y % len(filters)])
        cur = rows[y]
        left = np.concatenate([np.zeros(3, dtype=np.int32), cur[:-3]])
        upleft = np.concatenate([np.zeros(3, dtype=np.int32), prev[:-3]])
        if f == 0:
            enc = cur
        elif f == 1:
            enc = cur - left
        elif f == 2:
            enc = cur - prev
        elif f == 3:
            enc = cur - ((left + prev) >> 1)
        else:
            p = left + prev - upleft
            pa, pb, pc = np.abs(p - left), np.abs(p - prev), np.abs(p - upleft)
            enc = cur - np.where((pa <= pb) & (pa <= pc), left, np.where(pb <= pc, prev, upleft))
        out.append(f)
        out += (enc & 0xFF).astype(np.uint8).tobytes()
        prev = cur
    data = _SIG + _chunk(b"IHDR", struct.pack(">IIBBBBB", w, h, 8, 2, 0, 0, 0))
    data += _chunk(b"IDAT", zlib.compress(bytes(out), 9)) + _chunk(b"IEND", b"")
    with open(path, "wb") as f:
        f.write(data)


def resize_bilinear(img: np.ndarray, height: int, width: int) -> np.ndarray:
    """Bilinear resampling to (height, width) with pixel centres aligned."""
    h, w, _ = img.shape
    if (h, w) == (height, width):
        return img.copy()
    ys = np.clip((np.arange(height) + 0.5) * h / height - 0.5, 0, h - 1)
    xs = np.clip((np.arange(width) + 0.5) * w / width - 0.5, 0, w - 1)
    y0, x0 = np.floor(ys).astype(int), np.floor(xs).astype(int)
    y1, x1 = np.minimum(y0 + 1, h - 1), np.minimum(x0 + 1, w - 1)
    fy, fx = (ys - y0)[:, None, None], (xs - x0)[None, :, None]
    top = img[y0][:, x0] * (1 - fx) + img[y0][:, x1] * fx
    bot = img[y1][:, x0] * (1 - fx) + img[y1][:, x1] * fx
    return top * (1 - fy) + bot * fy


# ------------------------------------------------------------------ KDE

def kde_bandwidth(x: np.ndarray) -> float:
    """Silverman's rule as KernelDensity.jl states it: 0.9 min(std, IQR/1.34) n^(-1/5)."""
    x = np.asarray(x, dtype=np.float64)
    q75, q25 = np.percentile(x, [75, 25])
    width = min(np.std(x, ddof=1) if x.size > 1 else 0.0, (q75 - q25) / 1.34)
    if not width > 0:
        width = np.std(x, ddof=1) if x.size > 1 else 0.0
    if not width > 0:
        width = 1.0
    return 0.9 * width * x.size ** (-0.2)


def kde_grid(x: np.ndarray, npoints: int, bandwidth: float | None = None):
    """Gaussian KDE of x tabulated on npoints grid points (lo - 4h .. hi + 4h):
    linear binning, then circular convolution with N(0, h) via the FFT.
    Returns (grid, density) with density integrating to ~1 over the grid."""
    x = np.asarray(x, dtype=np.float64)
    h = kde_bandwidth(x) if bandwidth is None else bandwidth
    lo, hi = x.min() - 4.0 * h, x.max() + 4.0 * h
    grid = np.linspace(lo, hi, npoints)
    step = grid[1] - grid[0]
    pos = (x - lo) / step
    j = np.clip(np.floor(pos).astype(np.int64), 0, npoints - 2)
    fr = pos - j
    binned = np.zeros(npoints)
    np.add.at(binned, j, 1.0 - fr)
    np.add.at(binned, j + 1, fr)
    binned /= x.size * step
    freq = np.fft.rfftfreq(npoints, d=step)
    cf = np.exp(-0.5 * (2.0 * math.pi * freq * h) ** 2)   # Gaussian characteristic function
    density = np.fft.irfft(np.fft.rfft(binned) * cf, n=npoints)
    return grid, np.maximum(density, 0.0)


def kde_pdf(grid: np.ndarray, density: np.ndarray, x: np.ndarray) -> np.ndarray:
    """Quadratic spline interpolation of the grid density at x."""
    from scipy.interpolate import make_interp_spline
    return make_interp_spline(grid, density, k=2)(np.asarray(x, dtype=np.float64))


def kde_marginal(points: np.ndarray) -> np.ndarray:
    """ImgUtilities.jl:35-45: per-channel KDE (npoints = next power of two of
    the pixel count), each grid density divided by its 2-norm, evaluated at the
    pixels, summed over channels and normalised to sum 1."""
    pts = np.asarray(points, dtype=np.float64)
    n = pts.shape[0]
    npoints = int(2 ** math.ceil(math.log2(n)))
    total = np.zeros(n)
    for ch in range(pts.shape[1]):
        grid, dens = kde_grid(pts[:, ch], npoints)
        dens = dens / np.linalg.norm(dens)
        total += kde_pdf(grid, dens, pts[:, ch])
    return total / np.abs(total).sum()


# ------------------------------------------------------------------ reference API

def load_rgb(filepath: str, resolution: tuple = (), uniform_marginal: bool = False):
    """ImgUtilities.jl:30-52. Returns (points (N, 3), original_shape, marginal):
    points in [0, 1], one per pixel in column-major pixel order (i = y + h x),
    original_shape = (3, height, width)."""
    img = read_png(filepath)
    if resolution:
        img = resize_bilinear(img, int(resolution[0]), int(resolution[1]))
    h, w, _ = img.shape
    points = np.ascontiguousarray(img.transpose(1, 0, 2).reshape(h * w, 3))
    marginal = np.full(h * w, 1.0 / (h * w)) if uniform_marginal else kde_marginal(points)
    return points, (3, h, w), marginal


def save_image(path: str, flattened, original_shape: tuple) -> None:
    """ImgUtilities.jl:56-59: a flattened cloud (N, 3) back to an RGB PNG."""
    _, h, w = original_shape
    pts = np.asarray(flattened, dtype=np.float64).reshape(w, h, 3).transpose(1, 0, 2)
    write_png(path, pts)
