"""Seeded synthetic permeability fields in the SPE10 layout.

The reference reads the SPE10 model-2 file ``spe_perm.dat`` (3 x 1,122,000
values: the kx block, then ky, then kz; cell (i, j, k) of the 60x220x85 field is
entry ``k*13200 + j*60 + i``; modules/mesh/spe.cc:32-43, mesh.h:57-59). That file is
not distributed with the code, so the benchmark problems use seeded synthetic
fields of the same shape and layout. Every generator returns the full 60x220x85
field; a smaller grid (nx, ny, nz) uses the corner sub-block, exactly as
``SPEMesh::index_k`` does.

Models:
  * ``iid``       log10 kx ~ N(1.0, 1.5^2) i.i.d. per cell, clipped to [-3, 4.3];
  * ``layered``   layers 1-35 smooth, log10 k ~ N(1.5, 1.0^2) with a 3-cell box
                  filter; layers 36-85 channelised: binary facies from a seeded
                  Gaussian field elongated 20:1 along y thresholded at 40% sand,
                  sand log10 k ~ N(2.8, 0.4^2), shale log10 k ~ N(-1.5, 1.0^2).
In both, ky = kx and kz = 0.1 kx.
"""
from __future__ import annotations

import numpy as np

KNX, KNY, KNZ = 60, 220, 85
KN = KNX * KNY * KNZ


def _box3(a: np.ndarray) -> np.ndarray:
    """3-cell box filter along every axis (edges use the cells that exist)."""
    out = a.astype(np.float64, copy=True)
    for ax in range(a.ndim):
        s = np.zeros_like(out)
        c = np.zeros_like(out)
        n = out.shape[ax]
        for d in (-1, 0, 1):
            src = [slice(None)] * out.ndim
            dst = [slice(None)] * out.ndim
            if d < 0:
                src[ax] = slice(0, n + d)
                dst[ax] = slice(-d, n)
            elif d > 0:
                src[ax] = slice(d, n)
                dst[ax] = slice(0, n - d)
            s[tuple(dst)] += out[tuple(src)]
            c[tuple(dst)] += 1.0
        out = s / c
    return out


def _gauss1d(a: np.ndarray, sigma: float, ax: int) -> np.ndarray:
    """Separable Gaussian smoothing along one axis with reflecting edges."""
    if sigma <= 0:
        return a
    r = int(np.ceil(3 * sigma))
    w = np.exp(-0.5 * (np.arange(-r, r + 1) / sigma) ** 2)
    w /= w.sum()
    pad = [(0, 0)] * a.ndim
    pad[ax] = (r, r)
    p = np.pad(a, pad, mode="reflect" if a.shape[ax] > r else "edge")
    out = np.zeros_like(a)
    n = a.shape[ax]
    for t, wt in enumerate(w):
        sl = [slice(None)] * a.ndim
        sl[ax] = slice(t, t + n)
        out += wt * p[tuple(sl)]
    return out


def log10k_iid(seed: int, mean: float = 1.0, sd: float = 1.5,
               lo: float = -3.0, hi: float = 4.3) -> np.ndarray:
    """i.i.d. clipped normal log10 kx, shape (KNZ, KNY, KNX)."""
    rng = np.random.default_rng(seed)
    z = rng.standard_normal((KNZ, KNY, KNX))
    return np.clip(mean + sd * z, lo, hi)


def log10k_layered(seed: int) -> np.ndarray:
    """Smooth top (layers 1-35) over channelised bottom (36-85), (KNZ, KNY, KNX)."""
    rng = np.random.default_rng(seed)
    out = np.empty((KNZ, KNY, KNX))
    top = _box3(rng.standard_normal((35, KNY, KNX)))
    top = (top - top.mean()) / top.std()
    out[:35] = 1.5 + 1.0 * top
    g = rng.standard_normal((50, KNY, KNX))
    g = _gauss1d(g, 1.0, 2)   # x
    g = _gauss1d(g, 20.0, 1)  # y: 20:1 elongation
    g = _gauss1d(g, 1.0, 0)   # z
    thr = np.quantile(g, 0.60)           # top 40% is sand
    sand = g > thr
    sand_v = 2.8 + 0.4 * rng.standard_normal(sand.shape)
    shale_v = -1.5 + 1.0 * rng.standard_normal(sand.shape)
    out[35:] = np.where(sand, sand_v, shale_v)
    return out


def perm_from_log10(l10: np.ndarray):
    """kx = 10**l10, ky = kx, kz = 0.1*kx, each flattened in SPE10 order."""
    kx = np.power(10.0, l10).reshape(-1)
    return kx, kx.copy(), 0.1 * kx


def field(model: str, seed: int):
    """(kx, ky, kz) float64 arrays of length KN for a named model."""
    if model == "iid":
        return perm_from_log10(log10k_iid(seed))
    if model == "layered":
        return perm_from_log10(log10k_layered(seed))
    raise ValueError(f"unknown field model {model!r}")


def write_perm_bin(path: str, kx, ky, kz) -> None:
    """kx, ky, kz blocks as raw float64, the binary twin of spe_perm.dat."""
    np.concatenate([np.asarray(kx, np.float64), np.asarray(ky, np.float64),
                    np.asarray(kz, np.float64)]).tofile(path)
