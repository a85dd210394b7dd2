"""numpy restatement of CUBE's checkpoint power spectrum -- test infrastructure.

cicpower.f90:84-163 (CIC of unit-mass particles on ng^3 nodes centred in the
fine cells, delta = rho/mean - 1), cicpower.f90:199-214 (neutrino density
contrast sampled at the fine-cell centres) and powerspectrum.f90:27-137
(cross_power: mode skipping, |k| bins, CIC window, Delta^2 = |c|^2 4 pi k^3).
Sums in float64 (the reference's are FP32).
"""
from __future__ import annotations

import numpy as np


def particle_positions(st) -> np.ndarray:
    """Global coarse-cell coordinates [np, 3] of a checkpoint-layout state."""
    nc, nnt = st.nc, st.nnt
    nt = nc // nnt
    cells = np.arange(nc ** 3)
    l = cells % (nt ** 3)
    tile = cells // (nt ** 3)
    lx, ly, lz = l % nt, (l // nt) % nt, l // (nt * nt)
    tx, ty, tz = tile % nnt, (tile // nnt) % nnt, tile // (nnt * nnt)
    g = np.stack([tx * nt + lx, ty * nt + ly, tz * nt + lz], axis=1)
    cell_of = np.repeat(np.arange(nc ** 3), st.rhoc.astype(np.int64))
    mask = 0xFF if st.izipx == 1 else 0xFFFF
    u = (st.xp.astype(np.int64) & mask).astype(np.float64)
    frac = (u + 0.5) / (256.0 if st.izipx == 1 else 65536.0)
    return g[cell_of].astype(np.float64) + frac


def cic_delta(pos: np.ndarray, nc: int, ng: int) -> np.ndarray:
    p = (pos.astype(np.float32) * np.float32(ng) / np.float32(nc) - np.float32(0.5)).astype(np.float64)
    i0 = np.floor(p).astype(np.int64)
    w1 = (i0 + 1) - p
    rho = np.zeros((ng, ng, ng))
    for c in range(8):
        o = [(c >> d) & 1 for d in range(3)]
        w = np.ones(len(p))
        idx = []
        for d in range(3):
            w = w * (w1[:, d] if o[d] == 0 else 1.0 - w1[:, d])
            idx.append((i0[:, d] + o[d]) % ng)
        np.add.at(rho, (idx[2], idx[1], idx[0]), w)
    return rho / (rho.sum() / ng ** 3) - 1.0


def nu_delta(fluids, weights, ng: int) -> np.ndarray:
    """sum_k w_k CIC(rho_k)(n + 1/2) - 1 at every fine node n (hydrogr.f90:312-346)."""
    q = np.arange(ng) + 0.5
    out = np.zeros((ng, ng, ng))
    for fl, w in zip(fluids, weights):
        n = fl.shape[0]
        dx = ng // n
        xx = q / dx - 0.5
        lo = np.floor(xx).astype(int)
        d1 = (lo + 1) - xx
        r = fl[..., 0].astype(np.float64)
        den = np.zeros((ng, ng, ng))
        for c in range(8):
            ox, oy, oz = c & 1, (c >> 1) & 1, c >> 2
            wx = d1 if ox == 0 else 1 - d1
            ix = (lo + ox) % n
            den += (r[np.ix_((lo + oz) % n, (lo + oy) % n, ix)] * wx[None, None, :] *
                    (d1 if oy == 0 else 1 - d1)[None, :, None] * (d1 if oz == 0 else 1 - d1)[:, None, None])
        out += w * den
    return out - 1.0


def cross_power(d1: np.ndarray, d2: np.ndarray | None, box: float, log_bins: bool = False) -> np.ndarray:
    """xip(10, nbin) of powerspectrum.f90 as [nbin, 10]."""
    ng = d1.shape[0]
    nyq = ng // 2
    c1 = np.fft.rfftn(d1) / ng ** 3  # [kz][ky][kx], kx = 0..nyq
    c2 = np.fft.rfftn(d2) / ng ** 3 if d2 is not None else np.zeros_like(c1)
    kz, ky, kx = np.meshgrid(np.arange(ng), np.arange(ng), np.arange(nyq + 1), indexing="ij")
    ig, jg, kg = kx + 1, ky + 1, kz + 1
    skip = (ig == 1) & (jg == 1) & (kg == 1)
    skip |= ((ig == 1) | (ig == nyq + 1)) & (jg > nyq + 1)
    skip |= ((ig == 1) | (ig == nyq + 1)) & ((jg == 1) | (jg == nyq + 1)) & (kg > nyq + 1)
    f = [((g + nyq - 1) % ng - nyq).astype(np.float64) for g in (ig, jg, kg)]
    kr = np.sqrt(f[0] ** 2 + f[1] ** 2 + f[2] ** 2)
    sinc = np.ones_like(kr)
    for v in f:
        a = np.pi * v / ng
        sinc *= np.where(v == 0, 1.0, np.sin(np.where(v == 0, 1.0, a)) / np.where(v == 0, 1.0, a))
    if log_bins:
        nbin = int(np.floor(4 * np.log(nyq * np.sqrt(3.0) / 0.95) / np.log(2.0)))
        with np.errstate(divide="ignore"):
            rb = 4.0 / np.log(2.0) * np.log(np.where(kr > 0, kr, 1.0) / 0.95)
        ib = np.where(rb < 1, np.ceil(rb), np.floor(rb)).astype(int)
    else:
        nbin = int(np.rint(nyq * np.sqrt(3.0)))
        ib = np.floor(kr + 0.5).astype(int)
    keep = (~skip) & (ib >= 0) & (ib <= nbin)
    w = 4 * np.pi * kr ** 3 / sinc ** 4
    a11 = (np.abs(c1) ** 2) * w
    a22 = (np.abs(c2) ** 2) * w
    a12 = (c1.real * c2.real + c1.imag * c2.imag) * w
    xi = np.zeros((7, nbin + 1))
    for q, v in enumerate((np.ones_like(kr), kr, a11, a22, a12, 1 / sinc ** 2, 1 / sinc ** 4)):
        xi[q] = np.bincount(ib[keep], weights=v[keep], minlength=nbin + 1)[: nbin + 1]
    x = xi[:, 1:]
    out = np.zeros((nbin, 10))
    with np.errstate(divide="ignore", invalid="ignore"):
        out[:, 0] = x[0]
        out[:, 1] = x[1] / x[0] * 2 * np.pi / box
        for q in range(2, 7):
            out[:, q] = x[q] / x[0]
        out[:, 7] = out[:, 4] / np.sqrt(out[:, 2] * out[:, 3])
        out[:, 8] = np.sqrt(out[:, 3] / out[:, 2])
        out[:, 9] = out[:, 7] ** 4 / out[:, 8] ** 2 * out[:, 3]
    return out
