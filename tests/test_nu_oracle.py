"""CPU tests of the oracle's fluid neutrinos (hydrodf.f90, hydrogr.f90, hydro3d.f90,
hydro1d.f90) against an independent numpy restatement.

The numpy restatement below works on the periodic interior only (np.roll in place
of the halo cells), while the oracle keeps the reference's halo layout
(fld(5,1-ncb:nc+ncb,...), hg_buffer between the evolve calls).  Bit-identical
results pin both: the oracle's literal transcription, and the claim the CUDA
sweeps rely on, that with ncb >= 2 the halo form equals the periodic form.
"""
from __future__ import annotations

import numpy as np
import pytest

from cube_nufluid_b200 import ic
from cube_nufluid_b200.tables import read_coarse_table, read_fine_table
from helpers import nu_params
from oracle_ref import Oracle

f32 = np.float32
GAMMA = f32(5.0) / f32(3.0)

def oracle(p):
    fk, ck = read_fine_table(nf_cutoff=p.nf_cutoff), read_coarse_table()
    return Oracle(p, fk, ck, build_kernels=False)


# ---- numpy restatement of hydro1d / hydro3d on periodic pencils (axis 1) ----
def _mm(a, b, c):
    sa, sb, sc = np.copysign(f32(1), a), np.copysign(f32(1), b), np.copysign(f32(1), c)
    return ((f32(0.25) * np.abs(sa + sb)) * (sa + sc)) * np.minimum(np.minimum(np.abs(a), np.abs(b)), np.abs(c))


def _lb(u):
    um, up = np.roll(u, 1, axis=0), np.roll(u, -1, axis=0)
    return u + f32(0.5) * _mm(f32(1.5) * (u - um), f32(0.5) * (up - um), f32(1.5) * (up - u))


def _rb(u):
    up, upp = np.roll(u, -1, axis=0), np.roll(u, -2, axis=0)
    return up - f32(0.5) * _mm(f32(1.5) * (up - u), f32(0.5) * (upp - u), f32(1.5) * (upp - up))


def _kin(h):
    return (f32(0.5) * ((h[1] * h[1] + h[2] * h[2]) + h[3] * h[3])) / h[0]


def _pres(h, g):
    return np.maximum(f32(0), (h[4] - _kin(h)) * (g - f32(1)))


def _flux(h, g):
    p = _pres(h, g)
    m = h[1]
    return [m, m * (h[1] / h[0]) + p, m * (h[2] / h[0]), m * (h[3] / h[0]), h[4] * (h[1] / h[0])]


def _evolve_pencils(h, g, dt, dx):
    """h: list of 5 arrays [n, ...], sweep along axis 0, periodic."""
    p = _pres(h, g)
    hl, hr = [None] * 5, [None] * 5
    hl[0], hr[0] = _lb(h[0]), _rb(h[0])
    for d in (1, 2, 3):
        v = h[d] / h[0]
        hl[d], hr[d] = hl[0] * _lb(v), hr[0] * _rb(v)
    hl[4] = _lb(p) / (g - f32(1)) + _kin(hl)
    hr[4] = _rb(p) / (g - f32(1)) + _kin(hr)
    fl, fr = _flux(hl, g), _flux(hr, g)
    vl, vr = hl[1] / hl[0], hr[1] / hr[0]
    sl, sr = np.sqrt(_pres(hl, g) / hl[0]), np.sqrt(_pres(hr, g) / hr[0])
    ap = np.maximum(np.maximum(f32(0), vl + sl), vr + sr)
    am = np.maximum(np.maximum(f32(0), -vl + sl), -vr + sr)
    out = []
    for d in range(5):
        f = ((ap * fl[d] + am * fr[d]) - (ap * am) * (hr[d] - hl[d])) / (ap + am)
        r = -f + np.roll(f, 1, axis=0)
        out.append(h[d] + (dt * r) / dx)
    return out


def np_sweep(fld, axis, g, dt, dx):
    """fld [nc,nc,nc,5] (z,y,x,c); axis 0=x, 1=y, 2=z; the normal momentum goes to slot 2."""
    comp = [0, 1 + axis, 1 + (1 if axis != 1 else 0), 3 if axis != 2 else 1, 4]
    if axis == 0:
        comp = [0, 1, 2, 3, 4]
    elif axis == 1:
        comp = [0, 2, 1, 3, 4]
    else:
        comp = [0, 3, 2, 1, 4]
    arr_axis = 2 - axis  # x is the last array axis
    h = [np.moveaxis(fld[..., c], arr_axis, 0) for c in comp]
    o = _evolve_pencils(h, g, dt, dx)
    out = np.empty_like(fld)
    for slot, c in enumerate(comp):
        out[..., c] = np.moveaxis(o[slot], 0, arr_axis)
    return out


def np_timestep(fld, g, dx):
    rho = fld[..., 0]
    v = [np.abs(fld[..., 1 + d] / rho) for d in range(3)]
    h = [fld[..., c] for c in range(5)]
    s = np.sqrt(_pres(h, g) / rho)
    vmax = np.maximum(np.maximum(np.maximum(f32(0), v[0].max(axis=2)), v[1].max(axis=2)), v[2].max(axis=2))
    dts = (f32(0.71) * dx) / (vmax + s.max(axis=2))
    dt = f32(min(f32(1e9), dts.min()))
    return f32(1.0) if dt == f32(1e9) else dt


def np_evolve(fld, g, dt, dx, direction):
    order = (0, 1, 2) if direction > 0 else (2, 1, 0)
    for ax in order:
        fld = np_sweep(fld, ax, g, f32(dt), dx)
    return fld


# ---- tests --------------------------------------------------------------------
def test_fluid_setup_constants():
    p = nu_params()
    o = oracle(p)
    info = o.nu_info()
    nf = p.nc * p.ncell
    assert list(info["nc"]) == [nf // 2, nf // 4, nf // 8]
    # ncb = max(2, 1+floor(ncb*ncell/dx)) (hydrogr.f90:50)
    assert list(info["ncb"]) == [max(2, 1 + int(24 // d)) for d in (2, 4, 8)]
    # the reference prints the unnormalised weight sum beside 1.80305 = 3 zeta(3)/2, the
    # Fermi-Dirac integral the 3-point Gauss-Laguerre sum approximates (hydrodf.f90:80)
    v = np.array([0.41577456, 2.29428036, 6.28994508], f32)
    w = np.array([0.71109301, 0.27851773, 0.01038926], f32)
    raw = (w * ((v * v) / (np.exp(v) + f32(1)))) * np.exp(v)
    assert abs(float(raw.sum()) / 1.80305 - 1.0) < 0.01
    # numpy's float32 exp and the C library's expf may differ in the last place
    np.testing.assert_array_max_ulp(info["dwgts"], (raw / ((raw[0] + raw[1]) + raw[2])).astype(f32), maxulp=2)
    # sound speed: cs = GL_v/beta*c km/s in units of hg_dv (hydrodf.f90:71, hydrogr.f90:66)
    beta = f32(5966.34) * f32(0.1)
    hg_dv = f32(2 * nf) / ((f32(300.0) * np.sqrt(f32(p.omega_m))) * f32(p.box))
    for n in range(3):
        cs = (v[n] / beta) * f32(2.998e5)
        assert info["cs2"][n] == max(f32(1e-6), (cs * hg_dv) * (cs * hg_dv))


def test_rest_state_is_stationary():
    p = nu_params()
    o = oracle(p)
    info = o.nu_info()
    before = [o.nu_store(n) for n in range(3)]
    dtg = o.nu_evolve(0.05, 1000.0, 1, 0.5)
    for n in range(3):
        np.testing.assert_array_equal(o.nu_store(n), before[n])
    cs = np.sqrt(info["cs2"])
    expect = min(float((f32(0.71) * info["dx"][n]) / (f32(0) + f32(cs[n]))) for n in range(3))
    assert dtg == pytest.approx(expect, rel=0, abs=0)


def test_not_evolved_before_turn_on():
    p = nu_params()
    o = oracle(p)
    cs2 = o.nu_info()["cs2"]
    st = ic.nu_fluid_perturbed(int(o.nu_info()["nc"][0]), 5, cs2=float(cs2[0]))
    o.nu_load(0, st)
    dtg = o.nu_evolve(0.05, 1000.0, 1, 1.0 / 12.0)  # a < 1/(1+z_i_nu)
    np.testing.assert_array_equal(o.nu_store(0), st)
    assert dtg == 1000.0


@pytest.mark.parametrize("direction", [1, -1])
def test_oracle_sweeps_match_numpy_restatement(direction):
    p = nu_params(nc=8, nnt=1)
    o = oracle(p)
    info = o.nu_info()
    states = []
    for n in range(3):
        st = ic.nu_fluid_perturbed(int(info["nc"][n]), 11 + n, cs2=float(info["cs2"][n]))
        o.nu_load(n, st)
        states.append(st)
    dt = f32(0.3) * min(f32(info["dx"][n]) / np.sqrt(f32(info["cs2"][n])) for n in range(3))
    dtg = o.nu_evolve(float(dt), 1000.0, direction, 0.5)
    exp_dt = f32(1000.0)
    for n in range(3):
        dx = f32(info["dx"][n])
        ref = np_evolve(states[n], GAMMA, dt, dx, direction)
        got = o.nu_store(n)
        np.testing.assert_array_equal(got, ref)
        exp_dt = min(exp_dt, np_timestep(ref, GAMMA, dx))
        # the flux form conserves mass and momentum (FP32 rounding only)
        assert abs(float(ref[..., 0].astype(np.float64).sum() - states[n][..., 0].astype(np.float64).sum())) < 1e-3
    assert dtg == float(exp_dt)


# ---- gravity: closed form of the sequential scatter ---------------------------
def closed_form_gravity(fld, fine, coarse, a_mid, dt, nf, nc, dx, with_b=True):
    """The GPU's formulation in float64 numpy: per fluid cell A = sum dV a and
    B = sum dV (1-dV) |a|^2 over the reference's sources (fine cells; coarse
    sources also two layers beyond each face), then p += rho A,
    E += p.A + rho|A|^2/2 + rho B/2."""
    pif = f32(4.0) * np.arctan(f32(1.0))

    def scale(f):
        return (((f.astype(f32) * f32(a_mid)) * f32(dt)) / f32(6.0)) / pif

    q = np.arange(-2, nf + 2)
    # fine sources at q in [0, nf): force node q+1 (pm.f90:160-163)
    af = np.zeros((3, nf + 4, nf + 4, nf + 4))
    af[:, 2:nf + 2, 2:nf + 2, 2:nf + 2] = scale(np.roll(fine, -1, axis=(1, 2, 3)))
    # coarse sources: CIC of force_c at q + 1/2
    xc = (q + 0.5) / 4.0 - 0.5
    lo = np.floor(xc).astype(int)
    w1 = (lo + 1) - xc
    Wc = np.zeros((nf + 4, nc))
    Wc[np.arange(nf + 4), lo % nc] += w1
    Wc[np.arange(nf + 4), (lo + 1) % nc] += 1.0 - w1
    gc = scale(coarse).astype(np.float64)
    ac = np.einsum("zk,yj,xi,dkji->dzyx", Wc, Wc, Wc, gc)
    A = af + ac
    Q = (af ** 2).sum(0) + (ac ** 2).sum(0)
    n = nf // dx
    xx = (q + 0.5) / dx - 0.5
    tl = np.floor(xx).astype(int)
    wl = (tl + 1) - xx
    W = np.zeros((n, nf + 4))
    for t in range(n):
        W[t, tl == t] = wl[tl == t]
        W[t, tl == t - 1] = 1.0 - wl[tl == t - 1]
    Ar = np.einsum("zk,yj,xi,dkji->dzyx", W, W, W, A) / dx ** 3
    C1 = np.einsum("zk,yj,xi,kji->zyx", W, W, W, Q)
    C2 = np.einsum("zk,yj,xi,kji->zyx", W * W, W * W, W * W, Q)
    B = (C1 - C2) / dx ** 6
    out = fld.astype(np.float64).copy()
    rho = out[..., 0]
    p0 = out[..., 1:4].copy()
    Av = np.moveaxis(Ar, 0, -1)
    out[..., 1:4] = p0 + rho[..., None] * Av
    out[..., 4] += (p0 * Av).sum(-1) + 0.5 * rho * (Av ** 2).sum(-1) + (0.5 * rho * B if with_b else 0.0)
    return out


def test_gravity_closed_form_matches_sequential_scatter():
    from helpers import small_state
    st, _, s = small_state(nc=8, nnt=1, box=300.0, seed=29, amplitude=2.0)
    p = nu_params(nc=8, nnt=1, box=300.0)
    fk, ck = read_fine_table(nf_cutoff=p.nf_cutoff), read_coarse_table()
    o = Oracle(p, fk, ck, build_kernels=True)
    o.load(st.xp, st.vp, st.pid, st.rhoc, st.vfield)
    info = o.nu_info()
    before = []
    for k in range(3):
        fl = ic.nu_fluid_perturbed(int(info["nc"][k]), 51 + k, cs2=float(info["cs2"][k]))
        o.nu_load(k, fl)
        before.append(fl)
    nf, nc = p.nc * p.ncell, p.nc
    rng = np.random.default_rng(3)
    fine = rng.normal(size=(3, nf, nf, nf)).astype(f32) * f32(20.0)
    coarse = rng.normal(size=(3, nc, nc, nc)).astype(f32) * f32(5.0)
    s.a_mid, s.dt = 0.5, 0.05
    o.particle_mesh_with_force(s, fine.reshape(-1), coarse.reshape(-1), 1)
    for k in range(3):
        dx = int(info["dx"][k])
        ref = closed_form_gravity(before[k], fine, coarse, 0.5, 0.05, nf, nc, dx)
        got = o.nu_store(k).astype(np.float64)
        # the oracle adds its ~2(2dx)^3 increments one by one in FP32: allow
        # 8 sqrt(N) units in the last place of the largest value of the field
        nsrc = 2 * (2 * dx) ** 3
        for c in range(1, 5):
            tol = 8.0 * np.sqrt(nsrc) * np.abs(ref[..., c]).max() * 2.0 ** -24
            err = np.abs(got[..., c] - ref[..., c]).max()
            assert err <= tol, (k, c, err, tol)
        if k == 0:  # on the finest fluid the B term of the energy is far above that bound
            no_b = closed_form_gravity(before[k], fine, coarse, 0.5, 0.05, nf, nc, dx, with_b=False)
            tol_e = 8.0 * np.sqrt(nsrc) * np.abs(ref[..., 4]).max() * 2.0 ** -24
            assert np.abs(ref[..., 4] - no_b[..., 4]).max() > 20 * tol_e
