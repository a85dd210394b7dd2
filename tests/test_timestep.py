"""CPU tests of cube_timestep against a numpy restatement of timestep.f90:1-95.

The restatement keeps the reference's precisions: the real(4) scalars (dt, da,
ra, dt_e, a, the limits) as float32 and the real(8) internals of expansion
(timestep.f90:136-180) as float64, with the default-real literals and parameter
products evaluated in float32 before promotion.  Cases cover each limit being
the smallest, the ra_max retries and the snapping onto a checkpoint.
"""
import ctypes as C

import numpy as np
import pytest

from cube_nufluid_b200.abi import CubeScalars, make_params
from cube_nufluid_b200.cube import load_library

f32, f64 = np.float32, np.float64


def expansion_ref(p, a0, dt0):
    """timestep.f90:136-180 (the branch without new_expansion)."""
    om, ol, wde = f32(p.omega_m), f32(p.omega_l), f32(p.wde)
    a0, dt0 = f32(a0), f32(dt0)
    dt_x = dt0 / f32(2.0)
    omHsq = f64(f32(4.0) / f32(9.0))

    def half(a_x):
        a3rlm = (a_x ** f64(f32(-3.0) * wde)) * f64(ol) / f64(om)
        arkm = a_x * f64(f32(1.0) - om - ol) / f64(om)
        adot = np.sqrt(omHsq * (a_x * a_x * a_x) * (1.0 + arkm + a3rlm))
        addot = (a_x * a_x) * omHsq * (1.5 + 2.0 * arkm + f64(f32(1.5) * (f32(1.0) - wde)) * a3rlm)
        atdot = a_x * adot * omHsq * (3.0 + 6.0 * arkm +
                                      f64(f32(1.5) * (f32(2.0) - f32(3.0) * wde) * (f32(1.0) - wde)) * a3rlm)
        return f32(adot * f64(dt_x) + (addot * f64(dt_x * dt_x)) / 2.0 + (atdot * f64(dt_x * dt_x * dt_x)) / 6.0)

    da1 = half(f64(a0))
    da2 = half(f64(a0 + da1))
    return da1, da2


def timestep_ref(p, s, a_next):
    """timestep.f90:1-95 on the head image; returns (dt, da, a_mid, a, hit, retries)."""
    a = f32(s.a)
    dt_e = f32(p.dt_max)
    ntry = 0
    while True:
        ntry += 1
        d1, d2 = expansion_ref(p, a, dt_e)
        da = d1 + d2
        ra = da / (a + da)
        if ra > f32(p.ra_max):
            dt_e = dt_e * (f32(p.ra_max) / ra)
        else:
            break
        if ntry > 10:
            break
    nu = f32(s.dt_vmax_nu) if p.neutrino else f32(1000.0)
    dt = min(dt_e, f32(s.dt_fine), f32(s.dt_coarse), f32(s.dt_pp), f32(s.dt_vmax), nu, f32(s.dt_neu))
    d1, d2 = expansion_ref(p, a, dt)
    da = d1 + d2
    hit = False
    if a_next > 0 and da >= f32(a_next) - a:
        hit = True
        while abs((a + da) / f32(a_next) - f32(1.0)) >= f32(1e-6):
            dt = (dt * (f32(a_next) - a)) / da
            d1, d2 = expansion_ref(p, a, dt)
            da = d1 + d2
    return dt, da, a + da / f32(2.0), a + da, hit, ntry, dt_e


def run_lib(p, s, a_next):
    L = load_library()
    h = C.c_int32(0)
    L.cube_timestep(C.byref(p), C.byref(s), C.c_float(a_next), C.byref(h))
    return s, bool(h.value)


def scal(a, **lim):
    s = CubeScalars()
    s.a = a
    big = 1e3
    for k in ("dt_fine", "dt_coarse", "dt_pp", "dt_vmax", "dt_vmax_nu", "dt_neu"):
        setattr(s, k, lim.get(k, big))
    return s


def check(p, s, a_next=0.0):
    ref = timestep_ref(p, s, a_next)
    got, hit = run_lib(p, s.copy(), a_next)
    dt, da, a_mid, a1, rhit, _, dt_e = ref
    assert got.dt == dt and got.da == da and got.a_mid == a_mid and got.a == a1, (got.dt, dt, got.da, da)
    assert got.dt_e == dt_e
    assert hit == rhit
    return ref


@pytest.mark.parametrize("which", ["dt_fine", "dt_coarse", "dt_pp", "dt_vmax", "dt_neu"])
def test_each_limit_can_be_the_smallest(which):
    p = make_params(16, 2)
    p.dt_max = 1.0
    s = scal(0.5, **{which: 0.01234})
    dt = check(p, s)[0]
    assert dt == np.float32(0.01234)


def test_neutrino_velocity_limit_only_with_neutrinos():
    p = make_params(16, 2)
    s = scal(0.5, dt_vmax_nu=0.002)
    assert check(p, s)[0] > np.float32(0.002)          # merge(...,1000.,neutrino_flag): ignored
    p.neutrino = 1
    assert check(p, s)[0] == np.float32(0.002)


def test_expansion_limit_retries_on_ra_max():
    p = make_params(16, 2)
    p.dt_max = 50.0          # far beyond ra_max at a = 0.02
    s = scal(0.02)
    dt, da, _, a1, _, ntry, dt_e = check(p, s)
    assert ntry > 1 and dt == dt_e
    assert da / a1 <= np.float32(p.ra_max) * np.float32(1.0001)


def test_snaps_onto_a_checkpoint():
    p = make_params(16, 2)
    s = scal(0.5, dt_fine=0.2)
    dt0, da0 = timestep_ref(p, s, 0.0)[:2]
    a_next = float(np.float32(0.5) + da0 * np.float32(0.6))   # inside the step: snapped onto it
    dt, da, _, a1, hit, _, _ = check(p, s, a_next)
    assert hit and dt < dt0
    assert abs(a1 / np.float32(a_next) - 1) < 1e-6
    s2 = scal(0.5, dt_fine=0.2)
    assert not check(p, s2, float(np.float32(0.5) + da0 * np.float32(1.5)))[4]  # beyond the step: not hit


def test_expansion_matches_restatement():
    p = make_params(16, 2)
    L = load_library()
    for a0, dt0 in ((0.02, 0.3), (0.5, 0.05), (1.0, 0.01)):
        d1, d2 = C.c_float(), C.c_float()
        L.cube_expansion(C.byref(p), C.c_float(a0), C.c_float(dt0), C.byref(d1), C.byref(d2))
        r1, r2 = expansion_ref(p, a0, dt0)
        assert np.float32(d1.value) == r1 and np.float32(d2.value) == r2
