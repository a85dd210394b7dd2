"""GPU parity of the fluid neutrinos: the CUDA library through its C-ABI against
the CPU oracle's literal restatement of hydrodf/hydrogr/hydro3d/hydro1d and the
neutrino parts of pm.f90.

Bars: the sweeps, the CFL step and the neutrino density in both meshes are
bit-exact (same FP32 operations; 64-bit fixed point for the coarse deposit).
The gravity coupling is FP32 within tolerance: the oracle scatters sources one
by one in the reference's loop order, the GPU applies the closed form of that
chain (A = sum dV a, B = sum dV(1-dV)|a|^2) with a different summation order.
"""
import numpy as np
import pytest

from cube_nufluid_b200 import Cube, ic
from helpers import nu_params, small_state
from oracle_ref import Oracle

pytestmark = pytest.mark.gpu

# Gravity tolerance, per fluid and field: the oracle adds its N = 2 (2dx)^3
# increments one by one in FP32 and the GPU sums separable FP32 restrictions, so
# each side carries ~sqrt(N) units in the last place of the field; the bound is
# 16 sqrt(N) ulp of the field's largest value (the CPU test of the closed form
# pins the oracle alone to half of it).
def grav_tol(field_max, dx):
    return 16.0 * np.sqrt(2 * (2 * dx) ** 3) * field_max * 2.0 ** -24


def fluid_pair(p, tables, build=False, st=None):
    fk, ck = tables
    o = Oracle(p, fk, ck, build_kernels=build)
    g = Cube(p, np_capacity=(st.np + 1024) if st is not None else 1024, fk_table=fk, ck_table=ck)
    if st is not None:
        o.load(st.xp, st.vp, st.pid, st.rhoc, st.vfield)
        g.load_state(st.xp, st.vp, st.pid, st.rhoc, st.vfield)
    info = g.nu_info()
    states = []
    for k in range(3):
        fl = ic.nu_fluid_perturbed(int(info["nc"][k]), 31 + k, cs2=float(info["cs2"][k]))
        o.nu_load(k, fl)
        g.nu_load(k, fl)
        states.append(fl)
    return o, g, states


def test_nu_setup_matches_oracle(tables):
    p = nu_params()
    fk, ck = tables
    o = Oracle(p, fk, ck, build_kernels=False)
    g = Cube(p, np_capacity=1024, fk_table=fk, ck_table=ck)
    a, b = o.nu_info(), g.nu_info()
    for key in a:
        assert np.array_equal(np.asarray(a[key]), np.asarray(b[key])), key
    # hg_setup's rest state
    for k in range(3):
        fl = g.nu_store(k)
        assert np.array_equal(fl, o.nu_store(k))
        assert np.all(fl[..., 0] == 1.0) and np.all(fl[..., 1:4] == 0.0)


@pytest.mark.parametrize("direction", [1, -1])
def test_nu_evolve_bit_exact(tables, direction):
    p = nu_params(nc=16, nnt=2)
    o, g, _ = fluid_pair(p, tables)
    info = g.nu_info()
    dt = np.float32(0.3) * min(np.float32(info["dx"][k]) / np.sqrt(np.float32(info["cs2"][k])) for k in range(3))
    dto, dtg = 1000.0, 1000.0
    for rep in range(2):  # two half steps, the second one from the evolved state
        d = direction if rep == 0 else -direction
        dto = o.nu_evolve(float(dt), dto, d, 0.5)
        dtg = g.nu_evolve(float(dt), dtg, d, 0.5)
        assert dto == dtg
        for k in range(3):
            a, b = o.nu_store(k), g.nu_store(k)
            assert np.array_equal(a.view(np.int32), b.view(np.int32)), f"fluid {k} after half step {rep}"


def test_nu_evolve_waits_for_turn_on(tables):
    p = nu_params(nc=16, nnt=2)
    o, g, states = fluid_pair(p, tables)
    assert g.nu_evolve(0.05, 1000.0, 1, 0.08) == 1000.0  # a < 1/(1+z_i_nu)
    for k in range(3):
        assert np.array_equal(g.nu_store(k), states[k])


@pytest.mark.parametrize("a_mid", [0.5, 0.05])  # after / before z_i_nu
def test_nu_density_bit_exact(tables, a_mid):
    st, _, s = small_state(nc=16, nnt=2, box=300.0, seed=17, amplitude=2.0)
    p = nu_params(nc=16, nnt=2, box=300.0)
    o, g, _ = fluid_pair(p, tables, build=True, st=st)
    so, sg = s.copy(), s.copy()
    for x in (so, sg):
        x.a_mid = a_mid
        x.dt = 0.01
    o.particle_mesh(so, 1)
    g.debug_deposit(sg)
    assert np.array_equal(o.fetch(0).view(np.int32), g.fetch(0).view(np.int32))
    assert np.array_equal(o.fetch(1).view(np.int32), g.fetch(1).view(np.int32))
    assert sg.testrhof == pytest.approx(so.testrhof, rel=1e-6)
    assert sg.testrhoc == pytest.approx(so.testrhoc, rel=1e-7)


def test_nu_gravity_matches_sequential_scatter(tables):
    st, _, s = small_state(nc=16, nnt=2, box=300.0, seed=23, amplitude=3.0)
    p = nu_params(nc=16, nnt=2, box=300.0)
    o, g, before = fluid_pair(p, tables, build=True, st=st)
    so, sg = s.copy(), s.copy()
    for x in (so, sg):
        x.a_mid = 0.5
        x.dt = 0.05
    # the oracle's own step, then the GPU's kick + gravity on the oracle's forces
    o.particle_mesh(so, 1)
    g.kick_with_force(sg, o.fetch(2), o.fetch(3))
    info = g.nu_info()
    for k in range(3):
        fo = o.nu_store(k).astype(np.float64)
        fg = g.nu_store(k).astype(np.float64)
        assert np.array_equal(fg[..., 0], before[k][..., 0])  # gravity leaves rho alone
        for c in range(1, 5):
            assert np.abs(fo[..., c] - before[k][..., c]).max() > 0, (k, c)
            err = np.abs(fg[..., c] - fo[..., c]).max()
            tol = grav_tol(np.abs(fo[..., c]).max(), int(info["dx"][k]))
            assert err <= tol, (k, c, err, tol)


def test_nu_step_loop_runs_and_conserves_mass(tables):
    # the step of main.f90:49-64 with both neutrino half steps, on the GPU alone
    st, _, s = small_state(nc=16, nnt=2, box=300.0, seed=5, amplitude=2.0)
    p = nu_params(nc=16, nnt=2, box=300.0)
    fk, ck = tables
    g = Cube(p, np_capacity=st.np + 1024, fk_table=fk, ck_table=ck)
    g.load_state(st.xp, st.vp, st.pid, st.rhoc, st.vfield)
    info = g.nu_info()
    for k in range(3):
        g.nu_load(k, ic.nu_fluid_perturbed(int(info["nc"][k]), 40 + k, cs2=float(info["cs2"][k])))
    s.a = 0.3  # after the neutrino turn-on
    s.dt_neu = 1000.0
    m0 = [g.nu_store(k)[..., 0].astype(np.float64).sum() for k in range(3)]
    for _ in range(2):
        g.step(s)
        assert s.dt_neu < 1000.0
    for k in range(3):
        fl = g.nu_store(k)
        assert np.all(np.isfinite(fl))
        assert abs(fl[..., 0].astype(np.float64).sum() / m0[k] - 1.0) < 1e-5
