"""GPU tests of the FP64 Poisson mode (params.poisson_fp64): the FP64 run of the same
step that the FP32 results are measured against.

* its fine and coarse densities are the same 64-bit fixed-point sums as the FP32
  context's, written as doubles: rounded to FP32 they are the FP32 context's meshes;
* its forces are far closer to the CPU oracle's FP64 FFT than the FP32 forces are
  (the oracle stores its forces as FP32, so the FP64 path agrees with them to FP32
  rounding, about 5e-8, where the FP32 path is at about 2.5e-7);
* a full step (update_x, PP, particle_mesh) runs and its velocity codes differ from
  the FP32 step's only at rounding boundaries.
"""
import numpy as np
import pytest

from helpers import kick_chain, rel_rms, small_state
from oracle_ref import Oracle
from cube_nufluid_b200 import Cube
from cube_nufluid_b200.cube import CubeError

pytestmark = pytest.mark.gpu


def contexts(st, p, tables):
    fk, ck = tables
    g32 = Cube(p, st.np, fk, ck)
    p64 = type(p).from_buffer_copy(p)
    p64.poisson_fp64 = 1
    g64 = Cube(p64, st.np, fk, ck)
    for g in (g32, g64):
        g.load_state(st.xp, st.vp, st.pid, st.rhoc, st.vfield)
    return g32, g64


def test_fp64_mode_densities_and_forces(tables):
    fk, ck = tables
    st, p, s = small_state(nc=32, nnt=2, z_i=5.0, seed=91)
    g32, g64 = contexts(st, p, tables)
    for g in (g32, g64):
        g.debug_deposit(s.copy())
    for which in (0, 1):
        d32, d64 = g32.fetch(which), g64.fetch(which)
        assert d64.dtype == np.float64
        assert np.array_equal(d64.astype(np.float32).view(np.int32), d32.view(np.int32))
    s.a_mid, s.dt = s.a, 1.0
    s32, s64, so = s.copy(), s.copy(), s.copy()
    g32.particle_mesh(s32)
    g64.particle_mesh(s64)
    o = Oracle(p, fk, ck)
    o.load(st.xp, st.vp, st.pid, st.rhoc, st.vfield)
    o.particle_mesh(so, 1)
    for which in (2, 3):
        ref = kick_chain(o.fetch(which), s32.a_mid, s32.dt)  # the oracle's FP64 FFT, stored as FP32
        e32 = rel_rms(g32.fetch(which), ref)
        e64 = rel_rms(g64.fetch(which), ref)
        print(f"mesh {which}: FP32 path {e32:.2e}, FP64 path {e64:.2e} relative RMS against the oracle")
        assert e64 < 1e-7
        assert e64 < e32 / 3
    v32, v64 = g32.store_state()[1], g64.store_state()[1]
    assert np.mean(v32 != v64) < 5e-3
    assert s64.sigma_vi == s32.sigma_vi
    g32.close()
    g64.close()


def test_fp64_mode_full_step_with_pp(tables):
    st, p, s = small_state(nc=32, nnt=2, z_i=5.0, seed=92)
    p.ext_pp_force = 1
    g32, g64 = contexts(st, p, tables)
    s32, s64 = s.copy(), s.copy()
    for g, sc in ((g32, s32), (g64, s64)):
        g.timestep(sc)
        g.update_x(sc)
        g.ext_pp_force(sc)
        g.particle_mesh(sc)
    a, b = g32.store_state(), g64.store_state()
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[2], b[2])  # positions drift before the kick
    assert np.mean(a[1] != b[1]) < 5e-3
    assert s64.npairs == s32.npairs and s64.dt_pp == s32.dt_pp
    assert s64.f2_max_fine == pytest.approx(s32.f2_max_fine, rel=1e-5)
    g32.close()
    g64.close()


def test_fp64_mode_refuses_what_needs_fp32_meshes(tables):
    st, p, s = small_state(nc=16, nnt=2, seed=93)
    g32, g64 = contexts(st, p, tables)
    with pytest.raises(CubeError):
        g64.power_spectrum()
    g32.close()
    g64.close()
