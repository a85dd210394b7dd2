"""One full step on the tile layout of configuration 2, against the CPU oracle.

Configuration 2 (512^3 particles, nc = 256) runs on 8^3 tiles of nt = 32 coarse
cells.  Its full size is beyond the oracle, so the two halves of that layout are
checked at nc = 64 (128^3 particles at the same particle spacing, 1.95 Mpc/h):
tiles of nt = 32 (nnt = 2; extended tiles of 176 fine cells, the C2 tile shape)
and nnt = 8 tiles per side (nt = 8; the C2 tile count per side).  The state is a
Zel'dovich state at z = 5, so PP (on, pp_range = 1) finds many pairs.  One step
of main.f90:47-66 (timestep, update_x, ext_pp_force, particle_mesh):
  * update_x and ext_pp_force bit-exact (positions, codes, PIDs, counts, vfield,
    sigma statistics, npairs, f2_max_pp),
  * deposit bit-exact (64-bit fixed point on both arms),
  * fine and coarse forces within 1e-5 relative RMS of the FP64-FFT oracle,
  * kicked velocity codes equal except where the FP32 / FP64 force difference
    crosses a rounding boundary (< 0.5 % of components).
"""
import numpy as np
import pytest

from helpers import kick_chain, rel_rms
from test_gpu_parity import FORCE_TOL, assert_same_state, pair
from cube_nufluid_b200 import ic
from cube_nufluid_b200.abi import make_params
from cube_nufluid_b200.cube import load_library, scalars_from_ic

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("nnt", [2, 8])
def test_c2_tile_layout_step(tables, nnt):
    import ctypes as C
    nc, box = 64, 250.0
    st = ic.zeldovich(nc, nnt, box=box, z_i=5.0, seed=31, izipx=2, izipv=2)
    p = make_params(nc, nnt, box=box, izipx=2, izipv=2, ext_pp_force=True)
    o, g = pair(st, p, tables)
    s = scalars_from_ic(st)
    hit = C.c_int32(0)
    load_library().cube_timestep(C.byref(p), C.byref(s), C.c_float(0.0), C.byref(hit))
    so, sg = s.copy(), s.copy()
    o.update_x(so)
    g.update_x(sg)
    assert_same_state(o, g)
    assert so.sigma_vi_new == sg.sigma_vi_new and so.nlayer == sg.nlayer
    o.ext_pp_force(so)
    g.ext_pp_force(sg)
    assert so.itest1 == sg.itest1 == st.np
    assert so.npairs == sg.npairs > 1.5 * st.np
    assert so.f2_max_pp == sg.f2_max_pp and so.dt_pp == sg.dt_pp
    assert_same_state(o, g)
    sd = sg.copy()
    g.debug_deposit(sd)
    rho_f, rho_c = g.fetch(0), g.fetch(1)
    o.particle_mesh(so, 1)
    g.particle_mesh(sg)
    assert np.array_equal(rho_f.view(np.int32), o.fetch(0).view(np.int32))
    assert np.array_equal(rho_c.view(np.int32), o.fetch(1).view(np.int32))
    assert rel_rms(g.fetch(2), kick_chain(o.fetch(2), sg.a_mid, sg.dt)) <= FORCE_TOL
    assert rel_rms(g.fetch(3), kick_chain(o.fetch(3), sg.a_mid, sg.dt)) <= FORCE_TOL
    vo, vg = o.store()[1], g.store_state()[1]
    assert np.mean(vo != vg) < 5e-3
    assert sg.sigma_vi == so.sigma_vi
    g.close()
