"""Failure paths of the step, made on the host or with small states (no GPU fault):
status codes replace the reference's print + stop, and the context stays usable.

* a state larger than the context's capacity: CUBE_ERR_CAPACITY
  (the reference stops at update_particle.f90:90-96 when np_image_max is exceeded);
* cell counts that do not add up to nplocal: CUBE_ERR_PARAM;
* a drift farther than the ncb-cell buffer in one step: CUBE_ERR_MOVE (the
  reference's particles would leave the extended tile); the re-bin clamps what it
  indexes, reports the status and the context takes a fresh state afterwards;
* calls before a state is loaded: CUBE_ERR_STATE;
* a context created with PP off refuses ext_pp_force: CUBE_ERR_PARAM.
"""
import numpy as np
import pytest

from helpers import small_state
from cube_nufluid_b200 import Cube
from cube_nufluid_b200.cube import CubeError

pytestmark = pytest.mark.gpu


def test_capacity_and_inconsistent_counts(tables):
    fk, ck = tables
    st, p, s = small_state(nc=16, nnt=2, seed=31)
    g = Cube(p, st.np - 1, fk, ck)
    with pytest.raises(CubeError) as e:
        g.load_state(st.xp, st.vp, st.pid, st.rhoc, st.vfield)
    assert e.value.code == 2
    g.close()
    g = Cube(p, st.np, fk, ck)
    with pytest.raises(CubeError) as e:
        g.update_x(s.copy())
    assert e.value.code == 6
    rhoc = st.rhoc.copy()
    rhoc[0] += 1
    with pytest.raises(CubeError) as e:
        g.load_state(st.xp, st.vp, st.pid, rhoc, st.vfield)
    assert e.value.code == 1
    g.load_state(st.xp, st.vp, st.pid, st.rhoc, st.vfield)
    sc = s.copy()
    g.update_x(sc)
    with pytest.raises(CubeError) as e:
        g.ext_pp_force(sc)
    assert e.value.code == 1
    g.close()


def test_drift_beyond_the_buffer_is_reported_and_the_context_recovers(tables):
    fk, ck = tables
    st, p, s = small_state(nc=16, nnt=2, seed=32, amplitude=4.0)
    g = Cube(p, st.np, fk, ck)
    g.load_state(st.xp, st.vp, st.pid, st.rhoc, st.vfield)
    big = s.copy()
    # the fastest particles move about 10 coarse cells, beyond the ncb = 6 buffer
    # (nlayer = 2*ceiling(dt_mid*vz_max/ncell)+1 stays small)
    big.dt_old = big.dt = float(10.0 * p.ncell / s.vz_max)
    with pytest.raises(CubeError) as e:
        g.update_x(big)
    assert e.value.code == 4
    # the device status was reported, not a fault: the context takes a fresh state
    g.load_state(st.xp, st.vp, st.pid, st.rhoc, st.vfield)
    ok = s.copy()
    ok.dt_old = ok.dt = 1.0
    g.update_x(ok)
    g.particle_mesh(ok)
    assert g.store_state()[0].shape == st.xp.shape
    g.close()
