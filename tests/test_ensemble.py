"""Ensembles of independent boxes on one GPU: the reproducible box draws, the tile
layouts they get, and (GPU) that boxes stepped side by side on concurrent streams
end bit-identical to the same boxes stepped one after the other."""
import numpy as np
import pytest

from cube_nufluid_b200.ensemble import PARTICLES_PER_SIDE, BoxSpec, Ensemble, _nnt, ensemble_specs


def test_specs_are_reproducible_and_in_range():
    a = ensemble_specs(96, 7)
    b = ensemble_specs(96, 7)
    assert a == b and len(a) == 96
    assert ensemble_specs(96, 8) != a
    for sp in a:
        assert 2 * sp.nc in PARTICLES_PER_SIDE
        assert 50.0 <= sp.box <= 400.0
        assert 0.25 <= sp.omega_m <= 0.35 and 0.7 <= sp.sigma8 <= 0.9
    sides = {2 * sp.nc for sp in a}
    assert sides == set(PARTICLES_PER_SIDE)
    boxes = np.log([sp.box for sp in a])
    assert boxes.min() < np.log(100.0) and boxes.max() > np.log(200.0)


def test_tile_layouts_suit_the_kernels():
    for side in PARTICLES_PER_SIDE:
        nc = side // 2
        nnt = _nnt(nc)
        assert nc % nnt == 0 and (nc // nnt) % 4 == 0  # whole PP bricks per tile
        assert nc % 8 == 0                             # whole deposit bricks


@pytest.mark.gpu
def test_gpu_concurrent_boxes_match_sequential(tables):
    fk, ck = tables
    # every mesh size of the ensemble workload, so kernels shared across sizes run
    # side by side with different launch shapes
    specs = [BoxSpec(nc=16, box=60.0, omega_m=0.3, sigma8=0.8, seed=11),
             BoxSpec(nc=24, box=150.0, omega_m=0.27, sigma8=0.85, seed=12),
             BoxSpec(nc=32, box=300.0, omega_m=0.33, sigma8=0.75, seed=13),
             BoxSpec(nc=48, box=200.0, omega_m=0.29, sigma8=0.78, seed=14),
             BoxSpec(nc=64, box=350.0, omega_m=0.31, sigma8=0.82, seed=15),
             BoxSpec(nc=16, box=80.0, omega_m=0.31, sigma8=0.72, seed=16, pp=True)]
    seq = Ensemble(specs, fk, ck)
    r1 = seq.run(3, workers=1)
    s1 = seq.states()
    seq.close()
    par = Ensemble(specs, fk, ck)
    r6 = par.run(3, workers=6)
    s6 = par.states()
    par.close()
    assert r1["boxes"] == r6["boxes"] == 6 and r6["workers"] == 6
    for a, b in zip(s1, s6):
        for x, y in zip(a, b):
            assert np.array_equal(x, y)
    # the library's own thread pool (cube_run_steps) gives the same states and scalars
    nat = Ensemble(specs, fk, ck)
    rn = nat.run_native(3, workers=4)
    sn = nat.states()
    assert all(m.steps == 3 for m in nat.members)
    nat.close()
    assert rn["boxes"] == 6 and rn["workers"] == 4
    for a, b in zip(s1, sn):
        for x, y in zip(a, b):
            assert np.array_equal(x, y)


@pytest.mark.gpu
def test_gpu_native_runner_matches_python_steps_and_reports_errors(tables):
    from cube_nufluid_b200.cube import CubeError
    fk, ck = tables
    specs = [BoxSpec(nc=16, box=60.0, omega_m=0.3, sigma8=0.8, seed=21),
             BoxSpec(nc=32, box=250.0, omega_m=0.28, sigma8=0.82, seed=22, pp=True)]
    py = Ensemble(specs, fk, ck)
    py.run(2, workers=1)
    nat = Ensemble(specs, fk, ck)
    nat.run_native(2, workers=2)
    for a, b in zip(py.members, nat.members):
        assert a.s.as_dict() == b.s.as_dict()
    for a, b in zip(py.states(), nat.states()):
        for x, y in zip(a, b):
            assert np.array_equal(x, y)
    py.close()
    # a context without a loaded state is refused with its index
    import ctypes as C
    from cube_nufluid_b200 import Cube
    from cube_nufluid_b200.abi import CubeScalars
    fresh = Cube(nat.members[0].cube.p, np_capacity=4096, fk_table=fk, ck_table=ck)
    L = fresh.L
    handles = (C.c_void_p * 2)(nat.members[0].cube.h, fresh.h)
    ios = (CubeScalars * 2)()
    failed = C.c_int32(-5)
    rc = L.cube_run_steps(handles, ios, 2, 1, 2, C.byref(failed))
    assert rc == 6 and failed.value == 1  # CUBE_ERR_STATE, the second context
    fresh.close()
    nat.close()
