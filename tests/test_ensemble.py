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
