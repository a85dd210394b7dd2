"""The serving loop: reproducible Poisson request streams, the memory estimate its
admission uses, and (GPU) that an answer is the same whether the request is served
alone on a fresh context or among others on reused ones; cube_set_params refuses
changes that would need other allocations."""
import numpy as np
import pytest

from cube_nufluid_b200 import Cube, CubeError
from cube_nufluid_b200.abi import make_params
from cube_nufluid_b200.ensemble import BoxSpec
from cube_nufluid_b200.serving import SERVE_SIDES, Request, Server, footprint_bytes, request_stream


def test_request_stream_is_reproducible_poisson():
    a = request_stream(2000, 20.0, 5)
    assert a == request_stream(2000, 20.0, 5) and a != request_stream(2000, 20.0, 6)
    gaps = np.diff([0.0] + [r.arrival for r in a])
    assert np.all(gaps > 0) and abs(gaps.mean() - 0.05) < 0.005
    assert abs(np.std(gaps) / np.mean(gaps) - 1.0) < 0.1  # exponential: cv = 1
    sides = [2 * r.spec.nc for r in a]
    assert set(sides) == set(SERVE_SIDES)
    # log-uniform in count: the smallest and largest sizes get half a log-step each
    frac = np.mean(np.array(sides) == 64)
    assert 0.12 < frac < 0.22


def test_footprint_grows_with_size():
    f = [footprint_bytes(s // 2) for s in SERVE_SIDES]
    assert all(b > a for a, b in zip(f, f[1:]))
    assert 2e9 < footprint_bytes(128) < 8e9  # 256^3 particles, fine mesh 512^3


@pytest.mark.gpu
def test_gpu_set_params_refuses_size_changes(tables):
    fk, ck = tables
    g = Cube(make_params(16, 2, box=100.0), np_capacity=32 ** 3, fk_table=fk, ck_table=ck)
    g.set_params(make_params(16, 2, box=250.0, omega_m=0.27, omega_l=0.73))
    with pytest.raises(CubeError):
        g.set_params(make_params(32, 2, box=250.0))
    with pytest.raises(CubeError):
        g.set_params(make_params(16, 2, box=250.0, ext_pp_force=True))
    g.close()


@pytest.mark.gpu
def test_gpu_answers_do_not_depend_on_load_or_reuse(tables):
    fk, ck = tables
    specs = [BoxSpec(nc=16, box=60.0, omega_m=0.3, sigma8=0.8, seed=1),
             BoxSpec(nc=24, box=120.0, omega_m=0.27, sigma8=0.85, seed=2),
             BoxSpec(nc=16, box=200.0, omega_m=0.33, sigma8=0.72, seed=3),
             BoxSpec(nc=32, box=300.0, omega_m=0.31, sigma8=0.78, seed=4),
             BoxSpec(nc=24, box=90.0, omega_m=0.26, sigma8=0.88, seed=5),
             BoxSpec(nc=16, box=75.0, omega_m=0.34, sigma8=0.76, seed=6)]
    reqs = [Request(i, 0.0, sp, steps=12) for i, sp in enumerate(specs)]
    busy = Server(workers=3, fk_table=fk, ck_table=ck)
    got = busy.serve(reqs, realtime=False)
    busy.close()
    for i in (0, 2, 4):  # the later two ran on reused contexts of their size
        alone = Server(workers=1, fk_table=fk, ck_table=ck)
        ref = alone.answer(reqs[i])
        alone.close()
        assert np.array_equal(got[i].pk, ref.pk) and np.array_equal(got[i].sample, ref.sample)
        assert got[i].steps == ref.steps >= 12
    for a, sp in zip(got, specs):
        assert a.sample.shape == (-(-(2 * sp.nc) ** 3 // 64), 3)
        assert np.all(np.isfinite(a.pk)) and a.pk.shape[0] > 4
