"""GPU test of cube_coarse_density_noalloc, the allocation-free entry point.

Hosts that may not call cudaMalloc during a run (their device memory belongs to
another allocator, or each box got a fixed HBM budget at start-up) pass their
own device buffers; the entry point's accumulator is a static device array.
Its output must equal the coarse density of the context path bit for bit, on
two calls in a row (the shared accumulator is cleared by each call).
This file is collected last on purpose.
"""
import ctypes as C

import numpy as np
import pytest

from helpers import clustered_state
from cube_nufluid_b200 import Cube
from cube_nufluid_b200.cube import load_library

pytestmark = pytest.mark.gpu


def _bind():
    L = load_library()
    f = L.cube_coarse_density_noalloc
    f.argtypes = [C.c_int32, C.c_int32, C.c_int32, C.c_int64, C.c_void_p, C.c_void_p, C.c_float, C.c_void_p,
                  C.c_void_p]
    f.restype = C.c_int32
    return f


def test_noalloc_coarse_density_matches_context_deposit(tables):
    import torch
    fk, ck = tables
    nc, nnt = 32, 4
    st, p, s = clustered_state(nc=nc, nnt=nnt, npart=120000, seed=81)
    # reference: the coarse density of the context path
    g = Cube(p, st.np, fk, ck)
    g.load_state(st.xp, st.vp, st.pid, st.rhoc, st.vfield)
    sd = s.copy()
    g.debug_deposit(sd)
    ref = g.fetch(1)
    # caller-owned device buffers
    dev = torch.device("cuda:0")
    xp_soa = torch.from_numpy(np.ascontiguousarray(st.xp.T)).to(dev)          # [3][np] int16
    cs = torch.from_numpy(np.concatenate([[0], np.cumsum(st.rhoc)]).astype(np.int64)).to(dev)
    rho = torch.empty(nc ** 3, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream().cuda_stream
    f = _bind()
    for _ in range(2):
        rho.fill_(-1.0)
        rc = f(nc, nnt, 2, st.np, xp_soa.data_ptr(), cs.data_ptr(), st.mass_p_cdm, rho.data_ptr(), stream)
        torch.cuda.synchronize()
        assert rc == 0
        out = rho.cpu().numpy()
        assert np.array_equal(out.view(np.int32), ref.view(np.int32))
    # sizes beyond the static accumulator are refused before any launch
    assert f(128, 4, 2, st.np, xp_soa.data_ptr(), cs.data_ptr(), st.mass_p_cdm, rho.data_ptr(), stream) == 2
