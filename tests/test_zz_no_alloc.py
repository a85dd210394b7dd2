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


def _context_coarse(st, p, s, fk, ck):
    """The coarse density the context path deposits for this state."""
    g = Cube(p, st.np, fk, ck)
    g.load_state(st.xp, st.vp, st.pid, st.rhoc, st.vfield)
    g.debug_deposit(s.copy())
    ref = g.fetch(1)
    g.close()
    return ref


@pytest.mark.parametrize("nc,nnt,npart,izipx", [(32, 4, 120000, 2), (32, 4, 120000, 1), (64, 4, 400000, 2)])
def test_noalloc_coarse_density_matches_context_deposit(tables, nc, nnt, npart, izipx):
    import torch
    fk, ck = tables
    st, p, s = clustered_state(nc=nc, nnt=nnt, npart=npart, seed=81, izipx=izipx)
    ref = _context_coarse(st, p, s, fk, ck)
    # caller-owned device buffers
    dev = torch.device("cuda:0")
    xp_soa = torch.from_numpy(np.ascontiguousarray(st.xp.T)).to(dev)          # [3][np], 1 or 2 bytes
    cs = torch.from_numpy(np.concatenate([[0], np.cumsum(st.rhoc)]).astype(np.int64)).to(dev)
    rho = torch.empty(nc ** 3, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream().cuda_stream
    f = _bind()
    for _ in range(2):  # the shared accumulator keeps the last call's sums: each call clears it
        rho.fill_(-1.0)
        rc = f(nc, nnt, izipx, st.np, xp_soa.data_ptr(), cs.data_ptr(), st.mass_p_cdm, rho.data_ptr(), stream)
        torch.cuda.synchronize()
        assert rc == 0
        out = rho.cpu().numpy()
        assert np.array_equal(out.view(np.int32), ref.view(np.int32))


def test_noalloc_refuses_meshes_beyond_its_array():
    import torch
    dev = torch.device("cuda:0")
    xp = torch.zeros(3 * 8, dtype=torch.int16, device=dev)
    cs = torch.zeros(72 ** 3 + 1, dtype=torch.int64, device=dev)
    rho = torch.empty(8, dtype=torch.float32, device=dev)
    f = _bind()
    stream = torch.cuda.current_stream().cuda_stream
    # the first size over the 64^3 limit is refused before any launch, leaving rho alone
    rho.fill_(-1.0)
    assert f(72, 8, 2, 8, xp.data_ptr(), cs.data_ptr(), 8.0, rho.data_ptr(), stream) == 2
    torch.cuda.synchronize()
    assert bool((rho == -1.0).all())
