"""CPU tests that pin the oracle (the checker of the GPU parity tests).

The reference ships no golden outputs (its ICs are clock-seeded,
initial_conditions.f90:287-293) and cannot be built here (no Fortran compiler,
no FFTW).  The oracle is pinned piece by piece against independent numpy
restatements of the reference where that is possible: its FFT against numpy's,
its kernel_f / kernel_c against a numpy transcription of kernel_f.f90:25-37 and
kernel_c.f90:16-117, and its step against the reference's own run-time
invariants (mass sums pm.f90:108,280; particle count update_particle.f90:247-252;
PP touch count ext_pp_force.f90:154-158).
"""
import ctypes as C
import math

import numpy as np
import pytest

from helpers import clustered_state, small_state
from oracle_ref import Oracle, lib
from cube_nufluid_b200.abi import make_params


def test_oracle_fft_matches_numpy():
    rng = np.random.default_rng(0)
    for n in (12, 16, 20, 28):
        a = rng.normal(size=(n, n, n))
        out = np.zeros((n, n, n // 2 + 1, 2))
        lib().orc_rfft3(a.ctypes.data_as(C.c_void_p), n, out.ctypes.data_as(C.c_void_p))
        ref = np.fft.rfftn(a)
        got = out[..., 0] + 1j * out[..., 1]
        assert np.max(np.abs(got - ref)) < 1e-10 * np.max(np.abs(ref))


def numpy_kernel_f(fk, nfe, nfc=16, ext_pp=False, pp_range=1):
    """kernel_f.f90:25-37 transcribed with numpy (Fortran index i -> array [k,j,i])."""
    out = []
    for d in range(3):
        r = np.zeros((nfe, nfe, nfe))
        r[:nfc, :nfc, :nfc] = fk[d]
        if ext_pp:
            r[:pp_range + 1, :pp_range + 1, :pp_range + 1] = 0
        mf = [-1 if e == d else 1 for e in range(3)]
        r[:, :, nfe - nfc + 1:] = mf[0] * r[:, :, nfc - 1:0:-1]
        r[:, nfe - nfc + 1:, :] = mf[1] * r[:, nfc - 1:0:-1, :]
        r[nfe - nfc + 1:, :, :] = mf[2] * r[nfc - 1:0:-1, :, :]
        out.append(np.fft.rfftn(r).imag)
    return np.stack(out)


def separable_green(fk, n, nfc=16, ext_pp=False, pp_range=1):
    """The closed form the GPU evaluates (cube_green.cu): octant of Im K_d on an n^3 mesh."""
    kp = n // 2 + 1
    k = np.arange(kp)
    a = np.arange(nfc)
    ang = 2 * np.pi * np.outer(k, a) / n
    S = -2 * np.sin(ang)
    S[:, 0] = 0
    Cc = 2 * np.cos(ang)
    Cc[:, 0] = 1
    out = []
    for d in range(3):
        T = fk[d].astype(np.float64).copy()  # [az][ay][ax]
        if ext_pp:
            T[:pp_range + 1, :pp_range + 1, :pp_range + 1] = 0
        Fx = S if d == 0 else Cc
        Fy = S if d == 1 else Cc
        Fz = S if d == 2 else Cc
        out.append(np.einsum("zyx,kx,jy,iz->ijk", T, Fx, Fy, Fz))  # [kz][ky][kx]
    return np.stack(out)


@pytest.mark.parametrize("ext_pp", [False, True])
def test_oracle_kernel_f_matches_numpy_transcription(tables, ext_pp):
    fk, ck = tables
    p = make_params(16, 2, ext_pp_force=ext_pp)
    o = Oracle(p, fk, ck)
    nfe = 8 * 4 + 48
    got = o.fetch(4).reshape(3, nfe, nfe, nfe // 2 + 1)
    ref = numpy_kernel_f(fk, nfe, ext_pp=ext_pp)
    assert np.max(np.abs(got - ref)) < 1e-9 * np.max(np.abs(ref))


def test_separable_green_equals_fft_kernel(tables):
    # the GPU's closed-form multiplier equals the imaginary part of the FFT of the
    # mirrored table (checked on the oracle's nfe grid, octant part)
    fk, ck = tables
    nfe = 80
    ref = numpy_kernel_f(fk, nfe)
    kp = nfe // 2 + 1
    sep = separable_green(fk, nfe)
    assert np.max(np.abs(sep - ref[:, :kp, :kp, :kp])) < 1e-9 * np.max(np.abs(ref))
    # and the octant with sign flips reproduces the full half spectrum
    kz = np.arange(nfe)
    fz = np.where(kz <= nfe // 2, kz, nfe - kz)
    sz = np.where(kz <= nfe // 2, 1.0, -1.0)
    full_z = sep[2][fz][:, fz, :] * sz[:, None, None]
    assert np.max(np.abs(full_z - ref[2])) < 1e-9 * np.max(np.abs(ref))


def numpy_kernel_c(ck_table, nc, ncell=4):
    """kernel_c.f90:16-117 (LRCKCORR, one image) transcribed with numpy."""
    idx = np.arange(nc)
    off = ((idx + nc // 2) % nc) - nc // 2
    rx = ncell * np.stack(np.meshgrid(off, off, off, indexing="ij")[::-1])  # [d][z][y][x]
    r = np.sqrt((rx ** 2).sum(0))
    with np.errstate(divide="ignore", invalid="ignore"):
        direct = np.where(r == 0, 0.0, -rx / r ** 3)
    corr = direct.copy()
    for kz in range(-3, 4):
        for ky in range(-3, 4):
            for kx in range(-3, 4):
                for d in range(3):
                    v = ck_table[abs(kz), abs(ky), abs(kx), d]
                    o = (kx, ky, kz)[d]
                    corr[d, kz % nc, ky % nc, kx % nc] = -v if o < 0 else v
    kr_off = off
    out = []
    for d in range(3):
        C_ = np.fft.rfftn(corr[d]).imag
        D_ = np.fft.rfftn(direct[d]).imag
        kxs = kr_off[: nc // 2 + 1].copy()
        kxs[nc // 2] = -nc // 2
        KZ, KY, KX = np.meshgrid(kr_off, kr_off, kxs, indexing="ij")
        kr = np.sqrt(KX ** 2 + KY ** 2 + KZ ** 2)
        ks = [2 * np.sin(np.pi * K / nc) for K in (KX, KY, KZ)]
        ks2 = ks[0] ** 2 + ks[1] ** 2 + ks[2] ** 2
        kd = (KX, KY, KZ)[d]
        with np.errstate(divide="ignore", invalid="ignore"):
            rescaled = C_ * 0.25 * np.pi * ks[d] / ks2 / D_
        v = np.where((kr > 8) | (kd == 0), C_, rescaled)
        v = np.where(kd == -nc // 2, 0.0, v)
        out.append(v)
    return np.stack(out)


@pytest.mark.parametrize("nc", [16, 24])
def test_oracle_kernel_c_matches_numpy_transcription(tables, nc):
    fk, ck = tables
    o = Oracle(make_params(nc, 2), fk, ck)
    got = o.fetch(5).reshape(3, nc, nc, nc // 2 + 1)
    ref = numpy_kernel_c(ck, nc)
    assert np.max(np.abs(got - ref)) < 1e-9 * np.max(np.abs(ref))


def test_tree_sum_is_the_fixed_pairwise_tree():
    rng = np.random.default_rng(5)
    a = rng.normal(size=5000) * 10 ** rng.uniform(-5, 5, 5000)

    def tree(v):
        v = list(v)
        while len(v) > 1:
            out = []
            for b in range(0, len(v), 1024):
                loc = v[b:b + 1024] + [0.0] * (1024 - len(v[b:b + 1024]))
                s = 512
                while s >= 1:
                    for i in range(s):
                        loc[i] = loc[i] + loc[i + s]
                    s //= 2
                out.append(loc[0])
            v = out
        return v[0]

    got = lib().orc_tree_sum(a.ctypes.data_as(C.c_void_p), a.size)
    assert got == tree(a)
    assert abs(got - math.fsum(a)) < 1e-12 * np.sum(np.abs(a))


@pytest.fixture(scope="module")
def stepped(tables):
    """Two oracle steps on a 32^3-particle box: state after update_x and particle_mesh."""
    fk, ck = tables
    st, p, s = small_state(nc=16, nnt=2, seed=11)
    o = Oracle(p, fk, ck)
    o.load(st.xp, st.vp, st.pid, st.rhoc, st.vfield)
    from helpers import first_step_scalars
    first_step_scalars(p, s, 0.0)
    o.update_x(s)
    o.particle_mesh(s, 1)
    return st, p, s, o


def test_oracle_step_invariants(stepped):
    st, p, s, o = stepped
    xp, vp, pid, rhoc, vf = o.store()
    assert xp.shape[0] == st.np == rhoc.sum()                       # update_particle.f90:247-252
    assert np.array_equal(np.sort(pid), np.sort(st.pid))             # PID check :156-164
    assert abs(s.testrhof - st.np * st.mass_p_cdm) < 1e-6 * s.testrhof   # pm.f90:108,446
    assert abs(s.testrhoc - st.np * st.mass_p_cdm) < 1e-6 * s.testrhoc   # pm.f90:280
    assert 0 < s.sigma_vi_new < 1
    assert s.dt_fine > 0 and s.dt_coarse > 0 and s.dt_vmax > 0


def test_fixed_point_and_reference_order_deposits_agree(tables):
    fk, ck = tables
    st, p, s = small_state(nc=16, nnt=2, seed=2)
    dens = []
    for mode in (0, 1):
        o = Oracle(p, fk, ck)
        o.load(st.xp, st.vp, st.pid, st.rhoc, st.vfield)
        s2 = s.copy()
        s2.a_mid = s2.a
        s2.dt = 0.0
        o.particle_mesh(s2, mode)
        dens.append((o.fetch(0), o.fetch(1)))
    for a, b in zip(dens[0], dens[1]):
        assert np.max(np.abs(a - b)) <= 4e-6 * np.max(np.abs(b))


def test_pp_touches_every_particle_once(tables):
    fk, ck = tables
    st, p, s = clustered_state(nc=16, nnt=2, seed=4)
    p.ext_pp_force = 1
    o = Oracle(p, fk, ck, build_kernels=False)
    o.load(st.xp, st.vp, st.pid, st.rhoc, st.vfield)
    s.a_mid = s.a
    s.dt = 0.05
    o.ext_pp_force(s)
    assert s.itest1 == st.np                                        # ext_pp_force.f90:154-158
    assert s.npairs >= st.np
    assert s.f2_max_pp > 0 and s.dt_pp > 0
