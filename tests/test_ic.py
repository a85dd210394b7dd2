"""Initial conditions: the Philox4x32-10 noise shared by the host and the device
generator, the device power-spectrum constants, and cube_make_ic on the GPU against
the host Zel'dovich generator (initial_conditions.f90:268-900 packing rules)."""
import math

import numpy as np
import pytest

from cube_nufluid_b200 import Cube, ic
from cube_nufluid_b200.abi import make_params
from helpers import small_state


def test_philox_known_answers():
    # Known-answer vectors published with Philox4x32-10 (Salmon et al., SC 2011)
    cases = [
        ((0, 0, 0, 0), (0, 0), (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
        ((0xFFFFFFFF,) * 4, (0xFFFFFFFF, 0xFFFFFFFF), (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
        ((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0),
         (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1)),
    ]
    for ctr, key, out in cases:
        got = ic.philox4x32_10(np.array([ctr], np.uint32), key)[0]
        assert [int(v) for v in got] == list(out)


def test_uniform_noise_word_layout():
    # word i of the grid = output word i mod 4 of counter (i div 4, 0, 0, 0), key = seed
    seed = (7 << 32) | 12345
    n = 6
    u = ic.uniform_noise(n, seed).reshape(-1)
    for i in (0, 1, 2, 3, 4, 5, 97, n ** 3 - 1):
        w = ic.philox4x32_10(np.array([[i // 4, 0, 0, 0]], np.uint32), (seed & 0xFFFFFFFF, seed >> 32))[0, i % 4]
        assert u[i] == np.float32(int(w) >> 8) * np.float32(2.0 ** -24)
    assert u.min() >= 0.0 and u.max() < 1.0


def test_lattice_pid_encoding():
    # pid = iq_x + nf iq_y + nf^2 iq_z + 1 with iq = (ncell/np_nc) * lattice index
    pid = ic.lattice_pid(8, 2, 4)
    nf, npd = 32, 16
    assert pid.shape == (npd ** 3,) and pid[0] == 1 and pid[1] == 3 and pid[npd] == 2 * nf + 1
    assert pid[-1] == 30 + 30 * nf + 30 * nf * nf + 1
    assert np.unique(pid).size == pid.size and np.all(np.diff(pid) > 0)


def test_gaussian_noise_moments():
    g = ic.gaussian_noise(32, 5).astype(np.float64)
    assert abs(g.mean()) < 0.01 and abs(g.std() - 1.0) < 0.01


def test_potential_kernel_has_the_exact_near_field():
    """initial_conditions.f90:478-523 (correct_kernel): in real space the corrected
    kernel is -1/r within 8 cells and -2.5 at r = 0, up to the constant that the zeroed
    k = 0 mode removes; beyond 8 cells it is the discrete-Laplacian kernel shifted."""
    n = 40
    K = ic.potential_kernel(n)
    Kr = np.fft.ifftn(K).real
    c = Kr[1, 0, 0] + 1.0
    for r in [(0, 0, 0), (1, 0, 0), (0, 2, 0), (3, 4, 0), (0, 0, 8), (2, 3, 6), (5, 5, 5)]:
        d = math.sqrt(sum(x * x for x in r))
        exact = -2.5 if d == 0 else -1.0 / d
        if d <= 8:
            assert abs((Kr[r] - c) - exact) < 1e-12, (r, Kr[r] - c, exact)
    # far field: the uncorrected lattice Green function plus the shift, close to -1/r
    m = np.fft.fftfreq(n, d=1.0 / n)
    s2 = (2 * np.sin(np.pi * m / n)) ** 2
    kr = s2[:, None, None] + s2[None, :, None] + s2[None, None, :]
    K0 = np.where(kr > 0, -4 * np.pi / np.where(kr > 0, kr, 1.0), 0.0)
    K0r = np.fft.ifftn(K0).real
    phi8 = (K0r[8, 0, 0] + K0r[n - 8, 0, 0] + K0r[0, 8, 0] + K0r[0, n - 8, 0] + K0r[0, 0, 8] + K0r[0, 0, n - 8]) / 6
    for r in [(9, 0, 0), (6, 6, 3), (12, 5, 0)]:
        assert abs((Kr[r] - c) - (K0r[r] - (phi8 + 1 / 8))) < 1e-9
    # meshes too small for the 8-cell near field keep the plain kernel
    m16 = np.fft.fftfreq(16, d=1.0 / 16)
    s16 = (2 * np.sin(np.pi * m16 / 16)) ** 2
    k16 = s16[:, None, None] + s16[None, :, None] + s16[None, None, :]
    plain = np.where(k16 > 0, -4 * np.pi / np.where(k16 > 0, k16, 1.0), 0.0)
    assert np.array_equal(ic.potential_kernel(16), plain)


def test_zeldovich_displacement_is_the_central_difference_of_phi():
    """The generator's displacement at a lattice point equals -(phi(i+1) - phi(i-1))/(8 pi)
    of phi = IFFT(K' delta) on the fine mesh (initial_conditions.f90:794-796, 828)."""
    import scipy.fft as sfft
    nc, ncell, np_nc, box, z_i, seed = 8, 4, 2, 100.0, 49.0, 5
    nf = nc * ncell
    c = ic.Cosmology()
    a = 1.0 / (1.0 + z_i)
    dk, kx, ky, kz, _ = ic._linear_delta_k(nf, box, a, seed, c, 1.0)
    Kc = ic.potential_kernel(nf)[:, :, : nf // 2 + 1]
    phi = sfft.irfftn(Kc * dk, s=(nf, nf, nf))  # [z][y][x]
    gx = -(np.roll(phi, -1, axis=2) - np.roll(phi, 1, axis=2)) / (8 * np.pi)
    # the same from the generator's own k-space multiplier
    g = -np.sin(2 * np.pi * kx / nf) / (4 * np.pi)
    g = np.where(np.abs(kx) == nf // 2, 0.0, g)
    psi = sfft.irfftn(1j * g[None, None, :] * Kc * dk, s=(nf, nf, nf))
    # they differ only by the Nyquist-plane term that the generator drops
    dkn = dk.copy()
    dkn[:, :, : nf // 2] = 0
    nyq = -(np.roll(sfft.irfftn(Kc * dkn, s=(nf, nf, nf)), -1, axis=2)
            - np.roll(sfft.irfftn(Kc * dkn, s=(nf, nf, nf)), 1, axis=2)) / (8 * np.pi)
    assert np.allclose(psi, gx - nyq, atol=1e-6 * np.abs(gx).max())


def test_device_ic_params_reproduce_delta2():
    c = ic.Cosmology()
    z_i, box = 49.0, 200.0
    q = ic.device_ic_params(c, z_i, 16, box=box)
    k = np.logspace(-2, 1, 50)
    # the device expression: norm_d2 * T(k)^2 * k^(3+n_s), T from the EH constants
    k_mpc = k * q["h"]
    x = 0.43 * k_mpc * q["eh_s"]
    gamma = q["eh_omh"] * (q["eh_alpha"] + (1.0 - q["eh_alpha"]) / (1.0 + x ** 4))
    qq = k * q["eh_theta2"] / gamma
    l0 = np.log(2.0 * math.e + 1.8 * qq)
    c0 = 14.2 + 731.0 / (1.0 + 62.5 * qq)
    t = l0 / (l0 + c0 * qq * qq)
    dev = q["norm_d2"] * t * t * k ** (3.0 + q["n_s"])
    np.testing.assert_allclose(dev, ic.delta2(k, c, 1.0 / (1.0 + z_i)), rtol=1e-12)
    assert q["a"] == pytest.approx(1.0 / (1.0 + z_i))
    assert q["vf"] == pytest.approx(ic.vfactor(q["a"], c.omega_m, c.omega_l))


def _decode(st_like, nc, nnt, izipx, izipv, sigma):
    """Positions (coarse units) and velocities of a checkpoint-layout state, by PID."""
    xp, vp, pid, rhoc, vfield = st_like
    nt = nc // nnt
    cells = np.arange(nc ** 3)
    l = cells % nt ** 3
    tile = cells // nt ** 3
    g = np.stack([(tile % nnt) * nt + l % nt, ((tile // nnt) % nnt) * nt + (l // nt) % nt,
                  (tile // (nnt * nnt)) * nt + l // (nt * nt)], axis=1)
    cell_of = np.repeat(cells, rhoc.astype(np.int64))
    mask = 0xFF if izipx == 1 else 0xFFFF
    frac = ((xp.astype(np.int64) & mask) + 0.5) / (256.0 if izipx == 1 else 65536.0)
    pos = g[cell_of] + frac
    nvbin = 1 << (8 * izipv)
    pif = float(ic.pi_f32())
    coef = math.sqrt(pif / 2.0) / (sigma * 2.5)
    vel = np.tan(pif * vp.astype(np.float64) / (nvbin - 1)) / coef + vfield[cell_of].astype(np.float64)
    order = np.argsort(pid)
    return pid[order], pos[order], vel[order], cell_of[order]


@pytest.mark.gpu
@pytest.mark.parametrize("izip", [(2, 2), (1, 1), (2, 1)])
def test_gpu_ic_matches_host_generator(tables, izip):
    nc, nnt, box, z_i, seed = 32, 2, 200.0, 49.0, 21
    izipx, izipv = izip
    st, p, s_host = small_state(nc=nc, nnt=nnt, box=box, z_i=z_i, seed=seed, izipx=izipx, izipv=izipv)
    fk, ck = tables
    g = Cube(p, np_capacity=st.np, fk_table=fk, ck_table=ck)
    q = ic.device_ic_params(ic.Cosmology(), z_i, nc, box=box)
    s = g.make_ic(q, seed)
    xp, vp, pid, rhoc, vfield = g.store_state()
    assert xp.shape[0] == st.np and int(rhoc.sum()) == st.np
    # PIDs are 1 + the fine-mesh index of each lattice point (initial_conditions.f90:834-836),
    # each once, in lattice order inside a cell
    assert np.array_equal(np.sort(pid), np.sort(ic.lattice_pid(nc, 2)))
    assert np.array_equal(np.sort(pid), np.sort(st.pid))
    same_cell = np.repeat(np.arange(nc ** 3), rhoc)
    inner = same_cell[1:] == same_cell[:-1]
    assert np.all(pid[1:][inner] > pid[:-1][inner])
    # scalars
    assert s.a == pytest.approx(st.a, rel=1e-7)
    assert s.mass_p_cdm == st.mass_p_cdm
    assert s.sigma_vi == pytest.approx(st.sigma_vi, rel=1e-4)
    np.testing.assert_allclose(s.vmax[:], st.vmax, rtol=1e-4)
    assert s.nplocal == st.np and s.dt_vmax == pytest.approx(s_host.dt_vmax, rel=1e-4)
    # the FP32 FFTs of both generators differ by rounding only: a handful of particles
    # may land in the neighbouring cell, every position agrees to a few code steps
    assert np.mean(rhoc == st.rhoc) > 0.99
    a = _decode((xp, vp, pid, rhoc, vfield), nc, nnt, izipx, izipv, s.sigma_vi)
    b = _decode((st.xp, st.vp, st.pid, st.rhoc, st.vfield), nc, nnt, izipx, izipv, st.sigma_vi)
    assert np.array_equal(a[0], b[0])
    d = a[1] - b[1]
    d -= nc * np.round(d / nc)
    xres = 2.0 ** (-8 * izipx)
    assert np.max(np.abs(d)) <= 2 * xres + 1e-4
    assert np.mean(a[3] == b[3]) > 0.999
    # velocities agree to the codec's resolution at that velocity
    vs = float(np.std(b[2]))
    dv = np.abs(a[2] - b[2])
    tol = (5e-3 if izipv == 1 else 5e-5) * vs * (1.0 + (b[2] / vs) ** 2)
    assert np.mean(dv <= tol) > 0.999
    np.testing.assert_allclose(vfield[rhoc > 0].mean(axis=0), st.vfield[st.rhoc > 0].mean(axis=0), atol=1e-4 * vs)


@pytest.mark.gpu
def test_gpu_ic_then_steps(tables):
    nc, nnt, box, z_i, seed = 32, 2, 200.0, 49.0, 4
    p = make_params(nc, nnt, box=box)
    fk, ck = tables
    g = Cube(p, np_capacity=(2 * nc) ** 3, fk_table=fk, ck_table=ck)
    s = g.make_ic(ic.device_ic_params(ic.Cosmology(), z_i, nc, box=box), seed)
    n0 = s.nplocal
    for _ in range(2):
        g.step(s)
    assert s.nplocal == n0 and s.a > 1.0 / (1.0 + z_i)
    _, _, pid, rhoc, _ = g.store_state()
    assert int(rhoc.sum()) == n0 and np.array_equal(np.sort(pid), np.sort(ic.lattice_pid(nc, 2)))


@pytest.mark.gpu
def test_gpu_ic_rejects_bad_lattice(tables):
    nc, nnt = 16, 2
    p = make_params(nc, nnt, box=100.0)
    fk, ck = tables
    g = Cube(p, np_capacity=(2 * nc) ** 3, fk_table=fk, ck_table=ck)
    q = ic.device_ic_params(ic.Cosmology(), 49.0, nc, box=100.0, np_nc=3)
    with pytest.raises(Exception):
        g.make_ic(q, 1)  # 27 nc^3 particles exceed the capacity of 8 nc^3
