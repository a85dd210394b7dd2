"""Seeded Zel'dovich initial conditions in CUBE's compressed checkpoint layout.

This is the input harness of the particle-mesh step, restating the particle
creation of the reference IC program (CUBE_v2.0/work/utilities/initial_conditions.f90)
on a host with numpy:

* linear power: Eisenstein & Hu (1998, ApJ 496, 605) no-wiggle transfer function
  (their eqs. 26-31), n_s tilt, normalised to sigma_8 with the reference's top-hat
  integral (initial_conditions.f90:235-242, tophat :1017-1026);
* growth to z_i with the reference's Dgrow (initial_conditions.f90:1028-1041);
* unit Gaussian white noise from a counter-based generator (numpy's Philox4x32-10,
  Salmon et al. 2011) seeded explicitly, scaled as at initial_conditions.f90:373;
* the potential on the fine mesh with the reference's corrected discrete-Laplacian
  kernel (potential_kernel; initial_conditions.f90:449-523) and the Zel'dovich
  displacement -(phi(i+1) - phi(i-1))/(8 pi) at each lattice particle's fine cell,
  velocity v = psi * vfactor(a) (initial_conditions.f90:794-799, vfactor :1068-1079);
* zip packing as at initial_conditions.f90:797-838: cell g = ceiling(x),
  xp = floor(x/x_resolution) wrapped to the code width, vfield = mean particle
  velocity of the cell, vp = arctan code of v - vfield, pid = 1 + the fine-mesh
  index of the lattice point, iq = (ncell/np_nc)*lattice index per dimension,
  pid = iq_x + nf*iq_y + nf^2*iq_z + 1 (initial_conditions.f90:834-836).

Particles sit on a lattice of np_nc per coarse cell per dimension and are
ordered tile-major by coarse cell, lattice order inside a cell.  The linear power
comes from the Eisenstein-Hu formula where the reference reads a CAMB table, and
the noise from Philox where it calls the compiler's random_number.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np


@dataclass
class Cosmology:
    omega_m: float = 0.3
    omega_l: float = 0.7
    h: float = 0.7
    omega_b: float = 0.045
    n_s: float = 0.96
    sigma8: float = 0.8
    t_cmb: float = 2.7255


def eh_nowiggle(k_hmpc: np.ndarray, c: Cosmology) -> np.ndarray:
    """Eisenstein & Hu (1998) zero-baryon-oscillation transfer function, k in h/Mpc."""
    om = c.omega_m * c.h * c.h
    ob = c.omega_b * c.h * c.h
    fb = c.omega_b / c.omega_m
    theta = c.t_cmb / 2.7
    s = 44.5 * math.log(9.83 / om) / math.sqrt(1.0 + 10.0 * ob ** 0.75)  # Mpc
    alpha = 1.0 - 0.328 * math.log(431.0 * om) * fb + 0.38 * math.log(22.3 * om) * fb * fb
    k_mpc = k_hmpc * c.h
    gamma = c.omega_m * c.h * (alpha + (1.0 - alpha) / (1.0 + (0.43 * k_mpc * s) ** 4))
    q = k_hmpc * theta * theta / gamma
    l0 = np.log(2.0 * math.e + 1.8 * q)
    c0 = 14.2 + 731.0 / (1.0 + 62.5 * q)
    return l0 / (l0 + c0 * q * q)


# Philox4x32-10 (Salmon, Moraes, Dror and Shaw, "Parallel random numbers: as easy as
# 1, 2, 3", SC 2011): the counter-based generator shared by the host and the device
# initial conditions.  Word i of the noise grid is output word i mod 4 of the block
# with counter (i div 4 low 32 bits, high 32 bits, 0, 0) and key (seed low, seed high).
PHILOX_M0, PHILOX_M1 = 0xD2511F53, 0xCD9E8D57
PHILOX_W0, PHILOX_W1 = 0x9E3779B9, 0xBB67AE85


def philox4x32_10(ctr: np.ndarray, key: tuple[int, int]) -> np.ndarray:
    """ctr: uint32 [..., 4]; returns the uint32 [..., 4] output block."""
    c = [ctr[..., i].astype(np.uint64) for i in range(4)]
    k0, k1 = np.uint64(key[0] & 0xFFFFFFFF), np.uint64(key[1] & 0xFFFFFFFF)
    m32 = np.uint64(0xFFFFFFFF)
    for r in range(10):
        p0 = np.uint64(PHILOX_M0) * c[0]
        p1 = np.uint64(PHILOX_M1) * c[2]
        hi0, lo0 = p0 >> np.uint64(32), p0 & m32
        hi1, lo1 = p1 >> np.uint64(32), p1 & m32
        c = [(hi1 ^ c[1] ^ k0) & m32, lo1, (hi0 ^ c[3] ^ k1) & m32, lo0]
        k0 = (k0 + np.uint64(PHILOX_W0)) & m32
        k1 = (k1 + np.uint64(PHILOX_W1)) & m32
    return np.stack([x.astype(np.uint32) for x in c], axis=-1)


def uniform_noise(n: int, seed: int) -> np.ndarray:
    """Uniforms in [0,1) on an n^3 grid [z][y][x]: (word >> 8) * 2^-24 of the Philox stream."""
    total = n ** 3
    blocks = (total + 3) // 4
    out = np.empty(blocks * 4, np.float32)
    step = 1 << 22
    for b0 in range(0, blocks, step):
        b = np.arange(b0, min(blocks, b0 + step), dtype=np.uint64)
        ctr = np.zeros((len(b), 4), np.uint32)
        ctr[:, 0] = (b & np.uint64(0xFFFFFFFF)).astype(np.uint32)
        ctr[:, 1] = (b >> np.uint64(32)).astype(np.uint32)
        w = philox4x32_10(ctr, (seed & 0xFFFFFFFF, (seed >> 32) & 0xFFFFFFFF))
        out[4 * b0:4 * b0 + 4 * len(b)] = (w >> np.uint32(8)).astype(np.float32).reshape(-1) * np.float32(2.0 ** -24)
    return out[:total].reshape(n, n, n)


def gaussian_noise(n: int, seed: int) -> np.ndarray:
    """Unit Gaussian noise [z][y][x] (float32): Philox4x32-10 uniforms through the
    reference's Box-Muller pairing along x (initial_conditions.f90:320-336)."""
    if n % 2:
        raise ValueError("noise grid must be even along x")
    u = uniform_noise(n, seed)
    pif = pi_f32()
    theta = np.float32(2.0) * pif * u[..., 0::2]
    r = np.sqrt(np.float32(-2.0) * np.log(np.float32(1.0) - u[..., 1::2]))
    out = np.empty_like(u)
    out[..., 0::2] = r * np.cos(theta)
    out[..., 1::2] = r * np.sin(theta)
    return out


def _tophat(x):
    x = np.asarray(x, dtype=np.float64)
    out = np.ones_like(x)
    nz = x != 0
    xx = x[nz]
    out[nz] = 3.0 * (np.sin(xx) - np.cos(xx) * xx) / xx ** 3
    return out


def dgrow(a: float, om: float, ol: float) -> float:
    """Carroll-Press-Turner growth as in initial_conditions.f90:1028-1041."""
    def g(aa):
        hsq = om / aa ** 3 + (1 - om - ol) / aa ** 2 + ol
        oma = om / (aa ** 3 * hsq)
        ola = ol / hsq
        return 2.5 * oma / (oma ** (4.0 / 7) - ola + (1 + oma / 2) * (1 + ola / 70))
    return a * g(a) / g(1.0)


def vfactor(a: float, om: float, ol: float, f_neu: float = 0.0) -> float:
    """a^2 H(a) times the growth exponent, simulation units (initial_conditions.f90:1068-1079)."""
    npow = -(1.0 / 4.0) + (5.0 / 4.0) * math.sqrt(1 - 24.0 * f_neu / 25.0)
    lm = ol / om
    km = (1 - om - ol) / om
    hub = 2 / (3 * math.sqrt(a ** 3)) * math.sqrt(1 + a * km + a ** 3 * lm)
    return a * a * hub * npow


def delta2(k_hmpc, c: Cosmology, a: float):
    """Dimensionless linear power Delta^2(k) = k^3 P(k)/(2 pi^2) at scale factor a."""
    kk = np.logspace(-4, 2, 4000)
    t = eh_nowiggle(kk, c)
    d2 = t * t * kk ** (3 + c.n_s)
    w = _tophat(kk * 8.0)
    v8 = np.trapezoid(d2 * w * w / kk, kk)
    norm = c.sigma8 ** 2 / v8
    tk = eh_nowiggle(np.asarray(k_hmpc, dtype=np.float64), c)
    d = dgrow(a, c.omega_m, c.omega_l)
    return norm * tk * tk * np.asarray(k_hmpc, dtype=np.float64) ** (3 + c.n_s) * d * d


def pi_f32() -> np.float32:
    return np.float32(4.0) * np.arctan(np.float32(1.0))


def encode_velocity(v: np.ndarray, sigma: float, izipv: int, vrel_boost: float = 2.5) -> np.ndarray:
    """Host encode used only to pack ICs (the step's encode is cube_vencode on the device)."""
    pif = pi_f32()
    nvbin_m1 = np.float32((1 << (8 * izipv)) - 1)
    coef = float(np.sqrt(pif / np.float32(2.0))) / (float(np.float32(sigma)) * vrel_boost)
    q = (float(nvbin_m1) * np.arctan(coef * v)) / float(pif)
    code = np.sign(q) * np.floor(np.abs(q) + 0.5)
    dt = np.int8 if izipv == 1 else np.int16
    return code.astype(np.int64).astype(dt)


@dataclass
class ICState:
    nc: int
    nnt: int
    izipx: int
    izipv: int
    xp: np.ndarray       # [np,3] int8/int16
    vp: np.ndarray       # [np,3]
    pid: np.ndarray      # [np] int32
    rhoc: np.ndarray     # [ncells] int32, tile-major cell order
    vfield: np.ndarray   # [ncells,3] float32
    a: float
    sigma_vi: float
    mass_p_cdm: float
    vmax: np.ndarray     # [3]
    vsim2phys: float

    @property
    def np(self) -> int:
        return int(self.pid.shape[0])


def tile_major_cell_id(g: np.ndarray, nc: int, nnt: int) -> np.ndarray:
    """g: [...,3] zero-based global coarse cell -> tile-major cell id (Fortran rhoc order)."""
    nt = nc // nnt
    t = g // nt
    l = g % nt
    tile = (t[..., 2] * nnt + t[..., 1]) * nnt + t[..., 0]
    return ((tile * nt + l[..., 2]) * nt + l[..., 1]) * nt + l[..., 0]


def _linear_delta_k(npd: int, box: float, a: float, seed: int, c: Cosmology, amplitude: float):
    """Linear density contrast in Fourier space on an npd^3 grid (the fine mesh for
    the particles, the particle grid for the neutrino fluids) from the seeded noise
    (initial_conditions.f90:320-420): noise * sqrt(P(k)) at scale factor a."""
    import scipy.fft as sfft
    noise = gaussian_noise(npd, seed)  # [z][y][x]
    wk = sfft.rfftn(noise, workers=-1)
    del noise
    kx = np.fft.rfftfreq(npd, d=1.0 / npd).astype(np.float32)
    ky = np.fft.fftfreq(npd, d=1.0 / npd).astype(np.float32)
    kz = ky
    kr2 = kz[:, None, None] ** 2 + ky[None, :, None] ** 2 + kx[None, None, :] ** 2
    kr = np.sqrt(np.maximum(kr2, 1.0))
    d2 = delta2(2 * math.pi * kr / box, c, a).astype(np.float32)
    amp = np.sqrt(d2 / (4 * math.pi) * (npd / kr)) * (npd / kr) * amplitude
    dk = wk * amp
    dk[0, 0, 0] = 0
    return dk, kx, ky, kz, kr2


# radius (in mesh cells) inside which the potential kernel is the exact -1/r
EWALD_R = 8


def potential_kernel(n: int) -> np.ndarray:
    """The reference's potential kernel on a periodic n^3 mesh, in k space, full
    [z][y][x] (initial_conditions.f90:449-523): -4 pi/khat^2 with the discrete
    Laplacian khat^2 = sum_d (2 sin(pi m_d/n))^2, zero at k = 0; with its kernel
    correction (correct_kernel): its real-space form K_r (the inverse transform, 1/n^3
    normalised) is replaced within r <= 8 cells by the exact -1/r (-2.5 at r = 0) and
    shifted beyond by -(phi8 + 1/8), phi8 = the mean of K_r at distance 8 on the six
    axes, and transformed back.  As a correction in k space: K + FFT(w), w(r) =
    exact(r) - K_r(r) + phi8 + 1/8 on the cells within r <= 8 (the constant shift of
    every other cell only moves k = 0, which stays zero).  K is real and even, so its
    inverse transform is its forward one over n^3.  Meshes of fewer than 2*8+2 cells
    per side take the kernel without the correction."""
    m = np.fft.fftfreq(n, d=1.0 / n)
    s2 = (2.0 * np.sin(np.pi * m / n)) ** 2
    kr = s2[:, None, None] + s2[None, :, None] + s2[None, None, :]
    K = np.zeros_like(kr)
    nz = kr > 0
    K[nz] = -4.0 * np.pi / kr[nz]
    if n < 2 * EWALD_R + 2:
        return K
    Kr = np.fft.fftn(K).real / float(n) ** 3
    R = EWALD_R
    phi8 = (Kr[R, 0, 0] + Kr[n - R, 0, 0] + Kr[0, R, 0] + Kr[0, n - R, 0] + Kr[0, 0, R] + Kr[0, 0, n - R]) / 6.0
    r = np.arange(-R, R + 1)
    rz, ry, rx = np.meshgrid(r, r, r, indexing="ij")
    d = np.sqrt(rx * rx + ry * ry + rz * rz)
    sel = d <= R
    exact = np.where(d > 0, -1.0 / np.where(d > 0, d, 1.0), -2.5)
    iz, iy, ix = rz[sel] % n, ry[sel] % n, rx[sel] % n
    w = np.zeros((n, n, n))
    w[iz, iy, ix] = exact[sel] - Kr[iz, iy, ix] + (phi8 + 1.0 / R)
    K = K + np.fft.fftn(w).real
    K[0, 0, 0] = 0.0
    return K


def zeldovich(nc: int, nnt: int, box: float, z_i: float, seed: int, *, np_nc: int = 2,
              ncell: int = 4, izipx: int = 2, izipv: int = 2, cosmo: Cosmology | None = None,
              f_cdm: float = 1.0, amplitude: float = 1.0) -> ICState:
    """Build a seeded Zel'dovich state at z_i in checkpoint layout, by the reference's
    method (initial_conditions.f90:449-836): the linear density on the fine mesh, the
    potential phi = K * delta with the corrected discrete-Laplacian kernel of
    potential_kernel, and each particle (lattice spacing ncell/np_nc fine cells, at
    the centre of its fine cell) displaced by -(phi(i+1) - phi(i-1))/(8 pi) fine cells
    along each axis, with velocity that displacement times the growth factor vf.  The
    central difference is applied in k space, where it is the multiplier
    2 i sin(2 pi m_d/nf)."""
    c = cosmo or Cosmology()
    nf = nc * ncell
    npd = nc * np_nc
    st = ncell // np_nc
    if ncell % np_nc:
        raise ValueError("np_nc must divide ncell")
    a = 1.0 / (1.0 + z_i)
    import scipy.fft as sfft
    dk, kx, ky, kz, kr2 = _linear_delta_k(nf, box, a, seed, c, amplitude)
    Kc = potential_kernel(nf)[:, :, : nf // 2 + 1].astype(np.float32)
    disp = np.empty((3, npd, npd, npd), dtype=np.float32)
    for d, kk in enumerate((kx[None, None, :], ky[None, :, None], kz[:, None, None])):
        g = (-np.sin(2.0 * np.pi * kk.astype(np.float64) / nf) / (4.0 * np.pi)).astype(np.float32)
        g = np.where(np.abs(kk) == nf // 2, np.float32(0), g)  # zero on the own-dimension Nyquist plane
        psi_k = 1j * g * Kc * dk
        disp[d] = sfft.irfftn(psi_k, s=(nf, nf, nf), workers=-1)[::st, ::st, ::st]  # fine cells
        del psi_k
    del dk, Kc
    # lattice positions in coarse units: q = i/np_nc + 0.5/ncell (initial_conditions.f90:793)
    ii = np.arange(npd, dtype=np.float64) / np_nc + 0.5 / ncell
    zz, yy, xx = np.meshgrid(ii, ii, ii, indexing="ij")
    pos = np.stack([xx, yy, zz], axis=-1).reshape(-1, 3)
    del xx, yy, zz
    dsp = np.stack([disp[0], disp[1], disp[2]], axis=-1).reshape(-1, 3).astype(np.float64) / ncell
    del disp
    x = np.mod(pos + dsp, float(nc))
    vf = vfactor(a, c.omega_m, c.omega_l)
    vel = dsp * (ncell * vf)  # fine cells per unit time
    del pos, dsp
    return pack(x, vel, nc, nnt, ncell=ncell, izipx=izipx, izipv=izipv, a=a, box=box, omega_m=c.omega_m,
                f_cdm=f_cdm, pid_of=lattice_pid(nc, np_nc, ncell))


def lattice_pid(nc: int, np_nc: int, ncell: int = 4) -> np.ndarray:
    """PID of each lattice point (x fastest): 1 + its fine-mesh index on the nf^3
    mesh, iq = (ncell/np_nc)*(lattice index) per dimension (initial_conditions.f90:834-836)."""
    npd = nc * np_nc
    nf = nc * ncell
    iq = (ncell // np_nc) * np.arange(npd, dtype=np.int64)
    z, y, x = np.meshgrid(iq, iq, iq, indexing="ij")
    return (x + nf * y + nf * nf * z + 1).reshape(-1).astype(np.int32)



def clustered(nc: int, nnt: int, npart: int, seed: int, *, ncell: int = 4, izipx: int = 2, izipv: int = 2,
              clumps: int = 8, clump_frac: float = 0.5, clump_size: float = 0.6, vel: float = 0.02,
              box: float = 100.0) -> ICState:
    """A test state with uniform background plus dense clumps (crowded cells, PP pairs).

    Positions and velocities are drawn from Philox4x32-10 with the given seed
    and packed exactly as zeldovich() packs them.  Not a cosmological IC: it
    exercises the step on the clustering a late-time box has.
    """
    rng = np.random.Generator(np.random.Philox(seed))
    nclump = int(npart * clump_frac)
    nbg = npart - nclump
    xb = rng.uniform(0, nc, (nbg, 3))
    centers = rng.uniform(0, nc, (clumps, 3))
    which = rng.integers(0, clumps, nclump)
    xc = centers[which] + rng.normal(0, clump_size, (nclump, 3))
    x = np.mod(np.concatenate([xb, xc]), float(nc))
    v = rng.normal(0, vel, (npart, 3))
    v[nbg:] += rng.normal(0, 2 * vel, (clumps, 3))[which]
    return pack(x, v, nc, nnt, ncell=ncell, izipx=izipx, izipv=izipv, a=0.5, box=box)


def pack(x: np.ndarray, vel: np.ndarray, nc: int, nnt: int, *, ncell: int = 4, izipx: int = 2, izipv: int = 2,
         a: float = 0.02, box: float = 100.0, omega_m: float = 0.3, f_cdm: float = 1.0,
         pid_of: np.ndarray | None = None) -> ICState:
    """Zip packing of initial_conditions.f90:797-838 for positions x (coarse units) and velocities;
    pid_of[i] is particle i's PID (default i + 1)."""
    g = np.ceil(x).astype(np.int64) - 1
    g %= nc
    cid = tile_major_cell_id(g, nc, nnt)
    order = np.argsort(cid, kind="stable")
    cid = cid[order]
    x = x[order]
    vel = vel[order]
    pid = (order + 1).astype(np.int32) if pid_of is None else np.asarray(pid_of, np.int32)[order]
    ncells = nc ** 3
    rhoc = np.bincount(cid, minlength=ncells).astype(np.int32)
    vsum = np.stack([np.bincount(cid, weights=vel[:, d], minlength=ncells) for d in range(3)], axis=-1)
    vfield = (vsum / np.maximum(rhoc, 1)[:, None]).astype(np.float32)
    res = vel - vfield[cid].astype(np.float64)
    sigma_vi = float(np.float32(math.sqrt(float(np.mean(np.sum(res * res, axis=1)))) / math.sqrt(3.0)))
    xres = 2.0 ** (-8 * izipx)
    xcode = np.floor(x / xres).astype(np.int64)
    xdt = np.int8 if izipx == 1 else np.int16
    xp = (xcode & ((1 << (8 * izipx)) - 1)).astype(np.uint16 if izipx == 2 else np.uint8).view(xdt)
    vp = encode_velocity(res, sigma_vi, izipv)
    npart = x.shape[0]
    nf = nc * ncell
    mass_p = float(np.float32(f_cdm * float(nf) ** 3 / npart))
    vmax = np.max(np.abs(vel), axis=0)
    vsim2phys = (150.0 / a) * box * math.sqrt(omega_m) / nf
    return ICState(nc=nc, nnt=nnt, izipx=izipx, izipv=izipv, xp=np.ascontiguousarray(xp),
                   vp=np.ascontiguousarray(vp), pid=pid, rhoc=rhoc, vfield=vfield, a=a,
                   sigma_vi=sigma_vi, mass_p_cdm=mass_p, vmax=vmax.astype(np.float32), vsim2phys=vsim2phys)


def nu_fluid_perturbed(nc: int, seed: int, *, cs2: float, gamma: float = np.float32(5.0) / np.float32(3.0),
                       amp_rho: float = 0.2, amp_v: float = 0.5) -> np.ndarray:
    """A smooth seeded fluid state fld(1:5,1:nc,1:nc,1:nc) as float32 [nc,nc,nc,5]
    (z, y, x, component): rho = 1 + amp_rho*s, momentum = rho*v with
    v = amp_v*sqrt(cs2)*s', energy = rho*cs2/(g-1) + |m|^2/(2 rho) -- the
    composition neutrino_ic.f90 builds (density, isotropic stress, kinetic
    energy), on a band-limited random field instead of the linear one."""
    f32 = np.float32
    k = np.fft.fftfreq(nc) * nc
    kk = np.sqrt(k[:, None, None] ** 2 + k[None, :, None] ** 2 + k[None, None, :] ** 2)
    filt = np.exp(-(kk / max(nc / 8.0, 1.0)) ** 2)

    def field(s):
        w = np.fft.ifftn(np.fft.fftn(gaussian_noise(nc, s)) * filt).real
        return (w / max(np.abs(w).max(), 1e-30)).astype(f32)

    rho = (f32(1.0) + f32(amp_rho) * field(seed)).astype(f32)
    cs = f32(np.sqrt(f32(cs2)))
    out = np.zeros((nc, nc, nc, 5), f32)
    out[..., 0] = rho
    e = rho * f32(cs2) / (f32(gamma) - f32(1.0))
    for d in range(3):
        v = (f32(amp_v) * cs * field(seed + 1 + d)).astype(f32)
        m = (rho * v).astype(f32)
        out[..., 1 + d] = m
        e = (e + f32(0.5) * m * m / rho).astype(f32)
    out[..., 4] = e
    return out


def nu_fluid_linear(nc: int, box: float, z: float, seed: int, *, fluid_n: int, gl_v: float, m_nu_ev: float,
                    cs2: float, z_i_nu: float = 10.0, np_nc: int = 2, ncell: int = 4,
                    cosmo: Cosmology | None = None, amplitude: float = 1.0,
                    gamma: float = np.float32(5.0) / np.float32(3.0)) -> np.ndarray:
    """One Gauss-Laguerre fluid's initial state fld(1:5,1:n,1:n,1:n) as float32
    [n,n,n,5], following neutrino_ic.f90:46-181 on the seeded field of zeldovich():
    delta_nu = delta_L * 1/(1+l+l^2), v_nu = v_L * (1+1.5l+2l^2)/(1+l+l^2)^2 with
    l = k/k_fs, k_fs = sqrt(1.5 Om/(1+z_i_nu))*100 / v_nu and v_nu = u c/(beta m)
    (:11,:52-58,:77,:147); the fields are built on the particle grid and averaged
    to the fluid's n^3 cells (hydrogr.f90:288-308 set_fld); rho = 1 + delta,
    E = rho cs2/(g-1) + sum m_d^2/(2 rho) (:91-94,:162-166)."""
    import scipy.fft as sfft
    c = cosmo or Cosmology()
    npd = nc * np_nc
    a = 1.0 / (1.0 + z)
    dk, kx, ky, kz, kr2 = _linear_delta_k(npd, box, a, seed, c, amplitude)
    kgrid = 2 * math.pi / npd
    kphys = np.sqrt(kr2) * (2 * math.pi / box)
    kfs1 = math.sqrt(1.5 * c.omega_m / (1.0 + z_i_nu)) * 100.0
    vneu = gl_v / 5966.34 * 2.998e5 / m_nu_ev
    ll = (kphys / (kfs1 / vneu)).astype(np.float32)
    t_rho = 1.0 / (1.0 + ll + ll * ll)
    t_v = (1.0 + 1.5 * ll + 2.0 * ll * ll) * t_rho * t_rho
    if fluid_n <= 0 or npd % fluid_n:
        raise ValueError("the fluid mesh must divide the particle grid")
    r = npd // fluid_n

    def down(f):
        f = f.reshape(fluid_n, r, fluid_n, r, fluid_n, r).astype(np.float64)
        return f.mean(axis=(1, 3, 5)).astype(np.float32)

    rho = (1.0 + down(sfft.irfftn(dk * t_rho, s=(npd,) * 3, workers=-1))).astype(np.float32)
    out = np.zeros((fluid_n, fluid_n, fluid_n, 5), np.float32)
    out[..., 0] = rho
    e = (rho * np.float32(cs2) / (np.float32(gamma) - np.float32(1.0))).astype(np.float32)
    inv = np.where(kr2 > 0, 1.0 / (kgrid * kgrid * np.maximum(kr2, 1e-30)), 0.0).astype(np.float32)
    vf = vfactor(a, c.omega_m, c.omega_l) * ncell / np_nc  # displacement (grid cells) -> fine cells / time
    for d, kk in enumerate((kx[None, None, :], ky[None, :, None], kz[:, None, None])):
        vk = (1j * (kgrid * kk) * inv * dk) * (t_v * np.float32(vf))
        v = down(sfft.irfftn(vk, s=(npd,) * 3, workers=-1))
        m = (rho * v).astype(np.float32)
        out[..., 1 + d] = m
        e = (e + np.float32(0.5) * m * m / rho).astype(np.float32)
    out[..., 4] = e
    return out


def device_ic_params(c: Cosmology, z_i: float, nc: int, *, np_nc: int = 2, ncell: int = 4,
                     box: float = 200.0, amplitude: float = 1.0) -> dict:
    """The scalars the device initial conditions need (cube_make_ic): the linear power
    normalisation sigma8^2/v8 * D(a)^2 and the Eisenstein-Hu constants, so the device
    evaluates Delta^2(k) = norm * T(k)^2 * k^(3+n_s) per mode exactly as delta2() does."""
    a = 1.0 / (1.0 + z_i)
    kk = np.logspace(-4, 2, 4000)
    t = eh_nowiggle(kk, c)
    w = _tophat(kk * 8.0)
    v8 = np.trapezoid(t * t * kk ** (3 + c.n_s) * w * w / kk, kk)
    d = dgrow(a, c.omega_m, c.omega_l)
    om = c.omega_m * c.h * c.h
    ob = c.omega_b * c.h * c.h
    fb = c.omega_b / c.omega_m
    return {
        "norm_d2": c.sigma8 ** 2 / v8 * d * d, "n_s": c.n_s, "h": c.h,
        "eh_s": 44.5 * math.log(9.83 / om) / math.sqrt(1.0 + 10.0 * ob ** 0.75),
        "eh_alpha": 1.0 - 0.328 * math.log(431.0 * om) * fb + 0.38 * math.log(22.3 * om) * fb * fb,
        "eh_omh": c.omega_m * c.h, "eh_theta2": (c.t_cmb / 2.7) ** 2,
        "vf": vfactor(a, c.omega_m, c.omega_l), "a": a, "box": box, "amplitude": amplitude,
        "np_nc": np_nc, "ncell": ncell, "omega_m": c.omega_m,
    }
