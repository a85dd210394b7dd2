"""Shared set-up of the parity tests: seeded states and scalar blocks."""
from __future__ import annotations

import numpy as np

from cube_nufluid_b200 import ic
from cube_nufluid_b200.abi import CubeScalars, make_params
from cube_nufluid_b200.cube import scalars_from_ic


def small_state(nc=16, nnt=2, box=100.0, z_i=49.0, seed=1, izipx=2, izipv=2, amplitude=1.0):
    st = ic.zeldovich(nc, nnt, box=box, z_i=z_i, seed=seed, izipx=izipx, izipv=izipv, amplitude=amplitude)
    p = make_params(nc, nnt, box=box, izipx=izipx, izipv=izipv)
    s = scalars_from_ic(st)
    return st, p, s


def clustered_state(nc=16, nnt=2, npart=40000, seed=3, izipx=2, izipv=2, box=100.0):
    st = ic.clustered(nc, nnt, npart, seed, izipx=izipx, izipv=izipv, box=box)
    p = make_params(nc, nnt, box=box, izipx=izipx, izipv=izipv)
    s = scalars_from_ic(st)
    return st, p, s


def copy_scalars(s: CubeScalars) -> CubeScalars:
    return s.copy()


def first_step_scalars(p, s, a_next):
    """timestep() of the library for both arms, so oracle and GPU see the same dt."""
    from cube_nufluid_b200.cube import load_library
    import ctypes as C
    L = load_library()
    hit = C.c_int32(0)
    L.cube_timestep(C.byref(p), C.byref(s), a_next, C.byref(hit))
    return s


def rel_rms(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.sqrt(np.mean((a - b) ** 2)) / max(np.sqrt(np.mean(b ** 2)), 1e-300))


# fluid neutrinos: 3 x 0.1 eV at h=0.67 (parameters.f90:80-93), FP32 as there
_F32 = np.float32
OMEGA_NU = _F32(3.0) * _F32(0.1) * _F32(1.0) / _F32(93.14) / (_F32(0.67) ** 2)
F_NEU = float(OMEGA_NU / (_F32(0.27 + 0.05) + OMEGA_NU))


def nu_params(nc=16, nnt=2, box=300.0, **kw):
    """Parameters with the fluid neutrinos of the reference's defaults."""
    return make_params(nc, nnt, box=box, neutrino=True, f_neu=F_NEU, m_nu_ev=0.1, z_i_nu=10.0,
                       omega_m=float(_F32(0.32) + OMEGA_NU), h0=0.67, **kw)


def kick_chain(force, a_mid, dt):
    """(((f*a_mid)*dt)/6)/pi in FP32 (pm.f90:146): what the library's force meshes
    hold after particle_mesh."""
    f32 = np.float32
    pif = f32(4.0) * np.arctan(f32(1.0))
    return ((((np.asarray(force, f32) * f32(a_mid)) * f32(dt)) / f32(6.0)) / pif).astype(f32)


def planted_clumps(nc=16, nnt=2, centres=((3.0, 4.0, 5.0), (11.0, 9.5, 3.0), (6.5, 12.0, 12.5), (14.5, 2.0, 9.0)),
                   n_per=3000, sigma=0.3, nbg=20000, seed=5, izipx=2, izipv=2, box=100.0, vel=0.02):
    """Uniform background plus Gaussian clumps at known centres (coarse units), packed
    in checkpoint layout; each clump moves with its own bulk velocity."""
    rng = np.random.Generator(np.random.Philox(seed))
    c = np.asarray(centres, np.float64)
    xb = rng.uniform(0, nc, (nbg, 3))
    xc = np.repeat(c, n_per, axis=0) + rng.normal(0, sigma, (len(c) * n_per, 3))
    x = np.mod(np.concatenate([xb, xc]), float(nc))
    v = rng.normal(0, vel, (x.shape[0], 3))
    v[nbg:] += np.repeat(rng.normal(0, 2 * vel, (len(c), 3)), n_per, axis=0)
    st = ic.pack(x, v, nc, nnt, izipx=izipx, izipv=izipv, a=0.5, box=box)
    p = make_params(nc, nnt, box=box, izipx=izipx, izipv=izipv)
    return st, p, scalars_from_ic(st)


def particle_positions(st, nc, nnt, ncell=4):
    """Fine-unit positions of a checkpoint-layout state in storage order."""
    nt = nc // nnt
    cells = np.arange(nc ** 3)
    l = cells % nt ** 3
    tile = cells // nt ** 3
    g = np.stack([(tile % nnt) * nt + l % nt, ((tile // nnt) % nnt) * nt + (l // nt) % nt,
                  (tile // (nnt * nnt)) * nt + l // (nt * nt)], axis=1)
    cell_of = np.repeat(cells, st.rhoc.astype(np.int64))
    mask = 0xFF if st.izipx == 1 else 0xFFFF
    frac = ((st.xp.astype(np.int64) & mask) + 0.5) / (256.0 if st.izipx == 1 else 65536.0)
    return ncell * (g[cell_of] + frac)
