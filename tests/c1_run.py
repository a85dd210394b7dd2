"""Configuration 1 of the workload, run through the library and the CPU oracle in
lockstep -- test infrastructure.

Configuration 1: 64^3 CDM particles in a 200 Mpc/h periodic box, fine mesh 128^3,
coarse mesh 32^3 (2^3 tiles), PP off, int1 positions with int2 velocities, flat
LCDM (Om = 0.3, OL = 0.7, h = 0.7, s8 = 0.8, Eisenstein-Hu no-wiggle), seeded
Zel'dovich initial conditions at z = 49, 100 steps to z = 0 (the body of
main.f90:47-66: timestep, update_x, particle_mesh).

The 100 steps end on log-spaced scale factors: each step is the reference's
adaptive timestep (timestep.f90:1-95) snapped onto the next target the way its
checkpoints are (timestep.f90:46-61).  Both arms call the library's timestep with
the library's dt limits (dt_fine, dt_coarse, dt_vmax of the GPU arm), so they take
the same time steps and differ only by their step arithmetic.
"""
from __future__ import annotations

import numpy as np

from cube_nufluid_b200 import Cube, ic, tables
from cube_nufluid_b200.abi import make_params
from cube_nufluid_b200.cube import load_library, scalars_from_ic
from oracle_ref import Oracle
import pk_ref

C1 = dict(nc=32, nnt=2, box=200.0, z_i=49.0, izipx=1, izipv=2, steps=100)
LIMITS = ("dt_fine", "dt_coarse", "dt_pp", "dt_vmax", "dt_vmax_nu", "dt_neu")


def c1_state(seed: int = 2024):
    st = ic.zeldovich(C1["nc"], C1["nnt"], box=C1["box"], z_i=C1["z_i"], seed=seed, izipx=C1["izipx"],
                      izipv=C1["izipv"])
    p = make_params(C1["nc"], C1["nnt"], box=C1["box"], izipx=C1["izipx"], izipv=C1["izipv"], ext_pp_force=False)
    return st, p


def targets(a0: float, steps: int) -> np.ndarray:
    return np.geomspace(a0, 1.0, steps + 1)[1:]


def _timestep(p, s, a_next) -> bool:
    import ctypes as C
    hit = C.c_int32(0)
    load_library().cube_timestep(C.byref(p), C.byref(s), C.c_float(a_next), C.byref(hit))
    return bool(hit.value)


def run_lockstep(st, p, steps: int = 100, deposit_mode: int = 1, libm_codec: bool = False, max_substeps: int = 400):
    """Both arms from the same state over `steps` target scale factors; returns
    (final GPU state, final oracle state, GPU scalars, oracle scalars, steps taken)."""
    fk, ck = tables.read_fine_table(), tables.read_coarse_table()
    g = Cube(p, st.np, fk, ck)
    g.load_state(st.xp, st.vp, st.pid, st.rhoc, st.vfield)
    o = Oracle(p, fk, ck)
    o.load(st.xp, st.vp, st.pid, st.rhoc, st.vfield)
    if libm_codec:
        o.set_libm_codec(True)
    sg = scalars_from_ic(st)
    so = sg.copy()
    n = 0
    for a_next in targets(float(sg.a), steps):
        hit = False
        while not hit:
            for k in LIMITS:
                setattr(so, k, getattr(sg, k))
            hit = _timestep(p, sg, float(a_next))
            _timestep(p, so, float(a_next))
            assert sg.a == so.a and sg.dt == so.dt
            g.update_x(sg)
            o.update_x(so)
            g.particle_mesh(sg)
            o.particle_mesh(so, deposit_mode)
            n += 1
            assert n <= max_substeps
    out = g.store_state(), o.store(), sg, so, n
    g.close()
    return out


def positions_by_pid(state, nc, nnt, izipx) -> np.ndarray:
    """Coarse-unit positions [np, 3] ordered by PID."""
    xp, vp, pid, rhoc, vf = state

    class S:
        pass
    s = S()
    s.nc, s.nnt, s.izipx, s.xp, s.rhoc = nc, nnt, izipx, xp, rhoc
    pos = pk_ref.particle_positions(s)
    order = np.argsort(pid, kind="stable")
    return pos[order], pid[order]


def periodic_diff(a: np.ndarray, b: np.ndarray, n: float) -> np.ndarray:
    d = a - b
    return d - n * np.round(d / n)


def power(pos: np.ndarray, nc: int, box: float, ng: int, nbins32: int = 32):
    """P(k) of the positions: the reference's log bins (cross_power, 4 per octave)
    and 32 equal-log bins from the fundamental to the Nyquist frequency."""
    d = pk_ref.cic_delta(pos, nc, ng)
    xi = pk_ref.cross_power(d, None, box, log_bins=True)
    c = np.fft.rfftn(d) / ng ** 3
    kz, ky, kx = np.meshgrid(np.fft.fftfreq(ng, 1.0 / ng), np.fft.fftfreq(ng, 1.0 / ng), np.arange(ng // 2 + 1),
                             indexing="ij")
    kr = np.sqrt(kx ** 2 + ky ** 2 + kz ** 2)
    edges = np.geomspace(1.0, ng / 2, nbins32 + 1)
    ib = np.digitize(kr, edges) - 1
    keep = (ib >= 0) & (ib < nbins32) & (kr > 0)
    w = np.where(kx == 0, 1.0, 2.0)  # the half spectrum's mirrored modes
    p = np.bincount(ib[keep], weights=(w * np.abs(c) ** 2)[keep], minlength=nbins32)
    m = np.bincount(ib[keep], weights=w[keep], minlength=nbins32)
    return xi, p / np.maximum(m, 1), m
