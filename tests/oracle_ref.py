"""ctypes handle on the CPU oracle (oracle/liboracle.so) -- test infrastructure.

Only the tests, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
module, as the checker; the product never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from cube_nufluid_b200.abi import HALO_DTYPE, CubeHaloArgs, CubeHaloResult, CubeParams, CubeScalars

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
ORACLE_SO = os.path.join(ORACLE_DIR, "liboracle.so")

_lib = None


def build_oracle() -> str:
    subprocess.run(["make", "-s", "-C", ORACLE_DIR], check=True)
    return ORACLE_SO


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            build_oracle()
        L = C.CDLL(ORACLE_SO)
        P, S = C.POINTER(CubeParams), C.POINTER(CubeScalars)
        vp = C.c_void_p
        L.orc_create.restype = vp
        L.orc_create.argtypes = [P, vp, vp, C.c_int]
        L.orc_destroy.argtypes = [vp]
        L.orc_error.restype = C.c_char_p
        L.orc_error.argtypes = [vp]
        L.orc_load_state.argtypes = [vp, C.c_int64, vp, vp, vp, vp, vp]
        L.orc_store_state.argtypes = [vp, C.POINTER(C.c_int64), vp, vp, vp, vp, vp]
        L.orc_update_x.argtypes = [vp, S]
        L.orc_ext_pp_force.argtypes = [vp, S]
        L.orc_particle_mesh.argtypes = [vp, S, C.c_int]
        L.orc_particle_mesh_with_force.argtypes = [vp, S, C.c_int, vp, vp]
        L.orc_fetch.restype = C.c_int64
        L.orc_fetch.argtypes = [vp, C.c_int, vp, C.c_int64]
        L.orc_dt_constraints.argtypes = [vp, S]
        L.orc_halofind.argtypes = [vp, S, C.POINTER(CubeHaloArgs), C.POINTER(CubeHaloResult)]
        L.orc_set_tile_mask.argtypes = [vp, vp]
        L.orc_set_tile_mask.restype = None
        L.orc_coarse_poisson.argtypes = [vp]
        L.orc_coarse_poisson.restype = None
        L.orc_set_libm_codec.argtypes = [vp, C.c_int]
        L.orc_set_libm_codec.restype = None
        L.orc_tanf_code.restype = C.c_float
        L.orc_tanf_code.argtypes = [vp, C.c_int]
        L.orc_atan.restype = C.c_double
        L.orc_atan.argtypes = [C.c_double]
        L.orc_vencode.restype = C.c_int
        L.orc_vencode.argtypes = [vp, C.c_double, C.c_float]
        L.orc_vencode_libm.restype = C.c_int
        L.orc_vencode_libm.argtypes = [vp, C.c_double, C.c_float]
        L.orc_vdecode.restype = C.c_double
        L.orc_vdecode.argtypes = [vp, C.c_int, C.c_float]
        L.orc_tree_sum.restype = C.c_double
        L.orc_tree_sum.argtypes = [vp, C.c_int64]
        L.orc_nu_load.argtypes = [vp, C.c_int, vp]
        L.orc_nu_store.argtypes = [vp, C.c_int, vp]
        L.orc_nu_evolve.argtypes = [vp, C.c_float, C.POINTER(C.c_float), C.c_int, C.c_float]
        L.orc_nu_info.argtypes = [vp, vp]
        _lib = L
    return _lib


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class Oracle:
    def __init__(self, params: CubeParams, fk: np.ndarray, ck: np.ndarray, build_kernels: bool = True):
        self.p = params
        self.fk = np.ascontiguousarray(fk, dtype=np.float32)
        self.ck = np.ascontiguousarray(ck, dtype=np.float32)
        self.h = lib().orc_create(C.byref(params), _ptr(self.fk), _ptr(self.ck), int(build_kernels))
        self.nc = params.nc
        self.nf = params.nc * params.ncell

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_destroy(self.h)
            self.h = None

    def _check(self, rc):
        if rc != 0:
            raise RuntimeError(f"oracle error {rc}: {lib().orc_error(self.h).decode()}")

    def load(self, xp, vp, pid, rhoc, vfield):
        self._keep = (np.ascontiguousarray(xp), np.ascontiguousarray(vp),
                      None if pid is None else np.ascontiguousarray(pid, dtype=np.int32),
                      np.ascontiguousarray(rhoc, dtype=np.int32), np.ascontiguousarray(vfield, dtype=np.float32))
        x, v, p, r, f = self._keep
        self._check(lib().orc_load_state(self.h, x.shape[0], _ptr(x), _ptr(v), _ptr(p), _ptr(r), _ptr(f)))

    def set_libm_codec(self, on: bool = True):
        """Velocity encodes on the C library's atan, evaluated by the oracle itself
        (none of the library's codec code), instead of the shared project arctangent."""
        lib().orc_set_libm_codec(self.h, int(bool(on)))

    def set_tile_mask(self, mask):
        """Timing sample: the step routines run only the tiles marked in mask
        (nnt^3 entries, tile-major) and leave the state as it was; None clears it."""
        if mask is None:
            lib().orc_set_tile_mask(self.h, None)
        else:
            self._mask = np.ascontiguousarray(mask, dtype=np.int8)
            lib().orc_set_tile_mask(self.h, _ptr(self._mask))

    def coarse_poisson(self):
        """The global coarse Poisson solve of particle_mesh on the current r3."""
        lib().orc_coarse_poisson(self.h)

    def store(self):
        n = C.c_int64(0)
        lib().orc_store_state(self.h, C.byref(n), None, None, None, None, None)
        npart = n.value
        xdt = np.int8 if self.p.izipx == 1 else np.int16
        vdt = np.int8 if self.p.izipv == 1 else np.int16
        xp = np.zeros((npart, 3), xdt)
        vp = np.zeros((npart, 3), vdt)
        pid = np.zeros(npart, np.int32)
        rhoc = np.zeros(self.nc ** 3, np.int32)
        vf = np.zeros((self.nc ** 3, 3), np.float32)
        lib().orc_store_state(self.h, C.byref(n), _ptr(xp), _ptr(vp), _ptr(pid), _ptr(rhoc), _ptr(vf))
        return xp, vp, pid, rhoc, vf

    def update_x(self, s: CubeScalars):
        self._check(lib().orc_update_x(self.h, C.byref(s)))

    def ext_pp_force(self, s: CubeScalars):
        self._check(lib().orc_ext_pp_force(self.h, C.byref(s)))

    def particle_mesh(self, s: CubeScalars, deposit_mode: int = 1):
        self._check(lib().orc_particle_mesh(self.h, C.byref(s), deposit_mode))

    def particle_mesh_with_force(self, s: CubeScalars, fine: np.ndarray, coarse: np.ndarray, deposit_mode: int = 1):
        f = np.ascontiguousarray(fine, dtype=np.float32)
        c = np.ascontiguousarray(coarse, dtype=np.float32)
        self._check(lib().orc_particle_mesh_with_force(self.h, C.byref(s), deposit_mode, _ptr(f), _ptr(c)))

    def halofind(self, s: CubeScalars, *, den_odc: float = 200.0, capacity: int = 1 << 16,
                 member_capacity: int = 1 << 24, hid_len: int = 0):
        """halofind.f90 restated on the global periodic box (oracle hf::halofind):
        (halos as HALO_DTYPE, member PIDs, hid or None, number of density peaks)."""
        halos = np.zeros(capacity, HALO_DTYPE)
        mem = np.zeros(member_capacity, np.int32)
        hid = np.zeros(hid_len, np.int32) if hid_len > 0 else None
        a = CubeHaloArgs()
        a.den_odc, a.capacity, a.halos = float(den_odc), int(capacity), halos.ctypes.data
        a.member_pid, a.member_capacity = mem.ctypes.data, int(member_capacity)
        a.hid = hid.ctypes.data if hid is not None else None
        a.hid_len = int(hid_len)
        r = CubeHaloResult()
        self._check(lib().orc_halofind(self.h, C.byref(s), C.byref(a), C.byref(r)))
        return halos[:r.nhalo].copy(), mem[:r.nmember].copy(), hid, int(r.npeak)

    def fetch(self, which: int) -> np.ndarray:
        nf, nc = self.nf, self.nc
        p = self.p
        nt = nc // p.nnt
        nfe = nt * p.ncell + 2 * p.ncb * p.ncell
        sizes = {0: (nf ** 3, np.float32), 1: (nc ** 3, np.float32), 2: (3 * nf ** 3, np.float32),
                 3: (3 * nc ** 3, np.float32), 4: (3 * nfe * nfe * (nfe // 2 + 1), np.float64),
                 5: (3 * nc * nc * (nc // 2 + 1), np.float64)}
        n, dt = sizes[which]
        out = np.zeros(n, dt)
        got = lib().orc_fetch(self.h, which, _ptr(out), n)
        if got < 0:
            raise RuntimeError("orc_fetch failed")
        return out[:got]

    # ---- fluid neutrinos (hydrodf.f90) ----------------------------------------
    def nu_info(self) -> dict:
        out = np.zeros(4 + 15, np.float32)
        lib().orc_nu_info(self.h, _ptr(out))
        fl = out[4:].reshape(3, 5)
        return {"beta": float(out[0]), "dwgts": out[1:4].copy(), "nc": fl[:, 0].astype(int), "ncb": fl[:, 1].astype(int),
                "dx": fl[:, 2].copy(), "cs2": fl[:, 3].copy(), "dv": fl[:, 4].copy()}

    def nu_load(self, n: int, fld: np.ndarray):
        """fld: float32 [nc,nc,nc,5] (z,y,x,component) = the reference's fld(1:5,1:nc,1:nc,1:nc)."""
        a = np.ascontiguousarray(fld, dtype=np.float32)
        self._check(lib().orc_nu_load(self.h, n, _ptr(a)))

    def nu_store(self, n: int) -> np.ndarray:
        nc = int(self.nu_info()["nc"][n])
        a = np.zeros((nc, nc, nc, 5), np.float32)
        self._check(lib().orc_nu_store(self.h, n, _ptr(a)))
        return a

    def nu_evolve(self, dt: float, dtg: float, direction: int, a: float) -> float:
        g = C.c_float(dtg)
        self._check(lib().orc_nu_evolve(self.h, dt, C.byref(g), direction, a))
        return g.value
