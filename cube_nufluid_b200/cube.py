"""Host-side mirror of CUBE's step routines over the C-ABI (include/cube_gpu.h).

The reference drives one time step from its main program (CUBE_v2.0/work/main/main.f90:47-64):

    timestep; [neu%evolve]; update_x; buffer_grid; buffer_x; [ext_pp_force];
    particle_mesh; buffer_v; [neu%evolve]

`Cube` keeps those routine names and their meaning.  The buffer routines have
no device work on one GPU (every particle is stored once and neighbour cells
are read by periodic index), so `buffer_grid`, `buffer_x` and `buffer_v` are
accepted no-ops.  The scalar module variables (a, dt, sigma_vi, ...) live in a
`CubeScalars` block that each call reads and updates, as the reference's module
globals are read and updated by its no-argument subroutines.  Errors raise
`CubeError` with the library's status code, where the reference would print and
stop.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from .abi import ABI_VERSION, HALO_DTYPE, CubeHaloArgs, CubeHaloResult, CubeIcParams, CubeParams, CubeScalars
from . import tables

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "libcube_b200.so")

STATUS = {0: "ok", 1: "bad parameter", 2: "capacity exceeded", 3: "CUDA error", 4: "particle moved beyond the buffer",
          5: "device wait timed out", 6: "state error", 7: "cell too crowded for the re-bin sorter"}


class CubeError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"cube status {code} ({STATUS.get(code, '?')}): {msg}")
        self.code = code


_lib = None


def load_library():
    """Loads libcube_b200.so; raises if it is missing (there is no CPU fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is not built; run python -m cube_nufluid_b200.build")
    L = C.CDLL(LIB_PATH)
    P, S, vp = C.POINTER(CubeParams), C.POINTER(CubeScalars), C.c_void_p
    L.cube_abi_version.restype = C.c_int32
    L.cube_create.argtypes = [P, C.c_int64, vp, vp, C.POINTER(vp)]
    L.cube_create.restype = C.c_int32
    L.cube_load_state.argtypes = [vp, C.c_int64, vp, vp, vp, vp, vp]
    L.cube_load_state.restype = C.c_int32
    L.cube_run_steps.argtypes = [C.POINTER(vp), S, C.c_int32, C.c_int32, C.c_int32, C.POINTER(C.c_int32)]
    L.cube_run_steps.restype = C.c_int32
    L.cube_store_state.argtypes = [vp, C.POINTER(C.c_int64), vp, vp, vp, vp, vp]
    L.cube_store_state.restype = C.c_int32
    for name in ("cube_update_x", "cube_ext_pp_force", "cube_particle_mesh"):
        getattr(L, name).argtypes = [vp, S]
        getattr(L, name).restype = C.c_int32
    L.cube_timestep.argtypes = [P, S, C.c_float, C.POINTER(C.c_int32)]
    L.cube_timestep.restype = C.c_int32
    L.cube_expansion.argtypes = [P, C.c_float, C.c_float, C.POINTER(C.c_float), C.POINTER(C.c_float)]
    L.cube_expansion.restype = None
    L.cube_nu_evolve.argtypes = [vp, C.c_float, C.POINTER(C.c_float), C.c_int32, C.c_float]
    L.cube_nu_evolve.restype = C.c_int32
    for name in ("cube_nu_load", "cube_nu_store"):
        getattr(L, name).argtypes = [vp, C.c_int32, vp]
        getattr(L, name).restype = C.c_int32
    L.cube_nu_info.argtypes = [vp, vp]
    L.cube_nu_info.restype = C.c_int32
    L.cube_debug_encode_check.argtypes = [vp, C.c_int64, C.c_uint64, C.c_float, C.POINTER(C.c_int64)]
    L.cube_debug_encode_check.restype = C.c_int32
    L.cube_debug_division_check.argtypes = [vp, C.c_int64, C.c_uint64, C.POINTER(C.c_int64)]
    L.cube_debug_division_check.restype = C.c_int32
    L.cube_make_ic.argtypes = [vp, C.POINTER(CubeIcParams), S]
    L.cube_make_ic.restype = C.c_int32
    L.cube_halofind.argtypes = [vp, S, C.POINTER(CubeHaloArgs), C.POINTER(CubeHaloResult)]
    L.cube_halofind.restype = C.c_int32
    L.cube_power_spectrum.argtypes = [vp, C.c_int32, vp, C.c_int32, C.POINTER(C.c_int32)]
    L.cube_power_spectrum.restype = C.c_int32
    L.cube_phase_times.argtypes = [vp, C.POINTER(C.c_float)]
    L.cube_phase_times.restype = C.c_int32
    L.cube_launch_count.argtypes = [vp]
    L.cube_launch_count.restype = C.c_int64
    L.cube_set_params.argtypes = [vp, P]
    L.cube_set_params.restype = C.c_int32
    L.cube_set_stream.argtypes = [vp, vp]
    L.cube_set_stream.restype = C.c_int32
    L.cube_last_error.argtypes = [vp]
    L.cube_last_error.restype = C.c_char_p
    L.cube_destroy.argtypes = [vp]
    L.cube_destroy.restype = None
    L.cube_debug_fetch.argtypes = [vp, C.c_int32, vp, C.c_int64]
    L.cube_debug_fetch.restype = C.c_int64
    L.cube_debug_deposit.argtypes = [vp, S]
    L.cube_debug_deposit.restype = C.c_int32
    L.cube_debug_kick_with_force.argtypes = [vp, S, vp, vp]
    L.cube_debug_kick_with_force.restype = C.c_int32
    if L.cube_abi_version() != ABI_VERSION:
        raise ImportError("libcube_b200.so ABI version mismatch; rebuild")
    _lib = L
    return L


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def expansion(params: CubeParams, a0: float, dt0: float):
    """timestep.f90:136-180 through the library (FP64 inside, real(4) in and out)."""
    L = load_library()
    d1, d2 = C.c_float(), C.c_float()
    L.cube_expansion(C.byref(params), a0, dt0, C.byref(d1), C.byref(d2))
    return d1.value, d2.value


class Cube:
    """One image of CUBE's particle-mesh step on the current CUDA device."""

    def __init__(self, params: CubeParams, np_capacity: int, fk_table: np.ndarray | None = None,
                 ck_table: np.ndarray | None = None):
        self.L = load_library()
        self.p = params
        self.fk = np.ascontiguousarray(fk_table if fk_table is not None else tables.read_fine_table(
            nf_cutoff=params.nf_cutoff), dtype=np.float32)
        self.ck = np.ascontiguousarray(ck_table if ck_table is not None else tables.read_coarse_table(),
                                       dtype=np.float32)
        h = C.c_void_p()
        rc = self.L.cube_create(C.byref(params), int(np_capacity), _ptr(self.fk), _ptr(self.ck), C.byref(h))
        if rc:
            raise CubeError(rc, self.L.cube_last_error(None).decode())
        self.h = h
        self.np_capacity = int(np_capacity)
        self.nc = params.nc
        self.nf = params.nc * params.ncell

    def set_params(self, params: CubeParams):
        """cube_set_params: another box size and cosmology for this context (mesh
        sizes and options unchanged), e.g. before make_ic for the next box."""
        self._check(self.L.cube_set_params(self.h, C.byref(params)))
        self.p = params

    def close(self):
        if getattr(self, "h", None):
            self.L.cube_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def _check(self, rc):
        if rc:
            raise CubeError(rc, self.L.cube_last_error(self.h).decode())

    # ---- state -------------------------------------------------------------
    def load_state(self, xp, vp, pid, rhoc, vfield):
        xp = np.ascontiguousarray(xp)
        vp = np.ascontiguousarray(vp)
        pid = None if pid is None else np.ascontiguousarray(pid, dtype=np.int32)
        rhoc = np.ascontiguousarray(rhoc, dtype=np.int32)
        vfield = np.ascontiguousarray(vfield, dtype=np.float32)
        self._check(self.L.cube_load_state(self.h, xp.shape[0], _ptr(xp), _ptr(vp), _ptr(pid), _ptr(rhoc),
                                           _ptr(vfield)))

    def store_state(self):
        n = C.c_int64(0)
        self._check(self.L.cube_store_state(self.h, C.byref(n), None, None, None, None, None))
        npart = n.value
        xdt = np.int8 if self.p.izipx == 1 else np.int16
        vdt = np.int8 if self.p.izipv == 1 else np.int16
        xp = np.zeros((npart, 3), xdt)
        vp = np.zeros((npart, 3), vdt)
        pid = np.zeros(npart, np.int32)
        rhoc = np.zeros(self.nc ** 3, np.int32)
        vf = np.zeros((self.nc ** 3, 3), np.float32)
        self._check(self.L.cube_store_state(self.h, C.byref(n), _ptr(xp), _ptr(vp), _ptr(pid), _ptr(rhoc), _ptr(vf)))
        return xp, vp, pid, rhoc, vf

    # ---- the step routines (main.f90:47-64) --------------------------------
    def timestep(self, s: CubeScalars, a_next: float = 0.0) -> bool:
        hit = C.c_int32(0)
        self._check(self.L.cube_timestep(C.byref(self.p), C.byref(s), a_next, C.byref(hit)))
        return bool(hit.value)

    def update_x(self, s: CubeScalars):
        self._check(self.L.cube_update_x(self.h, C.byref(s)))

    def buffer_grid(self):
        """No device work: periodic neighbour cells are addressed directly."""

    def buffer_x(self):
        """No device work: buffer particles are not duplicated on the GPU."""

    def buffer_v(self):
        """No device work: buffer particles are not duplicated on the GPU."""

    def ext_pp_force(self, s: CubeScalars):
        self._check(self.L.cube_ext_pp_force(self.h, C.byref(s)))

    def particle_mesh(self, s: CubeScalars):
        self._check(self.L.cube_particle_mesh(self.h, C.byref(s)))

    def step(self, s: CubeScalars, a_next: float = 0.0) -> bool:
        """One pass of main.f90:49-64: timestep, neutrino half step, drift, PP,
        particle mesh, neutrino half step."""
        hit = self.timestep(s, a_next)
        if self.p.neutrino:
            s.dt_neu = self.nu_evolve(s.dt / 2.0, s.dt_neu, 1, s.a_mid)
        self.update_x(s)
        if self.p.ext_pp_force:
            self.ext_pp_force(s)
        self.particle_mesh(s)
        if self.p.neutrino:
            s.dt_neu = self.nu_evolve(s.dt / 2.0, s.dt_neu, -1, s.a_mid)
        return hit

    def debug_encode_check(self, n: int, seed: int, sigma: float) -> int:
        """Disagreements between the fast and the exact velocity encode over n velocities."""
        bad = C.c_int64(0)
        self._check(self.L.cube_debug_encode_check(self.h, int(n), int(seed), float(sigma), C.byref(bad)))
        return bad.value

    def debug_division_check(self, n: int, seed: int) -> int:
        """Quotients where the shared-reciprocal division differs from IEEE division."""
        bad = C.c_int64(0)
        self._check(self.L.cube_debug_division_check(self.h, int(n), int(seed), C.byref(bad)))
        return int(bad.value)

    def make_ic(self, ic: dict, seed: int, *, f_cdm: float = 1.0) -> CubeScalars:
        """Zel'dovich state made on the device (cube_make_ic) from the scalars of
        ic.device_ic_params; returns the initial scalar block."""
        q = CubeIcParams()
        q.seed = int(seed)
        q.np_nc = int(ic["np_nc"])
        for k in ("a", "norm_d2", "n_s", "h", "eh_s", "eh_alpha", "eh_omh", "eh_theta2", "vf", "amplitude"):
            setattr(q, k, float(ic[k]))
        q.f_cdm = float(f_cdm)
        s = CubeScalars()
        self._check(self.L.cube_make_ic(self.h, C.byref(q), C.byref(s)))
        return s

    def halofind(self, s: CubeScalars, *, den_odc: float = 200.0, capacity: int = 1 << 16,
                 members: bool = True, hid_len: int = 0):
        """Run-time halo finder (cube_halofind, halofind.f90:18-598) on the resident
        state.  Returns (halos as a HALO_DTYPE array, member PIDs by halo in radius
        order, hid array or None, number of density peaks)."""
        while True:
            halos = np.zeros(capacity, HALO_DTYPE)
            mcap = int(max(self.np_capacity, 1)) if members else 0
            mem = np.zeros(max(mcap, 1), np.int32)
            hid = np.zeros(hid_len, np.int32) if hid_len > 0 else None
            a = CubeHaloArgs()
            a.den_odc, a.capacity, a.halos = float(den_odc), int(capacity), halos.ctypes.data
            a.member_pid = mem.ctypes.data if members else None
            a.member_capacity = mcap
            a.hid = hid.ctypes.data if hid is not None else None
            a.hid_len = int(hid_len)
            r = CubeHaloResult()
            rc = self.L.cube_halofind(self.h, C.byref(s), C.byref(a), C.byref(r))
            if rc == 2 and r.nhalo > capacity:
                capacity = int(r.nhalo)
                continue
            self._check(rc)
            return halos[:r.nhalo].copy(), mem[:r.nmember].copy(), hid, int(r.npeak)

    def power_spectrum(self, log_bins: bool = False) -> np.ndarray:
        """xip(10, nbin) of cicpower / powerspectrum as float32 [nbin, 10]."""
        nb = C.c_int32(0)
        cap = 4096
        out = np.zeros((cap, 10), np.float32)
        self._check(self.L.cube_power_spectrum(self.h, int(log_bins), _ptr(out), cap, C.byref(nb)))
        return out[:nb.value].copy()

    # ---- fluid neutrinos (hydrodf.f90) ---------------------------------------
    def nu_evolve(self, dt: float, dtg: float, direction: int, a: float) -> float:
        """neu%evolve(dt, dtg, dir, a); returns the lowered dtg."""
        g = C.c_float(dtg)
        self._check(self.L.cube_nu_evolve(self.h, float(np.float32(dt)), C.byref(g), int(direction), float(a)))
        return g.value

    def nu_info(self) -> dict:
        out = np.zeros(19, np.float32)
        self._check(self.L.cube_nu_info(self.h, _ptr(out)))
        fl = out[4:].reshape(3, 5)
        return {"beta": float(out[0]), "dwgts": out[1:4].copy(), "nc": fl[:, 0].astype(int),
                "ncb": fl[:, 1].astype(int), "dx": fl[:, 2].copy(), "cs2": fl[:, 3].copy(), "dv": fl[:, 4].copy()}

    def nu_load(self, fluid: int, fld: np.ndarray):
        """fld: float32 [n,n,n,5] = the reference's fld(1:5,1:n,1:n,1:n)."""
        a = np.ascontiguousarray(fld, dtype=np.float32)
        n = int(self.nu_info()["nc"][fluid])
        if a.shape != (n, n, n, 5):
            raise ValueError(f"fluid {fluid} expects shape {(n, n, n, 5)}")
        self._check(self.L.cube_nu_load(self.h, int(fluid), _ptr(a)))

    def nu_store(self, fluid: int) -> np.ndarray:
        n = int(self.nu_info()["nc"][fluid])
        a = np.zeros((n, n, n, 5), np.float32)
        self._check(self.L.cube_nu_store(self.h, int(fluid), _ptr(a)))
        return a

    # ---- inspection --------------------------------------------------------
    def phase_times(self) -> list[float]:
        buf = (C.c_float * 8)()
        self._check(self.L.cube_phase_times(self.h, buf))
        return list(buf)

    def launch_count(self) -> int:
        return int(self.L.cube_launch_count(self.h))

    def fetch(self, which: int) -> np.ndarray:
        nf, nc = self.nf, self.nc
        sizes = {0: nf ** 3, 1: nc ** 3, 2: 3 * nf ** 3, 3: 3 * nc ** 3,
                 4: 3 * (nf // 2 + 1) ** 3, 5: 3 * (nc // 2 + 1) ** 3}
        fp64 = which <= 3 and bool(self.p.poisson_fp64)  # the FP64 Poisson mode's meshes
        out = np.zeros(sizes[which], np.float64 if fp64 else np.float32)
        got = self.L.cube_debug_fetch(self.h, which, _ptr(out), out.size)
        if got < 0:
            raise CubeError(3, "debug fetch failed")
        return out

    def debug_deposit(self, s: CubeScalars):
        """Deposit only; fetch(0) / fetch(1) then return the fine / coarse density."""
        self._check(self.L.cube_debug_deposit(self.h, C.byref(s)))

    def kick_with_force(self, s: CubeScalars, fine: np.ndarray, coarse: np.ndarray):
        f = np.ascontiguousarray(fine, dtype=np.float32)
        c = np.ascontiguousarray(coarse, dtype=np.float32)
        self._check(self.L.cube_debug_kick_with_force(self.h, C.byref(s), _ptr(f), _ptr(c)))


def scalars_from_ic(st) -> CubeScalars:
    """Initial scalar block for a state made by cube_nufluid_b200.ic (particle_initialization.f90:37-39)."""
    s = CubeScalars()
    s.a = st.a
    s.sigma_vi = st.sigma_vi
    s.sigma_vi_new = st.sigma_vi
    s.mass_p_cdm = st.mass_p_cdm
    s.vz_max = float(st.vmax[2])
    s.dt = 0.0
    s.dt_old = 0.0
    s.dt_fine = s.dt_coarse = s.dt_pp = s.dt_vmax = s.dt_vmax_nu = 1000.0
    s.dt_vmax = float(np.float32(0.9 * 20.0 / max(float(np.max(st.vmax)), 1e-30)))
    s.dt_neu = 1000.0
    s.npglobal = st.np
    s.nplocal = st.np
    s.vsim2phys = st.vsim2phys
    return s
