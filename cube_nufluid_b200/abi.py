"""ctypes mirror of include/cube_gpu.h (structs and entry points of the C-ABI)."""
from __future__ import annotations

import ctypes as C

import numpy as np

ABI_VERSION = 1


class CubeParams(C.Structure):
    _fields_ = [
        ("nc", C.c_int32), ("nnt", C.c_int32), ("ncell", C.c_int32), ("ncb", C.c_int32),
        ("np_nc", C.c_int32), ("izipx", C.c_int32), ("izipv", C.c_int32),
        ("nf_cutoff", C.c_int32), ("pp_range", C.c_int32), ("ext_pp_force", C.c_int32),
        ("use_pid", C.c_int32), ("neutrino", C.c_int32),
        ("rsoft", C.c_float), ("tile_buffer", C.c_float), ("image_buffer", C.c_float),
        ("vbuf", C.c_float), ("vrel_boost", C.c_double),
        ("box", C.c_float), ("h0", C.c_float), ("omega_m", C.c_float), ("omega_l", C.c_float),
        ("wde", C.c_float), ("ra_max", C.c_float), ("dt_max", C.c_float),
        ("z_i_nu", C.c_float), ("f_neu", C.c_float), ("m_nu_ev", C.c_float), ("deg_nu", C.c_float),
        ("nu_nc", C.c_int32 * 3), ("stockham_only", C.c_int32), ("poisson_fp64", C.c_int32),
        ("reserved", C.c_int32 * 6),
    ]


class CubeScalars(C.Structure):
    _fields_ = [
        ("a", C.c_float), ("a_mid", C.c_float), ("da", C.c_float),
        ("dt", C.c_float), ("dt_old", C.c_float), ("dt_mid", C.c_float),
        ("t", C.c_float), ("tau", C.c_float),
        ("sigma_vi", C.c_float), ("sigma_vi_new", C.c_float),
        ("mass_p_cdm", C.c_float), ("vz_max", C.c_float),
        ("dt_fine", C.c_float), ("dt_coarse", C.c_float), ("dt_pp", C.c_float),
        ("dt_vmax", C.c_float), ("dt_vmax_nu", C.c_float), ("dt_e", C.c_float), ("dt_neu", C.c_float),
        ("vmax", C.c_float * 3),
        ("f2_max_fine", C.c_float), ("f2_max_coarse", C.c_float), ("f2_max_pp", C.c_float),
        ("vsim2phys", C.c_float),
        ("nlayer", C.c_int32), ("timestep", C.c_int32),
        ("std_vsim", C.c_double), ("std_vsim_c", C.c_double), ("std_vsim_res", C.c_double),
        ("testrhof", C.c_double), ("testrhoc", C.c_double),
        ("nplocal", C.c_int64), ("npglobal", C.c_int64),
        ("npairs", C.c_int64), ("itest1", C.c_int64),
        ("reserved", C.c_int32 * 16),
    ]

    def copy(self) -> "CubeScalars":
        out = CubeScalars()
        C.memmove(C.byref(out), C.byref(self), C.sizeof(CubeScalars))
        return out

    def as_dict(self) -> dict:
        d = {}
        for name, _ in self._fields_:
            if name == "reserved":
                continue
            v = getattr(self, name)
            d[name] = list(v) if name == "vmax" else v
        return d


class CubeIcParams(C.Structure):
    """cube_ic_params of include/cube_gpu.h."""
    _fields_ = [
        ("seed", C.c_int64), ("np_nc", C.c_int32), ("pad0", C.c_int32),
        ("a", C.c_double), ("norm_d2", C.c_double), ("n_s", C.c_double), ("h", C.c_double),
        ("eh_s", C.c_double), ("eh_alpha", C.c_double), ("eh_omh", C.c_double), ("eh_theta2", C.c_double),
        ("vf", C.c_double), ("amplitude", C.c_double), ("f_cdm", C.c_double),
    ]


class CubeHalo(C.Structure):
    """cube_halo of include/cube_gpu.h: type_halo_info (halofind.f90:10-15), 42 floats."""
    _fields_ = [
        ("hpos", C.c_float * 3), ("mass_odc", C.c_float), ("radius_odc", C.c_float), ("v_disp", C.c_float),
        ("x_mean", C.c_float * 3), ("v_mean", C.c_float * 3), ("ang_mom", C.c_float * 3), ("var_x", C.c_float * 3),
        ("inertia", C.c_float * 9), ("q_mean", C.c_float * 3), ("inertia_q", C.c_float * 9), ("s_mean", C.c_float * 3),
    ]


class CubeHaloArgs(C.Structure):
    """cube_halo_args of include/cube_gpu.h."""
    _fields_ = [
        ("den_odc", C.c_float), ("capacity", C.c_int32), ("halos", C.c_void_p),
        ("member_pid", C.c_void_p), ("member_capacity", C.c_int64),
        ("hid", C.c_void_p), ("hid_len", C.c_int64),
    ]


class CubeHaloResult(C.Structure):
    """cube_halo_result of include/cube_gpu.h."""
    _fields_ = [("nhalo", C.c_int32), ("npeak", C.c_int32), ("nmember", C.c_int64)]


# numpy view of one cube_halo record
HALO_DTYPE = np.dtype([
    ("hpos", "<f4", 3), ("mass_odc", "<f4"), ("radius_odc", "<f4"), ("v_disp", "<f4"),
    ("x_mean", "<f4", 3), ("v_mean", "<f4", 3), ("ang_mom", "<f4", 3), ("var_x", "<f4", 3),
    ("inertia", "<f4", 9), ("q_mean", "<f4", 3), ("inertia_q", "<f4", 9), ("s_mean", "<f4", 3),
])


def make_params(nc: int, nnt: int, *, ncell: int = 4, ncb: int = 6, np_nc: int = 2, izipx: int = 2,
                izipv: int = 2, nf_cutoff: int = 16, pp_range: int = 1, ext_pp_force: bool = False,
                use_pid: bool = True, neutrino: bool = False, box: float = 200.0, h0: float = 0.7,
                omega_m: float = 0.3, omega_l: float = 0.7, z_i_nu: float = 10.0, f_neu: float = 0.0,
                m_nu_ev: float = 0.0, deg_nu: float = 3.0, nu_nc=(0, 0, 0)) -> CubeParams:
    p = CubeParams()
    p.nc, p.nnt, p.ncell, p.ncb, p.np_nc = nc, nnt, ncell, ncb, np_nc
    p.izipx, p.izipv, p.nf_cutoff, p.pp_range = izipx, izipv, nf_cutoff, pp_range
    p.ext_pp_force, p.use_pid, p.neutrino = int(ext_pp_force), int(use_pid), int(neutrino)
    p.rsoft, p.tile_buffer, p.image_buffer, p.vbuf, p.vrel_boost = 0.3, 1.5, 1.2, 0.9, 2.5
    p.box, p.h0, p.omega_m, p.omega_l = box, h0, omega_m, omega_l
    p.wde, p.ra_max, p.dt_max = -1.0, 0.2, 1.0
    p.z_i_nu, p.f_neu, p.m_nu_ev, p.deg_nu = z_i_nu, f_neu, m_nu_ev, deg_nu
    for i in range(3):
        p.nu_nc[i] = int(nu_nc[i])
    return p
