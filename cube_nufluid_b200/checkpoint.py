"""CUBE checkpoint files: the on-disk format of a CUBE run, so that a state can move
between this library and the reference (resume either way).

Per image and checkpoint redshift z the reference writes stream files
``<opath>image<i>/<z>_<name>_<i>.bin`` (basic_functions.fh:39-82, z formatted
f7.3 and trimmed) with name

    info   the sim_header record (parameters.f90:129-153), 224 bytes
    xp     int8|int16 xp(3, nplocal)            (checkpoint.f90:38)
    vp     int8|int16 vp(3, nplocal)            (:40)
    np     int32 rhoc(nt, nt, nt, nnt, nnt, nnt) (:42)
    vc     float32 vfield(3, nt, nt, nt, nnt^3)  (:44)
    id     int32 pid(nplocal)                    (:47, with -DPID)

and the fluid neutrinos ``<z>_neu<n>_<i>.bin`` (main.f90:79 -> hydrodf.f90:134-156):
m (real), gamma (real), isothermal (logical, 4 bytes), the three weights, then
each fluid's fld(5, 1-ncb:nc+ncb, ...)^3 with its halo cells.  The arrays are
exactly the layouts cube_load_state / cube_store_state and cube_nu_load /
cube_nu_store take, so reading and writing is a byte copy (plus the halo).
Resuming follows particle_initialization.f90:34-40: a = 1/(1+z), sigma_vi from
the header; the header's dt limits, mass and vz_max seed the next step.
"""
from __future__ import annotations

import os
from dataclasses import dataclass

import numpy as np

from .abi import HALO_DTYPE, CubeScalars

# sim_header (parameters.f90:129-153): 17 integer(8) then 22 real(4), no padding
SIM_HEADER = np.dtype([
    ("nplocal", "<i8"), ("npglobal", "<i8"), ("nplocal_nu", "<i8"), ("npglobal_nu", "<i8"),
    ("izipx", "<i8"), ("izipv", "<i8"), ("izipx_nu", "<i8"), ("izipv_nu", "<i8"),
    ("image", "<i8"), ("nn", "<i8"), ("nnt", "<i8"), ("nt", "<i8"), ("ncell", "<i8"), ("ncb", "<i8"),
    ("timestep", "<i8"), ("cur_checkpoint", "<i8"), ("cur_halofind", "<i8"),
    ("a", "<f4"), ("t", "<f4"), ("tau", "<f4"),
    ("dt_pp", "<f4"), ("dt_fine", "<f4"), ("dt_coarse", "<f4"), ("dt_vmax", "<f4"), ("dt_vmax_nu", "<f4"),
    ("mass_p_cdm", "<f4"), ("mass_p_nu", "<f4"), ("box", "<f4"),
    ("h0", "<f4"), ("omega_m", "<f4"), ("omega_l", "<f4"), ("s8", "<f4"), ("vsim2phys", "<f4"),
    ("sigma_vres", "<f4"), ("sigma_vi", "<f4"), ("sigma_vi_nu", "<f4"),
    ("z_i", "<f4"), ("z_i_nu", "<f4"), ("vz_max", "<f4"),
])
assert SIM_HEADER.itemsize == 224


def z_string(z: float) -> str:
    """Fortran write(str,'(f7.3)') z, adjusted left and trimmed."""
    return f"{np.float32(z):7.3f}".strip()


def file_name(opath: str, z: float, name: str, image: int = 1, with_z: bool = True) -> str:
    pre = f"{z_string(z)}_" if with_z else ""
    return os.path.join(opath, f"image{image}", f"{pre}{name}_{image}.bin")


@dataclass
class Checkpoint:
    header: np.ndarray  # one SIM_HEADER record
    xp: np.ndarray      # [np, 3]
    vp: np.ndarray      # [np, 3]
    rhoc: np.ndarray    # int32 [nnt^3 * nt^3]
    vfield: np.ndarray  # float32 [nnt^3 * nt^3, 3]
    pid: np.ndarray | None


def make_header(params, s: CubeScalars, *, image: int = 1, cur_checkpoint: int = 1, cur_halofind: int = 1,
                s8: float = 0.8, z_i: float = 49.0, sigma_vres: float = 0.0) -> np.ndarray:
    """checkpoint.f90:24-33: the header fields from the run's parameters and scalars."""
    h = np.zeros((), SIM_HEADER)
    nt = params.nc // params.nnt
    h["nplocal"] = h["npglobal"] = int(s.nplocal)
    h["izipx"], h["izipv"] = params.izipx, params.izipv
    h["izipx_nu"], h["izipv_nu"] = 2, 2  # parameters.f90:10-11
    h["image"], h["nn"], h["nnt"], h["nt"] = image, 1, params.nnt, nt
    h["ncell"], h["ncb"] = params.ncell, params.ncb
    h["timestep"], h["cur_checkpoint"], h["cur_halofind"] = int(s.timestep), cur_checkpoint, cur_halofind
    for k in ("a", "t", "tau", "dt_pp", "dt_fine", "dt_coarse", "dt_vmax", "dt_vmax_nu", "mass_p_cdm",
              "sigma_vi", "vz_max"):
        h[k] = getattr(s, k)
    f32 = np.float32
    h["box"], h["h0"], h["omega_m"], h["omega_l"] = params.box, params.h0, params.omega_m, params.omega_l
    h["s8"], h["z_i"], h["z_i_nu"], h["sigma_vres"] = s8, z_i, params.z_i_nu, sigma_vres
    # sim%vsim2phys=(1.5/a)*box*100.*sqrt(omega_m)/nf_global (checkpoint.f90:30)
    nf = params.nc * params.ncell
    h["vsim2phys"] = f32(f32(f32(f32(1.5) / f32(s.a)) * f32(params.box)) * f32(100.0)) * np.sqrt(f32(params.omega_m)) \
        / f32(nf)
    return h


def write(opath: str, z: float, ck: Checkpoint, image: int = 1) -> list[str]:
    os.makedirs(os.path.join(opath, f"image{image}"), exist_ok=True)
    files = []
    for name, arr in (("info", ck.header), ("xp", ck.xp), ("vp", ck.vp), ("np", ck.rhoc), ("vc", ck.vfield),
                      ("id", ck.pid)):
        if arr is None:
            continue
        fn = file_name(opath, z, name, image)
        with open(fn, "wb") as f:
            f.write(np.ascontiguousarray(arr).tobytes())
        files.append(fn)
    return files


def _checked_file(fn: str, nbytes: int, what: str) -> str:
    size = os.path.getsize(fn)
    if size != nbytes:
        raise ValueError(f"corrupted checkpoint: {what} file {fn} holds {size} bytes, the header implies {nbytes}")
    return fn


def read(opath: str, z: float, image: int = 1, *, with_pid: bool = True) -> Checkpoint:
    """particle_initialization.f90:34-56.  The header is checked against itself and
    against the sizes of the array files before anything is read: a truncated or
    corrupted checkpoint raises ValueError (the reference would read garbage)."""
    info = file_name(opath, z, "info", image)
    _checked_file(info, SIM_HEADER.itemsize, "info")
    h = np.fromfile(info, dtype=SIM_HEADER, count=1)[0]
    n = int(h["nplocal"])
    izx, izv, nnt, nt = int(h["izipx"]), int(h["izipv"]), int(h["nnt"]), int(h["nt"])
    if izx not in (1, 2) or izv not in (1, 2) or nnt <= 0 or nt <= 0 or n < 0:
        raise ValueError(f"corrupted checkpoint header: izipx={izx} izipv={izv} nnt={nnt} nt={nt} nplocal={n}")
    xdt = np.int8 if izx == 1 else np.int16
    vdt = np.int8 if izv == 1 else np.int16
    ncells = nnt ** 3 * nt ** 3
    xp = np.fromfile(_checked_file(file_name(opath, z, "xp", image), 3 * n * izx, "xp"), dtype=xdt,
                     count=3 * n).reshape(n, 3)
    vp = np.fromfile(_checked_file(file_name(opath, z, "vp", image), 3 * n * izv, "vp"), dtype=vdt,
                     count=3 * n).reshape(n, 3)
    rhoc = np.fromfile(_checked_file(file_name(opath, z, "np", image), 4 * ncells, "np"), dtype=np.int32,
                       count=ncells)
    if int(rhoc.astype(np.int64).sum()) != n or (rhoc < 0).any():
        raise ValueError("corrupted checkpoint: the cell counts do not add up to nplocal")
    vf = np.fromfile(_checked_file(file_name(opath, z, "vc", image), 12 * ncells, "vc"), dtype=np.float32,
                     count=3 * ncells).reshape(ncells, 3)
    pid = None
    fid = file_name(opath, z, "id", image)
    if with_pid and os.path.exists(fid):
        pid = np.fromfile(_checked_file(fid, 4 * n, "id"), dtype=np.int32, count=n)
    return Checkpoint(h, xp, vp, rhoc, vf, pid)


def scalars_from_header(h: np.ndarray, z: float) -> CubeScalars:
    """The scalar block a resumed run starts from (particle_initialization.f90:37-39:
    a = 1/(1+z), sigma_vi from the header; dt limits, mass and vz_max from sim)."""
    s = CubeScalars()
    f32 = np.float32
    s.a = float(f32(1.0) / (f32(1.0) + f32(z)))
    s.sigma_vi = s.sigma_vi_new = float(h["sigma_vi"])
    s.mass_p_cdm = float(h["mass_p_cdm"])
    s.t, s.tau = float(h["t"]), float(h["tau"])
    s.timestep = int(h["timestep"])
    for k in ("dt_pp", "dt_fine", "dt_coarse", "dt_vmax", "dt_vmax_nu", "vz_max", "vsim2phys"):
        setattr(s, k, float(h[k]))
    s.dt = s.dt_old = 0.0  # initialize.f90: a resumed run starts its first step from dt = 0
    s.dt_neu = 1000.0
    s.nplocal = s.npglobal = int(h["nplocal"])
    return s


# ---- fluid neutrinos (hydrodf.f90:134-185) ------------------------------------------
NU_HEAD = np.dtype([("m", "<f4"), ("g", "<f4"), ("iso", "<i4"), ("dwgts", "<f4", (3,))])


def add_halo(fld: np.ndarray, ncb: int) -> np.ndarray:
    """fld(1:5,1:n,1:n,1:n) [n,n,n,5] -> fld(5,1-ncb:n+ncb,...) with the periodic halo
    of hg_buffer (hydrogr.f90:240-284, one image)."""
    n = fld.shape[0]
    idx = np.arange(-ncb, n + ncb) % n
    return np.ascontiguousarray(fld[np.ix_(idx, idx, idx)])


def write_fluid(path: str, m_ev: float, gamma: float, dwgts, fluids, ncbs, iso: bool = True) -> None:
    """dfld_checkpoint: m, g, isothermal, dwgts, then each fluid with its halo."""
    h = np.zeros((), NU_HEAD)
    h["m"], h["g"], h["iso"], h["dwgts"] = m_ev, gamma, 1 if iso else 0, np.asarray(dwgts, np.float32)
    os.makedirs(os.path.dirname(path) or ".", exist_ok=True)
    with open(path, "wb") as f:
        f.write(h.tobytes())
        for fl, ncb in zip(fluids, ncbs):
            f.write(add_halo(np.asarray(fl, np.float32), int(ncb)).tobytes())


def read_fluid(path: str, ncs, ncbs):
    """dfld_restart: the header and each fluid's physical cells [n,n,n,5]; the fluid
    sizes come from the run's set-up (dfld_setup), as in the reference."""
    with open(path, "rb") as f:
        h = np.frombuffer(f.read(NU_HEAD.itemsize), NU_HEAD)[0]
        out = []
        for n, ncb in zip(ncs, ncbs):
            e = int(n) + 2 * int(ncb)
            a = np.frombuffer(f.read(4 * 5 * e ** 3), np.float32).reshape(e, e, e, 5)
            out.append(a[ncb:ncb + n, ncb:ncb + n, ncb:ncb + n].copy())
    return h, out


def save(cube, s: CubeScalars, opath: str, z: float, image: int = 1, **header_kw) -> list[str]:
    """checkpoint + neu%checkpoint of main.f90:72-81 for a resident Cube."""
    xp, vp, pid, rhoc, vf = cube.store_state()
    files = write(opath, z, Checkpoint(make_header(cube.p, s, image=image, **header_kw), xp, vp, rhoc, vf,
                                       pid if cube.p.use_pid else None), image)
    if cube.p.neutrino:
        info = cube.nu_info()
        fn = file_name(opath, z, "neu1", image)
        write_fluid(fn, cube.p.m_nu_ev, np.float32(5.0) / np.float32(3.0), info["dwgts"],
                    [cube.nu_store(k) for k in range(3)], info["ncb"])
        files.append(fn)
    return files


def restore(cube, opath: str, z: float, image: int = 1) -> CubeScalars:
    """particle_initialization (+ neu%restart) into a Cube; returns the scalars."""
    r = read(opath, z, image, with_pid=bool(cube.p.use_pid))
    if int(r.header["izipx"]) != cube.p.izipx or int(r.header["izipv"]) != cube.p.izipv:
        raise ValueError("zip format incompatible")  # particle_initialization.f90:41-45
    pid = r.pid if r.pid is not None else np.zeros(len(r.xp), np.int32)
    cube.load_state(r.xp, r.vp, pid, r.rhoc, r.vfield)
    if cube.p.neutrino:
        info = cube.nu_info()
        _, fl = read_fluid(file_name(opath, z, "neu1", image), info["nc"], info["ncb"])
        for k in range(3):
            cube.nu_load(k, fl[k])
    return scalars_from_header(r.header, z)


# ---- halo catalogue (halofind.f90:113-127, :417-513, :566-580) ---------------
HALO_HEADER = np.dtype([("nhalo_tot", "<i4"), ("nhalo", "<i4"), ("den_odc", "<f4")])


def write_halos(opath: str, z: float, halos: np.ndarray, members: np.ndarray | None, hid: np.ndarray | None,
                den_odc: float = 200.0, image: int = 1) -> list[str]:
    """The halofind output files of one image at redshift z:

    halo      nhalo_tot, nhalo (int32), den_odc (float32), then one type_halo_info
              record (42 float32, HALO_DTYPE) per halo;
    halo_pid  per halo: int32 i_odc, its i_odc PIDs by increasing radius, int32 0;
    hid       int16 per PID - 1 (halo number, 0 if none), nf^3 entries as the
              reference writes them (its integer(2) wraps above 32767).
    `members` is the concatenated PID list of cube_halofind (halos in order)."""
    os.makedirs(os.path.join(opath, f"image{image}"), exist_ok=True)
    files = []
    head = np.zeros(1, HALO_HEADER)
    head["nhalo_tot"] = head["nhalo"] = len(halos)
    head["den_odc"] = den_odc
    fn = file_name(opath, z, "halo", image)
    with open(fn, "wb") as f:
        f.write(head.tobytes())
        f.write(np.ascontiguousarray(halos).tobytes())
    files.append(fn)
    if members is not None:
        fn = file_name(opath, z, "halo_pid", image)
        counts = np.asarray(halos["mass_odc"], np.int64)
        if int(counts.sum()) != len(members):
            raise ValueError("member list does not match the halos' particle counts")
        with open(fn, "wb") as f:
            off = 0
            for n in counts:
                f.write(np.int32(n).tobytes())
                f.write(np.ascontiguousarray(members[off:off + n], dtype=np.int32).tobytes())
                f.write(np.int32(0).tobytes())
                off += int(n)
        files.append(fn)
    if hid is not None:
        fn = file_name(opath, z, "hid", image)
        with open(fn, "wb") as f:
            f.write(np.asarray(hid).astype(np.int16).tobytes())
        files.append(fn)
    return files


def read_halos(opath: str, z: float, image: int = 1):
    """(header, halos, list of per-halo PID arrays or None) of write_halos' files."""
    raw = np.fromfile(file_name(opath, z, "halo", image), dtype=np.uint8)
    head = raw[:HALO_HEADER.itemsize].view(HALO_HEADER)[0]
    halos = raw[HALO_HEADER.itemsize:].view(HALO_DTYPE)
    members = None
    fn = file_name(opath, z, "halo_pid", image)
    if os.path.exists(fn):
        w = np.fromfile(fn, dtype=np.int32)
        members, off = [], 0
        while off < len(w):
            n = int(w[off])
            members.append(w[off + 1:off + 1 + n].copy())
            if w[off + 1 + n] != 0:
                raise ValueError("halo_pid record does not end in 0")
            off += n + 2
    return head, halos, members
