"""Benchmark of the B200 PM step (one JSON line on stdout).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--config c2|c1|c3|c4|c5|c6|c2s|c3s] [--state-cache FILE]

Workload (default c2, the single-GPU precision configuration): 512^3 CDM
particles in a 1000 Mpc/h box, fine mesh 1024^3, coarse mesh 256^3, 8^3 tiles,
int2 positions and velocities, PP on (pp_range=1), synthetic seeded Zel'dovich
initial conditions at z_i=49 (Eisenstein-Hu no-wiggle, Philox noise).  A step
is one pass of the reference main loop body: timestep, update_x,
ext_pp_force, particle_mesh.  metric = particle-updates/s = Np * steps / time.

value : device time of K steps (CUDA events on the library's stream, state
        resident in HBM, meshes far larger than the 126 MB L2), max over ranks.
e2e   : the same steps through the C-ABI as a host that owns the arrays would
        drive it: per step cube_load_state from pinned host buffers (checkpoint
        layout), the step, cube_store_state back to pinned host buffers.
N > 1 : one independent box per rank (replicas, weak scaling), no collective
        on the data path; barrier and max-over-ranks timing through NCCL.
--impl reference: the CPU oracle (a restatement of the reference's Fortran
        step; the Fortran reference cannot be built here) on the host cores, on
        a bounded sample of the workload.
Other configurations: c3 (fluid neutrinos), c4 (ensemble of small boxes), c5
(serving a Poisson request stream), c6 (steps of a clustered z=0 state of a
256^3-particle, 50 Mpc/h box; --state-cache keeps the evolved state in a file),
c2s/c3s (profiling sizes).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

CONFIGS = {
    "c2": dict(nc=256, nnt=8, box=1000.0, izip=2, pp=True, z_i=49.0,
               workload="512^3 particles, 1000 Mpc/h, fine 1024^3, coarse 256^3, int2 x/v, PP on (pp_range=1)"),
    "c2s": dict(nc=128, nnt=4, box=500.0, izip=2, pp=True, z_i=49.0,
                workload="256^3 particles, 500 Mpc/h, fine 512^3, coarse 128^3, int2 x/v, PP on (profiling size)"),
    "c1": dict(nc=32, nnt=2, box=200.0, izip=2, pp=False, z_i=49.0,
               workload="64^3 particles, 200 Mpc/h, fine 128^3, coarse 32^3, int2 x/v, PP off"),
    # CDM + fluid neutrinos, started at the neutrino turn-on z_i_nu = 10 (the redshift
    # neutrino_ic.f90 builds the fluids at), so every timed step evolves the fluids
    "c3": dict(nc=256, nnt=8, box=500.0, izip=2, pp=True, z_i=10.0, nu=True,
               workload="512^3 CDM particles + fluid neutrinos (1 species, 3 x 0.1 eV; Gauss-Laguerre fluids "
                        "512^3, 256^3, 128^3), 500 Mpc/h, fine 1024^3, coarse 256^3, int2 x/v, PP on, from z=10"),
    # batched ensemble: 96 independent boxes of 32^3-128^3 particles, one context and
    # stream each, stepped by a pool of host threads (cube_nufluid_b200.ensemble)
    "c4": dict(nc=0, nnt=1, box=0.0, izip=2, pp=False, z_i=49.0, ensemble=96,
               workload="ensemble of 96 boxes, 32^3-128^3 particles (uniform over 32,48,64,96,128 per side), "
                        "50-400 Mpc/h log-uniform, Om~U[0.25,0.35], s8~U[0.7,0.9], per-box seeds, int2 x/v, PP off"),
    # serving: Poisson requests at 20/s of 32^3-256^3 particles, each evolved z=49 -> 0
    # in 48 steps and answered with P(k) and a 1/64 subsample (cube_nufluid_b200.serving)
    "c5": dict(nc=0, nnt=1, box=0.0, izip=2, pp=False, z_i=49.0, serving=60,
               workload="serving: Poisson arrivals at 20/s, 32^3-256^3 particles log-uniform, 50-400 Mpc/h, "
                        "Om~U[0.25,0.35], s8~U[0.7,0.9], 48 steps z=49->0, P(k) in 32 log bins + 1/64 "
                        "subsample, 160 GB HBM admission budget, int2 x/v, PP off"),
    # late times: a small box evolved from z=49 to z=0 (48 log-spaced targets, untimed;
    # cached with --state-cache), then timed steps of the clustered state (cells of up
    # to ~40,000 particles)
    "c6": dict(nc=128, nnt=4, box=50.0, izip=2, pp=False, z_i=49.0, late=True,
               workload="late-time clustered box: 256^3 particles, 50 Mpc/h, evolved z=49 -> 0 "
                        "(Om=0.3, s8=0.8), fine 512^3, coarse 128^3, int2 x/v, PP off"),
    "c3s": dict(nc=128, nnt=4, box=250.0, izip=2, pp=True, z_i=10.0, nu=True,
                workload="256^3 CDM particles + fluid neutrinos (fluids 256^3, 128^3, 64^3), 250 Mpc/h, "
                         "fine 512^3, coarse 128^3, int2 x/v, PP on, from z=10 (profiling size)"),
}

# fluid neutrinos of the C3 workload: one species of 0.1 eV, degeneracy 3, in a
# total Omega_m = 0.3 with h = 0.7 (Omega_cdm reduced by Omega_nu)
NU_M_EV, NU_DEG, NU_H = 0.1, 3.0, 0.7
NU_F = float(np.float32(NU_DEG * NU_M_EV / 93.14 / NU_H ** 2) / np.float32(0.3))
GL_V = (0.41577456, 2.29428036, 6.28994508)


def read_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock / throttle-reason samples during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.rows = []
        self.proc = None

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 9:
                self.rows.append(parts)

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def make_state(cfg, seed):
    """Seeded Zel'dovich state; cached under $TMPDIR so repeated runs on one host skip the host-side IC."""
    import pickle
    import tempfile
    from cube_nufluid_b200 import ic
    nu = bool(cfg.get("nu"))
    key = f"cube_ic_{cfg['nc']}_{cfg['nnt']}_{cfg['box']}_{cfg['z_i']}_{cfg['izip']}_{seed}_{int(nu)}.pkl"
    path = os.path.join(tempfile.gettempdir(), key)
    if os.path.exists(path):
        with open(path, "rb") as f:
            return pickle.load(f)
    st = ic.zeldovich(cfg["nc"], cfg["nnt"], box=cfg["box"], z_i=cfg["z_i"], seed=seed,
                      izipx=cfg["izip"], izipv=cfg["izip"], f_cdm=(1.0 - NU_F) if nu else 1.0)
    if nu:
        # fluid meshes nf/2, nf/4, nf/8 and hg_setup's cs2 = (u/beta*c * hg_dv)^2 (hydrogr.f90:66)
        f32 = np.float32
        nf = 4 * cfg["nc"]
        hg_dv = f32(2 * nf) / ((f32(300.0) * np.sqrt(f32(0.3))) * f32(cfg["box"]))
        beta = f32(5966.34) * f32(NU_M_EV)
        st.nu_fluids = []
        for k in range(3):
            cs = (f32(GL_V[k]) / beta) * f32(2.998e5) * hg_dv
            st.nu_fluids.append(ic.nu_fluid_linear(cfg["nc"], cfg["box"], cfg["z_i"], seed, fluid_n=nf >> (k + 1),
                                                   gl_v=GL_V[k], m_nu_ev=NU_M_EV, cs2=float(cs * cs)))
    try:
        with open(path + ".tmp", "wb") as f:
            pickle.dump(st, f, protocol=4)
        os.replace(path + ".tmp", path)
    except OSError:
        pass
    return st


def nu_params_for(cfg):
    from cube_nufluid_b200 import make_params
    return make_params(cfg["nc"], cfg["nnt"], box=cfg["box"], izipx=cfg["izip"], izipv=cfg["izip"],
                       ext_pp_force=cfg["pp"], neutrino=True, f_neu=NU_F, m_nu_ev=NU_M_EV, deg_nu=NU_DEG,
                       z_i_nu=10.0, omega_m=0.3, omega_l=0.7, h0=NU_H)


# DRAM bytes per step and phase (dram__bytes_read.sum + dram__bytes_write.sum summed
# over the phase's kernels), measured with
#   ncu --metrics gpu__time_duration.sum,dram__bytes_read.sum,dram__bytes_write.sum \
#       --clock-control none -c 400 --csv python bench.py --config <c> --steps 1 --warmup 3
# over the five steps that command runs; the roofline's "traffic" field.
MEASURED_DRAM_BYTES = {
    "c2": {"update_x": 21.063e9, "ext_pp_force": 2.530e9, "deposit": 5.916e9, "fine_fft_green": 87.852e9,
           "coarse_fft_green": 1.055e9, "kick": 15.925e9},
    "c3": {"update_x": 21.271e9, "ext_pp_force": 2.534e9, "deposit": 28.351e9, "fine_fft_green": 87.852e9,
           "coarse_fft_green": 1.055e9, "kick": 16.283e9, "nu_fluid": 80.798e9},
}


def algorithmic_bytes(cfg, npart):
    """Per-phase algorithmic bytes of one step (definitions of the survey, sec. 8(d))."""
    nc = cfg["nc"]
    nf = 4 * nc
    Nf, Nc = nf ** 3, nc ** 3
    bx = bv = 3 * cfg["izip"]
    kf = 3 * (nf // 2 + 1) ** 3 * 4
    kc = 3 * (nc // 2 + 1) ** 3 * 4
    out = {
        "update_x": npart * (2 * bx + 2 * bv + 8),
        "ext_pp_force": npart * (bx + 2 * bv),
        "deposit": npart * bx + Nc * 4 + Nf * 4 + Nc * 4,
        "fine_fft_green": 4 * 8 * Nf + kf,
        "coarse_fft_green": 4 * 8 * Nc + kc,
        "kick": npart * (bx + 2 * bv) + Nf * 12 + Nc * 12 + Nc * 12 + Nc * 8,
    }
    if cfg.get("nu"):
        # two half steps of 3 sweeps (5 floats in, 5 out per cell) and a CFL pass (5 in),
        # plus the gravity coupling: fine force once, the x/y restriction out and back
        # in, and 5 in + 4 out per fluid cell
        cells = sum((nf >> k) ** 3 for k in (1, 2, 3))
        planes = sum((nf >> k) ** 2 for k in (1, 2, 3))
        out["nu_fluid"] = 2 * (3 * 40 + 20) * cells + 12 * Nf + 2 * 20 * (nf + 4) * planes + 36 * cells
    return out


PHASES = ["update_x", "ext_pp_force", "deposit", "fine_fft_green", "coarse_fft_green", "kick"]


def run_ours(args, cfg, rank, world, local_rank):
    import torch
    import torch.distributed as dist
    from cube_nufluid_b200 import Cube, make_params, scalars_from_ic

    torch.cuda.set_device(local_rank)
    st = make_state(cfg, seed=1000 + rank)
    nu = bool(cfg.get("nu"))
    if nu:
        p = nu_params_for(cfg)
    else:
        p = make_params(cfg["nc"], cfg["nnt"], box=cfg["box"], izipx=cfg["izip"], izipv=cfg["izip"],
                        ext_pp_force=cfg["pp"])
    cube = Cube(p, np_capacity=st.np)
    stream = torch.cuda.Stream()
    cube.L.cube_set_stream(cube.h, stream.cuda_stream)
    cube.load_state(st.xp, st.vp, st.pid, st.rhoc, st.vfield)
    if nu:
        for k in range(3):
            cube.nu_load(k, st.nu_fluids[k])
    s = scalars_from_ic(st)
    npart = st.np
    nu_ms = [0.0]

    def step():
        # main.f90:49-64: timestep, neutrino half step, drift, PP, PM, neutrino half step
        cube.timestep(s)
        if nu:
            s.dt_neu = cube.nu_evolve(s.dt / 2.0, s.dt_neu, 1, s.a_mid)
            nu_ms[0] += cube.phase_times()[6]
        cube.update_x(s)
        if cfg["pp"]:
            cube.ext_pp_force(s)
        cube.particle_mesh(s)
        if nu:
            nu_ms[0] += cube.phase_times()[6]  # gravity on the fluids
            s.dt_neu = cube.nu_evolve(s.dt / 2.0, s.dt_neu, -1, s.a_mid)
            nu_ms[0] += cube.phase_times()[6]

    for _ in range(args.warmup):
        step()
    nu_ms[0] = 0.0
    phase_sum = np.zeros(len(PHASES))
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    l0 = cube.launch_count()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local_rank) as clk:
        with torch.cuda.stream(stream):
            ev0.record(stream)
            for _ in range(args.steps):
                step()
                pt = cube.phase_times()
                phase_sum += np.array([pt[0], pt[1], pt[2], pt[3], pt[4], pt[5]])
            ev1.record(stream)
        torch.cuda.synchronize()
    nu_timed = nu_ms[0]  # the end-to-end leg below runs step() again
    ms = ev0.elapsed_time(ev1)
    launches = cube.launch_count() - l0
    t = torch.tensor([ms], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dist.barrier()
    ms_max = float(t.item())

    # end to end through the C-ABI with host-resident arrays (pinned)
    pin = {}
    for name, a in (("xp", st.xp), ("vp", st.vp), ("pid", st.pid), ("rhoc", st.rhoc), ("vfield", st.vfield)):
        h = torch.empty(a.nbytes, dtype=torch.uint8, pin_memory=True)
        h.numpy()[:] = np.ascontiguousarray(a).view(np.uint8).reshape(-1)
        pin[name] = h
    xp_h = pin["xp"].numpy().view(st.xp.dtype).reshape(st.xp.shape)
    vp_h = pin["vp"].numpy().view(st.vp.dtype).reshape(st.vp.shape)
    pid_h = pin["pid"].numpy().view(np.int32)
    rhoc_h = pin["rhoc"].numpy().view(np.int32)
    vf_h = pin["vfield"].numpy().view(np.float32).reshape(st.vfield.shape)
    import ctypes as C

    def ptr(a):
        return a.ctypes.data_as(C.c_void_p)

    e2e_steps = max(1, min(args.steps, 3))
    h2d = xp_h.nbytes + vp_h.nbytes + pid_h.nbytes + rhoc_h.nbytes + vf_h.nbytes
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        e0.record(stream)
        for _ in range(e2e_steps):
            cube._check(cube.L.cube_load_state(cube.h, xp_h.shape[0], ptr(xp_h), ptr(vp_h), ptr(pid_h),
                                               ptr(rhoc_h), ptr(vf_h)))
            step()
            n = C.c_int64(0)
            cube._check(cube.L.cube_store_state(cube.h, C.byref(n), ptr(xp_h), ptr(vp_h), ptr(pid_h),
                                                ptr(rhoc_h), ptr(vf_h)))
        e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1)
    t2 = torch.tensor([e2e_ms], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(t2, op=dist.ReduceOp.MAX)
    e2e_ms = float(t2.item())
    if nu:
        phase_sum = np.append(phase_sum, nu_timed)
    return dict(ms=ms_max, npart=npart, launches=launches, phase_ms=phase_sum / args.steps, clocks=clk.summary(),
                e2e_ms=e2e_ms, e2e_steps=e2e_steps, h2d=h2d, d2h=h2d, scal=s.as_dict())


def cpu_sample(threads: int):
    """The CPU oracle on a bounded sample: one step (update_x + PP + particle_mesh)
    of a 64^3-particle box with the workload's method settings, OpenMP over all
    host threads where the reference's loops are parallel (its nlayer scheme)."""
    os.environ.setdefault("OMP_NUM_THREADS", str(threads))
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from oracle_ref import Oracle
    from cube_nufluid_b200 import ic, tables, make_params, scalars_from_ic

    st = ic.zeldovich(32, 2, box=200.0, z_i=49.0, seed=7)
    p = make_params(32, 2, box=200.0, ext_pp_force=True)
    o = Oracle(p, tables.read_fine_table(), tables.read_coarse_table())
    o.load(st.xp, st.vp, st.pid, st.rhoc, st.vfield)
    s = scalars_from_ic(st)
    s.dt_old = s.dt = 0.5
    s.a_mid = s.a
    t0 = time.perf_counter()
    o.update_x(s)
    o.ext_pp_force(s)
    o.particle_mesh(s, 0)
    dt = time.perf_counter() - t0
    return {"value": st.np / dt, "unit": "particle-updates/s", "cores": threads, "kind": "port",
            "sample": f"1 step (update_x + ext_pp_force + particle_mesh, FP32 reference-order deposit, FP64 FFT) "
                      f"of a {st.np}-particle box (nc=32, nf=128, 2^3 tiles) on {threads} host threads; "
                      f"{dt:.1f} s"}


def run_ensemble(args, cfg):
    """C4: box-steps/s of an ensemble of independent boxes on one GPU (per rank)."""
    import torch
    from cube_nufluid_b200 import build
    from cube_nufluid_b200.ensemble import Ensemble, ensemble_specs
    rank = int(os.environ.get("RANK", 0))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(local_rank)
    if rank == 0:
        build.build()
    specs = ensemble_specs(cfg["ensemble"], 2024 + rank)
    ens = Ensemble(specs)
    workers = 16
    ens.run(args.warmup, workers=workers)
    torch.cuda.synchronize()
    l0 = sum(m.cube.launch_count() for m in ens.members)
    with ClockSampler(local_rank) as clk:
        r = ens.run(args.steps, workers=workers)
        torch.cuda.synchronize()
    launches = sum(m.cube.launch_count() for m in ens.members) - l0
    npart = sum(sp.particles for sp in specs)
    line = {"metric": "ensemble box-steps/s", "value": r["box_steps_per_s"], "unit": "box-steps/s",
            "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": r["wall_s"] * 1e3 / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": cfg["workload"], "boxes": len(specs), "particles_total": npart,
                       "workers": r["workers"], "parallelism": "boxes on concurrent streams",
                       "timing": "host wall clock between device synchronisations (one stream per box)"},
            "particle_updates_per_s": r["particle_updates_per_s"], "gpu_launches": int(launches),
            "clocks": clk.summary()}
    ens.close()
    if rank == 0:
        print(json.dumps(line))


def run_late(args, cfg):
    """C6: particle-updates/s of steps of a clustered late-time state; device time of
    each step from the library's own events on its stream."""
    import torch
    from cube_nufluid_b200 import build, ic
    from cube_nufluid_b200.abi import CubeScalars, make_params
    from cube_nufluid_b200.cube import Cube
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(local_rank)
    build.build()
    nc, box = cfg["nc"], cfg["box"]
    cube = Cube(make_params(nc, cfg["nnt"], box=box, omega_m=0.3, omega_l=0.7, izipx=cfg["izip"], izipv=cfg["izip"],
                            ext_pp_force=cfg["pp"]), np_capacity=(2 * nc) ** 3)
    cache = args.state_cache
    if cache and os.path.exists(cache):
        d = np.load(cache)
        cube.load_state(d["xp"], d["vp"], d["pid"], d["rhoc"], d["vfield"])
        s = CubeScalars.from_buffer_copy(d["scal"].tobytes())
    else:
        cos = ic.Cosmology(omega_m=0.3, omega_l=0.7, sigma8=0.8)
        s = cube.make_ic(ic.device_ic_params(cos, cfg["z_i"], nc, box=box), 7)
        n = 0
        for a_next in np.geomspace(s.a, 1.0, 49)[1:]:
            while True:
                n += 1
                if cube.step(s, a_next=float(a_next)) or n > 2000:
                    break
        if cache:
            xp, vp, pid, rhoc, vfield = cube.store_state()
            np.savez(cache, xp=xp, vp=vp, pid=pid, rhoc=rhoc, vfield=vfield, scal=np.frombuffer(bytes(s), np.uint8))
    rhoc = cube.store_state()[3]
    for _ in range(args.warmup):
        cube.step(s)
    l0 = cube.launch_count()
    ph = np.zeros(8)
    with ClockSampler(local_rank) as clk:
        for _ in range(args.steps):
            cube.step(s)
            ph += np.array(cube.phase_times())
    launches = cube.launch_count() - l0
    npart = (2 * nc) ** 3
    ms = float(ph[7])
    line = {"metric": "late-time PM step particle-updates/s", "value": npart * args.steps / (ms / 1e3),
            "unit": "particle-updates/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic",
            "config": {"workload": cfg["workload"], "particles": npart, "nc": nc, "nf": 4 * nc,
                       "largest_cell": int(rhoc.max()), "cells_over_4096": int((rhoc > 4096).sum()),
                       "timing": "device time of each step (the library's CUDA events on its stream)"},
            "gpu_launches": int(launches),
            "phases_ms": {k: float(v) / args.steps for k, v in zip(PHASES, ph[:6])}, "clocks": clk.summary()}
    cube.close()
    print(json.dumps(line))


def run_serving(args, cfg):
    """C5: latency percentiles of a Poisson request stream served on one GPU, and the
    same percentiles relative to each request's plain service time (its size served
    alone on an idle GPU)."""
    import torch
    from cube_nufluid_b200 import build
    from cube_nufluid_b200.serving import SERVE_SIDES, Request, Server, request_stream
    from cube_nufluid_b200.ensemble import BoxSpec
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(local_rank)
    build.build()
    srv = Server(hbm_budget=160e9, workers=8)
    # warm-up: one request per size creates the contexts; then the plain service
    # time of each size on the idle server (contexts reused, as under load)
    plain = {}
    for rep in range(2):
        for i, side in enumerate(SERVE_SIDES):
            req = Request(-1, 0.0, BoxSpec(nc=side // 2, box=200.0, omega_m=0.3, sigma8=0.8, seed=77 + i))
            t = time.perf_counter()
            srv.answer(req)
            plain[side // 2] = time.perf_counter() - t
    reqs = request_stream(cfg["serving"], 20.0, 2025)
    with ClockSampler(local_rank) as clk:
        t0 = time.perf_counter()
        ans = srv.serve(reqs, realtime=True)
        wall = time.perf_counter() - t0
    srv.close()
    lat = np.array([a.latency for a in ans])
    slow = np.array([a.latency / plain[r.spec.nc] for a, r in zip(ans, reqs)])
    line = {"metric": "serving p99 latency", "value": float(np.percentile(lat, 99)), "unit": "s",
            "n_gpus": 1, "steps": 48, "warmup": 2 * len(SERVE_SIDES), "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": cfg["workload"], "requests": len(reqs), "workers": 8,
                       "timing": "host wall clock per request (arrival to answer)"},
            "latency_s": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                          "max": float(lat.max())},
            "vs_plain": {"p50": float(np.percentile(slow, 50)), "p99": float(np.percentile(slow, 99))},
            "plain_service_s": {str(2 * k): v for k, v in sorted(plain.items())},
            "requests_per_s": len(reqs) / wall, "steps_mean": float(np.mean([a.steps for a in ans])),
            "offered_gpu_s_per_s": 20.0 * float(np.mean([plain[r.spec.nc] for r in reqs])),
            "clocks": clk.summary()}
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="c2", choices=list(CONFIGS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--state-cache", default="", help="c6: file holding the evolved state (made if absent)")
    args = ap.parse_args()
    cfg = CONFIGS[args.config]
    if cfg.get("late"):
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the late-time state is made by this library's "
                              "own evolution; the reference's CPU path is timed on the single-box configurations"}))
            return
        run_late(args, cfg)
        return
    if cfg.get("serving"):
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the reference has no serving mode; "
                              "its CPU path is timed on the single-box configurations"}))
            return
        run_serving(args, cfg)
        return
    if cfg.get("ensemble"):
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the reference has no ensemble mode; "
                              "its CPU path is timed on the single-box configurations"}))
            return
        run_ensemble(args, cfg)
        return
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    npart = (2 * cfg["nc"]) ** 3
    config = {"workload": cfg["workload"], "particles": npart, "nc": cfg["nc"], "nf": 4 * cfg["nc"],
              "tiles": cfg["nnt"] ** 3, "parallelism": f"replicas x{args.gpus}",
              "l2": "inputs larger than L2 (meshes of GBs)", "ic": "Zel'dovich z=49, seeded (synthetic)"}
    metric = "PM step particle-updates/s"

    if args.impl == "reference":
        if rank != 0:
            return
        base = cpu_sample(os.cpu_count() or 1)
        line = {"impl": "reference", "metric": metric, "value": base["value"], "unit": "particle-updates/s",
                "n_gpus": args.gpus, "steps": 1, "warmup": 0, "higher_is_better": True, "config": config,
                "cpu_baseline": base, "e2e": {"value": base["value"], "unit": "particle-updates/s",
                                              "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
                "data": "synthetic", "dtype": "f32"}
        print(json.dumps(line))
        return

    import torch
    import torch.distributed as dist
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    from cube_nufluid_b200 import build
    if rank == 0:
        build.build()
    if world > 1:
        dist.barrier()
    r = run_ours(args, cfg, rank, world, local_rank)
    value = r["npart"] * world * args.steps / (r["ms"] / 1e3)
    e2e = r["npart"] * world * r["e2e_steps"] / (r["e2e_ms"] / 1e3)
    peak, peak_kind = read_peaks()
    ab = algorithmic_bytes(cfg, r["npart"])
    names = PHASES + (["nu_fluid"] if cfg.get("nu") else [])
    phases = {k: float(v) for k, v in zip(names, r["phase_ms"])}
    dom = max(phases, key=lambda k: phases[k])
    ach = ab[dom] / (phases[dom] / 1e3) / 1e9
    phase_gbs = {k: (ab[k] / (phases[k] / 1e3) / 1e9 if phases[k] > 0 else None) for k in names}
    line = {
        "metric": metric, "value": value, "unit": "particle-updates/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": r["ms"] / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic", "config": config,
        "e2e": {"value": e2e, "unit": "particle-updates/s", "h2d_bytes_per_step": r["h2d"],
                "d2h_bytes_per_step": r["d2h"], "steps": r["e2e_steps"]},
        "gpu_launches": int(r["launches"]),
        "roofline": {"kernel": dom, "bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s",
                     "frac": ach / peak, "peak_kind": peak_kind,
                     "traffic": MEASURED_DRAM_BYTES.get(args.config, {}).get(dom),
                     "algorithmic_bytes": ab[dom]},
        "phases_ms": phases, "phase_gbs": phase_gbs, "clocks": r["clocks"],
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_sample(os.cpu_count() or 1)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line))


if __name__ == "__main__":
    main()
