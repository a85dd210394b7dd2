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
    "c1": dict(nc=32, nnt=2, box=200.0, izip=2, izipx=1, izipv=2, pp=False, z_i=49.0,
               workload="64^3 particles, 200 Mpc/h, fine 128^3, coarse 32^3, int1 x / int2 v, PP off"),
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
    # precision study: the same 64 steps in FP32 and in the FP64 Poisson mode from one
    # seeded IC (force error against the FP64 run of the same step, P(k) ratio at z=0)
    "c2p": dict(nc=256, nnt=8, box=1000.0, izip=2, pp=True, z_i=49.0, precision=64,
                workload="precision study: 512^3 particles, 1000 Mpc/h, fine 1024^3, coarse 256^3, int2 x/v, "
                         "PP on; 64 steps z=49 -> 0 in FP32 and in the FP64 Poisson mode from the same IC"),
    "c2ps": dict(nc=128, nnt=4, box=500.0, izip=2, pp=True, z_i=49.0, precision=64,
                 workload="precision study (profiling size): 256^3 particles, 500 Mpc/h, fine 512^3, coarse "
                          "128^3, int2 x/v, PP on; 64 steps z=49 -> 0 in FP32 and in FP64 Poisson mode"),
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
    """nvidia-smi clock / throttle-reason samples during the timed region.

    start() launches nvidia-smi and waits for its first row, so that its start-up
    happens before the warm-up steps, not inside the timed region; the timed region
    is bracketed by `with sampler:` and summary() keeps the rows that arrived inside
    it (with the nearest row on either side when the region is shorter than the
    200 ms sampling period)."""

    def __init__(self, index: int):
        self.index = index
        self.rows = []  # (arrival time, fields)
        self.proc = None
        self.t0 = self.t1 = None

    def start(self, wait_s: float = 10.0):
        if self.proc is not None:
            return self
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            t_end = time.time() + wait_s
            while not self.rows and time.time() < t_end and self.proc.poll() is None:
                time.sleep(0.05)
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 9:
                self.rows.append((time.time(), parts))

    def __enter__(self):
        self.start()
        self.t0 = time.time()
        return self

    def __exit__(self, *a):
        self.t1 = time.time()
        time.sleep(0.25)  # one more row after the region
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        t0 = self.t0 if self.t0 is not None else 0.0
        t1 = self.t1 if self.t1 is not None else time.time()
        inside = [r for (t, r) in self.rows if t0 <= t <= t1]
        if not inside:
            before = [r for (t, r) in self.rows if t < t0][-1:]
            after = [r for (t, r) in self.rows if t > t1][:1]
            inside = before + after
        if not inside:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in inside if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in inside if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in inside for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(inside)}


def make_state(cfg, seed):
    """Seeded Zel'dovich state; cached under $TMPDIR so repeated runs on one host skip the host-side IC."""
    import pickle
    import tempfile
    from cube_nufluid_b200 import ic
    nu = bool(cfg.get("nu"))
    zx, zv = cfg.get("izipx", cfg["izip"]), cfg.get("izipv", cfg["izip"])
    key = f"cube_ic_{cfg['nc']}_{cfg['nnt']}_{cfg['box']}_{cfg['z_i']}_{zx}{zv}_{seed}_{int(nu)}.pkl"
    path = os.path.join(tempfile.gettempdir(), key)
    if os.path.exists(path):
        with open(path, "rb") as f:
            return pickle.load(f)
    st = ic.zeldovich(cfg["nc"], cfg["nnt"], box=cfg["box"], z_i=cfg["z_i"], seed=seed,
                      izipx=zx, izipv=zv, f_cdm=(1.0 - NU_F) if nu else 1.0)
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


def plain_params_for(cfg):
    from cube_nufluid_b200 import make_params
    return make_params(cfg["nc"], cfg["nnt"], box=cfg["box"], izipx=cfg.get("izipx", cfg["izip"]),
                       izipv=cfg.get("izipv", cfg["izip"]), ext_pp_force=cfg["pp"])


def nu_params_for(cfg):
    from cube_nufluid_b200 import make_params
    return make_params(cfg["nc"], cfg["nnt"], box=cfg["box"], izipx=cfg["izip"], izipv=cfg["izip"],
                       ext_pp_force=cfg["pp"], neutrino=True, f_neu=NU_F, m_nu_ev=NU_M_EV, deg_nu=NU_DEG,
                       z_i_nu=10.0, omega_m=0.3, omega_l=0.7, h0=NU_H)


# DRAM bytes per step and phase (dram__bytes_read.sum + dram__bytes_write.sum of the
# phase's kernels) from single-kernel ncu captures of the 256^3-particle case (c2s),
# summarised with their commands in profiles/: the fine solve is x r2c, four y passes
# (forward and three inverse, each as the forward one), z + Green and the c2r of the
# three components; the kick is one launch.  Particle counts and mesh sizes both grow
# by 8 from c2s to c2 (and the fine mesh is the same in c3), so these scale with the
# particle count; phases without a capture of every kernel have none.
TRAFFIC_C2S = {"fine_fft_green": (0.537 + 0.492) + 4 * (0.539 + 0.492) + (0.743 + 1.568) + (1.711 + 1.554),
               "kick": 1.894 + 0.100, "deposit": 0.135 + 0.498}  # GB per step at 256^3 particles


def phase_traffic(config, phase, npart):
    """DRAM bytes per step of a phase, scaled from the c2s captures (None if not captured)."""
    if config not in ("c2", "c2s", "c3", "c3s") or phase not in TRAFFIC_C2S:
        return None
    if config in ("c3", "c3s") and phase != "fine_fft_green":
        return None  # the neutrino densities and sources change the other phases
    return TRAFFIC_C2S[phase] * 1e9 * npart / 256 ** 3


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


def max_over_ranks(x: float, world: int, device: str = "cuda") -> float:
    """The largest of a per-rank figure (a device time) over the ranks; every rank
    calls it at the same point.  One rank: the figure itself."""
    if world <= 1:
        return float(x)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(npart_per_rank: int, world: int, steps: int, ms_max: float) -> float:
    """Whole-job particle-updates/s: every rank advances its own box of npart_per_rank
    particles (replicas, weak scaling), over the slowest rank's time."""
    return npart_per_rank * world * steps / (ms_max / 1e3)


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
        p = plain_params_for(cfg)
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

    clk = ClockSampler(local_rank).start()
    for _ in range(args.warmup):
        step()
    nu_ms[0] = 0.0
    phase_sum = np.zeros(len(PHASES))
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    l0 = cube.launch_count()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with clk:
        with torch.cuda.stream(stream):
            ev0.record(stream)
            for _ in range(args.steps):
                step()
                pt = cube.phase_times()
                phase_sum += np.array([pt[0], pt[1], pt[2], pt[3], pt[4], pt[5]])
            ev1.record(stream)
        torch.cuda.synchronize()
    nu_timed = nu_ms[0]  # the end-to-end leg below runs step() again
    npairs_timed = int(getattr(s, "npairs", 0))  # PP window entries of the last timed step
    ms = ev0.elapsed_time(ev1)
    launches = cube.launch_count() - l0
    ms_max = max_over_ranks(ms, world)
    if world > 1:
        dist.barrier()

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

    # the end-to-end leg continues the evolved state: it starts from the state the timed
    # steps left (stored untimed), and every step loads the state from and stores it to
    # pinned host memory around the step, for as many steps as the timed region
    n0 = C.c_int64(0)
    cube._check(cube.L.cube_store_state(cube.h, C.byref(n0), ptr(xp_h), ptr(vp_h), ptr(pid_h), ptr(rhoc_h),
                                        ptr(vf_h)))
    torch.cuda.synchronize()
    e2e_steps = max(1, args.steps)
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
    e2e_ms = max_over_ranks(e0.elapsed_time(e1), world)
    if nu:
        phase_sum = np.append(phase_sum, nu_timed)
    cufft = None
    if getattr(args, "cufft", False) and world == 1:
        cufft = cufft_comparison(cube, 4 * cfg["nc"])
    return dict(cufft=cufft, ms=ms_max, npart=npart, launches=launches, phase_ms=phase_sum / args.steps, clocks=clk.summary(),
                e2e_ms=e2e_ms, e2e_steps=e2e_steps, h2d=h2d, d2h=h2d, scal=s.as_dict(), npairs=npairs_timed)


def cufft_comparison(cube, nf: int, reps: int = 5) -> dict:
    """The fine-mesh Poisson solve of the library (its own FFT passes with the Green
    multiply and the kick scale fused) timed beside the same transforms done by
    cuFFT through torch.fft (one r2c, three c2r, the Green multiply as a separate
    elementwise pass) on a mesh of the same size.  A timed comparison only: cuFFT
    is never on the library's path."""
    import ctypes as C
    import torch
    ms = C.c_float(0.0)
    cube._check(cube.L.cube_debug_time_poisson(cube.h, reps, C.byref(ms)))
    ours = float(ms.value)
    x = torch.randn(nf, nf, nf, device="cuda", dtype=torch.float32)
    kern = torch.randn(3, nf, nf, nf // 2 + 1, device="cuda", dtype=torch.float32)

    def fft_only():
        X = torch.fft.rfftn(x)
        return [torch.fft.irfftn(X, s=x.shape) for _ in range(3)]

    def with_green():
        X = torch.fft.rfftn(x)
        return [torch.fft.irfftn(X * (1j * kern[d]), s=x.shape) for d in range(3)]

    out = {"library_ms": ours}
    for name, fn in (("cufft_transforms_ms", fft_only), ("cufft_with_green_ms", with_green)):
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            r = fn()
            del r
        e1.record()
        torch.cuda.synchronize()
        out[name] = e0.elapsed_time(e1) / reps
    del x, kern
    torch.cuda.empty_cache()
    out["mesh"] = f"{nf}^3, one r2c + three c2r (+ Green multiply), FP32"
    return out


def cpu_sample(threads: int, cfg=None, steps: int = 3, warmup: int = 1):
    """The CPU oracle (a restatement of the reference's step) on a bounded sample of
    the workload itself: the seeded state of the configuration, and per sample step
    one of its tiles run through the oracle's per-tile loops of update_x,
    ext_pp_force and particle_mesh (the reference's loop structure, FP32
    reference-order deposit, OpenMP where the reference's loops are parallel) with
    the particle state left as it was.  The global coarse Poisson solve is timed
    once and charged to each sample in proportion to its particles.  Rate =
    sampled particles / (their tiles' time + their share of the coarse solve)."""
    os.environ.setdefault("OMP_NUM_THREADS", str(threads))
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from oracle_ref import Oracle
    from cube_nufluid_b200 import tables, scalars_from_ic
    cfg = cfg or CONFIGS["c2"]
    t_setup = time.perf_counter()
    st = make_state(cfg, seed=1000)
    p = nu_params_for(cfg) if cfg.get("nu") else plain_params_for(cfg)
    o = Oracle(p, tables.read_fine_table(), tables.read_coarse_table())
    o.load(st.xp, st.vp, st.pid, st.rhoc, st.vfield)
    s = scalars_from_ic(st)
    import ctypes as C
    from cube_nufluid_b200.cube import load_library
    hit = C.c_int32(0)
    load_library().cube_timestep(C.byref(p), C.byref(s), C.c_float(0.0), C.byref(hit))
    nnt, nt = cfg["nnt"], cfg["nc"] // cfg["nnt"]
    ntiles = nnt ** 3
    tile_np = np.asarray(st.rhoc, dtype=np.int64).reshape(ntiles, nt ** 3).sum(axis=1)
    t0 = time.perf_counter()
    o.coarse_poisson()
    t_coarse = time.perf_counter() - t0
    t_setup = time.perf_counter() - t_setup
    rng = np.random.default_rng(7)
    order = rng.permutation(ntiles)
    done_np, done_t = 0, 0.0
    for i in range(warmup + steps):
        tile = int(order[i % ntiles])
        mask = np.zeros(ntiles, np.int8)
        mask[tile] = 1
        o.set_tile_mask(mask)
        ss = s.copy()
        t0 = time.perf_counter()
        o.update_x(ss)
        if cfg["pp"]:
            o.ext_pp_force(ss)
        o.particle_mesh(ss, 0)
        dt = time.perf_counter() - t0
        if i >= warmup:
            done_np += int(tile_np[tile])
            done_t += dt + t_coarse * float(tile_np[tile]) / float(st.np)
    o.set_tile_mask(None)
    return {"value": done_np / done_t, "unit": "particle-updates/s", "cores": threads, "kind": "port",
            "sample": f"{steps} sample steps (after {warmup} untimed), each one tile of the {st.np}-particle "
                      f"{cfg['nc']}^3-cell state ({nt}^3 coarse cells, about {int(tile_np.mean())} particles) "
                      f"through the CPU oracle's update_x + ext_pp_force + particle_mesh tile loops "
                      f"(FP32 reference-order deposit, FP64 FFT) on {threads} host threads, plus the global "
                      f"coarse Poisson solve ({t_coarse:.2f} s, timed once) charged per particle; "
                      f"{done_t:.1f} s timed, {t_setup:.0f} s set-up",
            "tiles_timed": steps, "coarse_solve_s": t_coarse}


def _rel_rms_chunked(a, b, scale_a=1.0, scale_b=1.0, chunk=1 << 26):
    """sqrt(sum((a/sa - b/sb)^2) / sum((b/sb)^2)) over large arrays, in chunks."""
    num = den = 0.0
    for i in range(0, a.size, chunk):
        x = a[i:i + chunk].astype(np.float64) / scale_a
        y = b[i:i + chunk].astype(np.float64) / scale_b
        num += float(np.sum((x - y) ** 2))
        den += float(np.sum(y * y))
    return float(np.sqrt(num / den))


def run_precision(args, cfg):
    """Precision study: the configuration's step run twice from the same seeded state,
    once in FP32 and once in the library's FP64 Poisson mode (FP64 meshes, FFT, Green
    and interpolation; the same integer deposit, codec and PP), in lockstep time steps
    (the FP64 run takes the FP32 run's dt limits).  Each run takes whole steps in the
    order of Cube.step and is never read or reloaded in the middle of one.  At
    checkpoint steps a third context, in the FP64 mode, takes the FP32 run's state
    after its step and runs that step's particle_mesh on it: the kick moves no
    particle, so its force meshes are the FP64 forces of the positions the FP32 run
    just deposited, and the relative RMS difference of the fine and coarse force meshes
    is the FP32 force error.  At z = 0 the power spectra of the two runs (the library's
    P(k), 4 log bins per octave) give the P(k) ratio."""
    import torch
    from cube_nufluid_b200 import Cube, build, scalars_from_ic
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(local_rank)
    build.build()
    st = make_state(cfg, seed=1000)
    p32 = plain_params_for(cfg)
    p64 = type(p32).from_buffer_copy(p32)
    p64.poisson_fp64 = 1
    g32, g64 = Cube(p32, st.np), Cube(p64, st.np)
    for g in (g32, g64):
        g.load_state(st.xp, st.vp, st.pid, st.rhoc, st.vfield)
    s32 = scalars_from_ic(st)
    s64 = s32.copy()
    nsteps = cfg["precision"]
    targets = np.geomspace(float(s32.a), 1.0, nsteps + 1)[1:]
    checks = {0, nsteps // 4, nsteps // 2, (3 * nsteps) // 4, nsteps - 1}
    limits = ("dt_fine", "dt_coarse", "dt_pp", "dt_vmax", "dt_vmax_nu", "dt_neu")
    rows = []
    n = 0
    pif = float(np.float32(4.0) * np.arctan(np.float32(1.0)))
    gp = None  # the probe context, made at the first checkpoint
    for i, a_next in enumerate(targets):
        hit = False
        while not hit:
            for k in limits:
                setattr(s64, k, getattr(s32, k))
            probe = None
            for g, sc in ((g32, s32), (g64, s64)):
                h = g.timestep(sc, float(a_next))
                g.update_x(sc)
                if cfg["pp"]:
                    g.ext_pp_force(sc)
                if g is g32:
                    hit = h
                    probe = s32.copy()  # the scalars particle_mesh starts from
                g.particle_mesh(sc)
            if hit and i in checks:
                # FP64 forces of the positions the FP32 run deposited in this step
                if gp is None:
                    gp = Cube(p64, st.np)
                gp.load_state(*g32.store_state())
                gp.particle_mesh(probe)
                f64, c64 = gp.fetch(2), gp.fetch(3)
                f32, c32 = g32.fetch(2), g32.fetch(3)
                # both meshes hold force * ((a_mid dt)/6)/pi: compare the forces
                k32 = float(np.float32(np.float32(np.float32(probe.a_mid) * np.float32(probe.dt)) / np.float32(6.0))
                            / np.float32(pif))
                k64 = ((float(probe.a_mid) * float(probe.dt)) / 6.0) / pif
                rows.append({"step": n, "a": float(s32.a), "fine": _rel_rms_chunked(f32, f64, k32, k64),
                             "coarse": _rel_rms_chunked(c32, c64, k32, k64)})
                del f64, c64, f32, c32
            n += 1
    if gp is not None:
        gp.close()
    # P(k) of both runs on the FP32 context (the FP64 mode's meshes are not FP32)
    pk32 = g32.power_spectrum(log_bins=True)
    g32.load_state(*g64.store_state())
    pk64 = g32.power_spectrum(log_bins=True)
    ok = pk64[:, 0] > 0
    ratio = pk32[ok, 2] / pk64[ok, 2]
    k = pk32[ok, 1]
    line = {"metric": "precision study: force RMS relative error and P(k) ratio, FP32 vs FP64 Poisson mode",
            "value": float(np.max(np.abs(ratio - 1.0))), "unit": "max |P32/P64 - 1| at z=0",
            "n_gpus": 1, "steps": n, "higher_is_better": False, "dtype": "f32 vs f64", "data": "synthetic",
            "config": {"workload": cfg["workload"], "particles": st.np, "nc": cfg["nc"], "nf": 4 * cfg["nc"]},
            "force_rms_rel_err": rows,
            "pk": {"k_h_per_mpc": [float(x) for x in k], "ratio": [float(x) for x in ratio],
                   "max_abs_dev": float(np.max(np.abs(ratio - 1.0))),
                   "max_abs_dev_k_below_half_nyquist": float(np.max(np.abs(ratio - 1.0)[k <= k.max() / 2]))},
            "a_final": float(s32.a)}
    g32.close()
    g64.close()
    print(json.dumps(line))


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
    clk = ClockSampler(local_rank).start()
    ens.run_native(args.warmup, workers=workers)
    torch.cuda.synchronize()
    l0 = sum(m.cube.launch_count() for m in ens.members)
    with clk:
        r = ens.run_native(args.steps, workers=workers)
        torch.cuda.synchronize()
    launches = sum(m.cube.launch_count() for m in ens.members) - l0
    npart = sum(sp.particles for sp in specs)
    # the same boxes one at a time (one thread, each box-step returns before the next
    # starts): the sequential rate the concurrent ensemble is compared with; and the
    # boxes stepped from Python threads instead of the library's pool
    seq_steps = max(1, min(args.steps, 2))
    seq = ens.run_native(seq_steps, workers=1)
    pyt = ens.run(seq_steps, workers=workers)
    torch.cuda.synchronize()
    line = {"metric": "ensemble box-steps/s", "value": r["box_steps_per_s"], "unit": "box-steps/s",
            "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": r["wall_s"] * 1e3 / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": cfg["workload"], "boxes": len(specs), "particles_total": npart,
                       "workers": r["workers"], "parallelism": "boxes on concurrent streams, stepped by the "
                                                          "library's thread pool (cube_run_steps)",
                       "timing": "host wall clock between device synchronisations (one stream per box)"},
            "particle_updates_per_s": r["particle_updates_per_s"], "gpu_launches": int(launches),
            "sequential": {"box_steps_per_s": seq["box_steps_per_s"], "steps": seq_steps, "workers": 1},
            "vs_sequential": r["box_steps_per_s"] / seq["box_steps_per_s"],
            "python_threads": {"box_steps_per_s": pyt["box_steps_per_s"], "steps": seq_steps,
                               "workers": pyt["workers"]},
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
    clk = ClockSampler(local_rank).start()
    for _ in range(args.warmup):
        cube.step(s)
    l0 = cube.launch_count()
    ph = np.zeros(8)
    with clk:
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
    clk = ClockSampler(local_rank).start()
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
    with clk:
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
    ap.add_argument("--cufft", action="store_true",
                    help="also time the fine Poisson solve against cuFFT (torch.fft) on the same mesh size")
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
    if cfg.get("precision"):
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the precision study compares the library's "
                              "FP32 and FP64 runs; the reference's CPU path is timed on the single-box "
                              "configurations"}))
            return
        run_precision(args, cfg)
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
        base = cpu_sample(os.cpu_count() or 1, cfg, steps=args.steps, warmup=args.warmup)
        line = {"impl": "reference", "metric": metric, "value": base["value"], "unit": "particle-updates/s",
                "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
                "config": config,
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
    value = job_rate(r["npart"], world, args.steps, r["ms"])
    e2e = job_rate(r["npart"], world, r["e2e_steps"], r["e2e_ms"])
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
                     "traffic": phase_traffic(args.config, dom, r["npart"]),
                     "traffic_source": "ncu DRAM bytes of the phase's kernels at 256^3 particles, scaled by the "
                                       "particle count (profiles/)",
                     "algorithmic_bytes": ab[dom]},
        "phases_ms": phases, "phase_gbs": phase_gbs, "clocks": r["clocks"],
    }
    if cfg["pp"]:
        # window entries the PP walks in the last timed step (ext_pp_force.f90's npairs: every
        # particle of every window fine cell, the target included) and their rate in the PP phase
        npairs = r["npairs"]
        line["pp"] = {"pairs_per_step": npairs, "pairs_per_particle": npairs / r["npart"],
                      "pairs_per_s": npairs / (phases["ext_pp_force"] / 1e3) if phases["ext_pp_force"] > 0 else None}
    if r.get("cufft"):
        line["cufft_comparison"] = r["cufft"]
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_sample(os.cpu_count() or 1, cfg, steps=2, warmup=1)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line))


if __name__ == "__main__":
    main()
