"""A serving loop on one GPU: boxes requested as (size, cosmology, seed), each made,
evolved from z_i to z = 0 and answered with its power spectrum and a particle
subsample.

Requests arrive as a Poisson process.  A pool of host threads serves them in
arrival order, each request on a context of its mesh size taken from a pool of
idle contexts (`cube_set_params` gives a reused context the request's box and
cosmology, `cube_make_ic` its initial state), so that after the first requests of
a size no device memory is allocated or freed: `cudaFree` would wait for the
whole device, stalling every request in flight.  Admission keeps the estimated
device memory of all contexts within an HBM budget; when a new context does not
fit, idle contexts of other sizes are released first, and a request that still
does not fit waits for running ones to finish.

A request's answer does not depend on the load: served alone or among others, on
a fresh or a reused context, it is bit-identical.
"""
from __future__ import annotations

import math
import threading
import time
from collections import deque
from dataclasses import dataclass, field

import numpy as np

from . import ic
from .abi import make_params
from .cube import Cube
from .ensemble import BoxSpec, _nnt

SERVE_SIDES = (32, 48, 64, 96, 128, 192, 256)  # particles per side the sizes snap to


@dataclass
class Request:
    rid: int
    arrival: float        # seconds after the start of the stream
    spec: BoxSpec
    steps: int = 48       # a-targets, log-spaced from 1/(1+z_i) to 1


@dataclass
class Answer:
    rid: int
    pk: np.ndarray        # [nbin, 2]: k (h/Mpc), Delta^2(k), log bins (at most 32)
    sample: np.ndarray    # [n, 3] float32 positions (fine-cell units) of every 64th particle
    steps: int            # steps taken (>= the a-targets)
    wait: float = 0.0     # seconds from arrival to start
    service: float = 0.0  # seconds from start to answer
    latency: float = 0.0


def request_stream(n: int, rate: float, master_seed: int, *, sides=SERVE_SIDES, steps: int = 48) -> list[Request]:
    """n requests with exponential inter-arrival times at `rate` per second, particle
    count log-uniform over sides[0]^3..sides[-1]^3 (snapped to the nearest size in
    log), box 50-400 Mpc/h log-uniform, Omega_m ~ U[0.25, 0.35], sigma_8 ~ U[0.7, 0.9]."""
    rng = np.random.Generator(np.random.Philox(master_seed))
    t = 0.0
    out = []
    logs = np.log(np.asarray(sides, np.float64))
    for i in range(n):
        t += float(rng.exponential(1.0 / rate))
        u = rng.uniform(logs[0], logs[-1])
        side = int(sides[int(np.argmin(np.abs(logs - u)))])
        box = float(math.exp(rng.uniform(math.log(50.0), math.log(400.0))))
        spec = BoxSpec(nc=side // 2, box=box, omega_m=float(rng.uniform(0.25, 0.35)),
                       sigma8=float(rng.uniform(0.7, 0.9)), seed=int(rng.integers(1, 2 ** 62)))
        out.append(Request(i, t, spec, steps))
    return out


def footprint_bytes(nc: int, izip: int = 2) -> int:
    """Estimated device memory of a context of nc coarse cells per side and 8 nc^3
    particles: fine and coarse meshes (density, three force meshes, scratch, Green
    octants), particle arrays (double-buffered codes and PIDs, re-bin scratch, work
    items) and per-cell arrays, plus the scratch that clustered late-time states
    grow (the block sorter's velocity columns, 58 MB; sort slots of cells beyond 4096
    particles, 148 x 32 B x the largest cell rounded up to a power of two, the
    largest cell taken as 0.3% of the particles; split deposit bricks, ~12 B per
    particle), with 10% margin."""
    nf = 4 * nc
    mesh = lambda n: 5 * n * n * (n + 32) * 4 + 3 * (n // 2 + 1) ** 3 * 4
    npart = 8 * nc ** 3
    per_particle = 2 * (6 * izip + 4) + 4 * 4 + 16 + 1 + 1
    per_cell = 2 * 4 + 2 * 8 + 2 * 12 + 24 + 4 + 8 + 1
    big_cell = 1 << max(0, math.ceil(math.log2(max(1.0, 0.003 * npart))))
    late = 58e6 + 148 * 32 * big_cell + 12 * npart
    return int(1.1 * (mesh(nf) + mesh(nc) + npart * per_particle + nc ** 3 * per_cell + late))


def positions(xp: np.ndarray, rhoc: np.ndarray, nc: int, nnt: int, izipx: int) -> np.ndarray:
    """Fine-unit positions of a checkpoint-layout state (storage order)."""
    nt = nc // nnt
    cells = np.arange(nc ** 3)
    l = cells % nt ** 3
    tile = cells // nt ** 3
    g = np.stack([(tile % nnt) * nt + l % nt, ((tile // nnt) % nnt) * nt + (l // nt) % nt,
                  (tile // (nnt * nnt)) * nt + l // (nt * nt)], axis=1)
    cell_of = np.repeat(cells, rhoc.astype(np.int64))
    mask = 0xFF if izipx == 1 else 0xFFFF
    frac = ((xp.astype(np.int64) & mask) + 0.5) / (256.0 if izipx == 1 else 65536.0)
    return (4.0 * (g[cell_of] + frac)).astype(np.float32)


@dataclass
class _Pool:
    idle: dict = field(default_factory=dict)   # nc -> [Cube]
    bytes_total: int = 0                       # estimate over idle and busy contexts


class Server:
    """Serves requests with `workers` host threads within `hbm_budget` bytes."""

    def __init__(self, hbm_budget: float = 160e9, workers: int = 8, fk_table=None, ck_table=None,
                 subsample: int = 64, max_bins: int = 32):
        self.budget = int(hbm_budget)
        self.workers = workers
        self.fk, self.ck = fk_table, ck_table
        self.subsample = subsample
        self.max_bins = max_bins
        self.pool = _Pool()
        self.lock = threading.Condition()

    # ---- contexts ----------------------------------------------------------
    def _params(self, sp: BoxSpec):
        return make_params(sp.nc, _nnt(sp.nc), box=sp.box, omega_m=sp.omega_m, omega_l=1.0 - sp.omega_m,
                           izipx=sp.izip, izipv=sp.izip, ext_pp_force=sp.pp)

    def _acquire(self, sp: BoxSpec) -> Cube:
        need = footprint_bytes(sp.nc, sp.izip)
        with self.lock:
            while True:
                free = self.pool.idle.get(sp.nc)
                if free:
                    return free.pop()
                # release idle contexts of other sizes while the new one does not fit
                while self.pool.bytes_total + need > self.budget:
                    victim = next((k for k, v in self.pool.idle.items() if v), None)
                    if victim is None:
                        break
                    c = self.pool.idle[victim].pop()
                    c.close()
                    self.pool.bytes_total -= footprint_bytes(victim)
                if self.pool.bytes_total + need <= self.budget:
                    self.pool.bytes_total += need
                    break
                self.lock.wait()  # a running request will return its context
        try:
            return Cube(self._params(sp), np_capacity=sp.particles, fk_table=self.fk, ck_table=self.ck)
        except Exception:
            with self.lock:
                self.pool.bytes_total -= need
                self.lock.notify_all()
            raise

    def _release(self, nc: int, cube: Cube):
        with self.lock:
            self.pool.idle.setdefault(nc, []).append(cube)
            self.lock.notify_all()

    def close(self):
        with self.lock:
            for v in self.pool.idle.values():
                for c in v:
                    c.close()
            self.pool.idle.clear()
            self.pool.bytes_total = 0

    # ---- one request ---------------------------------------------------------
    def answer(self, req: Request) -> Answer:
        sp = req.spec
        cube = self._acquire(sp)
        try:
            cube.set_params(self._params(sp))
            cos = ic.Cosmology(omega_m=sp.omega_m, omega_l=1.0 - sp.omega_m, sigma8=sp.sigma8)
            s = cube.make_ic(ic.device_ic_params(cos, sp.z_i, sp.nc, box=sp.box), sp.seed)
            targets = np.geomspace(s.a, 1.0, req.steps + 1)[1:]
            n = 0
            for a_next in targets:
                while True:
                    n += 1
                    if cube.step(s, a_next=float(a_next)) or n > 20 * req.steps:
                        break
            xip = cube.power_spectrum(log_bins=True)
            pk = xip[:self.max_bins, 1:3].copy()
            xp, _, _, rhoc, _ = cube.store_state()
            pos = positions(xp, rhoc, sp.nc, _nnt(sp.nc), sp.izip)
            return Answer(req.rid, pk, pos[::self.subsample].copy(), n)
        finally:
            self._release(sp.nc, cube)

    # ---- a stream ------------------------------------------------------------
    def serve(self, requests: list[Request], realtime: bool = True) -> list[Answer]:
        """Serves the requests in arrival order (waiting for each arrival time when
        realtime) and returns their answers with wait, service and latency."""
        queue = deque()
        answers = {}
        err = []
        done = threading.Event()
        cv = threading.Condition()
        t0 = time.perf_counter()

        def feeder():
            for r in requests:
                if realtime:
                    dt = r.arrival - (time.perf_counter() - t0)
                    if dt > 0:
                        time.sleep(dt)
                with cv:
                    queue.append(r)
                    cv.notify()
            with cv:
                done.set()
                cv.notify_all()

        def worker():
            while True:
                with cv:
                    while not queue and not done.is_set():
                        cv.wait()
                    if not queue:
                        return
                    r = queue.popleft()
                start = time.perf_counter() - t0
                try:
                    a = self.answer(r)
                except Exception as e:
                    err.append(e)
                    return
                end = time.perf_counter() - t0
                arrival = r.arrival if realtime else 0.0
                a.wait, a.service, a.latency = start - arrival, end - start, end - arrival
                answers[r.rid] = a

        threads = [threading.Thread(target=feeder)] + [threading.Thread(target=worker) for _ in range(self.workers)]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        if err:
            raise err[0]
        return [answers[r.rid] for r in requests]
