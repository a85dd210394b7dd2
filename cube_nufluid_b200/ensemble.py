"""Ensembles of independent boxes on one GPU.

Each box is its own `Cube` context (its own device state and CUDA stream); a pool
of host threads steps the boxes, so that the kernels of several boxes run on the
GPU at once.  The library's entry points release the interpreter lock while they
run (ctypes foreign calls), and every context synchronises only its own stream,
so boxes do not wait for one another.  A box's result does not depend on which
boxes run beside it: `run(..., workers=1)` and `run(..., workers=k)` give
bit-identical states.

`ensemble_specs` draws boxes as the batched-ensemble workload describes them:
particle counts uniform over {32^3, 48^3, 64^3, 96^3, 128^3} (two particles per
coarse cell per dimension, fine mesh 4x the coarse), box side log-uniform over
50-400 Mpc/h, Omega_m ~ U[0.25, 0.35] (flat), sigma_8 ~ U[0.7, 0.9], one seed per
box, all from one master seed.
"""
from __future__ import annotations

import math
import threading
import time
from dataclasses import dataclass, field

import numpy as np

from . import ic
from .abi import CubeScalars, make_params
from .cube import Cube

PARTICLES_PER_SIDE = (32, 48, 64, 96, 128)


@dataclass
class BoxSpec:
    nc: int              # coarse cells per side (particles per side / 2)
    box: float           # Mpc/h
    omega_m: float
    sigma8: float
    seed: int
    z_i: float = 49.0
    izip: int = 2
    pp: bool = False

    @property
    def particles(self) -> int:
        return (2 * self.nc) ** 3


def ensemble_specs(n: int, master_seed: int, *, sides=PARTICLES_PER_SIDE, box_range=(50.0, 400.0),
                   pp: bool = False) -> list[BoxSpec]:
    """n box specifications drawn reproducibly from master_seed."""
    rng = np.random.Generator(np.random.Philox(master_seed))
    out = []
    for _ in range(n):
        side = int(rng.choice(sides))
        box = float(math.exp(rng.uniform(math.log(box_range[0]), math.log(box_range[1]))))
        out.append(BoxSpec(nc=side // 2, box=box, omega_m=float(rng.uniform(0.25, 0.35)),
                           sigma8=float(rng.uniform(0.7, 0.9)), seed=int(rng.integers(1, 2 ** 62)), pp=pp))
    return out


def _nnt(nc: int) -> int:
    """Tiles per dimension: tiles of at least 8 coarse cells, a multiple of 4."""
    for nnt in (4, 2, 1):
        if nc % nnt == 0 and (nc // nnt) % 4 == 0 and nc // nnt >= 8:
            return nnt
    return 1


@dataclass
class Member:
    spec: BoxSpec
    cube: Cube
    s: CubeScalars
    steps: int = 0
    ms: list = field(default_factory=list)


class Ensemble:
    """Independent boxes, each with its own context and stream on the current GPU."""

    def __init__(self, specs: list[BoxSpec], fk_table=None, ck_table=None):
        self.members = []
        for sp in specs:
            p = make_params(sp.nc, _nnt(sp.nc), box=sp.box, omega_m=sp.omega_m, omega_l=1.0 - sp.omega_m,
                            izipx=sp.izip, izipv=sp.izip, ext_pp_force=sp.pp)
            cube = Cube(p, np_capacity=sp.particles, fk_table=fk_table, ck_table=ck_table)
            cos = ic.Cosmology(omega_m=sp.omega_m, omega_l=1.0 - sp.omega_m, sigma8=sp.sigma8)
            s = cube.make_ic(ic.device_ic_params(cos, sp.z_i, sp.nc, box=sp.box), sp.seed)
            self.members.append(Member(sp, cube, s))

    def run_native(self, steps: int, workers: int = 16) -> dict:
        """Advance every box by `steps` steps on `workers` native threads of the
        library (cube_run_steps: boxes dealt round-robin, each box-step the order of
        Cube.step); returns wall time, box-steps/s and particle-updates/s."""
        import ctypes as C
        n = len(self.members)
        L = self.members[0].cube.L if n else None
        handles = (C.c_void_p * max(n, 1))(*[m.cube.h for m in self.members])
        ios = (CubeScalars * max(n, 1))()
        for i, m in enumerate(self.members):
            C.memmove(C.byref(ios[i]), C.byref(m.s), C.sizeof(CubeScalars))
        failed = C.c_int32(-1)
        t0 = time.perf_counter()
        rc = L.cube_run_steps(handles, ios, n, int(steps), int(workers), C.byref(failed)) if n else 0
        wall = time.perf_counter() - t0
        for i, m in enumerate(self.members):
            C.memmove(C.byref(m.s), C.byref(ios[i]), C.sizeof(CubeScalars))
            m.steps += steps
        if rc:
            if failed.value < 0:
                from .cube import CubeError
                raise CubeError(rc, "cube_run_steps refused its arguments")
            self.members[failed.value].cube._check(rc)
        nsteps = steps * n
        npu = steps * sum(m.spec.particles for m in self.members)
        return {"boxes": n, "steps": steps, "workers": min(workers, max(n, 1)), "wall_s": wall,
                "box_steps_per_s": nsteps / wall, "particle_updates_per_s": npu / wall}

    def run(self, steps: int, workers: int = 8) -> dict:
        """Advance every box by `steps` steps with `workers` host threads (boxes dealt
        round-robin); returns wall time, box-steps/s and particle-updates/s."""
        err = []
        groups = [self.members[i::workers] for i in range(max(1, workers))]

        def work(ms):
            try:
                for _ in range(steps):
                    for m in ms:
                        m.cube.step(m.s)
                        m.steps += 1
            except Exception as e:  # surfaced after the join
                err.append(e)

        threads = [threading.Thread(target=work, args=(g,)) for g in groups if g]
        t0 = time.perf_counter()
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        wall = time.perf_counter() - t0
        if err:
            raise err[0]
        nsteps = steps * len(self.members)
        npu = steps * sum(m.spec.particles for m in self.members)
        return {"boxes": len(self.members), "steps": steps, "workers": len(threads), "wall_s": wall,
                "box_steps_per_s": nsteps / wall, "particle_updates_per_s": npu / wall}

    def states(self):
        """Checkpoint-layout state of every box (xp, vp, pid, rhoc, vfield)."""
        return [m.cube.store_state() for m in self.members]

    def close(self):
        for m in self.members:
            m.cube.close()
        self.members = []
