"""The precision study's loop in bench.py (run_precision), on CPU with a recording
stand-in for Cube: the FP32 and FP64 runs take whole steps in the order of Cube.step
(timestep, update_x, ext_pp_force, particle_mesh), neither is read or reloaded in the
middle of a step, and the force probe runs on a third context in the FP64 mode that
takes the FP32 run's state between steps with the scalars that step started from."""
import json
import os
import sys
import types

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

STEP = ["timestep", "update_x", "ext_pp_force", "particle_mesh"]
BETWEEN = {"store_state", "fetch2", "fetch3"}  # allowed only after a whole step


class RecordingCube:
    made = []

    def __init__(self, p, cap, *tables):
        self.p = p
        self.calls = []
        self.scale = None
        RecordingCube.made.append(self)

    def load_state(self, xp, vp, pid, rhoc, vfield):
        self.calls.append("load_state")
        self.state = (xp.copy(), vp.copy(), pid.copy(), rhoc.copy(), vfield.copy())

    def store_state(self):
        self.calls.append("store_state")
        return tuple(a.copy() for a in self.state)

    def timestep(self, s, a_next):
        self.calls.append("timestep")
        s.dt = float(a_next) - s.a
        s.a_mid = s.a + s.dt / 2
        s.a = float(a_next)
        return True

    def update_x(self, s):
        self.calls.append("update_x")

    def ext_pp_force(self, s):
        self.calls.append("ext_pp_force")

    def particle_mesh(self, s):
        self.calls.append("particle_mesh")
        # the meshes hold force * ((a_mid dt)/6)/pi in the context's precision
        if self.p.poisson_fp64:
            self.scale = ((s.a_mid * s.dt) / 6.0) / float(np.float32(np.pi))
        else:
            self.scale = float(np.float32(np.float32(np.float32(s.a_mid) * np.float32(s.dt)) / np.float32(6.0))
                               / np.float32(np.pi))
        s.sigma_vi = s.sigma_vi_new

    def fetch(self, which):
        self.calls.append(f"fetch{which}")
        base = np.linspace(-1.0, 1.0, 3 * 8 ** 3) * (1.0 + which)
        return base * self.scale if self.p.poisson_fp64 else (base * self.scale).astype(np.float32)

    def power_spectrum(self, log_bins=False):
        self.calls.append("power_spectrum")
        out = np.zeros((6, 10), np.float32)
        out[:, 0] = 10.0
        out[:, 1] = np.geomspace(0.01, 1.0, 6)
        out[:, 2] = 100.0
        return out

    def close(self):
        self.calls.append("close")


def _state(n=512, nc=8):
    st = types.SimpleNamespace()
    st.np = n
    st.xp = np.zeros((n, 3), np.int16)
    st.vp = np.zeros((n, 3), np.int16)
    st.pid = np.arange(1, n + 1, dtype=np.int32)
    st.rhoc = np.full(nc ** 3, n // nc ** 3, np.int32)
    st.vfield = np.zeros((nc ** 3, 3), np.float32)
    st.a, st.sigma_vi, st.mass_p_cdm, st.vsim2phys = 0.02, 1.0, 8.0, 1.0
    st.vmax = np.ones(3, np.float32)
    return st


@pytest.fixture
def study(monkeypatch, capsys):
    import torch
    import bench
    import cube_nufluid_b200
    import cube_nufluid_b200.build as cbuild
    RecordingCube.made = []
    monkeypatch.setattr(cube_nufluid_b200, "Cube", RecordingCube)
    monkeypatch.setattr(cbuild, "build", lambda *a, **k: None)
    monkeypatch.setattr(torch.cuda, "set_device", lambda *a, **k: None)
    monkeypatch.setattr(bench, "make_state", lambda cfg, seed: _state())
    cfg = dict(nc=8, nnt=2, box=100.0, izip=2, pp=True, z_i=49.0, precision=8, workload="harness check")
    bench.run_precision(types.SimpleNamespace(), cfg)
    line = json.loads(capsys.readouterr().out.strip().splitlines()[-1])
    return RecordingCube.made, line


def _steps(calls):
    """The calls of a lockstep run between its first load and its final P(k) reads,
    checked to be whole steps with reads only between them; returns the step count."""
    body = calls[1:]
    n = 0
    i = 0
    while i < len(body) and body[i] == "timestep":
        assert body[i:i + 4] == STEP, body[i:i + 4]
        i += 4
        n += 1
        while i < len(body) and body[i] in BETWEEN:
            i += 1
    return n, body[i:]


def test_lockstep_runs_take_whole_steps_and_are_never_reloaded_mid_step(study):
    made, line = study
    g32, g64, gp = made
    assert not g32.p.poisson_fp64 and g64.p.poisson_fp64 and gp.p.poisson_fp64
    assert g32.calls[0] == g64.calls[0] == "load_state"
    n32, tail32 = _steps(g32.calls)
    n64, tail64 = _steps(g64.calls)
    assert n32 == n64 == line["steps"] == 8
    # the FP64 run is read once, after its last step (its state for P(k)), and never loaded again
    assert tail64 == ["close"]
    assert g64.calls[-2:] == ["store_state", "close"] and g64.calls.count("store_state") == 1
    assert g64.calls.count("load_state") == 1
    assert tail32 == ["power_spectrum", "load_state", "power_spectrum", "close"]


def test_force_probe_runs_on_its_own_context_with_the_step_scalars(study):
    made, line = study
    gp = made[2]
    probes = len(line["force_rms_rel_err"])
    assert probes == 5
    assert gp.calls == ["load_state", "particle_mesh", "fetch2", "fetch3"] * probes + ["close"]
    for r in line["force_rms_rel_err"]:
        # the stand-in's meshes differ only by the FP32 rounding of the kick scale
        assert r["fine"] < 1e-6 and r["coarse"] < 1e-6
    assert line["pk"]["max_abs_dev"] == 0.0
