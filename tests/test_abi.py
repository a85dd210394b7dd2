"""CPU tests of the C-ABI library: it loads without a GPU and exports every
entry point that include/cube_gpu.h declares."""
import ctypes as C
import os
import re

import pytest

from cube_nufluid_b200 import build, cube

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            txt = open(os.path.join(ROOT, "include", fn)).read()
            names |= set(re.findall(r"^\s*(?:const\s+)?[\w\s\*]*?\b(cube_\w+)\s*\(", txt, re.M))
    return sorted(names)


def test_library_builds_and_loads():
    build.build()
    L = cube.load_library()
    assert L.cube_abi_version() == 1


def test_every_declared_entry_point_is_exported():
    L = cube.load_library()
    names = declared_symbols()
    assert len(names) >= 15
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_create_rejects_bad_parameters_without_a_gpu():
    from cube_nufluid_b200.abi import make_params
    p = make_params(16, 3)  # nc not divisible by nnt
    L = cube.load_library()
    h = C.c_void_p()
    fk = (C.c_float * (3 * 16 ** 3))()
    ck = (C.c_float * 192)()
    rc = L.cube_create(C.byref(p), 1000, fk, ck, C.byref(h))
    assert rc == 1
    assert b"invalid parameters" in L.cube_last_error(None)


def test_expansion_matches_a_direct_fp64_evaluation():
    from cube_nufluid_b200.abi import make_params
    import math
    p = make_params(16, 2)
    a0, dt0 = 0.02, 0.3
    d1, d2 = cube.expansion(p, a0, dt0)
    # timestep.f90:136-180 evaluated in plain double (FP32 literals aside)
    def half(a, dt):
        om, ol, wde = 0.3, 0.7, -1.0
        a3rlm = a ** (-3 * wde) * ol / om
        arkm = a * (1 - om - ol) / om
        adot = math.sqrt(4 / 9 * a ** 3 * (1 + arkm + a3rlm))
        addot = a * a * 4 / 9 * (1.5 + 2 * arkm + 1.5 * (1 - wde) * a3rlm)
        atdot = a * adot * 4 / 9 * (3 + 6 * arkm + 1.5 * (2 - 3 * wde) * (1 - wde) * a3rlm)
        return adot * dt + addot * dt * dt / 2 + atdot * dt ** 3 / 6
    r1 = half(a0, dt0 / 2)
    r2 = half(a0 + r1, dt0 / 2)
    assert abs(d1 - r1) < 1e-6 * r1 and abs(d2 - r2) < 1e-6 * r2
