"""CPU tests of the particle codec shared by the oracle and the CUDA library.

The velocity code is an arctangent compression (pm.f90:145,154; update_particle.f90:69,119);
the position code is the in-cell fixed point of parameters.f90:14-19.  The only
known-answer data the reference ships for the codec is the round trip of
velocity_conversion/test.f90:33-39.
"""
import ctypes as C
import math

import numpy as np
import pytest

from oracle_ref import Oracle, lib
from cube_nufluid_b200.abi import make_params


@pytest.fixture(scope="module")
def orc16(tables):
    fk, ck = tables
    return Oracle(make_params(16, 2), fk, ck, build_kernels=False)


@pytest.fixture(scope="module")
def orc8(tables):
    fk, ck = tables
    return Oracle(make_params(16, 2, izipx=1, izipv=1), fk, ck, build_kernels=False)


def _ulp_err(a, b):
    return abs(a - b) / math.ulp(b) if b != 0 else abs(a)


def test_project_atan_within_two_ulp():
    rng = np.random.default_rng(7)
    xs = np.concatenate([rng.uniform(-2, 2, 20000), np.sign(rng.uniform(-1, 1, 20000)) * 10 ** rng.uniform(-12, 12, 20000),
                         np.array([0.0, 1.0, -1.0, 0.2679491924311227, 1e300, -1e300])])
    worst = 0.0
    for x in xs:
        worst = max(worst, _ulp_err(lib().orc_atan(float(x)), math.atan(float(x))))
    assert worst <= 2.0, worst


def test_encode_flip_count_against_libm(orc16):
    # the project arctangent and the C library's differ by at most ~2 ulp; a code
    # flips only when nvbin*atan/pi lands within ~1e-11 of a half-integer
    rng = np.random.default_rng(3)
    sigma = np.float32(0.0023)
    vs = rng.normal(0, 3 * float(sigma), 100000)
    flips = sum(lib().orc_vencode(orc16.h, float(v), sigma) != lib().orc_vencode_libm(orc16.h, float(v), sigma)
                for v in vs)
    assert flips == 0


def test_tan_table_is_odd_and_monotone(orc16, orc8):
    for o, nv in ((orc16, 65536), (orc8, 256)):
        t = np.array([lib().orc_tanf_code(o.h, c) for c in range(-nv // 2, nv // 2)], np.float32)
        mid = nv // 2
        # code -nvbin/2 is never produced by the encode (|q| < nvbin/2-1/2); its FP32
        # argument lies just beyond -pi/2, where tan changes sign, as in the reference
        assert np.all(np.diff(t[1:]) > 0)
        assert np.array_equal(t[mid + 1:], -t[mid - 1:0:-1])


def test_tan_table_close_to_correctly_rounded(orc16):
    # the table holds the C library's tanf of the FP32 argument (what gfortran's
    # tan(real) calls); compare with the FP64 tangent rounded to FP32
    pif = np.float32(4.0) * np.arctan(np.float32(1.0))
    codes = np.arange(-32767, 32768)
    args = (pif * codes.astype(np.float32)) / np.float32(65535.0)
    cr = np.tan(args.astype(np.float64)).astype(np.float32)
    t = np.array([lib().orc_tanf_code(orc16.h, int(c)) for c in codes], np.float32)
    diff_ulp = np.abs(t.view(np.int32).astype(np.int64) - cr.view(np.int32).astype(np.int64))
    # glibc's tanf is within 1 ulp (not correctly rounded): the table carries exactly
    # the library's values, which is what the reference's tan(real) returns on this host
    assert diff_ulp.max() <= 1


def test_roundtrip_of_velocity_conversion_test(orc16):
    # velocity_conversion/test.f90:33-39: vtest=5 -> itest -> vtest, here with
    # vrel_boost folded in as in the step (pm.f90:145,154)
    sigma = np.float32(2.0)
    code = lib().orc_vencode(orc16.h, 5.0, sigma)
    back = lib().orc_vdecode(orc16.h, code, sigma)
    # one code step at v: dv = pi/(nvbin-1) * (1+y^2)/coef
    coef = float(np.sqrt(np.float32(np.pi) / 2)) / (float(sigma) * 2.5)
    step = math.pi / 65535 * (1 + (coef * 5) ** 2) / coef
    assert abs(back - 5.0) <= 0.5 * step
    assert 0 < code < 32767


@pytest.mark.parametrize("izip", [1, 2])
def test_position_code_matches_reference_expression(izip):
    # (int(xp+ishift,izipx)+rshift)*x_resolution with the integer(izipx) wrap
    bits = 8 * izip
    ishift = -(2 ** (bits - 1))
    rshift = 0.5 - ishift
    codes = np.arange(-(2 ** (bits - 1)), 2 ** (bits - 1), dtype=np.int64)
    wrapped = ((codes + ishift + 2 ** (bits - 1)) % (2 ** bits)) - 2 ** (bits - 1)
    ref = (wrapped + rshift) * 2.0 ** (-bits)
    ours = ((codes & (2 ** bits - 1)) + 0.5) * 2.0 ** (-bits)
    assert np.array_equal(ref, ours)
    assert ref.min() > 0 and ref.max() < 1


def test_constant_division_is_exact():
    """The force meshes divide by 6 and by pi_f with a precomputed reciprocal and one
    FMA correction (Brisebarre-Muller-Raina); over all 2^32 FP32 inputs it must equal
    IEEE division wherever the library uses it (|x| >= 2^-100)."""
    import ctypes as C
    from oracle_ref import lib
    L = lib()
    L.orc_check_const_div.restype = C.c_int64
    L.orc_check_const_div.argtypes = [C.c_float, C.POINTER(C.c_float)]
    pif = np.float32(4.0) * np.arctan(np.float32(1.0))
    for y in (6.0, float(pif)):
        worst = C.c_float(0.0)
        L.orc_check_const_div(y, C.byref(worst))
        assert worst.value < 2.0 ** -100, (y, worst.value)


@pytest.mark.gpu
@pytest.mark.parametrize("izipv", [2, 1])
def test_gpu_fast_encode_matches_exact(tables, izipv):
    # the reciprocal-based encode used by the kick, PP and re-bin falls back to the
    # exact FP64 encode within 1e-9 of a rounding boundary; it must never disagree
    from cube_nufluid_b200 import Cube
    from cube_nufluid_b200.abi import make_params
    fk, ck = tables
    g = Cube(make_params(16, 2, izipv=izipv), np_capacity=1024, fk_table=fk, ck_table=ck)
    for sigma in (0.00287, 0.05, 1.7):
        assert g.debug_encode_check(1 << 26, 12345, sigma) == 0
