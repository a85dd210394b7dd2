"""Power spectrum on the GPU (cicpower.f90 + powerspectrum.f90) against the numpy
restatement in pk_ref.py; the restatement itself is pinned on CPU by a plane
wave of known amplitude."""
import numpy as np
import pytest

from cube_nufluid_b200 import Cube, ic
from helpers import nu_params, small_state
from pk_ref import cic_delta, cross_power, nu_delta, particle_positions


def test_plane_wave_power_lands_in_its_bin():
    # delta = A cos(2 pi m x / ng): one mode pair of |c| = A/2, Delta^2 = (A/2)^2 4 pi m^3 / sinc^4 / N(bin)
    ng, m, A = 32, 5, 0.1
    x = np.arange(ng)
    d = np.broadcast_to(A * np.cos(2 * np.pi * m * x / ng)[None, None, :], (ng, ng, ng)).copy()
    xi = cross_power(d, None, box=100.0)
    b = m - 1  # bin m (nint(|k|) = m) is row m-1
    sinc = np.sin(np.pi * m / ng) / (np.pi * m / ng)
    expect = (A / 2) ** 2 * 4 * np.pi * m ** 3 / sinc ** 4 / xi[b, 0]
    assert xi[b, 2] == pytest.approx(expect, rel=1e-9)
    others = np.delete(xi[:, 2], b)
    assert np.nanmax(np.abs(others)) < 1e-20


def test_lattice_positions_round_trip():
    st, _, _ = small_state(nc=8, nnt=2, seed=3)
    pos = particle_positions(st)
    assert pos.shape == (st.np, 3) and np.all(pos >= 0) and np.all(pos < 8)


@pytest.mark.gpu
@pytest.mark.parametrize("log_bins", [False, True])
def test_gpu_power_spectrum_matches_restatement(tables, log_bins):
    st, p, s = small_state(nc=16, nnt=2, box=200.0, seed=9, amplitude=4.0)
    fk, ck = tables
    g = Cube(p, np_capacity=st.np, fk_table=fk, ck_table=ck)
    g.load_state(st.xp, st.vp, st.pid, st.rhoc, st.vfield)
    got = g.power_spectrum(log_bins)
    ref = cross_power(cic_delta(particle_positions(st), 16, 64), None, box=200.0, log_bins=log_bins)
    assert got.shape == ref.shape
    assert np.array_equal(got[:, 0], ref[:, 0].astype(np.float32))
    ok = ref[:, 0] > 0
    np.testing.assert_allclose(got[ok, 1], ref[ok, 1], rtol=1e-6)
    np.testing.assert_allclose(got[ok, 2], ref[ok, 2], rtol=2e-4)
    np.testing.assert_allclose(got[ok, 5:7], ref[ok, 5:7], rtol=1e-5)


@pytest.mark.gpu
@pytest.mark.parametrize("nc", [24, 48])
def test_gpu_power_spectrum_radix3_meshes(tables, nc):
    # nf = 96 and 192: the forward transform with a radix-3 first stage
    st, p, s = small_state(nc=nc, nnt=2, box=200.0, seed=19, amplitude=4.0)
    fk, ck = tables
    g = Cube(p, np_capacity=st.np, fk_table=fk, ck_table=ck)
    g.load_state(st.xp, st.vp, st.pid, st.rhoc, st.vfield)
    got = g.power_spectrum(True)
    ref = cross_power(cic_delta(particle_positions(st), nc, 4 * nc), None, box=200.0, log_bins=True)
    assert got.shape == ref.shape
    ok = ref[:, 0] > 0
    np.testing.assert_allclose(got[ok, 2], ref[ok, 2], rtol=2e-4)


@pytest.mark.gpu
def test_gpu_cross_power_with_neutrinos(tables):
    st, _, s = small_state(nc=16, nnt=2, box=300.0, seed=13, amplitude=2.0)
    p = nu_params(nc=16, nnt=2, box=300.0)
    fk, ck = tables
    g = Cube(p, np_capacity=st.np, fk_table=fk, ck_table=ck)
    g.load_state(st.xp, st.vp, st.pid, st.rhoc, st.vfield)
    info = g.nu_info()
    fl = [ic.nu_fluid_perturbed(int(info["nc"][k]), 61 + k, cs2=float(info["cs2"][k])) for k in range(3)]
    for k in range(3):
        g.nu_load(k, fl[k])
    got = g.power_spectrum()
    ref = cross_power(cic_delta(particle_positions(st), 16, 64), nu_delta(fl, info["dwgts"], 64), box=300.0)
    ok = ref[:, 0] > 0
    np.testing.assert_allclose(got[ok, 2], ref[ok, 2], rtol=2e-4)
    # The neutrino field is band-limited: above half the Nyquist frequency its power is
    # the FP32 rounding of delta_nu = rho - 1 (~6e-8 per cell, as the reference's real
    # rho_nu), times the CDM shot noise and the sinc^-4 window, which the FP64
    # restatement does not have.  Compare the neutrino terms where the field has power.
    low = ok & (np.arange(len(ref)) + 1 < 16)
    for q in (3, 4):
        np.testing.assert_allclose(got[low, q], ref[low, q], rtol=2e-4, atol=1e-4 * np.abs(ref[low, q]).max())
