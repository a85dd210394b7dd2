"""Run-time halo finder (halofind.f90:18-598): the CPU oracle against planted clumps,
a numpy restatement of its density-peak stage and a brute-force radius search;
the catalogue files; and cube_halofind on the GPU against the oracle (same peaks,
halos, member PIDs and hid; properties to FP64-summation rounding)."""
import ctypes as C
import math

import numpy as np
import pytest

from cube_nufluid_b200 import Cube, checkpoint, ic
from cube_nufluid_b200.abi import CubeHaloArgs, CubeHaloResult, HALO_DTYPE, make_params
from cube_nufluid_b200.cube import scalars_from_ic
from helpers import particle_positions, planted_clumps
from oracle_ref import Oracle

PI_F = float(np.float32(4.0) * np.arctan(np.float32(1.0)))


def oracle_for(st, p, tables):
    fk, ck = tables
    o = Oracle(p, fk, ck, build_kernels=False)
    o.load(st.xp, st.vp, st.pid, st.rhoc, st.vfield)
    return o


def numpy_peak_count(pos, nf, mass, den_odc=200.0, rmax=16):
    """Density peaks of halofind.f90:144-197 restated with numpy: fixed-point CIC at
    pos - 1/2, local maxima above 100, m_mesh over whole shells, m_mesh > 50 masses."""
    fix = 2.0 ** 32
    p = pos - 0.5
    f = np.floor(p)
    w1 = (f + 1.0) - p
    w2 = 1.0 - w1
    i1 = f.astype(np.int64)
    acc = np.zeros(nf ** 3, np.int64)
    for c in range(8):
        o = np.array([c & 1, (c >> 1) & 1, c >> 2])
        w = np.where(o[0], w2[:, 0], w1[:, 0]) * np.where(o[1], w2[:, 1], w1[:, 1])
        w = w * np.where(o[2], w2[:, 2], w1[:, 2])
        idx = (i1 + o) % nf
        np.add.at(acc, (idx[:, 2] * nf + idx[:, 1]) * nf + idx[:, 0], np.rint(w * fix).astype(np.int64))
    rho = acc.reshape(nf, nf, nf)
    unit = mass / fix
    nb = np.stack([np.roll(rho, (dz, dy, dx), axis=(0, 1, 2)) for dz in (-1, 0, 1) for dy in (-1, 0, 1)
                   for dx in (-1, 0, 1)])
    is_peak = (rho >= nb.max(axis=0)) & (rho * unit > 100.0)
    r = np.arange(-rmax, rmax + 1)
    gx, gy, gz = np.meshgrid(r, r, r, indexing="ij")
    r2 = (gx ** 2 + gy ** 2 + gz ** 2).ravel()
    keep = r2 <= rmax * rmax
    order = np.argsort(r2[keep], kind="stable")
    off = np.stack([gx.ravel()[keep], gy.ravel()[keep], gz.ravel()[keep]], axis=1)[order]
    r2s = r2[keep][order]
    count = 0
    for z, y, x in zip(*np.nonzero(is_peak)):
        vals = rho[(z + off[:, 2]) % nf, (y + off[:, 1]) % nf, (x + off[:, 0]) % nf]
        csum = np.cumsum(vals)
        m = csum[-1]
        for i in range(len(vals)):
            if i + 1 < len(vals) and r2s[i + 1] == r2s[i]:
                continue
            if i + 1 >= 19 and csum[i] * unit / (i + 1) < den_odc:
                m = csum[i]
                break
        count += int(m * unit > mass * 50.0)
    return count


def test_oracle_finds_the_planted_clumps(tables):
    st, p, s = planted_clumps()
    o = oracle_for(st, p, tables)
    halos, mem, hid, npeak = o.halofind(s, hid_len=st.np)
    centres = 4.0 * np.array([(3.0, 4.0, 5.0), (11.0, 9.5, 3.0), (6.5, 12.0, 12.5), (14.5, 2.0, 9.0)])
    assert len(halos) == 4 and npeak >= 4
    for h in halos:
        d = h["hpos"] - centres
        d -= 64.0 * np.round(d / 64.0)
        assert np.min(np.linalg.norm(d, axis=1)) < 1.0
        assert 1000 <= h["mass_odc"] <= 3200
        assert 1.5 < h["radius_odc"] < 4.0
    # densest first: the halos come out in order of their peak, each particle once
    assert len(mem) == int(halos["mass_odc"].sum()) and np.unique(mem).size == len(mem)
    off = 0
    for k, h in enumerate(halos):
        n = int(h["mass_odc"])
        assert np.all(hid[mem[off:off + n] - 1] == k + 1)
        off += n
    assert int((hid > 0).sum()) == len(mem)


def test_oracle_peak_stage_matches_numpy(tables):
    st, p, s = planted_clumps(n_per=1500, sigma=0.35, nbg=30000, seed=9)
    o = oracle_for(st, p, tables)
    _, _, _, npeak = o.halofind(s)
    pos = particle_positions(st, 16, 2)
    assert npeak == numpy_peak_count(pos, 64, float(s.mass_p_cdm))
    assert npeak >= 4


def test_oracle_first_halo_radius_matches_brute_force(tables):
    st, p, s = planted_clumps(seed=7)
    o = oracle_for(st, p, tables)
    halos, _, _, _ = o.halofind(s)
    h = halos[0]
    pos = particle_positions(st, 16, 2)
    d = pos - h["hpos"].astype(np.float64)
    d -= 64.0 * np.round(d / 64.0)
    r = np.sort(np.linalg.norm(d, axis=1))
    ii = np.arange(1, len(r) + 1)
    den = 0.75 / PI_F * ii * float(s.mass_p_cdm) / r ** 3
    first = int(np.nonzero((den < 200.0) & (ii >= 2))[0][0]) + 1  # 1-based ii
    assert abs(int(h["mass_odc"]) - (first - 1)) <= 1
    r1, r2 = r[first - 2], r[first - 1]
    d1, d2 = math.log10(den[first - 2]), math.log10(den[first - 1])
    lo = math.log10(200.0)
    expect = 10 ** (((lo - d2) * math.log10(r1) + (d1 - lo) * math.log10(r2)) / (d1 - d2))
    assert h["radius_odc"] == pytest.approx(expect, rel=2e-3)
    # the moments of the halo's particles, recomputed from the member positions
    assert h["v_disp"] > 0 and np.all(h["var_x"] > 0)


def test_oracle_no_halos_without_peaks(tables):
    rng = np.random.Generator(np.random.Philox(3))
    x = rng.uniform(0, 16, (20000, 3))
    st = ic.pack(x, rng.normal(0, 0.01, x.shape), 16, 2, a=0.5, box=100.0)
    p = make_params(16, 2, box=100.0)
    o = oracle_for(st, p, tables)
    halos, mem, _, npeak = o.halofind(scalars_from_ic(st))
    assert len(halos) == 0 and len(mem) == 0 and npeak == 0


def test_halo_catalogue_files_round_trip(tmp_path, tables):
    st, p, s = planted_clumps()
    o = oracle_for(st, p, tables)
    halos, mem, hid, _ = o.halofind(s, hid_len=64 ** 3)
    files = checkpoint.write_halos(str(tmp_path) + "/", 0.0, halos, mem, hid)
    assert [f.rsplit("/", 1)[1] for f in files] == ["0.000_halo_1.bin", "0.000_halo_pid_1.bin", "0.000_hid_1.bin"]
    head, h2, members = checkpoint.read_halos(str(tmp_path) + "/", 0.0)
    assert head["nhalo"] == head["nhalo_tot"] == len(halos) and head["den_odc"] == 200.0
    assert h2.tobytes() == halos.tobytes() and HALO_DTYPE.itemsize == 42 * 4
    assert np.array_equal(np.concatenate(members), mem)
    assert np.fromfile(files[2], np.int16).size == 64 ** 3


def _compare(hg, ho):
    assert len(hg) == len(ho)
    for f in ("hpos", "mass_odc"):
        assert np.array_equal(hg[f], ho[f]), f
    for f in ("x_mean", "q_mean", "s_mean"):
        np.testing.assert_allclose(hg[f], ho[f], rtol=0, atol=2e-5 * 64, err_msg=f)
    for f in ("radius_odc", "v_disp", "v_mean", "var_x", "ang_mom", "inertia", "inertia_q"):
        a, b = hg[f].astype(np.float64), ho[f].astype(np.float64)
        scale = np.maximum(np.abs(b).max(), 1e-30)
        np.testing.assert_allclose(a, b, rtol=2e-5, atol=2e-6 * scale, err_msg=f)


@pytest.mark.gpu
@pytest.mark.parametrize("izip", [(2, 2), (1, 1), (2, 1)])
def test_gpu_halofind_matches_oracle(tables, izip):
    st, p, s = planted_clumps(izipx=izip[0], izipv=izip[1], seed=11 + izip[0] + 2 * izip[1])
    fk, ck = tables
    g = Cube(p, np_capacity=st.np, fk_table=fk, ck_table=ck)
    g.load_state(st.xp, st.vp, st.pid, st.rhoc, st.vfield)
    hg, mg, idg, ng = g.halofind(s, hid_len=st.np)
    ho, mo, ido, no = oracle_for(st, p, tables).halofind(s, hid_len=st.np)
    assert ng == no and len(hg) == 4
    _compare(hg, ho)
    assert np.array_equal(mg, mo) and np.array_equal(idg, ido)


@pytest.mark.gpu
def test_gpu_halofind_on_an_evolved_box(tables):
    nc, nnt, box = 32, 2, 64.0
    fk, ck = tables
    p = make_params(nc, nnt, box=box)
    g = Cube(p, np_capacity=(2 * nc) ** 3, fk_table=fk, ck_table=ck)
    s = g.make_ic(ic.device_ic_params(ic.Cosmology(), 9.0, nc, box=box), 17)
    for _ in range(400):
        if g.step(s, a_next=1.0):
            break
    assert s.a > 0.3
    hg, mg, idg, ng = g.halofind(s, hid_len=(4 * nc) ** 3)
    xp, vp, pid, rhoc, vf = g.store_state()
    o = Oracle(p, fk, ck, build_kernels=False)
    o.load(xp, vp, pid, rhoc, vf)
    ho, mo, ido, no = o.halofind(s, hid_len=(4 * nc) ** 3)
    assert ng == no and len(hg) >= 3
    _compare(hg, ho)
    assert np.array_equal(mg, mo) and np.array_equal(idg, ido)
    # PIDs are fine-mesh indices of the IC lattice: the Lagrangian means lie near
    # lattice points' region, inside the box
    assert np.all((hg["q_mean"] >= 0) & (hg["q_mean"] < 4 * nc))


@pytest.mark.gpu
def test_gpu_halofind_reports_small_output_arrays(tables):
    st, p, s = planted_clumps()
    fk, ck = tables
    g = Cube(p, np_capacity=st.np, fk_table=fk, ck_table=ck)
    g.load_state(st.xp, st.vp, st.pid, st.rhoc, st.vfield)
    full, _, _, _ = g.halofind(s)
    out = np.zeros(2, HALO_DTYPE)
    a = CubeHaloArgs()
    a.den_odc, a.capacity, a.halos = 200.0, 2, out.ctypes.data
    r = CubeHaloResult()
    rc = g.L.cube_halofind(g.h, C.byref(s), C.byref(a), C.byref(r))
    assert rc == 2 and r.nhalo == len(full) == 4
    assert out.tobytes() == full[:2].tobytes()
