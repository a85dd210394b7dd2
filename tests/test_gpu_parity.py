"""GPU parity tests: the CUDA library through its C-ABI against the CPU oracle.

Bars: integer deposit, positions and velocity
re-quantisation bit-exact; forces within FP32 tolerance of the FP64-FFT oracle
(relative RMS <= 1e-5).  Sizes are small enough for the oracle to finish in
seconds; crowded cells come from the clustered test state.
"""
import numpy as np
import pytest

from helpers import clustered_state, first_step_scalars, kick_chain, rel_rms, small_state
from oracle_ref import Oracle
from cube_nufluid_b200 import Cube
from cube_nufluid_b200.abi import make_params

pytestmark = pytest.mark.gpu

FORCE_TOL = 1e-5   # relative RMS, FP32 FFT vs FP64 oracle


def pair(st, p, tables, build=True):
    fk, ck = tables
    o = Oracle(p, fk, ck, build_kernels=build)
    o.load(st.xp, st.vp, st.pid, st.rhoc, st.vfield)
    g = Cube(p, np_capacity=st.np + 1024, fk_table=fk, ck_table=ck)
    g.load_state(st.xp, st.vp, st.pid, st.rhoc, st.vfield)
    return o, g


def assert_same_state(o, g):
    a = o.store()
    b = g.store_state()
    for name, x, y in zip(("xp", "vp", "pid", "rhoc", "vfield"), a, b):
        assert x.shape == y.shape, name
        if x.dtype.kind == "f":
            assert np.array_equal(x.view(np.int32), y.view(np.int32)), name
        else:
            nbad = int(np.count_nonzero(x != y))
            assert nbad == 0, f"{name}: {nbad} entries differ"


@pytest.mark.parametrize("kind,izip", [("smooth", 2), ("clustered", 2), ("clustered", 1)])
def test_update_x_bit_exact(tables, kind, izip):
    if kind == "smooth":
        st, p, s = small_state(nc=16, nnt=2, seed=21, izipx=izip, izipv=izip, amplitude=8.0)
        s.dt_old, s.dt = 2.0, 2.0
    else:
        st, p, s = clustered_state(nc=16, nnt=2, seed=22, izipx=izip, izipv=izip)
        s.dt_old, s.dt = 60.0, 60.0
    o, g = pair(st, p, tables, build=False)
    so, sg = s.copy(), s.copy()
    o.update_x(so)
    g.update_x(sg)
    assert so.nlayer == sg.nlayer and so.nlayer >= 3
    assert_same_state(o, g)
    assert so.sigma_vi_new == sg.sigma_vi_new
    assert so.std_vsim == sg.std_vsim and so.std_vsim_c == sg.std_vsim_c and so.std_vsim_res == sg.std_vsim_res
    # particles did move between cells
    assert not np.array_equal(g.store_state()[3], st.rhoc)


@pytest.fixture(scope="module")
def pm_pair(tables):
    st, p, s = clustered_state(nc=16, nnt=2, seed=31)
    o, g = pair(st, p, tables)
    s.a, s.a_mid, s.dt = 0.5, 0.5, 20.0
    so, sg = s.copy(), s.copy()
    o.particle_mesh(so, 1)
    g.particle_mesh(sg)
    return st, p, s, o, g, so, sg


def test_deposit_bit_exact(pm_pair, tables):
    st, p, s, o, g, so, sg = pm_pair
    g2 = Cube(p, np_capacity=st.np, fk_table=tables[0], ck_table=tables[1])
    g2.load_state(st.xp, st.vp, st.pid, st.rhoc, st.vfield)
    sd = s.copy()
    g2.debug_deposit(sd)
    assert np.array_equal(o.fetch(0).view(np.int32), g2.fetch(0).view(np.int32))
    assert np.array_equal(o.fetch(1).view(np.int32), g2.fetch(1).view(np.int32))
    # the oracle sums the FP32-rounded nodes, the GPU the exact fixed-point integers
    assert so.testrhoc == pytest.approx(sd.testrhoc, rel=1e-7)
    assert sd.testrhof == pytest.approx(st.np * st.mass_p_cdm, rel=1e-9)


def test_deposit_bit_exact_after_a_smooth_drift(tables):
    # after a re-bin that leaves no cell beyond 32 particles the deposit launches one
    # block per brick without work items
    st, p, s = small_state(nc=16, nnt=2, seed=23, amplitude=8.0)
    s.dt_old, s.dt = 2.0, 2.0
    o, g = pair(st, p, tables)
    so, sg = s.copy(), s.copy()
    o.update_x(so)
    g.update_x(sg)
    assert g.store_state()[3].max() <= 32
    so.a, so.a_mid, so.dt = 0.5, 0.5, 20.0
    sg.a, sg.a_mid, sg.dt = 0.5, 0.5, 20.0
    o.particle_mesh(so, 1)
    g.debug_deposit(sg)
    assert np.array_equal(o.fetch(0).view(np.int32), g.fetch(0).view(np.int32))
    assert np.array_equal(o.fetch(1).view(np.int32), g.fetch(1).view(np.int32))


def test_deposit_bit_exact_on_dense_clumps(tables):
    # cells of 12,000 and 24,000 particles: thousands of weights collide on the same
    # shared-memory nodes and the 64-bit node sums (~1e14 in fixed point) carry out of
    # their low words many times
    from cube_nufluid_b200 import ic
    from cube_nufluid_b200.cube import scalars_from_ic
    rng = np.random.Generator(np.random.Philox(43))
    parts = [rng.uniform(0, 16, (20000, 3))]
    for c, n, sig in (((3.5, 4.5, 5.5), 12000, 0.08), ((10.5, 11.5, 2.5), 12000, 0.08), ((8.5, 8.5, 12.5), 24000, 0.02)):
        parts.append(np.asarray(c) + rng.normal(0, sig, (n, 3)))
    x = np.mod(np.concatenate(parts), 16.0)
    st = ic.pack(x, rng.normal(0, 0.02, x.shape), 16, 2, a=0.5, box=100.0)
    p = make_params(16, 2, box=100.0)
    s = scalars_from_ic(st)
    assert st.rhoc.max() > 20000
    o, g = pair(st, p, tables)
    s.a, s.a_mid, s.dt = 0.5, 0.5, 20.0
    so, sd = s.copy(), s.copy()
    o.particle_mesh(so, 1)
    g.debug_deposit(sd)
    assert np.array_equal(o.fetch(0).view(np.int32), g.fetch(0).view(np.int32))
    assert np.array_equal(o.fetch(1).view(np.int32), g.fetch(1).view(np.int32))
    assert sd.testrhof == pytest.approx(st.np * st.mass_p_cdm, rel=1e-9)


def test_forces_match_fp64_oracle(pm_pair):
    st, p, s, o, g, so, sg = pm_pair
    # the library's meshes hold force*a_mid*dt/6/pi; compare against the same chain
    # applied to the oracle's forces
    assert rel_rms(g.fetch(2), kick_chain(o.fetch(2), sg.a_mid, sg.dt)) <= FORCE_TOL
    assert rel_rms(g.fetch(3), kick_chain(o.fetch(3), sg.a_mid, sg.dt)) <= FORCE_TOL
    assert sg.f2_max_fine == pytest.approx(so.f2_max_fine, rel=1e-4)
    assert sg.f2_max_coarse == pytest.approx(so.f2_max_coarse, rel=1e-4)


def decode(codes, sigma, izipv=2):
    """Velocity decode of pm.f90:145 in numpy (FP32 argument and tan, FP64 divide)."""
    nvbin = 1 << (8 * izipv)
    pif = np.float32(4.0) * np.arctan(np.float32(1.0))
    arg = (pif * codes.astype(np.float32)) / np.float32(nvbin - 1)
    coef = float(np.sqrt(pif / np.float32(2.0))) / (float(np.float32(sigma)) * 2.5)
    return np.tan(arg).astype(np.float64) / coef


def test_kicked_velocities_close(pm_pair):
    st, p, s, o, g, so, sg = pm_pair
    vo = o.store()[1].astype(np.int32)
    vg = g.store_state()[1].astype(np.int32)
    # FP32 (GPU) vs FP64 (oracle) forces: the codes agree except where the force
    # difference crosses a rounding boundary; in velocity the difference is bounded
    # by the force tolerance times the kick, plus one code step either side
    assert np.mean(vo != vg) < 5e-3
    v_o, v_g = decode(vo, so.sigma_vi), decode(vg, so.sigma_vi)
    v0 = decode(st.vp.astype(np.int32), s.sigma_vi)
    kick = np.sqrt(np.mean((v_o - v0) ** 2))
    step = np.abs(decode(vo + 1, so.sigma_vi) - decode(vo - 1, so.sigma_vi))
    ok = np.abs(v_o - v_g) <= 1e-4 * kick + step
    assert ok[np.abs(vo) < 32700].all()
    assert sg.dt_fine == pytest.approx(so.dt_fine, rel=1e-4)
    assert sg.dt_coarse == pytest.approx(so.dt_coarse, rel=1e-4)
    assert sg.sigma_vi == so.sigma_vi


@pytest.mark.parametrize("izip", [2, 1])
def test_kick_bit_exact_on_identical_forces(tables, izip):
    st, p, s = clustered_state(nc=16, nnt=2, seed=41, izipx=izip, izipv=izip)
    o, g = pair(st, p, tables, build=False)
    s.a, s.a_mid, s.dt = 0.5, 0.5, 20.0
    s.sigma_vi_new = np.float32(s.sigma_vi * 1.01)
    rng = np.random.default_rng(9)
    nf, nc = 64, 16
    fine = rng.normal(0, 2.0, 3 * nf ** 3).astype(np.float32)
    coarse = rng.normal(0, 0.5, 3 * nc ** 3).astype(np.float32)
    so, sg = s.copy(), s.copy()
    o.particle_mesh_with_force(so, fine, coarse, 1)
    g.kick_with_force(sg, fine, coarse)
    assert_same_state(o, g)
    assert list(so.vmax) == list(sg.vmax)


def test_kick_bit_exact_on_cells_beyond_one_work_item(tables):
    # cells of 12,000 particles: the kick's work items cut their 64-cell groups into
    # runs of cells and the crowded cells into slices of 4096 particles
    from helpers import planted_clumps
    st, p, s = planted_clumps(nc=16, centres=((3.5, 4.5, 5.5), (10.5, 11.5, 2.5)), n_per=12000, sigma=0.08,
                              nbg=20000, seed=45)
    assert st.rhoc.max() > 2 * 4096  # three slices
    o, g = pair(st, p, tables, build=False)
    s.a, s.a_mid, s.dt = 0.5, 0.5, 20.0
    s.sigma_vi_new = np.float32(s.sigma_vi * 1.01)
    rng = np.random.default_rng(10)
    nf, nc = 64, 16
    fine = rng.normal(0, 2.0, 3 * nf ** 3).astype(np.float32)
    coarse = rng.normal(0, 0.5, 3 * nc ** 3).astype(np.float32)
    so, sg = s.copy(), s.copy()
    o.particle_mesh_with_force(so, fine, coarse, 1)
    g.kick_with_force(sg, fine, coarse)
    assert_same_state(o, g)
    assert list(so.vmax) == list(sg.vmax)


@pytest.mark.parametrize("izip", [2, 1])
def test_pp_bit_exact(tables, izip):
    st, p, s = clustered_state(nc=16, nnt=2, seed=51, izipx=izip, izipv=izip)
    p.ext_pp_force = 1
    o, g = pair(st, p, tables, build=False)
    s.a_mid, s.dt = 0.5, 5.0
    so, sg = s.copy(), s.copy()
    o.ext_pp_force(so)
    g.ext_pp_force(sg)
    assert so.itest1 == sg.itest1 == st.np
    assert so.npairs == sg.npairs
    assert so.f2_max_pp == sg.f2_max_pp
    assert so.dt_pp == sg.dt_pp
    assert_same_state(o, g)


def test_pp_division_through_a_shared_reciprocal_is_ieee(tables):
    # the pair term divides three components by one r^3: through RN(1/r^3) and two
    # FMA corrections, which must give the IEEE quotient in every bit
    fk, ck = tables
    st, p, s = small_state(nc=16, nnt=2, seed=5)
    g = Cube(p, np_capacity=st.np, fk_table=fk, ck_table=ck)
    assert g.debug_division_check(1 << 30, 12345) == 0
    g.close()


@pytest.mark.parametrize("z_i,izip", [(30.0, 2), (15.0, 2), (15.0, 1)])
def test_pp_bit_exact_on_a_smooth_state(tables, z_i, izip):
    # Zel'dovich states with no cell beyond 32 particles: at z = 30 almost every
    # brick takes the listed path (most targets alone in their window), at z = 15
    # about a third of the bricks do and the rest go to the staged brick kernel
    st, p, s = small_state(nc=32, nnt=2, z_i=z_i, seed=17, izipx=izip, izipv=izip)
    assert st.rhoc.max() <= 32
    p.ext_pp_force = 1
    o, g = pair(st, p, tables, build=False)
    s.a_mid, s.dt = s.a, 2.0
    so, sg = s.copy(), s.copy()
    o.ext_pp_force(so)
    g.ext_pp_force(sg)
    assert so.itest1 == sg.itest1 == st.np
    assert so.npairs == sg.npairs > 1.02 * st.np   # window entries beyond the targets themselves
    assert so.f2_max_pp == sg.f2_max_pp
    assert so.dt_pp == sg.dt_pp
    assert_same_state(o, g)


def test_fine_green_octant_matches_closed_form(tables):
    from test_oracle import separable_green
    fk, ck = tables
    st, p, s = small_state(nc=16, nnt=2, seed=1)
    g = Cube(p, np_capacity=st.np, fk_table=fk, ck_table=ck)
    nf = 64
    kp = nf // 2 + 1
    got = g.fetch(4).reshape(3, kp, kp, kp).astype(np.float64)      # [d][ky][kx][kz]
    ref = (separable_green(fk, nf) / nf ** 3).transpose(0, 2, 3, 1)  # [d][kz][ky][kx] -> [d][ky][kx][kz]
    assert np.max(np.abs(got - ref)) <= 1e-6 * np.max(np.abs(ref))


@pytest.mark.parametrize("nc", [24, 48])
def test_radix3_mesh_forces(tables, nc):
    # nf = 96 = 24*4 and 192 = 24*8: the register FFT with a radix-3 first stage on
    # the fine mesh; the coarse meshes (24, 48) take the Stockham passes
    st, p, s = clustered_state(nc=nc, nnt=2, npart=60000 * (nc // 24) ** 3, seed=61)
    o, g = pair(st, p, tables)
    s.a, s.a_mid, s.dt = 0.5, 0.5, 20.0
    so, sg = s.copy(), s.copy()
    g.debug_deposit(sg.copy())
    dens = g.fetch(0)
    o.particle_mesh(so, 1)
    g.particle_mesh(sg)
    assert np.array_equal(o.fetch(0).view(np.int32), dens.view(np.int32))
    assert rel_rms(g.fetch(2), kick_chain(o.fetch(2), sg.a_mid, sg.dt)) <= FORCE_TOL
    assert rel_rms(g.fetch(3), kick_chain(o.fetch(3), sg.a_mid, sg.dt)) <= FORCE_TOL


def test_multi_step_run_tracks_oracle(tables):
    # three full steps (timestep, update_x, particle_mesh) on a Zel'dovich box
    st, p, s = small_state(nc=16, nnt=2, seed=71, amplitude=4.0)
    o, g = pair(st, p, tables)
    so, sg = s.copy(), s.copy()
    for _ in range(3):
        first_step_scalars(p, so, 0.0)
        first_step_scalars(p, sg, 0.0)
        assert so.dt == sg.dt
        o.update_x(so)
        g.update_x(sg)
        o.particle_mesh(so, 1)
        g.particle_mesh(sg)
    xo, vo, po, ro, _ = o.store()
    xg, vg, pg, rg, _ = g.store_state()
    # compare per particle by PID: positions to the last code, velocities to one code
    io, ig = np.argsort(po), np.argsort(pg)
    assert np.array_equal(po[io], pg[ig])
    dx = np.abs(xo[io].astype(np.int32) - xg[ig].astype(np.int32))
    dx = np.minimum(dx, 65536 - dx)
    assert np.mean(dx == 0) > 0.99 and dx.max() <= 2
    dv = np.abs(vo[io].astype(np.int32) - vg[ig].astype(np.int32))
    assert np.mean(dv == 0) > 0.99


@pytest.mark.gpu
def test_update_x_bit_exact_with_cells_beyond_the_shared_sorter(tables):
    # two dense clumps put cells of more than 4096 particles through the global-
    # scratch sorter (and others through the shared-memory one)
    from helpers import planted_clumps
    st, p, s = planted_clumps(nc=16, centres=((3.5, 4.5, 5.5), (10.5, 11.5, 2.5)), n_per=12000, sigma=0.08,
                              nbg=20000, seed=41)
    assert st.rhoc.max() > 4096
    s.dt_old, s.dt = 20.0, 20.0
    o, g = pair(st, p, tables, build=False)
    so, sg = s.copy(), s.copy()
    o.update_x(so)
    g.update_x(sg)
    assert_same_state(o, g)
    assert so.sigma_vi_new == sg.sigma_vi_new and so.std_vsim == sg.std_vsim
    assert g.store_state()[3].max() > 4096
