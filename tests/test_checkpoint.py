"""CUBE checkpoint files (checkpoint.f90, particle_initialization.f90, hydrodf.f90)."""
import os

import numpy as np
import pytest

from cube_nufluid_b200 import checkpoint as ck, ic
from cube_nufluid_b200.cube import scalars_from_ic
from helpers import nu_params, small_state


def test_sim_header_layout():
    # 17 integer(8) then 22 real(4) in declaration order (parameters.f90:129-153)
    names = ck.SIM_HEADER.names
    assert names[0] == "nplocal" and names[16] == "cur_halofind" and names[17] == "a" and names[-1] == "vz_max"
    assert ck.SIM_HEADER.fields["a"][1] == 136 and ck.SIM_HEADER.itemsize == 224


def test_file_names_follow_output_name():
    assert ck.z_string(10.0) == "10.000" and ck.z_string(0.0) == "0.000"
    assert ck.file_name("/o/", 10.0, "xp", 3).endswith("image3/10.000_xp_3.bin")


def test_particle_checkpoint_round_trip(tmp_path):
    st, p, s = small_state(nc=16, nnt=2, seed=11)
    s.timestep, s.t, s.tau = 7, 1.5, 2.5
    h = ck.make_header(p, s, cur_checkpoint=2)
    files = ck.write(str(tmp_path), 10.0, ck.Checkpoint(h, st.xp, st.vp, st.rhoc, st.vfield, st.pid))
    assert len(files) == 6
    assert os.path.getsize(files[0]) == 224
    assert os.path.getsize(files[1]) == st.xp.nbytes
    r = ck.read(str(tmp_path), 10.0)
    for a, b in ((r.xp, st.xp), (r.vp, st.vp), (r.rhoc, st.rhoc), (r.vfield, st.vfield), (r.pid, st.pid)):
        assert np.array_equal(np.asarray(a), np.asarray(b))
    s2 = ck.scalars_from_header(r.header, 10.0)
    assert s2.a == pytest.approx(1 / 11, rel=1e-7) and s2.sigma_vi == np.float32(s.sigma_vi)
    assert s2.mass_p_cdm == np.float32(s.mass_p_cdm) and s2.timestep == 7 and s2.nplocal == st.np


def test_fluid_checkpoint_halo_and_round_trip(tmp_path):
    n, ncb = 8, 4
    fl = ic.nu_fluid_perturbed(n, 3, cs2=0.5)
    path = str(tmp_path / "neu1.bin")
    ck.write_fluid(path, 0.1, 5.0 / 3.0, [0.2, 0.5, 0.3], [fl, fl[::2, ::2, ::2], fl[::4, ::4, ::4]], [ncb, 4, 4])
    h, out = ck.read_fluid(path, [n, n // 2, n // 4], [ncb, 4, 4])
    assert h["iso"] == 1 and np.isclose(h["m"], 0.1)
    assert np.array_equal(out[0], fl)
    ext = ck.add_halo(fl, ncb)
    assert ext.shape == (n + 2 * ncb,) * 3 + (5,)
    # halo cells are the periodic images (hg_buffer)
    assert np.array_equal(ext[0, ncb, ncb], fl[n - ncb, 0, 0])
    assert np.array_equal(ext[n + 2 * ncb - 1, ncb, ncb], fl[ncb - 1, 0, 0])


@pytest.mark.gpu
def test_gpu_checkpoint_resume_is_exact(tables, tmp_path):
    # step, checkpoint, restore into a new context: the states are identical and the
    # next step from either is identical
    from cube_nufluid_b200 import Cube
    st, _, s = small_state(nc=16, nnt=2, box=300.0, seed=21, amplitude=2.0)
    p = nu_params(nc=16, nnt=2, box=300.0)
    fk, cc = tables
    g = Cube(p, np_capacity=st.np + 1024, fk_table=fk, ck_table=cc)
    g.load_state(st.xp, st.vp, st.pid, st.rhoc, st.vfield)
    info = g.nu_info()
    for k in range(3):
        g.nu_load(k, ic.nu_fluid_perturbed(int(info["nc"][k]), 70 + k, cs2=float(info["cs2"][k])))
    s.a = 0.3
    g.step(s)
    ck.save(g, s, str(tmp_path), 1.0 / s.a - 1.0)
    h = Cube(p, np_capacity=st.np + 1024, fk_table=fk, ck_table=cc)
    s2 = ck.restore(h, str(tmp_path), 1.0 / s.a - 1.0)
    for a, b in zip(g.store_state(), h.store_state()):
        assert np.array_equal(np.asarray(a), np.asarray(b))
    for k in range(3):
        assert np.array_equal(g.nu_store(k), h.nu_store(k))
    assert s2.sigma_vi == np.float32(s.sigma_vi) and s2.mass_p_cdm == np.float32(s.mass_p_cdm)


def test_corrupted_checkpoints_are_refused(tmp_path):
    st, p, s = small_state(nc=16, nnt=2, seed=12)
    h = ck.make_header(p, s)
    files = ck.write(str(tmp_path), 5.0, ck.Checkpoint(h, st.xp, st.vp, st.rhoc, st.vfield, st.pid))
    info, xpf = files[0], files[1]
    good = open(info, "rb").read()
    # a truncated header
    open(info, "wb").write(good[:200])
    with pytest.raises(ValueError, match="info"):
        ck.read(str(tmp_path), 5.0)
    # a header whose particle count does not match the array files
    bad = np.frombuffer(good, dtype=ck.SIM_HEADER).copy()
    bad["nplocal"] += 1
    open(info, "wb").write(bad.tobytes())
    with pytest.raises(ValueError, match="xp"):
        ck.read(str(tmp_path), 5.0)
    # an impossible code width
    bad = np.frombuffer(good, dtype=ck.SIM_HEADER).copy()
    bad["izipx"] = 3
    open(info, "wb").write(bad.tobytes())
    with pytest.raises(ValueError, match="header"):
        ck.read(str(tmp_path), 5.0)
    # a truncated position file
    open(info, "wb").write(good)
    data = open(xpf, "rb").read()
    open(xpf, "wb").write(data[:-6])
    with pytest.raises(ValueError, match="xp"):
        ck.read(str(tmp_path), 5.0)
    open(xpf, "wb").write(data)
    assert ck.read(str(tmp_path), 5.0).xp.shape == st.xp.shape
