"""Checkpoints (frame + integrator state) and the asynchronous trajectory
writer. A restored simulation continues the saved trajectory; a restart from
the frame alone (the reference's constructor from a file) does not, because it
loses the box, xi and the barostat state."""
import numpy as np
import pytest

import md_simulation_cuda_b200 as mdb
from md_simulation_cuda_b200 import workloads as wl

pytestmark = pytest.mark.gpu


def _nph_system():
    f, Lx, Ly = wl.lattice_frame(2000, 0.8, 1.0, 0.65, 0.9, seed=31, jitter=0.1)
    return f, wl.config_dict(2000, Lx, Ly, dt=0.002, T=0.9, barostat_mass=10.0)


def test_checkpoint_continues_nph_and_nose_hoover(built, tmp_path):
    f, cfg = _nph_system()
    a = mdb.MDSimulation(cfg, frame=f)
    a.step_single_nose_hoover(nsteps=40)
    a.step_single_NPH(2.0, nsteps=40)
    fp, sp = str(tmp_path / "ck.pframe"), str(tmp_path / "ck.json")
    a.save_checkpoint(fp, 80, sp)
    a.step_single_NPH(2.0, nsteps=30)
    ref = a.get_host_particles()
    b = mdb.MDSimulation(cfg, filename=fp, step=80, state_file=sp)
    assert b.t == pytest.approx(80 * 0.002)
    b.step_single_NPH(2.0, nsteps=30)
    got = b.get_host_particles()
    assert abs(b.get_Lx() - a.get_Lx()) <= 1e-12 * a.get_Lx()
    assert np.max(np.abs(got["pos"] - ref["pos"])) < 1e-8
    # the restored engine sums forces in another order (rounding differences
    # of FP32 pair terms, not lost state): velocities agree to ~1e-7
    assert np.max(np.abs(got["vel"] - ref["vel"])) < 1e-6
    # the reference's restart from the frame alone returns to the initial box
    c = mdb.MDSimulation(cfg, filename=fp, step=80)
    assert c.get_Lx() == cfg["box_w_global"] != a.get_Lx()


def test_checkpoint_piston_mode(built, tmp_path):
    f, Lx, Ly = wl.lattice_frame(1500, 0.8, 2.0, 0.65, 0.8, seed=32, jitter=0.1)
    cfg = wl.config_dict(1500, Lx, Ly, dt=0.001, barostat_mass=10.0, k_piston=100.0)
    a = mdb.MDSimulation(cfg, frame=f)
    a.step_single_NPH_piston(1.0, nsteps=50)
    fp, sp = str(tmp_path / "p.pframe"), str(tmp_path / "p.json")
    a.save_checkpoint(fp, 1, sp)
    a.step_single_NPH_piston(1.0, nsteps=20)
    b = mdb.MDSimulation(cfg, filename=fp, step=1, state_file=sp)
    b.step_single_NPH_piston(1.0, nsteps=20)
    assert abs(b.get_Ly() - a.get_Ly()) <= 1e-10 * a.get_Ly()
    assert abs(b.get_nph_piston_velocity() - a.get_nph_piston_velocity()) <= 1e-8
    assert np.max(np.abs(b.get_host_particles()["pos"] - a.get_host_particles()["pos"])) < 1e-8


def test_async_writer_matches_synchronous_frames(built, tmp_path):
    f, cfg = wl.nve_4096(seed=3)
    sim = mdb.MDSimulation(cfg, frame=f)
    path = str(tmp_path / "traj.pframe")
    expected = []
    with mdb.TrajectoryWriter(path, depth=2) as w:
        for k in range(5):
            sim.step_single_NVE(nsteps=7)
            w.write(sim, k * 7)  # queued on the stream; the host goes on
            sim.sample_collect()  # get_host_particles returns the last collected frame
            expected.append(sim.get_host_particles())
        w.flush()
    r = mdb.FileReader(path)
    for k in range(5):
        got = r.read(k * 7)
        assert got.tobytes() == expected[k].tobytes()
