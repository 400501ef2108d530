"""MD segments in batches (mdb_batch_add_md): every system of a batch follows
exactly the trajectory it follows alone through MDSimulation, bit for bit, and
stops after its own number of steps."""
import numpy as np
import pytest

import md_simulation_cuda_b200 as mdb
from md_simulation_cuda_b200 import workloads as wl

pytestmark = pytest.mark.gpu


def _systems():
    out = []
    for k, (N, aspect, T, nsteps) in enumerate([(1500, 1.0, 0.9, 150), (3000, 2.0, 0.7, 320),
                                                (700, 0.5, 1.1, 230)]):
        f, Lx, Ly = wl.lattice_frame(N, 0.8, aspect, 0.65, T, seed=20 + k, jitter=0.1)
        cfg = wl.config_dict(N, Lx, Ly, dt=0.002, T=T)
        out.append((f, cfg, nsteps))
    return out


@pytest.mark.parametrize("split", [False, True])
@pytest.mark.parametrize("nose_hoover", [True, False])
def test_batch_md_equals_solo(built, nose_hoover, split):
    """A system gives the same bits in a batch and alone when both handles
    use the same lanes setting: one lane (the batch default; the simulation
    handle asked for it) or split lanes (the simulation default; the batch
    asked for it)."""
    systems = _systems()
    b = mdb.Batch(lanes=mdb.LANES_SPLIT) if split else mdb.Batch()
    kind = mdb.JOB_NVT if nose_hoover else mdb.JOB_NVE
    ids = [b.add_md(cfg, f, kind, nsteps) for f, cfg, nsteps in systems]
    b.run(-1)
    assert b.progress() == (3, 3)
    for sid, (f, cfg, nsteps) in zip(ids, systems):
        n, done, steps = b.system_info(sid)
        assert done and steps == nsteps and n == len(f)
        sim = (mdb.MDSimulation(cfg, frame=f) if split
               else mdb.MDSimulation(cfg, frame=f, lanes=mdb.LANES_ONE))
        if nose_hoover:
            sim.step_single_nose_hoover(nsteps=nsteps)
        else:
            sim.step_single_NVE(nsteps=nsteps)
        solo = sim.get_host_particles()
        got = b.frame(sid)
        assert np.array_equal(got["pos"], solo["pos"])
        assert np.array_equal(got["vel"], solo["vel"])
        assert np.array_equal(got["acc"], solo["acc"])
        K, U, xi = b.energies(sid)
        assert abs(K - sim.cal_total_K()) <= 1e-12 * abs(K)
        assert abs(U - sim.cal_total_U()) <= 1e-12 * abs(U)
        if nose_hoover:
            assert xi == sim.xi


def test_batch_md_async_issue_and_collect(built):
    """mdb_batch_issue / query / collect advance a batch chunk by chunk to the
    same end state as mdb_batch_run."""
    systems = _systems()
    a = mdb.Batch()
    b = mdb.Batch()
    for f, cfg, nsteps in systems:
        a.add_md(cfg, f, mdb.JOB_NVT, nsteps)
        b.add_md(cfg, f, mdb.JOB_NVT, nsteps)
    a.run(-1)
    chunks = 0
    while True:
        k = b.issue(100)
        if k == 0:
            break
        chunks += 1
        while not b.idle():
            pass
        b.collect()
    assert chunks >= 4
    assert b.done_flags().all()
    assert b.device_bytes() > 0
    for sid in range(3):
        assert np.array_equal(a.frame(sid)["pos"], b.frame(sid)["pos"])
