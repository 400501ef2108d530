"""The serving loop (mdb_server_*): requests of mixed kinds submitted over
time are admitted into batches while others run, their work overlaps on the
device, and each result equals the same job run alone, bit for bit."""
import time

import numpy as np
import pytest

import md_simulation_cuda_b200 as mdb
from md_simulation_cuda_b200 import workloads as wl

pytestmark = pytest.mark.gpu


def _md_jobs():
    jobs = []
    for k, (N, T, nsteps, nh) in enumerate([(2000, 0.8, 400, True), (900, 1.1, 250, True),
                                            (4000, 0.6, 600, True), (1200, 1.0, 300, False)]):
        f, Lx, Ly = wl.lattice_frame(N, 0.8, 1.0, 0.65, T, seed=40 + k, jitter=0.1)
        jobs.append((f, wl.config_dict(N, Lx, Ly, dt=0.002, T=T), nsteps, nh))
    return jobs


def _fire_jobs():
    jobs = []
    for k, N in enumerate([300, 520]):
        f, L = wl.random_frame(N, 0.7, 0.5, 900 + k)
        jobs.append((f, wl.config_dict(N, L, L, dt=0.001, T=0.0, n_cap=N)))
    return jobs


def _fire_params():
    return mdb.FireParams(dt_init=0.001, dt_max=0.01, alpha0=0.1, f_inc=1.1, f_dec=0.5, N_min=5)


def test_server_results_equal_solo(built):
    md_jobs, fire_jobs = _md_jobs(), _fire_jobs()
    ids = []
    with mdb.Server(chunk=100) as srv:
        # staggered arrivals, kinds interleaved
        for k in range(max(len(md_jobs), len(fire_jobs))):
            if k < len(md_jobs):
                f, cfg, nsteps, nh = md_jobs[k]
                ids.append(("md", k, srv.submit_md(cfg, f, nsteps, nose_hoover=nh)))
            if k < len(fire_jobs):
                f, cfg = fire_jobs[k]
                ids.append(("fire", k, srv.submit_fire(cfg, f, 1e-4, 4000, _fire_params())))
            time.sleep(0.02)
        results = {}
        for kind, k, rid in ids:
            assert srv.wait(rid, timeout=300.0) == mdb.REQ_DONE
            results[(kind, k)] = srv.result(rid)
        st = srv.stats()
        assert st.finished == len(ids) and st.failed == 0 and st.queued == 0
        assert st.batches_admitted >= 2
    for k, (f, cfg, nsteps, nh) in enumerate(md_jobs):
        r = results[("md", k)]
        assert r.steps == nsteps and r.t_submit <= r.t_start <= r.t_done
        # the server's batches use one lane per particle, as a simulation
        # handle does when asked
        sim = mdb.MDSimulation(cfg, frame=f, lanes=mdb.LANES_ONE)
        if nh:
            sim.step_single_nose_hoover(nsteps=nsteps)
        else:
            sim.step_single_NVE(nsteps=nsteps)
        solo = sim.get_host_particles()
        assert np.array_equal(r.frame["pos"], solo["pos"])
        assert np.array_equal(r.frame["vel"], solo["vel"])
        assert abs(r.U - sim.cal_total_U()) <= 1e-12 * abs(r.U)
    for k, (f, cfg) in enumerate(fire_jobs):
        r = results[("fire", k)]
        solo = mdb.EnergyMinimizer(cfg).minimize_frame(f, 1e-4, 4000, _fire_params())
        assert r.steps == solo.steps and r.converged == solo.converged
        assert np.array_equal(r.frame["pos"], solo.frame["pos"])
        assert r.U == solo.potential_energy


def test_server_admits_while_busy(built):
    """A short request submitted while a long one runs finishes first: it is
    admitted as a second batch instead of waiting for the first."""
    f, Lx, Ly = wl.lattice_frame(40000, 0.8, 1.0, 0.65, 0.8, seed=77, jitter=0.1)
    long_cfg = wl.config_dict(40000, Lx, Ly, dt=0.002, T=0.8)
    g, Lx2, Ly2 = wl.lattice_frame(1000, 0.8, 1.0, 0.65, 0.8, seed=78, jitter=0.1)
    short_cfg = wl.config_dict(1000, Lx2, Ly2, dt=0.002, T=0.8)
    with mdb.Server(chunk=200) as srv:
        a = srv.submit_md(long_cfg, f, 6000)
        while srv.stats().running == 0:
            time.sleep(0.001)
        b = srv.submit_md(short_cfg, g, 200)
        assert srv.wait(b, timeout=300.0) == mdb.REQ_DONE
        assert srv.wait(a, timeout=0.0) != mdb.REQ_DONE
        rb = srv.result(b)
        assert srv.wait(a, timeout=300.0) == mdb.REQ_DONE
        ra = srv.result(a)
        assert rb.t_start < ra.t_done and rb.t_done < ra.t_done
        assert srv.stats().batches_admitted == 2


def test_server_budget_and_errors(built):
    f, Lx, Ly = wl.lattice_frame(5000, 0.8, 1.0, 0.65, 0.8, seed=5)
    cfg = wl.config_dict(5000, Lx, Ly, dt=0.002, T=0.8)
    with mdb.Server(hbm_budget_bytes=1 << 20) as srv:
        rid = srv.submit_md(cfg, f, 10)
        assert srv.wait(rid, timeout=60.0) == mdb.REQ_FAILED
        with pytest.raises(mdb.MDBError) as e:
            srv.result(rid)
        assert e.value.code == 3  # MDB_ERR_CAPACITY
        bad = dict(cfg, box_w_global=-1.0)
        with pytest.raises(mdb.MDBError):
            srv.submit_md(bad, f, 10)


@pytest.mark.parametrize("order, max_wait_ms, expect", [
    (mdb.ORDER_SHORTEST, 60000, ["small", "medium", "big"]),  # least work first
    (mdb.ORDER_SHORTEST, 1, ["big", "small", "medium"]),      # all overdue: oldest first
    (mdb.ORDER_FIFO, 60000, ["big", "small", "medium"]),
])
def test_server_admission_order(built, order, max_wait_ms, expect):
    """Three requests queued behind a running one, one batch at a time: they
    start in the admission order (work = particles x steps)."""
    def job(N, seed):
        f, Lx, Ly = wl.lattice_frame(N, 0.8, 1.0, 0.65, 0.8, seed=seed, jitter=0.1)
        return f, wl.config_dict(N, Lx, Ly, dt=0.002, T=0.8)
    with mdb.Server(chunk=100, max_active_batches=1, max_batch_systems=1, order=order,
                    max_wait_ms=max_wait_ms) as srv:
        f, cfg = job(2000, 60)
        blocker = srv.submit_md(cfg, f, 3000)
        while srv.stats().running == 0:
            time.sleep(0.001)
        ids = {}
        for name, N, nsteps, seed in [("big", 4000, 600, 61), ("small", 900, 250, 62),
                                      ("medium", 2000, 400, 63)]:
            f, cfg = job(N, seed)
            ids[name] = srv.submit_md(cfg, f, nsteps)
        assert srv.wait(blocker, timeout=300.0) == mdb.REQ_DONE
        for rid in ids.values():
            assert srv.wait(rid, timeout=300.0) == mdb.REQ_DONE
        starts = {name: srv.result(rid).t_start for name, rid in ids.items()}
    assert sorted(starts, key=starts.get) == expect
