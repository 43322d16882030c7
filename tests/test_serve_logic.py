"""Host logic of the continuous-batching server, on the CPU with a fake engine and clock:
admission order, job and memory caps, window boundaries, state hand-over and latencies."""
import numpy as np
import pytest

from omegagene_b200 import serve


class FakeClock:
    def __init__(self):
        self.t = 0.0

    def __call__(self):
        return self.t

    def sleep(self, dt):
        self.t += dt


class FakeEngine:
    """Advances every system's coordinates by +1 per step; one step costs 1 ms per 1000 atoms
    of the batch on the fake clock."""
    log = []

    def __init__(self, clock, fail_at=None):
        self.clock = clock
        self.systems = []
        self.fail_at = fail_at or {}  # system size -> coordinate value at which it faults
        self.faults = None

    def set_tuning(self, v):
        pass

    def tuning(self):
        return {"pair_variant": 0}

    def add_system(self, s, params, mcmd=None, first_step=0):
        self.systems.append({"crd": np.array(s["crd"], float), "vel": np.array(s["vel"], float),
                             "first_step": first_step, "n": s["n_atoms"]})

    def finalize(self):
        FakeEngine.log.append([(s["n"], s["first_step"]) for s in self.systems])

    def step(self, n):
        bad = [int(s["n"] in self.fail_at and s["crd"][0, 0] + n > self.fail_at[s["n"]]) * 4 for s in self.systems]
        if any(bad):  # like og_step: nothing advances, the faulted systems are named
            self.faults = np.array(bad, np.int32)
            raise serve.engine.OgError(serve.engine.OG_ERR_SYSTEM_FAULT, "fault")
        for s in self.systems:
            s["crd"] += n
        self.clock.t += n * 1e-3 * sum(s["n"] for s in self.systems) / 1000.0

    def system_faults(self):
        return self.faults

    def get_state(self, i):
        return self.systems[i]["crd"].copy(), self.systems[i]["vel"].copy()

    def set_state(self, i, crd=None, vel_next=None):
        if crd is not None:
            self.systems[i]["crd"] = np.array(crd, float)
        if vel_next is not None:
            self.systems[i]["vel"] = np.array(vel_next, float)

    def get_energies(self, i):
        return {"step": float(self.systems[i]["crd"][0, 0])}

    def close(self):
        pass


def _system(n):
    return {"n_atoms": n, "crd": np.zeros((n, 3)), "vel": np.zeros((n, 3))}


def _server(clock, fail_at=None, **kw):
    FakeEngine.log = []
    return serve.Server(0, hbm_budget_bytes=kw.pop("budget", 10 ** 12), clock=clock, sleep=clock.sleep,
                        engine_factory=lambda dev: FakeEngine(clock, fail_at), **kw)


def test_every_job_runs_exactly_its_steps():
    clock = FakeClock()
    p = {"nsgrid_update_intvl": 10}
    jobs = [serve.Job(k, _system(100 * (k + 1)), p, 10 * (k + 1), arrival_s=0.001 * k) for k in range(6)]
    res = _server(clock, max_jobs=3, window=20).run(jobs)
    assert res["n_jobs"] == 6
    for j in jobs:
        assert np.all(j.crd == j.n_steps)  # the fake engine adds 1 per step: no step lost or repeated
        assert j.steps_done == j.n_steps
        assert j.latency_s > 0


def test_first_step_carried_over_at_relayout():
    clock = FakeClock()
    p = {"nsgrid_update_intvl": 10}
    jobs = [serve.Job(0, _system(100), p, 60), serve.Job(1, _system(100), p, 20),
            serve.Job(2, _system(100), p, 20, arrival_s=0.0)]
    _server(clock, max_jobs=2, window=20).run(jobs)
    # job 0 starts at step 0, then continues at 20 beside job 2 after job 1 leaves
    assert FakeEngine.log[0] == [(100, 0), (100, 0)]
    assert FakeEngine.log[1] == [(100, 20), (100, 0)]
    assert all(fs % 10 == 0 for batch in FakeEngine.log for _, fs in batch)


def test_memory_budget_and_job_cap():
    clock = FakeClock()
    p = {"nsgrid_update_intvl": 10}
    jobs = [serve.Job(k, _system(1000), p, 20) for k in range(5)]
    srv = _server(clock, max_jobs=4, window=20, budget=2 * 1000 * serve.BYTES_PER_ATOM)
    res = srv.run(jobs)
    assert res["n_jobs"] == 5 and max(srv.batch_sizes) == 2


def test_idle_server_waits_for_arrivals():
    clock = FakeClock()
    p = {"nsgrid_update_intvl": 10}
    jobs = [serve.Job(0, _system(100), p, 10, arrival_s=5.0)]
    res = _server(clock, max_jobs=4, window=10).run(jobs)
    assert jobs[0].t_admit >= 5.0 and res["n_jobs"] == 1


def test_bad_window_and_steps_rejected():
    clock = FakeClock()
    with pytest.raises(ValueError):
        serve.Job(0, _system(10), {"nsgrid_update_intvl": 10}, 15)
    jobs = [serve.Job(0, _system(10), {"nsgrid_update_intvl": 10}, 20)]
    with pytest.raises(ValueError):
        _server(clock, window=15).run(jobs)


def test_fifo_latencies():
    lat, span = serve.fifo_latencies([0.0, 1.0, 1.5], [2.0, 1.0, 1.0])
    assert np.allclose(lat, [2.0, 2.0, 2.5]) and span == pytest.approx(4.0)


def test_faulted_job_retired_others_finish():
    """A job whose system faults mid-window leaves as failed with its state at the window's
    start; the window is redone for the others, which still run exactly their steps."""
    clock = FakeClock()
    p = {"nsgrid_update_intvl": 10}
    jobs = [serve.Job(k, _system(100 * (k + 1)), p, 60) for k in range(3)]
    res = _server(clock, fail_at={200: 30}, max_jobs=3, window=20).run(jobs)
    assert res["n_jobs"] == 2 and res["n_failed"] == 1
    bad = jobs[1]
    assert bad.failed and bad.fault == 4 and bad.steps_done == 20 and np.all(bad.crd == 20)
    for j in (jobs[0], jobs[2]):
        assert not j.failed and np.all(j.crd == 60)


@pytest.mark.parametrize("arrive", [0.0, 0.004])
def test_batches_built_ahead_match_boundary_builds(arrive):
    """The next batch built during the window (then given the continuing jobs' state) leaves
    every job where building it at the boundary does: same steps, same coordinates, same
    batches; with staggered arrivals some boundaries are not predictable and are built there."""
    out = []
    for ahead in (False, True):
        clock = FakeClock()
        p = {"nsgrid_update_intvl": 10}
        jobs = [serve.Job(k, _system(100 * (k % 3 + 1)), p, 20 * (k % 4 + 1), arrival_s=arrive * k)
                for k in range(9)]
        srv = _server(clock, max_jobs=3, window=20, prepare_ahead=ahead)
        res = srv.run(jobs)
        out.append((res, [(j.steps_done, j.crd[0, 0], j.t_admit, j.t_done) for j in jobs], list(FakeEngine.log),
                    srv.batch_sizes))
    (r0, j0, log0, b0), (r1, j1, log1, b1) = out
    assert j0 == j1 and b0 == b1 and r0["n_jobs"] == r1["n_jobs"] == 9
    assert r0["prepared_relayouts"] == 0 and r1["prepared_relayouts"] > 0
    assert sorted(map(tuple, log0)) == sorted(map(tuple, log1)) or arrive > 0


def test_failed_ahead_build_falls_back_to_the_boundary():
    """An engine built ahead that fails (say, two handles do not fit at once) is replaced by one
    built at the boundary; every job still runs exactly its steps."""
    import threading
    clock = FakeClock()
    p = {"nsgrid_update_intvl": 10}
    main = threading.current_thread()

    def factory(dev):
        if threading.current_thread() is not main:
            raise MemoryError("no room for a second handle")
        return FakeEngine(clock)

    jobs = [serve.Job(k, _system(100 * (k + 1)), p, 20 * (k % 3 + 1)) for k in range(6)]
    srv = serve.Server(0, hbm_budget_bytes=10 ** 12, max_jobs=3, window=20, clock=clock, sleep=clock.sleep,
                       engine_factory=factory)
    res = srv.run(jobs)
    assert res["n_jobs"] == 6 and res["prepared_relayouts"] == 0
    for j in jobs:
        assert np.all(j.crd == j.n_steps) and j.steps_done == j.n_steps
