"""Continuous batching: every job's result is the same alone and in the mix.

Five jobs, at most three on the device at once, so jobs join and leave a running batch at
window boundaries and continuing jobs are handed over to a new engine with their state and step
number.  Forces are fixed-point sums and every reduction is per system, so the final positions,
velocities and energies must equal those of the job run alone bit for bit.
"""
import numpy as np
import pytest

from omegagene_b200 import engine, serve, systems

pytestmark = pytest.mark.gpu


def _params(**kw):
    p = dict(engine.DEFAULT_PARAMS)
    p.update(kw)
    return p


def _jobs():
    heat = _params(nsgrid_update_intvl=10, time_step=2.0, thermostat="scaling", temperature=300.0,
                   temperature_init=200.0, heating_steps=50)
    nve = _params(nsgrid_update_intvl=10, time_step=2.0)
    spec = [(900, 40, heat), (1500, 60, nve), (600, 20, heat), (1200, 40, heat), (700, 60, nve)]
    return [serve.Job(k, systems.water_system(n, seed=40 + k), p, steps) for k, (n, steps, p) in enumerate(spec)]


def test_served_jobs_equal_alone_runs():
    jobs = _jobs()
    res = serve.Server(0, max_jobs=3, window=20).run(jobs)
    assert res["n_jobs"] == 5 and res["relayouts"] >= 3
    for j in jobs:
        _, ene, crd, vel = serve.run_alone(serve.Job(j.id, j.system, j.params, j.n_steps))
        assert np.array_equal(j.crd, crd) and np.array_equal(j.vel, vel), j.id
        assert j.energies == ene, j.id


def test_memory_budget_limits_admission():
    jobs = _jobs()
    budget = max(j.bytes for j in jobs) + min(j.bytes for j in jobs)
    srv = serve.Server(0, hbm_budget_bytes=budget, max_jobs=8, window=20)
    res = srv.run(jobs)
    assert res["n_jobs"] == 5
    assert max(srv.batch_sizes) <= 2
