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


@pytest.mark.parametrize("variant", [6, 10, "auto"])
def test_served_jobs_equal_alone_runs(variant):
    """Also with the j-list kernel (variant 10) and the autotuner's pick: a job's j lists are
    rebuilt when its own atoms pass the skin, never because another job's did."""
    jobs = _jobs()
    srv = serve.Server(0, max_jobs=3, window=20, pair_variant=variant)
    res = srv.run(jobs)
    assert res["n_jobs"] == 5 and res["relayouts"] >= 3
    used = srv.pair_variant  # "auto" resolves to the first engine's autotuned variant
    assert used != "auto"
    for j in jobs:
        _, ene, crd, vel = serve.run_alone(serve.Job(j.id, j.system, j.params, j.n_steps), pair_variant=used)
        assert np.array_equal(j.crd, crd) and np.array_equal(j.vel, vel), j.id
        assert j.energies == ene, j.id


def test_memory_budget_limits_admission():
    jobs = _jobs()
    budget = max(j.bytes for j in jobs) + min(j.bytes for j in jobs)
    srv = serve.Server(0, hbm_budget_bytes=budget, max_jobs=8, window=20, bytes_per_atom=serve.BYTES_PER_ATOM)
    res = srv.run(jobs)
    assert res["n_jobs"] == 5
    assert max(srv.batch_sizes) <= 2


def test_admission_by_measured_footprint_stays_within_budget():
    """The server measures every engine it builds (og_get_footprint) and admits by the largest
    bytes per atom seen: every batch's device footprint stays within the budget, and the
    estimate is the measurement, not the starting constant."""
    jobs = _jobs()
    budget = int(0.6 * sum(j.n_atoms for j in jobs) * 2000)
    srv = serve.Server(0, hbm_budget_bytes=budget, max_jobs=8, window=20)
    res = srv.run(jobs)
    assert res["n_jobs"] == 5
    assert srv.measured_bytes_per_atom > 0 and srv.bytes_per_atom != serve.BYTES_PER_ATOM
    assert max(peak for _, peak in srv.batch_footprints[1:]) <= budget, (srv.batch_footprints, budget)
    eng = engine.Engine(0)
    eng.add_system(jobs[0].system, jobs[0].params)
    eng.finalize()
    held, peak = eng.footprint()
    assert 0 < held <= peak
    eng.close()


def _engine(batch, variant=6):
    eng = engine.Engine(0)
    eng.set_tuning(variant)  # one pair kernel for every engine compared bitwise
    for s, p in batch:
        eng.add_system(s, p)
    eng.finalize()
    return eng


@pytest.mark.parametrize("variant", [6, 10])
def test_faulted_system_is_isolated(variant):
    """A caller-placed coordinate far outside one system's box makes og_step fail with
    OG_ERR_SYSTEM_FAULT naming that system only; every system is back at the call's start, and
    the others, stepped again without it, match their runs alone bit for bit."""
    p = _params(nsgrid_update_intvl=10, time_step=2.0, thermostat="scaling", temperature=300.0)
    sy = [systems.water_system(n, seed=60 + k) for k, n in enumerate((900, 700, 800))]
    eng = _engine([(s, p) for s in sy], variant)
    start = [eng.get_state(i) for i in range(3)]
    crd, vel = start[1]
    crd = crd.copy()
    crd[5, 0] += 1.0e5
    eng.set_state(1, crd, vel)
    with pytest.raises(engine.OgError) as ex:
        eng.step(20)
    assert ex.value.status == engine.OG_ERR_SYSTEM_FAULT
    f = eng.system_faults()
    assert f[0] == 0 and f[2] == 0 and f[1] & 4
    for i in (0, 2):
        c, v = eng.get_state(i)
        assert np.array_equal(c, start[i][0]) and np.array_equal(v, start[i][1])
    rest = _engine([(sy[0], p), (sy[2], p)], variant)
    rest.step(20)
    for k, i in enumerate((0, 2)):
        alone = _engine([(sy[i], p)], variant)
        alone.step(20)
        c1, v1 = alone.get_state(0)
        c2, v2 = rest.get_state(k)
        assert np.array_equal(c1, c2) and np.array_equal(v1, v2)


@pytest.mark.parametrize("graphs", [False, True])
def test_blown_up_large_system_faults_cleanly(graphs):
    """A 600,000-atom system whose velocities carry every atom far out of its box in one step:
    at the next list build (fixed schedule, every step) all its atoms fall into one MiniCell
    column of ~75,000 cells, whose cell pairs would number more than 2^31.  The system is
    faulted before the pair enumeration, which gives it no pairs (and the list offsets are
    64-bit besides), so the call ends in OG_ERR_SYSTEM_FAULT naming that system, with the other
    system back at the call's start."""
    p = _params(nsgrid_update_intvl=1, time_step=2.0)
    big = systems.water_system(200000, seed=70)
    big = dict(big, vel=np.asarray(big["vel"]) * 1e9)
    small = systems.water_system(800, seed=71)
    eng = _engine([(big, p), (small, p)], 10)
    eng.set_graphs(graphs)
    start = eng.get_state(1)
    with pytest.raises(engine.OgError) as ex:
        eng.step(3)
    assert ex.value.status == engine.OG_ERR_SYSTEM_FAULT
    f = eng.system_faults()
    assert f[0] != 0 and f[1] == 0
    c, v = eng.get_state(1)
    assert np.array_equal(c, start[0]) and np.array_equal(v, start[1])
    eng.close()


@pytest.mark.parametrize("variant", [6, 10])
def test_served_vmcmd_jobs_equal_alone_runs(variant):
    """V-McMD jobs handed between engines keep their virtual state and generator: the served
    virtual-state and lambda logs and final states equal the alone runs' bit for bit."""
    rt = 8.31451 / 4.184 * 1e-3 * 300.0
    jobs = []
    for k, (n, steps) in enumerate(((500, 60), (400, 40), (600, 80))):
        states = [dict(order=0, lambda_low=-1e9, lambda_high=1e9, prob_low=0.0 if v == 0 else 0.5,
                       prob_high=0.0 if v == 2 else 0.5, coef=[(0.98 + 0.02 * v) / rt], alpha_low=0.0,
                       alpha_high=0.0) for v in range(3)]
        vm = {"n_vs": 3, "interval": 3, "temperature": 300.0, "states": states, "init_vs": 2, "seed": 0}
        p = _params(nsgrid_update_intvl=10, time_step=2.0, thermostat="scaling", temperature=300.0,
                    random_seed=300 + k, print_intvl_extended_lambda=2)
        jobs.append(serve.Job(k, systems.water_system(n, seed=80 + k), p, steps, mcmd=vm))
    res = serve.Server(0, max_jobs=2, window=20, pair_variant=variant).run(jobs)
    assert res["n_jobs"] == 3 and res["relayouts"] >= 3
    for j in jobs:
        logs = {}
        fresh = serve.Job(j.id, j.system, j.params, j.n_steps, mcmd={k: v for k, v in j.mcmd.items()
                                                                      if k not in ("cur_vs", "mt_state")})
        _, ene, crd, vel = serve.run_alone(fresh, pair_variant=variant, logs=logs)
        assert np.array_equal(j.crd, crd) and np.array_equal(j.vel, vel), j.id
        assert j.vs_log == logs["vs"] and j.lambda_log == logs["lambda"], j.id
        assert len(j.vs_log) == (j.n_steps - 1) // 3 and len({v for _, v in j.vs_log}) > 1  # steps 3, 6 .. < n


@pytest.mark.parametrize("policy", ["fixed", "displacement"])
def test_column_overflow_faults_the_system_only(policy):
    """A caller piles one system's 5,100 atoms into one MiniCell column (beyond the 4,096 the
    engine sorts): og_step fails with OG_ERR_SYSTEM_FAULT naming that system with bit 2, every
    system is back at the call's start, and the list build that met the column left every index
    valid (the column is laid out unsorted and the call undone)."""
    p = _params(nsgrid_update_intvl=10, time_step=2.0)
    a = systems.water_system(900, seed=61)
    b = systems.water_system(1700, seed=62)
    eng = engine.Engine(0)
    eng.set_tuning(10)
    eng.set_list_policy(policy)
    for s in (a, b):
        eng.add_system(s, p)
    eng.finalize()
    start = [eng.get_state(i) for i in range(2)]
    crd, vel = start[1]
    crd = crd.copy()
    lo = b["pbc_val"][9:12] - 0.5 * b["pbc_val"][0]
    crd[:, 0] = lo[0] + 0.5 + 0.001 * (np.arange(len(crd)) % 7)  # one column: x, y within 0.01 A
    crd[:, 1] = lo[1] + 0.5 + 0.001 * (np.arange(len(crd)) % 5)
    eng.set_state(1, crd, vel)
    with pytest.raises(engine.OgError) as ex:
        eng.step(20)
    assert ex.value.status == engine.OG_ERR_SYSTEM_FAULT
    f = eng.system_faults()
    assert f[0] == 0 and f[1] & 2
    c0, v0 = eng.get_state(0)
    assert np.array_equal(c0, start[0][0]) and np.array_equal(v0, start[0][1])
    eng.close()
