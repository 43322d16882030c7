"""CUDA-graph replay of whole list intervals against kernel-by-kernel stepping.

og_step replays one captured graph per list interval (rebuild step + intvl-1 steps; the
thermostat-with-SHAKE loop is a device-side WHILE node).  Every per-step decision lives on the
device, so replayed and directly launched steps must give bitwise identical trajectories.
"""
import numpy as np
import pytest

from omegagene_b200 import engine, systems

pytestmark = pytest.mark.gpu


def _params(**kw):
    p = dict(engine.DEFAULT_PARAMS)
    p.update(kw)
    return p


def _mixed_batch():
    """Thermostat + SHAKE water, NVE water, and a McMD-scaled chain with SHAKE pairs under the
    thermostat: every branch of the step in one engine."""
    thermo = _params(nsgrid_update_intvl=10, time_step=2.0, thermostat="scaling", temperature=300.0)
    nve = _params(nsgrid_update_intvl=10, time_step=2.0)
    chain = systems.chain_water_system(300, 2500, seed=4, radius=12.0)
    mcmd = systems.mcmd_polynomial(-9000.0, 400.0, seed=7)
    return [(systems.water_system(1500, seed=5), thermo, None),
            (systems.water_system(700, seed=9), nve, None),
            (chain, thermo, mcmd)]


def _run(batch, n_steps, graphs, chunks=None, variant=6):
    eng = engine.Engine(0)
    eng.set_tuning(variant)  # one pair kernel for every engine compared bitwise
    eng.set_graphs(graphs)
    for s, p, m in batch:
        eng.add_system(s, p, m)
    eng.finalize()
    eng.set_trace(n_steps)
    for n in chunks or [n_steps]:
        eng.step(n)
    states = [eng.get_state(i) for i in range(len(batch))]
    return eng, eng.get_trace(n_steps), states


def test_graph_replay_equals_kernel_by_kernel():
    batch = _mixed_batch()
    n = 35  # three whole intervals replayed, five steps launched directly
    eg, tg, sg = _run(batch, n, True)
    ek, tk, sk = _run(batch, n, False)
    info = eg.graph_info()
    assert info["enabled"], info["note"]
    assert info["replays"] == 3 and info["kernels_per_replay"] > 100
    assert ek.graph_info()["replays"] == 0
    np.testing.assert_array_equal(tg, tk)
    for (c1, v1), (c2, v2) in zip(sg, sk):
        assert np.array_equal(c1, c2) and np.array_equal(v1, v2)
    assert eg.flags() == ek.flags()


def test_graph_split_calls_equal_one_call():
    """Calls of any length, aligned to the list interval or not, give the trajectory of one
    long call."""
    batch = _mixed_batch()[:2]
    _, t1, s1 = _run(batch, 40, True)
    _, t2, s2 = _run(batch, 40, True, chunks=[3, 7, 10, 20])
    np.testing.assert_array_equal(t1, t2)
    for (c1, v1), (c2, v2) in zip(s1, s2):
        assert np.array_equal(c1, c2) and np.array_equal(v1, v2)


def test_single_step_graph_equals_kernel_by_kernel():
    """og_step_async replays a captured one-step graph (with energies) for the last step of a
    call under the displacement list policy, whose rebuilds are conditional nodes.  Single-step
    calls with og_put_state in between, as an end-to-end caller makes them, give the trajectory
    and per-step energies of kernel-by-kernel steps bit for bit, rebuilds included; a batch with a
    thermostat-with-SHAKE system and an NVE system covers the WHILE node inside the graph."""
    thermo = _params(nsgrid_update_intvl=10, time_step=2.0, thermostat="scaling", temperature=300.0)
    hot = systems.water_system(1500, seed=5)
    hot = dict(hot, vel=np.asarray(hot["vel"]) * 4.0)  # passes the list margin within a few steps
    batch = [(hot, _params(nsgrid_update_intvl=10, time_step=2.0)), (systems.water_system(700, seed=9), thermo)]
    n = 40
    out = []
    for graphs in (True, False):
        eng = engine.Engine(0)
        eng.set_tuning(10)
        eng.set_list_policy("displacement")
        eng.set_graphs(graphs)
        for s, p in batch:
            eng.add_system(s, p)
        eng.finalize()
        eng.set_trace(n)
        b0 = eng.list_builds()
        for k in range(n):
            if k % 7 == 3:  # a caller's coordinates handed back between steps
                c = np.ascontiguousarray(eng.get_state(0)[0])
                eng.put_state_ptr(0, c.ctypes.data, 0)
            eng.step_async(1)
        eng.synchronize()
        assert eng.flags() & (8 | 16) == 0
        out.append((eng.get_state(0), eng.get_state(1), eng.get_trace(n).copy(), eng.list_builds() - b0,
                    eng.graph_info()))
        eng.close()
    (a0, a1, ta, ba, ga), (b0_, b1, tb, bb, gb) = out
    assert ba == bb and ba >= 2  # rebuilds happened inside the graph replays too
    assert ga["replays"] >= n - 1 and gb["replays"] == 0
    for x, y in ((a0, b0_), (a1, b1)):
        assert np.array_equal(x[0], y[0]) and np.array_equal(x[1], y[1])
    np.testing.assert_array_equal(ta, tb)
