"""No kernel of the step reads device memory that nothing wrote: with OG_DEBUG_POISON set, every
buffer the engine allocates starts filled with that byte, and runs with two different bytes
must agree bit for bit (positions, velocities and the per-step energies).  Covered: the
solvated chain (bonds, angles, SHAKE pairs and trios, two COM groups) with the thermostat loop,
both list policies, graphs on and off, and a water box."""
import os

import numpy as np
import pytest

from omegagene_b200 import engine, systems

pytestmark = pytest.mark.gpu
N = 60


def _run(s, p, poison, variant, policy, graphs):
    os.environ["OG_DEBUG_POISON"] = str(poison)
    try:
        eng = engine.Engine(0)
    finally:
        os.environ.pop("OG_DEBUG_POISON")
    eng.set_tuning(variant)
    eng.set_list_policy(policy)
    eng.set_graphs(graphs)
    eng.add_system(s, p)
    eng.finalize()
    eng.set_trace(N)
    eng.step(N)
    out = eng.get_state(0), eng.get_trace(N).copy()
    eng.close()
    return out


@pytest.mark.parametrize("kind,variant,policy,graphs", [
    ("chain", 10, "displacement", True), ("chain", 10, "fixed", False), ("chain", 1, "fixed", True),
    ("water", 10, "displacement", True)])
def test_results_do_not_depend_on_fresh_memory(kind, variant, policy, graphs):
    if kind == "chain":
        s = systems.chain_water_system(300, 2500, seed=4, radius=12.0)
    else:
        s = systems.water_system(1500, seed=5)
    p = dict(engine.DEFAULT_PARAMS)
    p.update(time_step=0.5, nsgrid_update_intvl=10, thermostat="scaling", temperature=300.0)
    (c0, v0), t0 = _run(s, p, 0, variant, policy, graphs)
    (c1, v1), t1 = _run(s, p, 255, variant, policy, graphs)
    assert np.array_equal(c0, c1) and np.array_equal(v0, v1)
    np.testing.assert_array_equal(t0, t1)
