"""The displacement-triggered cell-pair list (OG_LIST_DISPLACEMENT) against FP64 all-pairs
forces, and the reference's fixed schedule (DynamicsMode.cpp:480) for contrast.

A hot water box (velocities x4, NVE, 2 fs) moves atoms farther than the 1 A list margin within
the reference's 10-step interval.  Each step's forces of the FP64 pair variant over the engine's
(possibly several steps old) list are compared with the FP64 oracle's all-pairs forces at the
same positions: the list's grid coordinates (MiniCell::crd, which the reference rounds through
float at every build, MiniCell.cpp:413-470, and moves by each step's displacement since) for the
pair terms, the atoms' own coordinates for the excluded-pair term.  A list that holds every pair
within the cutoff gives the same forces to the fixed-point resolution, while one missed pair at
11.5 A is off by ~0.1 kcal/mol/A."""
import numpy as np
import pytest

from omegagene_b200 import cls_io, engine, systems
from oracle import ogo

pytestmark = pytest.mark.gpu

N_STEPS = 30


def _hot():
    s = systems.water_system(1500, seed=5)
    return dict(s, vel=np.asarray(s["vel"]) * 4.0)


def _params(intvl):
    p = dict(engine.DEFAULT_PARAMS)
    p.update(nsgrid_update_intvl=intvl, time_step=2.0)
    return p


def _run(s, policy, intvl, variant, graphs=True, n=N_STEPS):
    eng = engine.Engine(0)
    eng.set_tuning(variant)
    eng.set_list_policy(policy)
    eng.set_graphs(graphs)
    eng.add_system(s, _params(intvl))
    eng.finalize()
    b0 = eng.list_builds()
    eng.set_trace(n)
    eng.step(n)
    crd, vel = eng.get_state(0)
    out = crd, vel, eng.get_trace(n)[:, 0, :], eng.list_builds() - b0
    eng.close()
    return out


def _allpairs_work(s, grid_crd, crd):
    """FP64 pair work over all pairs at grid_crd plus the excluded-pair term at crd."""
    n, t = s["n_atoms"], s["topol"]
    nb = cls_io.nb15off_table(n, t["nb15off_pairs"])
    pbc = ogo.make_pbc(s["pbc_val"])
    L = np.array(pbc.L, np.float32).astype(np.float64)
    c6, c12 = cls_io.lj_tables(t)
    w, e, v = np.zeros(3 * n), np.zeros(2), np.zeros(9)
    ogo.lib().ogo_pair_allpairs_f64(L, n, np.ascontiguousarray(ogo.wrap_inbox(pbc, grid_crd).reshape(-1)),
                                    np.ascontiguousarray(t["charge"], np.float64), t["atom_type"].astype(np.int32),
                                    int(t["n_lj_types"]), c6.reshape(-1), c12.reshape(-1), nb.reshape(-1), 32, 12.0,
                                    w, e, v)
    ep = ogo.excess_pairs(n, nb).reshape(-1).astype(np.int32)
    ogo.lib().ogo_excess_f64(L, len(ep) // 2, ep, np.ascontiguousarray(crd.reshape(-1)),
                             np.ascontiguousarray(t["charge"], np.float64), 12.0, w, np.zeros(9))
    return w.reshape(-1, 3)


def _worst_force_error(s, policy):
    """Largest per-component difference, over N_STEPS one-step calls, between the engine's FP64
    forces on its own list and FP64 all-pairs forces at the same positions."""
    eng = engine.Engine(0)
    eng.set_tuning(engine.PAIR_VARIANT_F64)
    eng.set_list_policy(policy)
    eng.add_system(s, _params(10))
    eng.finalize()
    b0 = eng.list_builds()
    worst = 0.0
    for _ in range(N_STEPS):
        crd, _ = eng.get_state(0)
        g = eng.get_grid(0)  # the list's grid positions now, before the step moves them
        b = eng.list_builds()
        eng.step(1)
        if eng.list_builds() != b:  # rebuilt at this step's start: the grid is crd through float
            grid = crd.astype(np.float32).astype(np.float64)
        else:
            real = g["slot_atomid"] >= 0
            grid = np.zeros_like(crd)
            grid[g["slot_atomid"][real]] = g["slot_crd"][real]
        work, _, _ = eng.get_forces(0)
        worst = max(worst, float(np.abs(work - _allpairs_work(s, grid, crd)).max()))
    builds = eng.list_builds() - b0
    eng.close()
    return worst, builds


def test_displacement_policy_evaluates_every_pair():
    s = _hot()
    err_dis, b_dis = _worst_force_error(s, "displacement")
    err_fix, b_fix = _worst_force_error(s, "fixed")
    assert b_fix == 3
    assert 4 <= b_dis < N_STEPS, b_dis  # rebuilt when needed, not every step
    assert err_dis < 1e-6, err_dis
    # the reference's schedule misses pairs of this hot box: the contrast shows the test's power
    assert err_fix > 1e-3, err_fix


def test_displacement_policy_graph_equals_kernel_by_kernel():
    """Inside a captured graph the rebuild is a conditional node set on the device; launched
    kernel by kernel the host reads the same mark.  Both give the same trajectory bit for bit
    with the production j-list kernel."""
    s = _hot()
    c1, v1, t1, b1 = _run(s, "displacement", 10, 10, graphs=True)
    c2, v2, t2, b2 = _run(s, "displacement", 10, 10, graphs=False)
    assert b1 == b2 and 3 <= b1 < N_STEPS
    assert np.array_equal(c1, c2) and np.array_equal(v1, v2)
    np.testing.assert_array_equal(t1, t2)


def test_displacement_policy_any_split_of_a_run_is_the_same():
    """Calls of any length (kernel-by-kernel steps, then graph replays) make the same rebuild
    decisions: a run split into two calls gives the trajectory of one call."""
    s = _hot()
    p = dict(engine.DEFAULT_PARAMS)
    p.update(nsgrid_update_intvl=10, time_step=2.0)

    def run(chunks):
        eng = engine.Engine(0)
        eng.set_tuning(10)
        eng.set_list_policy("displacement")
        eng.add_system(s, p)
        eng.finalize()
        for n in chunks:
            eng.step(n)
        out = eng.get_state(0)
        eng.close()
        return out

    a = run([20])
    b = run([7, 13])
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
