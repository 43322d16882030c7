"""V-McMD virtual-state transitions on the engine.

* ala3 with the reference's four-state V-McMD run (fixture tests/golden/ala3_vmcmd.json, the
  reference's all-pairs CPU program): over steps 0-200 the engine takes the same 100 decisions
  (virtual-state log equal), its lambda log follows the reference's, and its generator ends in
  the state the oracle reaches replaying the reference's decisions (every word equal).
* The device generator across many twists: three walkers try a move at every step for 4,500
  steps (up to 9,000 draws each, 14 twists, and the 4,096-entry log ring drained mid-call); the
  oracle replays each walker's decisions from the engine's own lambda log and must take the same
  ones and end with the same generator words.  Graph replays and kernel-by-kernel steps give the
  same logs.
* A run handed from one engine to another (state, step number, virtual state and generator)
  continues exactly as the uninterrupted run; an og_step undone by a fault in another system
  leaves a walker's state, generator and logs as they were at the call's start.
"""
import importlib.util
import json
import os

import numpy as np
import pytest

from omegagene_b200 import engine, systems
from oracle import ogo

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden")
RT = 8.31451 / 4.184 * 1e-3 * 300.0


def _vm_golden():
    spec = importlib.util.spec_from_file_location("make_ala3_golden", os.path.join(GOLD, "make_ala3_golden.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod.load_system(), json.load(open(os.path.join(GOLD, "ala3_vmcmd.json")))


def _replay(vm, seed, lambdas):
    """Oracle decisions for the lambdas of successive transition steps: (states, generator)."""
    L = ogo.lib()
    lam = np.ascontiguousarray([[x["lambda_low"], x["lambda_high"]] for x in vm["states"]], np.float64).reshape(-1)
    prob = np.ascontiguousarray([[x["prob_low"], x["prob_high"]] for x in vm["states"]], np.float64).reshape(-1)
    st = np.zeros(625, np.uint32)
    L.ogo_mt_seed(st, seed)
    cur = vm.get("cur_vs", vm["init_vs"] - 1)
    out = []
    for x in lambdas:
        cur = L.ogo_vmcmd_transition(len(vm["states"]), lam, prob, cur, float(x), st)
        out.append(cur)
    return np.array(out, np.int32), st


def test_ala3_vmcmd_matches_reference_run():
    s, g = _vm_golden()
    eng = engine.Engine(0)
    eng.add_system(s, g["params"], g["vmcmd"])
    eng.finalize()
    eng.step(g["n_steps"] + 1)  # steps 0..n_steps, as the reference's loop and its last step
    steps, vs = eng.take_vs_log(0)
    assert [[int(a), int(b) + 1] for a, b in zip(steps, vs)] == g["vs"]
    lsteps, lam = eng.take_lambda_log(0)
    ref = np.array(g["lambda"])
    assert list(lsteps) == list(range(1, g["n_steps"] + 1))
    rel = np.abs(lam - ref) / np.abs(ref)
    # FP32 pair forces summed in another order than the reference's: ~1e-7 at the start,
    # growing along the trajectory
    assert rel[:10].max() <= 1e-6, rel[:10].max()
    assert rel.max() <= 1e-4, rel.max()
    states, mt = _replay(g["vmcmd"], g["random_seed"], [g["lambda"][st - 1] for st, _ in g["vs"]])
    cur, mt_dev = eng.vmcmd_state(0)
    assert cur == states[-1] and np.array_equal(mt_dev, mt)
    assert eng.take_vs_log(0)[0].size == 0  # taken entries are gone
    eng.close()


def _hopping_walkers(n=3):
    """Small water boxes whose four states all hold any lambda: a move is tried at every step."""
    out = []
    for k in range(n):
        s = systems.water_system(300, seed=70 + k)
        states = [dict(order=0, lambda_low=-1e9, lambda_high=1e9, prob_low=0.0 if v == 0 else 0.5,
                       prob_high=0.0 if v == 3 else 0.45, coef=[(0.97 + 0.02 * v) / RT], alpha_low=0.0,
                       alpha_high=0.0) for v in range(4)]
        vm = {"n_vs": 4, "interval": 1, "temperature": 300.0, "states": states, "init_vs": 2, "seed": 0}
        p = dict(engine.DEFAULT_PARAMS)
        p.update(nsgrid_update_intvl=10, time_step=2.0, thermostat="scaling", temperature=300.0,
                 random_seed=1000 + 17 * k, print_intvl_extended_lambda=1)
        out.append((s, p, vm))
    return out


def _run(walkers, n_steps, graphs=True, variant=6):
    eng = engine.Engine(0)
    eng.set_tuning(variant)
    eng.set_graphs(graphs)
    for s, p, vm in walkers:
        eng.add_system(s, p, vm)
    eng.finalize()
    eng.step(n_steps)
    res = [(eng.take_vs_log(i), eng.take_lambda_log(i), eng.vmcmd_state(i)) for i in range(len(walkers))]
    eng.close()
    return res


def test_device_generator_many_twists_and_ring_drain():
    walkers = _hopping_walkers()
    n = 4500
    res = _run(walkers, n)
    for (s, p, vm), ((vst, vs), (lst, lam), (cur, mt)) in zip(walkers, res):
        assert list(vst) == list(range(1, n)) and list(lst) == list(range(1, n))  # steps 0..n-1 ran
        states, mt_ref = _replay(vm, p["random_seed"], lam)
        assert np.array_equal(vs, states)
        assert cur == states[-1] and np.array_equal(mt, mt_ref)
        assert len(set(vs.tolist())) == 4
    plain = _run(walkers, n, graphs=False)
    for a, b in zip(res, plain):
        assert np.array_equal(a[0][1], b[0][1]) and np.array_equal(a[1][1], b[1][1])
        assert np.array_equal(a[2][1], b[2][1])


def test_handover_continues_the_run():
    (s, p, vm), = _hopping_walkers(1)
    whole = engine.Engine(0)
    whole.set_tuning(6)
    whole.add_system(s, p, vm)
    whole.finalize()
    whole.step(120)
    ref = (whole.take_vs_log(0), whole.take_lambda_log(0), whole.vmcmd_state(0), whole.get_state(0))
    whole.close()
    a = engine.Engine(0)
    a.set_tuning(6)
    a.add_system(s, p, vm)
    a.finalize()
    a.step(60)
    vs1, lam1 = a.take_vs_log(0), a.take_lambda_log(0)
    cur, mt = a.vmcmd_state(0)
    crd, vel = a.get_state(0)
    a.close()
    b = engine.Engine(0)
    b.set_tuning(6)
    b.add_system(dict(s, crd=crd, vel=vel), p, dict(vm, cur_vs=cur, mt_state=mt), first_step=60)
    b.finalize()
    b.step(60)
    vs2, lam2 = b.take_vs_log(0), b.take_lambda_log(0)
    got = (b.vmcmd_state(0), b.get_state(0))
    b.close()
    assert np.array_equal(np.concatenate([vs1[0], vs2[0]]), ref[0][0])
    assert np.array_equal(np.concatenate([vs1[1], vs2[1]]), ref[0][1])
    assert np.array_equal(np.concatenate([lam1[1], lam2[1]]), ref[1][1])
    assert got[0][0] == ref[2][0] and np.array_equal(got[0][1], ref[2][1])
    assert np.array_equal(got[1][0], ref[3][0]) and np.array_equal(got[1][1], ref[3][1])


def test_fault_undo_restores_vmcmd_state_and_logs():
    walkers = _hopping_walkers(2)
    eng = engine.Engine(0)
    eng.set_tuning(6)
    for s, p, vm in walkers:
        eng.add_system(s, p, vm)
    eng.finalize()
    eng.step(40)
    before = eng.vmcmd_state(0)
    crd, vel = eng.get_state(1)
    crd = crd.copy()
    crd[5, 0] += 1.0e5
    eng.set_state(1, crd, vel)
    with pytest.raises(engine.OgError) as ex:
        eng.step(20)
    assert ex.value.status == engine.OG_ERR_SYSTEM_FAULT
    after = eng.vmcmd_state(0)
    assert after[0] == before[0] and np.array_equal(after[1], before[1])
    steps, _ = eng.take_vs_log(0)
    assert list(steps) == list(range(1, 40))  # the 40 steps 0..39 of the first call
    eng.close()
