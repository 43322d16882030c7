"""V-McMD virtual-state transitions on the CPU: the oracle's generator and transition rule
against std::mt19937 and against the reference's own V-McMD run, plus the host-side config and
descriptor handling (no GPU).

Fixtures (tests/golden/make_vmcmd_golden.py): mt19937_vectors.json, draws of g++'s
std::mt19937; ala3_vmcmd.json, the reference's all-pairs CPU program run on its ala3 sample with
a four-state V-McMD section (virtual-state log, lambda log and printed energies).
"""
import importlib.util
import json
import os

import numpy as np
import pytest

from omegagene_b200 import engine
from oracle import ogo

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden")


def _vm_golden():
    spec = importlib.util.spec_from_file_location("make_ala3_golden", os.path.join(GOLD, "make_ala3_golden.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod.load_system(), json.load(open(os.path.join(GOLD, "ala3_vmcmd.json")))


def _ladder(vm):
    lam = np.ascontiguousarray([[x["lambda_low"], x["lambda_high"]] for x in vm["states"]], np.float64).reshape(-1)
    prob = np.ascontiguousarray([[x["prob_low"], x["prob_high"]] for x in vm["states"]], np.float64).reshape(-1)
    return lam, prob


def test_mt19937_matches_std_library():
    L = ogo.lib()
    gold = json.load(open(os.path.join(GOLD, "mt19937_vectors.json")))["draws"]
    for seed, draws in gold.items():
        st = np.zeros(625, np.uint32)
        L.ogo_mt_seed(st, int(seed))
        got = [L.ogo_mt_next(st) for _ in range(len(draws))]
        assert got == draws, seed


def test_mt19937_standard_known_answer():
    """The C++ standard ([rand.predef]): the 10000th draw of a default-constructed mt19937
    (seed 5489) is 4123659995."""
    L = ogo.lib()
    st = np.zeros(625, np.uint32)
    L.ogo_mt_seed(st, 5489)
    for _ in range(9999):
        L.ogo_mt_next(st)
    assert L.ogo_mt_next(st) == 4123659995


def test_oracle_transitions_replay_reference_log():
    """Fed the lambdas the reference logged, the oracle's transition rule and generator take
    every one of the reference's 100 decisions (ExtendedVMcMD::set_current_vstate)."""
    _, g = _vm_golden()
    L = ogo.lib()
    vm = g["vmcmd"]
    lam, prob = _ladder(vm)
    st = np.zeros(625, np.uint32)
    L.ogo_mt_seed(st, g["random_seed"])
    cur = vm["init_vs"] - 1
    moves = 0
    for step, vs1 in g["vs"]:
        nxt = L.ogo_vmcmd_transition(len(vm["states"]), lam, prob, cur, g["lambda"][step - 1], st)
        moves += nxt != cur
        cur = nxt
        assert cur + 1 == vs1, step
    assert moves >= 30  # the fixture exercises the rule, not one state


def test_transition_rule_edges():
    """Extend.cpp:160-177 case by case; the generator position shows which cases draw."""
    L = ogo.lib()
    lam = np.array([0.0, 10.0, 5.0, 15.0, 12.0, 20.0])      # three states
    prob = np.array([0.0, 1.0, 1.0, 1.0, 1.0, 0.0])         # down, up per state
    st = np.zeros(625, np.uint32)
    L.ogo_mt_seed(st, 1)
    # source out of its range: no draw, no move
    assert L.ogo_vmcmd_transition(3, lam, prob, 0, 11.0, st) == 0 and st[624] == 624
    # neighbour above out of range, bottom state cannot go down: no draw
    assert L.ogo_vmcmd_transition(3, lam, prob, 0, 2.0, st) == 0 and st[624] == 624
    # up with probability 1: one draw, moves up
    assert L.ogo_vmcmd_transition(3, lam, prob, 0, 6.0, st) == 1 and st[624] == 1
    # top state: up is never tried; down with probability 1
    assert L.ogo_vmcmd_transition(3, lam, prob, 2, 13.0, st) == 1 and st[624] == 2
    # probability 0 up: a draw, never a move; the state below does not hold lambda: no draw
    prob0 = np.array([0.0, 0.0, 0.0, 0.0, 0.0, 0.0])
    assert L.ogo_vmcmd_transition(3, lam, prob0, 1, 13.0, st) == 1 and st[624] == 3


def test_oracle_vmcmd_md_tracks_reference():
    """The oracle's leapfrog step with V-McMD scaling over the reference's first 100 steps: the
    same 50 virtual-state decisions and lambda (the potential energy) within 1e-6 relative (FP64
    over the cell list against the reference's FP32 all-pairs sums)."""
    s, g = _vm_golden()
    md = ogo.OracleMD(s, g["params"], mcmd=g["vmcmd"])
    for _ in range(101):
        md.step()
    assert [[a, b + 1] for a, b in md.vs_log] == g["vs"][:50]
    got = np.array([v for _, v in md.lambda_log])
    ref = np.array(g["lambda"][:100])
    assert [a for a, _ in md.lambda_log] == list(range(1, 101))
    assert np.max(np.abs(got - ref) / np.abs(ref)) <= 1e-6


def test_run_config_vmcmd_keys():
    p = engine.parse_run_config("--extended-ensemble v-mcmd\n--random-seed 42\n"
                                "--print-interval-extended-lambda 5\n--fn-o-vmcmd-log vs.log\n"
                                "--fn-o-extended-lambda lam.out\n--format-o-extended-lambda ascii\n")
    assert p["extended_ensemble"] == "v-mcmd" and p["random_seed"] == 42
    assert p["print_intvl_extended_lambda"] == 5 and p["fn_o_vmcmd_log"] == "vs.log"
    assert p["format_o_extended_lambda"] == "ascii"
    with pytest.raises(ValueError):
        engine.parse_run_config("--extended-ensemble vcmd")


def test_make_desc_vmcmd_fields():
    s, g = _vm_golden()
    p = dict(g["params"])
    d, keep = engine.make_desc(s, p, g["vmcmd"])
    assert d.n_vstates == 4 and d.vmcmd_trans_interval == 2 and d.vmcmd_init_vs == 0
    assert d.vmcmd_seed == g["random_seed"] and d.vmcmd_lambda_log_interval == 1
    assert list(keep.vs_order) == [2, 2, 2, 2] and len(keep.vs_coef) == 12
    assert keep.vs_prob[1] == 0.5 and keep.vs_prob[-1] == 0.0
    assert not d.vmcmd_mt_state
    mt = np.arange(625, dtype=np.uint32)
    mt[624] = 7
    d2, keep2 = engine.make_desc(s, p, dict(g["vmcmd"], cur_vs=3, mt_state=mt))
    assert d2.vmcmd_init_vs == 3 and d2.vmcmd_mt_state[624] == 7
    with pytest.raises(ValueError):
        engine.make_desc(s, p, dict(g["vmcmd"], mt_state=np.zeros(10, np.uint32)))
