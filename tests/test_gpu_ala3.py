"""The reference's ala3 sample (solvated tri-alanine, 6,207 atoms: bonds, angles, torsions,
impropers, 1-4 pairs, SHAKE pairs / trios / quads, COM cancel on two groups) on the engine.

* Forces and every energy term at the start against the FP64 oracle: force RMS relative error
  <= 1e-5; LJ + ZD energies within 1e-6 |E| + 2e-3 kcal/mol (FP32 pair terms); the FP64 bonded
  and 1-4 terms within 1e-9 relative.
* Ten steps against the energies the reference itself printed (samples/ala3/log03_md.txt, its
  all-pairs CPU build, fixture tests/golden/ala3_log.json): step 0 bonded and 1-4 terms within
  1e-9 relative, VDW / Ele within 1e-6; over ten steps every term within 1e-5 |E| + 1e-4
  kcal/mol (FP32 pair forces summed in another order start a separation of ~1e-7 per step).
"""
import importlib.util
import json
import os

import numpy as np
import pytest

from omegagene_b200 import engine
from oracle import ogo

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
BONDED = ("bond", "angle", "torsion", "improper", "vdw14", "ele14")


def _golden():
    spec = importlib.util.spec_from_file_location("make_ala3_golden", os.path.join(HERE, "golden", "make_ala3_golden.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod.load_system(), json.load(open(os.path.join(HERE, "golden", "ala3_log.json")))


def test_ala3_forces_and_terms_match_fp64_oracle():
    s, gold = _golden()
    p = gold["params"]
    eng = engine.Engine(0)
    eng.add_system(s, p)
    eng.finalize()
    eng.compute_forces()
    work, ene, _ = eng.get_forces(0)
    md = ogo.OracleMD(s, p)
    ref = md.forces()
    w64 = md.work.reshape(-1, 3)
    err = float(np.sqrt(((work - w64) ** 2).sum() / (w64 ** 2).sum()))
    assert err <= 1e-5, err
    for k in ("vdw", "ele"):
        assert abs(ene[k] - ref[k]) <= 1e-6 * abs(ref[k]) + 2e-3, (k, ene[k], ref[k])
    for k in BONDED:
        assert abs(ene[k] - ref[k]) <= 1e-9 * abs(ref[k]) + 1e-9, (k, ene[k], ref[k])
    assert abs(ene["potential"] - ref["potential"]) <= 1e-6 * abs(ref["potential"]) + 2e-3


def test_ala3_tracks_reference_log():
    s, gold = _golden()
    n = 10
    eng = engine.Engine(0)
    eng.add_system(s, gold["params"])
    eng.finalize()
    eng.set_trace(n)
    eng.step(n)
    tr = eng.get_trace(n)[:, 0, :]
    names = engine.ENERGY_NAMES
    row0 = gold["steps"][0]
    for k in BONDED:
        assert abs(tr[0, names.index(k)] - row0[k]) <= 1e-9 * abs(row0[k]), (k, tr[0, names.index(k)], row0[k])
    for k in ("vdw", "ele"):
        assert abs(tr[0, names.index(k)] - row0[k]) <= 1e-6 * abs(row0[k]), (k, tr[0, names.index(k)], row0[k])
    for i, row in enumerate(gold["steps"][:n]):
        for k, ref in row.items():
            if k == "step":
                continue
            got = tr[i, names.index(k)]
            assert abs(got - ref) <= 1e-5 * abs(ref) + 1e-4, (i, k, got, ref)


@pytest.mark.parametrize("run", ["shake", "shake_heating", "noshake"])
def test_ala3_thermostat_tracks_reference_runs(run):
    """The engine's velocity-scaling thermostat against the reference's own runs of the ala3
    sample (tests/golden/ala3_thermo.json): with SHAKE (the iterative loop of
    Thermostat.cpp:86-170, as a device-side loop), with a heating ramp, and without constraints
    (Thermostat.cpp:57-84).  Over ten steps every printed term within 1e-5 |E| + 1e-4 kcal/mol
    (the FP32 pair forces start a separation of ~1e-7 per step); the temperature within 1e-6
    relative of what the reference printed."""
    s, _ = _golden()
    gold = json.load(open(os.path.join(HERE, "golden", "ala3_thermo.json")))["runs"][run]
    n = 10
    eng = engine.Engine(0)
    eng.add_system(s, gold["params"])
    eng.finalize()
    eng.set_trace(n)
    eng.step(n)
    tr = eng.get_trace(n)[:, 0, :]
    names = engine.ENERGY_NAMES
    for i, row in enumerate(gold["steps"][:n]):
        for k, ref in row.items():
            if k == "step":
                continue
            got = tr[i, names.index(k)]
            tol = 1e-6 * abs(ref) if k == "temperature" else 1e-5 * abs(ref) + 1e-4
            assert abs(got - ref) <= tol, (run, i, k, got, ref)
    assert eng.flags() & 16 == 0  # the thermostat loop converged within its limit
