"""Electrostatics and nonbond models other than zero-dipole alpha = 0, on the CPU: the oracle's
FP32 all-pairs restatement against the reference's own runs of its ala3 sample in each model
(fixture tests/golden/ala3_models.json from make_ele_golden.py): zero-quadrupole / -octupole /
-hexadecapole at alpha 0, all four orders at alpha 0.1, Debye-Hueckel, and HPS.  Every energy the
reference printed for steps 0 and 1 (bond ... VDW, Ele, kinetic, total, temperature) is
reproduced to its 11 printed digits."""
import importlib.util
import json
import os

import pytest

from omegagene_b200 import cls_io, engine
from oracle import ogo

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden")


def _load(name):
    spec = importlib.util.spec_from_file_location(name, os.path.join(GOLD, name + ".py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


MODELS = json.load(open(os.path.join(GOLD, "ala3_models.json")))["models"]


@pytest.mark.parametrize("name", sorted(MODELS))
def test_oracle_reproduces_reference_model_run(name):
    mdl = MODELS[name]
    s = _load("make_ala3_golden").load_system()
    if name == "hps":
        s = _load("make_ele_golden").with_hps_lambdas(s)
    md = ogo.OracleMD(s, mdl["params"], pair_mode="allpairs_f32")
    assert not md.model.default
    for row in mdl["steps"][:2]:
        got = md.step()
        for key, ref in row.items():
            if key != "step":
                assert float("%.10e" % got[key]) == ref, (name, row["step"], key, got[key], ref)


def test_model_config_keys():
    p = engine.parse_run_config("--electrostatic zero-octupole\n--ele-alpha 0.2\n--nonbond hydrophobicity-scale-lj\n"
                                "--hydrophobicity-scale-epsiron 0.3\n--debye-huckel-dielectric 80\n")
    assert p["electrostatic"] == "zero-octupole" and p["ele_alpha"] == 0.2
    assert p["nonbond"] == "hydrophobicity-scale-lj" and p["hps_epsilon"] == 0.3 and p["dh_dielectric"] == 80.0
    with pytest.raises(ValueError):
        engine.parse_run_config("--electrostatic ewald")


def test_hps_tables_follow_record_order():
    s = _load("make_ala3_golden").load_system()
    cut, lam = cls_io.hps_tables(s["topol"])
    assert cut.shape == (40, 40) and (cut == cut.T).all() and not lam.any()
    t = _load("make_ele_golden").with_hps_lambdas(s)["topol"]
    _, lam2 = cls_io.hps_tables(t)
    assert lam2[0, 1] == _load("make_ele_golden").hps_lambda(1, 2) and (lam2 == lam2.T).all()
