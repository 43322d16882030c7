"""The reference's ala3 sample run, outputs included, on the engine: mdio.run with the sample's
output settings (a presto frame of the solute every 100 steps, the restart after the loop, the
energy log every step) against the files the reference wrote (fixtures from
tests/golden/make_output_golden.py) and the energies it printed (ala3_log.json).

The trajectory separates slowly from the reference's (FP32 pair forces summed in another order),
so the restart's positions are compared within 1e-3 A after 100 steps (measured on B200: 1.0e-4 A;
velocities 7e-5 relative, energies 1e-7).  The frame labelled step 100 must hold step 99's
positions (what the reference writes there, SubBox::crd_prev), which lie on average 9e-3 A from
step 100's; the engine's frame is within 1e-4 A of the reference's (measured: 1.3e-6 A, FP32
rounding).  The printed energies of all 101 steps agree within 1e-5 relative (measured: 1.2e-6).
"""
import importlib.util
import io
import json
import os

import numpy as np
import pytest

from omegagene_b200 import mdio

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden")


def _golden():
    spec = importlib.util.spec_from_file_location("make_ala3_golden", os.path.join(GOLD, "make_ala3_golden.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod, mod.load_system(), json.load(open(os.path.join(GOLD, "ala3_log.json")))


def _min_image(d, box):
    return d - box * np.round(d / box)


def test_ala3_run_outputs_match_reference_files(tmp_path):
    mod, s, gold = _golden()
    p = dict(gold["params"], n_steps=100, print_intvl_log=1, print_intvl_crd=[100],
             fn_o_crd=[str(tmp_path / "run.cod")], group_o_crd=["solute"], format_o_crd="presto",
             fn_o_restart=str(tmp_path / "run_o.restart"))
    log = io.StringIO()
    mdio.run(s, p, log=log)
    box = np.array([s["pbc_val"][0], s["pbc_val"][4], s["pbc_val"][8]])
    ours, ref = mdio.read_restart(tmp_path / "run_o.restart"), mdio.read_restart(os.path.join(GOLD, "ala3_run_o.restart"))
    assert ours["n_steps"] == ref["n_steps"] == 100 and ours["time"] == ref["time"]
    for k in ("e_potential", "e_kinetic", "e_total"):
        assert abs(ours[k] - ref[k]) <= 1e-5 * abs(ref[k]), (k, ours[k], ref[k])
    dx = np.abs(_min_image(ours["crd"] - ref["crd"], box)).max()
    dv = np.abs(ours["vel"] - ref["vel"]).max() / np.abs(ref["vel"]).max()
    assert dx <= 1e-3 and dv <= 1e-3, (dx, dv)
    (st, t, hdr, crd), = mdio.read_presto_frames(tmp_path / "run.cod")
    (rst, rt, rhdr, rcrd), = mdio.read_presto_frames(os.path.join(GOLD, "ala3_run.cod"))
    assert st == rst == 100 and t == rt
    # header: total, kinetic, temperature, potential, vdw of step 99
    for i in (2, 3, 4, 5, 7):
        assert abs(hdr[i] - rhdr[i]) <= 1e-4 * abs(rhdr[i]) + 1e-3, (i, hdr[i], rhdr[i])
    d_frame = np.abs(_min_image(crd - rcrd, box)).max()
    solute = np.asarray(s["groups"]["atoms"][s["groups"]["names"].index("solute")])
    d_wrong = np.abs(_min_image(ref["crd"][solute] - rcrd, box)).mean()
    assert d_frame <= 1e-4 and d_frame < 0.05 * d_wrong, (d_frame, d_wrong)
    rows = mod.parse_log(log.getvalue())
    assert [r["step"] for r in rows] == list(range(101))
    for r, g in zip(rows, gold["steps"]):
        for key in ("potential", "kinetic", "total", "vdw", "ele", "bond", "torsion"):
            assert abs(r[key] - g[key]) <= 1e-5 * abs(g[key]) + 1e-4, (r["step"], key, r[key], g[key])


def test_ala3_vmcmd_run_writes_reference_logs(tmp_path):
    """mdio.run with the reference's V-McMD settings writes the virtual-state log line for line
    as the reference did (ala3_vmcmd.json) and its ascii lambda log within 1e-4 relative."""
    g = json.load(open(os.path.join(GOLD, "ala3_vmcmd.json")))
    _, s, _ = _golden()
    p = dict(g["params"], n_steps=g["n_steps"], print_intvl_crd=[], fn_o_crd=[], fn_o_restart=str(tmp_path / "o.restart"),
             fn_o_vmcmd_log=str(tmp_path / "vs.log"), fn_o_extended_lambda=str(tmp_path / "lambda.out"),
             format_o_extended_lambda="ascii")
    mdio.run(s, p, mcmd=g["vmcmd"])
    assert open(tmp_path / "vs.log").read() == "".join("%d\t%d\n" % (a, b) for a, b in g["vs"])
    lam = np.loadtxt(tmp_path / "lambda.out")
    ref = np.array(g["lambda"])
    assert lam.shape == ref.shape and np.max(np.abs(lam - ref) / np.abs(ref)) <= 1e-4
    assert mdio.read_restart(tmp_path / "o.restart")["n_steps"] == g["n_steps"]
