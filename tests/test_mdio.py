"""Output formats against the reference's own files (no GPU): the restart and presto trajectory
of its ala3 sample run and the energy blocks it printed (fixtures from
tests/golden/make_output_golden.py), plus the config keys that drive the outputs."""
import importlib.util
import io
import os
import struct

import numpy as np

from omegagene_b200 import engine, mdio

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden")


def _log_steps():
    spec = importlib.util.spec_from_file_location("make_ala3_golden", os.path.join(GOLD, "make_ala3_golden.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    text = open(os.path.join(GOLD, "ala3_log_blocks.txt")).read()
    return {r["step"]: r for r in mod.parse_log(text)}, text


def test_restart_reproduces_reference_file(tmp_path):
    src = os.path.join(GOLD, "ala3_run_o.restart")
    r = mdio.read_restart(src)
    assert r["n_atoms"] == r["n_vel"] == 6207 and r["n_steps"] == 100 and r["time"] == 200.0
    steps, _ = _log_steps()
    # the restart after the 100-step loop carries step 99's energies
    assert float("%.10e" % r["e_potential"]) == steps[99]["potential"]
    assert float("%.10e" % r["e_kinetic"]) == steps[99]["kinetic"]
    out = tmp_path / "o.restart"
    mdio.write_restart(out, r["n_steps"], r["time"], r["e_potential"], r["e_kinetic"], r["crd"], r["vel"],
                       title=r["title"])
    assert open(out, "rb").read() == open(src, "rb").read()


def test_presto_frame_reproduces_reference_file():
    src = open(os.path.join(GOLD, "ala3_run.cod"), "rb").read()
    (step, time, hdr, crd), = mdio.read_presto_frames(os.path.join(GOLD, "ala3_run.cod"))
    assert step == 100 and time == 200.0 and crd.shape == (66, 3)
    steps, _ = _log_steps()
    e = dict(steps[99])  # frame 100 holds step 99's energies
    assert mdio.presto_frame(step, time, e, crd, cpu_time=hdr[1]) == src


def test_log_blocks_reproduce_reference_text():
    steps, text = _log_steps()
    ours = ""
    for k in (0, 1, 99, 100):
        e = steps[k]
        comput = float(text.split("Step: %8d" % k)[1].split("Comput Time:")[1].split()[0])
        ours += mdio.log_block(k, 2.0 * k, e, comput_time=comput)
    assert ours == text


def test_gromacs_frame_layout():
    crd = np.array([[1.0, 2.0, 3.0], [4.0, 5.0, 6.0]])
    b = mdio.gromacs_frame(7, 14.0, [30.0, 40.0, 50.0], crd)
    magic, n1, n2 = struct.unpack_from("<iii", b, 0)
    assert (magic, n1, n2) == (1993, 13, 12) and b[12:24] == b"GMX_trn_file"
    f = struct.unpack_from("<13i", b, 24)
    assert f[2] == 72 and f[7] == 48 and f[8] == 0 and f[10] == 2 and f[11] == 7
    t, lam = struct.unpack_from("<dd", b, 76)
    assert t == 14.0 and lam == 0.0
    box = np.frombuffer(b, "<f8", 9, 92)
    assert list(box[[0, 4, 8]]) == [3.0, 4.0, 5.0]
    x = np.frombuffer(b, "<f8", 6, 164).reshape(2, 3)
    assert np.allclose(x, crd * 0.1) and len(b) == 164 + 48


def test_run_config_output_keys():
    p = engine.parse_run_config("--n-steps 100\n--print-interval-log 1\n--print-interval-coord 100\n"
                                "--fn-o-coord run.cod\n--format-o-coord presto\n--group-o-coord solute\n"
                                "--fn-o-restart run_o.restart\n--print-interval-restart 50\n")
    assert p["n_steps"] == 100 and p["print_intvl_crd"] == [100] and p["fn_o_crd"] == ["run.cod"]
    assert p["group_o_crd"] == ["solute"] and p["fn_o_restart"] == "run_o.restart"
    assert p["print_intvl_restart"] == 50 and p["print_intvl_log"] == 1 and p["format_o_crd"] == "presto"


def test_lambda_log_header():
    assert mdio.lambda_log_header() == struct.pack("<iii", 66261, 8, 1)


def test_apply_restart():
    r = mdio.read_restart(os.path.join(GOLD, "ala3_run_o.restart"))
    s = {"n_atoms": 6207, "crd": np.zeros((6207, 3)), "vel": np.zeros((6207, 3))}
    t = mdio.apply_restart(s, r)
    assert np.array_equal(t["crd"], r["crd"]) and np.array_equal(t["vel"], r["vel"]) and not s["crd"].any()
