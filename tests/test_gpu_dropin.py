"""The drop-in: the reference's own program, built from its sources as its CELESTE_GPU build
(-DF_CUDA) and linked against libomegagene_celeste.so instead of its cuda_setup.cu
(oracle/_ref/omegagene_og, made by oracle/build.py), runs the ala3 sample with the cell-pair list
and the pair forces computed by this engine, and its host code doing the rest (MiniCell's host
grid, bonded and excluded-pair terms, leapfrog, SHAKE, COM cancel).

Its printed energies are checked against two references on the same inputs:
  * the reference's CPU cell-list program (oracle/_ref/omegagene_ns): the same host program
    with the pair list and forces computed on the CPU.  Step 0: VDW, Ele and the terms that
    depend on them (potential, total, and the kinetic energy of the half-step velocities) within
    1e-6 relative (FP32 pair terms summed in another order), the bonded terms to the printed 11
    digits; over 20 steps every term within 1e-5 |E| + 1e-3 kcal/mol;
  * the sample's own log (samples/ala3/log03_md.txt, its all-pairs build; fixture
    tests/golden/ala3_log.json): at step 0 the bonded terms to the printed digits and VDW
    within 1e-6.  The cell-list builds report Ele without the excluded-pair ZD energy (SubBox::
    calc_energy overwrites pote_ele with the pair sum, SubBox.cpp:939-941), so Ele plus that
    energy, computed by the oracle at the start, must equal the logged Ele within 1e-3.
"""
import importlib.util
import json
import os
import subprocess
import tempfile

import numpy as np
import pytest

from omegagene_b200 import cls_io
from oracle import ogo

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
N_STEPS = 20
TERMS = ("bond", "angle", "torsion", "improper", "vdw14", "ele14", "vdw", "ele", "potential", "kinetic", "total",
         "temperature")

# the sample's run settings (samples/ala3/md.inp.run), with --expected-num-density 1.0: the
# reference sizes its per-column arrays from that density and overflows them at its default
RUN = """--mode md
--integrator leapfrog-presto
--cutoff 12.0
--n-steps {n}
--time-step 2.0
--electrostatic zero-dipole
--ele-alpha 0
--thermostat none
--temperature 300
--com-motion cancel
--com-cancel-group-name solute
--com-cancel-group-name solvent
--print-interval-log 1
--print-interval-coord 1000
--fn-o-coord run.cod
--format-o-coord presto
--fn-o-log md.log
--fn-o-energy md.ene
--fn-o-restart run_o.restart
--nsgrid-cutoff 13.0
--nsgrid-update-intvl 10
--constraint shake
--const-max-loops 1000
--const-tolerance 0.0000001
--expected-num-density 1.0
"""


def _golden():
    spec = importlib.util.spec_from_file_location("make_ala3_golden", os.path.join(HERE, "golden", "make_ala3_golden.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _run(program, system, n_steps):
    exe = os.path.join(ROOT, "oracle", "_ref", program)
    if not os.path.exists(exe):
        pytest.skip("oracle/_ref/%s was not built (reference sources absent at build time)" % program)
    with tempfile.TemporaryDirectory() as tmp:
        cls_io.write_cls(os.path.join(tmp, "md.inp.cls"), system)
        open(os.path.join(tmp, "md.inp.run"), "w").write(RUN.format(n=n_steps))
        r = subprocess.run([exe, "--cfg", "md.inp.run", "--inp", "md.inp.cls"], cwd=tmp, capture_output=True,
                           text=True, timeout=900)
    steps = _golden().parse_log(r.stdout)
    assert r.returncode == 0 and len(steps) == n_steps + 1, (program, r.returncode, len(steps), r.stdout[-3000:],
                                                             r.stderr[-3000:])
    return steps


@pytest.fixture(scope="module")
def runs():
    system = _golden().load_system()
    # the sample's empty restraint sections (the reference frees the restraint arrays at exit
    # whether or not it loaded any)
    system["raw"] = {"dist_restraint": b"\0\0\0\0", "pos_restraint": b"\0\0\0\0"}
    return system, _run("omegagene_og", system, N_STEPS), _run("omegagene_ns", system, N_STEPS)


def test_dropin_matches_reference_cell_list_program(runs):
    _, og, ns = runs
    for k in TERMS:
        # the pair terms differ in the FP32 summation order, and with them the step-0 half-step
        # velocities behind the kinetic energy; the host's bonded terms are the same arithmetic
        tol = 1e-6 * abs(ns[0][k]) if k in ("vdw", "ele", "potential", "total", "kinetic", "temperature") else 0.0
        assert abs(og[0][k] - ns[0][k]) <= tol, ("step 0", k, og[0][k], ns[0][k])
    for a, b in zip(og, ns):
        for k in TERMS:
            assert abs(a[k] - b[k]) <= 1e-5 * abs(b[k]) + 1e-3, (a["step"], k, a[k], b[k])


def test_dropin_matches_sample_log(runs):
    system, og, _ = runs
    log = json.load(open(os.path.join(HERE, "golden", "ala3_log.json")))["steps"][0]
    for k in ("bond", "angle", "torsion", "improper", "vdw14", "ele14"):
        assert og[0][k] == log[k], (k, og[0][k], log[k])
    assert abs(og[0]["vdw"] - log["vdw"]) <= 1e-6 * abs(log["vdw"])
    # the excluded-pair ZD energy at the start (FP32, as the reference's host computes it)
    n, t = system["n_atoms"], system["topol"]
    nb = cls_io.nb15off_table(n, t["nb15off_pairs"])
    pbc = ogo.make_pbc(system["pbc_val"])
    crd = ogo.wrap_inbox(pbc, system["crd"]).reshape(-1)
    z, b, f = ogo.zd_constants(12.0)
    ep = ogo.excess_pairs(n, nb).reshape(-1).astype(np.int32)
    exc = ogo.lib().ogo_excess_f32(pbc, len(ep) // 2, ep, crd, t["charge"].astype(np.float32), b, f, np.zeros(3 * n))
    assert abs(og[0]["ele"] + exc - log["ele"]) <= 1e-3, (og[0]["ele"], exc, log["ele"])
