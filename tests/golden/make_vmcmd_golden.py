"""Writes the V-McMD fixtures (run here, where the reference tree and a C++ compiler are present;
the outputs are committed):

* mt19937_vectors.json: draws of std::mt19937 -- the generator random::Random wraps
  (src/celeste/random/Random.cpp:10-28) -- for several seeds, from a few-line C++ program
  compiled with g++ against the C++ standard library.
* ala3_vmcmd.json: the reference's own V-McMD run of its ala3 sample.  The sample's launch set
  (samples/ala3/md.inp.cls) gets a four-state "extended" section (the layout Read::load_ls_vmcmd
  reads, Read.cpp:521-560); md.inp.run gets --extended-ensemble v-mcmd, --random-seed and ascii
  logs of the virtual state and lambda every step.  The run is the reference's all-pairs CPU
  program built from its sources (oracle/_ref/omegagene_wons, oracle/build.py).  Recorded: the
  virtual-state log (WriteTTPVMcMDLog, "step<TAB>state+1"), the lambda log (%14.10e, one row per
  step) and the energies printed per step.  The reference program ends with a segmentation
  fault in its teardown after both logs are closed (its exit path, not the run); the script
  checks that every log line is there.

Usage: python tests/golden/make_vmcmd_golden.py <reference root>
"""
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

MT_SEEDS = [0, 1, 5489, 20261203, 4294967295]
MT_DRAWS = 1400  # three twists

MT_PROGRAM = r"""
#include <cstdio>
#include <cstdlib>
#include <random>
int main(int argc, char **argv) {
    std::mt19937 g;
    g.seed((std::mt19937::result_type)strtoul(argv[1], nullptr, 10));
    int n = atoi(argv[2]);
    for (int i = 0; i < n; i++) printf("%u\n", (unsigned)g());
    return 0;
}
"""

N_STEPS = 200          # --n-steps: steps 0..200 run (the reference's loop plus its last step)
SEED = 20261203        # --random-seed
TRANS_INTERVAL = 2
TEMPERATURE = 300.0
RT = 8.31451 / 4.184 * 1e-3 * TEMPERATURE


def _poly(e0, a, b):
    """d lnP / d lambda = (1 + a x + b x^2) / RT with x = (lambda - e0) / 1000, in raw powers of
    lambda as the reference's files hold it."""
    return [(1 - a * e0 / 1000 + b * e0 * e0 / 1e6) / RT, (a / 1000 - 2 * b * e0 / 1e6) / RT, (b / 1e6) / RT]


def vmcmd_section():
    """Four overlapping states over the potential energies of the sample's first 200 steps
    (-24,700 to -22,500 kcal/mol); the edge states cannot leave the ladder (probability 0)."""
    states = [
        dict(lambda_low=-25000.0, lambda_high=-22000.0, prob_low=0.0, prob_high=0.5, coef=_poly(-23500, 0.05, 0.01)),
        dict(lambda_low=-24000.0, lambda_high=-21000.0, prob_low=0.5, prob_high=0.4, coef=_poly(-22500, -0.04, 0.02)),
        dict(lambda_low=-23500.0, lambda_high=-20000.0, prob_low=0.3, prob_high=0.7, coef=_poly(-21750, 0.03, -0.01)),
        dict(lambda_low=-23000.0, lambda_high=-19000.0, prob_low=0.6, prob_high=0.0, coef=_poly(-21000, -0.02, 0.0)),
    ]
    for s in states:
        s.update(order=len(s["coef"]) - 1, alpha_low=0.0, alpha_high=0.0)
    return {"n_vs": len(states), "interval": TRANS_INTERVAL, "temperature": TEMPERATURE, "states": states,
            "init_vs": 1, "seed": 777}


def make_mt_vectors():
    with tempfile.TemporaryDirectory() as tmp:
        src = os.path.join(tmp, "mt.cpp")
        exe = os.path.join(tmp, "mt")
        open(src, "w").write(MT_PROGRAM)
        subprocess.run(["g++", "-O1", "-std=c++11", src, "-o", exe], check=True)
        out = {}
        for seed in MT_SEEDS:
            r = subprocess.run([exe, str(seed), str(MT_DRAWS)], check=True, capture_output=True, text=True)
            out[str(seed)] = [int(x) for x in r.stdout.split()]
    json.dump({"source": "std::mt19937 of g++ %s (libstdc++), seeded with seed(value)" % _gxx_version(),
               "draws": out}, open(os.path.join(HERE, "mt19937_vectors.json"), "w"))


def _gxx_version():
    return subprocess.run(["g++", "-dumpfullversion"], capture_output=True, text=True).stdout.strip()


def make_ala3_vmcmd(ref_root):
    from omegagene_b200 import cls_io, engine
    spec = __import__("importlib.util").util.spec_from_file_location(
        "make_ala3_golden", os.path.join(HERE, "make_ala3_golden.py"))
    mag = __import__("importlib.util").util.module_from_spec(spec)
    spec.loader.exec_module(mag)
    exe = os.path.join(ROOT, "oracle", "_ref", "omegagene_wons")
    if not os.path.exists(exe):
        raise SystemExit("build the reference programs first: python -c 'from oracle import build; build.build_ref()'")
    sample = os.path.join(ref_root, "samples", "ala3")
    run = open(os.path.join(sample, "md.inp.run")).read()
    run = run.replace("--n-steps                     100", "--n-steps                     %d" % N_STEPS)
    assert "--n-steps                     %d" % N_STEPS in run
    run += ("\n--extended-ensemble v-mcmd\n--random-seed %d\n--fn-o-vmcmd-log vs.log\n"
            "--fn-o-extended-lambda lambda.out\n--format-o-extended-lambda ascii\n"
            "--print-interval-extended-lambda 1\n" % SEED)
    vm = vmcmd_section()
    with tempfile.TemporaryDirectory() as tmp:
        s = cls_io.read_cls(os.path.join(sample, "md.inp.cls"))
        s["vmcmd"] = vm
        cls_io.write_cls(os.path.join(tmp, "md.inp.cls"), s)
        open(os.path.join(tmp, "md.inp.run"), "w").write(run)
        r = subprocess.run([exe, "--cfg", "md.inp.run", "--inp", "md.inp.cls"], cwd=tmp, capture_output=True,
                           text=True, timeout=600)
        vs = [[int(a), int(b)] for a, b in (ln.split() for ln in open(os.path.join(tmp, "vs.log")) if ln.strip())]
        lam = [float(x) for x in open(os.path.join(tmp, "lambda.out")).read().split()]
        steps = mag.parse_log(r.stdout)
        params = engine.parse_run_config(run)
    # every transition step 2..N and every lambda step 1..N is logged (the run completed)
    assert [v[0] for v in vs] == list(range(TRANS_INTERVAL, N_STEPS + 1, TRANS_INTERVAL)), vs[-3:]
    assert len(lam) == N_STEPS and len(steps) == N_STEPS + 1, (len(lam), len(steps))
    # distance of each transition step's lambda from the nearest range bound: the margin a
    # port's lambda may differ by and still take the same decisions
    bounds = np.array([[x["lambda_low"], x["lambda_high"]] for x in vm["states"]]).reshape(-1)
    margin = min(float(np.abs(bounds - lam[st - 1]).min()) for st, _ in vs)
    json.dump({"source": "oracle/_ref/omegagene_wons (the reference's all-pairs CPU program) on samples/ala3 with "
                         "the V-McMD section below; vs = [step, state + 1] lines of --fn-o-vmcmd-log, lambda = "
                         "rows of --fn-o-extended-lambda (steps 1..n_steps), steps = the energies it printed",
               "params": params, "vmcmd": vm, "random_seed": SEED, "n_steps": N_STEPS, "vs": vs, "lambda": lam,
               "lambda_margin": margin, "steps": steps, "reference_exit_status": r.returncode},
              open(os.path.join(HERE, "ala3_vmcmd.json"), "w"), indent=0)
    print("transitions logged %d, lambda margin %.3f kcal/mol, reference exit %d" % (len(vs), margin, r.returncode))


if __name__ == "__main__":
    make_mt_vectors()
    if len(sys.argv) != 2:
        sys.exit("usage: python %s <reference checkout root>" % os.path.basename(__file__))
    make_ala3_vmcmd(sys.argv[1])
