"""Writes the velocity-scaling thermostat fixture (run here, where the reference tree is present;
the output is committed):

* ala3_thermo.json: the reference's own runs of its ala3 sample (samples/ala3/md.inp.cls and
  md.inp.run) with the velocity-scaling thermostat switched on, through its all-pairs CPU
  program built from its sources (oracle/_ref/omegagene_wons, oracle/build.py).  Three runs:

  - "shake": --thermostat scaling at 300 K with the sample's SHAKE; every step takes the
    iterative thermostat-with-SHAKE loop (ThermostatScaling::apply_thermostat_with_shake,
    Thermostat.cpp:86-170, from DynamicsModePresto::apply_constraint, DynamicsMode.cpp:562-575);
  - "shake_heating": the same with --temperature-init 200 and --heating-steps 20, so the target
    temperature ramps (SubBox::update_thermostat, SubBox.cpp:1745-1757);
  - "noshake": --constraint none, dt 0.5 fs, --berendsen-tau 0.01: the unconstrained scaling
    (ThermostatScaling::apply_thermostat, Thermostat.cpp:57-84, from calc_in_each_step,
    DynamicsMode.cpp:526-532).

  Recorded per run: the md.inp.run text, the parsed run parameters and every energy block the
  program printed (steps 0..n_steps).

Usage: python tests/golden/make_thermo_golden.py <reference checkout root>
"""
import importlib.util
import json
import os
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

N_STEPS = 40

RUNS = {
    "shake": {"--thermostat": "scaling"},
    "shake_heating": {"--thermostat": "scaling", "--temperature-init": "200", "--heating-steps": "20"},
    "noshake": {"--thermostat": "scaling", "--constraint": "none", "--time-step": "0.5", "--berendsen-tau": "0.01"},
}


def _set(run_text, key, value):
    """The sample's md.inp.run with `key` set to `value` (an existing active line replaced, else
    appended); lines commented out with ';' stay as they are."""
    out, done = [], False
    for ln in run_text.splitlines():
        tok = ln.split()
        if tok and tok[0] == key:
            out.append("%s %s" % (key, value))
            done = True
        else:
            out.append(ln)
    if not done:
        out.append("%s %s" % (key, value))
    return "\n".join(out) + "\n"


def main(ref_root):
    from omegagene_b200 import engine
    spec = importlib.util.spec_from_file_location("make_ala3_golden", os.path.join(HERE, "make_ala3_golden.py"))
    mag = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mag)
    exe = os.path.join(ROOT, "oracle", "_ref", "omegagene_wons")
    if not os.path.exists(exe):
        raise SystemExit("build the reference programs first: python -c 'from oracle import build; build.build_ref()'")
    sample = os.path.join(ref_root, "samples", "ala3")
    base = open(os.path.join(sample, "md.inp.run")).read()
    out = {"source": "oracle/_ref/omegagene_wons (the reference's all-pairs CPU program) on samples/ala3, "
                     "md.inp.run with the settings of each run; steps = the energies it printed",
           "n_steps": N_STEPS, "runs": {}}
    for name, opts in RUNS.items():
        run = _set(base, "--n-steps", str(N_STEPS))
        for k, v in opts.items():
            run = _set(run, k, v)
        with tempfile.TemporaryDirectory() as tmp:
            os.symlink(os.path.join(sample, "md.inp.cls"), os.path.join(tmp, "md.inp.cls"))
            open(os.path.join(tmp, "md.inp.run"), "w").write(run)
            r = subprocess.run([exe, "--cfg", "md.inp.run", "--inp", "md.inp.cls"], cwd=tmp, capture_output=True,
                               text=True, timeout=1200)
        steps = mag.parse_log(r.stdout)
        if r.returncode != 0 or len(steps) != N_STEPS + 1:
            raise SystemExit("%s: reference exit %d, %d energy blocks\n%s" % (name, r.returncode, len(steps),
                                                                             r.stdout[-2000:]))
        out["runs"][name] = {"options": opts, "run": run, "params": engine.parse_run_config(run), "steps": steps}
        print(name, "T(0..3) =", [round(s["temperature"], 3) for s in steps[:4]])
    json.dump(out, open(os.path.join(HERE, "ala3_thermo.json"), "w"), indent=0)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python %s <reference checkout root>" % os.path.basename(__file__))
    main(sys.argv[1])
