"""Writes ala3_models.json: the energies the reference printed for steps 0-2 of its ala3 sample
under each electrostatics / nonbond model other than zero-dipole alpha = 0 (run here, where the
reference tree is present; the output is committed).

Each run is the reference's all-pairs CPU program (oracle/_ref/omegagene_wons, built from its
sources by oracle/build.py) on samples/ala3/md.inp.cls with samples/ala3/md.inp.run, --n-steps 2
and the model's options:
* --electrostatic zero-quadrupole / zero-octupole / zero-hexadecapole with --ele-alpha 0;
* zero-dipole / -quadrupole / -octupole / -hexadecapole with --ele-alpha 0.1;
* debye-huckel (dielectric 80, ionic strength 0.15 M, 300 K);
* --nonbond hydrophobicity-scale-lj (epsilon 0.2) with zero-dipole alpha = 0.  The sample's HPS
  records hold lambda = 0 for every type pair; this run rewrites them with
  lambda = ((31 a + 17 b) mod 11) / 10 for the type pair a <= b (1-based), cutoffs unchanged.

Usage: python tests/golden/make_ele_golden.py <reference root>
"""
import importlib.util
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

DH = ["--debye-huckel-dielectric", "80", "--debye-huckel-ionic-strength", "0.15", "--debye-huckel-temperature", "300"]
MODELS = [
    ("zq_a0", ["--electrostatic", "zero-quadrupole", "--ele-alpha", "0"]),
    ("zo_a0", ["--electrostatic", "zero-octupole", "--ele-alpha", "0"]),
    ("zh_a0", ["--electrostatic", "zero-hexadecapole", "--ele-alpha", "0"]),
    ("zd_a01", ["--electrostatic", "zero-dipole", "--ele-alpha", "0.1"]),
    ("zq_a01", ["--electrostatic", "zero-quadrupole", "--ele-alpha", "0.1"]),
    ("zo_a01", ["--electrostatic", "zero-octupole", "--ele-alpha", "0.1"]),
    ("zh_a01", ["--electrostatic", "zero-hexadecapole", "--ele-alpha", "0.1"]),
    ("dh", ["--electrostatic", "debye-huckel", "--ele-alpha", "0"] + DH),
    ("hps", ["--electrostatic", "zero-dipole", "--ele-alpha", "0", "--nonbond", "hydrophobicity-scale-lj",
             "--hydrophobicity-scale-epsiron", "0.2"]),
]


def hps_lambda(t1, t2):
    a, b = min(t1, t2), max(t1, t2)
    return ((31 * a + 17 * b) % 11) / 10.0


def with_hps_lambdas(s):
    """The launch set with the HPS lambdas of hps_lambda() (cutoffs kept)."""
    from omegagene_b200 import cls_io
    t = dict(s["topol"])
    rec = np.frombuffer(t["lj_hps_raw"], cls_io.HPS).copy()
    rec["lam"] = [hps_lambda(int(a), int(b)) for a, b in zip(rec["t1"], rec["t2"])]
    t["lj_hps_raw"] = rec.tobytes()
    return dict(s, topol=t)


def _strip_run_options(text):
    out = []
    for line in text.splitlines():
        key = line.split(";")[0].split("#")[0].split()
        if key and key[0] in ("--n-steps", "--electrostatic", "--ele-alpha", "--print-interval-coord",
                              "--fn-o-coord", "--format-o-coord", "--group-o-coord", "--fn-o-restart"):
            continue
        out.append(line)
    return "\n".join(out) + "\n"


def main(ref_root):
    from omegagene_b200 import cls_io, engine
    spec = importlib.util.spec_from_file_location("make_ala3_golden", os.path.join(HERE, "make_ala3_golden.py"))
    mag = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mag)
    exe = os.path.join(ROOT, "oracle", "_ref", "omegagene_wons")
    sample = os.path.join(ref_root, "samples", "ala3")
    base = _strip_run_options(open(os.path.join(sample, "md.inp.run")).read())
    s = cls_io.read_cls(os.path.join(sample, "md.inp.cls"))
    out = {"source": "oracle/_ref/omegagene_wons (the reference's all-pairs CPU program) on samples/ala3, steps 0-2 "
                     "per model", "hps_lambda": "((31 a + 17 b) mod 11) / 10 for LJ types a <= b (1-based)",
           "models": {}}
    for name, opts in MODELS:
        run = base + "--n-steps 2\n" + "".join("%s %s\n" % (opts[i], opts[i + 1]) for i in range(0, len(opts), 2))
        with tempfile.TemporaryDirectory() as tmp:
            cls_io.write_cls(os.path.join(tmp, "md.inp.cls"), with_hps_lambdas(s) if name == "hps" else s)
            open(os.path.join(tmp, "md.inp.run"), "w").write(run)
            r = subprocess.run([exe, "--cfg", "md.inp.run", "--inp", "md.inp.cls"], cwd=tmp, capture_output=True,
                               text=True, timeout=600)
        steps = mag.parse_log(r.stdout)
        if len(steps) != 3:
            raise SystemExit("%s: %d logged steps, exit %d\n%s" % (name, len(steps), r.returncode, r.stdout[-2000:]))
        out["models"][name] = {"options": opts, "params": engine.parse_run_config(run), "steps": steps}
        print(name, steps[0]["vdw"], steps[0]["ele"], flush=True)
    json.dump(out, open(os.path.join(HERE, "ala3_models.json"), "w"), indent=0)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python %s <reference checkout root>" % os.path.basename(__file__))
    main(sys.argv[1])
