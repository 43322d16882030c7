"""Writes the ala3 fixtures from the reference's own sample (run here, where the reference tree
is present; the outputs are committed):

* ala3_log.json: the energies the reference printed for steps 0-100 of its sample run
  (samples/ala3/log03_md.txt, all-pairs CPU build, md.inp.run: 2 fs, SHAKE, no thermostat,
  zero-dipole alpha 0, cutoff 12 A, COM cancel on the solute and solvent groups).
* ala3_system.npz: the sample's launch set (samples/ala3/md.inp.cls) as arrays, so that tests on a
  machine without the reference tree can rebuild the system dict.

Usage: python tests/golden/make_ala3_golden.py <reference root>
"""
import json
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

LABELS = {"Total": "total", "Potential": "potential", "Kinetic": "kinetic", "Bond": "bond", "Angle": "angle",
          "Torsion": "torsion", "Improper": "improper", "14-VDW": "vdw14", "14-Ele": "ele14", "VDW": "vdw",
          "Ele": "ele", "Temperature": "temperature"}


def parse_log(text):
    steps = []
    for blk in re.split(r"(?=Step:\s+\d+\s+Time)", text)[1:]:
        row = {"step": int(re.match(r"Step:\s+(\d+)", blk).group(1))}
        for lab, key in LABELS.items():
            m = re.search(r"(?<![\w-])%s:\s+([-0-9.eE+]+)" % re.escape(lab), blk)
            if m:
                row[key] = float(m.group(1))
        steps.append(row)
    return steps


def main(ref_root):
    from omegagene_b200 import cls_io
    sample = os.path.join(ref_root, "samples", "ala3")
    from omegagene_b200 import engine
    steps = parse_log(open(os.path.join(sample, "log03_md.txt")).read())
    params = engine.parse_run_config(open(os.path.join(sample, "md.inp.run")).read())
    json.dump({"source": "samples/ala3/log03_md.txt of the reference (all-pairs CPU build)",
               "inputs": "samples/ala3/md.inp.cls with samples/ala3/md.inp.run (parsed into params)",
               "params": params, "printed_digits": 11, "steps": steps},
              open(os.path.join(HERE, "ala3_log.json"), "w"), indent=0)
    s = cls_io.read_cls(os.path.join(sample, "md.inp.cls"))
    t, c, g = s["topol"], s["constraint"], s["groups"]
    arr = {"pbc_val": s["pbc_val"], "crd": s["crd"], "vel": s["vel"], "dof_extra": np.int32(s["dof_extra"]),
           "charge": t["charge"], "mass": t["mass"], "atom_type": t["atom_type"], "n_lj_types": np.int32(t["n_lj_types"]),
           "lj_pairs": t["lj_pairs"], "bonds": t["bonds"], "angles": t["angles"], "torsions": t["torsions"],
           "impros": t["impros"], "nb14_atoms": t["nb14"]["atoms"], "nb14_types": t["nb14"]["types"],
           "nb14_coeff_vdw": t["nb14"]["coeff_vdw"], "nb14_coeff_ele": t["nb14"]["coeff_ele"],
           "nb15off_pairs": t["nb15off_pairs"], "lj_hps_raw": np.frombuffer(t["lj_hps_raw"], np.uint8)}
    for k in ("pair_atoms", "pair_dist", "trio_atoms", "trio_dist", "quad_atoms", "quad_dist"):
        arr["cons_" + k] = c[k]
    arr["group_names"] = np.array(g["names"])
    for i, a in enumerate(g["atoms"]):
        arr["group_atoms_%d" % i] = np.asarray(a, np.int32)
    np.savez_compressed(os.path.join(HERE, "ala3_system.npz"), **arr)


def load_system(path=os.path.join(HERE, "ala3_system.npz")):
    """The ala3 launch set as the system dict cls_io.read_cls returns (the fields the engine,
    the oracle and the writer use)."""
    z = np.load(path)
    names = [str(x) for x in z["group_names"]]
    topol = {"charge": z["charge"], "mass": z["mass"], "atom_type": z["atom_type"], "n_lj_types": int(z["n_lj_types"]),
             "lj_pairs": z["lj_pairs"], "bonds": z["bonds"], "angles": z["angles"], "torsions": z["torsions"],
             "impros": z["impros"],
             "nb14": {"atoms": z["nb14_atoms"], "types": z["nb14_types"], "coeff_vdw": z["nb14_coeff_vdw"],
                      "coeff_ele": z["nb14_coeff_ele"]},
             "nb15off_pairs": z["nb15off_pairs"],
             "lj_hps_raw": z["lj_hps_raw"].tobytes() if "lj_hps_raw" in z else b""}
    cons = {k: z["cons_" + k] for k in ("pair_atoms", "pair_dist", "trio_atoms", "trio_dist", "quad_atoms", "quad_dist")}
    return {"pbc_val": z["pbc_val"], "n_atoms": len(z["crd"]), "crd": z["crd"], "vel": z["vel"], "topol": topol,
            "constraint": cons, "groups": {"names": names, "atoms": [z["group_atoms_%d" % i] for i in range(len(names))]},
            "dof_extra": int(z["dof_extra"])}


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python %s <reference checkout root>" % os.path.basename(__file__))
    main(sys.argv[1])
