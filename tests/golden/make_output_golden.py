"""Copies the reference's own output files of its ala3 sample run into the fixtures (run here,
where the reference tree is present; the copies are committed):

* ala3_run.cod: the presto trajectory (--print-interval-coord 100, --group-o-coord solute: one
  frame, labelled step 100, of the 66 solute atoms);
* ala3_run_o.restart: the restart written after the 100-step loop;
* ala3_log_blocks.txt: the energy blocks printed for steps 0, 1, 99 and 100
  (samples/ala3/log03_md.txt).

Usage: python tests/golden/make_output_golden.py <reference root>
"""
import os
import re
import shutil
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def main(ref_root):
    sample = os.path.join(ref_root, "samples", "ala3")
    shutil.copyfile(os.path.join(sample, "run.cod"), os.path.join(HERE, "ala3_run.cod"))
    shutil.copyfile(os.path.join(sample, "run_o.restart"), os.path.join(HERE, "ala3_run_o.restart"))
    text = open(os.path.join(sample, "log03_md.txt")).read()
    blocks = {int(m.group(1)): m.group(0) for m in re.finditer(r"Step:\s+(\d+)\s+Time:.*?Comput Time:[^\n]*\n", text, re.S)}
    with open(os.path.join(HERE, "ala3_log_blocks.txt"), "w") as f:
        for k in (0, 1, 99, 100):
            f.write(blocks[k])


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python %s <reference checkout root>" % os.path.basename(__file__))
    main(sys.argv[1])
