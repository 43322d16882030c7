"""Build recipes for the CPU oracle (TEST INFRASTRUCTURE).

* ``build_oracle()`` compiles the C restatement ``oracle/ogo.c`` into ``oracle/libogo.so``.
* ``build_ref()`` compiles pieces of the reference (myPresto/omegagene) straight from its
  source tree, unmodified, into ``oracle/_ref/``:

  - ``libogref_minicell.so``: MiniCell.cpp + PBC.cpp + CelesteObject.cpp with the
    ``ref_minicell_shim.cpp`` driver (cell assignment + cell-pair list of the reference);
  - ``omegagene_wons``: the all-pairs CPU program (``-DF_WO_NS``), which reproduces
    samples/ala3/log03_md.txt;
  - ``omegagene_ns``: the cell-list CPU program.  MiniCell.cpp is compiled with
    ``-DF_CUDA -DF_ECP`` so that it allocates its coordinate buffer (through the malloc
    stubs of ``ref_minicell_shim.cpp``); every other file is the plain CPU build, so the
    pair list and forces are the reference's CPU code;
  - ``omegagene_og``: the reference's GPU program (its CELESTE_GPU build: every file with
    ``-DF_CUDA``) linked against ``omegagene_b200/libomegagene_celeste.so`` in place of its
    ``cuda_setup.cu``: the drop-in, the reference's own host code driving this engine.

The reference's own CMake build is not used (it requires a .git directory).  Outputs
never go anywhere but ``oracle/`` and ``oracle/_ref/``.
"""
import concurrent.futures as cf
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
# The reference checkout this recipe compiles from, where it lies (read-only; nothing is written
# there).  OG_REFERENCE_ROOT, or the ref_root argument of build_ref, names another checkout.
REF_CHECKOUT = "/root/reference"
REF_ROOT = os.environ.get("OG_REFERENCE_ROOT") or REF_CHECKOUT
REF_OUT = os.path.join(HERE, "_ref")

CORE = [
    "Celeste.cpp", "CelesteObject.cpp", "COMMotion.cpp", "Config.cpp", "Constraint.cpp",
    "ConstraintShake.cpp", "DistRestraint.cpp", "DynamicsMode.cpp", "ElectrostaticObject.cpp",
    "Extend.cpp", "ForceField.cpp", "ForceFieldObject.cpp", "MiniCell.cpp", "MmSystem.cpp",
    "PBC.cpp", "PosRestraint.cpp", "Read.cpp", "RunMode.cpp", "SubBox.cpp", "Thermostat.cpp",
    "Write.cpp", "WriteTrr.cpp", "ZeroMultipoleSum.cpp",
]


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("command failed: %s\n%s%s" % (" ".join(cmd), r.stdout[-4000:], r.stderr[-4000:]))


def _newer(target, sources):
    if not os.path.exists(target):
        return False
    t = os.path.getmtime(target)
    return all(os.path.getmtime(s) <= t for s in sources if os.path.exists(s))


def build_oracle(force=False):
    src = os.path.join(HERE, "ogo.c")
    hdr = os.path.join(HERE, "ogo.h")
    out = os.path.join(HERE, "libogo.so")
    if force or not _newer(out, [src, hdr]):
        _run(["gcc", "-O2", "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-shared", "-o", out, src, "-lm"])
    return out


def reference_available(ref_root=None):
    return os.path.isdir(os.path.join(ref_root or REF_ROOT, "src", "celeste", "core"))


def build_ref(force=False, jobs=8, ref_root=None):
    """Compile the reference pieces; returns the output directory or None if absent."""
    REF_ROOT = ref_root or globals()["REF_ROOT"]
    if not reference_available(REF_ROOT):
        return None
    core = os.path.join(REF_ROOT, "src", "celeste", "core")
    rnd = os.path.join(REF_ROOT, "src", "celeste", "random", "Random.cpp")
    main = os.path.join(core, "main.cpp")
    shim = os.path.join(HERE, "ref_minicell_shim.cpp")
    objdir = os.path.join(REF_OUT, "obj")
    os.makedirs(objdir, exist_ok=True)
    base = ["g++", "-std=c++14", "-O3", "-fPIC", "-w",
            '-DMACRO_BUILD_VERSION="ref"', '-DMACRO_BUILD_TIMESTAMP="ref"',
            "-I", os.path.join(REF_ROOT, "src"), "-I", core]
    jobs_list = []  # (obj, src, extra flags)
    for f in CORE:
        src = os.path.join(core, f)
        stem = f[:-4]
        jobs_list.append((os.path.join(objdir, stem + ".wons.o"), src, ["-DF_WO_NS"]))
        if f == "MiniCell.cpp":
            jobs_list.append((os.path.join(objdir, stem + ".cudaecp.o"), src, ["-DF_CUDA", "-DF_ECP"]))
        jobs_list.append((os.path.join(objdir, stem + ".ns.o"), src, []))
        jobs_list.append((os.path.join(objdir, stem + ".cuda.o"), src, ["-DF_CUDA"]))
    jobs_list.append((os.path.join(objdir, "Random.o"), rnd, []))
    jobs_list.append((os.path.join(objdir, "main.cuda.o"), main, ["-DF_CUDA"]))
    jobs_list.append((os.path.join(objdir, "main.wons.o"), main, ["-DF_WO_NS"]))
    jobs_list.append((os.path.join(objdir, "main.ns.o"), main, []))
    jobs_list.append((os.path.join(objdir, "shim.o"), shim, []))

    def compile_one(job):
        obj, src, extra = job
        if not force and _newer(obj, [src]):
            return
        _run(base + extra + ["-c", src, "-o", obj])

    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        list(ex.map(compile_one, jobs_list))

    o = lambda name: os.path.join(objdir, name)
    wons_objs = [o(f[:-4] + ".wons.o") for f in CORE] + [o("Random.o"), o("main.wons.o")]
    ns_objs = [o(f[:-4] + (".cudaecp.o" if f == "MiniCell.cpp" else ".ns.o")) for f in CORE]
    ns_objs += [o("Random.o"), o("main.ns.o"), o("shim.o")]
    lib_objs = [o("MiniCell.cudaecp.o"), o("PBC.ns.o"), o("CelesteObject.ns.o"), o("shim.o")]
    og_dir = os.path.join(os.path.dirname(HERE), "omegagene_b200")
    og_objs = [o(f[:-4] + ".cuda.o") for f in CORE] + [o("Random.o"), o("main.cuda.o")]
    targets = [
        (os.path.join(REF_OUT, "omegagene_wons"), wons_objs, []),
        (os.path.join(REF_OUT, "omegagene_ns"), ns_objs, []),
        (os.path.join(REF_OUT, "libogref_minicell.so"), lib_objs, ["-shared"]),
    ]
    celeste = os.path.join(og_dir, "libomegagene_celeste.so")
    if os.path.exists(celeste):
        # the drop-in: found at run time relative to the program ($ORIGIN/../../omegagene_b200)
        targets.append((os.path.join(REF_OUT, "omegagene_og"), og_objs,
                        ["-L" + og_dir, "-l:libomegagene_celeste.so", "-l:libomegagene_b200.so",
                         "-Wl,-rpath,$ORIGIN/../../omegagene_b200"]))
    for out, objs, extra in targets:
        libs = [x for x in extra if x.startswith("-l") or x.startswith("-L") or x.startswith("-Wl")]
        flags = [x for x in extra if x not in libs]
        if force or not _newer(out, objs + ([celeste] if out.endswith("omegagene_og") else [])):
            _run(["g++", "-O3", "-fPIC"] + flags + ["-o", out] + objs + libs + ["-lm"])
    return REF_OUT


if __name__ == "__main__":
    print(build_oracle(force=True))
    print(build_ref())
