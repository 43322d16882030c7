"""Builds the CUDA engine for sm_100a in-tree: omegagene_b200/libomegagene_b200.so."""
import concurrent.futures as cf
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libomegagene_b200.so")
# the reference's CELESTE_GPU entry points on top of the engine (include/omegagene_celeste.h)
CELESTE_SRC = "og_celeste.cpp"
CELESTE_OUT = os.path.join(HERE, "libomegagene_celeste.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
SOURCES = ["og_grid.cu", "og_pair.cu", "og_integrate.cu", "og_engine.cu", "og_noalloc.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")


def _flags(src):
    f = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-I", INCLUDE] + ARCH
    if src == "og_grid.cu":
        # the cell-membership float arithmetic must not be contracted into FMAs
        f.append("-fmad=false")
    if src == "og_pair.cu":
        # no pair term comes near the subnormal range; flushing lets rsqrtf be one instruction
        f.append("-ftz=true")
    return f


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("%s\n%s%s" % (" ".join(cmd), r.stdout, r.stderr))
    return r.stdout + r.stderr


def build_celeste(force=False):
    """libomegagene_celeste.so: og_celeste.cpp against the engine library, found at run time
    beside it ($ORIGIN)."""
    src = os.path.join(CSRC, CELESTE_SRC)
    deps = [src, OUT, os.path.join(INCLUDE, "omegagene_celeste.h"), os.path.join(INCLUDE, "omegagene_b200.h")]
    if not force and os.path.exists(CELESTE_OUT) and os.path.getmtime(CELESTE_OUT) >= max(
            os.path.getmtime(d) for d in deps):
        return CELESTE_OUT
    _run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-I", INCLUDE, "-o", CELESTE_OUT, src, "-L", HERE,
          "-l:libomegagene_b200.so", "-Wl,-rpath,$ORIGIN"])
    return CELESTE_OUT


def build(force=False, verbose=False):
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f != CELESTE_SRC] + [
        os.path.join(INCLUDE, "omegagene_b200.h")]
    newest = max(os.path.getmtime(d) for d in deps)
    if not force and os.path.exists(OUT) and os.path.getmtime(OUT) >= newest:
        build_celeste(force)
        return OUT

    def one(src):
        obj = os.path.join(objdir, src.replace(".cu", ".o"))
        out = _run([NVCC, "-c", os.path.join(CSRC, src), "-o", obj] + _flags(src) +
                   (["-Xptxas", "-v"] if verbose else []))
        return obj, out

    with cf.ThreadPoolExecutor(len(SOURCES)) as ex:
        res = list(ex.map(one, SOURCES))
    if verbose:
        for _, out in res:
            print(out)
    _run([NVCC, "-shared", "-o", OUT] + [o for o, _ in res] + ARCH + ["-lcudart"])
    build_celeste(True)
    return OUT


if __name__ == "__main__":
    import sys
    print(build(force=True, verbose="-v" in sys.argv))
