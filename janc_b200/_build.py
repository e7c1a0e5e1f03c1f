"""Build the sm_100a shared library ``janc_b200/libjanc_b200.so`` in-tree.

Translation units: ``jb_strict*.cu`` (-fmad=false, the reference's rounding),
``jb_fast*.cu`` (FMA contraction, FP64 and mixed variants; each variant is
split into parts compiled in parallel, see ``jb_variant.inc``), ``jb_ensemble.cu``
(the persistent batched kernel and its C ABI), ``jb_adjoint.cu`` (the
reverse-mode kernels), ``jb_api.cu`` (the C ABI of the single-case solver),
``jb_noalloc.cu`` and ``jb_probe.cu``.
Compiled with nvcc for ``-gencode arch=compute_100a,code=sm_100a``.
"""
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libjanc_b200.so")
OBJ = os.path.join(HERE, "_objs")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr"]
# the slowest units first: they start before the pool fills
UNITS = [("jb_ensemble.cu", ["-fmad=true"]), ("jb_fast_flux32.cu", ["-fmad=true"]),
         ("jb_fast_god32.cu", ["-fmad=true"]), ("jb_fast_flux64.cu", ["-fmad=true"]),
         ("jb_fast_god64.cu", ["-fmad=true"]), ("jb_fast.cu", ["-fmad=true"]),
         ("jb_strict_flux.cu", ["-fmad=false"]), ("jb_strict_god.cu", ["-fmad=false"]),
         ("jb_strict.cu", ["-fmad=false"]), ("jb_strict_amr.cu", ["-fmad=false"]),
         ("jb_fast_amr.cu", ["-fmad=true"]), ("jb_adjoint.cu", ["-fmad=true"]), ("jb_api.cu", []),
         ("jb_probe.cu", []), ("jb_noalloc.cu", [])]


def _nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _sources():
    return [os.path.join(CSRC, f) for f in os.listdir(CSRC)
            if f.endswith((".cu", ".cuh", ".h", ".inc"))] + [
        os.path.join(HERE, "..", "include", "janc_b200.h")]


def up_to_date():
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(s) <= t for s in _sources())


def build(force=False, verbose=False):
    if not force and up_to_date():
        return LIB
    os.makedirs(OBJ, exist_ok=True)
    nvcc = _nvcc()

    def compile_unit(unit):
        src, extra = unit
        obj = os.path.join(OBJ, src.replace(".cu", ".o"))
        flags = os.environ.get("JB_NVCC_FLAGS", "").split()  # extra -D tuning constants
        cmd = [nvcc] + ARCH + COMMON + extra + flags + ["-c", os.path.join(CSRC, src), "-o", obj]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
        return obj

    with cf.ThreadPoolExecutor(len(UNITS)) as ex:
        objs = list(ex.map(compile_unit, UNITS))
    tmp = LIB + ".tmp"
    cmd = [nvcc] + ARCH + ["-shared", "-o", tmp] + objs + ["-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
