"""Build of the in-tree CUDA library (sm_100a) and of the CPU oracle.

``build()`` compiles every ``csrc/*.cu`` into ``otfwi_b200/lib/libotfwi.so``
with nvcc for sm_100a (no JIT, no torch extension cache) and also writes the
library under the file name the reference wrapper loads,
``lib/cuda_regression_PML_single.so``. Objects are rebuilt only when a source
or header is newer than the library.
"""
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIBDIR = os.path.join(PKG, "lib")
OBJDIR = os.path.join(PKG, "lib", "obj")
LIB = os.path.join(LIBDIR, "libotfwi.so")
DROPIN = os.path.join(LIBDIR, "cuda_regression_PML_single.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--fmad=true",
           "-Xptxas", "-warn-spills"] + ARCH


def _nvcc():
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the Otfwi CUDA library cannot be built")


def _sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))


def _deps():
    out = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    out.append(os.path.join(ROOT, "include", "otfwi.h"))
    return out


def _stale(target, inputs):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(p) > t for p in inputs)


def build(verbose=False, ptxas_info=False):
    """Compile the library if any source changed; return the library path."""
    os.makedirs(OBJDIR, exist_ok=True)
    nvcc = _nvcc()
    srcs = _sources()
    deps = _deps()
    jobs = []
    for s in srcs:
        obj = os.path.join(OBJDIR, os.path.basename(s)[:-3] + ".o")
        if _stale(obj, [s] + deps):
            cmd = [nvcc, "-c", s, "-o", obj, "-I", os.path.join(ROOT, "include")] + NVFLAGS
            if ptxas_info:
                cmd += ["-Xptxas", "-v"]
            jobs.append((s, cmd))

    def run(job):
        src, cmd = job
        r = subprocess.run(cmd, capture_output=True, text=True)
        return src, r

    if jobs:
        with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 4))) as ex:
            for src, r in ex.map(run, jobs):
                if verbose or ptxas_info:
                    sys.stdout.write(r.stdout + r.stderr)
                if r.returncode != 0:
                    raise RuntimeError(f"nvcc failed on {src}:\n{r.stdout}\n{r.stderr}")
    objs = [os.path.join(OBJDIR, os.path.basename(s)[:-3] + ".o") for s in srcs]
    if jobs or _stale(LIB, objs):
        cmd = [nvcc, "-shared", "-o", LIB] + objs + ARCH + ["-lcuda"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
        shutil.copyfile(LIB, DROPIN)
    elif not os.path.exists(DROPIN):
        shutil.copyfile(LIB, DROPIN)
    return LIB


def build_oracle():
    """Compile the CPU oracle (oracle/liborc.so); and, where the reference
    sources are present, the reference library oracle/_ref/ (test infra)."""
    odir = os.path.join(ROOT, "oracle")
    r = subprocess.run(["make", "-C", odir, "all"], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"oracle build failed:\n{r.stdout}\n{r.stderr}")
    ref = os.environ.get("OTFWI_REF", "/root/reference")
    if os.path.isdir(os.path.join(ref, "simulator", "src")):
        r = subprocess.run(["make", "-C", odir, "ref", f"REF={ref}"], capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"reference build failed:\n{r.stdout}\n{r.stderr}")


if __name__ == "__main__":
    print(build(verbose=True, ptxas_info="-v" in sys.argv))
    build_oracle()
