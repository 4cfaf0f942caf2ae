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
# second library: the CPML forward path under the reference's CPML library name
CPML_LIB = os.path.join(LIBDIR, "cuda_regression_CPML.so")

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


def _cpml_sources():
    d = os.path.join(CSRC, "cpml")
    return sorted(os.path.join(d, f) for f in os.listdir(d) if f.endswith(".cu")) + \
        [os.path.join(CSRC, "status.cu")]


def _deps():
    out = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    out.append(os.path.join(ROOT, "include", "otfwi.h"))
    out.append(os.path.join(ROOT, "include", "otfwi_cpml.h"))
    return out


def _stale(target, inputs):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(p) > t for p in inputs)


def _obj(src):
    rel = os.path.relpath(src, CSRC).replace(os.sep, "_")
    return os.path.join(OBJDIR, rel[:-3] + ".o")


def build(verbose=False, ptxas_info=False):
    """Compile the library if any source changed; return the library path."""
    os.makedirs(OBJDIR, exist_ok=True)
    nvcc = _nvcc()
    srcs = _sources()
    deps = _deps()
    jobs = []
    cpml_srcs = _cpml_sources()
    for s in sorted(set(srcs) | set(cpml_srcs)):
        obj = _obj(s)
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
    objs = [_obj(s) for s in srcs]
    cobjs = [_obj(s) for s in cpml_srcs]
    if jobs or _stale(CPML_LIB, cobjs):
        r = subprocess.run([nvcc, "-shared", "-o", CPML_LIB] + cobjs + ARCH, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"CPML link failed:\n{r.stdout}\n{r.stderr}")
    if jobs or _stale(LIB, objs):
        cmd = [nvcc, "-shared", "-o", LIB] + objs + ARCH + ["-lcuda", "-lcufft"]
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
    # the recipe knows where the reference tree lies (OTFWI_REF overrides it)
    # and builds nothing where it is absent
    r = subprocess.run(["make", "-C", odir, "ref-if-present"], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"reference build failed:\n{r.stdout}\n{r.stderr}")


if __name__ == "__main__":
    print(build(verbose=True, ptxas_info="-v" in sys.argv))
    build_oracle()
