"""Builds the native parts of sinksim_b200 in the source tree.

  libsinksim_b200.so      the engine: sm_100a kernels (the batch and its adjoint), the C++ host and the C ABI of
                          include/sinksim_b200.h
  bin/sinksim_cuda_run    drop-in for the reference's GPU batch runner (apps/sinksim_cuda_run.cpp)
  bin/sinksim_sweep       drop-in for the reference's sweep runner (apps/sinksim_sweep.cpp), on the GPU

Floating point is compiled without contraction (nvcc -fmad=false, host -ffp-contract=off -fexcess-precision=standard):
the portable numerics must round every operation once, as the reference's strict build does
(cmake/StrictFloatingPoint.cmake:12-17 of the reference).

    python -m sinksim_b200.build [--jobs N] [--force]
"""
import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(ROOT, "_build")
LIB = os.path.join(HERE, "libsinksim_b200.so")
BIN = os.path.join(HERE, "bin")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
HOST_FLAGS = "-fPIC,-ffp-contract=off,-fno-fast-math,-fexcess-precision=standard,-Wall,-Wextra,-Wno-unused-parameter"
NVCC_FLAGS = ARCH + ["-O3", "-std=c++17", "-fmad=false", "-lineinfo", "-Xptxas", "-v", "-diag-suppress", "222",
                     "-Xcompiler", HOST_FLAGS, "-I" + os.path.join(ROOT, "include"), "-I" + CSRC]

SOURCES = ["batch_kernel.cu", "adjoint_kernel.cu", "portable_math.cu", "probes.cu", "batch.cpp", "adjoint.cpp", "model.cpp", "json.cpp",
           "sweep.cpp", "capi.cpp"]
APPS = ["sinksim_cuda_run", "sinksim_sweep"]


def nvcc():
    for c in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _compile(src, obj, log):
    cmd = [nvcc()] + NVCC_FLAGS + ["-x", "cu" if src.endswith(".cu") else "c++", "-c", src, "-o", obj]
    if not src.endswith(".cu"):
        # host-only C++ through nvcc: same flags, no device code
        cmd = [nvcc()] + [f for f in NVCC_FLAGS if f not in ("-lineinfo",)] + ["-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    with open(log, "w") as f:
        f.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
    if r.returncode != 0:
        raise RuntimeError(f"compiling {os.path.basename(src)} failed:\n{r.stdout}{r.stderr}")
    return obj


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(jobs=8, force=False, verbose=False):
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(BIN, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    headers.append(os.path.join(ROOT, "include", "sinksim_b200.h"))
    objs, todo = [], []
    for s in SOURCES:
        src = os.path.join(CSRC, s)
        obj = os.path.join(BUILD, s + ".o")
        objs.append(obj)
        if force or _stale(obj, [src] + headers):
            todo.append((src, obj, os.path.join(BUILD, s + ".log")))
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        for f in [ex.submit(_compile, *t) for t in todo]:
            f.result()
    if force or todo or _stale(LIB, objs):
        cmd = [nvcc()] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"linking {LIB} failed:\n{r.stdout}{r.stderr}")
    for app in APPS:
        src = os.path.join(CSRC, "apps", app + ".cpp")
        exe = os.path.join(BIN, app)
        if force or _stale(exe, [src, LIB] + headers):
            cmd = [nvcc()] + ["-O2", "-std=c++17", "-Xcompiler", HOST_FLAGS, "-I" + os.path.join(ROOT, "include"), "-I" + CSRC,
                              src, "-o", exe, "-L" + HERE, "-lsinksim_b200", "-Xlinker", "-rpath,$ORIGIN/.."]
            r = subprocess.run(cmd, capture_output=True, text=True)
            if r.returncode != 0:
                raise RuntimeError(f"building {app} failed:\n{r.stdout}{r.stderr}")
    if verbose:
        for s in SOURCES:
            if s.endswith(".cu"):
                print(open(os.path.join(BUILD, s + ".log")).read())
    return LIB


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--jobs", type=int, default=8)
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    a = ap.parse_args(argv)
    print(build(a.jobs, a.force, a.verbose))


if __name__ == "__main__":
    sys.exit(main())
