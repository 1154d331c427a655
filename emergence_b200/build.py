"""Build the CUDA library libemergence_b200.so in-tree (sm_100a only).

Usage: python -m emergence_b200.build  (or import and call build()).

Translation units and their FMA policy:
  uniform.cu      host object, ghost/CFL/control kernels, C ABI  -fmad=false
  amr.cu          block-AMR host object, AMR kernels, C ABI      -fmad=false
  batch1d.cu      batched independent 1-D lines, C ABI           -fmad=false
  adjoint.cu      discrete adjoint of the uniform FP64 step      -fmad=false
  five.cu         five-equation two-phase system, C ABI           -fmad=false
  sweep_f64.cu    plain FP64 fused sweep                          -fmad=false
  sweep_mixed.cu  FP32-flux fused sweep                           -fmad=true
  sweep_fast.cu   fast FP64 fused sweep (within 1e-12)            -fmad=true
  five_fast.cu    fast FP64 five-equation sweep                   -fmad=true
The plain FP64 units keep every multiply and add separately rounded so that
their results round exactly as the reference CPU solver's.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libemergence_b200.so")
OUT_BC = os.path.join(HERE, "libemergence_b200_bc.so")
BUILD = os.path.join(HERE, "_build")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
          "-Xcompiler", "-ffp-contract=off", "--expt-relaxed-constexpr"]
UNITS = [
    ("uniform.cu", ["-fmad=false"]),
    ("amr.cu", ["-fmad=false"]),
    ("batch1d.cu", ["-fmad=false"]),
    ("adjoint.cu", ["-fmad=false"]),
    ("five.cu", ["-fmad=false"]),
    ("sweep_f64.cu", ["-fmad=false"]),
    ("sweep_mixed.cu", ["-fmad=true", "-use_fast_math"]),
    ("sweep_fast.cu", ["-fmad=true"]),
    ("five_fast.cu", ["-fmad=true"]),
]


def _nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _build_one(out, objdir, extra, verbose, force):
    os.makedirs(objdir, exist_ok=True)
    nvcc = _nvcc()
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    headers.append(os.path.join(HERE, "..", "include", "emergence_b200.h"))
    objs, jobs = [], []
    for src, flags in UNITS:
        s = os.path.join(CSRC, src)
        o = os.path.join(objdir, src.replace(".cu", ".o"))
        objs.append(o)
        if force or _stale(o, [s] + headers + [__file__]):
            cmd = [nvcc] + ARCH + COMMON + flags + extra + ["-c", s, "-o", o]
            if verbose:
                print(" ".join(cmd))
            jobs.append(subprocess.Popen(cmd))
    if any(j.wait() != 0 for j in jobs):
        raise subprocess.CalledProcessError(1, "nvcc")
    if force or _stale(out, objs):
        cmd = [nvcc] + ARCH + ["-shared", "-cudart", "static", "-o", out] + objs
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    return out


def build(verbose=False, force=False, bounds_check=True):
    """The product library and, unless bounds_check is False, the
    bounds-check variant libemergence_b200_bc.so (-DEMG_BOUNDS_CHECK: every
    global index of the sweeps, the ghost fill and the AMR pool accesses is
    checked and an out-of-range index is reported as EMG_ERR_BOUNDS; loaded
    instead of the product library when EMG_BOUNDS_CHECK=1 is set)."""
    _build_one(OUT, BUILD, [], verbose, force)
    if bounds_check:
        _build_one(OUT_BC, os.path.join(BUILD, "bc"), ["-DEMG_BOUNDS_CHECK"], verbose, force)
    return OUT


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv)
