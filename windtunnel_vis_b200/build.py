"""Build libwt.so (the C-ABI CUDA library) in-tree for sm_100a.

    python -m windtunnel_vis_b200.build [--force]

Each .cu in csrc/ is compiled by nvcc to an object in _build/, then linked into
windtunnel_vis_b200/libwt.so with the static CUDA runtime. The voxelizer, tracer and
derived-field units are compiled with -fmad=false (no contraction) so their f32 results are
bit-identical to the CPU restatement. So is the LBM unit, for another reason: without contraction
every rounding in it is the one written in the source (fused multiply-adds only where the code
asks for them), so a cell's update gives the same bits in every kernel that inlines it (the
per-step kernels, the batched kernels and the persistent multi-step kernel), whatever the
compiler's register budget or code placement there.
"""
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
OBJ = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libwt.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC",
          "-Xptxas", "-warn-spills", "-I", os.path.join(ROOT, "include")]
UNITS = {
    "wt_api.cu": [],
    "wt_lbm.cu": ["-fmad=false"],
    "wt_voxel.cu": ["-fmad=false"],
    "wt_tracer.cu": ["-fmad=false"],
    "wt_fields.cu": ["-fmad=false"],
    "wt_closure.cu": [],
}
HEADERS = ["wt_common.cuh", "wt_internal.h", "wt_closure.cuh", "wt_umma.cuh"]


def nvcc():
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _mtime(p):
    return os.path.getmtime(p) if os.path.exists(p) else 0.0


def build(force: bool = False, verbose: bool = False, extra=None) -> str:
    os.makedirs(OBJ, exist_ok=True)
    hdr_t = max(_mtime(os.path.join(CSRC, h)) for h in HEADERS)
    hdr_t = max(hdr_t, _mtime(os.path.join(ROOT, "include", "wt.h")), _mtime(os.path.abspath(__file__)))
    objs = []
    jobs = []
    for unit, flags in UNITS.items():
        src = os.path.join(CSRC, unit)
        obj = os.path.join(OBJ, unit.replace(".cu", ".o"))
        objs.append(obj)
        if force or _mtime(obj) < max(_mtime(src), hdr_t) or extra:
            cmd = [nvcc(), *ARCH, *COMMON, *flags, *(extra or []), "-c", src, "-o", obj]
            if verbose:
                print(" ".join(cmd))
            jobs.append((cmd, subprocess.Popen(cmd)))
    for cmd, proc in jobs:
        if proc.wait() != 0:
            raise subprocess.CalledProcessError(proc.returncode, cmd)
    rebuilt = bool(jobs)
    if rebuilt or not os.path.exists(LIB) or _mtime(LIB) < max(_mtime(o) for o in objs):
        cmd = [nvcc(), *ARCH, "-shared", "-Xcompiler", "-fPIC", "-cudart", "static", *objs, "-o", LIB + ".tmp"]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
        os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
