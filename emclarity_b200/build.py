"""Builds libemc_b200.so (sm_100a) in-tree from emclarity_b200/csrc/*.cu.

Run as ``python -m emclarity_b200.build`` or through ``__graft_entry__.build()``.
Objects are rebuilt only when a source or header is newer than the object.
"""
import glob
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libemc_b200.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
              "--expt-relaxed-constexpr", "-I", INCLUDE, "-I", CSRC]


def _nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.sep not in c or os.path.exists(c)):
            return c
    return "nvcc"


def _newest_header():
    hs = glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(INCLUDE, "*.h"))
    return max((os.path.getmtime(h) for h in hs), default=0.0)


def _compile(src, extra):
    obj = os.path.join(OBJ, os.path.basename(src) + ".o")
    if os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(src), _newest_header()):
        return obj
    cmd = [_nvcc(), *ARCH, *NVCC_FLAGS, *extra, "-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed for %s:\n%s\n%s" % (src, " ".join(cmd), r.stderr[-6000:]))
    return obj


def build(verbose=False, extra=()):
    os.makedirs(OBJ, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))
    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(lambda s: _compile(s, list(extra)), srcs))
    if os.path.exists(LIB) and os.path.getmtime(LIB) >= max(os.path.getmtime(o) for o in objs):
        return LIB
    cmd = [_nvcc(), *ARCH, "-shared", "-o", LIB, *objs, "-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("link failed:\n%s\n%s" % (" ".join(cmd), r.stderr[-4000:]))
    if verbose:
        print("built", LIB)
    return LIB


MEX_DIR = os.path.join(HERE, "mex")
MEX_OUT = os.path.join(MEX_DIR, "_shim")
GATEWAYS = ["mexXform3d_b200", "mexFFT_b200", "mexCTF_b200", "mexSF3D_b200", "mexEmcSearch", "mexEmcAverage"]


def build_mex(verbose=False):
    """Compiles every MEX gateway against the in-repo MEX stand-in (emclarity_b200/mex/shim) into
    emclarity_b200/mex/_shim/lib<gateway>.so, linked to libemc_b200.so.  With MATLAB installed the
    same sources build with `mex` instead (see the integration notes)."""
    lib = build(verbose=verbose)
    os.makedirs(MEX_OUT, exist_ok=True)
    shim = os.path.join(MEX_DIR, "shim", "mex_shim.cpp")
    outs = []
    for gw in GATEWAYS:
        src = os.path.join(MEX_DIR, gw + ".cpp")
        out = os.path.join(MEX_OUT, "lib%s.so" % gw)
        deps = [src, shim, os.path.join(MEX_DIR, "mex_common.h"), lib]
        if os.path.exists(out) and os.path.getmtime(out) >= max(os.path.getmtime(d) for d in deps):
            outs.append(out)
            continue
        cmd = [_nvcc(), "-O2", "-std=c++17", "-Xcompiler", "-fPIC", "-shared", "-I", os.path.join(MEX_DIR, "shim"),
               "-I", INCLUDE, "-I", MEX_DIR, src, shim, "-o", out, "-L", HERE, "-lemc_b200", "-lcudart",
               "-Xlinker", "-rpath=$ORIGIN/../.."]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("MEX gateway build failed for %s:\n%s\n%s" % (gw, " ".join(cmd), r.stderr[-4000:]))
        outs.append(out)
    return outs


if __name__ == "__main__":
    build(verbose=True, extra=sys.argv[1:])
    build_mex(verbose=True)
