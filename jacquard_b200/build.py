"""In-tree build of the native libraries (sm_100a).

  libjq_frontend.so    g++   csrc/frontend/*.cpp      (host script front end)
  libjacquard_b200.so  nvcc  csrc/*.cu                (interpreter kernels + C ABI)
  oracle/libjq_oracle.so, oracle/_ref/libref_kernel.so  (test infrastructure:
                       the CPU oracle and the reference kernel compiled from the
                       reference tree when it is present)
"""
import glob
import os
import shutil
import subprocess

from ._native import PKG_DIR, REPO_DIR

CSRC = os.path.join(PKG_DIR, "csrc")
NVCC_ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _gxx():
    return "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"


def _run(cmd, cwd=None):
    r = subprocess.run(cmd, cwd=cwd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"build failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return r


def _stale(out, srcs):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(s) > t for s in srcs)


def build_frontend(force=False):
    srcs = sorted(glob.glob(os.path.join(CSRC, "frontend", "*.cpp")))
    deps = srcs + glob.glob(os.path.join(CSRC, "frontend", "*.hpp")) + \
        [os.path.join(REPO_DIR, "include", "jacquard_frontend.h")]
    out = os.path.join(PKG_DIR, "libjq_frontend.so")
    if force or _stale(out, deps):
        _run([_gxx(), "-O2", "-std=c++17", "-fPIC", "-shared", "-pthread", "-o", out] + srcs)
    return out


def build_kernels(force=False):
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    deps = srcs + glob.glob(os.path.join(CSRC, "*.cuh")) + \
        [os.path.join(REPO_DIR, "include", "jacquard_b200.h")]
    out = os.path.join(PKG_DIR, "libjacquard_b200.so")
    if force or _stale(out, deps):
        nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
        _run([nvcc, "-O3", "-std=c++17", "-lineinfo", *NVCC_ARCH, "-Xcompiler", "-fPIC",
              "-shared", "-o", out] + srcs, cwd=CSRC)
    return out


def build_oracle(force=False):
    odir = os.path.join(REPO_DIR, "oracle")
    out = os.path.join(odir, "libjq_oracle.so")
    if force or _stale(out, [os.path.join(odir, "jq_oracle.c"), os.path.join(odir, "jq_oracle.h")]):
        _run(["make", "-C", odir, "-B" if force else "libjq_oracle.so"])
    ref = os.path.join(odir, "_ref", "libref_kernel.so")
    if force or not os.path.exists(ref):
        # builds from the reference tree where the recipe finds it, and keeps
        # the prebuilt library (or none) when the tree is absent
        _run([os.path.join(odir, "build_ref.sh")])
    return out


def build_all(force=False):
    build_frontend(force)
    build_kernels(force)
    build_oracle(force)
