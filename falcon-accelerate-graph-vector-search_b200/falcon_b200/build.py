"""Build recipe for libfalcon_b200.so (sm_100a), compiled in-tree with nvcc."""
import os
import subprocess
import sys

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
SRC_ROOT = os.path.dirname(PKG_DIR)
CSRC = os.path.join(SRC_ROOT, "csrc")
REPO = os.path.dirname(SRC_ROOT)
LIB_PATH = os.path.join(PKG_DIR, "libfalcon_b200.so")

SOURCES = ["falcon_kernels.cu", "falcon_capi.cu", "falcon_noalloc.cu", "falcon_serve.cu"]
HEADERS = ["falcon_internal.h"]
NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-std=c++17", "-lineinfo",
    # FP32 distances must not be contracted into FMAs: the reference adder
    # tree rounds every multiply and add separately.
    "--fmad=false",
    "-shared", "-Xcompiler", "-fPIC",
]


def _nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.sep not in cand or os.path.exists(cand)):
            return cand
    return "nvcc"


def sources():
    return [os.path.join(CSRC, s) for s in SOURCES]


def is_stale():
    if not os.path.exists(LIB_PATH):
        return True
    t = os.path.getmtime(LIB_PATH)
    deps = sources() + [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(REPO, "include", "falcon.h")]
    return any(os.path.getmtime(p) > t for p in deps if os.path.exists(p))


def build(force=False, verbose=False):
    """Compile the CUDA library if any source is newer than the .so."""
    if not force and not is_stale():
        return LIB_PATH
    cmd = [_nvcc()] + NVCC_FLAGS + sources() + ["-o", LIB_PATH + ".tmp"]
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + r.stdout[-6000:])
    if verbose:
        print(r.stdout)
    os.replace(LIB_PATH + ".tmp", LIB_PATH)
    return LIB_PATH


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
