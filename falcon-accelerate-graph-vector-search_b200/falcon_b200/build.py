"""Build recipe for libfalcon_b200.so (sm_100a), compiled in-tree with nvcc."""
import os
import subprocess
import sys

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
SRC_ROOT = os.path.dirname(PKG_DIR)
CSRC = os.path.join(SRC_ROOT, "csrc")
REPO = os.path.dirname(SRC_ROOT)
LIB_PATH = os.path.join(PKG_DIR, "libfalcon_b200.so")

SOURCES = ["falcon_kernels.cu", "falcon_capi.cu", "falcon_noalloc.cu", "falcon_serve.cu", "falcon_build.cu"]
HEADERS = ["falcon_internal.h"]
COMPILE_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-std=c++17", "-lineinfo",
    # FP32 distances must not be contracted into FMAs: the reference adder
    # tree rounds every multiply and add separately.
    "--fmad=false",
    "-Xcompiler", "-fPIC",
]
LINK_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-shared"]
# kept for callers that compile the sources in one nvcc invocation
NVCC_FLAGS = COMPILE_FLAGS + ["-shared"]


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


def _obj_dir():
    d = os.path.join(PKG_DIR, "_build")
    os.makedirs(d, exist_ok=True)
    return d


def build(force=False, verbose=False):
    """Compile the CUDA library if any source is newer than the .so: every
    source to an object file in parallel, then one link."""
    if not force and not is_stale():
        return LIB_PATH
    from concurrent.futures import ThreadPoolExecutor
    od = _obj_dir()
    objs = [os.path.join(od, os.path.splitext(s)[0] + ".o") for s in SOURCES]

    def compile_one(i):
        cmd = [_nvcc()] + COMPILE_FLAGS + ["-c", sources()[i], "-o", objs[i] + ".tmp"]
        r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
        if r.returncode == 0:
            os.replace(objs[i] + ".tmp", objs[i])
        return r

    with ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        results = list(ex.map(compile_one, range(len(SOURCES))))
    for r in results:
        if r.returncode != 0:
            raise RuntimeError("nvcc failed:\n" + r.stdout[-6000:])
        if verbose:
            print(r.stdout)
    r = subprocess.run([_nvcc()] + LINK_FLAGS + objs + ["-o", LIB_PATH + ".tmp"], stdout=subprocess.PIPE,
                       stderr=subprocess.STDOUT, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc link failed:\n" + r.stdout[-6000:])
    os.replace(LIB_PATH + ".tmp", LIB_PATH)
    return LIB_PATH


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
