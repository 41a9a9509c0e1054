"""Build recipe for the parity oracle (test infrastructure only).

Outputs:
  oracle/liboracle.so               the C restatement (falcon_oracle.c)
  oracle/_ref/libfalcon_ref_d{D}.so the reference's own v1.3 HLS kernel headers
                                    compiled as plain C++ through the harness
                                    in oracle/ref_harness/ (one per dimension D)
  oracle/_ref/libfalcon_ref_intra_d96_c{2,4}.so
                                    the reference's intra-query v1.5 kernel
                                    headers through ref_intra_harness.cpp
                                    (2 and 4 channels, D = 96)
  oracle/_ref/libfalcon_ref_trace_d128.so
                                    the same harness over the reference's trace
                                    variant (eval_trace_FPGA_inter_query_v1.3)
  oracle/_ref/libhnswlib_ref.so     the reference's vendored hnswlib (graph
                                    builder + CPU search baseline)
  oracle/_ref/CPU_client_simulator the reference's networked CPU client
                                    simulator (wire-format interop tests)
  oracle/_ref/murmur_golden,
  oracle/_ref/bloom_golden          drivers around the reference's software
                                    Murmur2 / Bloom, used to regenerate the
                                    golden fixtures in tests/golden/

The reference builds need the reference checkout at REF_ROOT; when it is
absent (a machine without the checkout) only the prebuilt files are used.  Reference sources are
compiled where they lie; the only copies are transient ones in a temporary
directory for the v1.3 kernel headers, which get three build-time edits
(listed in ref_harness/ref_inter_harness.cpp) before compilation.
"""
import os
import re
import shutil
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
REF_ROOT = "/root/reference"
REF_V13 = os.path.join(REF_ROOT, "FPGA_multi_DDR", "FPGA_inter_query_v1.3_longer_FIFO_alt_PR", "src")
REF_TRACE = os.path.join(REF_ROOT, "FPGA_multi_DDR", "eval_trace_FPGA_inter_query_v1.3", "src")
REF_V15 = os.path.join(REF_ROOT, "FPGA_multi_DDR", "FPGA_intra_query_v1.5_support_batching_longer_FIFO", "src")
REF_INTRA_VARIANTS = ((96, 2), (96, 4))   # (D, N_CHANNEL) of the intra-query v1.5 builds
REF_HNSWLIB = os.path.join(REF_ROOT, "networked_FPGA", "CPU_programs_oldest", "hnswlib")
REF_MURMUR = os.path.join(REF_ROOT, "unit_tests", "bloom_and_hash", "sw_murmur2", "murmur2.cpp")
REF_SWBLOOM = os.path.join(REF_ROOT, "unit_tests", "bloom_and_hash", "sw_bloom")
REF_DIMS = (96, 128, 384)
REF_OUT = os.path.join(HERE, "_ref")


def _run(cmd):
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed: %s\n%s" % (" ".join(cmd), r.stdout[-4000:]))


def _stale(out, srcs):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(s) > t for s in srcs if os.path.exists(s))


def build_oracle(force=False):
    src = os.path.join(HERE, "falcon_oracle.c")
    out = os.path.join(HERE, "liboracle.so")
    if force or _stale(out, [src]):
        _run(["gcc", "-O2", "-std=c11", "-fPIC", "-shared", "-ffp-contract=off", "-fno-fast-math",
              "-pthread", src, "-o", out + ".tmp", "-lm"])
        os.replace(out + ".tmp", out)
    return out


_EDITS = [
    # constructor-local arrays the HLS code points members at -> heap storage
    ("priority_queue.hpp", r"result_t queue_array\[hardware_queue_size\];",
     "result_t* queue_array = new result_t[hardware_queue_size];"),
    ("bloom_filter.hpp", r"ap_uint<512> hash_buckets\[num_512b_buckets_int\];",
     "ap_uint<512>* hash_buckets = new ap_uint<512>[num_512b_buckets_int];"),
    # result-queue hardware size 64 -> 256 (slots past ef are inert)
    ("constants.hpp", r"const int hardware_result_queue_size = 64;",
     "const int hardware_result_queue_size = 256;"),
]


def _patched_v13_copy(dst, dim, src=None, channels=None):
    names = ["constants.hpp", "types.hpp", "utils.hpp", "priority_queue.hpp", "bloom_filter.hpp",
             "compute.hpp", "DRAM_utils.hpp", "scheduler.hpp"]
    for n in names:
        shutil.copy(os.path.join(src or REF_V13, n), os.path.join(dst, n))
    if channels is not None:   # the intra-query v1.5 headers: channel count of the variant
        p = os.path.join(dst, "constants.hpp")
        s = open(p).read()
        s2, k = re.subn(r"#define N_CHANNEL \d+", "#define N_CHANNEL %d" % channels, s)
        if k != 1:
            raise RuntimeError("could not set N_CHANNEL in constants.hpp")
        open(p, "w").write(s2)
    for fname, pat, rep in _EDITS:
        p = os.path.join(dst, fname)
        s = open(p).read()
        s2, k = re.subn(pat, rep, s)
        if k != 1:
            raise RuntimeError("reference edit did not apply to %s: %s" % (fname, pat))
        open(p, "w").write(s2)
    p = os.path.join(dst, "constants.hpp")
    s = open(p).read()
    s2, k = re.subn(r"#define D 128\b", "#define D %d" % dim, s)
    if k != 1:
        raise RuntimeError("could not set D in constants.hpp")
    open(p, "w").write(s2)


def build_ref(force=False):
    """Build the reference-derived harnesses.  Returns False if the reference
    checkout is absent (prebuilt files are then used as they are)."""
    if not os.path.isdir(REF_ROOT):
        return False
    os.makedirs(REF_OUT, exist_ok=True)
    shim = os.path.join(HERE, "ref_harness", "shim")
    harness = os.path.join(HERE, "ref_harness", "ref_inter_harness.cpp")
    for dim in REF_DIMS:
        out = os.path.join(REF_OUT, "libfalcon_ref_d%d.so" % dim)
        srcs = [harness] + [os.path.join(shim, f) for f in os.listdir(shim)] + [os.path.abspath(__file__)]
        if not force and not _stale(out, srcs):
            continue
        with tempfile.TemporaryDirectory() as td:
            _patched_v13_copy(td, dim)
            _run(["g++", "-O1", "-std=c++17", "-fPIC", "-shared", "-ffp-contract=off", "-fno-fast-math",
                  "-Wno-unknown-pragmas", "-pthread", "-I", shim, "-I", td, harness, "-o", out + ".tmp"])
        os.replace(out + ".tmp", out)
    # the intra-query v1.5 kernel, one build per (D, N_CHANNEL)
    intra = os.path.join(HERE, "ref_harness", "ref_intra_harness.cpp")
    for dim, ch in REF_INTRA_VARIANTS:
        out = os.path.join(REF_OUT, "libfalcon_ref_intra_d%d_c%d.so" % (dim, ch))
        srcs = [intra] + [os.path.join(shim, f) for f in os.listdir(shim)] + [os.path.abspath(__file__)]
        if not force and not _stale(out, srcs):
            continue
        with tempfile.TemporaryDirectory() as td:
            _patched_v13_copy(td, dim, REF_V15, channels=ch)
            _run(["g++", "-O1", "-std=c++17", "-fPIC", "-shared", "-ffp-contract=off", "-fno-fast-math",
                  "-Wno-unknown-pragmas", "-pthread", "-I", shim, "-I", td, intra, "-o", out + ".tmp"])
        os.replace(out + ".tmp", out)
    # the trace variant of the same kernel (eval_trace_FPGA_inter_query_v1.3), D = 128
    out = os.path.join(REF_OUT, "libfalcon_ref_trace_d128.so")
    srcs = [harness] + [os.path.join(shim, f) for f in os.listdir(shim)] + [os.path.abspath(__file__)]
    if force or _stale(out, srcs):
        with tempfile.TemporaryDirectory() as td:
            _patched_v13_copy(td, 128, REF_TRACE)
            _run(["g++", "-O1", "-std=c++17", "-fPIC", "-shared", "-ffp-contract=off", "-fno-fast-math",
                  "-Wno-unknown-pragmas", "-pthread", "-DFALCON_REF_TRACE", "-I", shim, "-I", td, harness,
                  "-o", out + ".tmp"])
        os.replace(out + ".tmp", out)
    src = os.path.join(HERE, "ref_harness", "hnswlib_ref.cpp")
    # The library travels to other x86 hosts, so it is built for two ISA
    # levels and oracle.Hnsw loads the highest one the running CPU supports:
    # AVX2 + FMA, and x86-64-v4 (AVX-512 F/BW/CD/DQ/VL, which turns on
    # hnswlib's own AVX-512 distance, hnswlib.h:7-9).
    for name, isa in (("libhnswlib_ref.so", ["-mavx2", "-mfma"]), ("libhnswlib_ref_v4.so", ["-march=x86-64-v4"])):
        out = os.path.join(REF_OUT, name)
        if force or _stale(out, [src, os.path.abspath(__file__)]):
            _run(["g++", "-O3"] + isa + ["-std=c++17", "-fPIC", "-shared", "-pthread", "-I", REF_HNSWLIB,
                  src, "-o", out + ".tmp"])
            os.replace(out + ".tmp", out)
    # the networked client simulator (networked_FPGA/CPU_programs/CPU_client_simulator.cpp, the reference's
    # own Makefile recipe: g++ -std=c++20 ... -lpthread -fopenmp), for the wire-format interop tests
    out = os.path.join(REF_OUT, "CPU_client_simulator")
    src = os.path.join(REF_ROOT, "networked_FPGA", "CPU_programs", "CPU_client_simulator.cpp")
    if force or _stale(out, [src, os.path.abspath(__file__)]):
        _run(["g++", "-O2", "-std=c++20", src, "-lpthread", "-fopenmp", "-o", out + ".tmp"])
        os.replace(out + ".tmp", out)
    out = os.path.join(REF_OUT, "murmur_golden")
    src = os.path.join(HERE, "ref_harness", "murmur_golden.cpp")
    if force or _stale(out, [src]):
        with tempfile.TemporaryDirectory() as td:
            obj = os.path.join(td, "murmur2.o")
            _run(["g++", "-O1", "-c", "-Dmain=reference_murmur2_demo_main", REF_MURMUR, "-o", obj])
            _run(["g++", "-O1", src, obj, "-o", out])
    out = os.path.join(REF_OUT, "bloom_golden")
    src = os.path.join(HERE, "ref_harness", "bloom_golden.cpp")
    if force or _stale(out, [src]):
        _run(["g++", "-O1", "-I", REF_SWBLOOM, src, "-o", out])
    return True


def build_all(force=False):
    build_oracle(force)
    return build_ref(force)


if __name__ == "__main__":
    ok = build_all(force="--force" in sys.argv)
    print("oracle built; reference harnesses %s" % ("built" if ok else "skipped (no reference checkout)"))
