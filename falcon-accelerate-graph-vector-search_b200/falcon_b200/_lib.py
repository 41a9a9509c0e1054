"""ctypes binding of the C ABI in include/falcon.h (libfalcon_b200.so).

The library is required: importing this module on a machine without the built
.so raises, and so does every search when the library cannot run.  There is no
CPU fallback.
"""
import ctypes
import os

from .build import LIB_PATH

FALCON_OK = 0
FALCON_WARN_TRUNCATED = 1
FALCON_ERR_ARG = -1
FALCON_ERR_OOM = -2
FALCON_ERR_CUDA = -3
FALCON_ERR_IO = -4
FALCON_ERR_GRAPH = -5
FALCON_ERR_UNSUPPORTED = -6

STORE_F32, STORE_BF16, STORE_FP8 = 1, 2, 4
PREC_F32, PREC_BF16, PREC_FP8 = 0, 1, 2
MODE_INTER, MODE_INTRA = 0, 1
MEM_HOST, MEM_DEVICE = 0, 1


class FalconError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("falcon error %d: %s" % (code, msg))
        self.code = code


class IndexDesc(ctypes.Structure):
    _fields_ = [
        ("num_vectors", ctypes.c_int64),
        ("dim", ctypes.c_int32),
        ("max_degree", ctypes.c_int32),
        ("vectors", ctypes.c_void_p),
        ("vector_stride", ctypes.c_int64),
        ("links", ctypes.c_void_p),
        ("link_stride", ctypes.c_int64),
        ("ids_offset", ctypes.c_int32),
        ("entry_point", ctypes.c_int32),
        ("labels", ctypes.c_void_p),
        ("storage", ctypes.c_int32),
        ("device", ctypes.c_int32),
    ]


class IndexInfo(ctypes.Structure):
    _fields_ = [
        ("num_vectors", ctypes.c_int64),
        ("dim", ctypes.c_int32),
        ("dim_padded", ctypes.c_int32),
        ("max_degree", ctypes.c_int32),
        ("entry_point", ctypes.c_int32),
        ("storage", ctypes.c_int32),
        ("device", ctypes.c_int32),
        ("device_bytes", ctypes.c_int64),
    ]


class UpperLayersDesc(ctypes.Structure):
    _fields_ = [
        ("max_level", ctypes.c_int32),
        ("max_degree", ctypes.c_int32),
        ("entry_point", ctypes.c_int32),
        ("ids_offset", ctypes.c_int32),
        ("num_rows", ctypes.c_int64),
        ("row_stride", ctypes.c_int64),
        ("levels", ctypes.c_void_p),
        ("row_start", ctypes.c_void_p),
        ("rows", ctypes.c_void_p),
    ]


class SearchParams(ctypes.Structure):
    _fields_ = [
        ("k", ctypes.c_int32),
        ("ef", ctypes.c_int32),
        ("mc", ctypes.c_int32),
        ("mg", ctypes.c_int32),
        ("cand_queue_size", ctypes.c_int32),
        ("bloom_bits", ctypes.c_int32),
        ("hash_seed", ctypes.c_uint32),
        ("mode", ctypes.c_int32),
        ("channels", ctypes.c_int32),
        ("precision", ctypes.c_int32),
        ("rerank", ctypes.c_int32),
        ("max_hops", ctypes.c_int32),
    ]


class ServerConfig(ctypes.Structure):
    _fields_ = [
        ("device", ctypes.c_int32),
        ("ring_capacity", ctypes.c_int32),
        ("max_k", ctypes.c_int32),
        ("ef_max", ctypes.c_int32),
        ("cand_queue_max", ctypes.c_int32),
        ("bloom_bits_max", ctypes.c_int32),
        ("mc_max", ctypes.c_int32),
        ("mg_max", ctypes.c_int32),
        ("dim_max", ctypes.c_int32),
        ("idle_exit_us", ctypes.c_int64),
        ("memory_fraction", ctypes.c_double),
    ]


class ServerInfo(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int64) for n in
                ("ring_entries", "in_flight", "submitted", "kernel_launches", "warps", "device_bytes",
                 "concurrent_classes_max")]


# Every symbol include/falcon.h declares, with its ctypes signature.
_VP = ctypes.c_void_p
_I32 = ctypes.c_int32
_I64 = ctypes.c_int64
SIGNATURES = {
    "falcon_default_params": (None, [ctypes.POINTER(SearchParams)]),
    "falcon_index_create": (_I32, [ctypes.POINTER(IndexDesc), ctypes.POINTER(_VP)]),
    "falcon_index_load_fpga": (_I32, [ctypes.c_char_p, ctypes.c_char_p, _I32, _I32, _I32, ctypes.POINTER(_VP)]),
    "falcon_index_info_get": (_I32, [_VP, ctypes.POINTER(IndexInfo)]),
    "falcon_index_free": (_I32, [_VP]),
    "falcon_index_copy_storage": (_I32, [_VP, _I32, _VP, _I64]),
    "falcon_index_set_upper_layers": (_I32, [_VP, ctypes.POINTER(UpperLayersDesc)]),
    "falcon_descend": (_I32, [_VP, _VP, _I64, _I64, _VP, _VP, _I32, _VP]),
    "falcon_search": (_I32, [_VP, _VP, _I64, _I64, _VP, ctypes.POINTER(SearchParams), _I32,
                             _VP, _VP, _I32, _VP, _VP, _I32, _VP]),
    "falcon_search_trace": (_I32, [_VP, _VP, _I64, _I64, _VP, ctypes.POINTER(SearchParams), _VP, _VP, _I32, _VP,
                                   _VP, _VP, _VP, _I32, _VP, _VP, _I32, _VP, _I32, _VP]),
    "falcon_search_noalloc": (_I32, [_VP, _VP, _I64, _I64, _VP, ctypes.POINTER(SearchParams), _I32,
                                     _VP, _VP, _I32, _VP, _VP, _VP]),
    "falcon_vadd": (_I32, [_I32, _I32, _I32, _I32, _I32, _I32, _I32, ctypes.c_uint32, _I32, _I32, _I32, _I64,
                           _VP, _VP, _VP, _VP, _VP, _VP, _VP, _I32]),
    "falcon_graph_prune": (_I32, [_VP, _I64, _I32, _I64, _VP, _I64, _I32, _VP, _I64, ctypes.c_float, _I32, _VP,
                                  _I64, _VP, _I32, _VP]),
    "falcon_server_default_config": (None, [ctypes.POINTER(ServerConfig)]),
    "falcon_server_create": (_I32, [ctypes.POINTER(ServerConfig), ctypes.POINTER(_VP)]),
    "falcon_server_add_index": (_I32, [_VP, _VP, ctypes.POINTER(ctypes.c_int32)]),
    "falcon_server_submit": (_I32, [_VP, _I32, _VP, _VP, _I64, ctypes.POINTER(SearchParams), _I32, _VP]),
    "falcon_server_poll": (_I32, [_VP, _I64, _VP, _VP, ctypes.POINTER(_I32), ctypes.POINTER(_I32)]),
    "falcon_server_wait": (_I32, [_VP, _I64, _I64, _VP, _VP, ctypes.POINTER(_I32), ctypes.POINTER(_I32)]),
    "falcon_server_replay": (_I32, [_VP, _I32, _VP, _VP, _I64, ctypes.POINTER(SearchParams), _I32, _VP, _VP, _VP,
                                    _I32, _VP, _VP, _VP, _VP]),
    "falcon_server_info_get": (_I32, [_VP, ctypes.POINTER(ServerInfo)]),
    "falcon_server_free": (_I32, [_VP]),
    "falcon_last_error": (ctypes.c_char_p, []),
    "falcon_build_info": (ctypes.c_char_p, []),
}

_lib = None


def load(path=None):
    """Load libfalcon_b200.so (raises if it is missing or incomplete)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise FalconError(FALCON_ERR_IO, "libfalcon_b200.so not built at %s (run __graft_entry__.build())" % p)
    lib = ctypes.CDLL(p)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)   # AttributeError if the export is missing
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


def last_error():
    return load().falcon_last_error().decode()


def check(rc, allow_truncated=True):
    if rc == FALCON_OK or (allow_truncated and rc == FALCON_WARN_TRUNCATED):
        return rc
    raise FalconError(rc, last_error())
