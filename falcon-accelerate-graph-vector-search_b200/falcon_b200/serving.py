"""Continuous-batching search server over the C ABI (falcon_server_*).

A persistent kernel pulls single-query requests from a device ring while the
host keeps admitting new ones; requests carry their own index, precision and
k/ef/mc/mg.  See include/falcon.h for the contract.
"""
import ctypes

import numpy as np

from . import _lib
from .index import make_params


ServerConfig = _lib.ServerConfig
ServerInfo = _lib.ServerInfo


def _params_array(params, n):
    if isinstance(params, (list, tuple)):
        arr = (_lib.SearchParams * len(params))()
        for i, p in enumerate(params):
            arr[i] = p if isinstance(p, _lib.SearchParams) else make_params(**p)
        return arr, 1
    p = params if isinstance(params, _lib.SearchParams) else make_params(**(params or {}))
    return p, 0


class FalconServer:
    def __init__(self, device=0, **cfg):
        lib = _lib.load()
        c = ServerConfig()
        lib.falcon_server_default_config(ctypes.byref(c))
        c.device = device
        for k, v in cfg.items():
            setattr(c, k, v)
        h = ctypes.c_void_p()
        _lib.check(lib.falcon_server_create(ctypes.byref(c), ctypes.byref(h)))
        self._h, self.cfg, self._indexes, self._profile = h, c, [], None

    def set_profile(self, profile):
        """An autotuner profile (falcon_b200.autotune) that auto_params reads."""
        self._profile = profile

    def auto_params(self, index_id, k, ef, **overrides):
        """Request parameters for an index from the autotuner's profile: the
        candidate queue, (mc, mg) and Bloom size of the throughput entry for
        the index's (dimension, max degree) at or above `ef` (autotune.pick;
        the server runs inter-query requests), with the requested k and ef and
        `overrides` applied."""
        from .autotune import pick
        if self._profile is None:
            raise ValueError("no autotuner profile: call set_profile first")
        inf = self._indexes[index_id].info()
        p = pick(self._profile, inf.dim, inf.max_degree, ef, "throughput")
        p.update(k=k, ef=max(ef, k), mode="inter")
        p.update(overrides)
        return make_params(**p)

    def add_index(self, index):
        iid = ctypes.c_int32()
        _lib.check(_lib.load().falcon_server_add_index(self._h, index._h, ctypes.byref(iid)))
        self._indexes.append(index)
        return iid.value

    def submit(self, index_ids, queries, params):
        """Returns the request ids of the admitted prefix (possibly fewer than asked)."""
        q = np.ascontiguousarray(queries, dtype=np.float32)
        n = q.shape[0]
        ii = np.ascontiguousarray(np.broadcast_to(np.asarray(index_ids, dtype=np.int32), (n,)))
        rid = np.full(n, -1, dtype=np.int64)
        parr, pq = _params_array(params, n)
        pptr = ctypes.cast(parr, ctypes.POINTER(_lib.SearchParams)) if pq else ctypes.byref(parr)
        rc = _lib.load().falcon_server_submit(self._h, n, ii.ctypes.data, q.ctypes.data, q.shape[1], pptr, pq,
                                              rid.ctypes.data)
        if rc < 0:
            raise _lib.FalconError(rc, _lib.last_error())
        return rid[:rc]

    def poll(self, request_id, k):
        ids = np.empty(k, dtype=np.int32)
        d = np.empty(k, dtype=np.float32)
        h, v = ctypes.c_int32(), ctypes.c_int32()
        rc = _lib.load().falcon_server_poll(self._h, int(request_id), ids.ctypes.data, d.ctypes.data, ctypes.byref(h),
                                            ctypes.byref(v))
        if rc < 0:
            raise _lib.FalconError(rc, _lib.last_error())
        return (ids, d, h.value, v.value) if rc == 1 else None

    def wait(self, request_id, k, timeout_us=10_000_000):
        ids = np.empty(k, dtype=np.int32)
        d = np.empty(k, dtype=np.float32)
        h, v = ctypes.c_int32(), ctypes.c_int32()
        _lib.check(_lib.load().falcon_server_wait(self._h, int(request_id), int(timeout_us), ids.ctypes.data,
                                                  d.ctypes.data, ctypes.byref(h), ctypes.byref(v)))
        return ids, d, h.value, v.value

    def replay(self, index_ids, queries, params, arrival_us, out_stride):
        """Native load driver: returns latencies_us, ids, dists, hops, visited, elapsed_us."""
        q = np.ascontiguousarray(queries, dtype=np.float32)
        n = q.shape[0]
        ii = np.ascontiguousarray(np.broadcast_to(np.asarray(index_ids, dtype=np.int32), (n,)))
        arr = np.ascontiguousarray(arrival_us, dtype=np.float64)
        lat = np.zeros(n, dtype=np.float64)
        ids = np.full((n, out_stride), -1, dtype=np.int32)
        d = np.zeros((n, out_stride), dtype=np.float32)
        hops = np.zeros(n, dtype=np.int32)
        vis = np.zeros(n, dtype=np.int32)
        el = ctypes.c_double()
        parr, pq = _params_array(params, n)
        pptr = ctypes.cast(parr, ctypes.POINTER(_lib.SearchParams)) if pq else ctypes.byref(parr)
        _lib.check(_lib.load().falcon_server_replay(self._h, n, ii.ctypes.data, q.ctypes.data, q.shape[1], pptr, pq,
                                                    arr.ctypes.data, lat.ctypes.data, ids.ctypes.data, out_stride,
                                                    d.ctypes.data, hops.ctypes.data, vis.ctypes.data,
                                                    ctypes.byref(el)))
        return lat, ids, d, hops, vis, el.value

    def info(self):
        inf = ServerInfo()
        _lib.check(_lib.load().falcon_server_info_get(self._h, ctypes.byref(inf)))
        return inf

    def close(self):
        if getattr(self, "_h", None):
            _lib.load().falcon_server_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def poisson_arrivals(n, rate_qps, seed=0):
    """Arrival offsets in microseconds of a Poisson process of the given rate."""
    rng = np.random.default_rng(seed)
    return np.cumsum(rng.exponential(1e6 / rate_qps, size=n))
