"""The networked FPGA wire format, and a server that speaks it in front of the
continuous-batching server.

The reference's networked deployment streams queries from a CPU client to the
FPGA over TCP and reads results back on a second connection
(networked_FPGA/CPU_programs/README.md:50-72; CPU_client.cpp:183-199 sizes,
:449-520 send side, :545-612 receive side, :645-652 result parsing;
FPGA_simulator.cpp:55-70, :163-200 the FPGA side).  Everything travels in
64-byte packets (one 512-bit AXI word, constants.hpp:6-9):

  client -> FPGA, per batch: one header packet whose first int32 is the batch
      size (0 or -1: end of stream), then each query as ceil(D / 16) packets
      of float32, zero padded;
  FPGA -> client, per query in arrival order: one header packet (the first
      int32 is topK = ef), ceil(ef / 16) packets of int32 ids, ceil(ef / 16)
      packets of float32 distances, best first.

Connection order (CPU_client.cpp:522-545): the client listens on its F2C port
and the FPGA connects to it; only then does the client connect to the FPGA's
C2F port.  `WireServer` takes the FPGA's place: it listens on the C2F port,
connects back to the client's F2C port, then admits every query into a
`FalconServer` as soon as it has arrived (so queries of a batch overlap on the
GPU) and writes the results in arrival order.  The reference client therefore
talks to the GPU unchanged; `python -m falcon_b200.wire` serves an index saved
in the reference's FPGA file layout.
"""
import collections
import select
import socket
import struct
import threading
import time

import numpy as np

PACKET = 64            # bytes per 512-bit packet
FLOATS_PER_PACKET = 16


def _packets(n_words):
    return -(-int(n_words) // FLOATS_PER_PACKET)


def query_bytes(dim):
    """Bytes of one query on the client -> FPGA stream (header excluded)."""
    return _packets(dim) * PACKET


def result_bytes(ef):
    """Bytes of one query's answer on the FPGA -> client stream."""
    return PACKET + 2 * _packets(ef) * PACKET


def encode_header(batch_size):
    h = bytearray(PACKET)
    struct.pack_into("<i", h, 0, int(batch_size))
    return bytes(h)


def encode_query(q, dim):
    out = np.zeros(_packets(dim) * FLOATS_PER_PACKET, dtype="<f4")
    out[:dim] = np.asarray(q, dtype=np.float32)[:dim]
    return out.tobytes()


def encode_batch(queries):
    """A batch as the client sends it: header, then the padded queries."""
    q = np.asarray(queries, dtype=np.float32)
    return encode_header(len(q)) + b"".join(encode_query(v, q.shape[1]) for v in q)


def encode_end():
    return encode_header(-1)


def encode_result(ids, dists, ef):
    n = _packets(ef) * FLOATS_PER_PACKET
    h = bytearray(PACKET)
    struct.pack_into("<i", h, 0, int(ef))
    i = np.full(n, -1, dtype="<i4")
    d = np.zeros(n, dtype="<f4")
    k = min(len(ids), ef)
    i[:k] = np.asarray(ids, dtype=np.int32)[:k]
    d[:k] = np.asarray(dists, dtype=np.float32)[:k]
    return bytes(h) + i.tobytes() + d.tobytes()


def decode_result(buf, ef):
    """(ids[ef], dists[ef]) of one answer."""
    n = _packets(ef) * FLOATS_PER_PACKET
    ids = np.frombuffer(buf, dtype="<i4", count=n, offset=PACKET)[:ef].copy()
    dists = np.frombuffer(buf, dtype="<f4", count=n, offset=PACKET + 4 * n)[:ef].copy()
    return ids, dists


def decode_query(buf, dim):
    return np.frombuffer(buf, dtype="<f4", count=dim).copy()


def _recv_exact(sock, n):
    parts, got = [], 0
    while got < n:
        b = sock.recv(n - got)
        if not b:
            raise ConnectionError("peer closed the connection after %d of %d bytes" % (got, n))
        parts.append(b)
        got += len(b)
    return b"".join(parts)


class WireServer:
    """Serve one index over the FPGA wire format.

    engine: a FalconServer (or any object with submit(index_ids, queries,
    params) -> admitted request ids and wait(request_id, k) -> (ids, dists,
    hops, visited)); index_id: the engine's id of the index; dim, ef: the
    stream's vector length and answer length (topK = ef, as the FPGA);
    params: the search parameters of every query (k is set to ef)."""

    def __init__(self, engine, index_id, dim, ef, c2f_port, f2c_host, f2c_port, params=None, bind_host="0.0.0.0",
                 connect_timeout=60.0, max_group=256):
        self.engine, self.index_id, self.dim, self.ef = engine, int(index_id), int(dim), int(ef)
        self.params = dict(params or {})
        self.params["k"] = self.ef
        self.params["ef"] = max(self.ef, int(self.params.get("ef", self.ef)))
        self.c2f_port, self.f2c_host, self.f2c_port = int(c2f_port), f2c_host, int(f2c_port)
        self.bind_host, self.connect_timeout, self.max_group = bind_host, float(connect_timeout), int(max_group)
        self.queries_served = 0
        self.error = None
        self._lsock = socket.socket(socket.AF_INET, socket.SOCK_STREAM)
        self._lsock.setsockopt(socket.SOL_SOCKET, socket.SO_REUSEADDR, 1)
        self._lsock.bind((self.bind_host, self.c2f_port))
        self._lsock.listen(1)   # listening before the client is contacted, as the FPGA

    def _connect_back(self):
        t0 = time.time()
        while True:
            try:
                s = socket.create_connection((self.f2c_host, self.f2c_port), timeout=5.0)
                s.setsockopt(socket.IPPROTO_TCP, socket.TCP_NODELAY, 1)
                s.settimeout(None)
                return s
            except OSError:
                if time.time() - t0 > self.connect_timeout:
                    raise
                time.sleep(0.05)

    def _submit(self, qs):
        """Admit all of qs, retrying while the engine's ring is full."""
        rids = []
        while len(rids) < len(qs):
            got = self.engine.submit(np.full(len(qs) - len(rids), self.index_id, dtype=np.int32),
                                     np.ascontiguousarray(qs[len(rids):]), self.params)
            rids.extend(int(x) for x in got)
            if len(got) == 0:
                time.sleep(20e-6)
        return rids

    def serve(self):
        """Run until the client's end-of-stream header; returns the number of
        queries answered."""
        out = self._connect_back()
        self._lsock.settimeout(self.connect_timeout)
        inp, _ = self._lsock.accept()
        inp.settimeout(None)
        pending = collections.deque()
        cv = threading.Condition()
        state = {"done": False}

        def writer():
            try:
                while True:
                    with cv:
                        while not pending and not state["done"]:
                            cv.wait()
                        if not pending:
                            return
                        rid = pending.popleft()
                    ids, dists, _, _ = self.engine.wait(rid, self.ef)
                    out.sendall(encode_result(ids, dists, self.ef))
                    self.queries_served += 1
            except Exception as e:   # reported by serve()
                self.error = e

        wt = threading.Thread(target=writer, daemon=True)
        wt.start()
        qb = query_bytes(self.dim)
        try:
            while True:
                bs = struct.unpack_from("<i", _recv_exact(inp, PACKET), 0)[0]
                if bs <= 0:
                    break
                left = bs
                while left > 0:
                    # one query, then whatever else of the batch has already
                    # arrived, admitted together
                    group = [decode_query(_recv_exact(inp, qb), self.dim)]
                    left -= 1
                    while left > 0 and len(group) < self.max_group and select.select([inp], [], [], 0)[0]:
                        group.append(decode_query(_recv_exact(inp, qb), self.dim))
                        left -= 1
                    rids = self._submit(np.stack(group))
                    with cv:
                        pending.extend(rids)
                        cv.notify()
        finally:
            with cv:
                state["done"] = True
                cv.notify()
            wt.join()
            inp.close()
            out.close()
            self._lsock.close()
        if self.error is not None:
            raise self.error
        return self.queries_served


def main(argv=None):
    """Serve an index in the reference's FPGA file layout over the wire format:
    python -m falcon_b200.wire --index-dir D --dim 128 --graph HNSW --ef 64
        --c2f-port 8888 --client-host 10.0.0.1 --f2c-port 5001 [--mc 1 --mg 1 ...]"""
    import argparse
    from .formats import read_fpga_index
    from .index import FalconIndex
    from .serving import FalconServer
    ap = argparse.ArgumentParser(description=main.__doc__)
    ap.add_argument("--index-dir", required=True)
    ap.add_argument("--graph", default="HNSW", help="the file-name tag of the FPGA index files (HNSW or NSG)")
    ap.add_argument("--dim", type=int, required=True)
    ap.add_argument("--ef", type=int, required=True)
    ap.add_argument("--mc", type=int, default=1)
    ap.add_argument("--mg", type=int, default=1)
    ap.add_argument("--cand-queue-size", type=int, default=32)
    ap.add_argument("--bloom-bits", type=int, default=16)
    ap.add_argument("--c2f-port", type=int, required=True)
    ap.add_argument("--client-host", required=True)
    ap.add_argument("--f2c-port", type=int, required=True)
    ap.add_argument("--device", type=int, default=0)
    a = ap.parse_args(argv)
    g = read_fpga_index(a.index_dir, a.graph, a.dim)
    ix = FalconIndex(g, device=a.device)
    sv = FalconServer(device=a.device, ring_capacity=65536, max_k=a.ef, ef_max=a.ef, cand_queue_max=a.cand_queue_size,
                      bloom_bits_max=a.bloom_bits, mc_max=a.mc, mg_max=a.mg, dim_max=a.dim)
    iid = sv.add_index(ix)
    ws = WireServer(sv, iid, a.dim, a.ef, a.c2f_port, a.client_host, a.f2c_port,
                    params=dict(mc=a.mc, mg=a.mg, cand_queue_size=a.cand_queue_size, bloom_bits=a.bloom_bits))
    n = ws.serve()
    print("served %d queries" % n)
    sv.close()
    ix.close()
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
