"""The networked FPGA wire format (falcon_b200.wire).

* packet sizes and encode/decode round trips against the reference client's
  size formulas (networked_FPGA/CPU_programs/CPU_client.cpp:183-199);
* the reference's own CPU client simulator (CPU_client_simulator.cpp, built
  from its sources into oracle/_ref/ by oracle/build_oracle.py) runs its full
  protocol against WireServer on loopback: connection order, batch headers,
  per-query answers, end-of-stream;
* on the GPU, answers through WireServer + FalconServer equal falcon_search's,
  bit for bit.
"""
import os
import socket
import subprocess
import threading

import numpy as np
import pytest

from helpers import small_graph

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLIENT_SIM = os.path.join(REPO, "oracle", "_ref", "CPU_client_simulator")


def _free_ports(n):
    socks, ports = [], []
    for _ in range(n):
        s = socket.socket()
        s.bind(("127.0.0.1", 0))
        socks.append(s)
        ports.append(s.getsockname()[1])
    for s in socks:
        s.close()
    return ports


class FakeEngine:
    """submit/wait with a deterministic answer per query (CPU tests only)."""

    def __init__(self):
        self.q = []

    def submit(self, index_ids, queries, params):
        start = len(self.q)
        self.q.extend(np.asarray(queries, dtype=np.float32))
        return np.arange(start, len(self.q), dtype=np.int64)

    def wait(self, rid, k):
        base = int(abs(float(self.q[rid][0])) * 1000) + rid
        return (np.arange(base, base + k, dtype=np.int32), np.arange(k, dtype=np.float32) * 0.5, 1, k)


def test_wire_sizes_and_roundtrip():
    from falcon_b200 import wire
    # ceil(D / 16) and ceil(ef / 16) 64-byte packets, one header packet per answer
    assert [wire.query_bytes(d) for d in (96, 100, 128, 384)] == [384, 448, 512, 1536]
    assert [wire.result_bytes(e) for e in (10, 64, 100, 256)] == [192, 576, 960, 2112]
    q = np.random.default_rng(0).standard_normal((5, 100)).astype(np.float32)
    b = wire.encode_batch(q)
    assert len(b) == 64 + 5 * 448 and int(np.frombuffer(b[:4], "<i4")[0]) == 5
    for i in range(5):
        got = wire.decode_query(b[64 + i * 448:64 + (i + 1) * 448], 100)
        assert np.array_equal(got, q[i])
        assert not np.any(np.frombuffer(b[64 + i * 448 + 400:64 + (i + 1) * 448], "<f4"))   # zero padding
    ids, d = np.arange(37, dtype=np.int32), np.linspace(0, 1, 37, dtype=np.float32)
    r = wire.encode_result(ids, d, 37)
    assert len(r) == wire.result_bytes(37)
    i2, d2 = wire.decode_result(r, 37)
    assert np.array_equal(i2, ids) and np.array_equal(d2, d)
    assert int(np.frombuffer(wire.encode_end()[:4], "<i4")[0]) == -1


def _client(c2f, f2c, dim, ef, batches):
    """This side of the protocol, as the reference client runs it."""
    from falcon_b200 import wire
    ls = socket.socket()
    ls.setsockopt(socket.SOL_SOCKET, socket.SO_REUSEADDR, 1)
    ls.bind(("127.0.0.1", f2c))
    ls.listen(1)
    ls.settimeout(30)
    inp, _ = ls.accept()
    out = socket.create_connection(("127.0.0.1", c2f), timeout=30)
    res = []
    for qb in batches:
        out.sendall(wire.encode_batch(qb))
        for _ in range(len(qb)):
            res.append(wire.decode_result(wire._recv_exact(inp, wire.result_bytes(ef)), ef))
    out.sendall(wire.encode_end())
    out.close()
    inp.close()
    ls.close()
    return res


def test_wire_server_roundtrip_fake_engine():
    from falcon_b200.wire import WireServer
    c2f, f2c = _free_ports(2)
    eng = FakeEngine()
    ws = WireServer(eng, 0, 24, 20, c2f, "127.0.0.1", f2c, bind_host="127.0.0.1", connect_timeout=30)
    t = threading.Thread(target=ws.serve, daemon=True)
    t.start()
    rng = np.random.default_rng(1)
    batches = [rng.standard_normal((n, 24)).astype(np.float32) for n in (3, 17, 1)]
    res = _client(c2f, f2c, 24, 20, batches)
    t.join(30)
    assert not t.is_alive() and ws.error is None and ws.queries_served == 21
    allq = np.concatenate(batches)
    for j, (ids, d) in enumerate(res):
        want = eng.wait(j, 20)
        assert np.array_equal(ids, want[0]) and np.array_equal(d, want[1])
        assert np.array_equal(eng.q[j], allq[j])


@pytest.mark.skipif(not os.path.exists(CLIENT_SIM), reason="reference client simulator not built on this host")
def test_wire_server_with_reference_client_simulator(tmp_path):
    from falcon_b200.wire import WireServer
    c2f, f2c = _free_ports(2)
    ws = WireServer(FakeEngine(), 0, 128, 64, c2f, "127.0.0.1", f2c, bind_host="127.0.0.1", connect_timeout=30)
    t = threading.Thread(target=ws.serve, daemon=True)
    t.start()
    # <num_FPGA> <IP> <C2F port> <F2C port> <D> <ef> <query_num> <batch_size> <query_window> <batch_window>
    args = [CLIENT_SIM, "1", "127.0.0.1", str(c2f), str(f2c), "128", "64", "300", "32", "16", "2"]
    with open(tmp_path / "client.log", "w") as log:
        p = subprocess.run(args, cwd=tmp_path, stdout=log, stderr=subprocess.STDOUT, timeout=120)
    t.join(30)
    out = (tmp_path / "client.log").read_text()
    assert p.returncode == 0, out[-2000:]
    assert "End-to-end QPS" in out
    assert not t.is_alive() and ws.error is None and ws.queries_served == 300


@pytest.mark.gpu
def test_gpu_wire_answers_equal_search():
    from falcon_b200 import FalconIndex
    from falcon_b200.serving import FalconServer
    from falcon_b200.wire import WireServer
    g, q = small_graph("sift", 6000, 128, 32, 200, seed=51)
    ix = FalconIndex(g)
    sv = FalconServer(ring_capacity=1024, max_k=64, ef_max=64, dim_max=128, idle_exit_us=5000)
    iid = sv.add_index(ix)
    c2f, f2c = _free_ports(2)
    P = dict(mc=2, mg=2, cand_queue_size=32, bloom_bits=16)
    ws = WireServer(sv, iid, 128, 64, c2f, "127.0.0.1", f2c, params=P, bind_host="127.0.0.1", connect_timeout=30)
    t = threading.Thread(target=ws.serve, daemon=True)
    t.start()
    batches = [q[i:i + 32] for i in range(0, len(q), 32)]
    res = _client(c2f, f2c, 128, 64, batches)
    t.join(30)
    assert not t.is_alive() and ws.error is None
    r = ix.search(q, k=64, ef=64, **P)
    for j, (ids, d) in enumerate(res):
        assert np.array_equal(ids, r.ids[j]) and np.array_equal(d.view(np.uint32), r.dists[j].view(np.uint32))
    if os.path.exists(CLIENT_SIM):   # the reference's own client against the GPU server
        c2f, f2c = _free_ports(2)
        ws = WireServer(sv, iid, 128, 64, c2f, "127.0.0.1", f2c, params=P, bind_host="127.0.0.1",
                        connect_timeout=30)
        t = threading.Thread(target=ws.serve, daemon=True)
        t.start()
        args = [CLIENT_SIM, "1", "127.0.0.1", str(c2f), str(f2c), "128", "64", "500", "64", "32", "2"]
        p = subprocess.run(args, cwd="/tmp", stdout=subprocess.PIPE, stderr=subprocess.STDOUT, timeout=120)
        t.join(30)
        assert p.returncode == 0 and b"End-to-end QPS" in p.stdout
        assert ws.error is None and ws.queries_served == 500
    sv.close()
    ix.close()
