"""Host side of libsmx on CPU: the C-ABI library loads and exports every entry
point include/smx.h declares; text I/O, generators, k-core, RI order and
argument / format errors behave like the reference (or fail with a status
where the reference would exit)."""
from __future__ import annotations

import ctypes
import os
import re

import numpy as np
import pytest

import subgraphmatching_b200 as smx
from subgraphmatching_b200 import _lib
from helpers import TMP, host_graph, query_file

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "smx.h")).read()
    return sorted(set(re.findall(r"\b(smx_[a-z_0-9]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    names = declared_symbols()
    assert len(names) >= 30
    L = ctypes.CDLL(_lib.LIB_PATH)
    for name in names:
        assert hasattr(L, name), name
    assert {n for n, _, _ in _lib.SIGNATURES} == set(names)


def test_status_strings():
    assert _lib.lib.smx_status_str(0) == b"ok"
    assert _lib.lib.smx_status_str(1) == b"empty candidate set"


def test_generator_is_deterministic_and_exact():
    g1 = smx.Graph.generate(3000, 12000, 2.3, 1, 1.0, 42, device=-1)
    g2 = smx.Graph.generate(3000, 12000, 2.3, 1, 1.0, 42, device=-1)
    o1, n1, _ = g1.csr()
    o2, n2, _ = g2.csr()
    assert np.array_equal(o1, o2) and np.array_equal(n1, n2)
    assert g1.getEdgeCnt() == 12000
    deg = np.diff(o1.astype(np.int64))
    assert deg.sum() == 24000
    for v in range(3000):  # rows strictly ascending, no loops
        row = n1[o1[v]:o1[v + 1]]
        assert np.all(np.diff(row.astype(np.int64)) > 0) and v not in row
    assert g1.getMaxDgree() <= int(1.5 * np.sqrt(24000))


def test_zipf_labels():
    g = smx.Graph.generate(20000, 60000, 2.2, 32, 1.0, 3, device=-1)
    _, _, lab = g.csr()
    freq = np.bincount(lab, minlength=32) / len(lab)
    assert g.getLabelCnt() == 32
    assert abs(freq[0] - 1 / sum(1 / (i + 1) for i in range(32))) < 0.02
    assert freq[0] > freq[1] > freq[4] > freq[31]


def test_text_roundtrip():
    g, path = host_graph(2000, 9000, 2.5, 4, 3)
    g2 = smx.Graph.Load(path, device=-1)
    for a, b in zip(g.csr(), g2.csr()):
        assert np.array_equal(a, b)


def test_walk_queries(port):
    g, path = host_graph(9500, 35000, 2.5, 1, 1)
    for k in (4, 8, 16, 24, 32):
        for dense in (True, False):
            q = smx.Query.generate(g, k, dense, 100 + k)
            assert q.getVertexCnt() == k
            assert smx.isValid(smx.Order_RI(q), q)
            if not dense:
                assert q.getEdgeCnt() >= k - 1


def test_ri_order_and_kcore_match_oracle(port):
    g, gpath = host_graph(9500, 35000, 2.5, 1, 1)
    for seed in range(12):
        q, qpath = query_file(g, 4 + seed * 2, seed % 2 == 0, seed)
        qp = port.load_query(qpath)
        assert smx.Order_RI(q) == port.order_ri(qp)
        assert q.kcore() == [port.kcore(qp, v) for v in range(q.getVertexCnt())]


def _write(name, text):
    p = os.path.join(TMP, name)
    with open(p, "w") as f:
        f.write(text)
    return p


def test_bad_text_formats():
    cases = {
        "deg.txt": "t 3 2\nv 0 0 1\nv 1 0 1\nv 2 0 1\ne 0 1\ne 1 2\n",      # declared degree wrong
        "loop.txt": "t 2 1\nv 0 0 2\nv 1 0 0\ne 0 0\n",
        "dup.txt": "t 2 2\nv 0 0 2\nv 1 0 2\ne 0 1\ne 0 1\n",
        "range.txt": "t 2 1\nv 0 0 1\nv 1 0 1\ne 0 5\n",
        "count.txt": "t 2 2\nv 0 0 1\nv 1 0 1\ne 0 1\n",
        "junk.txt": "x 2 2\n",
    }
    for name, text in cases.items():
        with pytest.raises(smx.SmxError) as e:
            smx.Graph.Load(_write(name, text), device=-1)
        assert e.value.status == _lib.SMX_BAD_FORMAT, name
    with pytest.raises(smx.SmxError) as e:
        smx.Graph.Load(os.path.join(TMP, "missing.txt"), device=-1)
    assert e.value.status == _lib.SMX_IO_ERROR


def test_query_limits_and_validation():
    with pytest.raises(smx.SmxError) as e:
        smx.Query.from_edges(65, [(i, i + 1) for i in range(64)])
    assert e.value.status == _lib.SMX_TOO_LARGE
    with pytest.raises(smx.SmxError):
        smx.Query.from_csr(np.array([0, 1, 1], dtype=np.uint32), np.array([1], dtype=np.uint32))  # not symmetric
    q = smx.Query.from_edges(4, [(0, 1), (1, 2), (2, 3)])
    assert smx.isValid([1, 0, 2, 3], q)
    assert not smx.isValid([0, 2, 1, 3], q)   # 2 has no earlier neighbour
    assert not smx.isValid([0, 1, 1, 3], q)   # not a permutation
    assert smx.Order_RI(q) == [1, 2, 0, 3]  # RI tie-breaks, order.h:1182-1267


def test_device_calls_fail_loudly_without_gpu():
    if smx.device_count() > 0:
        pytest.skip("a GPU is present")
    with pytest.raises(smx.SmxError) as e:
        smx.Graph.generate(100, 300, 2.5, device=0)
    assert e.value.status == _lib.SMX_NO_DEVICE
    g = smx.Graph.generate(100, 300, 2.5, device=-1)
    q = smx.Query.from_edges(2, [(0, 1)])
    with pytest.raises(smx.SmxError) as e:
        smx.Filter_GQL(g, q, smx.CandidateParam(g, q))
    assert e.value.status == _lib.SMX_NO_DEVICE
