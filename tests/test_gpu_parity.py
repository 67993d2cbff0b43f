"""Parity of the CUDA path with the oracle on a B200 (marked gpu).

Calls go through the C ABI (the package's ctypes layer).  Integer work, so the
bar is bit-exact: candidate arrays, edge-table CSRs, orders and embedding
counts equal the reference's golden vectors (tests/golden/golden.json, made
by the reference's own code) or the oracle's, on every query; at full size,
size-independent invariants (count independent of explorer, order and
filter; a capped count equals the cap).
"""
from __future__ import annotations

import threading
import time

import numpy as np
import pytest

import subgraphmatching_b200 as smx
from subgraphmatching_b200 import _lib
from helpers import host_graph, query_file, sha

pytestmark = pytest.mark.gpu

# exhaustive golden counts above this many embeddings are checked by the
# dedicated large-count test only
BIG = 2_000_000_000


def device_graph(n, m, gamma, labels, seed):
    g, path = host_graph(n, m, gamma, labels, seed)
    off, nb, lab = g.csr()
    return g, smx.Graph.from_csr(off, nb, lab, device=0), path


def filter_record(can, n):
    rec = {"ok": can.ok, "counts": can.candidates_count}
    if can.ok:
        rec["cand_sha"] = sha(can.candidates(u) for u in range(n))
        tabs, total = [], 0
        for a in range(n):
            for b in range(n):
                t = can.edge_matrix(a, b)
                if t is not None:
                    tabs += [np.array([a, b, t._max_degree]), t._offset, t._edge, t._edge_v]
                    total += len(t._edge)
        rec["table_entries"] = total
        rec["table_sha"] = sha(tabs)
    return rec


def test_golden_filters_orders_and_counts(gpu, golden):
    for gcase in golden["graphs"]:
        hg, dg, _ = device_graph(gcase["n"], gcase["m"], gcase["gamma"], gcase["labels"], gcase["seed"])
        for qc in gcase["queries"]:
            q, _ = query_file(hg, qc["k"], qc["dense"], qc["seed"])
            n = qc["k"]
            can_n = smx.CandidateParam(dg, q)
            smx.Filter_NLF(dg, q, can_n)
            assert filter_record(can_n, n) == qc["nlf"], (gcase["name"], n, "nlf")
            can = smx.CandidateParam(dg, q)
            smx.Filter_GQL(dg, q, can)
            assert filter_record(can, n) == qc["gql"], (gcase["name"], n, "gql")
            assert smx.Order_RI(q) == qc["order_ri"]
            assert q.kcore() == qc["kcore"]
            if not can.ok:
                continue
            assert smx.Order_GQL(dg, q, can) == qc["order_gql"]
            if qc["cap"] == 0 and qc["count"] > BIG:
                continue
            for mode in (smx.EXPLORE_CANDIDATES, smx.EXPLORE_CACHE_DAF):
                st = smx.explore(dg, q, can, qc["order_ri"], smx.EnumOptions(explore=mode), qc["cap"])
                assert st.status == 0
                assert st.count == qc["count"], (gcase["name"], n, qc["seed"], mode, st.count)


def test_random_small_graphs_match_oracle(gpu, port):
    rng = np.random.default_rng(11)
    for trial in range(6):
        labels = int(rng.choice([1, 2, 5]))
        hg, dg, gpath = device_graph(1500, 6000, 2.4, labels, 100 + trial)
        gp = port.load_graph(gpath)
        for k in (3, 4, 5, 6, 7):
            dense = bool(rng.integers(2))
            q, qpath = query_file(hg, k, dense, 1000 * trial + k)
            qp = port.load_query(qpath)
            for kind in (smx.NLF, smx.GQL):
                can = smx.CandidateParam(dg, q)
                ok = (smx.Filter_NLF if kind == smx.NLF else smx.Filter_GQL)(dg, q, can)
                cp = port.filter(gp, qp, kind)
                assert ok == cp.ok
                assert can.candidates_count == port.counts(cp)
                if not ok:
                    continue
                for order in (smx.Order_RI(q), smx.Order_GQL(dg, q, can)):
                    ref = port.explore(gp, qp, cp, order, 50_000_000, 8)[0]
                    for mode in (smx.EXPLORE_CANDIDATES, smx.EXPLORE_CACHE_DAF):
                        for tma in (0, 1):
                            st = smx.explore(dg, q, can, order, smx.EnumOptions(explore=mode, use_tma=tma),
                                             50_000_000)
                            assert st.count == ref, (trial, k, kind, mode, tma)


def test_intersection_modes_agree(gpu, port):
    """Merge (staged) and galloping intersections, tiny and large chunks."""
    hg, dg, gpath = device_graph(9500, 35000, 2.5, 1, 1)
    gp = port.load_graph(gpath)
    q, qpath = query_file(hg, 6, True, 14)
    qp = port.load_query(qpath)
    can = smx.CandidateParam(dg, q)
    smx.Filter_GQL(dg, q, can)
    cp = port.filter(gp, qp, 1)
    order = smx.Order_RI(q)
    ref = port.explore(gp, qp, cp, order, 0, 8)[0]
    for chunk, ratio, wpb, grab in ((64, 1, 8, 1), (64, 1_000_000, 4, 16), (4096, 4, 8, 4), (32, 2, 2, 64)):
        for mode in (0, 1):
            opts = smx.EnumOptions(explore=mode, stage_chunk=chunk, gallop_ratio=ratio, warps_per_block=wpb,
                                   task_grab=grab)
            assert smx.explore(dg, q, can, order, opts).count == ref


def test_lane_depths_agree(gpu, golden):
    """Per-lane subtree enumeration from every possible lane depth (0 = off,
    -1 = chosen from the query) gives the golden counts, with galloping on and
    off."""
    for gcase in golden["graphs"]:
        hg, dg, _ = device_graph(gcase["n"], gcase["m"], gcase["gamma"], gcase["labels"], gcase["seed"])
        for qc in gcase["queries"]:
            if qc["k"] < 5 or (qc["cap"] == 0 and qc["count"] > BIG):
                continue
            q, _ = query_file(hg, qc["k"], qc["dense"], qc["seed"])
            can = smx.CandidateParam(dg, q)
            if not smx.Filter_GQL(dg, q, can):
                continue
            for ld in [-1, 0] + list(range(2, qc["k"] - 1)):
                for ratio in (16, 1):
                    opts = smx.EnumOptions(explore=smx.EXPLORE_CANDIDATES, lane_depth=ld, gallop_ratio=ratio)
                    st = smx.explore(dg, q, can, qc["order_ri"], opts, qc["cap"])
                    assert st.status == 0
                    assert st.count == qc["count"], (gcase["name"], qc["k"], qc["seed"], ld, ratio, st.count)


def test_leaf_bitmap_agrees(gpu, golden):
    """Last-depth counts through the membership bitmap (forced on from one
    element, default threshold, off) give the golden counts."""
    for gcase in golden["graphs"]:
        hg, dg, _ = device_graph(gcase["n"], gcase["m"], gcase["gamma"], gcase["labels"], gcase["seed"])
        for qc in gcase["queries"]:
            if qc["k"] < 4 or (qc["cap"] == 0 and qc["count"] > BIG):
                continue
            q, _ = query_file(hg, qc["k"], qc["dense"], qc["seed"])
            can = smx.CandidateParam(dg, q)
            if not smx.Filter_GQL(dg, q, can):
                continue
            for bmin in (1, 0, -1):
                opts = smx.EnumOptions(explore=smx.EXPLORE_CANDIDATES, bitmap_min=bmin)
                st = smx.explore(dg, q, can, qc["order_ri"], opts, qc["cap"])
                assert st.status == 0
                assert st.count == qc["count"], (gcase["name"], qc["k"], qc["seed"], bmin, st.count)


def test_edge_cases(gpu):
    hg, dg, _ = device_graph(2000, 9000, 2.5, 4, 3)
    _, _, lab = hg.csr()
    # one-vertex query: count = |C(u)|
    q1 = smx.Query.from_csr(np.array([0, 0], dtype=np.uint32), np.zeros(0, dtype=np.uint32), [2])
    can = smx.CandidateParam(dg, q1)
    assert smx.Filter_GQL(dg, q1, can)
    assert smx.explore(dg, q1, can).count == int(np.sum(lab == 2))
    # two-vertex query: ordered adjacent pairs with the right labels
    q2 = smx.Query.from_edges(2, [(0, 1)], [1, 1])
    can = smx.CandidateParam(dg, q2)
    assert smx.Filter_GQL(dg, q2, can)
    off, nb, _ = hg.csr()
    expect = sum(1 for v in range(hg.getVertexCnt()) if lab[v] == 1
                 for w in nb[off[v]:off[v + 1]] if lab[w] == 1)
    for mode in (0, 1):
        assert smx.explore(dg, q2, can, opts=smx.EnumOptions(explore=mode)).count == expect
    # a label the data graph does not have: empty candidates, filter returns False
    qx = smx.Query.from_edges(3, [(0, 1), (1, 2)], [0, 9, 0])
    can = smx.CandidateParam(dg, qx)
    assert not smx.Filter_NLF(dg, qx, can)
    assert not smx.Filter_GQL(dg, qx, can)
    with pytest.raises(smx.SmxError) as e:
        smx.explore(dg, qx, can)
    assert e.value.status == _lib.SMX_EMPTY_CANDIDATES
    # disconnected order
    q3 = smx.Query.from_edges(4, [(0, 1), (1, 2), (2, 3)])
    can = smx.CandidateParam(dg, q3)
    smx.Filter_GQL(dg, q3, can)
    with pytest.raises(smx.SmxError) as e:
        smx.explore(dg, q3, can, [0, 2, 1, 3])
    assert e.value.status == _lib.SMX_INVALID_ORDER
    # cache explorer without tables, candidate explorer needs them
    can = smx.CandidateParam(dg, q3, build_tables=False)
    smx.Filter_GQL(dg, q3, can)
    with pytest.raises(smx.SmxError):
        smx.explore(dg, q3, can, opts=smx.EnumOptions(explore=0))
    assert smx.explore(dg, q3, can, opts=smx.EnumOptions(explore=1)).count > 0


def golden_count(golden, graph, k, seed):
    for g in golden["graphs"]:
        if g["name"] == graph:
            for q in g["queries"]:
                if q["k"] == k and q["seed"] == seed:
                    return q["count"]
    raise KeyError((graph, k, seed))


def test_limit_semantics(gpu, golden):
    hg, dg, gpath = device_graph(9500, 35000, 2.5, 1, 1)
    q, qpath = query_file(hg, 5, True, 12)
    can = smx.CandidateParam(dg, q)
    smx.Filter_GQL(dg, q, can)
    full = smx.explore(dg, q, can).count
    assert full == golden_count(golden, "cl9500_unlabelled", 5, 12)  # the reference's count
    for lim in (1, 999, full - 1, full, full + 1):
        for mode in (0, 1):
            st = smx.explore(dg, q, can, opts=smx.EnumOptions(explore=mode), output_limit=lim)
            assert st.count == min(full, lim)
            assert st.limit_reached == (lim <= full)


def test_batch_matches_single(gpu):
    hg, dg, _ = device_graph(9500, 35000, 2.5, 8, 2)
    qs, cans, singles = [], [], []
    for i, (k, dense) in enumerate([(4, True), (6, True), (8, False), (5, True), (12, True), (3, False)]):
        q, _ = query_file(hg, k, dense, 500 + i)
        can = smx.CandidateParam(dg, q)
        smx.Filter_GQL(dg, q, can)
        qs.append(q)
        cans.append(can)
        singles.append(smx.explore(dg, q, can, output_limit=5_000_000).count if can.ok else 0)
    # an empty-candidate query inside the batch counts 0
    qx = smx.Query.from_edges(3, [(0, 1), (1, 2)], [0, 31, 0])
    cx = smx.CandidateParam(dg, qx)
    smx.Filter_GQL(dg, qx, cx)
    qs.append(qx)
    cans.append(cx)
    singles.append(0)
    for mode in (0, 1):
        counts, st = smx.explore_batch(dg, qs, cans, opts=smx.EnumOptions(explore=mode), output_limit=5_000_000)
        assert counts == singles


LONG = ("cl9500_unlabelled", 6, False, 13)  # 28.3 billion embeddings (reference count)


def test_time_budget_returns_partial_count(gpu, golden):
    hg, dg, _ = device_graph(9500, 35000, 2.5, 1, 1)
    q, _ = query_file(hg, LONG[1], LONG[2], LONG[3])
    full = golden_count(golden, LONG[0], LONG[1], LONG[3])
    can = smx.CandidateParam(dg, q)
    smx.Filter_GQL(dg, q, can)
    t0 = time.time()
    st = smx.explore(dg, q, can, opts=smx.EnumOptions(time_budget_ms=50))
    assert st.status == _lib.SMX_TIMEOUT
    assert 0 < st.count < full
    assert time.time() - t0 < 30


def test_batch_budget_per_query(gpu, golden):
    """With budget_per_query the budget runs for each query from its first
    task: the 28.3-billion query stops with SMX_TIMEOUT and a partial count,
    the small queries of the same launch finish with their exact counts."""
    hg, dg, _ = device_graph(9500, 35000, 2.5, 1, 1)
    specs = [(LONG[1], LONG[2], LONG[3]), (4, True, 11), (5, True, 12)]
    qs, cans = [], []
    for k, dense, seed in specs:
        q, _ = query_file(hg, k, dense, seed)
        can = smx.CandidateParam(dg, q)
        smx.Filter_GQL(dg, q, can)
        qs.append(q)
        cans.append(can)
    counts, st = smx.explore_batch(dg, qs, cans, opts=smx.EnumOptions(time_budget_ms=20, budget_per_query=1))
    assert st.status == _lib.SMX_TIMEOUT
    assert st.query_status == [_lib.SMX_TIMEOUT, 0, 0]
    assert 0 < counts[0] < golden_count(golden, LONG[0], LONG[1], LONG[3])
    assert counts[1] == golden_count(golden, "cl9500_unlabelled", 4, 11)
    assert counts[2] == golden_count(golden, "cl9500_unlabelled", 5, 12)


def test_stop_flag_from_another_thread(gpu, golden):
    # a dense 8-vertex query on the 1M-vertex graph runs for minutes uncapped
    hg, dg, _ = device_graph(1_000_000, 10_000_000, 2.2, 1, 2)
    q, _ = query_file(hg, 8, True, 10_000)
    can = smx.CandidateParam(dg, q)
    smx.Filter_GQL(dg, q, can)
    flag = smx.StopFlag(0)
    timer = threading.Timer(1.0, flag.set)
    timer.start()
    t0 = time.time()
    st = smx.explore(dg, q, can, stop=flag)
    timer.join()
    assert st.status == _lib.SMX_STOPPED
    assert st.count > 0 and time.time() - t0 < 30
    flag.clear()   # the context stays usable
    hg, dg, _ = device_graph(9500, 35000, 2.5, 1, 1)
    q2, _ = query_file(hg, 4, True, 11)
    can2 = smx.CandidateParam(dg, q2)
    smx.Filter_GQL(dg, q2, can2)
    assert smx.explore(dg, q2, can2, stop=flag).count == golden_count(golden, "cl9500_unlabelled", 4, 11)


def test_large_exhaustive_count(gpu, golden):
    """28,302,124,178 embeddings, exhaustive, against the reference's count."""
    hg, dg, _ = device_graph(9500, 35000, 2.5, 1, 1)
    q, _ = query_file(hg, LONG[1], LONG[2], LONG[3])
    can = smx.CandidateParam(dg, q)
    smx.Filter_GQL(dg, q, can)
    st = smx.explore(dg, q, can, opts=smx.EnumOptions(time_budget_ms=300_000))
    assert st.status == 0
    assert st.count == golden_count(golden, LONG[0], LONG[1], LONG[3])


def test_scale_invariants(gpu):
    """cfg-2-sized graph (1M vertices, 10M edges): the capped count is the
    same for both explorers, both orders and both filters."""
    dg = smx.Graph.generate(1_000_000, 10_000_000, 2.2, 1, 1.0, 2, device=0)
    cap = 10_000_000
    for i, (k, dense) in enumerate([(8, True), (8, False), (12, True), (12, False)]):
        q = smx.Query.generate(dg, k, dense, 70 + i)
        counts = set()
        for kind in (smx.NLF, smx.GQL):
            can = smx.CandidateParam(dg, q)
            assert (smx.Filter_NLF if kind == smx.NLF else smx.Filter_GQL)(dg, q, can)
            for order in (smx.Order_RI(q), smx.Order_GQL(dg, q, can)):
                for mode in (0, 1):
                    st = smx.explore(dg, q, can, order, smx.EnumOptions(explore=mode, time_budget_ms=60_000), cap)
                    assert st.status == 0
                    counts.add(st.count)
        assert len(counts) == 1, (k, dense, counts)
