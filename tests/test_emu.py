"""The product's CUDA kernels (filter, edge tables, both explorers, batching)
executed by the CPU warp emulator (tests/emu) and checked bit-exactly against
the oracle on small seeded graphs.  Same kernel sources as the GPU build;
this catches warp-logic errors (divergent shuffles, slot bookkeeping,
failing-set pruning) before a GPU run."""
from __future__ import annotations

import os

import numpy as np
import pytest

from emu_driver import p32
from helpers import TMP, host_graph, query_file


def smx_generate(n, m, seed):
    import subgraphmatching_b200 as smx

    return smx.Graph.generate(n, m, 2.2, 1, 1.0, seed=seed, device=-1)


def smx_query(g, k, seed):
    import subgraphmatching_b200 as smx

    return smx.Query.generate(g, k, dense=True, seed=seed)

CASES = [  # (n, m, labels, seed, [(k, dense, qseed)], filter kinds)
    (300, 900, 1, 5, [(4, True, 2), (5, False, 3)], (1,)),
    (300, 900, 3, 6, [(5, True, 6)], (0, 1)),
]


@pytest.mark.parametrize("n,m,labels,seed,queries,kinds", CASES)
def test_emulated_pipeline_matches_oracle(emu, port, n, m, labels, seed, queries, kinds):
    g, gpath = host_graph(n, m, 2.5, labels, seed)
    off, nb, lab = g.csr()
    dg = emu.graph(off, nb, lab)
    gp = port.load_graph(gpath)
    for k, dense, qseed in queries:
        q, qpath = query_file(g, k, dense, qseed)
        qp = port.load_query(qpath)
        qo, qn, ql = q.csr()
        dq = emu.query(qo, qn, ql)
        for kind in kinds:
            c, ok = emu.filter(dg, dq, kind)
            cp = port.filter(gp, qp, kind)
            assert ok == cp.ok
            cnt = emu.counts(c, k)
            assert list(cnt) == port.counts(cp)
            if not ok:
                continue
            for u in range(k):
                assert np.array_equal(emu.candidates(c, u, int(cnt[u])), port.candidates(cp, u))
            for a in range(k):
                for b in range(k):
                    t, tp = emu.table(c, a, b), port.table(cp, a, b)
                    assert (t is None) == (tp is None)
                    if t is not None:
                        assert np.array_equal(t[0], tp.offset) and np.array_equal(t[1], tp.edge)
                        assert np.array_equal(t[2], tp.edge_v) and t[3] == tp.max_degree
            order = emu.order_ri(dq, k)
            ref = port.explore(gp, qp, cp, order, 0, 4)[0]
            for mode in (0, 1):
                st = emu.enumerate(dg, dq, c, order, explore=mode)
                assert st.count == ref, (k, kind, mode)
            # failing sets off: same count
            st = emu.enumerate(dg, dq, c, order, explore=1, failing_sets=0)
            assert st.count == ref


def test_emulated_limit_and_batch(emu, port):
    g, gpath = host_graph(300, 900, 2.5, 1, 5)
    off, nb, lab = g.csr()
    dg = emu.graph(off, nb, lab)
    gp = port.load_graph(gpath)
    qs, cs, refs, orders = [], [], [], []
    for k, dense, qseed in [(3, True, 11), (4, False, 12), (4, True, 14)]:
        q, qpath = query_file(g, k, dense, qseed)
        qo, qn, ql = q.csr()
        dq = emu.query(qo, qn, ql)
        c, ok = emu.filter(dg, dq, 1)
        qp = port.load_query(qpath)
        cp = port.filter(gp, qp, 1)
        order = emu.order_ri(dq, k)
        refs.append(port.explore(gp, qp, cp, order, 0, 2)[0] if ok else 0)
        qs.append(dq)
        cs.append(c)
        orders.append(order)
    for mode in (0, 1):
        counts, st = emu.batch(dg, qs, cs, explore=mode)
        assert counts == refs
    # a limit below the count is reported as the limit (explore.h:587-590)
    big = max(range(len(refs)), key=lambda i: refs[i])
    lim = max(1, refs[big] // 3)
    st = emu.enumerate(dg, qs[big], cs[big], orders[big], explore=0, limit=lim)
    assert st.count == lim and st.limit_reached == 1 and st.raw_count >= lim


def test_emulated_lane_subtrees_and_galloping(emu, port):
    """Per-lane subtree enumeration below the lane depth (chosen from the
    query, or forced to depth 2), the galloping intersection (ratio 1, so
    every long row is probed by binary search) and the last-depth bitmap give
    the oracle's counts."""
    g, gpath = host_graph(900, 4000, 2.2, 1, 5)
    off, nb, lab = g.csr()
    dg = emu.graph(off, nb, lab)
    gp = port.load_graph(gpath)
    for k, dense, qseed in [(5, True, 2), (6, True, 3)]:
        q, qpath = query_file(g, k, dense, qseed)
        qp = port.load_query(qpath)
        qo, qn, ql = q.csr()
        dq = emu.query(qo, qn, ql)
        c, ok = emu.filter(dg, dq, 1)
        assert ok
        order = emu.order_ri(dq, k)
        ref = port.explore(gp, qp, port.filter(gp, qp, 1), order, 0, 4)[0]
        assert ref > 0
        for lane_depth in (-1, 2):
            assert emu.enumerate(dg, dq, c, order, explore=0, lane_depth=lane_depth).count == ref
        assert emu.enumerate(dg, dq, c, order, explore=0, lane_depth=0, gallop_ratio=1).count == ref
        for bmin in (1, -1):  # last depth through the bitmap from one element / never
            assert emu.enumerate(dg, dq, c, order, explore=0, bitmap_min=bmin).count == ref
        assert emu.enumerate(dg, dq, c, order, explore=1, gallop_ratio=1).count == ref


def test_emulated_graph_destroyed_before_its_candidates(emu):
    """Finalizers may run in any order (Python's cycle collector): a data graph
    destroyed before a candidate set built on it frees that set's device
    memory and detaches it; the set's handle then refuses device reads with
    SMX_BAD_ARGUMENT and can still be destroyed."""
    g, _ = host_graph(300, 900, 2.5, 1, 5)
    off, nb, lab = g.csr()
    dg = emu.graph(off, nb, lab)
    q, _ = query_file(g, 4, True, 2)
    qo, qn, ql = q.csr()
    dq = emu.query(qo, qn, ql)
    c, ok = emu.filter(dg, dq, 1)
    assert ok
    emu.L.smx_graph_destroy(dg)
    assert emu.table(c, 0, 1) is None
    assert emu.L.smx_cand_export(c, 0, p32(np.zeros(8, dtype=np.uint32))) == 6  # SMX_BAD_ARGUMENT
    emu.L.smx_cand_destroy(c)
    emu.L.smx_query_destroy(dq)


def test_emulated_factored_tail(emu, port):
    """Queries whose last two depths close on shallow vertices (the factored
    tail: one sum per shallow node, corrected per node by inclusion-exclusion
    over the embedded vertices) against the oracle, with the tail on (default)
    and off (bitmap_min = -1)."""
    for gn, gm, gs, k, seed in [(600, 2400, 7, 8, 1055), (900, 4000, 5, 7, 1046), (600, 2400, 7, 7, 1110)]:
        g = smx_generate(gn, gm, gs)
        off, nb, lab = g.csr()
        dg = emu.graph(off, nb, lab)
        path = os.path.join(TMP, f"g{gn}_{gm}_{gs}.txt")
        g.save(path)
        gp = port.load_graph(path)
        q = smx_query(g, k, seed)
        qpath = os.path.join(TMP, f"tail_q{seed}.txt")
        q.save(qpath)
        qp = port.load_query(qpath)
        qo, qn, ql = q.csr()
        dq = emu.query(qo, qn, ql)
        c, ok = emu.filter(dg, dq, 1)
        assert ok
        order = emu.order_ri(dq, k)
        ref = min(port.explore(gp, qp, port.filter(gp, qp, 1), order, 3_000_000, 8)[0], 3_000_000)
        assert ref > 0
        for bmin in (0, -1):
            assert emu.enumerate(dg, dq, c, order, explore=0, limit=3_000_000, bitmap_min=bmin).count == ref
