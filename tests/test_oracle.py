"""The oracle pinned against the reference (CPU).

* the C restatement (oracle/port) reproduces the golden vectors that the
  reference itself produced (tests/golden/golden.json);
* where the reference sources are present, the known answers on the
  reference's bundled hprd graph (densest 4- and 5-vertex subgraphs of its
  n16 query: 7,362,038 and 34,149,984 embeddings) are reproduced by both the
  port and the compiled reference;
* an independent brute-force enumerator agrees with the port on tiny graphs.
"""
from __future__ import annotations

import itertools
import os

import numpy as np
import pytest

from helpers import brute_force_count, file_sha, host_graph, query_file, sha

REF = "/root/reference"
EXHAUSTIVE_CPU_LIMIT = 2_000_000_000  # larger exhaustive counts are GPU-only tests


def _golden_cases(golden):
    for gcase in golden["graphs"]:
        for qcase in gcase["queries"]:
            yield gcase, qcase


def test_golden_graphs_regenerate(golden):
    for gcase in golden["graphs"]:
        g, path = host_graph(gcase["n"], gcase["m"], gcase["gamma"], gcase["labels"], gcase["seed"])
        assert file_sha(path) == gcase["sha256"], f"generator drift on {gcase['name']}"
        assert g.getMaxDgree() == gcase["max_degree"]


def _filter_record(port, gp, qp, kind, n):
    c = port.filter(gp, qp, kind)
    rec = {"ok": c.ok, "counts": port.counts(c)}
    if c.ok:
        rec["cand_sha"] = sha(port.candidates(c, u) for u in range(n))
        tabs, total = [], 0
        for a in range(n):
            for b in range(n):
                t = port.table(c, a, b)
                if t is not None:
                    tabs += [np.array([a, b, t.max_degree]), t.offset, t.edge, t.edge_v]
                    total += len(t.edge)
        rec["table_entries"] = total
        rec["table_sha"] = sha(tabs)
    return c, rec


def test_port_matches_golden(golden, port):
    for gcase, qcase in _golden_cases(golden):
        g, gpath = host_graph(gcase["n"], gcase["m"], gcase["gamma"], gcase["labels"], gcase["seed"])
        q, qpath = query_file(g, qcase["k"], qcase["dense"], qcase["seed"])
        assert file_sha(qpath) == qcase["sha256"]
        gp, qp = port.load_graph(gpath), port.load_query(qpath)
        n = qcase["k"]
        _, nlf = _filter_record(port, gp, qp, 0, n)
        cg, gql = _filter_record(port, gp, qp, 1, n)
        assert nlf == qcase["nlf"], (gcase["name"], n)
        assert gql == qcase["gql"], (gcase["name"], n)
        assert port.order_ri(qp) == qcase["order_ri"]
        assert [port.kcore(qp, v) for v in range(n)] == qcase["kcore"]
        if not cg.ok:
            continue
        assert port.order_gql(gp, qp, cg) == qcase["order_gql"]
        if qcase["cap"] == 0 and qcase["count"] > EXHAUSTIVE_CPU_LIMIT:
            continue
        cnt, _, _ = port.explore(gp, qp, cg, qcase["order_ri"], qcase["cap"], 8)
        assert cnt == qcase["count"], (gcase["name"], n, qcase["seed"])


def _dk_query(k: int) -> str:
    """Densest connected induced k-subgraph of the reference's n16 query
    (first in itertools.combinations order), relabelled 0..k-1."""
    lines = open(os.path.join(REF, "data", "query", "n16_query.txt")).read().split("\n")
    edges = [tuple(map(int, ln.split()[1:3])) for ln in lines if ln.startswith("e")]
    best = None
    for S in itertools.combinations(range(16), k):
        s = set(S)
        E = [e for e in edges if e[0] in s and e[1] in s]
        adj = {v: set() for v in S}
        for a, b in E:
            adj[a].add(b)
            adj[b].add(a)
        seen, st = {S[0]}, [S[0]]
        while st:
            x = st.pop()
            for y in adj[x]:
                if y not in seen:
                    seen.add(y)
                    st.append(y)
        if len(seen) == k and (best is None or len(E) > len(best[1])):
            best = (S, E)
    S, E = best
    rl = {v: i for i, v in enumerate(S)}
    deg = [0] * k
    for a, b in E:
        deg[rl[a]] += 1
        deg[rl[b]] += 1
    from helpers import TMP

    path = os.path.join(TMP, f"d{k}.txt")
    with open(path, "w") as f:
        f.write(f"t {k} {len(E)}\n")
        for i in range(k):
            f.write(f"v {i} 0 {deg[i]}\n")
        for a, b in E:
            f.write(f"e {rl[a]} {rl[b]}\n")
    return path


@pytest.mark.skipif(not os.path.isdir(REF), reason="reference fixtures not present")
@pytest.mark.parametrize("k,expected", [(4, 7_362_038), (5, 34_149_984)])
def test_hprd_known_answers(port, k, expected):
    hprd = os.path.join(REF, "data", "data", "hprd.txt")
    gp = port.load_graph(hprd)
    qpath = _dk_query(k)
    qp = port.load_query(qpath)
    for kind in (0, 1):
        c = port.filter(gp, qp, kind)
        order = port.order_ri(qp)
        assert port.explore(gp, qp, c, order, 0, 8)[0] == expected


@pytest.mark.skipif(not os.path.isdir(REF), reason="reference fixtures not present")
def test_hprd_n16_filters_match_reference(port, ref):
    hprd = os.path.join(REF, "data", "data", "hprd.txt")
    q16 = os.path.join(REF, "data", "query", "n16_query.txt")
    gp, qp = port.load_graph(hprd), port.load_query(q16)
    gr, qr = ref.load_graph(hprd), ref.load_query(q16)
    for kind in (0, 1):
        cp, cr = port.filter(gp, qp, kind), ref.filter(gr, qr, kind)
        assert port.counts(cp) == ref.counts(cr)
        for u in range(16):
            assert np.array_equal(port.candidates(cp, u), ref.candidates(cr, u))
    assert port.order_ri(qp) == ref.order_ri(qr) == [0, 4, 2, 12, 14, 11, 15, 1, 10, 7, 5, 6, 9, 13, 3, 8]


def _tiny_case(rng, n, p, labels, k):
    adj = [[] for _ in range(n)]
    for a in range(n):
        for b in range(a + 1, n):
            if rng.random() < p:
                adj[a].append(b)
                adj[b].append(a)
    lab = [int(rng.integers(labels)) for _ in range(n)]
    # query: random connected induced subgraph of the data graph
    start = int(rng.integers(n))
    while not adj[start]:
        start = int(rng.integers(n))
    vs = [start]
    while len(vs) < k:
        cand = sorted({y for x in vs for y in adj[x]} - set(vs))
        if not cand:
            break
        vs.append(int(rng.choice(cand)))
    idx = {v: i for i, v in enumerate(vs)}
    qadj = [sorted(idx[y] for y in adj[v] if y in idx) for v in vs]
    qlab = [lab[v] for v in vs]
    return adj, lab, qadj, qlab


def _csr(adj):
    off = np.zeros(len(adj) + 1, dtype=np.uint64)
    for i, a in enumerate(adj):
        off[i + 1] = off[i] + len(a)
    nb = np.array([x for a in adj for x in sorted(a)], dtype=np.uint32)
    return off, nb


def test_port_matches_brute_force(port):
    rng = np.random.default_rng(5)
    for trial in range(25):
        n = int(rng.integers(6, 12))
        adj, lab, qadj, qlab = _tiny_case(rng, n, 0.45, int(rng.integers(1, 3)), int(rng.integers(2, 5)))
        k = len(qadj)
        off, nb = _csr(adj)
        gp = port.graph_from_csr(off, nb, np.array(lab, dtype=np.uint32))
        qoff, qnb = _csr(qadj)
        qp = port.graph_from_csr(qoff, qnb, np.array(qlab, dtype=np.uint32))
        expect = brute_force_count(n, adj, lab, k, qadj, qlab)
        c = port.filter(gp, qp, 1)
        got = port.explore(gp, qp, c, port.order_ri(qp), 0, 2)[0] if c.ok else 0
        assert got == expect, (trial, n, k)
