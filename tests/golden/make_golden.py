"""Generate tests/golden/golden.json from the reference itself.

Runs the reference's own code (oracle/_ref/libsmx_refdriver.so, built from the
reference sources by oracle/Makefile) on seeded synthetic inputs made by this
project's generator, and records its outputs: candidate counts and hashes
(Filter_NLF / Filter_GQL), edge-table sizes and hashes (buildTables), RI and
GQL orders, and embedding counts (explore_Intersection_Recursive with
CandidatesBuffer, cross-checked with explore_Intersection_Cache_DAF_Filter).

The synthetic inputs stand in for the reference's bundled hprd fixture (a
9,460-vertex / 34,998-edge protein network): Chung-Lu graphs with the same
shape (9,500 vertices, 35,000 edges, degree exponent 2.5), unlabelled and with
8 Zipf(1) labels, and random-walk queries.  The graph text is regenerated from
its seed at test time; its sha256 is recorded so generator drift is caught.

Usage (needs the reference build, i.e. run where the reference sources are):
    python tests/golden/make_golden.py
"""
from __future__ import annotations

import hashlib
import json
import os
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.abspath(os.path.join(HERE, "..", ".."))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

# Graph / query cases: (name, n, m, gamma, labels, seed, [(k, dense, seed, cap)])
CASES = [
    ("cl9500_unlabelled", 9500, 35000, 2.5, 1, 1, [
        (4, True, 11, 0), (5, True, 12, 0), (6, False, 13, 0), (6, True, 14, 0),
        (8, True, 15, 0), (8, False, 16, 10_000_000), (12, True, 17, 10_000_000),
        (16, True, 18, 10_000_000), (16, False, 19, 1_000_000),
    ]),
    ("cl9500_labels8", 9500, 35000, 2.5, 8, 2, [
        (4, True, 21, 0), (6, True, 22, 0), (8, True, 23, 0), (8, False, 24, 0),
        (12, True, 25, 0), (16, True, 26, 10_000_000), (24, True, 27, 10_000_000),
    ]),
    ("cl2000_labels4", 2000, 9000, 2.5, 4, 3, [
        (5, True, 31, 0), (7, True, 32, 0), (10, False, 33, 1_000_000),
    ]),
]


def sha(arrays) -> str:
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a, dtype=np.uint32).tobytes())
        h.update(b"|")
    return h.hexdigest()


def file_sha(path: str) -> str:
    with open(path, "rb") as f:
        return hashlib.sha256(f.read()).hexdigest()


def describe_filter(R, gr, qr, kind):
    c = R.filter(gr, qr, kind)
    n = c.n
    out = {"ok": c.ok, "counts": R.counts(c)}
    if c.ok:
        out["cand_sha"] = sha(R.candidates(c, u) for u in range(n))
        tabs = []
        total = 0
        for a in range(n):
            for b in range(n):
                t = R.table(c, a, b)
                if t is not None:
                    tabs += [np.array([a, b, t.max_degree]), t.offset, t.edge, t.edge_v]
                    total += len(t.edge)
        out["table_entries"] = total
        out["table_sha"] = sha(tabs)
    return c, out


def main() -> None:
    import subgraphmatching_b200 as smx
    from oracle import GQL, NLF, RefOracle

    R = RefOracle()
    golden = {"generator": "smx_graph_generate / smx_query_generate (Chung-Lu, random walk)", "graphs": []}
    with tempfile.TemporaryDirectory() as tmp:
        for name, n, m, gamma, labels, seed, queries in CASES:
            g = smx.Graph.generate(n, m, gamma, labels, 1.0, seed, device=-1)
            gpath = os.path.join(tmp, name + ".txt")
            g.save(gpath)
            gr = R.load_graph(gpath)
            entry = {"name": name, "n": n, "m": m, "gamma": gamma, "labels": labels, "seed": seed,
                     "sha256": file_sha(gpath), "max_degree": g.getMaxDgree(), "queries": []}
            for k, dense, qseed, cap in queries:
                q = smx.Query.generate(g, k, dense, qseed)
                qpath = os.path.join(tmp, f"{name}_q{k}_{qseed}.txt")
                q.save(qpath)
                qr = R.load_query(qpath)
                qe = {"k": k, "dense": dense, "seed": qseed, "edges": q.getEdgeCnt(), "sha256": file_sha(qpath),
                      "cap": cap}
                cn, qe["nlf"] = describe_filter(R, gr, qr, NLF)
                cg, qe["gql"] = describe_filter(R, gr, qr, GQL)
                qe["order_ri"] = R.order_ri(qr)
                qe["kcore"] = [R.kcore(qr, v) for v in range(k)]
                if cg.ok:
                    qe["order_gql"] = R.order_gql(gr, qr, cg)
                    cnt, ms, _ = R.explore(gr, qr, cg, qe["order_ri"], cap, 8, R.CANDIDATES)
                    cnt2, ms2, _ = R.explore(gr, qr, cg, qe["order_ri"], cap, 8, R.CACHE_DAF_FILTER)
                    assert cnt == cnt2, (name, k, qseed, cnt, cnt2)
                    qe["count"] = cnt
                    qe["ref_ms"] = round(ms, 1)
                    print(f"{name} k={k} dense={dense} seed={qseed}: count={cnt} (cap {cap}) {ms:.0f} ms", flush=True)
                else:
                    qe["count"] = 0
                entry["queries"].append(qe)
            golden["graphs"].append(entry)
    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump(golden, f, indent=1)


if __name__ == "__main__":
    main()
