"""Small helpers shared by the tests (graph generation cached per session,
writing text files for the oracle, hashes as in tests/golden/make_golden.py)."""
from __future__ import annotations

import functools
import hashlib
import os
import tempfile

import numpy as np

import subgraphmatching_b200 as smx

TMP = tempfile.mkdtemp(prefix="smx_tests_")


def sha(arrays) -> str:
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a, dtype=np.uint32).tobytes())
        h.update(b"|")
    return h.hexdigest()


def file_sha(path: str) -> str:
    with open(path, "rb") as f:
        return hashlib.sha256(f.read()).hexdigest()


@functools.lru_cache(maxsize=None)
def host_graph(n, m, gamma, labels, seed):
    """Host-only graph plus its text file path."""
    g = smx.Graph.generate(n, m, gamma, labels, 1.0, seed, device=-1)
    path = os.path.join(TMP, f"g_{n}_{m}_{gamma}_{labels}_{seed}.txt")
    g.save(path)
    return g, path


def query_file(g, k, dense, seed):
    q = smx.Query.generate(g, k, dense, seed)
    path = os.path.join(TMP, f"q_{id(g)}_{k}_{int(dense)}_{seed}.txt")
    q.save(path)
    return q, path


def brute_force_count(n_data, adj_data, lab_data, n_q, adj_q, lab_q):
    """Independent count of injective, label- and edge-preserving maps (tiny graphs)."""
    adj_sets = [set(a) for a in adj_data]
    order = []
    seen = set()
    # BFS order over the query for pruning
    for s in range(n_q):
        if s in seen:
            continue
        stack = [s]
        seen.add(s)
        while stack:
            x = stack.pop(0)
            order.append(x)
            for y in adj_q[x]:
                if y not in seen:
                    seen.add(y)
                    stack.append(y)
    pos = {u: i for i, u in enumerate(order)}
    m = [None] * n_q
    used = set()

    def rec(i):
        if i == n_q:
            return 1
        u = order[i]
        total = 0
        for v in range(n_data):
            if v in used or lab_data[v] != lab_q[u]:
                continue
            ok = all(m[w] in adj_sets[v] for w in adj_q[u] if pos[w] < i)
            if not ok:
                continue
            m[u] = v
            used.add(v)
            total += rec(i + 1)
            used.discard(v)
            m[u] = None
        return total

    return rec(0)
