"""smx_enumerate_noalloc against smx_enumerate on a B200 (marked gpu).

smx_enumerate allocates device memory on every call.  Callers whose device
memory is owned by someone else's allocator, or that must not take
cudaMalloc's implicit synchronisation or its failure mid-run, use
smx_enumerate_noalloc instead: the same kernel with its working memory in a
static device array the library reserves at load time.  Both are called
through the C ABI on the same inputs, the allocation-free one twice in a
row (the array keeps the previous call's contents, so the second call checks
that everything that must start at zero is cleared).  Counts are integers:
they must be equal.

The file is named to be collected last, so a run that stops at the first
failure has run every other test before this one.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

import subgraphmatching_b200 as smx
from subgraphmatching_b200 import _lib
from helpers import host_graph, query_file

pytestmark = pytest.mark.gpu

CASES = [  # (graph name in the golden file, query size, dense, seed)
    ("cl9500_unlabelled", 5, True, 12),
    ("cl9500_unlabelled", 8, True, 15),
    ("cl9500_unlabelled", 12, True, 17),
    ("cl9500_labels8", 8, False, 24),
    ("cl2000_labels4", 10, False, 33),
]


def golden_query(golden, name, k, seed):
    for g in golden["graphs"]:
        if g["name"] == name:
            for q in g["queries"]:
                if q["k"] == k and q["seed"] == seed:
                    return g, q
    return None, None


def run(fn, dg, q, can, order, explore, limit):
    o = smx.EnumOptions(explore=explore).to_c()
    st = _lib.StatsC()
    arr = np.ascontiguousarray(order, dtype=np.uint32)
    rc = fn(dg._h, q._h, can._h, arr.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)), ctypes.byref(o), limit, None,
            ctypes.byref(st))
    return rc, st


@pytest.mark.parametrize("name,k,dense,seed", CASES)
def test_noalloc_matches_enumerate(gpu, golden, name, k, dense, seed):
    gcase, qc = golden_query(golden, name, k, seed)
    if qc is None:
        pytest.skip("query not in the golden file")
    hg, _ = host_graph(gcase["n"], gcase["m"], gcase["gamma"], gcase["labels"], gcase["seed"])
    off, nb, lab = hg.csr()
    dg = smx.Graph.from_csr(off, nb, lab, device=0)
    q, _ = query_file(hg, k, dense, seed)
    can = smx.CandidateParam(dg, q)
    if not smx.Filter_GQL(dg, q, can):
        pytest.skip("empty candidate set")
    order = smx.Order_RI(q)
    limit = qc["cap"]  # 0: exhaustive
    for explore in (smx.EXPLORE_CANDIDATES, smx.EXPLORE_CACHE_DAF):
        rc, ref = run(_lib.lib.smx_enumerate, dg, q, can, order, explore, limit)
        assert rc == 0 and ref.status == 0
        for _ in range(2):
            rc, st = run(_lib.lib.smx_enumerate_noalloc, dg, q, can, order, explore, limit)
            assert rc == 0, _lib.lib.smx_last_error()
            assert st.status == 0
            assert st.count == ref.count, (name, k, seed, explore, st.count, ref.count)
            assert st.limit_reached == ref.limit_reached
        assert ref.count == qc["count"]
