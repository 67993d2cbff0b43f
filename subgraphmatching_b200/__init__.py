"""smx: B200-native subgraph matching behind the reference's plugin surface.

Python mirror of Orrinn/SubgraphMatching's filter / order / explore API
(inc/graph.h, inc/api.h, inc/filter.h, inc/order.h, inc/explore.h) over the C
ABI of libsmx (include/smx.h).  Names follow the reference so a driver written
against it reads the same:

    data = Graph.Load("data.txt")                 # Graph::Load, graph.h:190
    query = Query.Load("query.txt")               # Query::Load, graph.h:474
    can = CandidateParam(data, query)             # api.h:24
    ok = Filter_GQL(data, query, can)             # filter.h:1057
    order = Order_RI(query)                       # order.h:1138
    cfg = Config(useFilter=True, can=can)         # api.h:184
    ans, ms = explore_Intersection_Recursive(data, query, order, cfg)   # explore.h:613

All compute runs in libsmx's CUDA kernels on the device; there is no CPU
fallback.  Importing fails loudly if libsmx.so has not been built, and device
calls raise SmxError when no GPU is present.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import SmxError, check, lib

__all__ = [
    "Graph", "Query", "CandidateParam", "StopFlag", "Edges", "Config", "EnumOptions", "Stats",
    "Filter_NLF", "Filter_GQL", "Order_RI", "Order_GQL", "isValid", "explore",
    "explore_Intersection_Recursive", "explore_Intersection_Cache_DAF_Filter", "explore_batch",
    "SmxError", "device_count", "NLF", "GQL", "EXPLORE_CANDIDATES", "EXPLORE_CACHE_DAF",
]

NLF = 0
GQL = 1
EXPLORE_CANDIDATES = 0
EXPLORE_CACHE_DAF = 1

_u32p = ctypes.POINTER(ctypes.c_uint32)
_u64p = ctypes.POINTER(ctypes.c_uint64)


def _p32(a: np.ndarray):
    return a.ctypes.data_as(_u32p)


def _p64(a: np.ndarray):
    return a.ctypes.data_as(_u64p)


def device_count() -> int:
    return int(lib.smx_device_count())


class Graph:
    """Data graph resident in HBM (Graph, graph.h:51-380).  device=-1 keeps it host-only."""

    def __init__(self, handle):
        self._h = handle

    @classmethod
    def Load(cls, path: str, device: int = 0) -> "Graph":
        h = ctypes.c_void_p()
        check(lib.smx_graph_load_text(os.fsencode(path), device, ctypes.byref(h)))
        return cls(h)

    @classmethod
    def from_csr(cls, offsets, neighbors, labels=None, device: int = 0) -> "Graph":
        off = np.ascontiguousarray(offsets, dtype=np.uint64)
        nb = np.ascontiguousarray(neighbors if len(neighbors) else np.zeros(1), dtype=np.uint32)
        lab = None if labels is None else np.ascontiguousarray(labels, dtype=np.uint32)
        h = ctypes.c_void_p()
        check(lib.smx_graph_create(_p64(off), _p32(nb), None if lab is None else _p32(lab),
                                   len(off) - 1, int(off[-1]), device, ctypes.byref(h)))
        return cls(h)

    @classmethod
    def generate(cls, n: int, m: int, gamma: float, num_labels: int = 1, zipf_s: float = 1.0,
                 seed: int = 1, device: int = 0) -> "Graph":
        """Seeded Chung-Lu power-law graph (see smx_graph_generate)."""
        h = ctypes.c_void_p()
        check(lib.smx_graph_generate(n, m, gamma, num_labels, zipf_s, seed, device, ctypes.byref(h)))
        return cls(h)

    def __del__(self):
        if getattr(self, "_h", None) and lib is not None:
            lib.smx_graph_destroy(self._h)
            self._h = None

    def _info(self):
        n, m2, md, lc = ctypes.c_uint32(), ctypes.c_uint64(), ctypes.c_uint32(), ctypes.c_uint32()
        check(lib.smx_graph_info(self._h, ctypes.byref(n), ctypes.byref(m2), ctypes.byref(md), ctypes.byref(lc)))
        return n.value, m2.value, md.value, lc.value

    def getVertexCnt(self) -> int:
        return self._info()[0]

    def getEdgeCnt(self) -> int:
        return self._info()[1] // 2

    def getMaxDgree(self) -> int:
        return self._info()[2]

    def getLabelCnt(self) -> int:
        return self._info()[3]

    def csr(self):
        n, m2, _, _ = self._info()
        off = np.empty(n + 1, dtype=np.uint64)
        nb = np.empty(max(m2, 1), dtype=np.uint32)
        lab = np.empty(max(n, 1), dtype=np.uint32)
        check(lib.smx_graph_export(self._h, _p64(off), _p32(nb), _p32(lab)))
        return off, nb[:m2], lab[:n]

    def save(self, path: str) -> None:
        check(lib.smx_graph_save_text(self._h, os.fsencode(path)))


class Query:
    """Query graph (Query, graph.h:382-495)."""

    def __init__(self, handle):
        self._h = handle

    @classmethod
    def Load(cls, path: str) -> "Query":
        h = ctypes.c_void_p()
        check(lib.smx_query_load_text(os.fsencode(path), ctypes.byref(h)))
        return cls(h)

    @classmethod
    def from_csr(cls, offsets, neighbors, labels=None) -> "Query":
        off = np.ascontiguousarray(offsets, dtype=np.uint32)
        nb = np.ascontiguousarray(neighbors if len(neighbors) else np.zeros(1), dtype=np.uint32)
        lab = None if labels is None else np.ascontiguousarray(labels, dtype=np.uint32)
        h = ctypes.c_void_p()
        check(lib.smx_query_create(_p32(off), _p32(nb), None if lab is None else _p32(lab), len(off) - 1,
                                   ctypes.byref(h)))
        return cls(h)

    @classmethod
    def from_edges(cls, n: int, edges, labels=None) -> "Query":
        adj = [[] for _ in range(n)]
        for a, b in edges:
            adj[a].append(b)
            adj[b].append(a)
        off = np.zeros(n + 1, dtype=np.uint32)
        for i in range(n):
            off[i + 1] = off[i] + len(adj[i])
        nb = np.array([x for row in adj for x in sorted(row)], dtype=np.uint32)
        return cls.from_csr(off, nb, labels)

    @classmethod
    def generate(cls, data: Graph, k: int, dense: bool, seed: int) -> "Query":
        """Seeded random-walk query (see smx_query_generate)."""
        h = ctypes.c_void_p()
        check(lib.smx_query_generate(data._h, k, 1 if dense else 0, seed, ctypes.byref(h)))
        return cls(h)

    def __del__(self):
        if getattr(self, "_h", None) and lib is not None:
            lib.smx_query_destroy(self._h)
            self._h = None

    def _info(self):
        n, m, md = ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_uint32()
        check(lib.smx_query_info(self._h, ctypes.byref(n), ctypes.byref(m), ctypes.byref(md)))
        return n.value, m.value, md.value

    def getVertexCnt(self) -> int:
        return self._info()[0]

    def getEdgeCnt(self) -> int:
        return self._info()[1]

    def getMaxDgree(self) -> int:
        return self._info()[2]

    def csr(self):
        n, m, _ = self._info()
        off = np.empty(n + 1, dtype=np.uint32)
        nb = np.empty(max(2 * m, 1), dtype=np.uint32)
        lab = np.empty(n, dtype=np.uint32)
        check(lib.smx_query_export(self._h, _p32(off), _p32(nb), _p32(lab)))
        return off, nb[: 2 * m], lab

    def getVertexDegree(self, u: int) -> int:
        off, _, _ = self.csr()
        return int(off[u + 1] - off[u])

    def kcore(self) -> list[int]:
        n = self.getVertexCnt()
        out = np.empty(n, dtype=np.uint32)
        check(lib.smx_query_kcore(self._h, _p32(out)))
        return [int(x) for x in out]

    def getKCoreValue(self, u: int) -> int:
        return self.kcore()[u]

    def save(self, path: str) -> None:
        check(lib.smx_query_save_text(self._h, os.fsencode(path)))


@dataclass
class Edges:
    """edge_matrix[a][b] (Edges, graph.h:13-49), copied to the host."""

    _offset: np.ndarray
    _edge: np.ndarray
    _edge_v: np.ndarray
    _max_degree: int

    @property
    def _v_cnt(self) -> int:
        return len(self._offset) - 1

    @property
    def _e_cnt(self) -> int:
        return len(self._edge)

    def getNeb(self, i: int) -> np.ndarray:
        return self._edge[self._offset[i]: self._offset[i + 1]]


class CandidateParam:
    """Candidate sets and edge tables on the device (CandidateParam, api.h:9-164).

    Filled by Filter_NLF / Filter_GQL.  ``build_tables=False`` skips the edge
    tables (the cache explorer needs none)."""

    def __init__(self, data: Graph, query: Query, build_tables: bool = True):
        self.data = data
        self.query = query
        self.build_tables = build_tables
        self._h = None
        self.ok = False

    def _set(self, handle, ok: bool):
        self._release()
        self._h = handle
        self.ok = ok

    def _release(self):
        if getattr(self, "_h", None) is not None and lib is not None:
            lib.smx_cand_destroy(self._h)
        self._h = None

    def __del__(self):
        self._release()

    @property
    def candidates_count(self) -> list[int]:
        n = self.query.getVertexCnt()
        out = np.zeros(n, dtype=np.uint32)
        if self._h is not None:
            check(lib.smx_cand_counts(self._h, _p32(out)))
        return [int(x) for x in out]

    def candidates(self, u: int) -> np.ndarray:
        cnt = self.candidates_count[u]
        out = np.empty(max(cnt, 1), dtype=np.uint32)
        if cnt:
            check(lib.smx_cand_export(self._h, u, _p32(out)))
        return out[:cnt]

    def edge_matrix(self, a: int, b: int) -> Edges | None:
        if self._h is None:
            return None
        vc, ec, md = ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_uint32()
        if lib.smx_table_info(self._h, a, b, ctypes.byref(vc), ctypes.byref(ec), ctypes.byref(md)) != 0:
            return None
        off = np.empty(vc.value + 1, dtype=np.uint32)
        e = np.empty(max(ec.value, 1), dtype=np.uint32)
        ev = np.empty(max(ec.value, 1), dtype=np.uint32)
        check(lib.smx_table_export(self._h, a, b, _p32(off), _p32(e), _p32(ev)))
        return Edges(off, e[: ec.value], ev[: ec.value], md.value)

    def timing_ms(self) -> list[float]:
        out = (ctypes.c_double * 4)()
        check(lib.smx_cand_timing(self._h, out))
        return list(out)


def _filter(kind: int, data: Graph, query: Query, can: CandidateParam) -> bool:
    h = ctypes.c_void_p()
    rc = lib.smx_filter(data._h, query._h, kind, 1 if can.build_tables else 0, ctypes.byref(h))
    if rc not in (_lib.SMX_OK, _lib.SMX_EMPTY_CANDIDATES):
        check(rc)
    can._set(h, rc == _lib.SMX_OK)
    return rc == _lib.SMX_OK


def Filter_NLF(data: Graph, query: Query, can: CandidateParam) -> bool:
    """Filter_NLF (filter.h:1049-1055); returns False like the reference on an empty set."""
    return _filter(NLF, data, query, can)


def Filter_GQL(data: Graph, query: Query, can: CandidateParam) -> bool:
    """Filter_GQL (filter.h:1057-1063); returns False like the reference on an empty set."""
    return _filter(GQL, data, query, can)


def Order_RI(query: Query) -> list[int]:
    """Order_RI (order.h:1138-1281)."""
    n = query.getVertexCnt()
    out = np.empty(n, dtype=np.uint32)
    check(lib.smx_order_ri(query._h, _p32(out)))
    return [int(x) for x in out]


def Order_GQL(data: Graph, query: Query, can: CandidateParam) -> list[int]:
    """Order_GQL (order.h:563-597)."""
    n = query.getVertexCnt()
    out = np.empty(n, dtype=np.uint32)
    check(lib.smx_order_gql(query._h, can._h, _p32(out)))
    return [int(x) for x in out]


def isValid(order, query: Query) -> bool:
    """isValid (order.h:104-124)."""
    o = np.ascontiguousarray(order, dtype=np.uint32)
    if len(o) != query.getVertexCnt():
        return False
    return bool(lib.smx_order_valid(query._h, _p32(o)))


@dataclass
class Config:
    """Config (api.h:184-227)."""

    useFilter: bool = True
    useCache: bool = False
    useDAFFailingPrune: bool = False
    can: CandidateParam | None = None

    def Check(self) -> None:
        if self.useFilter and self.can is None:
            raise SmxError(_lib.SMX_BAD_ARGUMENT, "config error, use filter but canParam is nullptr")


@dataclass
class EnumOptions:
    explore: int = EXPLORE_CANDIDATES
    warps_per_block: int = 8
    blocks_per_sm: int = 0
    task_grab: int = 4
    stage_chunk: int = 1024
    gallop_ratio: int = 16
    bitmap_min: int = 0
    use_tma: int = 1
    failing_sets: int = 1
    lane_depth: int = 0
    time_budget_ms: float = 0.0
    budget_per_query: int = 0

    def to_c(self):
        o = _lib.EnumOpts()
        lib.smx_enum_opts_default(ctypes.byref(o))
        for k in ("explore", "warps_per_block", "blocks_per_sm", "task_grab", "stage_chunk", "gallop_ratio",
                  "bitmap_min", "use_tma", "failing_sets", "lane_depth", "budget_per_query"):
            setattr(o, k, int(getattr(self, k)))
        o.time_budget_ms = float(self.time_budget_ms)
        return o


@dataclass
class Stats:
    count: int = 0
    raw_count: int = 0
    intersections: int = 0
    nodes: int = 0
    bytes: int = 0
    pruned: int = 0
    tasks: int = 0
    kernel_ms: float = 0.0
    limit_reached: bool = False
    status: int = 0
    query_status: list | None = None  # explore_batch: SMX_OK / SMX_TIMEOUT per query

    @classmethod
    def from_c(cls, s) -> "Stats":
        return cls(s.count, s.raw_count, s.intersections, s.nodes, s.bytes, s.pruned, s.tasks, s.kernel_ms,
                   bool(s.limit_reached), s.status)


def explore(data: Graph, query: Query, can: CandidateParam, order=None, opts: EnumOptions | None = None,
            output_limit: int = 0, stop=None) -> Stats:
    """Count embeddings on the device; returns Stats (count = min(count, limit)).

    Timeouts and stops return normally with ``status`` set and a partial count."""
    opts = opts or EnumOptions()
    o = opts.to_c()
    st = _lib.StatsC()
    ord_arr = None if order is None else np.ascontiguousarray(order, dtype=np.uint32)
    stop_ptr = stop.ptr if isinstance(stop, StopFlag) else stop
    rc = lib.smx_enumerate(data._h, query._h, can._h, None if ord_arr is None else _p32(ord_arr), ctypes.byref(o),
                           output_limit, stop_ptr, ctypes.byref(st))
    if rc not in (_lib.SMX_OK, _lib.SMX_TIMEOUT, _lib.SMX_STOPPED):
        check(rc)
    out = Stats.from_c(st)
    out.status = rc
    return out


class StopFlag:
    """Pinned, device-mapped stop word (smx_stop_flag_create): the reference's
    std::atomic<bool> stop_flag.  ``set()`` from any host thread ends a running
    explore() with status SMX_STOPPED and a partial count."""

    def __init__(self, device: int = 0):
        self._p = _u32p()
        check(lib.smx_stop_flag_create(device, ctypes.byref(self._p)))

    def set(self, value: int = 1) -> None:
        self._p[0] = value

    def clear(self) -> None:
        self._p[0] = 0

    @property
    def ptr(self):
        return self._p

    def __del__(self):
        if getattr(self, "_p", None) and lib is not None:
            lib.smx_stop_flag_destroy(self._p)
            self._p = None


def explore_Intersection_Recursive(data: Graph, query: Query, order, cfg: Config, output_limit: int = 0,
                                   opts: EnumOptions | None = None):
    """explore_Intersection_Recursive<CandidatesBuffer> (explore.h:613-670): returns (ans, time_ms)."""
    cfg.Check()
    opts = opts or EnumOptions()
    opts.explore = EXPLORE_CANDIDATES
    st = explore(data, query, cfg.can, order, opts, output_limit)
    return st.count, st.kernel_ms


def explore_Intersection_Cache_DAF_Filter(data: Graph, query: Query, order, cfg: Config, output_limit: int = 0,
                                          opts: EnumOptions | None = None):
    """explore_Intersection_Cache_DAF_Filter (explore.h:1073-1129): returns (ans, time_ms)."""
    cfg.Check()
    opts = opts or EnumOptions()
    opts.explore = EXPLORE_CACHE_DAF
    opts.failing_sets = 1
    st = explore(data, query, cfg.can, order, opts, output_limit)
    return st.count, st.kernel_ms


def explore_batch(data: Graph, queries, cans, orders=None, opts: EnumOptions | None = None, output_limit: int = 0):
    """All queries in one persistent launch under a CUDA graph; returns (counts, Stats)."""
    opts = opts or EnumOptions()
    nq = len(queries)
    qs = (ctypes.c_void_p * nq)(*[q._h for q in queries])
    cs = (ctypes.c_void_p * nq)(*[c._h for c in cans])
    keep = []
    os_ = None
    if orders is not None:
        os_ = (_u32p * nq)()
        for i, o in enumerate(orders):
            if o is not None:
                a = np.ascontiguousarray(o, dtype=np.uint32)
                keep.append(a)
                os_[i] = _p32(a)
    counts = np.zeros(max(nq, 1), dtype=np.uint64)
    qstat = np.zeros(max(nq, 1), dtype=np.int32)
    st = _lib.StatsC()
    o = opts.to_c()
    rc = lib.smx_enumerate_batch(data._h, qs, cs, os_, nq, ctypes.byref(o), output_limit, _p64(counts),
                                 ctypes.byref(st), qstat.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)))
    if rc not in (_lib.SMX_OK, _lib.SMX_TIMEOUT, _lib.SMX_STOPPED):
        check(rc)
    out = Stats.from_c(st)
    out.status = rc
    out.query_status = [int(x) for x in qstat[:nq]]
    return [int(x) for x in counts[:nq]], out


# ---------------------------------------------------------------------- learned order
MLP_INPUTS = 64
MLP_PARAMS = 82689


def _pf(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


class MLP:
    """The learned-order cost model on a device (smx_mlp_*): 64-256-256-1,
    ReLU, BF16 weights / activations, FP32 accumulation, Adam on FP32 masters.
    No counterpart in the reference."""

    def __init__(self, device: int = 0, max_batch: int = 4096, seed: int = 0):
        h = ctypes.c_void_p()
        check(lib.smx_mlp_create(device, max_batch, seed, ctypes.byref(h)))
        self._h = h
        self.max_batch = max_batch

    def __del__(self):
        if getattr(self, "_h", None) and lib is not None:
            lib.smx_mlp_destroy(self._h)
            self._h = None

    @property
    def params(self) -> np.ndarray:
        p = np.zeros(MLP_PARAMS, dtype=np.float32)
        check(lib.smx_mlp_get_params(self._h, _pf(p), MLP_PARAMS))
        return p

    @params.setter
    def params(self, p) -> None:
        p = np.ascontiguousarray(p, dtype=np.float32)
        check(lib.smx_mlp_set_params(self._h, _pf(p), len(p)))

    def forward(self, x) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.float32).reshape(-1, MLP_INPUTS)
        y = np.zeros(len(x), dtype=np.float32)
        for i in range(0, len(x), self.max_batch):
            xs = np.ascontiguousarray(x[i:i + self.max_batch])
            ys = np.zeros(len(xs), dtype=np.float32)
            check(lib.smx_mlp_forward(self._h, _pf(xs), len(xs), _pf(ys)))
            y[i:i + len(xs)] = ys
        return y

    def gradients(self, x, t):
        x = np.ascontiguousarray(x, dtype=np.float32).reshape(-1, MLP_INPUTS)
        t = np.ascontiguousarray(t, dtype=np.float32)
        g = np.zeros(MLP_PARAMS, dtype=np.float32)
        loss = np.zeros(1, dtype=np.float32)
        check(lib.smx_mlp_gradients(self._h, _pf(x), _pf(t), len(x), _pf(g), _pf(loss)))
        return g, float(loss[0])

    def train_step(self, x, t, lr: float = 1e-3) -> float:
        x = np.ascontiguousarray(x, dtype=np.float32).reshape(-1, MLP_INPUTS)
        t = np.ascontiguousarray(t, dtype=np.float32)
        loss = np.zeros(1, dtype=np.float32)
        check(lib.smx_mlp_train_step(self._h, _pf(x), _pf(t), len(x), float(lr), _pf(loss)))
        return float(loss[0])

    def save(self, path: str) -> None:
        np.save(path, self.params)

    def load(self, path: str) -> None:
        self.params = np.load(path)


def order_features(query: Query, can: CandidateParam, order) -> np.ndarray:
    o = np.ascontiguousarray(order, dtype=np.uint32)
    f = np.zeros(MLP_INPUTS, dtype=np.float32)
    check(lib.smx_order_features(query._h, can._h, _p32(o), _pf(f)))
    return f


def order_beam(query: Query, can: CandidateParam, beam: int = 32, seed: int = 0) -> list[list[int]]:
    """RI, GQL and seeded randomized greedy orders (distinct, valid)."""
    n = query.getVertexCnt()
    out = np.zeros(beam * n, dtype=np.uint32)
    k = ctypes.c_uint32()
    check(lib.smx_order_beam(query._h, can._h, beam, seed, _p32(out), ctypes.byref(k)))
    return [[int(v) for v in out[i * n:(i + 1) * n]] for i in range(k.value)]


def Order_Learned(model: MLP, query: Query, can: CandidateParam, beam: int = 32, seed: int = 0) -> list[int]:
    """The beam order with the smallest predicted enumeration work."""
    n = query.getVertexCnt()
    out = np.zeros(n, dtype=np.uint32)
    pred = ctypes.c_float()
    check(lib.smx_order_learned(model._h, query._h, can._h, beam, seed, _p32(out), ctypes.byref(pred)))
    return [int(v) for v in out]
