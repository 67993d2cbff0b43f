"""Oracles for the filter -> edge table -> order -> enumerate path.

TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and bench.py's
cpu_baseline / reference legs may import this package, and only as the
checker.  The product (subgraphmatching_b200 / libsmx) never imports it.

Two interchangeable back ends with one Python surface:

* ``PortOracle``  -- oracle/port/oracle.c, a C restatement of the reference
  algorithms (built by ``make -C oracle port`` into oracle/lib/).
* ``RefOracle``   -- the reference's own headers compiled where they lie with
  oracle/ref_driver.cpp (``make -C oracle ref`` into oracle/_ref/).  Present
  only where the reference sources were available at build time; the built
  library travels with the repository snapshot.

Both expose: load_graph / load_query, filter (NLF=0 / GQL=1), candidates,
counts, table, order_ri, order_gql, order_valid, kcore, explore.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_LIB = os.path.join(HERE, "lib", "libsmx_oracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libsmx_refdriver.so")

NLF = 0
GQL = 1

_vp = ctypes.c_void_p
_u32 = ctypes.c_uint32
_u64 = ctypes.c_uint64
_pu32 = ctypes.POINTER(ctypes.c_uint32)
_pdbl = ctypes.POINTER(ctypes.c_double)
_pu64 = ctypes.POINTER(ctypes.c_uint64)


def _ptr(a: np.ndarray, ctype=ctypes.c_uint32):
    return a.ctypes.data_as(ctypes.POINTER(ctype))


@dataclass
class Table:
    offset: np.ndarray
    edge: np.ndarray
    edge_v: np.ndarray
    max_degree: int


class _Handle:
    def __init__(self, ptr, free):
        self.ptr = ptr
        self._free = free

    def __del__(self):
        if self.ptr:
            self._free(self.ptr)
            self.ptr = None


class _Oracle:
    prefix = ""
    path = ""

    def __init__(self):
        if not os.path.exists(self.path):
            raise FileNotFoundError(f"oracle library missing: {self.path} (run __graft_entry__.build())")
        L = ctypes.CDLL(self.path)
        p = self.prefix
        self.L = L
        self._f = lambda name: getattr(L, p + name)
        f = self._f
        f("graph_free").argtypes = [_vp]
        f("cand_free").argtypes = [_vp]
        f("filter").restype = _vp
        f("filter").argtypes = [_vp, _vp, ctypes.c_int, _pdbl]
        f("cand_ok").argtypes = [_vp]
        f("cand_count").argtypes = [_vp, _u32]
        f("cand_count").restype = _u32
        f("cand_copy").argtypes = [_vp, _u32, _pu32]
        f("table_info").argtypes = [_vp, _u32, _u32, _pu32, _pu32, _pu32]
        f("table_copy").argtypes = [_vp, _u32, _u32, _pu32, _pu32, _pu32]
        f("order_ri").argtypes = [_vp, _pu32]
        f("order_gql").argtypes = [_vp, _vp, _vp, _pu32]
        f("order_valid").argtypes = [_vp, _pu32, _u32]
        f("query_kcore").argtypes = [_vp, _u32]
        f("query_kcore").restype = _u32
        f("graph_vcount").argtypes = [_vp]
        f("graph_vcount").restype = _u32

    def load_graph(self, path: str):
        raise NotImplementedError

    def load_query(self, path: str):
        return self.load_graph(path)

    def vcount(self, g) -> int:
        return int(self._f("graph_vcount")(g.ptr))

    def kcore(self, q, v: int) -> int:
        return int(self._f("query_kcore")(q.ptr, v))

    def filter(self, data, query, kind: int):
        ms = ctypes.c_double()
        c = self._f("filter")(data.ptr, query.ptr, kind, ctypes.byref(ms))
        h = _Handle(c, self._f("cand_free"))
        h.ok = bool(self._f("cand_ok")(c))
        h.ms = ms.value
        h.n = self.vcount(query)
        return h

    def candidates(self, cand, u: int) -> np.ndarray:
        n = self._f("cand_count")(cand.ptr, u)
        out = np.empty(max(n, 1), dtype=np.uint32)
        if n:
            self._f("cand_copy")(cand.ptr, u, _ptr(out))
        return out[:n]

    def counts(self, cand) -> list[int]:
        return [int(self._f("cand_count")(cand.ptr, u)) for u in range(cand.n)]

    def table(self, cand, a: int, b: int) -> Table | None:
        vc, ec, md = _u32(), _u32(), _u32()
        if not self._f("table_info")(cand.ptr, a, b, ctypes.byref(vc), ctypes.byref(ec), ctypes.byref(md)):
            return None
        off = np.empty(vc.value + 1, dtype=np.uint32)
        e = np.empty(max(ec.value, 1), dtype=np.uint32)
        ev = np.empty(max(ec.value, 1), dtype=np.uint32)
        self._f("table_copy")(cand.ptr, a, b, _ptr(off), _ptr(e), _ptr(ev))
        return Table(off, e[: ec.value], ev[: ec.value], md.value)

    def order_ri(self, query) -> list[int]:
        n = self.vcount(query)
        out = np.zeros(n, dtype=np.uint32)
        self._f("order_ri")(query.ptr, _ptr(out))
        return [int(x) for x in out]

    def order_gql(self, data, query, cand) -> list[int]:
        n = self.vcount(query)
        out = np.zeros(n, dtype=np.uint32)
        self._f("order_gql")(data.ptr, query.ptr, cand.ptr, _ptr(out))
        return [int(x) for x in out]

    def order_valid(self, query, order) -> bool:
        o = np.asarray(order, dtype=np.uint32)
        return bool(self._f("order_valid")(query.ptr, _ptr(o), len(o)))


class PortOracle(_Oracle):
    """C restatement (oracle/port/oracle.c)."""

    prefix = "smxo_"
    path = PORT_LIB

    def __init__(self):
        super().__init__()
        f = self._f
        f("graph_load").restype = _vp
        f("graph_load").argtypes = [ctypes.c_char_p]
        f("graph_from_csr").restype = _vp
        f("graph_from_csr").argtypes = [_u32, _pu64, _pu32, _pu32]
        f("explore").restype = _u64
        f("explore").argtypes = [_vp, _vp, _vp, _pu32, _u64, ctypes.c_int, _pdbl, _pu64]

    def load_graph(self, path: str):
        p = self._f("graph_load")(os.fsencode(path))
        if not p:
            raise OSError(f"cannot load {path}")
        return _Handle(p, self._f("graph_free"))

    def graph_from_csr(self, offsets: np.ndarray, neighbors: np.ndarray, labels: np.ndarray | None):
        off = np.ascontiguousarray(offsets, dtype=np.uint64)
        nb = np.ascontiguousarray(neighbors if len(neighbors) else np.zeros(1), dtype=np.uint32)
        lab = None if labels is None else np.ascontiguousarray(labels, dtype=np.uint32)
        n = len(off) - 1
        p = self._f("graph_from_csr")(n, _ptr(off, ctypes.c_uint64), _ptr(nb), None if lab is None else _ptr(lab))
        h = _Handle(p, self._f("graph_free"))
        return h

    def explore(self, data, query, cand, order, limit: int = 0, threads: int = 1):
        """Candidate-table enumeration count (explore.h:613-670): (count, ms, bytes)."""
        o = np.asarray(order, dtype=np.uint32)
        ms = ctypes.c_double()
        wb = _u64()
        n = self._f("explore")(data.ptr, query.ptr, cand.ptr, _ptr(o), limit, threads, ctypes.byref(ms),
                               ctypes.byref(wb))
        return int(n), ms.value, int(wb.value)


class RefOracle(_Oracle):
    """The reference's own code (oracle/_ref/libsmx_refdriver.so)."""

    prefix = "smxref_"
    path = REF_LIB

    CANDIDATES = 0
    CACHE_DAF_FILTER = 1
    CANDIDATES_DAF = 2

    def __init__(self):
        super().__init__()
        f = self._f
        f("graph_load").restype = _vp
        f("graph_load").argtypes = [ctypes.c_char_p]
        f("query_load").restype = _vp
        f("query_load").argtypes = [ctypes.c_char_p]
        f("query_free").argtypes = [_vp]
        f("explore").restype = _u64
        f("explore").argtypes = [_vp, _vp, _vp, _pu32, ctypes.c_int, _u64, ctypes.c_int, _pdbl, _pu64]

    def load_graph(self, path: str):
        if not os.path.exists(path):
            raise OSError(f"cannot load {path}")
        return _Handle(self._f("graph_load")(os.fsencode(path)), self._f("graph_free"))

    def load_query(self, path: str):
        if not os.path.exists(path):
            raise OSError(f"cannot load {path}")
        return _Handle(self._f("query_load")(os.fsencode(path)), self._f("query_free"))

    def explore(self, data, query, cand, order, limit: int = 0, threads: int = 1, explorer: int = 0):
        """The reference explorer `explorer` (see ref_driver.cpp): (count, ms, intersections)."""
        o = np.asarray(order, dtype=np.uint32)
        ms = ctypes.c_double()
        it = _u64()
        n = self._f("explore")(data.ptr, query.ptr, cand.ptr, _ptr(o), explorer, limit, threads, ctypes.byref(ms),
                               ctypes.byref(it))
        return int(n), ms.value, int(it.value)


def available() -> dict[str, bool]:
    return {"port": os.path.exists(PORT_LIB), "ref": os.path.exists(REF_LIB)}
