"""Thin driver over a library that exports include/smx.h, used by the tests to
run the CPU warp emulator build (tests/emu/libsmx_emu.so) of the product's
kernels.  TEST INFRASTRUCTURE ONLY."""
from __future__ import annotations

import ctypes
import os

import numpy as np

from subgraphmatching_b200 import _lib

HERE = os.path.dirname(os.path.abspath(__file__))
EMU_PATH = os.path.join(HERE, "emu", "libsmx_emu.so")

_u32p = ctypes.POINTER(ctypes.c_uint32)
_u64p = ctypes.POINTER(ctypes.c_uint64)


def p32(a):
    return a.ctypes.data_as(_u32p)


def p64(a):
    return a.ctypes.data_as(_u64p)


class Driver:
    def __init__(self, path: str = EMU_PATH):
        self.L = _lib.load(path)

    def check(self, rc):
        if rc != 0:
            raise _lib.SmxError(rc, self.L.smx_last_error().decode())

    def graph(self, off, nb, lab):
        off = np.ascontiguousarray(off, dtype=np.uint64)
        nb = np.ascontiguousarray(nb if len(nb) else np.zeros(1), dtype=np.uint32)
        lab = np.ascontiguousarray(lab, dtype=np.uint32)
        h = ctypes.c_void_p()
        self.check(self.L.smx_graph_create(p64(off), p32(nb), p32(lab), len(off) - 1, int(off[-1]), 0,
                                           ctypes.byref(h)))
        return h

    def query(self, off, nb, lab):
        off = np.ascontiguousarray(off, dtype=np.uint32)
        nb = np.ascontiguousarray(nb if len(nb) else np.zeros(1), dtype=np.uint32)
        lab = np.ascontiguousarray(lab, dtype=np.uint32)
        h = ctypes.c_void_p()
        self.check(self.L.smx_query_create(p32(off), p32(nb), p32(lab), len(off) - 1, ctypes.byref(h)))
        return h

    def filter(self, g, q, kind, tables=True):
        h = ctypes.c_void_p()
        rc = self.L.smx_filter(g, q, kind, 1 if tables else 0, ctypes.byref(h))
        if rc not in (0, 1):
            self.check(rc)
        return h, rc == 0

    def counts(self, c, n):
        out = np.zeros(n, dtype=np.uint32)
        self.check(self.L.smx_cand_counts(c, p32(out)))
        return out

    def candidates(self, c, u, cnt):
        out = np.zeros(max(cnt, 1), dtype=np.uint32)
        self.check(self.L.smx_cand_export(c, u, p32(out)))
        return out[:cnt]

    def table(self, c, a, b):
        vc, ec, md = ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_uint32()
        if self.L.smx_table_info(c, a, b, ctypes.byref(vc), ctypes.byref(ec), ctypes.byref(md)) != 0:
            return None
        off = np.zeros(vc.value + 1, dtype=np.uint32)
        e = np.zeros(max(ec.value, 1), dtype=np.uint32)
        ev = np.zeros(max(ec.value, 1), dtype=np.uint32)
        self.check(self.L.smx_table_export(c, a, b, p32(off), p32(e), p32(ev)))
        return off, e[: ec.value], ev[: ec.value], md.value

    def order_ri(self, q, n):
        out = np.zeros(n, dtype=np.uint32)
        self.check(self.L.smx_order_ri(q, p32(out)))
        return [int(x) for x in out]

    def enumerate(self, g, q, c, order, explore=0, limit=0, **kw):
        o = _lib.EnumOpts()
        self.L.smx_enum_opts_default(ctypes.byref(o))
        o.explore = explore
        o.use_tma = 0
        o.warps_per_block = kw.get("warps_per_block", 2)
        o.stage_chunk = kw.get("stage_chunk", 64)
        o.gallop_ratio = kw.get("gallop_ratio", 4)
        o.task_grab = kw.get("task_grab", 1)
        o.failing_sets = kw.get("failing_sets", 1)
        o.lane_depth = kw.get("lane_depth", 0)
        o.bitmap_min = kw.get("bitmap_min", 0)
        st = _lib.StatsC()
        arr = np.ascontiguousarray(order, dtype=np.uint32)
        rc = self.L.smx_enumerate(g, q, c, p32(arr), ctypes.byref(o), limit, None, ctypes.byref(st))
        self.check(rc)
        return st

    def batch(self, g, qs, cs, explore=0, limit=0, **kw):
        o = _lib.EnumOpts()
        self.L.smx_enum_opts_default(ctypes.byref(o))
        o.explore = explore
        o.use_tma = 0
        o.warps_per_block = kw.get("warps_per_block", 2)
        o.stage_chunk = kw.get("stage_chunk", 64)
        o.gallop_ratio = kw.get("gallop_ratio", 4)
        o.task_grab = kw.get("task_grab", 2)
        nq = len(qs)
        qa = (ctypes.c_void_p * nq)(*qs)
        ca = (ctypes.c_void_p * nq)(*cs)
        counts = np.zeros(nq, dtype=np.uint64)
        st = _lib.StatsC()
        self.check(self.L.smx_enumerate_batch(g, qa, ca, None, nq, ctypes.byref(o), limit, p64(counts),
                                              ctypes.byref(st), None))
        return [int(x) for x in counts], st
