"""The learned-order cost model on CPU: the numpy restatement (oracle/mlp.py)
against finite differences, and the CUDA kernels of csrc/mlp.cu run by the
CPU warp emulator against that restatement (forward, gradients, Adam steps),
plus the order features and beam."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from emu_driver import p32
from helpers import host_graph, query_file
from oracle import mlp as ref

_pf = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))  # noqa: E731


def init_params(seed):
    rng = np.random.default_rng(seed)
    p = np.zeros(ref.N_PARAMS, dtype=np.float32)
    P = ref.split(p)
    P["W1"][:] = rng.normal(0, np.sqrt(2 / 64), P["W1"].shape)
    P["W2"][:] = rng.normal(0, np.sqrt(2 / 256), P["W2"].shape)
    P["W3"][:] = rng.normal(0, np.sqrt(1 / 256), P["W3"].shape)
    P["b1"][:] = rng.normal(0, 0.05, 256)
    P["b2"][:] = rng.normal(0, 0.05, 256)
    P["b3"][:] = 0.3
    return p


def test_oracle_gradients_match_finite_differences():
    rng = np.random.default_rng(1)
    p = init_params(2).astype(np.float64)
    x = rng.normal(0, 1, (9, 64))
    t = rng.normal(0, 1, 9)
    g, _ = ref.gradients(p, x, t, rounding=False)
    for idx in list(rng.choice(ref.N_PARAMS, 40, replace=False)) + [ref.N_PARAMS - 1]:
        e = np.zeros_like(p)
        e[idx] = 1e-6
        fd = (ref.gradients(p + e, x, t, rounding=False)[1] - ref.gradients(p - e, x, t, rounding=False)[1]) / 2e-6
        assert abs(fd - g[idx]) <= 1e-5 + 1e-4 * abs(fd), idx


def test_bf16_rounding_is_nearest_even():
    x = np.array([1.0, 1.00390625, 1.005859375, 3.0e38, -2.5, 0.0], dtype=np.float32)
    r = ref.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0078125 and r[4] == -2.5 and r[5] == 0.0


@pytest.fixture(scope="module")
def emu_mlp(emu):
    h = ctypes.c_void_p()
    emu.check(emu.L.smx_mlp_create(0, 512, 7, ctypes.byref(h)))
    yield emu, h
    emu.L.smx_mlp_destroy(h)


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a, dtype=np.float64) - b) / max(np.linalg.norm(b), 1e-12))


def test_emulated_kernels_match_oracle(emu_mlp):
    emu, h = emu_mlp
    L = emu.L
    p = init_params(3)
    L.smx_mlp_set_params(h, _pf(p), len(p))
    rng = np.random.default_rng(4)
    for n in (1, 37, 300):
        x = rng.normal(0, 1, (n, 64)).astype(np.float32)
        t = rng.normal(0, 1, n).astype(np.float32)
        y = np.zeros(n, dtype=np.float32)
        emu.check(L.smx_mlp_forward(h, _pf(x), n, _pf(y)))
        assert rel(y, ref.forward(p, x)[3]) < 1e-2
        g = np.zeros(ref.N_PARAMS, dtype=np.float32)
        loss = np.zeros(1, dtype=np.float32)
        emu.check(L.smx_mlp_gradients(h, _pf(x), _pf(t), n, _pf(g), _pf(loss)))
        gr, lr_ = ref.gradients(p, x, t)
        assert rel(g, gr) < 2e-2
        assert abs(loss[0] - lr_) <= 1e-3 * max(1.0, lr_)
    # Adam: three steps follow the oracle's updates
    x = rng.normal(0, 1, (64, 64)).astype(np.float32)
    t = rng.normal(0, 1, 64).astype(np.float32)
    pr, m, v = p.copy(), np.zeros_like(p), np.zeros_like(p)
    for step in range(1, 4):
        loss = np.zeros(1, dtype=np.float32)
        emu.check(L.smx_mlp_train_step(h, _pf(x), _pf(t), 64, ctypes.c_float(1e-3), _pf(loss)))
        gr, _ = ref.gradients(pr, x, t)
        pr, m, v = ref.adam(pr, gr, m, v, step, 1e-3)
    got = np.zeros(ref.N_PARAMS, dtype=np.float32)
    emu.check(L.smx_mlp_get_params(h, _pf(got), len(got)))
    assert rel(got - p, pr - p) < 5e-2
    # too large a batch is refused
    assert L.smx_mlp_forward(h, _pf(np.zeros((513, 64), np.float32)), 513, _pf(np.zeros(513, np.float32))) == 3


def test_emulated_order_features_and_beam(emu):
    g, _ = host_graph(300, 900, 2.5, 1, 5)
    off, nb, lab = g.csr()
    dg = emu.graph(off, nb, lab)
    q, _ = query_file(g, 6, True, 3)
    qo, qn, ql = q.csr()
    dq = emu.query(qo, qn, ql)
    c, ok = emu.filter(dg, dq, 1)
    assert ok
    n = 6
    out = np.zeros(16 * n, dtype=np.uint32)
    k = ctypes.c_uint32()
    emu.check(emu.L.smx_order_beam(dq, c, 16, 5, p32(out), ctypes.byref(k)))
    orders = [tuple(out[i * n:(i + 1) * n]) for i in range(k.value)]
    assert 2 <= len(orders) <= 16 and len(set(orders)) == len(orders)
    assert list(orders[0]) == emu.order_ri(dq, n)
    counts = set()
    for o in orders:
        oa = np.ascontiguousarray(o, dtype=np.uint32)
        assert emu.L.smx_order_valid(dq, p32(oa)) == 1
        f = np.zeros(64, dtype=np.float32)
        emu.check(emu.L.smx_order_features(dq, c, p32(oa), _pf(f)))
        assert np.isfinite(f).all() and f[0] == n / 32
        counts.add(emu.enumerate(dg, dq, c, list(o), explore=0).count)
    assert len(counts) == 1  # the order never changes the count
