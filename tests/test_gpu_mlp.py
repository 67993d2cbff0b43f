"""The learned-order cost model on a B200 (marked gpu): the CUDA forward /
backward / Adam kernels against the numpy restatement (oracle/mlp.py), and
the learned order end to end on the 1M-vertex graph — it never changes a
count, and after training its predictions rank held-out orders by their
measured enumeration time."""
from __future__ import annotations

import numpy as np
import pytest

import subgraphmatching_b200 as smx
from subgraphmatching_b200 import learned_order as lo
from helpers import host_graph
from oracle import mlp as ref

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a, dtype=np.float64) - b) / max(np.linalg.norm(b), 1e-12))


def test_mlp_kernels_match_oracle(gpu):
    m = smx.MLP(0, 2048, seed=11)
    p = m.params
    rng = np.random.default_rng(5)
    for n in (1, 255, 2048):
        x = rng.normal(0, 1, (n, 64)).astype(np.float32)
        t = rng.normal(0, 1, n).astype(np.float32)
        assert rel(m.forward(x), ref.forward(p, x)[3]) < 1e-2   # bf16 activations: summation order only
        g, loss = m.gradients(x, t)
        gr, lr_ = ref.gradients(p, x, t)
        assert rel(g, gr) < 2e-2
        assert abs(loss - lr_) <= 1e-3 * max(1.0, lr_)
    x = rng.normal(0, 1, (512, 64)).astype(np.float32)
    t = rng.normal(0, 1, 512).astype(np.float32)
    pr, mo, vo = p.copy(), np.zeros_like(p), np.zeros_like(p)
    for step in range(1, 6):
        m.train_step(x, t, 1e-3)
        gr, _ = ref.gradients(pr, x, t)
        pr, mo, vo = ref.adam(pr, gr, mo, vo, step, 1e-3)
    assert rel(m.params - p, pr - p) < 5e-2


def test_mlp_fits_a_smooth_target(gpu):
    rng = np.random.default_rng(6)
    x = rng.uniform(0, 1, (4096, 64)).astype(np.float32)
    t = (np.sin(3 * x[:, 0]) + x[:, 1] * x[:, 2] + 0.5 * x[:, 3]).astype(np.float32)
    m = smx.MLP(0, 4096, seed=1)
    first = m.gradients(x, t)[1]
    for _ in range(300):
        idx = rng.integers(0, len(x), 256)
        m.train_step(x[idx], t[idx], 2e-3)
    assert m.gradients(x, t)[1] < first / 10


def test_learned_order_keeps_counts_and_ranks_orders(gpu):
    hg, _ = host_graph(1_000_000, 10_000_000, 2.2, 1, 2)
    off, nb, lab = hg.csr()
    dg = smx.Graph.from_csr(off, nb, lab, device=0)
    qs = [smx.Query.generate(hg, 8 if i % 3 else 10, i % 2 == 0, 50_000 + i) for i in range(48)]
    train_s = lo.collect(dg, qs[:36], beam=8, cap=5_000_000, budget_ms=300)
    test_s = lo.collect(dg, qs[36:], beam=8, cap=5_000_000, budget_ms=300, seed=999)
    m = smx.MLP(0, 1024, seed=3)
    losses = lo.train(m, train_s, epochs=60, batch=128, lr=2e-3)
    assert losses[-1] < losses[0]
    pred = m.forward(test_s.x)
    assert lo.rank_correlation(pred, test_s.t) > 0.2
    ev = lo.evaluate(dg, qs[36:], m, beam=8, cap=5_000_000)   # raises if any counts differ
    print("held-out total ms: RI %.1f GQL %.1f learned %.1f" % (ev["ri_total_ms"], ev["gql_total_ms"],
                                                               ev["learned_total_ms"]))
