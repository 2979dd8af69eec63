"""GPU tests of learned truncation: the tensor-core network against the FP64 CPU reference
(oracle/mlp_ref.py), its training, and term-budget truncation against a host selection."""

import numpy as np
import pytest

from oracle import mlp_ref as M
from ppvm_b200 import circuits as C
from ppvm_b200.learned import TermPriorityNet, split_layers
from ppvm_b200.paulisum import PauliSum

pytestmark = pytest.mark.gpu


def rand_net(seed):
    rng = np.random.default_rng(seed)
    net = TermPriorityNet(seed=seed)
    p = M.unpack(rng.normal(0, 1, M.N_PARAMS))
    p["W1"] *= 0.35
    p["W2"] *= 0.125
    p["w3"] *= 0.125
    p["b1"] *= 0.1
    p["b2"] *= 0.1
    net.params = M.pack(p).astype(np.float32)
    return net, rng


def test_forward_matches_reference():
    net, rng = rand_net(1)
    X = rng.normal(0, 1, (1000, 8)).astype(np.float32)
    y = net.predict(X)
    want, _ = M.forward(net.params.astype(np.float64), X, tc=True)
    assert np.max(np.abs(y - want) / (1 + np.abs(want))) < 1e-2
    exact, _ = M.forward(net.params.astype(np.float64), X, tc=False)
    assert np.max(np.abs(y - exact) / (1 + np.abs(exact))) < 5e-2


def test_gradient_matches_reference():
    net, rng = rand_net(2)
    X = rng.normal(0, 1, (2000, 8)).astype(np.float32)
    t = rng.normal(0, 1, 2000).astype(np.float32)
    g, loss = net.grad(X, t)
    want_loss, want = M.loss_and_grad(net.params.astype(np.float64), X, t, tc=True)
    assert abs(loss - want_loss) < 1e-2 * (1 + want_loss)
    rel = np.linalg.norm(g - want) / np.linalg.norm(want)
    cos = float(g @ want / (np.linalg.norm(g) * np.linalg.norm(want)))
    assert rel < 5e-2 and cos > 0.998, (rel, cos)
    for name, sl in (("W1", slice(0, 512)), ("W2", slice(576, 4672)), ("w3", slice(4736, 4800))):
        r = np.linalg.norm(g[sl] - want[sl]) / np.linalg.norm(want[sl])
        assert r < 6e-2, (name, r)


def test_training_fits_a_smooth_target():
    net, rng = rand_net(3)
    X = rng.uniform(-1, 1, (20000, 8)).astype(np.float32)
    t = (np.sin(2 * X[:, 0]) + X[:, 1] * X[:, 2] - 0.5 * X[:, 3] ** 2).astype(np.float32)
    before = float(np.mean((net.predict(X) - t) ** 2))
    net.train(X, t, epochs=30, batch=512, lr=3e-3, seed=1)
    after = float(np.mean((net.predict(X) - t) ** 2))
    assert after < 0.05 * before and after < 0.02, (before, after)


def test_training_is_deterministic():
    """Same data, seed and start: bit-identical gradients and trained parameters (no float
    atomics: per-warp copies, per-block slabs, fixed-order sums)."""
    rng = np.random.default_rng(6)
    X = rng.normal(0, 1, (3000, 8)).astype(np.float32)
    t = rng.normal(0, 1, 3000).astype(np.float32)
    runs = []
    for _ in range(2):
        net, _ = rand_net(5)
        g, loss = net.grad(X, t)
        net.train(X, t, epochs=3, batch=256, lr=1e-3, seed=9)
        runs.append((g, loss, net.params))
    assert np.array_equal(runs[0][0], runs[1][0]) and runs[0][1] == runs[1][1]
    assert np.array_equal(runs[0][2], runs[1][2])


def test_adam_step_and_repacked_weights():
    """One full-batch step: Adam's first update is -lr * sign(g) (bias-corrected moments), and
    the packed tensor-core weights follow the updated FP32 parameters."""
    net, rng = rand_net(4)
    X = rng.normal(0, 1, (1024, 8)).astype(np.float32)
    t = rng.normal(0, 1, 1024).astype(np.float32)
    p0 = net.params.astype(np.float64)
    g, _ = net.grad(X, t)
    lr = 1e-3
    net.train(X, t, epochs=1, batch=len(t), lr=lr, seed=0)
    p1 = net.params.astype(np.float64)
    big = np.abs(g) > 1e-3  # eps = 1e-8 is negligible against sqrt(v) = 0.0316 |g|
    assert big.sum() > 0.5 * len(g)
    np.testing.assert_allclose(p1[big] - p0[big], -lr * np.sign(g[big]), rtol=1e-3, atol=1e-8)
    y = net.predict(X)
    want, _ = M.forward(p1, X, tc=True)
    assert np.max(np.abs(y - want) / (1 + np.abs(want))) < 1e-2


def _sum_after(L=5, layers=3):
    wl = C.kicked_ising_random_h(L=L, layers=layers, seed=5, thr=1e-7, obs=(L // 2, L // 2))
    s = PauliSum([wl.observable[0][0]], wl.n_qubits, [1.0], min_abs_coeff=1e-7, clifford_angles=True)
    for part in split_layers(wl.ops)[:layers]:
        s.run(part)
    return s


def _expected_kept(keys, B):
    order = np.lexsort((np.arange(len(keys)), -keys.astype(np.int64)))  # by key desc, then index
    return np.sort(order[:B])


@pytest.mark.parametrize("bits", [8, 11])
def test_budget_truncation_plain_keeps_the_top_by_magnitude(bits):
    s = _sum_after()
    terms = s.terms
    n = len(terms)
    assert n > 3000
    c = np.array([abs(v) for _, v in terms])
    keys = (c.view(np.uint64) >> np.uint64(32)).astype(np.uint64)
    for B in (n // 3, 1000, 1):
        t = _sum_after()
        t.truncate_budget(B, digit_bits=bits)
        kept = _expected_kept(keys, B)
        assert t.terms == [terms[i] for i in kept]


def test_budget_truncation_learned_keeps_the_top_scores():
    net, _ = rand_net(4)
    s = _sum_after()
    terms = s.terms
    f = s.features(5, 2)
    score = net.predict(f)
    u = score.view(np.uint32).astype(np.uint64)
    keys = np.where(u & 0x80000000, (~u) & 0xFFFFFFFF, u | 0x80000000)
    B = len(terms) // 4
    s.truncate_budget(B, net, 5, 2)
    assert s.terms == [terms[i] for i in _expected_kept(keys, B)]
    s.truncate_budget(10 ** 9, net, 5, 2)  # larger than the sum: nothing changes
    assert len(s) == B


def test_trained_network_beats_plain_budget_truncation():
    """What the trained network gains: at matched term budgets the learned priority gives a
    smaller <O> error than |c| on a circuit the network never saw (10x10, seeded angles;
    trained on 6x6 circuits with other angles).  The budgets bind between layers 2 and 3."""
    from ppvm_b200 import learned

    X, y = learned.make_training_set(L=6, layers=4, seeds=(11, 12, 13, 14, 15, 16, 17, 18), per_layer=2048,
                                     label_thr=1e-5)
    net = TermPriorityNet(seed=7)
    net.train(X, y, epochs=300, batch=512, lr=2e-3, seed=3)
    wl = C.kicked_ising_random_h(L=10, layers=4, seed=2, thr=1e-7)
    ref, _ = learned.run_with_budget(wl, None)
    errs = {"plain": [], "learned": []}
    for B in (2000, 4000, 8000):
        for kind, nn in (("plain", None), ("learned", net)):
            v, _ = learned.run_with_budget(wl, B, nn, 10)
            errs[kind].append(max(abs(v - ref), 1e-12))
    gp = float(np.exp(np.mean(np.log(errs["plain"]))))
    gl = float(np.exp(np.mean(np.log(errs["learned"]))))
    print("geometric-mean |err|: plain", gp, "learned", gl, errs)
    assert gl < 0.5 * gp, (gl, gp, errs)
