"""Learned output-tree proposal: the network's forward/backward kernels against a float64 CPU
implementation, and the learned apply against the plain apply (identical trees and coefficients)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

WORLD = (-2, (-5, -5, -5), (10, 10, 10))


def cpu_forward(layers, x):
    acts = [x.astype(np.float64)]
    h = acts[0]
    for i, (W, b) in enumerate(layers):
        z = h @ W.astype(np.float64).T + b.astype(np.float64)
        h = np.maximum(z, 0.0) if i + 1 < len(layers) else z
        acts.append(h)
    return acts


def cpu_gradient(layers, x, y, w):
    acts = cpu_forward(layers, x)
    z = acts[-1][:, 0]
    n = len(x)
    loss = np.mean(w * (np.logaddexp(0.0, z) - y * z))
    dz = (w * (1.0 / (1.0 + np.exp(-z)) - y) / n)[:, None]
    grads = []
    d = dz
    for i in range(len(layers) - 1, -1, -1):
        W, b = layers[i]
        gW = d.T @ acts[i]
        gb = d.sum(axis=0)
        grads.append((gW, gb))
        if i > 0:
            d = (d @ W.astype(np.float64)) * (acts[i] > 0)
    flat = []
    for gW, gb in reversed(grads):
        flat += [gW.ravel(), gb.ravel()]
    return loss, np.concatenate(flat)


def test_network_forward_and_gradient_match_cpu(gpu_mod):
    G = gpu_mod
    net = G.ProposalNet(hidden_layers=3, width=128, seed=7)
    rng = np.random.default_rng(3)
    x = rng.normal(0.0, 1.0, (37, net.nfeatures)).astype(np.float32)
    y = (rng.uniform(size=37) < 0.3).astype(np.float32)
    w = rng.uniform(0.5, 2.0, 37).astype(np.float32)
    layers = net.layers()
    z_gpu = net.forward(x)
    z_cpu = cpu_forward(layers, x)[-1][:, 0]
    assert np.max(np.abs(z_gpu - z_cpu)) < 1e-4 * max(1.0, np.max(np.abs(z_cpu)))
    loss_gpu, g_gpu = net.gradient(x, y, w)
    loss_cpu, g_cpu = cpu_gradient(layers, x, y, w)
    assert abs(loss_gpu - loss_cpu) < 1e-5 * max(1.0, abs(loss_cpu))
    assert np.max(np.abs(g_gpu - g_cpu)) < 1e-4 * np.max(np.abs(g_cpu))


def _setup(G, m, seed, n, prec):
    from mrchem_b200 import workloads as W

    orbs = W.orbitals(n, seed=seed)
    mus = W.helmholtz_mus(n, seed=seed)
    inps, ops = [], []
    for f, mu in zip(orbs, mus):
        t = G.FunctionTree(m)
        G.project(prec, t, f)
        inps.append(t)
        ops.append(G.HelmholtzOperator(m, mu, prec))
    return inps, ops


def _assert_identical(a, b):
    ea, eb = a.export(), b.export()
    ka = {(int(d), *map(int, t)): i for i, (d, t) in enumerate(zip(ea["depth"], ea["trans"]))}
    kb = {(int(d), *map(int, t)): i for i, (d, t) in enumerate(zip(eb["depth"], eb["trans"]))}
    assert set(ka) == set(kb)
    for q in ka:
        assert np.array_equal(ea["coef"][ka[q]], eb["coef"][kb[q]])
        assert (ea["child0"][ka[q]] < 0) == (eb["child0"][kb[q]] < 0)


@pytest.mark.parametrize("flags", [0, 1])
def test_learned_apply_equals_plain_with_untrained_network(gpu_mod, flags):
    """Whatever the network proposes, the exact check restores the plain result."""
    G = gpu_mod
    prec = 1e-5
    m = G.MultiResolutionAnalysis(*WORLD, 7, 14)
    inps, ops = _setup(G, m, 21, 3, prec)
    plain = [G.FunctionTree(m) for _ in inps]
    G.apply_batched(prec, plain, ops, inps, flags)
    net = G.ProposalNet(seed=1)
    for tau in (0.5, 0.05):
        learned = [G.FunctionTree(m) for _ in inps]
        st = G.apply_learned(prec, learned, ops, inps, net, tau=tau, flags=flags)
        for a, b in zip(learned, plain):
            _assert_identical(a, b)
        assert st["out_nodes"] == sum(t.nnodes() for t in plain)


def test_trained_network_saves_passes(gpu_mod):
    """Trained on plain applies of one set of orbitals, the network proposes the trees of fresh
    orbitals: the result is unchanged and the apply needs fewer passes than the plain refinement."""
    G = gpu_mod
    prec = 1e-6
    m = G.MultiResolutionAnalysis(*WORLD, 9, 15)
    net = G.ProposalNet(seed=2)
    inps, ops = _setup(G, m, 31, 8, prec)
    outs = [G.FunctionTree(m) for _ in inps]
    G.apply_batched(prec, outs, ops, inps)
    for o, op, t in zip(outs, ops, inps):
        net.collect(o, op, t)
    n, npos = net.dataset()
    assert n > 1000 and 0 < npos < n
    loss = net.train(epochs=30, batch=2048, lr=2e-3, seed=0)
    assert loss < 0.5
    inps2, ops2 = _setup(G, m, 77, 6, prec)
    plain = [G.FunctionTree(m) for _ in inps2]
    G.apply_batched(prec, plain, ops2, inps2)
    plain_passes = max(G.apply_stats(t)[2] for t in plain)
    learned = [G.FunctionTree(m) for _ in inps2]
    st = G.apply_learned(prec, learned, ops2, inps2, net, tau=0.5)
    for a, b in zip(learned, plain):
        _assert_identical(a, b)
    total = st["out_nodes"]
    assert st["missed"] * 8 < 0.1 * total, st
    assert st["pruned"] < 0.2 * total, st
    assert st["passes"] < plain_passes, (st, plain_passes)


def test_network_of_another_context_rejected(gpu_mod):
    """Handles of different contexts (streams) are never mixed in one call."""
    G = gpu_mod
    prec = 1e-4
    m = G.MultiResolutionAnalysis(*WORLD, 5, 12)
    inps, ops = _setup(G, m, 3, 1, prec)
    other = G.ProposalNet(ctx=G.Context(0), hidden_layers=1, width=16, seed=1)
    with pytest.raises(G.MWError):
        G.apply_learned(prec, [G.FunctionTree(m)], ops, inps, other, tau=0.5)
