"""Host-side pieces of the 2D flow sampler (no GPU): the natural<->even/odd
permutation, the coupling-layer masks, the independence MH chain and the
Gamma-method autocorrelation time."""
import math

import numpy as np
import pytest

from latticeu1_b200.flow import Coupling, eo_permutation, independence_mh, tau_int
from tests.torch_ref import link_index


def test_eo_permutation_matches_reference_index():
    L0, L1 = 8, 6
    perm = eo_permutation(L0, L1)
    V = L0 * L1
    lex = np.arange(V)
    X = np.stack([lex % L0, lex // L0, np.zeros(V, int), np.zeros(V, int)])
    for mu in range(2):
        eo = link_index((L0, L1, 1, 1), X, mu)
        assert np.array_equal(perm[eo], mu * V + lex)
    assert np.array_equal(np.sort(perm), np.arange(2 * V))


@pytest.mark.parametrize("layer", range(8))
def test_coupling_masks(layer):
    L = 8
    c = Coupling(L, layer % 2, (layer // 2) % 4, K=2, hidden=4)
    upd = np.zeros(2 * L * L, bool)
    upd[c.mu * L * L + c.link_idx.numpy()] = True
    frozen = c.frozen.numpy()[0, 0].reshape(-1)
    act = np.zeros(L * L, bool)
    act[c.act_idx.numpy()] = True
    for x1 in range(L):
        for x0 in range(L):
            links = [(0, x1, x0, 1), (1, x1, (x0 + 1) % L, 1), (0, (x1 + 1) % L, x0, -1), (1, x1, x0, -1)]
            hit = [(s, upd[m * L * L + a * L + b]) for m, a, b, s in links]
            n = sum(h for _, h in hit)
            p = x1 * L + x0
            if frozen[p]:
                assert n == 0
            if act[p]:
                assert n == 1 and [s for s, h in hit if h] == [1]
            assert n <= 1


def test_tau_int_ar1():
    rng = np.random.default_rng(0)
    phi, N = 0.8, 200000
    x = np.empty(N)
    x[0] = 0.0
    e = rng.normal(size=N)
    for i in range(1, N):
        x[i] = phi * x[i - 1] + e[i]
    t, dt, W = tau_int(x)
    exact = 0.5 * (1 + phi) / (1 - phi)
    assert abs(t - exact) < 4 * dt + 0.1
    assert W > 0


def test_independence_mh():
    rng = np.random.default_rng(1)
    logw = np.zeros(1000)
    idx, acc = independence_mh(logw, rng.uniform(size=1000))
    assert acc == 1.0 and np.array_equal(idx, np.arange(1000))
    logw = np.array([0.0, -math.inf] * 50)
    idx, acc = independence_mh(logw, rng.uniform(size=100))
    assert np.all(idx[1::2] == idx[0::2])
