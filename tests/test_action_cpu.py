"""The float64 torch restatement of the action used by the adjoint tests,
checked on the CPU against the FP64 oracle (value and autograd gradient)."""
import numpy as np
import pytest
import torch

from oracle.oracle import Oracle
from tests.torch_ref import plaquette_tables, torch_action

CASES = [(4, (4, 6, 4, 8), 1.3, 1.0), (4, (4, 4, 6, 4), 0.9, 1.7), (3, (6, 4, 0, 8), 1.1, 0.8),
         (2, (8, 0, 0, 6), 2.0, 1.0)]


@pytest.mark.parametrize("case", CASES)
def test_torch_reference_matches_oracle(case):
    dims, N, beta, aniso = case
    o = Oracle(dims, N, beta, aniso)
    th = np.random.default_rng(3).uniform(0, 2 * np.pi, o.nlinks)
    s_o, g_o = o.action(th, grad=True)
    t = torch.tensor(th[None, :], dtype=torch.float64, requires_grad=True)
    s = torch_action(t, plaquette_tables(dims, o.grid), beta, aniso)
    s.sum().backward()
    assert abs(float(s[0].detach()) - s_o) <= 1e-11 * abs(s_o)
    assert np.abs(t.grad[0].numpy() - g_o).max() <= 1e-11


def test_oracle_charge_is_integer():
    o = Oracle(2, (8, 0, 0, 8), 2.0)
    for seed in range(4):
        th = np.random.default_rng(seed).uniform(0, 2 * np.pi, o.nlinks)
        q = o.topological_charge_2d(th)
        assert abs(q - round(q)) < 1e-9
