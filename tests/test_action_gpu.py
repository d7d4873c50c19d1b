"""GPU parity of the Wilson action and its hand-written adjoint.

* FP64: action and gradient equal the FP64 oracle and the float64 torch
  restatement (autograd) to 1e-12 relative; the gradient equals FP64 central
  differences of the GPU action (h = 1e-6) to 2e-5 absolute on sampled links;
* FP32: action within 2e-6 relative, gradient within 5e-5 absolute of FP64;
* batched calls equal per-configuration calls bit for bit, and backward
  scales each configuration's gradient by its grad_output;
* 2D topological charge: integer to 1e-9 (FP64) and equal to the oracle.
"""
import numpy as np
import pytest
import torch

from latticeu1_b200.action import WilsonAction
from oracle.oracle import Oracle
from tests.torch_ref import plaquette_tables, torch_action

pytestmark = pytest.mark.gpu

CASES = [(4, (8, 8, 8, 8), 1.0, 1.0), (4, (8, 6, 4, 8), 0.9, 1.7), (3, (8, 8, 0, 12), 1.4, 0.8),
         (2, (32, 0, 0, 32), 2.0, 1.0), (2, (16, 0, 0, 16), 6.0, 1.0)]
IDS = [f"{c[0]}d-{'x'.join(map(str, c[1]))}-b{c[2]}-xi{c[3]}" for c in CASES]


def _theta(o, seed, B=1):
    return np.random.default_rng(seed).uniform(0, 2 * np.pi, (B, o.nlinks))


@pytest.mark.parametrize("case", CASES, ids=IDS)
def test_fp64_matches_oracle_and_torch(case):
    dims, N, beta, aniso = case
    o = Oracle(dims, N, beta, aniso)
    th = _theta(o, 11)
    S = WilsonAction(dims, N, beta, aniso)
    t = torch.tensor(th, dtype=torch.float64, device="cuda", requires_grad=True)
    s = S(t)
    s.sum().backward()
    s = s.detach()
    s_o, g_o = o.action(th[0], grad=True)
    assert abs(float(s[0]) - s_o) <= 1e-12 * abs(s_o)
    g = t.grad[0].cpu().numpy()
    assert np.abs(g - g_o).max() <= 1e-12 * max(1.0, np.abs(g_o).max())
    tr = torch.tensor(th, dtype=torch.float64, requires_grad=True)
    sr = torch_action(tr, plaquette_tables(dims, o.grid), beta, aniso)
    sr.sum().backward()
    assert abs(float(s[0]) - float(sr[0].detach())) <= 1e-12 * abs(s_o)
    assert np.abs(g - tr.grad[0].numpy()).max() <= 1e-12 * max(1.0, np.abs(g_o).max())


@pytest.mark.parametrize("case", [CASES[0], CASES[3]], ids=[IDS[0], IDS[3]])
def test_adjoint_vs_central_differences(case):
    dims, N, beta, aniso = case
    o = Oracle(dims, N, beta, aniso)
    th = torch.tensor(_theta(o, 5), dtype=torch.float64, device="cuda")
    S = WilsonAction(dims, N, beta, aniso)
    t = th.clone().requires_grad_(True)
    S(t).sum().backward()
    g = t.grad[0]
    h = 1e-6
    links = np.random.default_rng(9).choice(o.nlinks, 64, replace=False)
    # all perturbed configurations in one batched call
    pert = th.repeat(2 * len(links), 1)
    for j, l in enumerate(links):
        pert[2 * j, l] += h
        pert[2 * j + 1, l] -= h
    with torch.no_grad():
        vals = S(pert).cpu().numpy()
    fd = (vals[0::2] - vals[1::2]) / (2 * h)
    assert np.abs(fd - g[links].cpu().numpy()).max() <= 2e-5


@pytest.mark.parametrize("case", CASES, ids=IDS)
def test_fp32_close_to_fp64(case):
    dims, N, beta, aniso = case
    o = Oracle(dims, N, beta, aniso)
    th = _theta(o, 21)
    S = WilsonAction(dims, N, beta, aniso)
    t32 = torch.tensor(th, dtype=torch.float32, device="cuda", requires_grad=True)
    s32 = S(t32)
    s32.sum().backward()
    s32 = s32.detach()
    assert t32.grad.dtype == torch.float32
    s_o, g_o = o.action(th[0], grad=True)
    assert abs(float(s32[0]) - s_o) <= 2e-6 * abs(s_o)
    assert np.abs(t32.grad[0].cpu().numpy().astype(np.float64) - g_o).max() <= 5e-5 * max(1.0, beta * aniso)


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_batched_equals_single_and_scales(dtype):
    dims, N, beta, aniso = CASES[1]
    o = Oracle(dims, N, beta, aniso)
    th = torch.tensor(_theta(o, 2, B=3), dtype=dtype, device="cuda")
    S = WilsonAction(dims, N, beta, aniso)
    tb = th.clone().requires_grad_(True)
    sb = S(tb)
    w = torch.tensor([0.5, -2.0, 3.0], dtype=torch.float64, device="cuda")
    (sb * w).sum().backward()
    for b in range(3):
        t1 = th[b].clone().requires_grad_(True)
        s1 = S(t1)
        s1.backward()
        assert float(s1.detach()) == float(sb[b].detach())
        ref = (t1.grad * w[b].to(dtype))
        assert torch.allclose(tb.grad[b], ref, rtol=1e-6 if dtype == torch.float32 else 1e-14, atol=0)


def test_charge_2d():
    o = Oracle(2, (16, 0, 0, 16), 2.0)
    th = _theta(o, 4, B=8)
    S = WilsonAction(2, (16, 0, 0, 16), 2.0)
    q = S.charge(torch.tensor(th, dtype=torch.float64, device="cuda")).cpu().numpy()
    for b in range(8):
        assert abs(q[b] - round(q[b])) < 1e-9
        assert abs(q[b] - o.topological_charge_2d(th[b])) < 1e-9


def test_argument_errors():
    S = WilsonAction(4, (4, 4, 4, 4), 1.0)
    with pytest.raises(TypeError):
        S(torch.zeros(S.nlinks, dtype=torch.float16, device="cuda"))
    with pytest.raises(ValueError):
        S(torch.zeros(S.nlinks, dtype=torch.float64))
    with pytest.raises(ValueError):
        S(torch.zeros(S.nlinks + 1, dtype=torch.float64, device="cuda"))
