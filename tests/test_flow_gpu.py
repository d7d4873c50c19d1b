"""GPU checks of the flow kernels and the 2D flow sampler.

* the circular coupling transform (forward, inverse) equals a float64 torch
  restatement of the mixture of non-compact projections (1e-5), its backward
  passes equal torch autograd of that restatement (inverse: through Newton
  steps from the kernel's solution, i.e. the implicit derivative);
* a coupling layer's log-det equals log|det J| of its Jacobian computed by
  autograd through the library kernels; layers are gauge-equivariant;
* the flow inverts (log_prob(sample) = log q of the sample), and a short
  reverse-KL run lowers the loss.
"""
import math

import numpy as np
import pytest
import torch

from latticeu1_b200.flow import Coupling, Flow2D, ncp_forward, ncp_inverse, plaquettes_no

pytestmark = pytest.mark.gpu

TWO_PI = 2 * math.pi


def ref_H(xc, p, K):
    """float64 mixture value and derivative, xc in [-pi, pi]."""
    a = torch.clamp(p[:, :K], -8, 8)
    al = torch.exp(a)
    w = torch.softmax(p[:, K:2 * K], dim=1)
    s, c = torch.sin(xc / 2)[:, None], torch.cos(xc / 2)[:, None]
    g = 2 * torch.atan2(al * s, c)
    gp = al / (c * c + al * al * s * s)
    return (w * g).sum(1), (w * gp).sum(1)


def _inputs(n, K, seed=0, scale=1.0):
    g = torch.Generator(device="cuda").manual_seed(seed)
    x = (torch.rand(n, device="cuda", generator=g) * 4 - 2) * math.pi
    p = torch.randn(n, 2 * K + 1, device="cuda", generator=g) * scale
    return x, p


@pytest.mark.parametrize("K", [1, 4, 6, 8])
def test_ncp_forward_and_backward(K):
    x, p = _inputs(4096, K, seed=K)
    x.requires_grad_(True)
    p.requires_grad_(True)
    dy, logd = ncp_forward(x, p, K)
    gdy = torch.randn_like(dy)
    gl = torch.randn_like(logd)
    (dy * gdy + logd * gl).sum().backward()
    x64 = x.detach().double().requires_grad_(True)
    p64 = p.detach().double().requires_grad_(True)
    xc = torch.remainder(x64 + math.pi, TWO_PI) - math.pi
    H, Hp = ref_H(xc, p64, K)
    dy_r = H + p64[:, 2 * K] - xc
    logd_r = torch.log(Hp)
    assert (dy.double() - dy_r).abs().max() < 2e-5
    assert (logd.double() - logd_r).abs().max() < 2e-5
    (dy_r * gdy.double() + logd_r * gl.double()).sum().backward()
    assert torch.allclose(x.grad.double(), x64.grad, atol=2e-4, rtol=1e-3)
    assert torch.allclose(p.grad.double(), p64.grad, atol=2e-4, rtol=1e-3)


@pytest.mark.parametrize("K", [2, 6])
def test_ncp_inverse_and_backward(K):
    y, p = _inputs(4096, K, seed=10 + K)
    y.requires_grad_(True)
    p.requires_grad_(True)
    dx, logd = ncp_inverse(y, p, K)
    # round trip: the forward map at the solution reproduces y (mod 2 pi)
    z = torch.remainder(y.detach() - p.detach()[:, 2 * K] + math.pi, TWO_PI) - math.pi
    xs = (dx.detach() + z + p.detach()[:, 2 * K])
    H, Hp = ref_H(xs.double(), p.detach().double(), K)
    err = torch.remainder(H + p.detach().double()[:, 2 * K] - y.detach().double() + math.pi, TWO_PI) - math.pi
    assert err.abs().max() < 5e-5
    assert (logd.double() - torch.log(Hp)).abs().max() < 5e-5
    gdx = torch.randn_like(dx)
    gl = torch.randn_like(logd)
    (dx * gdx + logd * gl).sum().backward()
    # float64 reference: Newton steps from the solution carry the implicit derivative
    y64 = y.detach().double().requires_grad_(True)
    p64 = p.detach().double().requires_grad_(True)
    z64 = torch.remainder(y64 - p64[:, 2 * K] + math.pi, TWO_PI) - math.pi
    xk = xs.double().detach()
    for _ in range(3):
        Hk, Hpk = ref_H(xk, p64, K)
        xk = xk - (Hk - z64) / Hpk
    dx_r = xk - z64 - p64[:, 2 * K]
    logd_r = torch.log(ref_H(xk, p64, K)[1])
    (dx_r * gdx.double() + logd_r * gl.double()).sum().backward()
    assert torch.allclose(y.grad.double(), y64.grad, atol=5e-4, rtol=2e-3)
    assert torch.allclose(p.grad.double(), p64.grad, atol=5e-4, rtol=2e-3)


def _random_layer(L, layer, K=4, seed=0):
    torch.manual_seed(seed)
    c = Coupling(L, layer % 2, (layer // 2) % 4, K=K, hidden=8).cuda()
    with torch.no_grad():
        for m in c.net:
            if isinstance(m, torch.nn.Conv2d):
                m.weight.normal_(0, 0.3)
                m.bias.normal_(0, 0.3)
    return c


@pytest.mark.parametrize("layer", [0, 1, 2, 7])
def test_coupling_logdet_is_log_abs_det_jacobian(layer):
    L = 4
    c = _random_layer(L, layer, seed=layer)
    th = (torch.rand(1, 2, L, L, device="cuda") * TWO_PI)
    out, ld = c(th)

    def f(v):
        return c(v.reshape(1, 2, L, L))[0].reshape(-1)

    J = torch.autograd.functional.jacobian(f, th.reshape(-1))
    sign, logabs = torch.linalg.slogdet(J.double())
    assert sign.item() > 0
    assert abs(logabs.item() - ld.item()) < 2e-3


@pytest.mark.parametrize("layer", [0, 3])
def test_coupling_gauge_equivariance(layer):
    L = 8
    c = _random_layer(L, layer, seed=5)
    th = torch.rand(3, 2, L, L, device="cuda") * TWO_PI
    alpha = torch.rand(3, L, L, device="cuda") * TWO_PI
    g = torch.stack([alpha - torch.roll(alpha, -1, dims=-1), alpha - torch.roll(alpha, -1, dims=-2)], 1)
    out, ld = c(th)
    out_g, ld_g = c(th + g)
    d = torch.remainder(out_g - (out + g) + math.pi, TWO_PI) - math.pi
    assert d.abs().max() < 1e-4
    assert (ld - ld_g).abs().max() < 1e-3
    assert (torch.remainder(plaquettes_no(th + g) - plaquettes_no(th) + math.pi, TWO_PI) - math.pi).abs().max() < 1e-5


def test_flow_inverts_and_trains():
    torch.manual_seed(0)
    flow = Flow2D(8, beta=2.0, n_layers=8, K=4, hidden=16).cuda()
    with torch.no_grad():
        for layer in flow.layers:
            layer.net[2].weight.normal_(0, 0.05)
    th, logq = flow.sample(64)
    lq2 = flow.log_prob(th)
    assert (lq2 - logq).abs().max() < 5e-3
    opt = torch.optim.Adam(flow.parameters(), lr=2e-3)
    first = [flow.reverse_kl_step(opt, 256)["loss"] for _ in range(5)]
    for _ in range(120):
        last = flow.reverse_kl_step(opt, 256)
    assert last["loss"] < np.mean(first) - 1.0


def _layer_ref_fp32(c, th):
    """The coupling layer in plain torch FP32 with bf16-rounded weights (the
    fused kernel's arithmetic; the rounding passes gradients straight
    through): returns (theta', logdet)."""
    import torch.nn.functional as Fn
    from latticeu1_b200.flow import ncp_forward, plaquettes_no
    r = lambda t: t + (t.detach().to(torch.bfloat16).float() - t.detach())
    torch.backends.cudnn.allow_tf32 = False  # plain FP32 convolutions for the reference
    B = th.shape[0]
    P = plaquettes_no(th)
    ctx = torch.stack([torch.cos(P), torch.sin(P)], 1) * c.frozen
    h = Fn.conv2d(Fn.pad(ctx, (1, 1, 1, 1), mode="circular"), r(c.net[0].weight), r(c.net[0].bias))
    h = Fn.leaky_relu(h, c.net[1].negative_slope)
    prm = Fn.conv2d(Fn.pad(h, (1, 1, 1, 1), mode="circular"), r(c.net[2].weight), r(c.net[2].bias))
    prm = prm.reshape(B, 2 * c.K + 1, -1)[:, :, c.act_idx].permute(0, 2, 1).reshape(-1, 2 * c.K + 1)
    Pa = P.reshape(B, -1)[:, c.act_idx].reshape(-1)
    dy, logd = ncp_forward(Pa, prm, c.K)
    return c._apply_delta(th, dy), logd.reshape(B, -1).sum(1)


@pytest.mark.parametrize("L,layer", [(8, 0), (8, 1), (16, 2), (16, 5), (32, 7)])
def test_fused_layer_forward_matches_torch(L, layer):
    import ctypes as C
    from latticeu1_b200._lib import check, lib
    torch.manual_seed(layer)
    c = Coupling(L, layer % 2, (layer // 2) % 4, K=6, hidden=32).cuda()
    with torch.no_grad():
        for m in c.net:
            if isinstance(m, torch.nn.Conv2d):
                m.weight.normal_(0, 0.2)
                m.bias.normal_(0, 0.2)
    B = 16
    th = torch.rand(B, 2, L, L, device="cuda") * TWO_PI
    want, want_ld = _layer_ref_fp32(c, th)
    out = torch.empty_like(th)
    ld = torch.empty(B, device="cuda")
    p = lambda t: C.c_void_p(t.data_ptr())
    check(lib.u1_flow_layer_forward(p(th), p(out), p(ld), B, L, c.mu, c.off, c.K, 32, p(c.net[0].weight),
                                    p(c.net[0].bias), p(c.net[2].weight), p(c.net[2].bias),
                                    C.c_float(c.net[1].negative_slope), None), "u1_flow_layer_forward")
    torch.cuda.synchronize()
    d = torch.remainder(out - want + math.pi, TWO_PI) - math.pi
    assert d.abs().max().item() < 2e-4
    assert (ld - want_ld).abs().max().item() < 2e-3


def test_fused_sampler_consistent_with_inverse():
    """Proposals from the fused layers carry log q consistent with the inverse flow."""
    torch.manual_seed(1)
    flow = Flow2D(8, beta=2.0, n_layers=8, K=4, hidden=16).cuda()
    with torch.no_grad():
        for layer in flow.layers:
            layer.net[2].weight.normal_(0, 0.05)
            layer.net[2].weight.copy_(layer.net[2].weight.to(torch.bfloat16).float())
            layer.net[2].bias.copy_(layer.net[2].bias.to(torch.bfloat16).float())
            layer.net[0].weight.copy_(layer.net[0].weight.to(torch.bfloat16).float())
            layer.net[0].bias.copy_(layer.net[0].bias.to(torch.bfloat16).float())
    th, logq = flow.sample_fused(64)
    assert torch.isfinite(logq).all()
    # the torch inverse runs its convolutions in bf16 (autocast), so agreement is to bf16 level
    lq2 = flow.log_prob(th)
    assert (lq2 - logq).abs().max().item() < 0.5


def _layer_ref_fp32_inverse(c, th):
    """The inverse coupling layer in plain torch FP32 with bf16-rounded
    weights and the library's elementwise inverse transform (its analytic
    backward is checked against float64 in test_ncp_inverse_and_backward)."""
    import torch.nn.functional as Fn
    from latticeu1_b200.flow import ncp_inverse, plaquettes_no
    r = lambda t: t + (t.detach().to(torch.bfloat16).float() - t.detach())
    torch.backends.cudnn.allow_tf32 = False
    B = th.shape[0]
    P = plaquettes_no(th)
    ctx = torch.stack([torch.cos(P), torch.sin(P)], 1) * c.frozen
    h = Fn.conv2d(Fn.pad(ctx, (1, 1, 1, 1), mode="circular"), r(c.net[0].weight), r(c.net[0].bias))
    h = Fn.leaky_relu(h, c.net[1].negative_slope)
    prm = Fn.conv2d(Fn.pad(h, (1, 1, 1, 1), mode="circular"), r(c.net[2].weight), r(c.net[2].bias))
    prm = prm.reshape(B, 2 * c.K + 1, -1)[:, :, c.act_idx].permute(0, 2, 1).reshape(-1, 2 * c.K + 1)
    Pa = P.reshape(B, -1)[:, c.act_idx].reshape(-1)
    dx, logd = ncp_inverse(Pa, prm, c.K)
    return c._apply_delta(th, dx), logd.reshape(B, -1).sum(1)


def _random_coupling(L, layer, seed):
    torch.manual_seed(seed)
    c = Coupling(L, layer % 2, (layer // 2) % 4, K=6, hidden=32).cuda()
    with torch.no_grad():
        for m in c.net:
            if isinstance(m, torch.nn.Conv2d):
                m.weight.normal_(0, 0.2)
                m.bias.normal_(0, 0.2)
    return c


@pytest.mark.parametrize("L,layer", [(8, 1), (16, 6), (32, 3)])
def test_fused_inverse_layer(L, layer):
    """u1_flow_layer_inverse undoes u1_flow_layer_forward, returns the same
    log-det, and equals the torch inverse layer (FP32, bf16-rounded weights)."""
    c = _random_coupling(L, layer, 30 + layer)
    th = torch.rand(16, 2, L, L, device="cuda") * TWO_PI
    with torch.no_grad():
        fw, ld_f = c.forward_fused(th)
        back, ld_i = c.inverse_fused(fw)
        want, want_ld = _layer_ref_fp32_inverse(c, fw)
    d = torch.remainder(back - th + math.pi, TWO_PI) - math.pi
    assert d.abs().max().item() < 5e-4
    assert (ld_i - ld_f).abs().max().item() < 5e-3
    d = torch.remainder(back - want + math.pi, TWO_PI) - math.pi
    assert d.abs().max().item() < 2e-4
    assert (ld_i - want_ld).abs().max().item() < 2e-3


@pytest.mark.parametrize("L,layer", [(8, 2), (32, 5)])
def test_fused_inverse_backward_matches_autograd(L, layer):
    """Gradients of the fused inverse layer equal torch autograd through the
    FP32 inverse reference layer."""
    c = _random_coupling(L, layer, 40 + layer)
    B = 8
    th0 = torch.rand(B, 2, L, L, device="cuda") * TWO_PI
    R = torch.randn(B, 2, L, L, device="cuda")
    r = torch.randn(B, device="cuda")

    def run(fn):
        c.zero_grad(set_to_none=True)
        th = th0.clone().requires_grad_(True)
        out, ld = fn(th)
        ((out * R).sum() + (ld * r).sum()).backward()
        return th.grad.clone(), [p.grad.clone() for p in c.parameters()]

    g_f, w_f = run(c.inverse_fused)
    g_r, w_r = run(lambda t: _layer_ref_fp32_inverse(c, t))
    assert torch.allclose(g_f, g_r, atol=3e-3, rtol=3e-3)
    for a, b in zip(w_f, w_r):
        assert torch.allclose(a, b, atol=5e-3 * max(1.0, b.abs().max().item()), rtol=3e-3)


@pytest.mark.parametrize("L,layer", [(8, 0), (8, 3), (16, 4), (16, 7), (32, 1), (32, 6)])
def test_fused_layer_backward_matches_autograd(L, layer):
    """Gradients of the fused layer (theta and all weights) equal torch autograd
    through the FP32 reference layer with the same bf16-rounded weights."""
    torch.manual_seed(10 + layer)
    c = Coupling(L, layer % 2, (layer // 2) % 4, K=6, hidden=32).cuda()
    with torch.no_grad():
        for m in c.net:
            if isinstance(m, torch.nn.Conv2d):
                m.weight.normal_(0, 0.2)
                m.bias.normal_(0, 0.2)
    B = 8
    th0 = torch.rand(B, 2, L, L, device="cuda") * TWO_PI
    R = torch.randn(B, 2, L, L, device="cuda")
    r = torch.randn(B, device="cuda")

    def run(fn):
        c.zero_grad(set_to_none=True)
        th = th0.clone().requires_grad_(True)
        out, ld = fn(th)
        ((out * R).sum() + (ld * r).sum()).backward()
        return th.grad.clone(), [p.grad.clone() for p in c.parameters()]

    g_f, w_f = run(c.forward_fused)
    g_r, w_r = run(lambda t: _layer_ref_fp32(c, t))
    assert torch.allclose(g_f, g_r, atol=2e-3, rtol=2e-3)
    for a, b in zip(w_f, w_r):
        assert torch.allclose(a, b, atol=5e-3 * max(1.0, b.abs().max().item()), rtol=2e-3)
