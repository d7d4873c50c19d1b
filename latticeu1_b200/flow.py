"""Gauge-equivariant normalizing flow for 2D U(1) and an independence
Metropolis-Hastings sampler built on it.

Method after Kanwar et al., "Equivariant flow-based sampling for lattice
gauge theory", arXiv:2003.06413 (restated, not copied): masked coupling
layers transform plaquette angles with an invertible circular map whose
parameters come from a convolutional net over the plaquettes the layer leaves
unchanged; the updated link absorbs the change of its "active" plaquette, so
the map is gauge-equivariant and its Jacobian is the product of the circular
map's derivatives.  The reference has no flow; its 2D Wilson action and
Metropolis + overrelaxation chain (src/update.cu, include/staple.h) are the
target distribution and the baseline sampler.

Layout inside the flow: theta[b, mu, x1, x0] (the reference's natural order
with x0 fastest, include/index.h:51-56), mu = 0 along x0, mu = 1 along x1
(the time direction of the 2D lattice).  The action is evaluated by the
library's kernel (latticeu1_b200.action) after a permutation to the
even/odd layout.

Library kernels on this path: the circular coupling transform and its
inverse with analytic backward passes (u1_ncp_*), the Wilson action and its
adjoint (u1_wilson_action*), and for proposals one fused kernel per coupling
layer (u1_flow_layer_forward: context net, transform, link update, log-det).
In training the 3x3 convolutions run through cuDNN in bfloat16 with FP32
accumulation.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np
import torch
from torch import nn

from ._lib import check, lib
from .action import WilsonAction

__all__ = ["Flow2D", "eo_permutation", "plaquettes_no", "independence_mh", "tau_int", "sample_mc",
           "plain_chain_q", "run_experiment"]

TWO_PI = 2.0 * math.pi


def _stream(t: torch.Tensor) -> C.c_void_p:
    return C.c_void_p(torch.cuda.current_stream(t.device).cuda_stream)


def _p(t: torch.Tensor | None) -> C.c_void_p:
    return C.c_void_p(t.data_ptr() if t is not None else 0)


class _NCP(torch.autograd.Function):
    """(x, params) -> (dy, logd), elementwise; x: (n,), params: (n, 2K+1)."""

    @staticmethod
    def forward(ctx, x, params, K: int):
        x = x.contiguous().float()
        params = params.contiguous().float()
        n = x.numel()
        dy = torch.empty_like(x)
        logd = torch.empty_like(x)
        with torch.cuda.device(x.device):
            check(lib.u1_ncp_forward(_p(x), _p(params), n, K, _p(dy), _p(logd), _stream(x)), "u1_ncp_forward")
        ctx.save_for_backward(x, params)
        ctx.K = K
        return dy, logd

    @staticmethod
    def backward(ctx, gdy, glogd):
        x, params = ctx.saved_tensors
        gx = torch.empty_like(x)
        gp = torch.empty_like(params)
        gdy = gdy.contiguous().float() if gdy is not None else None
        glogd = glogd.contiguous().float() if glogd is not None else None
        with torch.cuda.device(x.device):
            check(lib.u1_ncp_backward(_p(x), _p(params), _p(gdy), _p(glogd), x.numel(), ctx.K, _p(gx), _p(gp),
                                      _stream(x)), "u1_ncp_backward")
        return gx, gp, None


class _NCPInverse(torch.autograd.Function):
    """(y, params) -> (dx, logd) of the inverse map (bisection solve)."""

    @staticmethod
    def forward(ctx, y, params, K: int):
        y = y.contiguous().float()
        params = params.contiguous().float()
        n = y.numel()
        dx = torch.empty_like(y)
        xs = torch.empty_like(y)
        logd = torch.empty_like(y)
        with torch.cuda.device(y.device):
            check(lib.u1_ncp_inverse(_p(y), _p(params), n, K, _p(dx), _p(xs), _p(logd), _stream(y)),
                  "u1_ncp_inverse")
        ctx.save_for_backward(xs, params)
        ctx.K = K
        return dx, logd

    @staticmethod
    def backward(ctx, gdx, glogd):
        xs, params = ctx.saved_tensors
        gy = torch.empty_like(xs)
        gp = torch.empty_like(params)
        gdx = gdx.contiguous().float() if gdx is not None else None
        glogd = glogd.contiguous().float() if glogd is not None else None
        with torch.cuda.device(xs.device):
            check(lib.u1_ncp_inverse_backward(_p(xs), _p(params), _p(gdx), _p(glogd), xs.numel(), ctx.K, _p(gy),
                                              _p(gp), _stream(xs)), "u1_ncp_inverse_backward")
        return gy, gp, None


def ncp_forward(x, params, K):
    return _NCP.apply(x, params, K)


def ncp_inverse(y, params, K):
    return _NCPInverse.apply(y, params, K)


class _FusedLayer(torch.autograd.Function):
    """A whole coupling layer as the library's fused kernels:
    (theta, W1, B1, W2, B2) -> (theta_out, logdet) with u1_flow_layer_forward
    (or, inverse, u1_flow_layer_inverse), gradients with
    u1_flow_layer_backward (u1_flow_layer_inverse_backward); L <= 32."""

    @staticmethod
    def forward(ctx, th, W1, B1, W2, B2, meta, inverse=False):
        L, mu, off, K, H, slope = meta
        th = th.contiguous()
        out = torch.empty_like(th)
        ld = torch.empty(th.shape[0], device=th.device)
        fn, name = ((lib.u1_flow_layer_inverse, "u1_flow_layer_inverse") if inverse
                    else (lib.u1_flow_layer_forward, "u1_flow_layer_forward"))
        with torch.cuda.device(th.device):
            check(fn(_p(th), _p(out), _p(ld), th.shape[0], L, mu, off, K, H, _p(W1), _p(B1), _p(W2), _p(B2),
                     C.c_float(slope), _stream(th)), name)
        ctx.save_for_backward(th, W1, B1, W2, B2)
        ctx.meta = meta
        ctx.inverse = inverse
        return out, ld

    @staticmethod
    def backward(ctx, g_out, g_ld):
        th, W1, B1, W2, B2 = ctx.saved_tensors
        L, mu, off, K, H, slope = ctx.meta
        fn, name = ((lib.u1_flow_layer_inverse_backward, "u1_flow_layer_inverse_backward") if ctx.inverse
                    else (lib.u1_flow_layer_backward, "u1_flow_layer_backward"))
        B = th.shape[0]
        C2 = 2 * K + 1
        nw = H * 18 + H + C2 * H * 9 + C2
        g_out = torch.zeros_like(th) if g_out is None else g_out.contiguous()
        g_ld = None if g_ld is None else g_ld.contiguous().float()
        gth = torch.empty_like(th)
        part = torch.empty((B, nw), device=th.device)
        wg = torch.empty(nw, device=th.device)
        with torch.cuda.device(th.device):
            check(fn(_p(th), _p(g_out), _p(g_ld), _p(gth), _p(part), _p(wg), B, L, mu, off, K, H, _p(W1), _p(B1),
                     _p(W2), _p(B2), C.c_float(slope), _stream(th)), name)
        o = 0
        gW1 = wg[o:o + H * 18].view_as(W1)
        o += H * 18
        gB1 = wg[o:o + H]
        o += H
        gW2 = wg[o:o + C2 * H * 9].view_as(W2)
        o += C2 * H * 9
        gB2 = wg[o:o + C2]
        return gth, gW1, gB1, gW2, gB2, None, None


def plaquettes_no(th: torch.Tensor) -> torch.Tensor:
    """P(x) = th_0(x) + th_1(x + e0) - th_0(x + e1) - th_1(x) for th[b, mu, x1, x0]."""
    t0, t1 = th[:, 0], th[:, 1]
    return t0 + torch.roll(t1, -1, dims=-1) - torch.roll(t0, -1, dims=-2) - t1


def eo_permutation(L0: int, L1: int) -> np.ndarray:
    """perm with theta_eo = theta_no.reshape(B, -1)[:, perm]: the reference's
    EO link index e = eo + parity V/2 + mu V (include/index.h:114-153) taken
    from the natural-order index mu V + lex, lex = x0 + L0 x1."""
    V = L0 * L1
    lex = np.arange(V)
    x0, x1 = lex % L0, lex // L0
    par = (x0 + x1) & 1
    eo_pos = (lex >> 1) + par * (V // 2)
    perm = np.empty(2 * V, dtype=np.int64)
    for mu in range(2):
        perm[mu * V + eo_pos] = mu * V + lex
    return perm


class Coupling(nn.Module):
    """One masked coupling layer: links of direction mu at sites with
    x_nu = off (mod 4), nu = 1 - mu, are updated through the plaquette in
    which they enter with a + sign; the context is the plaquettes that hold
    no updated link."""

    def __init__(self, L: int, mu: int, off: int, K: int = 6, hidden: int = 32):
        super().__init__()
        self.L, self.mu, self.off, self.K = L, mu, off, K
        self.net = nn.Sequential(
            nn.Conv2d(2, hidden, 3, padding=1, padding_mode="circular"),
            nn.LeakyReLU(),
            nn.Conv2d(hidden, 2 * K + 1, 3, padding=1, padding_mode="circular"),
        )
        nn.init.zeros_(self.net[2].weight)  # start at the identity map (alpha = 1, uniform weights, no shift)
        nn.init.zeros_(self.net[2].bias)
        r = np.arange(L)
        # coordinate along nu (the axis the stripes are offset on), in tensor axes [x1, x0]
        if mu == 0:
            link = (r % 4 == off)[:, None] & np.ones(L, bool)[None, :]           # x1 = off
            active = link                                                       # P(x)
            frozen = np.isin((r - off) % 4, (1, 2))[:, None] & np.ones(L, bool)[None, :]  # x1 = off+1, off+2
        else:
            link = np.ones(L, bool)[:, None] & (r % 4 == off)[None, :]           # x0 = off
            active = np.ones(L, bool)[:, None] & (r % 4 == (off - 1) % 4)[None, :]  # P(x - e0)
            frozen = np.ones(L, bool)[:, None] & np.isin((r - off) % 4, (1, 2))[None, :]  # x0 = off+1, off+2
        # the active plaquette of link (x1, x0) is at (x1, x0) (mu = 0) or (x1, x0 - 1) (mu = 1)
        li = np.argwhere(link)
        ai = li.copy()
        if mu == 1:
            ai[:, 1] = (ai[:, 1] - 1) % L
        assert active[ai[:, 0], ai[:, 1]].all()
        self.register_buffer("link_idx", torch.as_tensor(li[:, 0] * L + li[:, 1]))
        self.register_buffer("act_idx", torch.as_tensor(ai[:, 0] * L + ai[:, 1]))
        self.register_buffer("frozen", torch.as_tensor(frozen, dtype=torch.float32)[None, None])

    def _params(self, P: torch.Tensor) -> torch.Tensor:
        ctx = torch.stack([torch.cos(P), torch.sin(P)], 1) * self.frozen
        with torch.autocast("cuda", dtype=torch.bfloat16, cache_enabled=False):
            prm = self.net(ctx)
        B = P.shape[0]
        prm = prm.float().reshape(B, 2 * self.K + 1, -1)[:, :, self.act_idx]  # (B, 2K+1, n)
        return prm.permute(0, 2, 1).reshape(-1, 2 * self.K + 1)

    def _apply_delta(self, th: torch.Tensor, delta: torch.Tensor) -> torch.Tensor:
        B = th.shape[0]
        flat = th.reshape(B, 2, -1)
        upd = flat[:, self.mu].index_add(1, self.link_idx, delta.reshape(B, -1))
        parts = [upd, flat[:, 1]] if self.mu == 0 else [flat[:, 0], upd]
        return torch.stack(parts, 1).reshape_as(th)

    def forward_fused(self, th: torch.Tensor):
        """The layer as the library's fused forward/backward kernels:
        bf16-rounded weights, FP32 arithmetic."""
        c1, c2 = self.net[0], self.net[2]
        meta = (self.L, self.mu, self.off, self.K, c1.out_channels, self.net[1].negative_slope)
        return _FusedLayer.apply(th, c1.weight, c1.bias, c2.weight, c2.bias, meta)

    def inverse_fused(self, th: torch.Tensor):
        """The inverse layer as the library's fused kernels (differentiable)."""
        c1, c2 = self.net[0], self.net[2]
        meta = (self.L, self.mu, self.off, self.K, c1.out_channels, self.net[1].negative_slope)
        return _FusedLayer.apply(th, c1.weight, c1.bias, c2.weight, c2.bias, meta, True)

    def forward(self, th: torch.Tensor):
        B = th.shape[0]
        P = plaquettes_no(th)
        prm = self._params(P)
        Pa = P.reshape(B, -1)[:, self.act_idx].reshape(-1)
        dy, logd = ncp_forward(Pa, prm, self.K)
        return self._apply_delta(th, dy), logd.reshape(B, -1).sum(1)

    def inverse(self, th: torch.Tensor):
        B = th.shape[0]
        P = plaquettes_no(th)
        prm = self._params(P)  # the context plaquettes are unchanged by the layer
        Pa = P.reshape(B, -1)[:, self.act_idx].reshape(-1)
        dx, logd = ncp_inverse(Pa, prm, self.K)
        return self._apply_delta(th, dx), logd.reshape(B, -1).sum(1)


class Flow2D(nn.Module):
    """n_layers coupling layers (mu = l % 2, stripe offset (l // 2) % 4) on
    an L x L lattice; prior: uniform (Haar) link angles."""

    def __init__(self, L: int, beta: float, n_layers: int = 8, K: int = 6, hidden: int = 32):
        super().__init__()
        if L % 4:
            raise ValueError("L must be a multiple of 4")
        self.L, self.beta = L, float(beta)
        self.layers = nn.ModuleList([Coupling(L, l % 2, (l // 2) % 4, K, hidden) for l in range(n_layers)])
        self.action = WilsonAction(2, (L, 0, 0, L), beta)
        self.register_buffer("perm", torch.as_tensor(eo_permutation(L, L)))
        self.log_prior = -2 * L * L * math.log(TWO_PI)

    def to_eo(self, th: torch.Tensor) -> torch.Tensor:
        return th.reshape(th.shape[0], -1)[:, self.perm]

    def from_eo(self, th_eo: torch.Tensor) -> torch.Tensor:
        out = torch.empty_like(th_eo)
        out[:, self.perm] = th_eo
        return out.reshape(-1, 2, self.L, self.L)

    def sample(self, B: int, generator: torch.Generator | None = None, fused: bool = False):
        """(theta, log q(theta)) for B flow samples; fused: each layer through
        the library's fused kernels (differentiable)."""
        dev = self.perm.device
        th = torch.rand((B, 2, self.L, self.L), device=dev, generator=generator) * TWO_PI
        logq = torch.full((B,), self.log_prior, device=dev)
        for layer in self.layers:
            th, ld = layer.forward_fused(th) if fused else layer(th)
            logq = logq - ld
        return torch.remainder(th, TWO_PI), logq

    @torch.no_grad()
    def sample_fused(self, B: int, generator: torch.Generator | None = None):
        """As sample(), each coupling layer one library kernel
        (u1_flow_layer_forward: context net with bf16-rounded weights and FP32
        arithmetic, transform, link update, log-det), for proposals."""
        dev = self.perm.device
        th = torch.rand((B, 2, self.L, self.L), device=dev, generator=generator) * TWO_PI
        buf = torch.empty_like(th)
        ld = torch.empty(B, device=dev)
        logq = torch.full((B,), self.log_prior, device=dev)
        with torch.cuda.device(dev):
            stream = torch.cuda.current_stream(dev).cuda_stream
            for layer in self.layers:
                c1, c2 = layer.net[0], layer.net[2]
                check(lib.u1_flow_layer_forward(_p(th), _p(buf), _p(ld), B, self.L, layer.mu, layer.off, layer.K,
                                                c1.out_channels, _p(c1.weight), _p(c1.bias), _p(c2.weight),
                                                _p(c2.bias), C.c_float(layer.net[1].negative_slope),
                                                C.c_void_p(stream)), "u1_flow_layer_forward")
                logq -= ld
                th, buf = buf, th
        return torch.remainder(th, TWO_PI), logq

    def log_prob(self, th: torch.Tensor, fused: bool = False) -> torch.Tensor:
        """log q(theta) through the inverse flow; fused: each inverse layer
        through the library's fused kernels (differentiable)."""
        logq = torch.full((th.shape[0],), self.log_prior, device=th.device)
        for layer in reversed(self.layers):
            th, ld = layer.inverse_fused(th) if fused else layer.inverse(th)
            logq = logq - ld
        return logq

    def S(self, th: torch.Tensor) -> torch.Tensor:
        return self.action(self.to_eo(th))

    def charge(self, th: torch.Tensor) -> torch.Tensor:
        return self.action.charge(self.to_eo(th.detach()).double())

    def reverse_kl_step(self, opt, B: int) -> dict:
        th, logq = self.sample(B)
        S = self.S(th)
        loss = (logq + S).mean()
        opt.zero_grad(set_to_none=True)
        loss.backward()
        opt.step()
        with torch.no_grad():
            lw = -(S + logq).double()
            ess = (torch.exp(2 * torch.logsumexp(lw, 0) - torch.logsumexp(2 * lw, 0)) / B).item()
        return {"loss": loss.item(), "ess": ess}

    def graphed_reverse_kl(self, opt, B: int, fused: bool = False):
        """The reverse-KL step (sampling, flow, action, backward, optimizer)
        captured once as a CUDA graph; returns a function that replays it and
        the static (loss, S, logq) tensors it refreshes.  opt must be built
        with capturable=True (e.g. Adam(..., capturable=True)).  fused: the
        layers run as the library's fused kernels."""
        def body():
            th, logq = self.sample(B, fused=fused)
            S = self.S(th)
            loss = (logq + S).mean()
            loss.backward()
            opt.step()
            return loss.detach(), S.detach(), logq.detach()

        side = torch.cuda.Stream()
        side.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(side):
            for _ in range(3):  # warm-up outside the graph (allocations, autograd state)
                opt.zero_grad(set_to_none=False)
                body()
        torch.cuda.current_stream().wait_stream(side)
        graph = torch.cuda.CUDAGraph()
        opt.zero_grad(set_to_none=False)
        with torch.cuda.graph(graph):
            opt.zero_grad(set_to_none=False)
            static = body()

        def step():
            graph.replay()
            return static

        step.graph = graph
        return step, static

    def forward_kl_step(self, opt, data: torch.Tensor, fused: bool = False) -> float:
        loss = -self.log_prob(data, fused=fused).mean()
        opt.zero_grad(set_to_none=True)
        loss.backward()
        opt.step()
        return loss.item()


def independence_mh(logw: np.ndarray, u: np.ndarray) -> tuple[np.ndarray, float]:
    """Independence Metropolis-Hastings over proposals with log weights
    logw = -S - log q, in order: index of the state after each step, and
    the acceptance rate.  u: uniforms in (0, 1), one per proposal."""
    n = len(logw)
    idx = np.empty(n, dtype=np.int64)
    cur = 0
    acc = 0
    for i in range(n):
        if i > 0 and math.log(u[i]) < logw[i] - logw[cur]:
            cur = i
            acc += 1
        idx[i] = cur
    return idx, acc / max(1, n - 1)


def tau_int(x: np.ndarray, S: float = 1.5) -> tuple[float, float, int]:
    """Integrated autocorrelation time with Wolff's automatic window
    (U. Wolff, Comput. Phys. Commun. 156 (2004) 143; the reference's
    calculateCorTime, src/actime.cpp:19-145): (tau_int, its error, W)."""
    x = np.asarray(x, dtype=np.float64)
    N = len(x)
    d = x - x.mean()
    f = np.fft.rfft(d, 2 * N)
    G = np.fft.irfft(f * np.conj(f))[:N] / (N - np.arange(N))
    if G[0] == 0.0:
        return 0.5, 0.0, 0
    W = N // 2
    acc = 0.0
    for t in range(1, N // 2):
        acc += G[t] / G[0]
        tau = S / math.log((acc + 1.0) / acc) if acc > 0 else 1e-16
        g = math.exp(-t / tau) - tau / math.sqrt(t * N)
        if g < 0:
            W = t
            break
    C0 = G[0] + 2 * G[1:W + 1].sum()
    Gc = G + C0 / N
    tint = 0.5 + Gc[1:W + 1].sum() / Gc[0]
    return float(tint), float(tint * 2 * math.sqrt((W - tint + 0.5) / N)), int(W)


def sample_mc(L: int, beta: float, n_chains: int, n_per_chain: int, therm: int = 200, every: int = 5,
              seed: int = 1234, ctx=None) -> torch.Tensor:
    """Configurations from the library's Metropolis + 4 OR chains (one batch
    of n_chains), as a float32 CUDA tensor theta[b, mu, x1, x0]."""
    from .lattice import Batch, Context
    ctx = ctx or Context(0)
    b = Batch(ctx, [(2, (L, 0, 0, L), beta)] * n_chains, seed=seed)
    stream = torch.cuda.current_stream()
    b.set_stream(stream.cuda_stream)
    b.hot_start()
    for _ in range(therm):
        b.update(1, 4)
    perm = torch.as_tensor(eo_permutation(L, L), device="cuda")
    out = torch.empty((n_per_chain, n_chains, 2 * L * L), dtype=torch.float32, device="cuda")
    for k in range(n_per_chain):
        for _ in range(every):
            b.update(1, 4)
        eo = b.export_all().reshape(n_chains, 2 * L * L)
        out[k][:, perm] = eo.float()
    torch.cuda.synchronize()
    b.close()
    return out.reshape(-1, 2, L, L)


def plain_chain_q(L: int, beta: float, n_chains: int, n_sweeps: int, therm: int = 500, seed: int = 99,
                  ctx=None) -> tuple[np.ndarray, np.ndarray, float]:
    """Topological charge and mean cos(theta_P) after every sweep (1 Met + 4 OR)
    of n_chains independent chains: arrays (n_sweeps, n_chains), and the
    device seconds per sweep of one chain (batched)."""
    from .lattice import Batch, Context
    ctx = ctx or Context(0)
    b = Batch(ctx, [(2, (L, 0, 0, L), beta)] * n_chains, seed=seed)
    stream = torch.cuda.current_stream()
    b.set_stream(stream.cuda_stream)
    b.hot_start()
    for _ in range(therm):
        b.update(1, 4)
    S = WilsonAction(2, (L, 0, 0, L), beta)
    q = torch.empty((n_sweeps, n_chains), dtype=torch.float64, device="cuda")
    pl = torch.empty_like(q)
    for k in range(n_sweeps):
        b.update(1, 4)
        th = b.export_all().reshape(n_chains, 2 * L * L)
        with torch.no_grad():
            q[k] = S.charge(th)
            pl[k] = 1.0 - S(th) / (beta * L * L)
    # device time of the sweeps alone
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(64):
        b.update(1, 4)
    e1.record(stream)
    e1.synchronize()
    t_sweep = e0.elapsed_time(e1) * 1e-3 / 64
    b.close()
    return q.cpu().numpy(), pl.cpu().numpy(), t_sweep / n_chains


def run_experiment(L: int = 16, beta: float = 2.0, n_layers: int = 8, K: int = 6, hidden: int = 32,
                   batch: int = 1024, n_warm: int = 10000, warm_epochs: int = 10, rkl_steps: int = 1000,
                   lr: float = 1e-3, n_props: int = 65536, plain_chains: int = 256, plain_sweeps: int = 2048,
                   seed: int = 0, fused: bool | None = None) -> dict:
    """Config: 2D U(1) L x L at beta; flow of n_layers coupling layers
    (2 conv 3x3 layers of `hidden` channels each) warm-started by forward KL
    on n_warm Metropolis + OR configurations and trained by reverse KL; an
    independence MH chain of n_props flow proposals is compared with plain
    Metropolis + OR chains: acceptance, <cos theta_P> against the exact
    I1(beta)/I0(beta) and tau_int of the topological charge."""
    import time

    from scipy.special import ive
    torch.manual_seed(seed)
    if fused is None:
        fused = L <= 32  # the fused layer kernels (forward, inverse and their backward) cover L <= 32
    res = {"L": L, "beta": beta, "layers": n_layers, "K": K, "hidden": hidden, "batch": batch,
           "training_layers": "fused kernels" if fused else "torch/cuDNN"}
    flow = Flow2D(L, beta, n_layers, K, hidden).cuda()
    opt = torch.optim.Adam(flow.parameters(), lr=lr)
    # warm start: forward KL on Markov-chain configurations
    t0 = time.perf_counter()
    per_chain = max(1, n_warm // 1000)
    data = sample_mc(L, beta, n_warm // per_chain, per_chain, therm=300, every=10, seed=seed + 1)
    res["warm_data_s"] = time.perf_counter() - t0
    t0 = time.perf_counter()
    fkl = []
    for ep in range(warm_epochs):
        idx = torch.randperm(data.shape[0], device="cuda")
        for i in range(0, data.shape[0] - batch + 1, batch):
            fkl.append(flow.forward_kl_step(opt, data[idx[i:i + batch]], fused=fused))
    torch.cuda.synchronize()
    res["warm_s"] = time.perf_counter() - t0
    res["forward_kl_first_last"] = [fkl[0], fkl[-1]] if fkl else None
    # reverse KL, one CUDA graph per step (optimizer state moved to a capturable Adam)
    opt2 = torch.optim.Adam(flow.parameters(), lr=lr, capturable=True)
    opt2.load_state_dict(opt.state_dict())
    for grp in opt2.param_groups:
        grp["capturable"] = True
    for st in opt2.state.values():
        if "step" in st and not st["step"].is_cuda:
            st["step"] = st["step"].cuda()
    step, (loss_t, S_t, logq_t) = flow.graphed_reverse_kl(opt2, batch, fused=fused)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    losses, ess = [], []
    for it in range(rkl_steps):
        step()
        if it % 100 == 0 or it == rkl_steps - 1:
            lw = -(S_t + logq_t).double()
            ess.append((torch.exp(2 * torch.logsumexp(lw, 0) - torch.logsumexp(2 * lw, 0)) / batch).item())
            losses.append(loss_t.item())
    torch.cuda.synchronize()
    res["rkl_s"] = time.perf_counter() - t0
    res["rkl_step_ms"] = 1e3 * res["rkl_s"] / max(1, rkl_steps)
    res["reverse_kl_loss_first_last"] = [losses[0], losses[-1]] if losses else None
    res["ess_last"] = float(np.mean(ess[-3:])) if ess else None
    res["min_loss_exact"] = -(2 * L * L * math.log(TWO_PI) + L * L * math.log(float(ive(0, beta))))
    # proposals
    lw, qs, pls = [], [], []
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record()
    with torch.no_grad():
        for _ in range(n_props // batch):
            th, logq = flow.sample_fused(batch)  # log q from the same kernels that make the sample
            S = flow.S(th)
            lw.append((-S - logq).double())
            qs.append(flow.charge(th))
            pls.append(1.0 - S.double() / (beta * L * L))
    ev1.record()
    ev1.synchronize()
    res["proposal_s_per_sample"] = ev0.elapsed_time(ev1) * 1e-3 / (n_props // batch * batch)
    lw = torch.cat(lw).cpu().numpy()
    qs = torch.cat(qs).cpu().numpy()
    pls = torch.cat(pls).cpu().numpy()
    u = np.random.default_rng(seed + 7).uniform(size=len(lw))
    idx, acc = independence_mh(lw, u)
    q_chain, p_chain = qs[idx], pls[idx]
    res["mh_acceptance"] = acc
    t_q, dt_q, _ = tau_int(np.round(q_chain))
    res["flow_tau_int_Q"] = [t_q, dt_q]
    t_p, _, _ = tau_int(p_chain)
    exact = float(ive(1, beta) / ive(0, beta))
    res["exact_cosP"] = exact
    res["flow_cosP"] = [float(p_chain.mean()), float(p_chain.std() * math.sqrt(2 * t_p / len(p_chain)))]
    res["flow_Q2"] = float(np.mean(np.round(q_chain) ** 2))
    # plain Metropolis + OR chains
    qp, pp, s_sweep = plain_chain_q(L, beta, plain_chains, plain_sweeps, seed=seed + 11)
    taus = [tau_int(np.round(qp[:, c]))[0] for c in range(plain_chains)]
    res["plain_tau_int_Q"] = [float(np.mean(taus)), float(np.std(taus) / math.sqrt(plain_chains))]
    tp = float(np.mean([tau_int(pp[:, c])[0] for c in range(min(plain_chains, 32))]))
    res["plain_cosP"] = [float(pp.mean()), float(pp.std() * math.sqrt(2 * tp / pp.size))]
    res["plain_Q2"] = float(np.mean(np.round(qp) ** 2))
    res["plain_s_per_sweep_per_chain"] = s_sweep
    # cost of one independent Q sample (2 tau_int steps)
    res["s_per_indep_Q_flow"] = 2 * t_q * res["proposal_s_per_sample"]
    res["s_per_indep_Q_plain"] = 2 * res["plain_tau_int_Q"][0] * s_sweep
    return res
