"""Plain float64 torch restatement of the Wilson action, for the adjoint tests.

Index tables follow the reference's even/odd layout (include/index.h:114-153):
lexicographic id = x0 + N0 (x1 + N1 (x2 + N2 x3)), EO index = id >> 1,
parity = (x0 + x1 + x2 + x3) & 1, link (x, mu) at EO + parity V/2 + mu V.
"""
from __future__ import annotations

import itertools

import numpy as np


def link_index(grid, x, mu):
    """Link array index of (x, mu) for coordinate arrays x = (x0, x1, x2, x3)."""
    N0, N1, N2, N3 = grid
    V = N0 * N1 * N2 * N3
    xs = [np.mod(c, n) for c, n in zip(x, grid)]
    lid = xs[0] + N0 * (xs[1] + N1 * (xs[2] + N2 * xs[3]))
    par = (xs[0] + xs[1] + xs[2] + xs[3]) & 1
    return (lid >> 1) + par * (V // 2) + mu * V


def plaquette_tables(dims: int, grid) -> tuple[np.ndarray, np.ndarray]:
    """For every site and mu < nu: the four link indices (a, b, c, d) with
    theta_P = th[a] + th[b] - th[c] - th[d], and whether nu is the time
    direction (dims - 1)."""
    axes = [np.arange(n) for n in grid]
    X = np.stack(np.meshgrid(*axes, indexing="ij"), 0).reshape(4, -1)
    rows, temporal = [], []
    for mu, nu in itertools.combinations(range(dims), 2):
        e = np.eye(4, dtype=np.int64)
        a = link_index(grid, X, mu)
        b = link_index(grid, X + e[mu][:, None], nu)
        c = link_index(grid, X + e[nu][:, None], mu)
        d = link_index(grid, X, nu)
        rows.append(np.stack([a, b, c, d], 1))
        temporal.append(np.full(a.shape, nu == dims - 1))
    return np.concatenate(rows, 0), np.concatenate(temporal, 0)


def torch_action(theta, tables, beta: float, aniso: float):
    """S per configuration for theta of shape (B, V*d) (any float dtype)."""
    import torch
    idx, temporal = tables
    idx_t = torch.as_tensor(idx, device=theta.device)
    w = torch.where(torch.as_tensor(temporal, device=theta.device),
                    torch.tensor(aniso, dtype=theta.dtype, device=theta.device),
                    torch.tensor(1.0 / aniso, dtype=theta.dtype, device=theta.device))
    th = theta[:, idx_t[:, 0]] + theta[:, idx_t[:, 1]] - theta[:, idx_t[:, 2]] - theta[:, idx_t[:, 3]]
    return beta * (w * (1.0 - torch.cos(th))).sum(dim=1)
