"""Reference of the fixed-assignment reconstruction loss, for gradient checks.

TEST INFRASTRUCTURE ONLY.  Plain PyTorch ops (gather, einsum, index_add), any
dtype and device, differentiable by torch.autograd: the tests use it in
float64 as the autograd reference gradient and for the central finite
differences that pin the hand-written adjoint of ``kilosort_b200.adjoint``.

    R[c, tau] = sum_s amps[s] * sum_p U[k_s, p, c] * W[p, tau - tau_s + nt//2]
    loss      = sum_{c, tau} (X - R)[c, tau]^2

R restates the residual subtraction of kilosort/template_matching.py:237
(``Xres[:, iX + tiwave] -= amp * einsum('ijk, jl -> kil', U[iY], W)``) for a
fixed spike set; taps that fall outside [0, L) are dropped.
"""
from __future__ import annotations

import torch

__all__ = ["recon_residual", "recon_loss"]


def recon_residual(X, st, amps, U, W, chunk=4096):
    """X - R (differentiable in amps, U and W)."""
    C, L = X.shape
    nt = W.shape[1]
    half = nt // 2
    tiwave = torch.arange(-half, half + 1, device=X.device)
    R = torch.zeros((C, L + 1), dtype=X.dtype, device=X.device)   # column L collects dropped taps
    amps = amps.reshape(-1)
    for s0 in range(0, st.shape[0], chunk):
        tau = st[s0:s0 + chunk, 0]
        k = st[s0:s0 + chunk, 1]
        waves = torch.einsum("spc,pt->cst", U[k], W)              # [C, n, nt]
        contrib = waves * amps[s0:s0 + chunk].reshape(1, -1, 1)
        cols = tau[:, None] + tiwave[None, :]
        cols = torch.where((cols >= 0) & (cols < L), cols, torch.full_like(cols, L))
        R = R.index_add(1, cols.reshape(-1), contrib.reshape(C, -1))
    return X - R[:, :L]


def recon_loss(X, st, amps, U, W):
    return (recon_residual(X, st, amps, U, W) ** 2).sum()
