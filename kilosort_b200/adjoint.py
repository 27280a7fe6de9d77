"""Reconstruction loss with a hand-written adjoint, for template refinement.

For a fixed spike assignment (the ``st`` and ``amps`` that ``run_matching``
returns) the reconstruction of a batch is

    R[c, tau] = sum_s amps[s] * sum_p U[k_s, p, c] * wPCA[p, tau - tau_s + nt//2]

-- the subtraction kilosort/template_matching.py:237 applies spike by spike --
and ``reconstruction_loss`` returns ``||X - R||^2``.  Its backward is the
sm_100a adjoint kernel of ``libks_b200.so`` (``ks_recon_adjoint``): gradients
with respect to U, wPCA and the amplitudes (and X), recomputing the template
waveforms U x wPCA per block instead of storing them.  Both directions are
deterministic.

    loss = reconstruction_loss(X, st, amps, U, wPCA)
    loss.backward()          # U.grad, wPCA.grad, amps.grad
"""
from __future__ import annotations

import torch

from . import _lib
from .template_matching import _need, _ptr, _stream

__all__ = ["reconstruction_loss", "reconstruct", "ReconstructionLoss"]


class _Scratch:
    def __init__(self):
        self.buf = {}

    def get(self, device, nbytes):
        key = (device.type, device.index)
        b = self.buf.get(key)
        if b is None or b.numel() < nbytes:
            b = torch.empty(max(int(nbytes), 256), dtype=torch.uint8, device=device)
            self.buf[key] = b
        return b


_scratch = _Scratch()


def _shapes(X, st, amps, U, W):
    C, L = X.shape
    K, P, Cu = U.shape
    if Cu != C:
        raise ValueError(f"U has {Cu} channels but X has {C}")
    if W.shape[0] != P or W.shape[1] % 2 == 0:
        raise ValueError(f"wPCA must be [{P}, odd nt], got {tuple(W.shape)}")
    if st.dim() != 2 or st.shape[1] != 2:
        raise ValueError("st must be [N, 2] (time, template)")
    if amps.numel() != st.shape[0]:
        raise ValueError("amps must hold one amplitude per spike")
    return C, L, K, P, W.shape[1], st.shape[0]


def _check_status(status, what):
    s = int(status.item())
    if s != _lib.KS_OK:
        raise _lib.KilosortB200Error(s, f"{what}: a spike's time or template is out of range")


def _forward(X, st, amps_f, U, W):
    C, L, K, P, nt, N = _shapes(X, st, amps_f, U, W)
    dev = X.device
    lib = _lib.load()
    ws = _scratch.get(dev, lib.ks_recon_workspace_size(C, L, K, P, nt, N))
    Xres = torch.empty_like(X)
    loss = torch.empty((), dtype=torch.float64, device=dev)
    status = torch.empty(1, dtype=torch.int32, device=dev)
    _lib.check(lib.ks_recon_loss(_ptr(X), _ptr(st), _ptr(amps_f), N, _ptr(U), _ptr(W),
                                 C, L, K, P, nt, _ptr(Xres), _ptr(loss), _ptr(status),
                                 _ptr(ws), ws.numel(), _stream(dev)), "ks_recon_loss")
    _check_status(status, "ks_recon_loss")
    return Xres, loss


def reconstruct(X, st, amps, U, wPCA):
    """``(X - R, ||X - R||^2)`` without autograd (loss as a float64 tensor)."""
    return _forward(_need(X, "X", ndim=2), _need(st, "st", dtype=torch.int64, ndim=2),
                    _need(amps, "amps").reshape(-1), _need(U, "U", ndim=3),
                    _need(wPCA, "wPCA", ndim=2))


class ReconstructionLoss(torch.autograd.Function):
    """loss = ||X - R(st, amps, U, wPCA)||^2 with the hand-written adjoint."""

    @staticmethod
    def forward(ctx, X, amps, U, W, st):
        X = _need(X, "X", ndim=2)
        U = _need(U, "U", ndim=3)
        W = _need(W, "wPCA", ndim=2)
        st = _need(st, "st", dtype=torch.int64, ndim=2)
        amps_f = _need(amps.detach(), "amps").reshape(-1)
        Xres, loss = _forward(X, st, amps_f, U.detach(), W.detach())
        ctx.save_for_backward(Xres, amps_f, U, W, st)
        ctx.amps_shape = amps.shape
        return loss.to(torch.float32)

    @staticmethod
    def backward(ctx, dloss):
        Xres, amps_f, U, W, st = ctx.saved_tensors
        C, L = Xres.shape
        K, P, _ = U.shape
        nt, N = W.shape[1], st.shape[0]
        dev = Xres.device
        g = dloss.detach().to(device=dev, dtype=torch.float32).reshape(1).contiguous()
        dU = torch.empty_like(U)
        dW = torch.empty_like(W)
        damps = torch.empty(max(N, 1), dtype=torch.float32, device=dev)
        status = torch.empty(1, dtype=torch.int32, device=dev)
        lib = _lib.load()
        ws = _scratch.get(dev, lib.ks_recon_workspace_size(C, L, K, P, nt, N))
        _lib.check(lib.ks_recon_adjoint(_ptr(Xres), _ptr(st), _ptr(amps_f), N, _ptr(U), _ptr(W),
                                        C, L, K, P, nt, _ptr(g), _ptr(dU), _ptr(dW),
                                        _ptr(damps), _ptr(status), _ptr(ws), ws.numel(),
                                        _stream(dev)), "ks_recon_adjoint")
        dX = 2.0 * g * Xres if ctx.needs_input_grad[0] else None
        return dX, damps[:N].reshape(ctx.amps_shape), dU, dW, None


def reconstruction_loss(X, st, amps, U, wPCA):
    """``||X - R||^2`` for spikes ``st`` [N, 2] with amplitudes ``amps`` [N] or [N, 1]."""
    return ReconstructionLoss.apply(X, amps, U, wPCA, st)
