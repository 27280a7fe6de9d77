"""CPU oracle for Kilosort4's template-matching hot path.

TEST INFRASTRUCTURE ONLY.  This module restates, on the CPU with PyTorch
tensor ops, the algorithm of ``kilosort/template_matching.py`` (the reference
package's `run_matching`, `prepare_matching`, `prepare_extract` and the
per-batch feature step of `extract`).  Only the tests, the smoke check and the
benchmark's CPU-baseline leg use it, and only as the checker: the product
path in ``kilosort_b200`` never imports it.

Parity of this restatement is pinned against outputs of the reference itself
(``tests/golden/make_golden.py`` runs the reference's own functions on seeded
inputs and stores their outputs; ``tests/test_oracle_golden.py`` asserts that
this module reproduces them bit for bit in float32).

Every function runs in the dtype and on the device of its inputs, so the same
code gives the float64 oracle used for error statements and, on CUDA tensors,
the reference's own op sequence on the GPU (the benchmark's reference-on-GPU
timing).
"""
from __future__ import annotations

import numpy as np
import torch
import torch.nn.functional as F

__all__ = [
    "template_energy",
    "project_scores",
    "peel",
    "run_matching",
    "prepare_matching",
    "prepare_extract",
    "spike_features",
]

# kilosort/template_matching.py:186-188 preallocates this many spike rows per batch.
SPIKE_CAPACITY = 100000


def template_energy(U: torch.Tensor) -> torch.Tensor:
    """nm[k] = sum_{p,c} U[k,p,c]^2, summed over channels first.

    Follows kilosort/template_matching.py:176.
    """
    sq = U * U
    return sq.sum(dim=2).sum(dim=1)


def project_scores(X: torch.Tensor, U: torch.Tensor, W: torch.Tensor, nt: int):
    """Score matrix B[k, tau] = sum_{p,c} U[k,p,c] * (X[c] (*) W[p])[tau].

    The temporal projection is a zero-padded cross-correlation of every
    channel with every basis row (kilosort/template_matching.py:180); the
    channel/component contraction follows at :181.
    """
    Y = F.conv1d(X[:, None, :], W[:, None, :], padding=nt // 2)   # [C, P, L]
    # torch.einsum flattens contracted labels in label order; "q" (component)
    # before "r" (channel) sums in the same order as the reference's equation.
    return torch.einsum("kqr,rqt->kt", U, Y)


def _peak_columns(B, nm, Th, nt):
    """One detection pass (kilosort/template_matching.py:197-212).

    Returns (tau, best template, pooled score) for every column whose best
    score is the maximum of its +-nt neighbourhood and exceeds Th^2.
    """
    L = B.shape[1]
    score = torch.relu(B) ** 2 / nm[:, None]
    score[:, :nt] = 0
    score[:, L - nt:] = 0
    best, arg = torch.max(score, dim=0)
    pooled = F.max_pool1d(best[None, None, :], 2 * nt + 1, stride=1,
                          padding=nt)[0, 0]
    keep = (pooled > Th ** 2) & (torch.abs(pooled - best) < 1e-9)
    tau = torch.nonzero(keep)[:, 0]
    return tau, arg[tau], pooled


def peel(B, Xres, U, W, ctc, nm, Th, nt, max_peels, capacity=SPIKE_CAPACITY):
    """Greedy matching pursuit on a score matrix, in place on B and Xres.

    Follows kilosort/template_matching.py:183-244: every iteration detects all
    isolated peaks of the best per-column score, records (tau, k), the
    amplitude B[k, tau] / nm[k] and sqrt(pooled score), then subtracts the
    fitted waveforms from Xres and the template cross-correlations from B,
    even-indexed peaks first, odd-indexed peaks second.
    Returns (st [N,2] int64, amps [N,1], th_amps [N,1], n_iterations).
    """
    dt = B.dtype
    dev = B.device          # the reference's buffers live on its device (:186-188)
    lags = torch.arange(-nt, nt + 1, device=dev)
    taps = torch.arange(-(nt // 2), nt // 2 + 1, device=dev)
    st = torch.zeros((capacity, 2), dtype=torch.int64, device=dev)
    amps = torch.zeros((capacity, 1), dtype=dt, device=dev)
    th_amps = torch.zeros((capacity, 1), dtype=dt, device=dev)
    n = 0
    it = 0
    for it in range(max_peels):
        tau, k, pooled = _peak_columns(B, nm, Th, nt)
        m = int(tau.numel())
        if m == 0:
            break
        if n + m > capacity:
            raise RuntimeError(
                f"spike buffer overflow: {n + m} spikes > capacity {capacity}")
        st[n:n + m, 0] = tau
        st[n:n + m, 1] = k
        a = (B[k, tau] / nm[k])[:, None]
        amps[n:n + m] = a
        th_amps[n:n + m, 0] = pooled[tau] ** .5
        n += m
        for g in range(2):
            tg, kg, ag = tau[g::2], k[g::2], a[g::2]
            wave = torch.einsum("kpc,pt->ckt", U[kg], W)          # [C, m_g, nt]
            Xres[:, tg[:, None] + taps] -= ag * wave
            B[:, tg[:, None] + lags] -= ag * ctc[:, kg, :]
    return st[:n], amps[:n], th_amps[:n], it


def run_matching(ops, X, U, ctc, capacity=SPIKE_CAPACITY):
    """Oracle of kilosort/template_matching.py:170-244 (CPU tensors)."""
    nt = int(ops["nt"])
    W = ops["wPCA"].contiguous()
    nm = template_energy(U)
    B = project_scores(X, U, W, nt)
    Xres = X.clone()
    st, amps, th_amps, _ = peel(B, Xres, U, W, ctc, nm, ops["Th_learned"], nt,
                                int(ops["max_peels"]), capacity)
    return st, amps, th_amps, Xres


def prepare_matching(ops, U):
    """ctc[i, j, l] = sum_{k,m} (U_i U_j^T)[k, m] * WtW[k, m, l].

    WtW is the full cross-correlation of the basis rows, time-reversed
    (kilosort/template_matching.py:155-167).
    """
    nt = int(ops["nt"])
    W = ops["wPCA"].contiguous()
    WtW = F.conv1d(W[:, None, :], W[:, None, :], padding=nt)
    WtW = torch.flip(WtW, dims=[2])
    UtU = torch.einsum("ikc,jmc->ijkm", U, U)
    return torch.einsum("ijkm,kml->ijl", UtU, WtW)


def prepare_extract(xc, yc, U, nC, position_limit):
    """Neighbour channels and per-template feature loadings.

    Follows kilosort/template_matching.py:14-53: iCC[:, c] are the nC channels
    nearest to c (numpy argsort of squared distances), iCC_mask marks those
    within position_limit, iU[k] is the channel of largest sum_p U^2 and
    Ucc[i, k, p] = U[k, p, iCC[i, iU[k]]].
    """
    d2 = (xc[None, :] - xc[:, None]) ** 2 + (yc[None, :] - yc[:, None]) ** 2
    iCC = torch.from_numpy(np.argsort(d2, 0)[:nC])
    mask = torch.from_numpy(np.sort(d2, 0)[:nC] < position_limit ** 2)
    iU = torch.argmax((U ** 2).sum(1), -1)
    Ucc = U[torch.arange(U.shape[0]), :, iCC[:, iU]]
    return iCC, mask, iU, Ucc


def spike_features(Xres, st, amps, W, iCC, iU, Ucc, nt):
    """PC features of each spike on its template's nC nearest channels.

    Follows kilosort/template_matching.py:85-86: the residual around the
    spike, projected on the basis, plus the template's own loading times the
    amplitude.  Returns [nC, N, P].
    """
    taps = torch.arange(-(nt // 2), nt // 2 + 1)
    chans = iCC[:, iU[st[:, 1:2]]]                    # [nC, N, 1]
    window = Xres[chans, st[:, :1] + taps]            # [nC, N, nt]
    feat = window @ W.T
    feat += amps * Ucc[:, st[:, 1]]
    return feat
