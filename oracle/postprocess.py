"""CPU oracle of the output consumers of `extract`.

TEST INFRASTRUCTURE ONLY.  Restates with the same PyTorch ops:

* ``spike_positions`` -- kilosort/postprocessing.py:33-62
  (compute_spike_positions): per spike, the 2-norm of its PC features on each
  of the nC channels nearest its template's peak channel, masked by
  ``iCC_mask``, normalised to sum 1, weights the channels' x and y;
* ``amplitudes`` -- kilosort/io.py:353: the 2-norm of each spike's features;
* ``similarity`` -- kilosort/CCG.py:94-102: the maximum over lags of the
  cross-correlation of the unit-norm templates (UtU over channels, WtW the
  flipped full cross-correlation of the wPCA rows);
* ``remove_duplicates`` -- kilosort/postprocessing.py:10-30 (a per-spike loop
  in index order, as the reference's numba function);
* ``phy_templates`` -- kilosort/io.py:383-387 (templates.npy, templates_ind.npy).

Pinned against tests/golden/golden_post.npz and tests/golden/golden_phy.npz
(the reference's own outputs; the latter from its save_to_phy).
"""
from __future__ import annotations

import numpy as np
import torch


def spike_positions(st, tF, iCC, iCC_mask, iU, xc, yc):
    tmass = torch.norm(tF, 2, dim=-1)
    tmask = iCC_mask[:, iU[st[:, 1]]].T
    tmass = tmass * tmask
    tmass = tmass / tmass.sum(1, keepdim=True)
    chs = iCC[:, iU[st[:, 1]]]
    xc0 = torch.from_numpy(xc)[chs.T]
    yc0 = torch.from_numpy(yc)[chs.T]
    return (xc0 * tmass).sum(1).numpy(), (yc0 * tmass).sum(1).numpy()


def amplitudes(tF):
    return torch.norm(tF, dim=[-2, -1]).numpy()


def similarity(Wall, W, nt=61):
    from torch.nn.functional import conv1d
    WtW = conv1d(W.reshape(-1, 1, nt), W.reshape(-1, 1, nt), padding=nt)
    WtW = torch.flip(WtW, [2])
    mu = (Wall ** 2).sum((1, 2), keepdims=True) ** .5
    Wnorm = Wall / (1e-6 + mu)
    UtU = torch.einsum('ilk, jlm -> ijkm', Wnorm, Wnorm)
    return torch.einsum('ijkm, kml -> ijl', UtU, WtW).numpy().max(axis=-1)


def remove_duplicates(spike_times, spike_clusters, dt=15):
    """kilosort/postprocessing.py:10-30: spikes in index order; a spike is
    kept when its time is at least dt after the last kept spike of its
    cluster (the first spike of a cluster is kept).  Returns
    (spike_times[keep], spike_clusters[keep], keep)."""
    spike_times = np.asarray(spike_times, dtype=np.int64)
    spike_clusters = np.asarray(spike_clusters, dtype=np.int32)
    keep = np.zeros(spike_times.size, bool)
    last = {}
    for i in range(spike_times.size):
        t, c = int(spike_times[i]), int(spike_clusters[i])
        t0 = last.get(c, t - dt)
        if t >= t0 + dt:
            last[c] = t
            keep[i] = True
    return spike_times[keep], spike_clusters[keep], keep


def phy_templates(Wall, W):
    """kilosort/io.py:383-387: templates [K, nt, C] = the products
    Wall[k, c, p] * W[p, t] summed over p, and templates_ind [K, C]."""
    templates = (Wall.unsqueeze(-1).cpu() * W.cpu()).sum(axis=-2).numpy()
    templates = templates.transpose(0, 2, 1)
    ind = np.tile(np.arange(Wall.shape[1])[np.newaxis, :], (templates.shape[0], 1))
    return templates, ind
