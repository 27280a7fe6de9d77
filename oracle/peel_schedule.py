"""CPU model of a segment-skewed schedule of the greedy peel.

TEST INFRASTRUCTURE ONLY.  Nothing in ``kilosort_b200`` imports it.  It models
a schedule in which the batch's columns are cut into segments that advance
through the peel's iterations on their own, instead of all columns finishing
iteration i before any column starts iteration i + 1 (the order of
kilosort/template_matching.py:195-238 and of ``matching.peel``).  The test
next to it checks that every order such a schedule may take gives the spikes,
amplitudes, pooled scores and final score matrix of ``matching.peel`` bit for
bit; that is the condition for running the peel this way on the device, where
a segment's score rows could then be re-read from L2 between iterations.

Tasks, for segment s (columns [s*w, (s+1)*w), w >= nt) and iteration i:

* detect(s, i): the peak test of kilosort/template_matching.py:197-212 on the
  segment's columns.  It reads the best scores within +-nt of them, so it runs
  once update(s', i-1) has rescored segments s-1, s and s+1.
* update(s, i): the subtractions of :235-238 on the segment's columns from the
  iteration's peaks within +-nt (segments s-1, s, s+1), then the rescoring of
  those columns.  The reference applies even-indexed peaks before odd-indexed
  ones, where the index counts all of the iteration's peaks in time order.
  So the task also needs the peak counts of every segment left of it (a
  look-back), and runs once detect(s', i) is done for all s' <= s + 1.

The tasks run in a seeded random order among those whose dependencies are
met, standing for the device's asynchronous progress.  Arithmetic is the same
torch float32 element operations as ``matching.peel``.  The residual is not
modelled: it is applied from the records after the loop, as the device does.
"""
from __future__ import annotations

import numpy as np
import torch
import torch.nn.functional as F


def peel_skewed(B, nm, ctc, Th, nt, max_peels, width, seed=0):
    """Greedy peel of B (in place) under a random segment-skewed order.

    Returns (st [N,2] int64, amps [N,1], th_amps [N,1], n_iterations) in the
    record order of ``matching.peel`` (iteration, then time)."""
    K, L = B.shape
    if width < nt:
        raise ValueError("segments must be at least nt columns wide")
    nseg = (L + width - 1) // width
    bounds = [(s * width, min(L, (s + 1) * width)) for s in range(nseg)]
    th2 = Th ** 2
    best = torch.zeros(L, dtype=B.dtype)
    arg = torch.zeros(L, dtype=torch.int64)

    def rescore(s):
        lo, hi = bounds[s]
        score = torch.relu(B[:, lo:hi]) ** 2 / nm[:, None]
        c = torch.arange(lo, hi)
        score[:, (c < nt) | (c >= L - nt)] = 0
        best[lo:hi], arg[lo:hi] = torch.max(score, dim=0)

    for s in range(nseg):
        rescore(s)

    peaks = {}                      # (i, s) -> list of (tau, k, amp, th)
    det = np.full(nseg, -1)         # last iteration detected, per segment
    upd = np.full(nseg, -1)         # last iteration updated, per segment
    empty_at = None                 # first iteration without peaks anywhere
    rng = np.random.default_rng(seed)

    def detect(s, i):
        lo, hi = bounds[s]
        a, b = max(0, lo - nt), min(L, hi + nt)
        pooled = F.max_pool1d(best[a:b][None, None, :], 2 * nt + 1, stride=1,
                              padding=nt)[0, 0][lo - a:hi - a]
        keep = (pooled > th2) & (torch.abs(pooled - best[lo:hi]) < 1e-9)
        out = []
        for j in torch.nonzero(keep)[:, 0].tolist():
            tau = lo + j
            k = int(arg[tau])
            amp = B[k, tau] / nm[k]
            out.append((tau, k, amp, pooled[j] ** .5))
        peaks[(i, s)] = out

    def update(s, i):
        lo, hi = bounds[s]
        first = 0                   # global index of the first peak of segment 0..
        touching = []
        for s2 in range(0, min(nseg, s + 2)):
            lst = peaks[(i, s2)]
            if s2 >= s - 1:
                for e, (tau, k, amp, _) in enumerate(lst):
                    if tau + nt >= lo and tau - nt < hi:
                        touching.append((first + e, tau, k, amp))
            first += len(lst)
        touching.sort(key=lambda t: (t[0] & 1, t[0]))
        for _, tau, k, amp in touching:
            c0, c1 = max(lo, tau - nt), min(hi, tau + nt + 1)
            B[:, c0:c1] -= amp * ctc[:, k, c0 - tau + nt:c1 - tau + nt]
        rescore(s)

    def limit():
        return max_peels if empty_at is None else min(max_peels, empty_at + 1)

    while True:
        ready = []
        lim = limit()
        for s in range(nseg):
            i = det[s] + 1
            if i < lim and upd[s] == i - 1 and all(upd[t] >= i - 1 for t in (s - 1, s + 1)
                                                   if 0 <= t < nseg):
                ready.append(("detect", s, i))
            i = upd[s] + 1
            if i <= det[s] and i < lim and (empty_at is None or i < empty_at) \
                    and det[:min(nseg, s + 2)].min() >= i:
                ready.append(("update", s, i))
        if not ready:
            break
        kind, s, i = ready[rng.integers(len(ready))]
        if kind == "detect":
            detect(s, i)
            det[s] = i
            if empty_at is None and det.min() >= i and \
                    sum(len(peaks[(i, t)]) for t in range(nseg)) == 0:
                empty_at = i
        else:
            update(s, i)
            upd[s] = i

    n_iter = limit() if empty_at is None else empty_at
    rows = []
    for i in range(n_iter):
        for s in range(nseg):
            for tau, k, amp, th in peaks.get((i, s), []):
                rows.append((tau, k, amp, th))
    n = len(rows)
    st = torch.zeros((n, 2), dtype=torch.int64)
    amps = torch.zeros((n, 1), dtype=B.dtype)
    th_amps = torch.zeros((n, 1), dtype=B.dtype)
    for r, (tau, k, amp, th) in enumerate(rows):
        st[r, 0], st[r, 1] = tau, k
        amps[r, 0] = amp
        th_amps[r, 0] = th
    return st, amps, th_amps, n_iter
