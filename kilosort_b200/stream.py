"""Streaming matcher: raw int16 on the host -> whitening -> batched matching.

The batches of kilosort/io.py (BinaryRWFile.padded_batch_to_torch, :789-831,
batch edges :771-783) are cut from a raw int16 recording ``raw`` [samples,
channels] in host memory: batch b covers samples [b*NT - nt, (b+1)*NT + nt),
the first batch's left pad repeats its first sample and a later batch that
ends early (the last) is padded with its last sample.  Per group of batches:

* copy stream: one host->device copy per batch window, straight from the
  page-locked source (the recording's memory is registered once; the two
  edge windows are assembled in a small page-locked staging buffer);
* compute stream: ``ks_whiten_int16`` (X = scale * Wrot @ raw, split-BF16 on
  the tensor cores) -- or, with ``preprocess`` settings (chan_map, hp_filter,
  do_CAR, invert_sign, artifact_threshold), the whole batch filter of
  kilosort/io.py:994-1026 (``ks_preprocess_int16``) -- writes each batch into
  a ``BatchedMatcher``'s inputs, then its captured graph matches the group
  (grouped contraction, team-split peel);
* two matchers alternate, so the host reads one group's spikes while the GPU
  matches the next;
* every ``refine_every`` groups the templates take one gradient step on the
  reconstruction loss of a matched batch (the hand-written adjoint), and the
  cross-correlations are recomputed in place (the captured graphs read them).
"""
from __future__ import annotations

from typing import List, Optional

import numpy as np
import torch

from . import _lib
from .adjoint import reconstruction_loss
from .batched import BatchedMatcher, Recording
from .preprocess import Preprocessor
from .template_matching import _ptr, _stream, prepare_matching


def batch_windows(n_samples: int, NT: int, nt: int):
    """(start, stop, left_pad, n_batches) of each padded batch, as io.py cuts them."""
    n_batches = int(np.ceil(n_samples / NT))
    out = []
    for b in range(n_batches):
        if b == 0:
            start, stop = 0, min(n_samples, NT + nt)
            left = nt
        else:
            start = b * NT - nt
            stop = min(n_samples, start + NT + 2 * nt)
            left = 0
        out.append((start, stop, left))
    return out


def padded_raw_window(raw: np.ndarray, b: int, NT: int, nt: int, out: np.ndarray):
    """The raw samples of padded batch b in ``out`` [NT + 2nt, C].

    As io.py:813-824 pads them: the first batch's left pad repeats its first
    sample and whatever follows its data stays zero (also when it is the only
    batch); a later batch that ends early repeats its last sample.
    """
    start, stop, left = batch_windows(raw.shape[0], NT, nt)[b]
    n = stop - start
    out[left:left + n] = raw[start:stop]
    if left:
        out[:left] = raw[start]
    if left + n < out.shape[0]:
        out[left + n:] = 0 if b == 0 else raw[stop - 1]
    return out


class Whitener:
    """``ks_whiten_int16`` with its own workspace and status word."""

    def __init__(self, Wrot: torch.Tensor, scale: float, L: int, device):
        self.Wrot = Wrot.to(device=device, dtype=torch.float32).contiguous()
        self.scale = float(scale)
        self.C = self.Wrot.shape[0]
        lib = _lib.load()
        self.ws = torch.empty(lib.ks_whiten_int16_workspace_size(L, self.C), dtype=torch.uint8,
                              device=device)
        self.flags = torch.zeros(1, dtype=torch.int32, device=device)

    def __call__(self, raw_dev: torch.Tensor, X: torch.Tensor):
        T, C = raw_dev.shape
        lib = _lib.load()
        _lib.check(lib.ks_whiten_int16(_ptr(raw_dev), T, C, raw_dev.stride(0), _ptr(self.Wrot),
                                       self.scale, _ptr(X), X.stride(0), _ptr(self.flags),
                                       _ptr(self.ws), self.ws.numel(), _stream(X.device)),
                   "ks_whiten_int16")
        return X

    def status(self):
        """(device status, artifact) of the last call (synchronises)."""
        return int(self.flags.item()), False


class StreamMatcher:
    """Match a raw int16 recording batch by batch, whitened on the GPU."""

    def __init__(self, raw: np.ndarray, Wrot: torch.Tensor, scale: float, ops, U: torch.Tensor,
                 NT: int, group: int = 8, teams: Optional[int] = 0, projection: str = "bf16x3",
                 refine_every: int = 0, refine_lr: float = 1e-4, device=None,
                 preprocess: Optional[dict] = None):
        if raw.dtype != np.int16 or raw.ndim != 2:
            raise TypeError("raw must be an int16 [samples, channels] array")
        self.raw = np.ascontiguousarray(raw)
        self.device = device or U.device
        self.NT, self.nt = int(NT), int(ops["nt"])
        self.L = self.NT + 2 * self.nt
        self.C = raw.shape[1]
        self.group = int(group)
        self.ops = ops
        self.U = U
        self.ctc = prepare_matching(ops, U)
        self.rec = Recording.from_ops(ops, U, self.ctc)
        self.windows = batch_windows(raw.shape[0], self.NT, self.nt)
        self.n_batches = len(self.windows)
        if preprocess is None:
            self.whiten = Whitener(Wrot, scale, self.L, self.device)
        else:
            # the whole filter of kilosort/io.py:994-1026 on each padded batch
            W = torch.as_tensor(Wrot, dtype=torch.float32) * float(scale)
            self.whiten = Preprocessor(self.C, self.L, whiten=W, device=self.device,
                                       **preprocess)
        self.refine_every = int(refine_every)
        self.refine_lr = float(refine_lr)
        self.refinements = 0
        self.copy_stream = torch.cuda.Stream(self.device)
        # page-locked source: the recording's own memory, registered once
        self._registered = False
        nbytes = self.raw.nbytes
        if nbytes:
            rc = torch.cuda.cudart().cudaHostRegister(self.raw.ctypes.data, nbytes, 0)
            self._registered = int(rc) == 0
        self.staging = torch.empty((2, self.L, self.C), dtype=torch.int16).pin_memory()
        self.raw_dev = [torch.empty((self.group, self.L, self.C), dtype=torch.int16,
                                    device=self.device) for _ in range(2)]
        self.copied = [torch.cuda.Event() for _ in range(2)]
        self.freed = [torch.cuda.Event() for _ in range(2)]
        self.done = [torch.cuda.Event() for _ in range(2)]
        self.readback = torch.cuda.Stream(self.device)
        n_grp = min(self.group, self.n_batches)
        self._short = {}
        self.matchers = [BatchedMatcher([self.rec], [(self.L, 0)] * n_grp, projection,
                                        teams=teams, graph=True) for _ in range(2)]

    def close(self):
        if self._registered:
            torch.cuda.cudart().cudaHostUnregister(self.raw.ctypes.data)
            self._registered = False

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -------------------------------------------------------------- pieces
    def _host_window(self, b: int):
        start, stop, left = self.windows[b]
        if left == 0 and stop - start == self.L:
            if self._registered:
                return torch.from_numpy(self.raw[start:stop])
            return torch.from_numpy(self.raw[start:stop]).pin_memory()
        slot = self.staging[0 if b == 0 else 1]
        padded_raw_window(self.raw, b, self.NT, self.nt, slot.numpy())
        return slot

    def _enqueue_copy(self, g: int, batches: List[int]):
        buf = self.raw_dev[g % 2]
        with torch.cuda.stream(self.copy_stream):
            self.copy_stream.wait_event(self.freed[g % 2])
            for i, b in enumerate(batches):
                buf[i].copy_(self._host_window(b), non_blocking=True)
            self.copied[g % 2].record(self.copy_stream)

    def _matcher(self, g: int, n: int) -> BatchedMatcher:
        """The matcher of group g: one of the two full-size ones, or (for a short
        last group) one of its own size, built once and kept for later runs."""
        if n == len(self.matchers[0].X):
            return self.matchers[g % 2]
        key = (g % 2, n)
        if key not in self._short:
            self._short[key] = BatchedMatcher([self.rec], [(self.L, 0)] * n,
                                              self.matchers[0].projection,
                                              teams=self.matchers[0].teams, graph=True)
        return self._short[key]

    def _enqueue_match(self, g: int, batches: List[int], m: BatchedMatcher):
        cur = torch.cuda.current_stream(self.device)
        cur.wait_event(self.copied[g % 2])
        for i in range(len(batches)):
            self.whiten(self.raw_dev[g % 2][i], m.X[i])
        self.freed[g % 2].record(cur)
        m.launch()
        self.done[g % 2].record(cur)

    def _refine(self, m: BatchedMatcher):
        """One gradient step on U from the reconstruction loss of the group's
        first batch, on each template's footprint only: the channels whose
        loading norm is at least 1e-3 of the template's largest.  Templates
        stay as sparse as they were (Kilosort4's live on their nearest
        channels); a dense step would spread every template over the probe
        and, through ctc, make every peel update touch every template group."""
        st, amps, _, _ = m.results()[0]
        if len(st) == 0:
            return
        Uq = self.U.detach().clone().requires_grad_(True)
        loss = reconstruction_loss(m.X[0], st, amps.reshape(-1), Uq, self.ops["wPCA"])
        loss.backward()
        with torch.no_grad():
            norm = self.U.norm(dim=1)                                   # [K, C]
            support = norm >= 1e-3 * norm.amax(dim=1, keepdim=True)
            self.U.sub_(self.refine_lr * Uq.grad * support.unsqueeze(1))
            self.ctc.copy_(prepare_matching(self.ops, self.U))
            lib = _lib.load()
            K = self.U.shape[0]
            _lib.check(lib.ks_ctc_transpose(_ptr(self.ctc), K, self.nt, _ptr(self.rec.ctcT),
                                            _stream(self.device)), "ks_ctc_transpose")
        self.refinements += 1

    # ------------------------------------------------------------------ run
    def run(self):
        """Match every batch; returns (times [N] int64 recording samples,
        templates [N] int64, amplitudes [N] float32, batch [N] int64)."""
        groups = [list(range(g0, min(g0 + self.group, self.n_batches)))
                  for g0 in range(0, self.n_batches, self.group)]
        times, templ, amps, bidx = [], [], [], []

        ms = [self._matcher(g, len(b)) for g, b in enumerate(groups)]

        def collect(g):
            # read group g on a side stream: the host waits for that group
            # only, while the compute stream runs the next one
            m = ms[g]
            with torch.cuda.stream(self.readback):
                self.readback.wait_event(self.done[g % 2])
                info = m.info.to("cpu", non_blocking=True)
                self.readback.synchronize()
                info = info.numpy()
                host = []
                for i in range(len(groups[g])):
                    n, status = int(info[i, 0]), int(info[i, 1])
                    if status != _lib.KS_OK:
                        raise _lib.KilosortB200Error(status, f"stream: batch {groups[g][i]}: "
                                                     f"device status {status}")
                    host.append((m.outs[i].st[:n].to("cpu", non_blocking=True),
                                 m.outs[i].amps[:n].to("cpu", non_blocking=True)))
                self.readback.synchronize()
            for i, b in enumerate(groups[g]):
                st_h = host[i][0].numpy()
                a = host[i][1]
                # padded-batch sample -> recording sample, as kilosort/template_matching.py:103
                # computes it before aligning to nt0min
                times.append(st_h[:, 0] - self.nt + b * self.NT)
                templ.append(st_h[:, 1])
                amps.append(a.reshape(-1).cpu().numpy())
                bidx.append(np.full(len(st_h), b, dtype=np.int64))
            if self.refine_every and (g + 1) % self.refine_every == 0:
                self._refine(m)

        if groups:
            self._enqueue_copy(0, groups[0])
        for g, batches in enumerate(groups):
            if g + 1 < len(groups):
                self._enqueue_copy(g + 1, groups[g + 1])
            self._enqueue_match(g, batches, ms[g])
            if g >= 1:
                collect(g - 1)
        if groups:
            collect(len(groups) - 1)
        code, _ = self.whiten.status()
        if code != _lib.KS_OK:
            raise _lib.KilosortB200Error(code, f"stream: whitening device status {code}")
        cat = (lambda xs, dt: np.concatenate(xs).astype(dt) if xs else np.zeros(0, dt))
        return (cat(times, np.int64), cat(templ, np.int64), cat(amps, np.float32),
                cat(bidx, np.int64))
