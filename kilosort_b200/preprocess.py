"""Preprocessing of raw int16 batches on the device.

The filter kilosort/io.py:994-1026 (``BinaryFiltered.filter``) applies to each
padded batch -- channel map, sign inversion, per-channel mean removal, common
average reference, high-pass, artifact zeroing, whitening (with the drift
matrix of kilosort/preprocessing.py:44-69 folded in) -- as one call of
``ks_preprocess_int16``.

The reference high-passes in the Fourier domain over the whole batch
(kilosort/preprocessing.py:138-154 pads or crops its filter to the batch
length, io.py:1008-1010 multiplies by the conjugate spectrum and shifts by half
a batch), which is a circular correlation with the filter; the device computes
that correlation directly with the filter's centre taps (``highpass_taps``).
"""
from __future__ import annotations

import math
from typing import Optional

import numpy as np
import torch

from . import _lib
from .template_matching import _stream, to_host


def _ptr(t) -> int:
    return 0 if t is None else t.data_ptr()


def highpass_filter(fs: float = 30000, cutoff: float = 300) -> torch.Tensor:
    """The reference's time-domain high-pass (kilosort/preprocessing.py:121-136):
    the response of a 3rd-order Butterworth high-pass run forwards and
    backwards (scipy ``filtfilt``) to a unit impulse at the centre of 30122
    samples, float32."""
    from scipy.signal import butter, filtfilt
    n = 30122
    b, a = butter(3, cutoff, fs=fs, btype="high")
    x = np.zeros(n)
    x[n // 2] = 1
    return torch.from_numpy(filtfilt(b, a, x).copy()).float()


def highpass_taps(hp_filter, L: int, ntaps: int = 1023):
    """(taps float32 [n], centre): X'[n] = sum_j taps[j] X[(n + j - centre) mod L].

    ``hp_filter`` is the reference's time-domain filter (odd or even length,
    centred at len // 2, kilosort/preprocessing.py:121-136).  Padding or
    cropping it to L samples (preprocessing.py:144-153) puts its centre at
    ``cpos``; the half-batch shift then reads sample n + d + (cpos - L//2) for
    the tap at distance d.  At most ``ntaps`` taps are kept, and no more than
    the padded or cropped filter holds on either side of its centre.
    """
    h = hp_filter.detach().double().cpu().numpy() if torch.is_tensor(hp_filter) \
        else np.asarray(hp_filter, np.float64)
    ft = h.shape[0]
    if ft < L:
        cpos = (L - ft) // 2 + ft // 2
    elif ft > L:
        cpos = ft // 2 - (ft - L) // 2
    else:
        cpos = ft // 2
    half = min(ntaps // 2, cpos, L - 1 - cpos)
    c = ft // 2
    taps = np.zeros(2 * half + 1)
    lo, hi = max(0, c - half), min(ft, c + half + 1)
    taps[lo - (c - half):hi - (c - half)] = h[lo:hi]
    return taps.astype(np.float32), half - (cpos - L // 2)


class Preprocessor:
    """Device preprocessing of padded raw batches of one length.

    raw batches are int16 ``[L, n_chan_bin]`` device tensors (the file's
    layout); the output is ``[C, L]`` float32 with C = len(chan_map).
    """

    def __init__(self, n_chan_bin: int, L: int, whiten: Optional[torch.Tensor] = None,
                 chan_map=None, hp_filter=None, do_CAR: bool = True,
                 invert_sign: bool = False, artifact_threshold: float = math.inf,
                 device=None, ntaps: int = 1023):
        self.device = torch.device(device) if device is not None else torch.device("cuda")
        self.n_chan_bin, self.L = int(n_chan_bin), int(L)
        if chan_map is None:
            self.chan_map = None
            self.C = self.n_chan_bin
        else:
            cm = torch.as_tensor(np.asarray(chan_map), dtype=torch.int64)
            self.chan_map = cm.to(self.device).contiguous()
            self.C = int(cm.numel())
        self.whiten = None if whiten is None else \
            torch.as_tensor(whiten, dtype=torch.float32).to(self.device).contiguous()
        if self.whiten is not None and tuple(self.whiten.shape) != (self.C, self.C):
            raise ValueError(f"whitening matrix must be {self.C} x {self.C}")
        if hp_filter is not None:
            taps, self.centre = highpass_taps(hp_filter, self.L, ntaps)
            self.taps = torch.from_numpy(taps).to(self.device)
        else:
            self.taps, self.centre = None, 0
        self.do_CAR, self.invert_sign = bool(do_CAR), bool(invert_sign)
        self.artifact_threshold = float(artifact_threshold)
        lib = _lib.load()
        self.ws = torch.empty(lib.ks_preprocess_workspace_size(self.L, self.C,
                                                               int(self.whiten is not None)),
                              dtype=torch.uint8, device=self.device)
        self.flags = torch.zeros(2, dtype=torch.int32, device=self.device)

    def __call__(self, raw: torch.Tensor, X: Optional[torch.Tensor] = None,
                 drift: Optional[torch.Tensor] = None) -> torch.Tensor:
        if raw.dtype != torch.int16 or raw.dim() != 2 or raw.shape[0] != self.L \
                or raw.shape[1] < self.n_chan_bin or raw.stride(1) != 1:
            raise ValueError(f"raw must be an int16 [{self.L}, {self.n_chan_bin}] row-major tensor")
        if X is None:
            X = torch.empty((self.C, self.L), dtype=torch.float32, device=self.device)
        W = self.whiten
        if drift is not None:
            if W is None:
                raise ValueError("a drift matrix needs a whitening matrix")
            W = (torch.as_tensor(drift, dtype=torch.float32, device=self.device) @ W).contiguous()
        lib = _lib.load()
        _lib.check(lib.ks_preprocess_int16(
            _ptr(raw), self.L, raw.stride(0), _ptr(self.chan_map), self.C,
            int(self.invert_sign), int(self.do_CAR), _ptr(self.taps),
            0 if self.taps is None else self.taps.numel(), self.centre,
            self.artifact_threshold, _ptr(W), _ptr(X), X.stride(0), _ptr(self.flags),
            _ptr(self.ws), self.ws.numel(), _stream(self.device)), "ks_preprocess_int16")
        return X

    def status(self):
        """(device status, artifact) of the last call (synchronises)."""
        f = to_host(self.flags)[0].tolist()
        return int(f[0]), bool(f[1])


def filter_batch(raw: torch.Tensor, **kw) -> torch.Tensor:
    """One padded raw batch [L, n_chan_bin] int16 -> [C, L] float32."""
    p = Preprocessor(raw.shape[1], raw.shape[0], device=raw.device, **kw)
    X = p(raw)
    status, _ = p.status()
    if status != _lib.KS_OK:
        raise _lib.KilosortB200Error(status, f"ks_preprocess_int16: device status {status}")
    return X
