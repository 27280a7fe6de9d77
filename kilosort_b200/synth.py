"""Seeded synthetic recordings for the template-matching hot path.

The reference measures `run_matching` / `extract` on real Neuropixels data that
is not available offline, so every test and benchmark here runs on recordings
drawn from one explicit generative model:

* probe geometry: a linear probe at 20 um pitch, or a Neuropixels-1.0-like
  probe with four staggered columns (x in {43, 11, 59, 27} um, two contacts per
  20 um row);
* each unit has a biphasic waveform (negative unit trough at sample
  ``t_trough`` = 20, positive lobe ~12 samples = 0.4 ms later, per-unit shape
  jitter), a Gaussian spatial footprint (sigma 30 um) around a continuously
  drawn site, and an amplitude in standard deviations of the noise;
* the temporal basis ``wPCA`` is the top ``n_pcs`` right singular vectors of
  5000 unit-norm waveforms drawn from the same shape distribution (the
  reference learns it the same way from detected clips,
  kilosort/spikedetect.py:57-78);
* the spatial components are the templates projected on that basis,
  ``U[k, p, c] = sum_t T_k[c, t] * wPCA[p, t]``;
* the whitened signal is N(0, 1) float32 noise plus every spike's template
  added at its trough time; units fire as Poisson trains with a refractory
  period of ``nt`` samples.

Template pairs whose projected templates have cosine similarity above
``max_cos`` are redrawn: (near-)proportional templates tie in the
``relu(B)^2 / |U|^2`` score and make the argmax over templates depend on
rounding, which real pipelines avoid by merging such units
(kilosort/template_matching.py:144-152).

All randomness comes from ``numpy.random.default_rng(seed)`` streams, so a
recording is identical on every machine with the same numpy build.
"""
from __future__ import annotations

import dataclasses
from typing import List, Optional, Sequence

import numpy as np

__all__ = [
    "Recording",
    "probe_geometry",
    "make_recording",
    "config_recording",
    "CONFIGS",
    "raw_recording",
    "FilteredBinary",
]


def probe_geometry(kind: str, n_chan: int):
    """Contact coordinates (xc, yc) in um as float64 arrays."""
    idx = np.arange(n_chan)
    if kind == "linear":
        xc = np.zeros(n_chan)
        yc = 20.0 * idx
    elif kind == "np1":
        xc = np.array([43.0, 11.0, 59.0, 27.0])[idx % 4]
        yc = 20.0 * (idx // 2)
    else:
        raise ValueError(f"unknown probe kind {kind!r}")
    return xc.astype(np.float64), yc.astype(np.float64)


def _waveforms(rng, n, nt, t_trough, shift_sd=0.0):
    """Biphasic unit-trough waveforms, one per row, shape [n, nt] float64."""
    t = np.arange(nt, dtype=np.float64)[None, :]
    s1 = rng.uniform(1.2, 2.2, size=(n, 1))
    s2 = rng.uniform(3.0, 6.0, size=(n, 1))
    r = rng.uniform(0.2, 0.6, size=(n, 1))
    d = rng.uniform(10.0, 14.0, size=(n, 1))
    t0 = t_trough + (rng.normal(0.0, shift_sd, size=(n, 1)) if shift_sd else 0.0)
    w = -np.exp(-((t - t0) ** 2) / (2 * s1 ** 2)) \
        + r * np.exp(-((t - t0 - d) ** 2) / (2 * s2 ** 2))
    w /= -w.min(axis=1, keepdims=True)
    return w


def _basis(rng, nt, n_pcs, t_trough, n_wave=5000):
    """Top ``n_pcs`` right singular vectors of unit-norm jittered waveforms."""
    w = _waveforms(rng, n_wave, nt, t_trough, shift_sd=1.0)
    w /= np.sqrt((w ** 2).sum(1, keepdims=True))
    _, _, vt = np.linalg.svd(w, full_matrices=False)
    basis = vt[:n_pcs].copy()
    # fix the sign convention: the largest-magnitude entry of each row is positive
    sgn = np.sign(basis[np.arange(n_pcs), np.abs(basis).argmax(1)])
    return (basis * sgn[:, None]).astype(np.float32)


@dataclasses.dataclass
class Recording:
    """A synthetic recording cut into padded batches.

    ``batch(b)`` returns the padded batch ``[C, NT_b + 2*nt]`` float32 that
    `run_matching` consumes; ``batch_lengths`` holds the unpadded ``NT_b``.
    """

    xc: np.ndarray
    yc: np.ndarray
    wPCA: np.ndarray          # [P, nt] float32, orthonormal rows
    U: np.ndarray             # [K, P, C] float32
    templates: np.ndarray     # [K, C, nt] float32 (before projection)
    spike_times: np.ndarray   # int64 trough sample in the continuous signal
    spike_units: np.ndarray   # int64
    batch_starts: np.ndarray  # first unpadded sample of each batch
    batch_lengths: np.ndarray
    nt: int
    signal: np.ndarray        # [C, total] float32 continuous whitened signal
    min_one_minus_cos: float

    @property
    def n_chan(self):
        return self.U.shape[2]

    @property
    def n_templates(self):
        return self.U.shape[0]

    @property
    def n_batches(self):
        return len(self.batch_lengths)

    def batch(self, b: int) -> np.ndarray:
        s = int(self.batch_starts[b])
        n = int(self.batch_lengths[b])
        return self.signal[:, s: s + n + 2 * self.nt]


def make_recording(
    seed: int,
    n_chan: int = 96,
    probe: str = "linear",
    n_templates: int = 80,
    batch_lengths: Sequence[int] = (60000,),
    nt: int = 61,
    n_pcs: int = 6,
    t_trough: int = 20,
    rate_hz=(5.0, 5.0),
    amp_sd=(8.0, 25.0),
    fs: float = 30000.0,
    sigma_um: float = 30.0,
    max_cos: float = 0.99,
    duplicate_pairs: int = 0,
) -> Recording:
    """Draw one recording.

    ``duplicate_pairs`` > 0 copies that many templates exactly onto other
    template slots (ties in the score, used to pin argmax tie-breaking).
    """
    root = np.random.SeedSequence(seed)
    s_geom, s_basis, s_units, s_trains, s_noise = root.spawn(5)
    xc, yc = probe_geometry(probe, n_chan)
    wPCA = _basis(np.random.default_rng(s_basis), nt, n_pcs, t_trough)
    rng = np.random.default_rng(s_units)

    K = n_templates
    xlo, xhi = xc.min(), xc.max()
    ylo, yhi = yc.min(), yc.max()

    def draw(n):
        sx = rng.uniform(xlo, xhi, size=n)
        sy = rng.uniform(ylo, yhi, size=n)
        w = _waveforms(rng, n, nt, t_trough)
        a = rng.uniform(amp_sd[0], amp_sd[1], size=n)
        d2 = (xc[None, :] - sx[:, None]) ** 2 + (yc[None, :] - sy[:, None]) ** 2
        sp = np.exp(-d2 / (2 * sigma_um ** 2))
        T = (a[:, None, None] * sp[:, :, None] * w[:, None, :]).astype(np.float32)
        return T

    def project(T):
        # U[k,p,c] = sum_t T[k,c,t] W[p,t]
        return np.einsum("kct,pt->kpc", T.astype(np.float64),
                         wPCA.astype(np.float64)).astype(np.float32)

    T = draw(K)
    U = project(T)
    # redraw units whose projected template is too similar to an earlier one
    for _ in range(50):
        f = U.reshape(K, -1).astype(np.float64)
        f = f / np.linalg.norm(f, axis=1, keepdims=True)
        cos = f @ f.T
        np.fill_diagonal(cos, -1.0)
        bad = np.unique(np.nonzero(np.triu(cos > max_cos))[1])
        if len(bad) == 0:
            break
        T[bad] = draw(len(bad))
        U[bad] = project(T[bad])
    f = U.reshape(K, -1).astype(np.float64)
    f = f / np.linalg.norm(f, axis=1, keepdims=True)
    cos = f @ f.T
    np.fill_diagonal(cos, -1.0)
    min_one_minus_cos = float(1.0 - cos.max()) if K > 1 else 1.0

    if duplicate_pairs:
        for i in range(duplicate_pairs):
            T[K - 1 - i] = T[i]
            U[K - 1 - i] = U[i]
        min_one_minus_cos = 0.0

    lengths = np.asarray(batch_lengths, dtype=np.int64)
    starts = np.concatenate([[0], np.cumsum(lengths)[:-1]]).astype(np.int64)
    total = int(lengths.sum()) + 2 * nt

    # Poisson trains with an nt-sample refractory period
    trng = np.random.default_rng(s_trains)
    rates = trng.uniform(rate_hz[0], rate_hz[1], size=K)
    times, units = [], []
    lo, hi = t_trough, total - (nt - t_trough)
    for k in range(K):
        mean_isi = fs / rates[k]
        n_draw = int((hi - lo) / mean_isi * 1.5) + 16
        isi = nt + trng.exponential(max(mean_isi - nt, 1.0), size=n_draw)
        t = lo + np.floor(np.cumsum(isi)).astype(np.int64)
        t = t[t < hi]
        times.append(t)
        units.append(np.full(len(t), k, dtype=np.int64))
    spike_times = np.concatenate(times) if times else np.zeros(0, np.int64)
    spike_units = np.concatenate(units) if units else np.zeros(0, np.int64)
    order = np.argsort(spike_times, kind="stable")
    spike_times, spike_units = spike_times[order], spike_units[order]

    nrng = np.random.default_rng(s_noise)
    signal = nrng.standard_normal((n_chan, total), dtype=np.float32)
    tw = np.arange(nt)
    for k in range(K):
        tk = times[k]
        if len(tk) == 0:
            continue
        chans = np.nonzero(np.abs(T[k]).max(1) > 0)[0]
        if len(chans) == 0:
            continue
        idx = (tk[:, None] - t_trough + tw[None, :])          # [n, nt]
        sub = signal[np.ix_(chans, idx.ravel())].reshape(len(chans), len(tk), nt)
        sub += T[k][chans][:, None, :]
        signal[np.ix_(chans, idx.ravel())] = sub.reshape(len(chans), -1)

    return Recording(xc=xc, yc=yc, wPCA=wPCA, U=U, templates=T,
                     spike_times=spike_times, spike_units=spike_units,
                     batch_starts=starts, batch_lengths=lengths, nt=nt,
                     signal=signal, min_one_minus_cos=min_one_minus_cos)


# The measurement workloads.  Seeds follow numpy.random.default_rng(1000 + i).
CONFIGS = {
    1: dict(n_chan=96, probe="linear", n_templates=80, n_batches=10,
            rate_hz=(5.0, 5.0), amp_sd=(8.0, 25.0)),
    2: dict(n_chan=384, probe="np1", n_templates=600, n_batches=20,
            rate_hz=(2.0, 15.0), amp_sd=(6.0, 30.0)),
    4: dict(n_chan=384, probe="np1", n_templates=600, n_batches=1,
            rate_hz=(5.0, 37.0), amp_sd=(6.0, 30.0)),      # ~25000 spikes per batch
    5: dict(n_chan=384, probe="np1", n_templates=2000, n_batches=1800,
            rate_hz=(1.0, 30.0), amp_sd=(5.0, 40.0)),
}


def config_recording(cfg: int, n_batches: Optional[int] = None,
                     batch_size: int = 60000, n_templates: Optional[int] = None,
                     n_chan: Optional[int] = None) -> Recording:
    """Recording for one of the numbered workloads (optionally truncated)."""
    c = dict(CONFIGS[cfg])
    nb = c.pop("n_batches")
    if n_batches is not None:
        nb = n_batches
    if n_templates is not None:
        c["n_templates"] = n_templates
    if n_chan is not None:
        c["n_chan"] = n_chan
    return make_recording(1000 + cfg, batch_lengths=[batch_size] * nb, **c)


def uneven_recordings(seed: int = 1003, n_batches_total: int = 200,
                      lo: int = 8000, hi: int = 60000) -> List[Recording]:
    """Three recordings with uneven batch lengths (96/150, 384/600, 384/1000).

    Batch lengths are drawn uniformly from [lo, hi]; the last batch of each
    recording is a short tail.
    """
    rng = np.random.default_rng(seed)
    specs = [
        dict(n_chan=96, probe="linear", n_templates=150, rate_hz=(5.0, 5.0),
             amp_sd=(8.0, 25.0)),
        dict(n_chan=384, probe="np1", n_templates=600, rate_hz=(2.0, 15.0),
             amp_sd=(6.0, 30.0)),
        dict(n_chan=384, probe="np1", n_templates=1000, rate_hz=(2.0, 15.0),
             amp_sd=(6.0, 30.0)),
    ]
    counts = [n_batches_total // 3 + (1 if i < n_batches_total % 3 else 0)
              for i in range(3)]
    recs = []
    for i, (spec, nb) in enumerate(zip(specs, counts)):
        lengths = rng.integers(lo, hi + 1, size=nb)
        lengths[-1] = max(lo // 2, int(lengths[-1]) // 4)
        recs.append(make_recording(seed * 10 + i, batch_lengths=lengths, **spec))
    return recs


class SyntheticBinary:
    """Batch source with the duck type `extract` expects of a binary file.

    Mirrors the three members of the reference's ``BinaryFiltered`` that
    kilosort/template_matching.py:73,83,102 use: ``n_batches``,
    ``batch_downsampling`` and ``padded_batch_to_torch(ibatch, ops)``, which
    returns the padded batch ``[C, NT + 2*nt]`` as a float32 tensor on
    ``device``.
    """

    def __init__(self, rec: Recording, device="cpu"):
        if len(set(int(n) for n in rec.batch_lengths)) != 1:
            raise ValueError("extract needs equal batch lengths")
        self.rec = rec
        self.n_batches = rec.n_batches
        self.batch_downsampling = 1
        self.device = device

    def padded_batch_to_torch(self, ibatch, ops=None):
        import torch
        x = np.ascontiguousarray(self.rec.batch(int(ibatch)))
        return torch.from_numpy(x).to(self.device)


def raw_batch(seed: int, n_chan_bin: int, L: int, fs: float = 30000.0,
              n_spikes: int = 40) -> np.ndarray:
    """A raw int16 batch in the file layout [L, n_chan_bin], with what the
    preprocessing removes: per-channel offsets (-500..500), a slow per-channel
    drift (1-8 Hz, amplitude 20-120), a common-mode signal on every channel
    (amplitude 60, 50 Hz plus noise), white noise (sd 20) and negative spikes
    (amplitude 80-300, trough 0.3 ms wide, on 3 neighbouring channels)."""
    rng = np.random.default_rng(seed)
    t = np.arange(L) / fs
    off = rng.uniform(-500, 500, n_chan_bin)
    f_drift = rng.uniform(1, 8, n_chan_bin)
    a_drift = rng.uniform(20, 120, n_chan_bin)
    ph = rng.uniform(0, 2 * np.pi, n_chan_bin)
    common = 60 * np.sin(2 * np.pi * 50 * t) + 15 * rng.standard_normal(L)
    x = (off[None, :] + a_drift[None, :] * np.sin(2 * np.pi * f_drift[None, :] * t[:, None]
                                                   + ph[None, :])
         + common[:, None] + 20 * rng.standard_normal((L, n_chan_bin)))
    w = np.exp(-0.5 * ((np.arange(-15, 16)) / 4.5) ** 2)
    for _ in range(n_spikes):
        s = int(rng.integers(20, max(21, L - 20)))
        c = int(rng.integers(0, n_chan_bin))
        a = rng.uniform(80, 300)
        for dc, g in ((-1, 0.5), (0, 1.0), (1, 0.5)):
            cc = c + dc
            if 0 <= cc < n_chan_bin:
                lo, hi = max(0, s - 15), min(L, s + 16)
                x[lo:hi, cc] -= a * g * w[lo - (s - 15):hi - (s - 15)]
    return np.clip(np.round(x), -32768, 32767).astype(np.int16)


def raw_recording(rec: Recording, n_chan_bin: int, chan_map, seed: int, gain: float = 25.0,
                  fs: float = 30000.0, chunk: int = 65536) -> np.ndarray:
    """The whole of ``rec`` as a raw int16 file ``[T, n_chan_bin]``.

    Every file channel carries what preprocessing removes (as in `raw_batch`,
    but continuous over the recording: a per-channel offset, a slow sinusoidal
    drift, a common-mode 50 Hz signal with noise, white noise of sd 20); the
    channels ``chan_map`` (in order) add ``round(gain * rec.signal)``, so a
    whitening matrix ``eye / gain`` brings the signal back to its scale.
    Generated in chunks of ``chunk`` samples in float32.
    """
    chan_map = np.asarray(chan_map)
    if len(chan_map) != rec.n_chan:
        raise ValueError("chan_map must name one file channel per recording channel")
    T = rec.signal.shape[1]
    rng = np.random.default_rng(seed)
    off = rng.uniform(-500, 500, n_chan_bin).astype(np.float32)
    f_drift = rng.uniform(1, 8, n_chan_bin)
    a_drift = rng.uniform(20, 120, n_chan_bin).astype(np.float32)
    ph = rng.uniform(0, 2 * np.pi, n_chan_bin)
    out = np.empty((T, n_chan_bin), np.int16)
    for s in range(0, T, chunk):
        e = min(T, s + chunk)
        t = np.arange(s, e) / fs
        x = np.sin(2 * np.pi * f_drift[None, :] * t[:, None] + ph[None, :]).astype(np.float32)
        x *= a_drift
        x += off
        common = 60 * np.sin(2 * np.pi * 50 * t) + 15 * rng.standard_normal(e - s)
        x += common.astype(np.float32)[:, None]
        x += 20 * rng.standard_normal((e - s, n_chan_bin), dtype=np.float32)
        x[:, chan_map] += gain * rec.signal[:, s:e].T
        np.clip(np.round(x), -32768, 32767, out=x)
        out[s:e] = x
    return out


class FilteredBinary:
    """An in-memory stand-in for the reference's ``BinaryFiltered``
    (kilosort/io.py:968-1045) over a raw int16 (or uint16) array
    ``[T, n_chan_bin]``, with ``tmin = 0``, ``tmax = inf``, no scale or shift.

    It has the members a ``BinaryFiltered`` carries and `extract` reads:
    ``file``, ``NT``, ``nt``, ``n_chan_bin``, ``dtype``, the filter settings
    (``chan_map``, ``hp_filter``, ``whiten_mat``, ``dshift``, ``do_CAR``,
    ``invert_sign``, ``artifact_threshold``), ``imin``/``imax``,
    ``n_batches``, ``batch_downsampling`` and ``_get_batch_edges``, with the
    batch count and edges of io.py:646-656 and :771-787: ``ceil(T / NT)``
    batches, the last one dropped (and ``imax`` cut back) when it would hold
    fewer than ``nt`` samples past its left pad; batch 0 covers
    ``[imin, imin + NT + nt)``, batch b ``[imin + b NT - nt,
    min(imax, imin + (b+1) NT + nt))``.  ``padded_batch_to_torch`` filters on
    the device (``filtered.FilteredBatches``).
    """

    def __init__(self, data: np.ndarray, NT: int = 60000, nt: int = 61, chan_map=None,
                 hp_filter=None, whiten_mat=None, dshift=None, do_CAR: bool = True,
                 invert_sign: bool = False, artifact_threshold: float = np.inf,
                 batch_downsampling: int = 1, device="cuda"):
        self.file = data
        self.dtype = str(data.dtype)
        self.NT, self.nt = int(NT), int(nt)
        self.n_chan_bin = int(data.shape[1])
        self.chan_map, self.hp_filter, self.whiten_mat = chan_map, hp_filter, whiten_mat
        self.dshift, self.do_CAR, self.invert_sign = dshift, do_CAR, invert_sign
        self.artifact_threshold = artifact_threshold
        self.scale = self.shift = None
        self.device = device
        self.imin, self.imax = 0, int(data.shape[0])
        self.n_batches_raw = int(np.ceil((self.imax - self.imin) / self.NT))
        a, b = self._get_batch_edges(self.n_batches_raw - 1)
        tail = b - a - self.nt
        if tail < self.nt:
            self.n_batches_raw -= 1
            self.imax -= tail
        self.batch_downsampling = int(batch_downsampling)
        self.n_batches = int(self.n_batches_raw / self.batch_downsampling)
        self._device_batches = None

    def _get_batch_edges(self, ibatch: int):
        if ibatch == 0:
            return self.imin, self.imin + self.NT + self.nt
        start = self.imin + int(ibatch) * self.NT - self.nt
        return start, min(self.imax, start + self.NT + 2 * self.nt)

    def padded_batch_to_torch(self, ibatch: int, ops=None):
        from .filtered import FilteredBatches
        if self._device_batches is None:
            self._device_batches = FilteredBatches(self, self.device, copy_threads=1)
        X = self._device_batches.batch(ibatch, ops)
        self._device_batches.check()
        return X


class TiledSamples:
    """A read-only ``[reps * T, n_chan_bin]`` sample array that repeats ``base``
    ``reps`` times along time, without copying it: a long file for the
    sharded benchmark (every rank's batches hold the same recording).
    Slicing returns a numpy array (a copy where the slice crosses a repeat)."""

    def __init__(self, base: np.ndarray, reps: int):
        self.base = base
        self.reps = int(reps)
        self.dtype = base.dtype
        self.shape = (base.shape[0] * self.reps, base.shape[1])

    def __len__(self):
        return self.shape[0]

    def __getitem__(self, idx):
        if not isinstance(idx, slice) or idx.step not in (None, 1):
            raise TypeError("TiledSamples supports contiguous time slices only")
        start, stop, _ = idx.indices(self.shape[0])
        T = self.base.shape[0]
        if stop <= start:
            return self.base[:0]
        if start // T == (stop - 1) // T:
            o = (start // T) * T
            return self.base[start - o:stop - o]
        parts, s = [], start
        while s < stop:
            o = (s // T) * T
            e = min(stop, o + T)
            parts.append(self.base[s - o:e - o])
            s = e
        return np.concatenate(parts, 0)
