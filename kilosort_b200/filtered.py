"""Device batch source for the reference's filtered binary file.

The reference's ``extract`` reads each padded batch with
``bfile.padded_batch_to_torch(ibatch, ops)`` (kilosort/template_matching.py:83).
On a ``BinaryFiltered`` (kilosort/io.py:968-1045) that is the raw window of
``BinaryRWFile.padded_batch_to_torch`` (io.py:789-831: a numpy slice of the
file, transposed, copied to the device and converted to float32, its edges
repeated for the first and last batch) followed by ``filter`` (io.py:990-1026:
channel map, sign, mean, common average reference, Fourier-domain high-pass,
artifact zeroing, whitening with the batch's drift matrix).

``FilteredBatches`` makes the same batch from the same object on the device:

* the window is cut from ``bfile.file`` straight into pinned host memory in the
  file's own ``[samples, channels]`` layout (no transpose), on a few host
  threads;
* it crosses to the device as int16 (half the bytes of float32), from pinned
  memory, on the caller's stream;
* one ``ks_preprocess_int16`` call filters it, with the drift matrix of
  kilosort/preprocessing.py:44-69 (``drift_matrix``) folded into the
  whitening matrix as the reference folds it (``(M @ whiten_mat) @ X``).

It serves files whose samples are int16, or uint16 (shifted by 2**15 exactly
as io.py:796-799 does, which in int16 is the top bit flipped), without
``scale`` or ``shift``; `supports` says whether a file qualifies, and `extract`
falls back to ``bfile.padded_batch_to_torch`` when it does not.
"""
from __future__ import annotations

import threading
import weakref
from concurrent.futures import ThreadPoolExecutor
from typing import Optional

import numpy as np
import torch

from . import _lib
from .preprocess import Preprocessor
from .template_matching import to_host

# attributes of the reference's BinaryFiltered (io.py:569-659, 968-988) that
# the device path reads
_ATTRS = ("file", "_get_batch_edges", "NT", "nt", "n_chan_bin", "n_batches",
          "batch_downsampling", "chan_map", "hp_filter", "whiten_mat", "do_CAR",
          "invert_sign", "artifact_threshold")
_COPY_ROWS = 8192          # rows per host copy task


def _dtype_name(bfile) -> str:
    try:
        return str(np.dtype(getattr(bfile, "dtype", "int16")))
    except TypeError:
        return ""


def supports(bfile) -> bool:
    """True when ``bfile`` has the members of the reference's ``BinaryFiltered``
    and holds int16 or uint16 samples with neither ``scale`` nor ``shift``
    (io.py:801-804 makes such batches float32 on the host)."""
    if not all(hasattr(type(bfile), a) or hasattr(bfile, a) for a in _ATTRS):
        return False
    if getattr(bfile, "scale", None) is not None or getattr(bfile, "shift", None) is not None:
        return False
    return _dtype_name(bfile) in ("int16", "uint16")


def drift_matrix(ops, dshift, device) -> torch.Tensor:
    """The drift-correction matrix of one batch, as kilosort/preprocessing.py:44-69
    forms it: the batch's shifts (one per block; with several blocks,
    interpolated linearly to every channel's depth and extrapolated past the
    ends, scipy ``interp1d``), the channel positions moved up by them, a
    Gaussian kernel of width ``sig_interp`` between moved and original
    positions (kernel2D_torch, :37-41), times ``ops['iKxx']``.  Computed with
    the same torch operations on ``device``, in the dtype of the probe
    coordinates (float32 for a loaded probe)."""
    if ops["nblocks"] == 1:
        shifts = dshift
    else:
        from scipy.interpolate import interp1d
        shifts = interp1d(ops["yblk"], dshift, fill_value="extrapolate",
                          kind="linear")(ops["probe"]["yc"])
    pos = np.vstack((ops["probe"]["xc"], ops["probe"]["yc"])).T
    moved = pos.copy()
    moved[:, 1] -= shifts
    # pinned, non-blocking: a pageable copy would wait for the device in the
    # driver while the batch reader prepares the next batch
    pos_t = _to_device(pos, device)
    moved_t = _to_device(moved, device)
    sig = ops["settings"]["sig_interp"]
    d2 = ((moved_t.unsqueeze(1) - pos_t) ** 2).sum(-1)
    return torch.exp(-d2 / (2 * sig ** 2)) @ torch.as_tensor(ops["iKxx"]).to(device)


def _to_device(a: np.ndarray, device) -> torch.Tensor:
    t = torch.from_numpy(np.ascontiguousarray(a))
    if torch.device(device).type != "cuda":
        return t
    return t.pin_memory().to(device, non_blocking=True)


def padded_window(bfile, ibatch: int, out: np.ndarray, copy=None) -> np.ndarray:
    """The raw samples of padded batch ``ibatch`` in ``out`` [NT + 2nt, n_chan_bin]
    int16, as io.py:789-824 lays them out before the float conversion.

    The batch index is scaled by ``batch_downsampling`` and its edges come from
    the file's own ``_get_batch_edges`` (io.py:771-783).  The first batch puts
    its samples after ``nt`` copies of its first sample and leaves the rest
    zero; the batch whose scaled index is ``n_batches - 1`` repeats its last
    sample to the end; any other batch must fill the window (the reference
    fails there too).  uint16 samples are stored as ``u - 2**15``.
    ``copy(dst, src)`` moves the samples (default: one numpy copy).
    """
    NT, nt = int(bfile.NT), int(bfile.nt)
    L = NT + 2 * nt
    if out.shape[0] != L or out.dtype != np.int16:
        raise ValueError(f"window buffer must be int16 with {L} rows")
    ib = int(ibatch) * int(bfile.batch_downsampling)
    bstart, bend = bfile._get_batch_edges(ib)
    data = bfile.file[bstart:bend]
    n = int(data.shape[0])
    put = copy if copy is not None else _copy_samples
    if ib == 0:
        if n > L - nt:
            raise ValueError(f"first batch holds {n} samples, more than {L - nt}")
        if n:
            put(out[nt:nt + n], data)
            out[:nt] = out[nt]
        else:
            out[:nt] = 0
        out[nt + n:] = 0
    elif ib == int(bfile.n_batches) - 1:
        if n == 0 or n > L:
            raise ValueError(f"last batch holds {n} samples, expected 1..{L}")
        put(out[:n], data)
        out[n:] = out[n - 1]
    else:
        if n != L:
            raise ValueError(f"batch {ib} holds {n} samples, expected {L}")
        put(out, data)
    return out


def _copy_samples(dst: np.ndarray, src) -> None:
    if src.dtype == np.uint16:
        np.bitwise_xor(src, np.uint16(0x8000), out=dst.view(np.uint16))
    elif src.dtype == np.int16:
        np.copyto(dst, src)
    else:
        raise TypeError(f"samples of type {src.dtype} need the file's own batch reader")


class FilteredBatches:
    """Filtered padded batches ``[C, NT + 2nt]`` float32 of a ``BinaryFiltered``
    on ``device`` (see the module docstring).

    ``batch(ibatch, ops)`` enqueues the copy and the filter on the current
    stream and returns the batch tensor; ``check()`` synchronises with the
    last filter and raises if the device reported an error.  Two pinned
    windows and two device copies of them alternate, so the host cuts the
    next window while the previous one crosses to the device; a window is
    rewritten only after its copy has finished, and its device copy only after
    the filter that read it.
    """

    def __init__(self, bfile, device, copy_threads: int = 4, ntaps: int = 1023):
        if not supports(bfile):
            raise ValueError("the batch source is not an int16/uint16 BinaryFiltered "
                             "without scale or shift")
        self.bfile = bfile
        self.device = torch.device(device)
        if self.device.type != "cuda":
            raise ValueError("FilteredBatches runs on a CUDA device")
        self.signature = _signature(bfile)
        self.NT, self.nt = int(bfile.NT), int(bfile.nt)
        self.L = self.NT + 2 * self.nt
        self.n_chan_bin = int(bfile.n_chan_bin)
        whiten = bfile.whiten_mat
        if whiten is not None:
            whiten = torch.as_tensor(whiten).detach().to(self.device, torch.float32).clone()
        self.whiten = whiten
        self.pre = Preprocessor(self.n_chan_bin, self.L, whiten=whiten,
                                chan_map=bfile.chan_map, hp_filter=bfile.hp_filter,
                                do_CAR=bool(bfile.do_CAR), invert_sign=bool(bfile.invert_sign),
                                artifact_threshold=float(bfile.artifact_threshold),
                                device=self.device, ntaps=ntaps)
        self.C = self.pre.C
        self.host = [torch.empty((self.L, self.n_chan_bin), dtype=torch.int16).pin_memory()
                     for _ in range(2)]
        self.raw = [torch.empty((self.L, self.n_chan_bin), dtype=torch.int16, device=self.device)
                    for _ in range(2)]
        self.copied = [None, None]               # events: copy out of host[i] done
        self.used = [None, None]                 # events: filter of raw[i] done
        self.slot = 0
        # the largest device status of every batch filtered since the last check
        self.sticky = torch.zeros(1, dtype=torch.int32, device=self.device)
        self.pool = ThreadPoolExecutor(copy_threads, thread_name_prefix="ks-window") \
            if copy_threads > 1 else None

    def _copy(self, dst: np.ndarray, src) -> None:
        n = src.shape[0]
        if self.pool is None or n < 2 * _COPY_ROWS:
            _copy_samples(dst, src)
            return
        edges = list(range(0, n, _COPY_ROWS)) + [n]
        jobs = [self.pool.submit(_copy_samples, dst[a:b], src[a:b])
                for a, b in zip(edges[:-1], edges[1:])]
        for j in jobs:
            j.result()

    def _drift(self, ops, ibatch) -> Optional[torch.Tensor]:
        # io.py:1019-1023: the drift matrix needs whitening, dshift and ops
        dshift = getattr(self.bfile, "dshift", None)
        if self.whiten is None or dshift is None or ops is None:
            return None
        return drift_matrix(ops, dshift[int(ibatch)], self.device).to(torch.float32)

    def batch(self, ibatch: int, ops=None, out: Optional[torch.Tensor] = None) -> torch.Tensor:
        i = self.slot
        self.slot ^= 1
        if self.copied[i] is not None:
            self.copied[i].synchronize()
        padded_window(self.bfile, ibatch, self.host[i].numpy(), copy=self._copy)
        stream = torch.cuda.current_stream(self.device)
        if self.used[i] is not None:
            stream.wait_event(self.used[i])
        self.raw[i].copy_(self.host[i], non_blocking=True)
        self.copied[i] = torch.cuda.Event()
        self.copied[i].record(stream)
        if out is None:
            out = torch.empty((self.C, self.L), dtype=torch.float32, device=self.device)
        X = self.pre(self.raw[i], out, drift=self._drift(ops, ibatch))
        torch.maximum(self.sticky, self.pre.flags[:1], out=self.sticky)
        self.used[i] = torch.cuda.Event()
        self.used[i].record(stream)
        return X

    def check(self) -> None:
        """Raise if any batch filtered since the last check reported an error
        (synchronises with the last one).  Call it when no batch is being
        filtered on another stream: the status word is cleared here."""
        status = int(to_host(self.sticky)[0][0])
        self.sticky.zero_()
        if status != _lib.KS_OK:
            raise _lib.KilosortB200Error(
                status, f"ks_preprocess_int16: device status {_lib.status_message(status)}")

    def close(self) -> None:
        if self.pool is not None:
            self.pool.shutdown(wait=True)
            self.pool = None


def _tensor_key(t):
    if t is None:
        return None
    if torch.is_tensor(t):
        return ("tensor", id(t), t._version)
    a = np.asarray(t)
    return ("array", a.dtype.str, a.shape, a.tobytes())


def _signature(bfile):
    """What the device filter is built from: a file whose settings differ (a
    new or changed channel map, filter or whitening tensor, other flags or
    sizes) gets a new FilteredBatches."""
    return (int(bfile.NT), int(bfile.nt), int(bfile.n_chan_bin), _dtype_name(bfile),
            _tensor_key(bfile.chan_map), _tensor_key(bfile.hp_filter),
            _tensor_key(bfile.whiten_mat), bool(bfile.do_CAR), bool(bfile.invert_sign),
            float(bfile.artifact_threshold))


_cache = weakref.WeakKeyDictionary()
_cache_lock = threading.Lock()


def batches_for(bfile, device) -> FilteredBatches:
    """The FilteredBatches of ``bfile`` on ``device``, kept with the file object
    (weakly) and reused while its settings are unchanged, so repeated
    `extract` calls on one file keep their pinned windows and filter state."""
    device = torch.device(device)
    sig = _signature(bfile)
    with _cache_lock:
        try:
            per_dev = _cache.setdefault(bfile, {})
        except TypeError:                 # not weakly referenceable: no reuse
            return FilteredBatches(bfile, device)
        fb = per_dev.get(device)
        if fb is None or fb.signature != sig:
            if fb is not None:
                fb.close()
            fb = per_dev[device] = FilteredBatches(bfile, device)
        return fb
