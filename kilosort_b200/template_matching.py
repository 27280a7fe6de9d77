"""Drop-in replacements for ``kilosort.template_matching`` on a B200.

Same signatures, argument meanings, outputs and error behaviour as the
reference functions (kilosort/template_matching.py):

* ``prepare_extract(xc, yc, U, nC, position_limit, device)``   (:14-53)
* ``extract(ops, bfile, U, device, progress_bar)``              (:56-126)
* ``prepare_matching(ops, U)``                                  (:155-167)
* ``run_matching(ops, X, U, ctc, device)``                      (:170-244)

PyTorch only holds device memory and supplies the current CUDA stream; every
computation runs in the sm_100a kernels of ``libks_b200.so``.  There is no CPU
path: inputs must be float32 CUDA tensors on a B200.

Extra ``ops`` keys understood here (the reference ignores them):
``projection`` -- ``"fp32"`` (plain FP32 contraction, the default) or
``"bf16x3"`` (split-BF16 on tensor cores); ``spike_capacity`` -- spike rows
per batch (default 100000, the reference's fixed buffer size);
``read_ahead`` -- `extract` reads the next batch while matching the current
one (default True; set False for a batch source whose
``padded_batch_to_torch`` returns the same buffer on every call).
"""
from __future__ import annotations

import logging
import threading
import weakref

import numpy as np
import torch

from . import _lib

logger = logging.getLogger(__name__)

DEFAULT_CAPACITY = 100000
_PROJECTIONS = {"fp32": _lib.KS_PROJ_FP32, "bf16x3": _lib.KS_PROJ_BF16X3}
_default_projection = "fp32"


def set_default_projection(name: str) -> None:
    """Select the projection used when ``ops`` has no ``projection`` key."""
    global _default_projection
    if name not in _PROJECTIONS:
        raise ValueError(f"projection must be one of {sorted(_PROJECTIONS)}")
    _default_projection = name


def _projection(ops) -> int:
    name = ops.get("projection", _default_projection) if hasattr(ops, "get") else _default_projection
    if name not in _PROJECTIONS:
        raise ValueError(f"ops['projection'] must be one of {sorted(_PROJECTIONS)}")
    return _PROJECTIONS[name]


def _ptr(t: torch.Tensor) -> int:
    return t.data_ptr()


def _stream(device) -> int:
    return torch.cuda.current_stream(device).cuda_stream


def _need(t, name, dtype=torch.float32, ndim=None):
    if not isinstance(t, torch.Tensor):
        raise TypeError(f"{name} must be a torch.Tensor")
    if not t.is_cuda:
        raise ValueError(f"{name} must be a CUDA tensor (this path has no CPU fallback)")
    if t.dtype != dtype:
        raise TypeError(f"{name} must be {dtype}, got {t.dtype}")
    if ndim is not None and t.dim() != ndim:
        raise ValueError(f"{name} must have {ndim} dims, got shape {tuple(t.shape)}")
    return t.contiguous()


class _Workspace:
    """One growable device scratch buffer per device, reused across calls."""

    def __init__(self):
        self._bufs = {}

    def get(self, device, nbytes: int) -> torch.Tensor:
        key = (device.type, device.index)
        buf = self._bufs.get(key)
        if buf is None or buf.numel() < nbytes:
            self._bufs.pop(key, None)
            buf = torch.empty(max(int(nbytes), 256), dtype=torch.uint8, device=device)
            self._bufs[key] = buf
        return buf


_ws = _Workspace()


class _HostStage:
    """Device->host reads through pinned staging.

    The copies are queued (non-blocking) on the current stream of the
    tensors' device into one pinned buffer per host thread, and waited for
    with a CUDA event, which does not hold the GIL.  A pageable copy would
    wait for the stream in the driver instead, and a host thread that waits
    there for a long peel stalls the other threads' copies and launches (the
    batch reader of `extract` filters the next batch meanwhile).  Returns
    numpy copies, so the buffer is free again when `fetch` returns.
    """

    def __init__(self):
        self._local = threading.local()

    def _buffer(self, nbytes: int) -> torch.Tensor:
        buf = getattr(self._local, "buf", None)
        if buf is None or buf.numel() < nbytes:
            buf = torch.empty(max(4096, int(nbytes * 1.25)), dtype=torch.uint8, pin_memory=True)
            self._local.buf = buf
        return buf

    def fetch(self, *tensors: torch.Tensor):
        ts = [t.detach().contiguous() for t in tensors]
        dev = next((t.device for t in ts if t.is_cuda), None)
        if dev is None:                       # host tensors (the CPU checks of the loop)
            return [t.numpy().copy() for t in ts]
        offs, total = [], 0
        for t in ts:
            offs.append(total)
            total += -(-t.numel() * t.element_size() // 64) * 64
        buf = self._buffer(total)
        views = []
        for t, o in zip(ts, offs):
            nb = t.numel() * t.element_size()
            v = buf[o:o + nb].view(t.dtype).view(t.shape)
            if nb:
                v.copy_(t, non_blocking=True)
            views.append(v)
        ev = torch.cuda.Event()
        ev.record(torch.cuda.current_stream(dev))
        ev.synchronize()
        return [v.numpy().copy() for v in views]


_host = _HostStage()


def to_host(*tensors: torch.Tensor):
    """numpy copies of device tensors, read through pinned staging (`_HostStage`)."""
    return _host.fetch(*tensors)


class _TransposedCtc:
    """The most recent ctc in the peel's layout, ctcT[k][j][lag] = ctc[j][k][lag].

    `extract` matches every batch with the same ctc tensor; transposing it once
    instead of per batch saves a full pass over K*K*(2nt+1) floats per batch.
    The entry belongs to that tensor object (a weak reference: a new tensor
    that happens to reuse the freed storage of an old one is a new entry) and
    to its version counter, so an in-place change of ctc invalidates it.
    """

    def __init__(self):
        self._ref = None
        self._version = None
        self._val = None

    def get(self, ctc: torch.Tensor, nt: int) -> torch.Tensor:
        if self._ref is not None and self._ref() is ctc and self._version == ctc._version:
            return self._val
        self._ref, self._version, self._val = None, None, None
        K = ctc.shape[0]
        out = torch.empty_like(ctc)
        lib = _lib.load()
        _lib.check(lib.ks_ctc_transpose(_ptr(ctc), K, nt, _ptr(out), _stream(ctc.device)),
                   "ks_ctc_transpose")
        self._ref, self._version, self._val = weakref.ref(ctc), ctc._version, out
        return out


_ctcT = _TransposedCtc()


def th2_of(Th) -> float:
    """Th_learned**2 as the reference's float32 comparison sees it."""
    return float(np.float32(float(Th) ** 2))


# ------------------------------------------------------------------ building blocks
def template_energy(U: torch.Tensor) -> torch.Tensor:
    """nm[k] = sum_{p,c} U[k,p,c]^2 (kilosort/template_matching.py:176)."""
    U = _need(U, "U", ndim=3)
    K, P, Cn = U.shape
    nm = torch.empty(K, dtype=torch.float32, device=U.device)
    lib = _lib.load()
    _lib.check(lib.ks_template_energy(_ptr(U), K, P, Cn, _ptr(nm), _stream(U.device)),
               "ks_template_energy")
    return nm


def project_scores(X, U, W, nt, projection="fp32", tiled=False, check_status=True):
    """Score matrix B (kilosort/template_matching.py:180-181).

    Returns B [K, L] (a view of a row-padded buffer), or with ``tiled`` the
    peel's blocked layout Bt [ceil(L/32), K, 32], Bt[b, k, i] = B[k, 32*b + i].
    ``check_status`` reads the device status (one host synchronisation).
    """
    X = _need(X, "X", ndim=2)
    U = _need(U, "U", ndim=3)
    W = _need(W, "wPCA", ndim=2)
    Cn, L = X.shape
    K, P, Cu = U.shape
    if Cu != Cn or W.shape != (P, nt):
        raise ValueError("shape mismatch between X, U and wPCA")
    prec = _PROJECTIONS[projection]
    lib = _lib.load()
    if tiled:
        B = torch.empty(((L + 31) // 32, K, 32), dtype=torch.float32, device=X.device)
        ldb, layout = 0, _lib.KS_B_TILED
    else:
        ldb = ((L + 63) // 64) * 64
        B = torch.empty((K, ldb), dtype=torch.float32, device=X.device)
        layout = _lib.KS_B_ROWS
    nbytes = lib.ks_project_workspace_size(Cn, L, K, P, prec)
    ws = _ws.get(X.device, nbytes)
    status = torch.zeros(1, dtype=torch.int32, device=X.device)
    _lib.check(lib.ks_project(_ptr(X), _ptr(U), _ptr(W), Cn, L, K, P, nt, prec,
                              _ptr(B), ldb, layout, _ptr(status), _ptr(ws), ws.numel(),
                              _stream(X.device)), "ks_project")
    if check_status:
        st = int(status.item())
        if st != _lib.KS_OK:
            raise _lib.KilosortB200Error(st, f"ks_project: device status {st} "
                                         f"({_lib.status_message(st)})")
    return B if tiled else B[:, :L]


def _info_status(info, what):
    n, status, iters, need = (int(v) for v in to_host(info)[0].tolist())
    if status == _lib.KS_ERR_OVERFLOW:
        raise RuntimeError(
            f"{what}: {need} spikes in one batch exceed the spike buffer "
            f"(capacity {n} written so far); raise ops['spike_capacity']")
    if status != _lib.KS_OK:
        raise _lib.KilosortB200Error(status, f"{what}: device status {status} "
                                     f"({_lib.status_message(status)})")
    return n, iters


def peel(B, Xres, U, W, ctc, nm, Th, nt, max_peels, capacity=DEFAULT_CAPACITY,
         ctc_transposed=False):
    """Greedy peel on a given score matrix, in place on B and Xres.

    ``B`` is either [K, L] with contiguous rows (any row stride) or the tiled
    [ceil(L/32), K, 32] layout of ``project_scores(..., tiled=True)``.  ``ctc``
    is in the reference layout, or ctcT[k][j][lag] with ``ctc_transposed``.
    Returns (st [N,2] int64, amps [N,1], th_amps [N,1], iterations), in the
    order of kilosort/template_matching.py:183-244.
    """
    Xres = _need(Xres, "Xres", ndim=2)
    U = _need(U, "U", ndim=3)
    W = _need(W, "wPCA", ndim=2)
    ctc = _need(ctc, "ctc", ndim=3)
    nm = _need(nm, "nm", ndim=1)
    K, P, Cn = U.shape
    L = Xres.shape[1]
    if not (isinstance(B, torch.Tensor) and B.is_cuda and B.dtype == torch.float32):
        raise ValueError("B must be a float32 CUDA tensor")
    if B.dim() == 3:
        if B.shape != ((L + 31) // 32, K, 32) or not B.is_contiguous():
            raise ValueError("tiled B must be a contiguous [ceil(L/32), K, 32] tensor")
        ldb, layout = 0, _lib.KS_B_TILED
    else:
        if not (B.dim() == 2 and B.shape == (K, L) and B.stride(1) == 1
                and B.stride(0) >= L):
            raise ValueError("B must be [K, L] with contiguous rows")
        ldb, layout = B.stride(0), _lib.KS_B_ROWS
    if ctc.shape != (K, K, 2 * nt + 1):
        raise ValueError("shape mismatch between U and ctc")
    clayout = _lib.KS_CTC_KJL if ctc_transposed else _lib.KS_CTC_JKL
    dev = Xres.device
    st = torch.zeros((capacity, 2), dtype=torch.int64, device=dev)
    amps = torch.zeros((capacity, 1), dtype=torch.float32, device=dev)
    th_amps = torch.zeros((capacity, 1), dtype=torch.float32, device=dev)
    info = torch.zeros(4, dtype=torch.int64, device=dev)
    lib = _lib.load()
    ws = _ws.get(dev, lib.ks_peel_workspace_size(L, K, nt, layout, clayout))
    _lib.check(lib.ks_peel(_ptr(B), ldb, layout, _ptr(Xres), _ptr(U), _ptr(W), _ptr(ctc),
                           clayout, _ptr(nm), Cn, L, K, P, nt, th2_of(Th), int(max_peels),
                           int(capacity), _ptr(st), _ptr(amps), _ptr(th_amps), _ptr(info),
                           _ptr(ws), ws.numel(), _stream(dev)), "ks_peel")
    n, iters = _info_status(info, "ks_peel")
    return st[:n], amps[:n], th_amps[:n], iters


def transpose_ctc(ctc, nt):
    """ctcT[k][j][lag] = ctc[j][k][lag], the layout the peel streams."""
    ctc = _need(ctc, "ctc", ndim=3)
    out = torch.empty_like(ctc)
    lib = _lib.load()
    _lib.check(lib.ks_ctc_transpose(_ptr(ctc), ctc.shape[0], nt, _ptr(out),
                                    _stream(ctc.device)), "ks_ctc_transpose")
    return out


# ------------------------------------------------------------------ drop-in API
def run_matching(ops, X, U, ctc, device=torch.device("cuda")):
    """Greedy template matching of one padded batch.

    Same contract as kilosort/template_matching.py:170-244: returns
    ``(st [N,2] int64, amps [N,1] float32, th_amps [N,1] float32, Xres [C,L])``
    with spikes in (iteration, time) order; ``X`` is not modified.
    """
    Th = ops["Th_learned"]
    nt = int(ops["nt"])
    max_peels = int(ops["max_peels"])
    W = _need(ops["wPCA"], "ops['wPCA']", ndim=2)
    X = _need(X, "X", ndim=2)
    U = _need(U, "U", ndim=3)
    ctc = _need(ctc, "ctc", ndim=3)
    Cn, L = X.shape
    K, P, Cu = U.shape
    if Cu != Cn:
        raise ValueError(f"U has {Cu} channels but X has {Cn}")
    if W.shape != (P, nt):
        raise ValueError(f"wPCA must be [{P}, {nt}], got {tuple(W.shape)}")
    if ctc.shape != (K, K, 2 * nt + 1):
        raise ValueError(f"ctc must be [{K}, {K}, {2 * nt + 1}], got {tuple(ctc.shape)}")
    capacity = int(ops.get("spike_capacity", DEFAULT_CAPACITY)) if hasattr(ops, "get") \
        else DEFAULT_CAPACITY
    prec = _projection(ops)
    dev = X.device
    # only the first info[0] rows are returned, and the peel writes all of info
    st = torch.empty((capacity, 2), dtype=torch.int64, device=dev)
    amps = torch.empty((capacity, 1), dtype=torch.float32, device=dev)
    th_amps = torch.empty((capacity, 1), dtype=torch.float32, device=dev)
    Xres = torch.empty_like(X)
    info = torch.empty(4, dtype=torch.int64, device=dev)
    lib = _lib.load()
    ctcT = _ctcT.get(ctc, nt)
    ws = _ws.get(dev, lib.ks_run_matching_workspace_size(Cn, L, K, P, nt, prec,
                                                         _lib.KS_CTC_KJL))
    _lib.check(lib.ks_run_matching(_ptr(X), _ptr(U), _ptr(W), _ptr(ctcT), _lib.KS_CTC_KJL,
                                   Cn, L, K, P, nt,
                                   th2_of(Th), max_peels, prec, capacity, _ptr(st),
                                   _ptr(amps), _ptr(th_amps), _ptr(Xres), _ptr(info),
                                   _ptr(ws), ws.numel(), _stream(dev)), "ks_run_matching")
    n, _ = _info_status(info, "run_matching")
    return st[:n], amps[:n], th_amps[:n], Xres


def prepare_matching(ops, U):
    """Template cross-correlations ctc [K, K, 2nt+1] (template_matching.py:155-167)."""
    nt = int(ops["nt"])
    W = _need(ops["wPCA"], "ops['wPCA']", ndim=2)
    U = _need(U, "U", ndim=3)
    K, P, Cn = U.shape
    ctc = torch.empty((K, K, 2 * nt + 1), dtype=torch.float32, device=U.device)
    lib = _lib.load()
    ws = _ws.get(U.device, lib.ks_ctc_workspace_size(K, P, Cn, nt))
    _lib.check(lib.ks_ctc(_ptr(U), _ptr(W), K, P, Cn, nt, _ptr(ctc), _ptr(ws), ws.numel(),
                          _stream(U.device)), "ks_ctc")
    return ctc


def prepare_extract(xc, yc, U, nC, position_limit, device=torch.device("cuda")):
    """Nearest channels, masks, peak channels and loadings (template_matching.py:14-53).

    The channel neighbourhoods are host-side numpy, as in the reference; the
    per-template peak channel ``iU`` and loadings ``Ucc`` come from the GPU.
    """
    ds = (xc - xc[:, np.newaxis]) ** 2 + (yc - yc[:, np.newaxis]) ** 2
    iCC = np.argsort(ds, 0)[:nC]
    iCC = torch.from_numpy(iCC).to(device)
    iCC_mask = np.sort(ds, 0)[:nC] < position_limit ** 2
    iCC_mask = torch.from_numpy(iCC_mask).to(device)
    U = _need(U, "U", ndim=3)
    K, P, Cn = U.shape
    iCCd = iCC.to(U.device).contiguous()
    iU = torch.empty(K, dtype=torch.int64, device=U.device)
    Ucc = torch.empty((nC, K, P), dtype=torch.float32, device=U.device)
    lib = _lib.load()
    _lib.check(lib.ks_template_channels(_ptr(U), _ptr(iCCd), K, P, Cn, nC, _ptr(iU),
                                        _ptr(Ucc), _stream(U.device)),
               "ks_template_channels")
    return iCC, iCC_mask, iU, Ucc


def spike_features(Xres, st, amps, W, iCC, iU, Ucc):
    """Per-spike PC features [N, nC, P] (template_matching.py:85-86, 108)."""
    Xres = _need(Xres, "Xres", ndim=2)
    W = _need(W, "wPCA", ndim=2)
    st = _need(st, "st", dtype=torch.int64, ndim=2)
    amps = _need(amps, "amps").reshape(-1)
    iCC = _need(iCC, "iCC", dtype=torch.int64, ndim=2)
    iU = _need(iU, "iU", dtype=torch.int64, ndim=1)
    Ucc = _need(Ucc, "Ucc", ndim=3)
    nC, K, P = Ucc.shape
    Cn, L = Xres.shape
    nt = W.shape[1]
    N = st.shape[0]
    tF = torch.empty((N, nC, P), dtype=torch.float32, device=Xres.device)
    if N == 0:
        return tF
    lib = _lib.load()
    _lib.check(lib.ks_features(_ptr(Xres), _ptr(st), _ptr(amps), _ptr(W), _ptr(iCC),
                               _ptr(iU), _ptr(Ucc), Cn, L, K, P, nt, nC, N, _ptr(tF),
                               _stream(Xres.device)), "ks_features")
    return tF


def _match_features(ops, W, iCCd, iU, Ucc):
    """Default per-batch matcher and feature step of `extract` (this library)."""
    def match(X, U, ctc, device):
        return run_matching(ops, X, U, ctc, device=device)

    def features(Xres, st, amps):
        return spike_features(Xres, st, amps, W, iCCd, iU, Ucc)     # [N, nC, P]
    return match, features


_reader_pools = {}
_reader_lock = threading.Lock()


def _reader(device):
    """(worker thread, stream) that read batches ahead for ``device``; kept for
    the process, so repeated `extract` calls reuse the thread's library
    handles."""
    key = (device.type, device.index)
    with _reader_lock:
        r = _reader_pools.get(key)
        if r is None:
            from concurrent.futures import ThreadPoolExecutor
            pool = ThreadPoolExecutor(1, thread_name_prefix="ks-batch-reader")
            stream = torch.cuda.Stream(device) if device.type == "cuda" else None
            r = _reader_pools[key] = (pool, stream)
        return r


class _BatchReader:
    """Reads padded batches one ahead on a worker thread, so the next batch's
    file read, host->device copy and filter overlap the current batch's
    matching.

    A reference ``BinaryFiltered`` with int16 or uint16 samples (and no
    scale or shift) on a CUDA device is read through
    ``filtered.FilteredBatches``: the raw window goes into pinned memory,
    crosses as int16 and is filtered on the device by ``ks_preprocess_int16``
    -- the batch ``bfile.padded_batch_to_torch(ibatch, ops)`` returns
    (kilosort/io.py:1037-1045), made on the device.  ``ops['device_filter'] =
    False`` keeps the file's own ``padded_batch_to_torch``; any other source
    uses it too.

    On a CUDA device the read runs on the reader's own stream and is complete
    when handed over (the stream is synchronised in the worker); the tensor is
    then recorded on the consumer's stream so its memory is not reused while
    that stream may still read it.
    """

    def __init__(self, bfile, order, ops, device=None, ahead=True, depth=1):
        self.bfile, self.order, self.ops = bfile, list(order), ops
        self.device = torch.device(device) if device is not None else None
        self.pool = None
        self.stream = None
        self.pending = []               # futures of order[self.submitted - len(pending):]
        self.submitted = 0
        self.depth = max(1, int(depth))
        self.filtered = None
        from . import filtered          # imports this module's stream helper
        if self.device is not None and self.device.type == "cuda" \
                and ops.get("device_filter", True) and filtered.supports(bfile):
            self.filtered = filtered.batches_for(bfile, self.device)
        if ahead and len(self.order) > 1:
            self.pool, self.stream = _reader(self.device or torch.device("cpu"))
            self._fill()

    def _fill(self):
        while len(self.pending) < self.depth and self.submitted < len(self.order):
            self.pending.append(self.pool.submit(self._read, self.order[self.submitted]))
            self.submitted += 1

    def _load(self, ibatch):
        if self.filtered is None:
            return self.bfile.padded_batch_to_torch(ibatch, self.ops)
        return self.filtered.batch(ibatch, self.ops)

    def _read(self, ibatch):
        """(X, event): the event marks the end of X's copy and filter on the
        reader's stream (None: X is complete)."""
        dev = self.device
        if self.pool is None or dev is None or dev.type != "cuda":
            X = self._load(ibatch)
            if self.filtered is not None:
                self.filtered.check()
            return X, None
        s = self.stream
        with torch.cuda.device(dev), torch.cuda.stream(s):
            X = self._load(ibatch)
            if self.filtered is not None:
                # the device source is stream-ordered: the consumer waits on
                # the event, and the host cuts the next window meanwhile
                ev = torch.cuda.Event()
                ev.record(s)
                return X, ev
        s.synchronize()
        return X, None

    def get(self, pos):
        """The batch ``order[pos]``; positions are taken in increasing order,
        with up to ``depth`` reads in flight ahead of the consumer."""
        if self.pool is None:
            return self._read(self.order[pos])[0]
        X, ev = self.pending.pop(0).result()
        self._fill()
        if isinstance(X, torch.Tensor) and X.is_cuda:
            cur = torch.cuda.current_stream(X.device)
            if ev is not None:
                cur.wait_event(ev)
            X.record_stream(cur)
        return X

    def close(self):
        # leave no read of ours running on the shared worker
        for f in self.pending:
            if not f.cancel():
                try:
                    f.result()
                except Exception:
                    pass
        self.pending = []
        self.pool = None
        self.filtered = None

    def check(self):
        """Raise if the device batch source reported an error for any batch
        read so far (call after the last batch is consumed)."""
        if self.filtered is not None:
            self.filtered.check()


def _rows_host(ops, bfile, ibatch, st_h, th_h, tf_h):
    """Host rows ``[N, 3]`` and features of one matched batch, as
    kilosort/template_matching.py:88-108 forms them: batch 0 drops the spikes
    whose aligned time would be negative, the time is shifted by the batch's
    start and aligned to nt0min in float64 (exact for sample indices)."""
    nt = ops["nt"]
    if ibatch == 0:
        keep = ~((st_h[:, 0] - nt - nt // 2 + ops["nt0min"]) < 0)
        st_h, th_h, tf_h = st_h[keep], th_h[keep], tf_h[keep]
    t_shift = ibatch * bfile.batch_downsampling * (ops["batch_size"])
    rows = np.empty((len(st_h), 3), "float64")
    rows[:, 0] = ((st_h[:, 0].astype("float64") - nt) + t_shift) - nt // 2 + ops["nt0min"]
    rows[:, 1] = st_h[:, 1]
    rows[:, 2] = th_h.reshape(-1)
    return rows, torch.from_numpy(np.ascontiguousarray(tf_h))


def _batch_rows(ops, bfile, ibatch, stt, th_amps, xfeat):
    return _rows_host(ops, bfile, ibatch, *to_host(stt, th_amps, xfeat))


def extract_batches(ops, bfile, batches, U, ctc, match, features, progress_bar=None,
                    read_ahead=True, reader=None):
    """Rows ``[N, 3]`` (time, template, th_amp; float64 numpy) and features
    ``[N, nC, P]`` (CPU tensor) of the given batches, in batch order, before
    the final sort -- the loop body of kilosort/template_matching.py:79-110.

    ``match(X, U, ctc, device)`` returns ``(st, amps, th_amps, Xres)`` and
    ``features(Xres, st, amps)`` the ``[N, nC, P]`` features of one batch.
    With ``read_ahead`` the next batch is read while the current one is
    matched (the same batches in the same order), so the batch source must
    return a new tensor per call (the reference's ``BinaryFiltered`` does); a
    source that refills one buffer needs ``read_ahead=False``
    (``ops['read_ahead'] = False`` through `extract`).  Rows are gathered per
    batch and joined once at the end (the reference grows preallocated
    buffers of 10**6 rows; the returned rows are the same).
    """
    try:
        from tqdm import tqdm
    except ImportError:  # pragma: no cover
        tqdm = None
    nt = ops["nt"]
    nC = ops["settings"]["nearest_chans"]
    sts, tFs = [], []
    prog = tqdm(batches, miniters=200 if progress_bar else None,
                mininterval=60 if progress_bar else None) if tqdm else batches
    ibatch = -1
    if reader is None:
        reader = _BatchReader(bfile, [int(b) for b in batches], ops, device=U.device,
                              ahead=read_ahead)
    try:
        for pos, ibatch in enumerate(prog):
            ibatch = int(ibatch)
            if ibatch % 100 == 0 and torch.cuda.is_available():
                logger.debug(f"Batch {ibatch}: {torch.cuda.memory_allocated() / 2**30:.2f} GiB allocated")
            X = reader.get(pos)
            stt, amps, th_amps, Xres = match(X, U, ctc, X.device)
            xfeat = features(Xres, stt, amps)
            rows, tf = _batch_rows(ops, bfile, ibatch, stt, th_amps, xfeat)
            sts.append(rows)
            tFs.append(tf)
            if progress_bar is not None:
                progress_bar.emit(int((ibatch + 1) / bfile.n_batches * 100))
        reader.check()
    except Exception:
        logger.exception(f"Error in kilosort_b200.extract on batch {ibatch}")
        raise
    finally:
        reader.close()
    st = np.concatenate(sts) if sts else np.zeros((0, 3), "float64")
    tF = torch.cat(tFs) if tFs else torch.zeros((0, nC, ops["settings"]["n_pcs"]))
    return st, tF


def extract_grouped(ops, bfile, batches, U, ctc, feat, group=4, teams=None,
                    progress_bar=None, reader=None):
    """`extract_batches` with the batches matched ``group`` at a time by one
    ``ks_match_batches`` launch (the batched matcher: each batch's peel
    equals its own ``run_matching``, bit for bit), so a team of blocks works on
    every batch of the group at once instead of the whole device on one batch.
    ``feat`` = (wPCA, iCC, iU, Ucc) on the device.

    Group sizes ramp up as 1, 2, 4, ... to ``group``, so the first launch
    starts after one batch is read.  The reader keeps a group and one batch in
    flight ahead of the matcher.
    Each group's PC features are enqueued right behind its launch with the
    spike counts read on the device (``ks_features_counted``), so nothing
    waits for the host between the launches.  Two sets of outputs alternate:
    while group g is matched, the rows and features of group g-1 are copied to
    the host on a side stream (copies only, which run beside the peel), and
    group g+1 is launched once they have arrived.  ``teams`` defaults to one
    team per batch.  Returns the same rows and features, in batch order, as
    `extract_batches`.
    """
    from . import batched as bt
    batches = [int(b) for b in batches]
    dev = U.device
    nt = int(ops["nt"])
    proj = ops.get("projection", _default_projection)
    W, iCC, iU, Ucc = feat
    nC, K, P = Ucc.shape
    cap = int(ops.get("spike_capacity", DEFAULT_CAPACITY))
    rec = bt.Recording(U=U, wPCA=ops["wPCA"], ctc=ctc, Th=ops["Th_learned"], nt=nt,
                       max_peels=int(ops["max_peels"]), capacity=cap, ctcT=_ctcT.get(ctc, nt))
    if reader is None:
        reader = _BatchReader(bfile, batches, ops, device=dev, ahead=True, depth=group + 1)
    main = torch.cuda.current_stream(dev)
    aux = torch.cuda.Stream(dev)
    lib = _lib.load()
    sts, tFs = [], []
    slots = [None, None]                  # (outs, info, tF buffers) per parity
    ws = None
    prev = None
    ibatch = -1

    def finish(prev):
        nonlocal ibatch
        grp, outs, info, tfs, done, _items = prev
        with torch.cuda.stream(aux):
            aux.wait_event(done)
            host = to_host(info)[0]
            counts = []
            for i, ib in enumerate(grp):
                ibatch = ib
                n, status, _it, need = (int(v) for v in host[i])
                if status == _lib.KS_ERR_OVERFLOW:
                    raise RuntimeError(f"extract: batch {ib} needs {need} spikes, above the "
                                       f"capacity {cap}; raise ops['spike_capacity']")
                if status != _lib.KS_OK:
                    raise _lib.KilosortB200Error(status, f"extract: batch {ib}: device status "
                                                 f"{status} ({_lib.status_message(status)})")
                counts.append(n)
            parts = []
            for i, n in enumerate(counts):
                parts += [outs[i].st[:n], outs[i].th_amps[:n], tfs[i][:n]]
            got = to_host(*parts)
        for i, ib in enumerate(grp):
            rows, tf = _rows_host(ops, bfile, ib, *got[3 * i:3 * i + 3])
            sts.append(rows)
            tFs.append(tf)
            if progress_bar is not None:
                progress_bar.emit(int((ib + 1) / bfile.n_batches * 100))

    # group sizes 1, 2, 4, ... up to `group`: the first launch starts after one
    # batch is read instead of a whole group
    sizes, left, g = [], len(batches), 1
    while left > 0:
        sizes.append(min(g, group, left))
        left -= sizes[-1]
        g *= 2
    try:
        pos = 0
        for gi, size in enumerate(sizes):
            g0 = pos
            grp = batches[g0:g0 + size]
            Xs = [reader.get(pos + i) for i in range(len(grp))]
            pos += len(grp)
            items = [(X, 0) for X in Xs]
            slot = gi % 2
            if slots[slot] is None or slots[slot][0][0].Xres.shape != Xs[0].shape:
                # a full group's outputs; smaller groups use the first entries
                Cn, L = Xs[0].shape
                slots[slot] = ([bt._Outputs(rec, Cn, L, dev) for _ in range(group)],
                               torch.empty((group, 4), dtype=torch.int64, device=dev),
                               [torch.empty((cap, nC, P), dtype=torch.float32, device=dev)
                                for _ in range(group)])
            outs, info, tfs = (slots[slot][0][:len(grp)], slots[slot][1][:len(grp)],
                               slots[slot][2][:len(grp)])
            t = int(teams) if teams else len(grp)
            need = bt.workspace_size([rec], items, proj, t)
            if ws is None or ws.numel() < need:
                ws = torch.empty(need, dtype=torch.uint8, device=dev)
            bt._launch([rec], items, outs, info, ws, proj, t)
            for i, (X, o) in enumerate(zip(Xs, outs)):
                Cn, L = o.Xres.shape
                _lib.check(lib.ks_features_counted(
                    _ptr(o.Xres), _ptr(o.st), _ptr(o.amps), _ptr(W), _ptr(iCC), _ptr(iU),
                    _ptr(Ucc), Cn, L, K, P, W.shape[1], nC, _ptr(info[i]), cap,
                    _ptr(tfs[i]), _stream(dev)), "ks_features_counted")
            done = torch.cuda.Event()
            done.record(main)
            if prev is not None:
                finish(prev)
            prev = (grp, outs, info, tfs, done, items)
        if prev is not None:
            finish(prev)
            prev = None
        main.wait_stream(aux)
        reader.check()
    except Exception:
        logger.exception(f"Error in kilosort_b200.extract on batch {ibatch}")
        raise
    finally:
        reader.close()
    st = np.concatenate(sts) if sts else np.zeros((0, 3), "float64")
    tF = torch.cat(tFs) if tFs else torch.zeros((0, nC, ops["settings"]["n_pcs"]))
    return st, tF


def sort_spikes(st, tF):
    """The final ordering of kilosort/template_matching.py:122-124 (numpy's
    default argsort of the times, as the reference calls it)."""
    isort = np.argsort(st[:, 0])
    return st[isort], tF[isort]


def extract(ops, bfile, U, device=torch.device("cuda"), progress_bar=None):
    """Match every batch of ``bfile`` and collect spikes and PC features.

    Same contract as kilosort/template_matching.py:56-126: returns
    ``(st [N,3] float64 numpy (time, template, th_amp), tF [N,nC,P] CPU
    tensor, ops)`` sorted by time, and stores ``iCC``, ``iCC_mask``, ``iU``
    in ``ops``.
    """
    nC = ops["settings"]["nearest_chans"]
    position_limit = ops["settings"]["position_limit"]
    batches = np.arange(bfile.n_batches, dtype=np.int64)
    group = int(ops.get("batch_group", 4))
    ahead = bool(ops.get("read_ahead", True))
    grouped = ahead and group > 1 and len(batches) > 1 and U.is_cuda
    # the first batches are read (and filtered) while the templates are prepared
    reader = _BatchReader(bfile, [int(b) for b in batches], ops, device=U.device,
                          ahead=ahead, depth=group + 1 if grouped else 1)
    try:
        iCC, iCC_mask, iU, Ucc = prepare_extract(ops["xc"], ops["yc"], U, nC,
                                                 position_limit, device=device)
        ops["iCC"] = iCC
        ops["iCC_mask"] = iCC_mask
        ops["iU"] = iU
        ctc = prepare_matching(ops, U)
        W = ops["wPCA"].contiguous()
        iCCd = iCC.to(U.device).contiguous()
        match, features = _match_features(ops, W, iCCd, iU, Ucc)
    except Exception:
        reader.close()
        raise
    if grouped:
        st, tF = extract_grouped(ops, bfile, batches, U, ctc, (W, iCCd, iU, Ucc),
                                 group=group, teams=ops.get("batch_teams"),
                                 progress_bar=progress_bar, reader=reader)
    else:
        st, tF = extract_batches(ops, bfile, batches, U, ctc, match, features, progress_bar,
                                 reader=reader)
    st, tF = sort_spikes(st, tF)
    return st, tF, ops


def install(module=None):
    """Route the reference's template matching through this implementation.

    Replaces ``run_matching``, ``prepare_matching``, ``prepare_extract`` and
    ``extract`` on ``kilosort.template_matching`` (or on ``module``).  The
    reference's ``extract`` resolves ``run_matching`` as a module global, so
    patching the attribute reroutes it as well.  Returns the patched module.
    """
    if module is None:
        import importlib
        module = importlib.import_module("kilosort.template_matching")
    module.run_matching = run_matching
    module.prepare_matching = prepare_matching
    module.prepare_extract = prepare_extract
    module.extract = extract
    return module
