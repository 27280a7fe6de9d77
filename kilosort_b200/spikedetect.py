"""Universal-template spike detection on the device (drop-in for
kilosort/spikedetect.py's ``template_match`` and ``run``).

The host part is the reference's own bookkeeping, done the same way in numpy:
template positions on a grid (``template_centers``, spikedetect.py:97-130),
the nearest channels of each position and the nearest positions of each
(``nearest_chans``, :181-187), the Gaussian size weights (:221-246).  The
per-batch part -- the convolution with the universal waveforms, the weighted
sums over sizes and waveforms, the neighbourhood maximum, the max-pool and
the peak test, the amplitudes, y positions and PC features -- is one call of
``ks_detect`` (no tensor of all the sums is ever stored).

The universal waveforms and basis come from ``ops['wTEMP']``/``ops['wPCA']``
(the reference's built-in templates file, or templates learned from data
elsewhere); learning them here (``templates_from_data``: k-means and SVD of
snippets) is not on the device path.
"""
from __future__ import annotations

from typing import Optional

import numpy as np
import torch

from . import _lib
from .template_matching import _stream


def _ptr(t) -> int:
    return 0 if t is None else t.data_ptr()


def template_centers(ops):
    """Template positions yup, xup (spikedetect.py:97-130); sets ops['dmin'], ops['dminx']."""
    shank_idx = ops["kcoords"]
    xc, yc = ops["xc"], ops["yc"]
    dmin = ops["settings"]["dmin"]
    if dmin is None:
        y_uniq = np.unique(yc)
        dmin = 1 if y_uniq.size == 1 else np.median(np.diff(np.unique(y_uniq)))
    ops["dmin"] = dmin
    ops["dminx"] = dminx = ops["settings"]["dminx"]
    yup, xup = np.array([]), np.array([])
    for i in np.unique(shank_idx):
        xc_i, yc_i = xc[shank_idx == i], yc[shank_idx == i]
        xmin, xmax, ymin, ymax = xc_i.min(), xc_i.max(), yc_i.min(), yc_i.max()
        yup = np.concatenate([yup, np.arange(ymin, ymax + .01, dmin / 2)])
        nx = np.round((xmax - xmin) / (dminx / 2)) + 1
        xup = np.concatenate([xup, np.linspace(xmin, xmax, int(nx))])
    ops["yup"], ops["xup"] = np.unique(yup), np.unique(xup)
    return ops


def nearest_chans(ys, yc, xs, xc, nC, device=torch.device("cuda")):
    """The nC nearest of (xc, yc) to each (xs, ys), and the squared distances."""
    ds = (ys - yc[:, np.newaxis]) ** 2 + (xs - xc[:, np.newaxis]) ** 2
    iC = np.argsort(ds, 0)[:nC]
    return torch.from_numpy(iC).to(device), np.sort(ds, 0)[:nC]


def geometry(ops, device=torch.device("cuda")):
    """(iC, iC2, weigh) of run() (spikedetect.py:221-246); sets ops['ycup'], ops['xcup']."""
    ops = template_centers(ops)
    ys, xs = np.meshgrid(ops["yup"], ops["xup"])
    ys, xs = ys.flatten(), xs.flatten()
    xc, yc = ops["xc"], ops["yc"]
    s = ops["settings"]
    iC, ds = nearest_chans(ys, yc, xs, xc, s["nearest_chans"], device=device)
    igood = ds[0, :] <= ops["max_channel_distance"] ** 2
    iC, ds, ys, xs = iC[:, igood], ds[:, igood], ys[igood], xs[igood]
    ops["ycup"], ops["xcup"] = ys, xs
    iC2, _ = nearest_chans(ys, ys, xs, xs, s["nearest_templates"], device=device)
    ds_t = torch.from_numpy(ds).to(device).float()
    sizes = s["min_template_size"] * (1 + torch.arange(s["template_sizes"], device=device))
    weigh = torch.exp(-ds_t.unsqueeze(-1) / sizes ** 2)
    weigh = torch.permute(weigh, (2, 0, 1)).contiguous()
    weigh = weigh / (weigh ** 2).sum(1).unsqueeze(1) ** .5
    return iC, iC2, weigh


class Detector:
    """``ks_detect`` for batches [C, L] with fixed geometry and templates."""

    def __init__(self, ops, iC, iC2, weigh, device=None, capacity: int = 200000):
        self.device = torch.device(device) if device is not None else iC.device
        if self.device.type != "cuda":
            raise ValueError("detection runs on a CUDA device (no CPU fallback)")
        d = self.device
        self.iC = iC.to(d, torch.int64).contiguous()
        self.iC2 = iC2.to(d, torch.int64).contiguous()
        self.weigh = weigh.to(d, torch.float32).contiguous()
        self.wTEMP = ops["wTEMP"].to(d, torch.float32).contiguous()
        self.wPCA = ops["wPCA"].to(d, torch.float32).contiguous()
        self.yc = torch.as_tensor(np.asarray(ops["yc"], np.float32)).to(d)
        self.nt = int(ops["nt"])
        self.nt0 = int(ops["settings"]["nt0min"])
        self.th = float(ops["Th_universal"])
        self.capacity = int(capacity)
        self.info = torch.zeros(4, dtype=torch.int64, device=d)
        self._ws = None

    def _alloc(self, cap):
        nC, P = self.iC.shape[0], self.wPCA.shape[0]
        d = self.device
        return dict(xy=torch.empty((cap, 2), dtype=torch.int64, device=d),
                    imax=torch.empty(cap, dtype=torch.int64, device=d),
                    amp=torch.empty(cap, dtype=torch.float32, device=d),
                    adist=torch.empty((nC, cap), dtype=torch.float32, device=d),
                    yct=torch.empty(cap, dtype=torch.float32, device=d),
                    tF=torch.empty((cap, nC, P), dtype=torch.float32, device=d))

    def __call__(self, X: torch.Tensor):
        """One batch -> (xy [n, 2], imax [n], amp [n], adist [nC, n], yct [n], tF [n, nC, P])."""
        X = X.to(self.device, torch.float32).contiguous()
        C, L = X.shape
        nC, Nfilt = self.iC.shape
        lib = _lib.load()
        need = lib.ks_detect_workspace_size(C, L, self.wTEMP.shape[0], Nfilt)
        if self._ws is None or self._ws.numel() < need:
            self._ws = torch.empty(need, dtype=torch.uint8, device=self.device)
        cap = self.capacity
        while True:
            o = self._alloc(cap)
            _lib.check(lib.ks_detect(
                _ptr(X), C, L, _ptr(self.wTEMP), self.wTEMP.shape[0], self.nt, _ptr(self.iC),
                nC, _ptr(self.iC2), self.iC2.shape[0], _ptr(self.weigh), self.weigh.shape[0],
                Nfilt, self.nt0, self.th, _ptr(self.wPCA), self.wPCA.shape[0], _ptr(self.yc),
                cap, _ptr(o["xy"]), _ptr(o["imax"]), _ptr(o["amp"]), _ptr(o["adist"]),
                _ptr(o["yct"]), _ptr(o["tF"]), _ptr(self.info), _ptr(self._ws), self._ws.numel(),
                _stream(self.device)), "ks_detect")
            n, status, _, found = (int(v) for v in self.info.cpu().tolist())
            if status == _lib.KS_ERR_OVERFLOW:
                cap = int(found * 1.25) + 1024       # detect again with room for all
                self.capacity = max(self.capacity, cap)
                continue
            if status != _lib.KS_OK:
                raise _lib.KilosortB200Error(status, f"ks_detect: device status {status}")
            return (o["xy"][:n], o["imax"][:n], o["amp"][:n], o["adist"][:, :n], o["yct"][:n],
                    o["tF"][:n])


def template_match(X, ops, iC, iC2, weigh, device=torch.device("cuda")):
    """Same inputs and outputs as kilosort/spikedetect.py:133-178:
    (xy [n, 2] (position, sample), imax [n], amp [n], adist [nC, n])."""
    xy, imax, amp, adist, _, _ = Detector(ops, iC, iC2, weigh, device)(X)
    return xy, imax, amp, adist


def run(ops, bfile, device=torch.device("cuda"), progress_bar=None, clear_cache=False,
        verbose=False):
    """Same inputs and outputs as kilosort/spikedetect.py:199-307 with the
    universal templates already in ops ('wTEMP', 'wPCA'): (st [n, 6] float64 --
    time in s, y, amplitude, index, batch, position --, tF [n, nC, P], ops)."""
    if "wTEMP" not in ops or "wPCA" not in ops:
        raise ValueError("ops['wTEMP'] and ops['wPCA'] are needed (learning them is not on "
                         "the device path)")
    iC, iC2, weigh = geometry(ops, device=device)
    det = Detector(ops, iC, iC2, weigh, device)
    nt = ops["nt"]
    sts, tFs = [], []
    for ibatch in range(bfile.n_batches):
        X = bfile.padded_batch_to_torch(ibatch, ops)
        xy, imax, amp, _, yct, tF = det(X)
        xy_h = xy.cpu().numpy()
        st = np.zeros((len(xy_h), 6), "float64")
        t_shift = ibatch * bfile.batch_downsampling * (ops["batch_size"] / ops["fs"])
        st[:, 0] = (xy_h[:, 1] - nt) / ops["fs"] + t_shift
        st[:, 1] = yct.cpu().numpy()
        st[:, 2] = amp.cpu().numpy()
        st[:, 3] = imax.cpu().numpy()
        st[:, 4] = ibatch
        st[:, 5] = xy_h[:, 0]
        sts.append(st)
        tFs.append(tF.cpu().numpy())
        if progress_bar is not None:
            progress_bar.emit(int((ibatch + 1) / bfile.n_batches * 100))
    ops["iC"], ops["iC2"], ops["weigh"] = iC, iC2, weigh
    nC, P = iC.shape[0], ops["wPCA"].shape[0]
    st = np.concatenate(sts) if sts else np.zeros((0, 6))
    tF = np.concatenate(tFs) if tFs else np.zeros((0, nC, P), np.float32)
    return st, tF, ops
