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

The universal waveforms and basis come, as in the reference's ``run``
(:205-216), either from its built-in templates file (``get_waves``, read from
the same place the reference keeps its download, $KILOSORT_LOCAL_DOWNLOADS_PATH
or ~/.kilosort; this library does not download it) or, with
``settings['templates_from_data']``, from the data (``extract_wPCA_wTEMP``,
:50-92): the isolated single-channel peaks of every 25th batch
(``ks_snippets``), the exact truncated-SVD basis of their unit-norm snippets
(``ks_snippet_gram`` on the device, the 61 x 61 symmetric eigenproblem on the
host, rows signed as sklearn's TruncatedSVD signs them) and k-means of the
snippets (k-means++ seeding and Lloyd steps on the device:
``ks_kmeans_mindist``, ``ks_kmeans_candidates``, ``ks_kmeans_step``; ten
seeded starts, the lowest inertia kept, as sklearn's KMeans with
n_init=10).  The reference's TruncatedSVD and KMeans are randomized
(random_state=None); these are deterministic for a given ``seed``.
"""
from __future__ import annotations

import os
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


def template_path(basename="wTEMP.npz"):
    """Where the reference keeps its built-in universal templates
    (kilosort/utils.py:22-38): $KILOSORT_LOCAL_DOWNLOADS_PATH, else
    ~/.kilosort, file ``basename``."""
    base = os.environ.get("KILOSORT_LOCAL_DOWNLOADS_PATH") or os.path.join(
        os.path.expanduser("~"), ".kilosort")
    return os.path.join(base, basename)


def get_waves(ops, device=torch.device("cuda")):
    """kilosort/spikedetect.py:94-98: (wPCA, wTEMP) of the built-in templates
    file.  The reference downloads the file when it is missing; this library
    has no download and raises FileNotFoundError instead."""
    path = template_path()
    if not os.path.exists(path):
        raise FileNotFoundError(
            f"{path} not found: place the reference's wTEMP.npz there (or set "
            "KILOSORT_LOCAL_DOWNLOADS_PATH), or set settings['templates_from_data']")
    dd = np.load(path)
    return (torch.from_numpy(dd["wPCA"]).to(device), torch.from_numpy(dd["wTEMP"]).to(device))


def extract_snippets(X, nt, twav_min, Th_single_ch, device=None):
    """Same inputs and output as kilosort/spikedetect.py:33-48: the snippets
    [n, nt] of the isolated single-channel peaks of one padded batch X [C, L],
    in (channel, sample) order, on the device (``ks_snippets``)."""
    dev = torch.device(device) if device is not None else X.device
    if dev.type != "cuda":
        raise ValueError("snippets are extracted on a CUDA device (no CPU fallback)")
    Xd = X.to(dev, torch.float32).contiguous()
    C, L = Xd.shape
    # isolated peaks are more than 6 channels or 30 samples apart: at most
    # (C + 7) (L + 31) / (7 * 31) of them
    cap = (C + 7) * (L + 31) // (7 * 31) + 1
    clips = torch.empty((cap, nt), dtype=torch.float32, device=dev)
    n = _snippets_into(Xd, nt, twav_min, Th_single_ch, clips, 0)
    return clips[:n]


def _snippets_into(Xd, nt, twav_min, th, clips, base):
    """Snippets of one batch written at clips[base:]; returns the batch's count."""
    lib = _lib.load()
    C, L = Xd.shape
    ws = torch.empty(lib.ks_snippets_workspace_size(C, L), dtype=torch.uint8, device=Xd.device)
    count = torch.zeros(1, dtype=torch.int32, device=Xd.device)
    _lib.check(lib.ks_snippets(_ptr(Xd), C, L, int(nt), int(twav_min), float(th), int(base),
                               clips.shape[0], _ptr(clips), _ptr(count), _ptr(ws), ws.numel(),
                               _stream(Xd.device)), "ks_snippets")
    return int(count.item())


def svd_basis(clips, n_pcs):
    """The top ``n_pcs`` right singular vectors [n_pcs, nt] of the snippets
    after each is scaled to unit norm (in place): the Gram matrix on the
    device (``ks_snippet_gram``, double), its eigenvectors on the host in
    descending eigenvalue order, each row signed so its largest-magnitude
    entry is positive (sklearn's TruncatedSVD convention, which the
    reference's wPCA follows).  float32 on the device of ``clips``."""
    n, nt = clips.shape
    dev = clips.device
    lib = _lib.load()
    G = torch.empty((nt, nt), dtype=torch.float64, device=dev)
    ws = torch.empty(lib.ks_snippet_gram_workspace_size(n, nt), dtype=torch.uint8, device=dev)
    _lib.check(lib.ks_snippet_gram(_ptr(clips), n, nt, _ptr(G), _ptr(ws), ws.numel(),
                                   _stream(dev)), "ks_snippet_gram")
    w, V = np.linalg.eigh(G.cpu().numpy())
    comp = V[:, np.argsort(w)[::-1][:n_pcs]].T
    sgn = np.sign(comp[np.arange(comp.shape[0]), np.abs(comp).argmax(1)])
    sgn[sgn == 0] = 1.0
    return torch.from_numpy((comp * sgn[:, None]).astype(np.float32)).to(dev)


def kmeans(X, k, n_init=10, max_iter=300, tol=1e-4, seed=0):
    """k-means of the rows of X [n, d] (float32, CUDA), as sklearn's KMeans
    (k-means++ seeding with 2 + log(k) local trials, Lloyd steps until the
    labels stop changing or the squared center shift is at most tol times
    the mean per-feature variance, ``n_init`` starts, the lowest inertia
    kept), with its random choices drawn from numpy's RandomState(seed).
    Returns (centers [k, d] float32 on X's device, inertia)."""
    n, d = X.shape
    dev = X.device
    lib = _lib.load()
    stream = _stream(dev)
    ws = torch.empty(lib.ks_kmeans_workspace_size(n, d, max(k, 1)), dtype=torch.uint8,
                     device=dev)
    if ws.numel() == 0:
        raise ValueError("kmeans: need n >= 1 and d, k <= 64")
    labels = torch.empty(n, dtype=torch.int32, device=dev)
    sums = torch.empty((max(k, 1), d), dtype=torch.float64, device=dev)
    counts = torch.empty(max(k, 1), dtype=torch.int64, device=dev)
    stats = torch.empty(2, dtype=torch.float64, device=dev)

    def step(centers):
        labels_k = centers.shape[0]
        _lib.check(lib.ks_kmeans_step(_ptr(X), n, d, _ptr(centers), labels_k, _ptr(labels),
                                      _ptr(sums), _ptr(counts), _ptr(stats), _ptr(ws),
                                      ws.numel(), stream), "ks_kmeans_step")
        return (sums[:labels_k].cpu().numpy(), counts[:labels_k].cpu().numpy(),
                stats.cpu().numpy())

    # tolerance: tol x the mean per-feature variance (one step against the origin)
    labels.fill_(-1)
    s1, _, st1 = step(torch.zeros((1, d), dtype=torch.float32, device=dev))
    tol_s = tol * (st1[0] / n - float((s1[0] / n) @ (s1[0] / n))) / d
    rng = np.random.RandomState(seed)
    d2 = torch.empty(n, dtype=torch.float64, device=dev)
    pots = torch.empty(64, dtype=torch.float64, device=dev)
    trials = 2 + int(np.log(k))
    best = None
    for _ in range(n_init):
        # k-means++ seeding
        first = int(rng.randint(n))
        centers = [X[first].clone()]
        _lib.check(lib.ks_kmeans_mindist(_ptr(X), n, d, _ptr(centers[0]), 1, _ptr(d2), stream),
                   "ks_kmeans_mindist")
        d2h = d2.cpu().numpy()
        pot = float(d2h.sum())
        for _c in range(1, k):
            cand = np.searchsorted(np.cumsum(d2h), rng.uniform(size=trials) * pot)
            cand = np.minimum(cand, n - 1)
            cx = X[torch.from_numpy(cand).to(dev)].contiguous()
            _lib.check(lib.ks_kmeans_candidates(_ptr(X), n, d, _ptr(cx), trials, _ptr(d2),
                                                _ptr(pots), _ptr(ws), ws.numel(), stream),
                       "ks_kmeans_candidates")
            b = int(np.argmin(pots[:trials].cpu().numpy()))
            centers.append(cx[b].clone())
            _lib.check(lib.ks_kmeans_mindist(_ptr(X), n, d, _ptr(centers[-1]), 0, _ptr(d2),
                                             stream), "ks_kmeans_mindist")
            d2h = d2.cpu().numpy()
            pot = float(d2h.sum())
        C = torch.stack(centers).contiguous()
        Ch = C.cpu().numpy().astype(np.float64)
        labels.fill_(-1)
        for _it in range(max_iter):
            sm, cn, st = step(C)
            new = np.where(cn[:, None] > 0, sm / np.maximum(cn, 1)[:, None], Ch)
            shift = float(((new - Ch) ** 2).sum())
            Ch = new
            C = torch.from_numpy(Ch.astype(np.float32)).to(dev)
            if st[1] == 0 or shift <= tol_s:
                break
        inertia = float(step(C)[2][0])
        if best is None or inertia < best[1]:
            best = (C, inertia)
    return best


def extract_wPCA_wTEMP(ops, bfile, nt=61, twav_min=20, Th_single_ch=6, nskip=25,
                       device=torch.device("cuda"), seed=0):
    """Same inputs and outputs as kilosort/spikedetect.py:50-92: the snippets
    of the isolated peaks of batches 0, nskip, 2 nskip, ... (up to 500000;
    the batch that would pass that is left out, and the reading stops), wPCA
    [n_pcs, nt] = their truncated-SVD basis (``svd_basis``), wTEMP
    [n_templates, nt] = their k-means centers (``kmeans``) scaled to unit
    norm; both float32 on ``device``."""
    dev = torch.device(device)
    if dev.type != "cuda":
        raise ValueError("templates are learned on a CUDA device (no CPU fallback)")
    cap = 500000
    clips = torch.empty((cap, nt), dtype=torch.float32, device=dev)
    i = 0
    for j in range(0, bfile.n_batches, nskip):
        X = bfile.padded_batch_to_torch(j, ops).to(dev, torch.float32).contiguous()
        nnew = _snippets_into(X, nt, twav_min, Th_single_ch, clips, i)
        if i + nnew > cap:
            break
        i += nnew
    clips = clips[:i].contiguous()
    s = ops["settings"]
    wPCA = svd_basis(clips, s["n_pcs"])
    wTEMP, _ = kmeans(clips, s["n_templates"], n_init=10, seed=seed)
    wTEMP = wTEMP / (wTEMP ** 2).sum(1).unsqueeze(1) ** .5
    return wPCA, wTEMP


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
    """Same inputs and outputs as kilosort/spikedetect.py:199-307: (st [n, 6]
    float64 -- time in s, y, amplitude, index, batch, position --, tF
    [n, nC, P], ops).  The universal templates ops['wPCA'], ops['wTEMP'] come
    from the data when settings['templates_from_data'] is set
    (extract_wPCA_wTEMP), else from the built-in templates file (get_waves),
    as the reference sets them (:205-216)."""
    s = ops["settings"]
    if s.get("templates_from_data", True):
        ops["wPCA"], ops["wTEMP"] = extract_wPCA_wTEMP(
            ops, bfile, nt=ops["nt"], twav_min=ops["nt0min"], Th_single_ch=s["Th_single_ch"],
            nskip=25, device=device)
    else:
        ops["wPCA"], ops["wTEMP"] = get_waves(ops, device=device)
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
