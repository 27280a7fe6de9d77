"""CPU oracle of the universal-template spike detection.

TEST INFRASTRUCTURE ONLY.  Restates kilosort/spikedetect.py with the same
PyTorch/numpy operations, in the same order:

* ``template_centers`` -- :97-130: template positions on a grid of dmin/2
  vertically (dmin: median spacing of the contact rows when unset) and
  dminx/2 horizontally, per shank;
* ``nearest_chans`` -- :181-187: the nC nearest channels of each position;
* ``setup`` -- :221-246 of ``run``: positions farther than
  max_channel_distance from every channel dropped, the nC2 nearest template
  positions of each, the Gaussian size weights (template_sizes multiples of
  min_template_size) normalised per size and position;
* ``template_match`` -- :133-178: the universal waveforms convolved with the
  batch, the weighted sums over each position's nearest channels for every
  size and waveform, the signed index of the largest magnitude, the maximum
  over the nC2 nearest positions, edges zeroed, a (2*nt0min+1) max-pool in
  time, peaks above Th_universal;
* ``yweighted`` -- :190-197;
* ``run_batches`` -- the per-batch loop of ``run`` (:250-285): st (time in
  seconds, y, amplitude, signed index, batch, position) and the PC features;
* ``extract_snippets`` -- :33-48, the isolated single-channel peaks and their
  snippets (templates_from_data);
* ``svd_basis`` -- the exact truncated-SVD basis of the unit-norm snippets
  with sklearn's sign convention (the reference's TruncatedSVD, :72-73, is
  randomized and approximates it).

Pinned against tests/golden/golden_detect.npz and golden_learn.npz (the
reference's own run() and extract_snippets).
"""
from __future__ import annotations

import numpy as np
import torch
import torch.nn.functional as F
from torch.nn.functional import conv1d, max_pool1d


def template_centers(xc, yc, kcoords, dmin=None, dminx=32.0):
    if dmin is None:
        y_uniq = np.unique(yc)
        dmin = 1 if y_uniq.size == 1 else np.median(np.diff(np.unique(y_uniq)))
    yup, xup = np.array([]), np.array([])
    for i in np.unique(kcoords):
        xc_i, yc_i = xc[kcoords == i], yc[kcoords == i]
        xmin, xmax, ymin, ymax = xc_i.min(), xc_i.max(), yc_i.min(), yc_i.max()
        yup = np.concatenate([yup, np.arange(ymin, ymax + .01, dmin / 2)])
        nx = np.round((xmax - xmin) / (dminx / 2)) + 1
        xup = np.concatenate([xup, np.linspace(xmin, xmax, int(nx))])
    return np.unique(yup), np.unique(xup), dmin


def nearest_chans(ys, yc, xs, xc, nC):
    ds = (ys - yc[:, np.newaxis]) ** 2 + (xs - xc[:, np.newaxis]) ** 2
    iC = np.argsort(ds, 0)[:nC]
    return torch.from_numpy(iC), np.sort(ds, 0)[:nC]


def setup(xc, yc, kcoords, settings, max_channel_distance):
    yup, xup, dmin = template_centers(xc, yc, kcoords, settings["dmin"], settings["dminx"])
    ys, xs = np.meshgrid(yup, xup)
    ys, xs = ys.flatten(), xs.flatten()
    iC, ds = nearest_chans(ys, yc, xs, xc, settings["nearest_chans"])
    igood = ds[0, :] <= max_channel_distance ** 2
    iC, ds, ys, xs = iC[:, igood], ds[:, igood], ys[igood], xs[igood]
    iC2, _ = nearest_chans(ys, ys, xs, xs, settings["nearest_templates"])
    ds_t = torch.from_numpy(ds).float()
    sizes = settings["min_template_size"] * (1 + torch.arange(settings["template_sizes"]))
    weigh = torch.exp(-ds_t.unsqueeze(-1) / sizes ** 2)
    weigh = torch.permute(weigh, (2, 0, 1)).contiguous()
    weigh = weigh / (weigh ** 2).sum(1).unsqueeze(1) ** .5
    return iC, iC2, weigh, ys, xs, dmin


def template_match(X, wTEMP, iC, iC2, weigh, nt, nt0, Th_universal):
    nk = wTEMP.shape[0]
    NT = X.shape[-1]
    Nfilt = iC.shape[1]
    niter = 40
    nb = (NT - 1) // niter + 1
    B = conv1d(X.unsqueeze(1), wTEMP.unsqueeze(1), padding=nt // 2)
    As = torch.zeros((Nfilt, NT))
    Amaxs = torch.zeros((Nfilt, NT))
    imaxs = torch.zeros((Nfilt, NT), dtype=torch.int64)
    ti = torch.arange(Nfilt)
    tj = torch.arange(nb)
    for t in range(niter):
        A = torch.einsum('ijk, jklm-> iklm', weigh, B[iC, :, nb * t:nb * (t + 1)])
        A = A.transpose(1, 2)
        A = A.reshape(-1, Nfilt, A.shape[-1])
        Aa, imax = torch.max(A.abs(), 0)
        imax = (1 + imax) * A[imax, ti.unsqueeze(-1), tj[:A.shape[-1]]].sign()
        As[:, nb * t:nb * (t + 1)] = Aa
        imaxs[:, nb * t:nb * (t + 1)] = imax
        Amax = torch.max(Aa[iC2], 0)[0]
        Amaxs[:, nb * t:nb * (t + 1)] = Amax
    Amaxs[:, :nt] = 0
    Amaxs[:, -nt:] = 0
    Amaxs = max_pool1d(Amaxs.unsqueeze(0), (2 * nt0 + 1), stride=1, padding=nt0).squeeze(0)
    xy = torch.logical_and(Amaxs == As, As > Th_universal).nonzero()
    imax = imaxs[xy[:, 0], xy[:, 1]]
    amp = As[xy[:, 0], xy[:, 1]]
    ssign = imax.sign()
    imax = imax.abs() - 1
    adist = B[iC[:, xy[:, 0]], imax % nk, xy[:, 1]] * ssign
    return xy, imax, amp, adist


def yweighted(yc, iC, adist, xy):
    yy = torch.from_numpy(yc)[iC]
    cF0 = torch.nn.functional.relu(adist)
    cF0 = cF0 / cF0.sum(0)
    return (cF0 * yy[:, xy[:, 0]]).sum(0)


def run_batches(batches, wTEMP, wPCA, iC, iC2, weigh, yc, nt, nt0, Th_universal,
                batch_size, fs, batch_downsampling=1):
    """st [N, 6] float64 and tF [N, nC, P] float32 over the padded batches."""
    tarange = torch.arange(-(nt // 2), nt // 2 + 1)
    sts, tFs = [], []
    for ibatch, X in enumerate(batches):
        xy, imax, amp, adist = template_match(X, wTEMP, iC, iC2, weigh, nt, nt0, Th_universal)
        yct = yweighted(yc, iC, adist, xy)
        xsub = X[iC[:, xy[:, :1]], xy[:, 1:2] + tarange]
        xfeat = xsub @ wPCA.T
        st = np.zeros((len(xy), 6), 'float64')
        t_shift = ibatch * batch_downsampling * (batch_size / fs)
        st[:, 0] = (xy[:, 1].numpy() - nt) / fs + t_shift
        st[:, 1] = yct.numpy()
        st[:, 2] = amp.numpy()
        st[:, 3] = imax.numpy()
        st[:, 4] = ibatch
        st[:, 5] = xy[:, 0].numpy()
        sts.append(st)
        tFs.append(xfeat.transpose(0, 1).numpy())
    return np.concatenate(sts), np.concatenate(tFs)


def extract_snippets(X, nt, twav_min, Th_single_ch, loc_range=(4, 5), long_range=(6, 30)):
    """kilosort/spikedetect.py:33-48 with the same torch ops: isolated
    single-channel peaks (max_pool2d window, avg_pool2d count times its area
    equal to 1), zero within nt of both edges, snippets in nonzero order."""
    Xabs = X.abs()
    Xmax = F.max_pool2d(Xabs.unsqueeze(0), [2 * loc_range[0] + 1, 2 * loc_range[1] + 1],
                        stride=[1, 1], padding=[loc_range[0], loc_range[1]])[0]
    ispeak = torch.logical_and(Xmax == Xabs, Xabs > Th_single_ch).float()
    area = (2 * long_range[0] + 1) * (2 * long_range[1] + 1)
    ispeak_sum = F.avg_pool2d(ispeak.unsqueeze(0), [2 * long_range[0] + 1, 2 * long_range[1] + 1],
                              stride=[1, 1], padding=[long_range[0], long_range[1]])[0] * area
    is_peak_iso = (ispeak_sum == 1) * (ispeak == 1)
    is_peak_iso[:, :nt] = 0
    is_peak_iso[:, -nt:] = 0
    xy = is_peak_iso.nonzero()
    return X[xy[:, :1], xy[:, 1:2] - twav_min + torch.arange(nt)]


def svd_basis(clips, n_pcs):
    """The exact top right singular vectors [n_pcs, nt] (float64) of the
    unit-norm snippets, each row signed so its largest-magnitude entry is
    positive (the sign convention of sklearn's TruncatedSVD, which
    kilosort/spikedetect.py:72-73 uses)."""
    x = np.asarray(clips, dtype=np.float64)
    x = x / np.sqrt((x ** 2).sum(1, keepdims=True))
    _, _, vt = np.linalg.svd(x, full_matrices=False)
    comp = vt[:n_pcs]
    sgn = np.sign(comp[np.arange(comp.shape[0]), np.abs(comp).argmax(1)])
    return comp * sgn[:, None]
