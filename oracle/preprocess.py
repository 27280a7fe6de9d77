"""CPU oracle of the batch preprocessing (the filter applied to each padded batch).

TEST INFRASTRUCTURE ONLY.  Restates with the same PyTorch operations, in the
same order:

* ``highpass_filter`` -- kilosort/preprocessing.py:121-136: the impulse
  response (length 30122, centre 15061) of a 3rd-order Butterworth high-pass
  applied forwards and backwards (scipy ``butter`` + ``filtfilt``);
* ``fft_highpass`` -- kilosort/preprocessing.py:138-154: that response padded
  or cropped (centred) to the batch length, in the Fourier domain;
* ``filter_batch`` -- kilosort/io.py:994-1026 (BinaryFiltered.filter): channel
  map, sign inversion, per-channel mean removal, common average reference
  (lower median over channels), Fourier-domain high-pass with the half-length
  shift, artifact zeroing, whitening (drift matrix folded in as M @ Wrot);
* ``drift_matrix`` -- kilosort/preprocessing.py:44-69 with one block
  (kernel2D_torch, datashift.py:176-179; iKxx as datashift.py:216-223);
* ``drift_matrix_ops`` -- kilosort/preprocessing.py:44-69 as the filter calls
  it, from ``ops`` (blocks, their depths, probe, ``iKxx``, ``sig_interp``);
* ``padded_batch`` -- kilosort/io.py:789-831 (BinaryRWFile.padded_batch_to_torch):
  the file slice transposed, copied to the device as it is (pageable), made
  float32 (uint16 shifted by 2**15), its edges repeated for the first and last
  batch;
* ``filtered_batch`` -- kilosort/io.py:1037-1045: ``padded_batch`` then
  ``filter_batch`` with the batch's drift matrix.

Pinned against tests/golden/golden_pre.npz (the reference's own filter run on
the same inputs, tests/golden/make_golden_pre.py).
"""
from __future__ import annotations

import numpy as np
import torch
from torch.fft import fft, fftshift, ifft


def highpass_filter(fs=30000, cutoff=300):
    from scipy.signal import butter, filtfilt
    n = 30122
    b, a = butter(3, cutoff, fs=fs, btype="high")
    x = np.zeros(n)
    x[n // 2] = 1
    return torch.from_numpy(filtfilt(b, a, x).copy()).float()


def fft_highpass(hp, n):
    ft = hp.shape[0]
    if ft < n:
        pad = (n - ft) // 2
        z = lambda k: torch.zeros(k, dtype=hp.dtype, device=hp.device)
        return fft(torch.cat((z(pad), hp, z(pad + (n - pad * 2 - ft)))))
    if ft > n:
        crop = (ft - n) // 2
        return fft(hp[crop:crop + n])
    return fft(hp)


def filter_batch(X, chan_map=None, invert_sign=False, do_car=True, hp=None,
                 artifact_threshold=np.inf, whiten=None, drift=None):
    """X: [n_chan_bin, L] float32 (the padded batch); returns [C, L]."""
    if chan_map is not None:
        X = X[chan_map]
    if invert_sign:
        X = X * -1
    X = X - X.mean(1).unsqueeze(1)
    if do_car:
        X = X - torch.median(X, 0)[0]
    if hp is not None:
        fwav = fft_highpass(hp, X.shape[1])
        X = torch.real(ifft(fft(X) * torch.conj(fwav)))
        X = fftshift(X, dim=-1)
    if artifact_threshold < np.inf:
        if torch.any(torch.abs(X) >= artifact_threshold):
            return torch.zeros_like(X)
    if whiten is not None:
        X = ((drift @ whiten) if drift is not None else whiten) @ X
    return X


def kernel2d(x, y, sig):
    ds = ((x.unsqueeze(1) - y) ** 2).sum(-1)
    return torch.exp(-ds / (2 * sig ** 2))


def drift_matrix(xc, yc, shift, sig_interp=20.0):
    xp = np.vstack((xc, yc)).T
    Kxx = kernel2d(torch.from_numpy(xp), torch.from_numpy(xp), sig_interp)
    iKxx = torch.linalg.inv(Kxx + 0.01 * torch.eye(Kxx.shape[0]))
    yp = xp.copy()
    yp[:, 1] -= shift
    Kyx = kernel2d(torch.from_numpy(yp), torch.from_numpy(xp), sig_interp)
    return Kyx @ iKxx


def drift_matrix_ops(ops, dshift, device):
    if ops["nblocks"] == 1:
        shifts = dshift
    else:
        from scipy.interpolate import interp1d
        f = interp1d(ops["yblk"], dshift, fill_value="extrapolate", kind="linear")
        shifts = f(ops["probe"]["yc"])
    xp = np.vstack((ops["probe"]["xc"], ops["probe"]["yc"])).T
    yp = xp.copy()
    yp[:, 1] -= shifts
    Kyx = kernel2d(torch.from_numpy(yp).to(device), torch.from_numpy(xp).to(device),
                   ops["settings"]["sig_interp"])
    return Kyx @ ops["iKxx"].to(device)


def centre_offset(ft, L):
    """Where the filter's centre (index ft//2) lands relative to L//2 once
    fft_highpass has padded or cropped it to L samples: the shifted
    correlation reads sample n + d + offset for the tap at distance d."""
    if ft < L:
        cpos = (L - ft) // 2 + ft // 2
    elif ft > L:
        cpos = ft // 2 - (ft - L) // 2
    else:
        cpos = ft // 2
    return cpos - L // 2, cpos


def centre_taps(hp, L, ntaps=1023):
    """(taps, centre): X'[n] = sum_j taps[j] X[(n + j - centre) mod L] equals
    the reference's Fourier-domain high-pass up to the filter's tail beyond
    the taps kept (at most ntaps, and no more than the padded or cropped
    filter holds on either side of its centre)."""
    hp = hp.double().numpy() if torch.is_tensor(hp) else np.asarray(hp, np.float64)
    ft = hp.shape[0]
    off, cpos = centre_offset(ft, L)
    h = min(ntaps // 2, cpos, L - 1 - cpos)
    c = ft // 2
    taps = np.zeros(2 * h + 1)
    lo, hi = max(0, c - h), min(ft, c + h + 1)
    taps[lo - (c - h):hi - (c - h)] = hp[lo:hi]
    return taps, h - off


def filter_batch_taps(X, taps, centre=None, chan_map=None, invert_sign=False, do_car=True,
                      artifact_threshold=np.inf, whiten=None, drift=None):
    """float64 restatement with the high-pass as a circular correlation with
    centre taps (the form the device computes)."""
    X = X.double()
    if chan_map is not None:
        X = X[chan_map]
    if invert_sign:
        X = -X
    X = X - X.mean(1, keepdim=True)
    if do_car:
        X = X - torch.median(X, 0)[0]
    if taps is not None:
        Y = torch.zeros_like(X)
        for j, w in enumerate(taps):
            if w != 0.0:
                Y += float(w) * torch.roll(X, -(j - centre), dims=1)
        X = Y
    if artifact_threshold < np.inf and torch.any(torch.abs(X) >= artifact_threshold):
        return torch.zeros_like(X)
    if whiten is not None:
        W = whiten.double()
        if drift is not None:
            W = drift.double() @ W
        X = W @ X
    return X


def padded_batch(bfile, ibatch, device):
    ibatch = int(ibatch) * bfile.batch_downsampling
    bstart, bend = bfile._get_batch_edges(ibatch)
    data = bfile.file[bstart:bend].T
    if str(data.dtype) == "uint16":
        data = data.astype("float32") - 2 ** 15
    nsamp = data.shape[-1]
    nt = bfile.nt
    X = torch.zeros((bfile.n_chan_bin, bfile.NT + 2 * nt), device=device)
    if ibatch == 0:
        X[:, nt:nt + nsamp] = torch.from_numpy(data).to(device).float()
        X[:, :nt] = X[:, nt:nt + 1]
    elif ibatch == bfile.n_batches - 1:
        X[:, :nsamp] = torch.from_numpy(data).to(device).float()
        X[:, nsamp:] = X[:, nsamp - 1:nsamp]
    else:
        X[:] = torch.from_numpy(data).to(device).float()
    return X


def filtered_batch(bfile, ibatch, ops, device):
    X = padded_batch(bfile, ibatch, device)
    drift = None
    if bfile.whiten_mat is not None and bfile.dshift is not None and ops is not None:
        drift = drift_matrix_ops(ops, bfile.dshift[ibatch], device)
    cmap = None if bfile.chan_map is None else torch.as_tensor(bfile.chan_map, device=device)
    hp = None if bfile.hp_filter is None else bfile.hp_filter.to(device)
    W = None if bfile.whiten_mat is None else bfile.whiten_mat.to(device)
    return filter_batch(X, chan_map=cmap, invert_sign=bfile.invert_sign, do_car=bfile.do_CAR,
                        hp=hp, artifact_threshold=bfile.artifact_threshold, whiten=W,
                        drift=drift)
