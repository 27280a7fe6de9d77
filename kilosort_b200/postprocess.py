"""Output consumers of `extract` on the GPU (kernel ``ks_spike_positions``).

* ``compute_spike_positions(st, tF, ops)`` -- same signature and outputs as
  kilosort/postprocessing.py:33-62: x and y (float64 numpy) of each spike as
  the feature-norm-weighted mean of the positions of the nC channels nearest
  its template's peak channel (channels beyond ``position_limit`` weigh 0).
* ``spike_amplitudes(tF)`` -- the Phy-export amplitudes of kilosort/io.py:353,
  ``||tF[s]||`` (float32 numpy).
* ``template_similarity(Wall, W, nt)`` -- kilosort/CCG.py:94-102, Phy's
  similar_templates (io.py:377), on the device (kernel ``ks_similarity``).
* ``remove_duplicates(spike_times, spike_clusters, dt)`` --
  kilosort/postprocessing.py:10-30 on the device (``ks_remove_duplicates``).
* ``phy_templates(Wall, wPCA)`` -- templates.npy and templates_ind.npy of
  kilosort/io.py:383-387 (``ks_phy_templates``).
* ``phy_arrays(st, clu, tF, Wall, ops, imin)`` / ``save_phy_arrays`` -- the
  arrays save_to_phy (kilosort/io.py:248-470) derives from the matching
  outputs, under the reference's file names: spike times, clusters,
  detection templates, positions and amplitudes after duplicate removal, the
  kept-spike mask, the template waveforms, their channel indices and the
  template similarity.  The rest of save_to_phy (probe and whitening files,
  pc_features.npy, which regroups features per cluster through the
  clustering module, the refractoriness labels, params.py) is not produced
  here.

``st`` and ``tF`` may be the host arrays `extract` returns; they are moved to
the device of ``ops['iU']`` (which must be a CUDA device).
"""
from __future__ import annotations

import numpy as np
import torch

from . import _lib
from .template_matching import _ptr, _stream


def _device_of(ops):
    dev = ops["iU"].device if isinstance(ops.get("iU"), torch.Tensor) else None
    if dev is None or dev.type != "cuda":
        raise ValueError("ops['iU'] must be a CUDA tensor (this path has no CPU fallback)")
    return dev


def _positions(st, tF, ops):
    dev = _device_of(ops)
    tFd = torch.as_tensor(tF).to(device=dev, dtype=torch.float32).contiguous()
    N, nC, P = tFd.shape
    templ = torch.as_tensor(np.asarray(st)[:, 1] if not isinstance(st, torch.Tensor)
                            else st[:, 1]).to(device=dev, dtype=torch.int64).contiguous()
    iCC = ops["iCC"].to(device=dev, dtype=torch.int64).contiguous()
    mask = ops["iCC_mask"].to(device=dev, dtype=torch.uint8).contiguous()
    iU = ops["iU"].to(device=dev, dtype=torch.int64).contiguous()
    xc = torch.as_tensor(np.asarray(ops["xc"], dtype=np.float64)).to(dev)
    yc = torch.as_tensor(np.asarray(ops["yc"], dtype=np.float64)).to(dev)
    C, K = iCC.shape[1], iU.shape[0]
    if iCC.shape[0] != nC or mask.shape != iCC.shape:
        raise ValueError("tF, iCC and iCC_mask disagree on the number of nearest channels")
    xs = torch.empty(N, dtype=torch.float64, device=dev)
    ys = torch.empty(N, dtype=torch.float64, device=dev)
    amps = torch.empty(N, dtype=torch.float32, device=dev)
    status = torch.empty(1, dtype=torch.int32, device=dev)
    lib = _lib.load()
    _lib.check(lib.ks_spike_positions(_ptr(tFd), _ptr(templ), _ptr(iCC), _ptr(mask), _ptr(iU),
                                      _ptr(xc), _ptr(yc), N, nC, P, C, K, _ptr(xs), _ptr(ys),
                                      _ptr(amps), _ptr(status), _stream(dev)),
               "ks_spike_positions")
    if int(status.item()) != _lib.KS_OK:
        raise _lib.KilosortB200Error(_lib.KS_ERR_ARG, "ks_spike_positions: template index out of range")
    return xs, ys, amps


def compute_spike_positions(st, tF, ops):
    """x, y positions of spikes (kilosort/postprocessing.py:33-62)."""
    xs, ys, _ = _positions(st, tF, ops)
    return xs.cpu().numpy(), ys.cpu().numpy()


def spike_amplitudes(tF, ops):
    """Phy-export amplitudes ||tF[s]|| (kilosort/io.py:353)."""
    st = np.zeros((torch.as_tensor(tF).shape[0], 2))
    _, _, amps = _positions(st, tF, ops)
    return amps.cpu().numpy()


def template_similarity(Wall: torch.Tensor, W: torch.Tensor, nt: int = 61,
                        to_host: bool = True):
    """Same inputs and output as kilosort/CCG.py:94-102 (``similarity``):
    ``Wall`` [K, C, P] templates, ``W`` = wPCA [P, nt]; returns [K, K] float32,
    the maximum over lags of the cross-correlation of the unit-norm templates
    (numpy on the host, as the reference returns it, unless ``to_host`` is
    False).  Runs on the device of ``Wall`` (``ks_similarity``)."""
    if not isinstance(Wall, torch.Tensor) or Wall.device.type != "cuda":
        raise ValueError("Wall must be a CUDA tensor (this path has no CPU fallback)")
    dev = Wall.device
    Wd = Wall.to(torch.float32).contiguous()
    Wp = W.to(device=dev, dtype=torch.float32).contiguous()
    K, C, P = Wd.shape
    lib = _lib.load()
    ws = torch.empty(lib.ks_similarity_workspace_size(K, C, P, nt), dtype=torch.uint8, device=dev)
    sim = torch.empty((K, K), dtype=torch.float32, device=dev)
    _lib.check(lib.ks_similarity(_ptr(Wd), _ptr(Wp), K, C, P, nt, _ptr(sim), _ptr(ws),
                                 ws.numel(), _stream(dev)), "ks_similarity")
    return sim.cpu().numpy() if to_host else sim


def template_amplitudes(Wall: torch.Tensor) -> np.ndarray:
    """kilosort/io.py:378: ``||Wall[k]||`` over channels and components."""
    return torch.norm(Wall, dim=[-2, -1]).cpu().numpy()


def remove_duplicates(spike_times, spike_clusters, dt=15, device=None):
    """Same inputs and outputs as kilosort/postprocessing.py:10-30: spikes in
    index order, a spike kept when its time is at least ``dt`` after the last
    kept spike of its cluster; returns (spike_times[keep],
    spike_clusters[keep], keep) as numpy arrays.  Runs on ``device`` (default
    cuda:0) through ``ks_remove_duplicates``."""
    dev = torch.device(device) if device is not None else torch.device("cuda", 0)
    if dev.type != "cuda":
        raise ValueError("remove_duplicates runs on a CUDA device (no CPU fallback)")
    t_host = np.asarray(spike_times, dtype=np.int64)
    c_host = np.asarray(spike_clusters, dtype=np.int32)
    if t_host.shape != c_host.shape or t_host.ndim != 1:
        raise ValueError("spike_times and spike_clusters must be 1-D and of equal length")
    N = t_host.size
    if N == 0:
        return t_host.copy(), c_host.copy(), np.zeros(0, bool)
    t = torch.from_numpy(t_host).to(dev)
    c = torch.from_numpy(c_host).to(dev)
    keep = torch.empty(N, dtype=torch.uint8, device=dev)
    lib = _lib.load()
    ws = torch.empty(lib.ks_remove_duplicates_workspace_size(N), dtype=torch.uint8, device=dev)
    _lib.check(lib.ks_remove_duplicates(_ptr(t), _ptr(c), N, int(dt), _ptr(keep), _ptr(ws),
                                        ws.numel(), _stream(dev)), "ks_remove_duplicates")
    k = keep.cpu().numpy().astype(bool)
    return t_host[k], c_host[k], k


def phy_templates(Wall: torch.Tensor, W: torch.Tensor):
    """templates.npy and templates_ind.npy of kilosort/io.py:383-387: the
    waveform of each template from its PC loadings Wall [K, C, P] and the
    basis W = wPCA [P, nt], as [K, nt, C] float32, and the channel indices
    [K, C] (every channel, in order).  Runs on the device of ``Wall``."""
    if not isinstance(Wall, torch.Tensor) or Wall.device.type != "cuda":
        raise ValueError("Wall must be a CUDA tensor (this path has no CPU fallback)")
    dev = Wall.device
    Wd = Wall.to(torch.float32).contiguous()
    Wp = W.to(device=dev, dtype=torch.float32).contiguous()
    K, C, P = Wd.shape
    nt = Wp.shape[1]
    out = torch.empty((K, nt, C), dtype=torch.float32, device=dev)
    _lib.check(_lib.load().ks_phy_templates(_ptr(Wd), _ptr(Wp), K, C, P, nt, _ptr(out),
                                            _stream(dev)), "ks_phy_templates")
    ind = np.tile(np.arange(C)[np.newaxis, :], (K, 1))
    return out.cpu().numpy(), ind


def phy_arrays(st, clu, tF, Wall: torch.Tensor, ops, imin: int = 0):
    """The arrays kilosort/io.py:248-470 (save_to_phy) derives from the
    matching outputs, keyed by their file names without ``.npy``.  ``st``
    [N, >=2] (time in samples, template), ``clu`` [N] cluster per spike
    (int32), ``tF`` [N, nC, P] features, ``Wall`` [K, C, P] cluster loadings
    on the device, ``ops`` with iCC, iCC_mask, iU, xc, yc, wPCA, nt and
    duplicate_spike_bins; ``imin`` shifts the exported times
    (io.py:350-389)."""
    st = np.asarray(st)
    spike_times = st[:, 0].astype("int64") + imin
    spike_templates = st[:, 1].astype("int32")
    xs, ys, amps = _positions(st, tF, ops)
    spike_positions = np.vstack([xs.cpu().numpy(), ys.cpu().numpy()]).T
    amplitudes = amps.cpu().numpy()
    dev = _device_of(ops)
    spike_times, spike_clusters, kept = remove_duplicates(
        spike_times, np.asarray(clu, dtype=np.int32), dt=ops["duplicate_spike_bins"], device=dev)
    templates, templates_ind = phy_templates(Wall, ops["wPCA"])
    return {
        "spike_times": spike_times,
        "spike_templates": spike_clusters,
        "spike_clusters": spike_clusters,
        "spike_positions": spike_positions[kept],
        "spike_detection_templates": spike_templates[kept],
        "amplitudes": amplitudes[kept],
        "kept_spikes": kept,
        "similar_templates": template_similarity(Wall, ops["wPCA"], nt=int(ops["nt"])),
        "templates": templates,
        "templates_ind": templates_ind,
    }


def save_phy_arrays(results_dir, arrays):
    """Write ``phy_arrays`` output as <name>.npy files in results_dir, the
    names and contents save_to_phy gives them."""
    import os
    os.makedirs(results_dir, exist_ok=True)
    for name, value in arrays.items():
        np.save(os.path.join(results_dir, name + ".npy"), value)
