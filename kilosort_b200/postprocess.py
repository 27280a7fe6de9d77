"""Output consumers of `extract` on the GPU (kernel ``ks_spike_positions``).

* ``compute_spike_positions(st, tF, ops)`` -- same signature and outputs as
  kilosort/postprocessing.py:33-62: x and y (float64 numpy) of each spike as
  the feature-norm-weighted mean of the positions of the nC channels nearest
  its template's peak channel (channels beyond ``position_limit`` weigh 0).
* ``spike_amplitudes(tF)`` -- the Phy-export amplitudes of kilosort/io.py:353,
  ``||tF[s]||`` (float32 numpy).
* ``template_similarity(Wall, W, nt)`` -- kilosort/CCG.py:94-102, Phy's
  similar_templates (io.py:377), on the device (kernel ``ks_similarity``).

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
