"""One process per GPU: `extract` over contiguous batch ranges.

Batches are independent given U, ctc and wPCA (the only cross-batch state of
kilosort/template_matching.py:56-126 is each batch's time offset, :102, and
the final sort, :122-124), so the recording shards by batch with no
collective on the data path:

* rank 0's templates and basis are replicated by one broadcast each;
* rank r matches the contiguous range ``batch_range(n_batches, world, r)``;
* the per-rank rows and features go to ``dst`` (counts by all-gather, data by
  point-to-point, in rank order = batch order) and ``dst`` applies the
  reference's final sort, so the result equals a single-process `extract`.

For template refinement over several GPUs, ``allreduce_gradients`` sums the
per-rank adjoint gradients (dU, dwPCA) in place.
"""
from __future__ import annotations

from typing import Callable, Optional, Sequence, Tuple

import numpy as np
import torch
import torch.distributed as dist

from . import template_matching as tm


def batch_range(n_batches: int, world: int, rank: int) -> Tuple[int, int]:
    """Contiguous, balanced ``[start, stop)`` of batches for ``rank``."""
    if world < 1 or not 0 <= rank < world or n_batches < 0:
        raise ValueError("need world >= 1, 0 <= rank < world, n_batches >= 0")
    base, extra = divmod(n_batches, world)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def _comm_device(group):
    return torch.device("cuda", torch.cuda.current_device()) \
        if dist.get_backend(group) == "nccl" else torch.device("cpu")


def broadcast_templates(U: torch.Tensor, wPCA: torch.Tensor, src: int = 0, group=None):
    """Replicate rank ``src``'s U and wPCA (in place) on every rank."""
    if not (dist.is_available() and dist.is_initialized()):
        return U, wPCA
    dev = _comm_device(group)
    for t in (U, wPCA):
        buf = t.detach().to(dev).contiguous()
        dist.broadcast(buf, src=src, group=group)
        with torch.no_grad():
            t.copy_(buf.to(t.device))
    return U, wPCA


def _gather_rows(st: np.ndarray, tF: torch.Tensor, dst: int, group):
    """Concatenate every rank's (rows, features) on ``dst`` in rank order."""
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    dev = _comm_device(group)
    n = torch.tensor([st.shape[0]], dtype=torch.int64, device=dev)
    counts = [torch.zeros_like(n) for _ in range(world)]
    dist.all_gather(counts, n, group=group)
    counts = [int(c.item()) for c in counts]
    feat_shape = tuple(tF.shape[1:])
    if rank != dst:
        if st.shape[0]:
            dist.send(torch.from_numpy(np.ascontiguousarray(st)).to(dev), dst, group=group)
            dist.send(tF.contiguous().to(dev), dst, group=group)
        return None, None
    rows, feats = [], []
    for r in range(world):
        if counts[r] == 0:
            continue
        if r == rank:
            rows.append(st)
            feats.append(tF)
            continue
        b_st = torch.empty((counts[r], 3), dtype=torch.float64, device=dev)
        b_tf = torch.empty((counts[r],) + feat_shape, dtype=tF.dtype, device=dev)
        dist.recv(b_st, r, group=group)
        dist.recv(b_tf, r, group=group)
        rows.append(b_st.cpu().numpy())
        feats.append(b_tf.cpu())
    if not rows:
        return np.zeros((0, 3)), torch.zeros((0,) + feat_shape)
    return np.concatenate(rows, 0), torch.cat(feats, 0)


def extract_sharded(ops, bfile, U, device=None, dst: int = 0, group=None,
                    match: Optional[Callable] = None, features: Optional[Callable] = None,
                    prepare: Optional[Callable] = None, progress_bar=None):
    """`extract` with the batches split over the ranks of ``group``.

    Returns ``(st, tF, ops)`` on ``dst`` (equal to a single-process
    ``extract``) and ``(None, None, ops)`` on the other ranks; every rank's
    ``ops`` gets ``iCC``, ``iCC_mask`` and ``iU``.  ``match``, ``features``
    and ``prepare`` default to this library's kernels; ``prepare(ops, U)``
    returns ``(iCC, iCC_mask, iU, Ucc, ctc)``.
    """
    distributed = dist.is_available() and dist.is_initialized()
    rank = dist.get_rank(group) if distributed else 0
    world = dist.get_world_size(group) if distributed else 1
    if distributed:
        broadcast_templates(U, ops["wPCA"], src=dst, group=group)
    start, stop = batch_range(int(bfile.n_batches), world, rank)
    batches = np.arange(start, stop, dtype=np.int64)
    bgroup = int(ops.get("batch_group", 4))
    ahead = bool(ops.get("read_ahead", True))
    # this library's matcher: groups of batches per launch, as `extract` does
    grouped = (match is None and features is None and ahead and bgroup > 1
               and len(batches) > 1 and U.is_cuda)
    # this rank's first batches are read while the templates are prepared
    reader = tm._BatchReader(bfile, [int(b) for b in batches], ops, device=U.device,
                             ahead=ahead, depth=bgroup + 1 if grouped else 1)
    try:
        st, tF = _match_range(ops, bfile, batches, U, device, match, features, prepare,
                              progress_bar, reader, bgroup if grouped else 0)
    finally:
        reader.close()
    if distributed:
        st, tF = _gather_rows(st, tF, dst, group)
        if rank != dst:
            return None, None, ops
    st, tF = tm.sort_spikes(st, tF)
    return st, tF, ops


def _match_range(ops, bfile, batches, U, device, match, features, prepare, progress_bar,
                 reader, group=0):
    if prepare is None:
        def prepare(o, Ut):
            iCC, iCC_mask, iU, Ucc = tm.prepare_extract(
                o["xc"], o["yc"], Ut, o["settings"]["nearest_chans"],
                o["settings"]["position_limit"], device=device or Ut.device)
            return iCC, iCC_mask, iU, Ucc, tm.prepare_matching(o, Ut)
    iCC, iCC_mask, iU, Ucc, ctc = prepare(ops, U)
    ops["iCC"], ops["iCC_mask"], ops["iU"] = iCC, iCC_mask, iU
    if match is None or features is None:
        W = ops["wPCA"].contiguous()
        m, f = tm._match_features(ops, W, iCC.to(U.device).contiguous(), iU, Ucc)
        match = match or m
        features = features or f
    if group:
        W = ops["wPCA"].contiguous()
        return tm.extract_grouped(ops, bfile, batches, U, ctc,
                                  (W, iCC.to(U.device).contiguous(), iU, Ucc), group=group,
                                  teams=ops.get("batch_teams"), progress_bar=progress_bar,
                                  reader=reader)
    return tm.extract_batches(ops, bfile, batches, U, ctc, match, features, progress_bar,
                              reader=reader)


def allreduce_gradients(tensors: Sequence[torch.Tensor], group=None):
    """Sum gradients (e.g. U.grad, wPCA.grad of each rank's batches) over ranks, in place."""
    if not (dist.is_available() and dist.is_initialized()):
        return tensors
    dev = _comm_device(group)
    for t in tensors:
        buf = t.detach().to(dev).contiguous()
        dist.all_reduce(buf, op=dist.ReduceOp.SUM, group=group)
        with torch.no_grad():
            t.copy_(buf.to(t.device))
    return tensors
