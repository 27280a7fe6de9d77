"""Many batches of several recordings per launch sequence (``ks_match_batches``).

The reference matches one padded batch per ``run_matching`` call
(kilosort/template_matching.py:79-84, the loop of ``extract``).  Here a whole
group of batches -- up to 256, of up to 8 recordings (template sets), of any
lengths -- goes through one grouped tensor-core contraction, one cooperative
peel launch whose grid is split into teams of co-resident blocks, and one
residual launch.  Each batch gets exactly what ``run_matching`` returns for it.

* ``Recording``      one template set: U, wPCA, ctc (transposed once), Th, nt,
                     max_peels, spike capacity per batch
* ``match_batches``  one call over a list of ``(X, recording index)``
* ``BatchedMatcher`` fixed shapes: preallocated inputs, outputs and workspace,
                     optionally captured once in a CUDA graph and replayed
* ``autotune_teams`` times candidate team counts on the device and caches the
                     fastest per workload signature; ``autotune_schedule``
                     also picks the number of pipelined groups
* ``MatcherSequence`` several matchers in turn (one shared workspace) captured
                     in one CUDA graph: a long workload's pass is one launch
* ``HostPipeline``   batches in host memory: two captured matchers alternate
                     so transfers and read-back overlap the matching
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence, Tuple

import torch

from . import _lib
from .template_matching import (DEFAULT_CAPACITY, _PROJECTIONS, _need, _ptr, _stream,
                                th2_of, transpose_ctc)


@dataclass
class Recording:
    """A template set and its peel settings (one ``ks_rec_desc``)."""

    U: torch.Tensor
    wPCA: torch.Tensor
    ctc: torch.Tensor
    Th: float
    nt: int
    max_peels: int = 100
    capacity: int = DEFAULT_CAPACITY
    ctcT: Optional[torch.Tensor] = field(default=None, repr=False)

    def __post_init__(self):
        self.U = _need(self.U, "U", ndim=3)
        self.wPCA = _need(self.wPCA, "wPCA", ndim=2)
        self.ctc = _need(self.ctc, "ctc", ndim=3)
        K, P, _ = self.U.shape
        if self.wPCA.shape != (P, self.nt):
            raise ValueError(f"wPCA must be [{P}, {self.nt}], got {tuple(self.wPCA.shape)}")
        if self.ctc.shape != (K, K, 2 * self.nt + 1):
            raise ValueError("shape mismatch between U and ctc")
        if self.ctcT is None:
            self.ctcT = transpose_ctc(self.ctc, self.nt)

    @classmethod
    def from_ops(cls, ops, U, ctc, capacity=None):
        cap = int(ops.get("spike_capacity", DEFAULT_CAPACITY)) if capacity is None else capacity
        return cls(U=U, wPCA=ops["wPCA"], ctc=ctc, Th=ops["Th_learned"], nt=int(ops["nt"]),
                   max_peels=int(ops["max_peels"]), capacity=cap)

    @property
    def shape(self):
        K, P, Cn = self.U.shape
        return Cn, K, P

    def desc(self) -> _lib.RecDesc:
        Cn, K, P = self.shape
        return _lib.RecDesc(_ptr(self.U), _ptr(self.wPCA), _ptr(self.ctcT), Cn, K, P, self.nt,
                            th2_of(self.Th), int(self.max_peels), int(self.capacity))


class _Outputs:
    """Device outputs of one batch."""

    def __init__(self, rec: Recording, Cn: int, L: int, device, Xres=None):
        cap = int(rec.capacity)
        self.st = torch.empty((cap, 2), dtype=torch.int64, device=device)
        self.amps = torch.empty((cap, 1), dtype=torch.float32, device=device)
        self.th_amps = torch.empty((cap, 1), dtype=torch.float32, device=device)
        self.Xres = torch.empty((Cn, L), dtype=torch.float32, device=device) if Xres is None else Xres


def _check_group(recs: Sequence[Recording], items: Sequence[Tuple[torch.Tensor, int]]):
    if not 1 <= len(recs) <= _lib.KS_MAX_RECORDINGS:
        raise ValueError(f"1..{_lib.KS_MAX_RECORDINGS} recordings per call")
    if not 1 <= len(items) <= _lib.KS_MAX_BATCHES:
        raise ValueError(f"1..{_lib.KS_MAX_BATCHES} batches per call")
    dev = recs[0].U.device
    for X, r in items:
        if not 0 <= r < len(recs):
            raise ValueError(f"recording index {r} out of range")
        X = _need(X, "X", ndim=2)
        if X.shape[0] != recs[r].shape[0]:
            raise ValueError(f"batch has {X.shape[0]} channels, recording {r} has {recs[r].shape[0]}")
        if X.device != dev:
            raise ValueError("all tensors must be on one device")
    return dev


def _descs(recs, items, outs, info):
    rd = (_lib.RecDesc * len(recs))(*[r.desc() for r in recs])
    bd = (_lib.BatchDesc * len(items))()
    for i, ((X, r), o) in enumerate(zip(items, outs)):
        bd[i] = _lib.BatchDesc(_ptr(X), _ptr(o.Xres), X.shape[1], r, _ptr(o.st), _ptr(o.amps),
                               _ptr(o.th_amps), _ptr(info[i]))
    return rd, bd


def workspace_size(recs, items, projection="bf16x3", teams=0) -> int:
    rd = (_lib.RecDesc * len(recs))(*[r.desc() for r in recs])
    bd = (_lib.BatchDesc * len(items))()
    for i, (X, r) in enumerate(items):
        # pointers are not read by the size query; shapes are
        bd[i] = _lib.BatchDesc(1, 1, X.shape[1], r, 1, 1, 1, 1)
    n = _lib.load().ks_match_batches_workspace_size(C.byref(rd), len(recs), C.byref(bd),
                                                    len(items), _PROJECTIONS[projection],
                                                    int(teams))
    if n == 0:
        raise _lib.KilosortB200Error(_lib.KS_ERR_ARG, "ks_match_batches_workspace_size: "
                                     + _lib.load().ks_last_error().decode(errors="replace"))
    return n


def _launch(recs, items, outs, info, ws, projection, teams, groups=1, aux=None):
    rd, bd = _descs(recs, items, outs, info)
    lib = _lib.load()
    _lib.check(lib.ks_match_batches(C.byref(rd), len(recs), C.byref(bd), len(items),
                                    _PROJECTIONS[projection], int(teams), int(groups),
                                    _ptr(ws), ws.numel(), _stream(ws.device),
                                    aux.cuda_stream if (aux is not None and groups > 1) else None),
               "ks_match_batches")


def _results(outs, info, what="ks_match_batches"):
    """(st, amps, th_amps, Xres) per batch; raises on the first failed batch."""
    host = info.cpu().tolist()
    res = []
    for i, (o, (n, status, _it, need)) in enumerate(zip(outs, host)):
        if status == _lib.KS_ERR_OVERFLOW:
            raise RuntimeError(f"{what}: batch {i} needs {need} spikes, above the capacity "
                               f"{o.st.shape[0]} of its recording")
        if status != _lib.KS_OK:
            raise _lib.KilosortB200Error(status, f"{what}: batch {i}: device status {status}")
        res.append((o.st[:n], o.amps[:n], o.th_amps[:n], o.Xres))
    return res


def match_batches(recs: Sequence[Recording], items: Sequence[Tuple[torch.Tensor, int]],
                  projection: str = "bf16x3", teams: int = 0, groups: int = 1):
    """Match every ``(X, recording index)`` of ``items``.

    Returns a list of ``(st, amps, th_amps, Xres)``, one per batch, equal to
    what ``run_matching`` returns for that batch alone.  Groups larger than
    256 batches are split into consecutive calls.  ``groups`` > 1 pipelines
    the projections of one group of batches with the peel of the previous
    one on a second stream.
    """
    recs = list(recs)
    items = [(_need(X, "X", ndim=2), int(r)) for X, r in items]
    out = []
    for g0 in range(0, len(items), _lib.KS_MAX_BATCHES):
        grp = items[g0:g0 + _lib.KS_MAX_BATCHES]
        dev = _check_group(recs, grp)
        outs = [_Outputs(recs[r], X.shape[0], X.shape[1], dev) for X, r in grp]
        info = torch.empty((len(grp), 4), dtype=torch.int64, device=dev)
        ws = torch.empty(workspace_size(recs, grp, projection, teams), dtype=torch.uint8,
                         device=dev)
        aux = torch.cuda.Stream(dev) if groups > 1 else None
        _launch(recs, grp, outs, info, ws, projection, teams, groups, aux)
        out.extend(_results(outs, info))
    return out


# ------------------------------------------------------------------ autotuner
_TEAMS_CACHE: Dict[tuple, int] = {}


def _signature(recs, lengths_recs, projection):
    dev = recs[0].U.device
    return (torch.cuda.get_device_name(dev), projection,
            tuple((r.shape, r.nt, int(r.max_peels)) for r in recs),
            tuple(sorted(lengths_recs)))


def autotune_teams(recs: Sequence[Recording], items: Sequence[Tuple[torch.Tensor, int]],
                   projection: str = "bf16x3", candidates=(1, 2, 4, 8, 16, 32),
                   reps: int = 2, groups: int = 1) -> int:
    """Fastest team count for this workload, timed with CUDA events.

    Every candidate runs the full call (warm-up once, then ``reps`` timed
    runs); the winner is cached per (device, projection, template-set shapes,
    batch lengths) so later calls with the same signature skip the search.
    """
    recs = list(recs)
    items = [(_need(X, "X", ndim=2), int(r)) for X, r in items]
    key = _signature(recs, [(X.shape[1], r) for X, r in items], projection) + (groups,)
    if key in _TEAMS_CACHE:
        return _TEAMS_CACHE[key]
    dev = _check_group(recs, items)
    outs = [_Outputs(recs[r], X.shape[0], X.shape[1], dev) for X, r in items]
    info = torch.empty((len(items), 4), dtype=torch.int64, device=dev)
    cands = [t for t in candidates if 1 <= t <= len(items)] or [1]
    ws = torch.empty(max(workspace_size(recs, items, projection, t) for t in cands),
                     dtype=torch.uint8, device=dev)
    best, best_ms = cands[0], float("inf")
    aux = torch.cuda.Stream(dev) if groups > 1 else None
    for t in cands:
        _launch(recs, items, outs, info, ws, projection, t, groups, aux)
        _results(outs, info, "autotune_teams")
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            _launch(recs, items, outs, info, ws, projection, t, groups, aux)
        e1.record()
        torch.cuda.synchronize(dev)
        _results(outs, info, "autotune_teams")
        ms = e0.elapsed_time(e1) / reps
        if ms < best_ms:
            best, best_ms = t, ms
    _TEAMS_CACHE[key] = best
    return best


def autotune_schedule(recs: Sequence[Recording], items: Sequence[Tuple[torch.Tensor, int]],
                      projection: str = "bf16x3", teams=(4, 8, 16, 20), groups=(1, 2, 4),
                      reps: int = 2) -> Tuple[int, int]:
    """Fastest (teams, groups) pair: teams tuned per group count, then the
    group counts compared on their best team count (CUDA-event timing)."""
    best = None
    for g in groups:
        if g > len(items):
            continue
        t = autotune_teams(recs, items, projection, candidates=teams, reps=reps, groups=g)
        ms = _time_schedule(recs, items, projection, t, g, reps)
        if best is None or ms < best[0]:
            best = (ms, t, g)
    return best[1], best[2]


def _time_schedule(recs, items, projection, teams, groups, reps):
    items = [(_need(X, "X", ndim=2), int(r)) for X, r in items]
    dev = _check_group(list(recs), items)
    outs = [_Outputs(recs[r], X.shape[0], X.shape[1], dev) for X, r in items]
    info = torch.empty((len(items), 4), dtype=torch.int64, device=dev)
    ws = torch.empty(workspace_size(recs, items, projection, teams), dtype=torch.uint8, device=dev)
    aux = torch.cuda.Stream(dev) if groups > 1 else None
    _launch(recs, items, outs, info, ws, projection, teams, groups, aux)
    _results(outs, info, "autotune_schedule")
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        _launch(recs, items, outs, info, ws, projection, teams, groups, aux)
    e1.record()
    torch.cuda.synchronize(dev)
    return e0.elapsed_time(e1) / reps


# ------------------------------------------------------------------ fixed shapes
class BatchedMatcher:
    """Repeated matching of batches with fixed shapes, optionally as a CUDA graph.

    ``lengths`` lists ``(L, recording index)`` per batch.  The matcher owns
    input buffers ``X[i]`` (fill them, e.g. ``X[i].copy_(pinned, non_blocking=True)``),
    outputs and workspace, so the launch sequence can be captured once
    (``graph=True``) and replayed with no per-call host work beyond the replay.
    ``teams=None`` runs the autotuner on the first inputs given to ``run``.
    """

    def __init__(self, recs: Sequence[Recording], lengths: Sequence[Tuple[int, int]],
                 projection: str = "bf16x3", teams: Optional[int] = 0, graph: bool = True,
                 in_place: bool = False, workspace: Optional[torch.Tensor] = None,
                 groups: int = 1):
        if projection not in _PROJECTIONS:
            raise ValueError(f"projection must be one of {sorted(_PROJECTIONS)}")
        if len(lengths) > _lib.KS_MAX_BATCHES:
            raise ValueError(f"at most {_lib.KS_MAX_BATCHES} batches")
        self.recs = list(recs)
        self.projection = projection
        self.graph_enabled = graph
        dev = self.recs[0].U.device
        self.device = dev
        self.X = [torch.zeros((self.recs[r].shape[0], int(L)), dtype=torch.float32, device=dev)
                  for L, r in lengths]
        self.items = [(X, int(r)) for X, (_, r) in zip(self.X, lengths)]
        _check_group(self.recs, self.items)
        self.outs = [_Outputs(self.recs[r], X.shape[0], X.shape[1], dev,
                              Xres=X if in_place else None) for X, r in self.items]
        self.info = torch.empty((len(self.items), 4), dtype=torch.int64, device=dev)
        self.teams = teams
        self.groups = max(1, int(groups))
        self._aux = torch.cuda.Stream(dev) if self.groups > 1 else None
        # matchers whose launches never overlap (one stream) may share one
        # workspace of the largest size they need (workspace_bytes())
        self._ws = workspace
        self._graph = None

    def workspace_bytes(self, teams: Optional[int] = None) -> int:
        t = self.teams if teams is None else teams
        return workspace_size(self.recs, self.items, self.projection, 0 if t is None else t)

    def _prepare(self):
        if self.teams is None:
            self.teams = autotune_teams(self.recs, self.items, self.projection,
                                        groups=self.groups)
        need = workspace_size(self.recs, self.items, self.projection, self.teams)
        if self._ws is None:
            self._ws = torch.empty(need, dtype=torch.uint8, device=self.device)
        elif self._ws.numel() < need or self._ws.device != self.device:
            raise ValueError(f"shared workspace holds {self._ws.numel()} bytes, need {need}")

    def launch(self):
        """Enqueue one matching pass on the current stream (no host sync)."""
        self._prepare()
        if self.graph_enabled:
            if self._graph is None:
                # warm-up: first-use set-up out of capture; a residual written
                # in place overwrites the inputs, so they are put back after it
                saved = [X.clone() for X, o in zip(self.X, self.outs) if o.Xres is X]
                self._enqueue()
                for X, s in zip((X for X, o in zip(self.X, self.outs) if o.Xres is X), saved):
                    X.copy_(s)
                del saved
                torch.cuda.synchronize(self.device)
                g = torch.cuda.CUDAGraph()
                s = torch.cuda.Stream(self.device)
                s.wait_stream(torch.cuda.current_stream(self.device))
                with torch.cuda.stream(s):
                    g.capture_begin(capture_error_mode="thread_local")
                    try:
                        self._enqueue()
                    finally:
                        g.capture_end()
                torch.cuda.current_stream(self.device).wait_stream(s)
                self._graph = g
            self._graph.replay()
        else:
            self._enqueue()

    def _enqueue(self):
        _launch(self.recs, self.items, self.outs, self.info, self._ws, self.projection,
                self.teams, self.groups, self._aux)

    def launch_eager(self):
        """Enqueue one pass without the graph (for stage tracing or debugging)."""
        self._prepare()
        self._enqueue()

    def results(self):
        """Per batch ``(st, amps, th_amps, Xres)`` (synchronises to read the status).

        The tensors are views of the matcher's own buffers: the next launch
        overwrites them (clone what must outlive it).
        """
        return _results(self.outs, self.info)

    def run(self, Xs: Optional[Sequence[torch.Tensor]] = None):
        if Xs is not None:
            if len(Xs) != len(self.X):
                raise ValueError(f"expected {len(self.X)} batches")
            for dst, src in zip(self.X, Xs):
                dst.copy_(src, non_blocking=True)
        self.launch()
        return self.results()


class MatcherSequence:
    """Several BatchedMatchers run one after another on one stream (for
    instance the groups of a long uneven workload sharing one workspace),
    captured in one CUDA graph: a whole pass is one graph launch.

    Each matcher runs once eagerly first (first-use set-up and autotuning stay
    out of the capture); a matcher whose residual is written in place gets its
    inputs put back after that run.
    """

    def __init__(self, matchers: Sequence["BatchedMatcher"]):
        self.matchers = list(matchers)
        if not self.matchers:
            raise ValueError("no matchers")
        self.device = self.matchers[0].device
        self._graph = None

    def launch(self):
        if self._graph is None:
            for m in self.matchers:
                saved = [X.clone() for X, o in zip(m.X, m.outs) if o.Xres is X]
                m.launch_eager()
                for X, sv in zip((X for X, o in zip(m.X, m.outs) if o.Xres is X), saved):
                    X.copy_(sv)
            torch.cuda.synchronize(self.device)
            g = torch.cuda.CUDAGraph()
            s = torch.cuda.Stream(self.device)
            s.wait_stream(torch.cuda.current_stream(self.device))
            with torch.cuda.stream(s):
                g.capture_begin(capture_error_mode="thread_local")
                try:
                    for m in self.matchers:
                        m._enqueue()
                finally:
                    g.capture_end()
            torch.cuda.current_stream(self.device).wait_stream(s)
            self._graph = g
        self._graph.replay()

    def results(self):
        return [r for m in self.matchers for r in m.results()]


class HostPipeline:
    """Match batches held in host memory, transfers overlapped with matching.

    The batches are split into consecutive groups whose sizes ramp 1, 2, 4, ...
    up to ``group`` (the first launch waits for one batch's copy instead of a
    whole group's); two captured ``BatchedMatcher`` graphs alternate, so while
    group g is matched the
    copies of group g+1 into the other matcher's inputs (copy stream) and
    the read-back of group g-1's spikes (read-back stream) proceed.  Host
    batches should be page-locked (``pin_memory``) for the copies to be
    asynchronous.  ``run`` returns per batch ``(st, amps, th_amps)`` on the
    host, in input order, equal to what ``run_matching`` returns for that
    batch.
    """

    def __init__(self, recs: Sequence[Recording], lengths: Sequence[Tuple[int, int]],
                 projection: str = "bf16x3", teams: Optional[int] = 0, group: int = 5):
        self.recs = list(recs)
        self.lengths = [(int(L), int(r)) for L, r in lengths]
        self.projection = projection
        self.teams = teams
        self.group = max(1, int(group))
        self.device = self.recs[0].U.device
        n = len(self.lengths)
        self.groups, b0, size = [], 0, 1
        while b0 < n:
            k = min(size, self.group, n - b0)
            self.groups.append(list(range(b0, b0 + k)))
            b0 += k
            size *= 2
        self._matchers = {}
        self.copy = torch.cuda.Stream(self.device)
        self.readback = torch.cuda.Stream(self.device)
        self.copied = [torch.cuda.Event() for _ in range(2)]
        self.done = [torch.cuda.Event() for _ in range(2)]

    def _matcher(self, g: int) -> BatchedMatcher:
        shape = tuple(self.lengths[b] for b in self.groups[g])
        key = (g % 2, shape)
        if key not in self._matchers:
            self._matchers[key] = BatchedMatcher(self.recs, list(shape), self.projection,
                                                 teams=self.teams, graph=True)
        return self._matchers[key]

    def run(self, Xh: Sequence[torch.Tensor]):
        if len(Xh) != len(self.lengths):
            raise ValueError(f"expected {len(self.lengths)} batches, got {len(Xh)}")
        ms = [self._matcher(g) for g in range(len(self.groups))]
        cur = torch.cuda.current_stream(self.device)
        out = [None] * len(Xh)

        def enqueue_copy(g):
            m = ms[g]
            with torch.cuda.stream(self.copy):
                # the matcher's previous launch has finished reading its inputs
                self.copy.wait_event(self.done[g % 2])
                for i, b in enumerate(self.groups[g]):
                    m.X[i].copy_(Xh[b], non_blocking=True)
                self.copied[g % 2].record(self.copy)

        def collect(g):
            m = ms[g]
            with torch.cuda.stream(self.readback):
                self.readback.wait_event(self.done[g % 2])
                info = m.info.to("cpu", non_blocking=True)
                self.readback.synchronize()
                host = []
                for i, b in enumerate(self.groups[g]):
                    n, status, _, need = (int(v) for v in info[i].tolist())
                    if status == _lib.KS_ERR_OVERFLOW:
                        raise RuntimeError(f"HostPipeline: batch {b} needs {need} spikes, above "
                                           f"the capacity {m.outs[i].st.shape[0]}")
                    if status != _lib.KS_OK:
                        raise _lib.KilosortB200Error(status, f"HostPipeline: batch {b}: "
                                                     f"device status {status}")
                    o = m.outs[i]
                    host.append((b, o.st[:n].to("cpu", non_blocking=True),
                                 o.amps[:n].to("cpu", non_blocking=True),
                                 o.th_amps[:n].to("cpu", non_blocking=True)))
                self.readback.synchronize()
            for b, st, amps, th in host:
                out[b] = (st, amps, th)

        if self.groups:
            enqueue_copy(0)
        for g in range(len(self.groups)):
            if g + 1 < len(self.groups):
                enqueue_copy(g + 1)
            cur.wait_event(self.copied[g % 2])
            ms[g].launch()
            self.done[g % 2].record(cur)
            if g >= 1:
                collect(g - 1)
        if self.groups:
            collect(len(self.groups) - 1)
        return out
