"""Batched matching (ks_match_batches) against one run_matching call per batch.

The batched path runs the same per-batch arithmetic (same temporal
projection, same contraction tiles and accumulation order, same peel and
residual), only grouped into fewer launches, so every output must be
bit-identical to run_matching's for that batch: spike times and templates,
amplitudes, threshold amplitudes and the residual.
"""
import numpy as np
import pytest
import torch

import kilosort_b200 as kb
from kilosort_b200 import _lib, synth
from kilosort_b200.batched import (BatchedMatcher, Recording, autotune_teams,
                                   match_batches)

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0")


def _recordings():
    """Two template sets with different C, K and nt, uneven batch lengths."""
    a = synth.make_recording(7001, n_chan=96, n_templates=80,
                             batch_lengths=[3000, 12000, 7000, 20000, 1500])
    b = synth.make_recording(7002, n_chan=64, probe="linear", n_templates=130, nt=41,
                             batch_lengths=[5000, 15000, 9000])
    return [a, b]


def _setup(recs, capacity=100000):
    out = []
    for r in recs:
        U = torch.from_numpy(r.U).to(DEV)
        W = torch.from_numpy(r.wPCA).to(DEV)
        ops = dict(Th_learned=8.0, nt=r.nt, max_peels=100, wPCA=W, spike_capacity=capacity)
        ctc = kb.prepare_matching(ops, U)
        out.append((ops, U, ctc, Recording.from_ops(ops, U, ctc)))
    return out


def _items(recs):
    items = []
    for i, r in enumerate(recs):
        for b in range(r.n_batches):
            items.append((torch.from_numpy(np.ascontiguousarray(r.batch(b))).to(DEV), i))
    # interleave the recordings so the tile table and team order are exercised
    return items[::2] + items[1::2]


def _assert_same(res, ref):
    for (st, amps, th, xres), (st_r, amps_r, th_r, xres_r) in zip(res, ref):
        assert torch.equal(st, st_r)
        assert torch.equal(amps, amps_r)
        assert torch.equal(th, th_r)
        assert torch.equal(xres, xres_r)


def _reference(setup, items, projection):
    ref = []
    for X, r in items:
        ops, U, ctc, _ = setup[r]
        ref.append(kb.run_matching(dict(ops, projection=projection), X, U, ctc, device=DEV))
    return ref


@pytest.mark.parametrize("projection", ["fp32", "bf16x3"])
@pytest.mark.parametrize("teams,groups", [(0, 1), (1, 1), (3, 1), (8, 1), (2, 3), (8, 2)])
def test_batched_equals_per_batch(cuda_device, projection, teams, groups):
    recs = _recordings()
    setup = _setup(recs)
    items = _items(recs)
    ref = _reference(setup, items, projection)
    assert sum(len(r[0]) for r in ref) > 100
    res = match_batches([s[3] for s in setup], items, projection=projection, teams=teams,
                        groups=groups)
    _assert_same(res, ref)


def test_overflowing_batch_reports_and_others_complete(cuda_device):
    recs = _recordings()
    setup = _setup(recs)
    items = _items(recs)
    ref = _reference(setup, items, "bf16x3")
    counts = [len(r[0]) for r in ref]
    cap = sorted(counts)[len(counts) // 2]          # about half the batches overflow
    small = [Recording(U=s[3].U, wPCA=s[3].wPCA, ctc=s[3].ctc, Th=8.0, nt=s[3].nt,
                       capacity=cap, ctcT=s[3].ctcT) for s in setup]
    m = BatchedMatcher(small, [(X.shape[1], r) for X, r in items], "bf16x3", teams=2,
                       graph=False)
    for dst, (X, _) in zip(m.X, items):
        dst.copy_(X)
    m.launch()
    info = m.info.cpu().numpy()
    for i, n in enumerate(counts):
        if n > cap:
            assert info[i, 1] == _lib.KS_ERR_OVERFLOW
            assert info[i, 3] >= cap
        else:
            assert info[i, 1] == _lib.KS_OK and info[i, 0] == n
            assert torch.equal(m.outs[i].st[:n], ref[i][0])
    with pytest.raises(RuntimeError, match="capacity"):
        m.results()


@pytest.mark.parametrize("projection,groups", [("fp32", 1), ("bf16x3", 1), ("bf16x3", 3)])
def test_graph_replay_with_new_inputs(cuda_device, projection, groups):
    recs = _recordings()
    setup = _setup(recs)
    items = _items(recs)
    ref = _reference(setup, items, projection)
    m = BatchedMatcher([s[3] for s in setup], [(X.shape[1], r) for X, r in items],
                       projection, teams=4, graph=True, groups=groups)
    # first replay on zeros-scaled inputs, then on the real ones: the graph
    # reads the buffers, not values captured at capture time
    # results are views of the matcher's buffers: keep copies across runs
    res0 = [tuple(t.clone() for t in r) for r in m.run([X * 0.5 for X, _ in items])]
    assert m._graph is not None
    res = m.run([X for X, _ in items])
    _assert_same(res, ref)
    ref_half = _reference(setup, [(X * 0.5, r) for X, r in items], projection)
    _assert_same(res0, ref_half)


def test_autotuner_picks_and_caches(cuda_device):
    recs = _recordings()
    setup = _setup(recs)
    items = _items(recs)
    rs = [s[3] for s in setup]
    t = autotune_teams(rs, items, "bf16x3", candidates=(1, 2, 4), reps=1)
    assert t in (1, 2, 4)
    assert autotune_teams(rs, items, "bf16x3", candidates=(8,), reps=1) == t   # cached
    res = match_batches(rs, items, "bf16x3", teams=t)
    _assert_same(res, _reference(setup, items, "bf16x3"))


@pytest.mark.parametrize("graph", [False, True])
def test_in_place_residual(cuda_device, graph):
    """The residual written over the inputs; with a graph, the warm-up pass
    before capture must not leave its residual as the first run's input."""
    recs = _recordings()
    setup = _setup(recs)
    items = _items(recs)
    ref = _reference(setup, items, "fp32")
    m = BatchedMatcher([s[3] for s in setup], [(X.shape[1], r) for X, r in items],
                       "fp32", teams=2, graph=graph, in_place=True)
    for _ in range(2):
        res = m.run([X for X, _ in items])
        _assert_same(res, ref)
        assert all(res[i][3].data_ptr() == m.X[i].data_ptr() for i in range(len(items)))


def test_host_pipeline_equals_per_batch(cuda_device):
    """Batches in pinned host memory through the pipelined front end: groups
    of 3 alternate between two captured matchers (the last group is short)."""
    from kilosort_b200.batched import HostPipeline
    recs = _recordings()
    setup = _setup(recs)
    items = _items(recs)
    ref = _reference(setup, items, "bf16x3")
    pipe = HostPipeline([s[3] for s in setup], [(X.shape[1], r) for X, r in items], "bf16x3",
                        teams=2, group=3)
    host = [X.cpu().pin_memory() for X, _ in items]
    for _ in range(2):                       # a second run replays the graphs
        res = pipe.run(host)
        for (st, amps, th), (st_r, amps_r, th_r, _) in zip(res, ref):
            assert torch.equal(st, st_r.cpu())
            assert torch.equal(amps, amps_r.cpu())
            assert torch.equal(th, th_r.cpu())


def test_matcher_sequence_equals_separate_matchers(cuda_device):
    """Groups captured in one graph (MatcherSequence, one shared workspace)
    give what each group's own matcher gives."""
    import numpy as np
    import torch
    from kilosort_b200 import synth
    from kilosort_b200.batched import BatchedMatcher, MatcherSequence, Recording, workspace_size
    import kilosort_b200 as kb
    dev = torch.device("cuda:0")
    recs = synth.uneven_recordings(seed=1003, n_batches_total=6)
    mrecs, items = [], []
    for i, r in enumerate(recs):
        U = torch.from_numpy(r.U).to(dev)
        ops = dict(Th_learned=8.0, nt=r.nt, max_peels=100, wPCA=torch.from_numpy(r.wPCA).to(dev))
        mrecs.append(Recording.from_ops(ops, U, kb.prepare_matching(ops, U)))
        for b in range(r.n_batches):
            items.append((torch.from_numpy(np.ascontiguousarray(r.batch(b))).to(dev), i))
    groups = [items[0:3], items[3:6]]
    ws = torch.empty(max(workspace_size(mrecs, g, "bf16x3", 2) for g in groups),
                     dtype=torch.uint8, device=dev)
    seq_m = [BatchedMatcher(mrecs, [(X.shape[1], r) for X, r in g], "bf16x3", teams=2,
                            graph=False, workspace=ws) for g in groups]
    ref_m = [BatchedMatcher(mrecs, [(X.shape[1], r) for X, r in g], "bf16x3", teams=2,
                            graph=True) for g in groups]
    for ms in (seq_m, ref_m):
        for m, g in zip(ms, groups):
            for dst, (X, _) in zip(m.X, g):
                dst.copy_(X)
    seq = MatcherSequence(seq_m)
    seq.launch()
    seq.launch()                     # the graph replay
    got = seq.results()
    want = []
    for m in ref_m:
        m.launch()
        want.extend(m.results())
    assert len(got) == len(want) == 6
    for (st, amps, th, _), (st_r, amps_r, th_r, _) in zip(got, want):
        assert torch.equal(st, st_r) and torch.equal(amps, amps_r) and torch.equal(th, th_r)
