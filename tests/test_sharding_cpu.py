"""Multi-process host logic of kilosort_b200.sharding, on CPU with gloo.

Two ranks split the batches of the golden `extract` case; the per-batch
matcher is the oracle (bit-exact to the reference), so rank 0's merged and
sorted result must equal the reference's own `extract` output bit for bit.
The gradient all-reduce is checked against the gradient of the summed loss.
"""
import ast
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from kilosort_b200 import sharding, synth
from oracle import adjoint as oa
from oracle import matching as om
from tests import golden_util as gu


def test_batch_range_partitions_contiguously():
    for n in (0, 1, 7, 20, 1800):
        for world in (1, 2, 3, 8):
            ranges = [sharding.batch_range(n, world, r) for r in range(world)]
            assert ranges[0][0] == 0 and ranges[-1][1] == n
            for (a, b), (c, d) in zip(ranges, ranges[1:]):
                assert b == c
            sizes = [b - a for a, b in ranges]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        sharding.batch_range(5, 2, 2)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _golden_case():
    g = gu.load("extract")
    kw = ast.literal_eval(str(g["seed_kwargs"]))
    rec = synth.make_recording(**kw)
    assert gu.sha(rec.signal) == str(g["signal_sha"])
    return g, rec


def _oracle_fns(rec, ops):
    U = torch.from_numpy(rec.U)
    W = torch.from_numpy(rec.wPCA)
    nt = ops["nt"]
    iCC, mask, iU, Ucc = om.prepare_extract(rec.xc, rec.yc, U, 10, 100)
    ctc = om.prepare_matching(ops, U)

    def prepare(o, Ut):
        return iCC, mask, iU, Ucc, ctc

    def match(X, Ut, c, device):
        return om.run_matching(ops, X, Ut, c)

    def features(Xres, st, amps):
        return om.spike_features(Xres, st, amps, W, iCC, iU, Ucc, nt).transpose(0, 1)
    return prepare, match, features


def _ops(rec):
    return dict(Th_learned=8.0, nt=61, max_peels=100, wPCA=torch.from_numpy(rec.wPCA),
                nt0min=20, batch_size=3000, xc=rec.xc, yc=rec.yc,
                settings=dict(nearest_chans=10, position_limit=100, n_pcs=6))


def _extract_worker(rank, world, port, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    try:
        torch.set_num_threads(2)
        _, rec = _golden_case()
        ops = _ops(rec)
        prepare, match, features = _oracle_fns(rec, ops)
        bfile = synth.SyntheticBinary(rec, device="cpu")
        U = torch.from_numpy(rec.U).clone()
        if rank != 0:
            U.zero_()               # replaced by rank 0's templates (broadcast)
        st, tF, ops = sharding.extract_sharded(ops, bfile, U, device="cpu", prepare=prepare,
                                               match=match, features=features)
        if rank == 0:
            np.save(os.path.join(out_dir, "st.npy"), st)
            np.save(os.path.join(out_dir, "tF.npy"), tF.numpy())
        else:
            assert st is None and tF is None
            assert torch.equal(U, torch.from_numpy(rec.U))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_sharded_extract_equals_reference_extract(tmp_path):
    g, _ = _golden_case()
    mp.start_processes(_extract_worker, args=(2, _free_port(), str(tmp_path)), nprocs=2,
                       join=True, start_method="spawn")
    st = np.load(tmp_path / "st.npy")
    tF = np.load(tmp_path / "tF.npy")
    np.testing.assert_array_equal(st, g["st"])
    np.testing.assert_array_equal(tF, g["tF"])


def test_single_process_sharded_extract_equals_reference_extract():
    g, rec = _golden_case()
    ops = _ops(rec)
    prepare, match, features = _oracle_fns(rec, ops)
    st, tF, _ = sharding.extract_sharded(ops, synth.SyntheticBinary(rec, device="cpu"),
                                         torch.from_numpy(rec.U), device="cpu",
                                         prepare=prepare, match=match, features=features)
    np.testing.assert_array_equal(st, g["st"])
    np.testing.assert_array_equal(tF.numpy(), g["tF"])


def _grad_worker(rank, world, port, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    try:
        U, W, batches = _grad_case()
        X, st, amps = batches[rank]
        Ud = U.clone().requires_grad_(True)
        Wd = W.clone().requires_grad_(True)
        oa.recon_loss(X, st, amps, Ud, Wd).backward()
        sharding.allreduce_gradients([Ud.grad, Wd.grad])
        np.save(os.path.join(out_dir, f"dU{rank}.npy"), Ud.grad.numpy())
        np.save(os.path.join(out_dir, f"dW{rank}.npy"), Wd.grad.numpy())
        dist.barrier()
    finally:
        dist.destroy_process_group()


def _grad_case():
    rec = synth.make_recording(5151, n_chan=32, n_templates=12, batch_lengths=[2000, 2000])
    U = torch.from_numpy(rec.U).double()
    W = torch.from_numpy(rec.wPCA).double()
    rng = np.random.default_rng(3)
    batches = []
    for b in range(2):
        X = torch.from_numpy(np.ascontiguousarray(rec.batch(b))).double()
        n = 40
        st = torch.stack([torch.from_numpy(rng.integers(61, X.shape[1] - 61, n)),
                          torch.from_numpy(rng.integers(0, U.shape[0], n))], 1)
        amps = torch.from_numpy(rng.uniform(5, 20, n))
        batches.append((X, st, amps))
    return U, W, batches


def test_gradient_allreduce_equals_gradient_of_summed_loss(tmp_path):
    mp.start_processes(_grad_worker, args=(2, _free_port(), str(tmp_path)), nprocs=2,
                       join=True, start_method="spawn")
    U, W, batches = _grad_case()
    Ud = U.clone().requires_grad_(True)
    Wd = W.clone().requires_grad_(True)
    sum(oa.recon_loss(X, st, a, Ud, Wd) for X, st, a in batches).backward()
    for r in range(2):
        np.testing.assert_allclose(np.load(tmp_path / f"dU{r}.npy"), Ud.grad.numpy(),
                                   rtol=1e-12, atol=1e-9)
        np.testing.assert_allclose(np.load(tmp_path / f"dW{r}.npy"), Wd.grad.numpy(),
                                   rtol=1e-12, atol=1e-9)


class _CountingSource:
    """A batch source that records the order of reads and can fail on one."""

    def __init__(self, n, fail_at=None):
        self.n_batches, self.batch_downsampling = n, 1
        self.reads, self.fail_at = [], fail_at

    def padded_batch_to_torch(self, ibatch, ops=None):
        self.reads.append(int(ibatch))
        if ibatch == self.fail_at:
            raise OSError(f"cannot read batch {ibatch}")
        return torch.full((2, 5), float(ibatch))


@pytest.mark.parametrize("ahead", [False, True])
def test_batch_reader_order_and_errors(ahead):
    from kilosort_b200.template_matching import _BatchReader
    src = _CountingSource(6)
    r = _BatchReader(src, [3, 4, 5], None, device="cpu", ahead=ahead)
    assert [r.get(i)[0, 0].item() for i in range(3)] == [3.0, 4.0, 5.0]
    r.close()
    assert src.reads == [3, 4, 5]
    src = _CountingSource(6, fail_at=1)
    r = _BatchReader(src, range(4), None, device="cpu", ahead=ahead)
    assert r.get(0)[0, 0].item() == 0.0
    with pytest.raises(OSError, match="batch 1"):
        r.get(1)
    r.close()


def test_extract_read_ahead_equals_reference_extract():
    """extract_batches with and without the read-ahead reader give the
    reference's own extract output (oracle matcher, CPU)."""
    from kilosort_b200 import template_matching as tm
    g, rec = _golden_case()
    ops = _ops(rec)
    _, match, features = _oracle_fns(rec, ops)
    U = torch.from_numpy(rec.U)
    ctc = om.prepare_matching(ops, U)
    batches = np.arange(synth.SyntheticBinary(rec).n_batches, dtype=np.int64)
    for ahead in (False, True):
        st, tF = tm.extract_batches(ops, synth.SyntheticBinary(rec, device="cpu"), batches, U,
                                    ctc, match, features, read_ahead=ahead)
        st, tF = tm.sort_spikes(st, tF)
        np.testing.assert_array_equal(st, g["st"])
        np.testing.assert_array_equal(tF.numpy(), g["tF"])


class _RefillingSource(synth.SyntheticBinary):
    """A batch source that refills one buffer on every call."""

    def padded_batch_to_torch(self, ibatch, ops=None):
        x = torch.from_numpy(np.ascontiguousarray(self.rec.batch(int(ibatch))))
        if not hasattr(self, "_buf"):
            self._buf = torch.empty_like(x)
        return self._buf.copy_(x)


def test_refilling_source_without_read_ahead_equals_reference_extract():
    g, rec = _golden_case()
    ops = dict(_ops(rec), read_ahead=False)
    prepare, match, features = _oracle_fns(rec, ops)
    st, tF, _ = sharding.extract_sharded(ops, _RefillingSource(rec, device="cpu"),
                                         torch.from_numpy(rec.U), device="cpu",
                                         prepare=prepare, match=match, features=features)
    np.testing.assert_array_equal(st, g["st"])
    np.testing.assert_array_equal(tF.numpy(), g["tF"])
