"""The host side of the device batch source for a ``BinaryFiltered``
(kilosort_b200/filtered.py, synth.FilteredBinary), against the reference's own
``BinaryFiltered`` run on the same raw file (tests/golden/golden_filtered.npz,
made by tests/golden/make_golden_filtered.py):

* the stand-in's batch count, cut-back end and batch edges equal the
  reference object's (io.py:646-656, :771-787);
* every padded raw window cut by ``filtered.padded_window`` equals the
  reference's ``BinaryRWFile.padded_batch_to_torch`` window (io.py:789-831)
  sample for sample, first (left pad), middle and ragged last batch;
* a uint16 file gives the same windows as the int16 file it shifts;
* ``filtered.drift_matrix`` and the oracle's ``drift_matrix_ops`` equal the
  reference's ``get_drift_matrix`` (preprocessing.py:44-69) over two blocks
  bit for bit, and the oracle filter of the last
  batch with it matches the reference's filtered batch;
* ``supports`` accepts int16/uint16 BinaryFiltered-like sources only.
"""
import ast
import hashlib

import numpy as np
import pytest
import torch

from kilosort_b200 import filtered, synth
from oracle import preprocess as op
from tests.golden import make_golden_filtered as mk

G = np.load(mk.__file__.replace("make_golden_filtered.py", "golden_filtered.npz"))


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()[:16]


@pytest.fixture(scope="module")
def case():
    rec = synth.make_recording(**ast.literal_eval(str(G["rec_kwargs"])))
    raw = mk.make_raw(rec)
    assert _sha(raw) == str(G["raw_sha"])
    return rec, raw


def _source(raw, **kw):
    return synth.FilteredBinary(raw, NT=int(G["NT"]), nt=61, chan_map=G["chan_map"],
                                whiten_mat=torch.from_numpy(G["W"]), dshift=G["dshift"],
                                device="cpu", **kw)


def _ops():
    return dict(nblocks=2, yblk=G["yblk"], probe=dict(xc=G["xc"], yc=G["yc"]),
                iKxx=torch.from_numpy(G["iKxx"]), settings=dict(sig_interp=float(G["sig_interp"])))


def test_batch_geometry(case):
    _, raw = case
    src = _source(raw)
    assert src.n_batches == int(G["n_batches"])
    assert src.imax == int(G["imax"])
    edges = np.array([src._get_batch_edges(b) for b in range(src.n_batches)])
    np.testing.assert_array_equal(edges, G["edges"])


def test_padded_windows_equal_reference(case):
    _, raw = case
    src = _source(raw)
    L = src.NT + 2 * src.nt
    out = np.empty((L, src.n_chan_bin), np.int16)
    for b in range(src.n_batches):
        out.fill(12345)                 # nothing of a previous batch may survive
        filtered.padded_window(src, b, out)
        assert _sha(out.T) == str(G["window_sha"][b]), b


def test_uint16_file_gives_the_same_windows(case):
    _, raw = case
    u = (raw.astype(np.int32) + 32768).astype(np.uint16)
    a, b = _source(raw), _source(u)
    assert filtered.supports(b) and b.dtype == "uint16"
    L = a.NT + 2 * a.nt
    wa, wb = (np.empty((L, a.n_chan_bin), np.int16) for _ in range(2))
    for i in range(a.n_batches):
        np.testing.assert_array_equal(filtered.padded_window(a, i, wa),
                                      filtered.padded_window(b, i, wb))


def test_threaded_copy_equals_single_copy(case):
    _, raw = case
    src = _source(raw)
    L = src.NT + 2 * src.nt
    wa, wb = (np.empty((L, src.n_chan_bin), np.int16) for _ in range(2))

    def halves(dst, s):             # a copy split as the device source splits it
        h = s.shape[0] // 2
        filtered._copy_samples(dst[:h], s[:h])
        filtered._copy_samples(dst[h:], s[h:])

    for i in range(src.n_batches):
        np.testing.assert_array_equal(filtered.padded_window(src, i, wa),
                                      filtered.padded_window(src, i, wb, copy=halves))


def test_drift_matrix_equals_reference():
    ops = _ops()
    nb = int(G["n_batches"])
    for b, ref in ((0, G["M0"]), (nb - 1, G["Mlast"])):
        M = filtered.drift_matrix(ops, G["dshift"][b], torch.device("cpu"))
        assert M.dtype == torch.float32
        np.testing.assert_array_equal(M.numpy(), ref)           # same torch ops on the CPU
        np.testing.assert_array_equal(op.drift_matrix_ops(ops, G["dshift"][b], "cpu").numpy(),
                                      ref)


def test_oracle_filter_of_last_batch_matches_reference(case):
    _, raw = case
    src = _source(raw)
    nb = src.n_batches
    win = filtered.padded_window(src, nb - 1, np.empty((src.NT + 2 * src.nt, src.n_chan_bin),
                                                         np.int16))
    M = filtered.drift_matrix(_ops(), G["dshift"][nb - 1], torch.device("cpu"))
    X = op.filter_batch(torch.from_numpy(win.T.astype(np.float32)),
                        chan_map=torch.from_numpy(G["chan_map"]), hp=op.highpass_filter(),
                        whiten=torch.from_numpy(G["W"]), drift=M)
    ref = G["Xlast_rows"]
    got = X[:ref.shape[0]].numpy()
    np.testing.assert_allclose(got, ref, rtol=0, atol=1e-5 * np.abs(ref).max())


def test_supports():
    raw = np.zeros((7000, 4), np.int16)
    assert filtered.supports(synth.FilteredBinary(raw, NT=3000))
    s = synth.FilteredBinary(raw, NT=3000)
    s.scale = 0.5
    assert not filtered.supports(s)
    assert not filtered.supports(synth.FilteredBinary(raw.astype(np.float32), NT=3000))
    rec = synth.make_recording(1, n_chan=8, n_templates=4, batch_lengths=[1000])
    assert not filtered.supports(synth.SyntheticBinary(rec))


def test_short_middle_batch_is_an_error():
    raw = np.zeros((9000, 4), np.int16)
    src = synth.FilteredBinary(raw, NT=3000)
    src.file = raw[:5000]               # the file shrank under the object
    with pytest.raises(ValueError):
        filtered.padded_window(src, 1, np.empty((3122, 4), np.int16))


def test_oracle_padded_batch_equals_reference_windows(case):
    _, raw = case
    src = _source(raw)
    for b in range(src.n_batches):
        X = op.padded_batch(src, b, "cpu")
        assert _sha(X.numpy().astype(np.int16)) == str(G["window_sha"][b]), b
    u = _source((raw.astype(np.int32) + 32768).astype(np.uint16))
    assert torch.equal(op.padded_batch(u, 2, "cpu"), op.padded_batch(src, 2, "cpu"))


def test_tiled_samples_repeat_the_base_file():
    base = np.arange(60, dtype=np.int16).reshape(20, 3)
    t = synth.TiledSamples(base, 4)
    full = np.concatenate([base] * 4)
    assert t.shape == full.shape and t.dtype == base.dtype
    for s, e in [(0, 20), (3, 17), (18, 23), (5, 75), (0, 80), (79, 80), (40, 40)]:
        np.testing.assert_array_equal(t[s:e], full[s:e])
    src = synth.FilteredBinary(t, NT=9, nt=2, device="cpu")
    assert src.n_batches == int(np.ceil(80 / 9))


def test_downsampled_batches_match_the_oracle_read(case):
    """batch_downsampling = 2: batch i reads the file's batch 2i (io.py:791, 788),
    through filtered.padded_window and through the oracle's restatement of
    padded_batch_to_torch; the last scaled batch is padded as the reference
    pads the batch whose scaled index is n_batches - 1."""
    _, raw = case
    src = _source(raw, batch_downsampling=2)
    assert src.n_batches == int(G["n_batches"]) // 2
    L = src.NT + 2 * src.nt
    out = np.empty((L, src.n_chan_bin), np.int16)
    for b in range(src.n_batches):
        filtered.padded_window(src, b, out)
        ref = op.padded_batch(src, b, "cpu").numpy()
        np.testing.assert_array_equal(out.T.astype(np.float32), ref)


class _CountingSource:
    """A batch source that records the order of its reads."""

    def __init__(self, n):
        self.n_batches, self.batch_downsampling = n, 1
        self.reads = []

    def padded_batch_to_torch(self, ibatch, ops=None):
        self.reads.append(int(ibatch))
        return torch.full((2, 5), float(ibatch))


@pytest.mark.parametrize("depth", [1, 3, 8])
def test_batch_reader_reads_ahead_in_order(depth):
    """The extract loop's reader hands over the batches in order with up to
    `depth` reads in flight, reads each batch once, and close() leaves no read
    running (a partly consumed reader included)."""
    from kilosort_b200 import template_matching as tm
    src = _CountingSource(7)
    order = [0, 1, 2, 3, 4, 5, 6]
    r = tm._BatchReader(src, order, {}, device=None, ahead=True, depth=depth)
    got = [int(r.get(p)[0, 0]) for p in range(len(order))]
    r.close()
    assert got == order and src.reads == order
    src2 = _CountingSource(7)
    r2 = tm._BatchReader(src2, order, {}, device=None, ahead=True, depth=depth)
    assert int(r2.get(0)[0, 0]) == 0
    r2.close()
    assert not r2.pending and src2.reads == sorted(src2.reads)
    assert len(src2.reads) <= 1 + depth


def test_device_source_signature_follows_the_settings():
    """extract keeps a file's device source while the settings it was built
    from are unchanged: the same object gives the same signature; a new
    channel map, an in-place change of the whitening matrix, or other flags
    give a new one."""
    raw = np.zeros((7000, 6), np.int16)
    W = torch.eye(4)
    src = synth.FilteredBinary(raw, NT=3000, chan_map=np.arange(4), whiten_mat=W)
    sig = filtered._signature(src)
    assert filtered._signature(src) == sig
    src.chan_map = np.arange(4)                   # equal values: the same source
    assert filtered._signature(src) == sig
    src.chan_map = np.array([0, 1, 2, 5])
    assert filtered._signature(src) != sig
    src.chan_map = np.arange(4)
    W.mul_(2.0)                                    # the same tensor, changed in place
    assert filtered._signature(src) != sig
    sig2 = filtered._signature(src)
    src.do_CAR = False
    assert filtered._signature(src) != sig2
