"""``extract`` over a ``BinaryFiltered``-style int16 file, through the device
batch source (kilosort_b200/filtered.py: pinned raw windows, int16 copies,
``ks_preprocess_int16`` with the drift matrix folded into the whitening).

* Golden case (tests/golden/golden_filtered.npz: the reference's own
  ``extract`` over its own ``BinaryFiltered`` on the same raw file; 64
  channels on a permutation of 66 file channels, high-pass, whitening, drift
  over two blocks, six batches with a ragged last one): >= 99.5 % exact
  (time, template) agreement; on the matched spikes th_amp within 2e-3 and
  features within 2e-3 of their maximum.  The device filter is not the
  reference's Fourier-domain arithmetic (a 1023-tap circular correlation, the
  whitening in split BF16): the filtered batch agrees to 1e-4 of its maximum
  (test_gpu_preprocess.py), which moves amplitudes by up to ~1e-3.
* Full size (385 file channels, 384 mapped, K = 600, NT = 60000, two full
  batches and a ragged tail, one-block drift): the device batch source
  against the same ``extract`` fed by the oracle restatement of the
  reference's batch filter on the GPU (``ops['device_filter'] = False``),
  same bar.
* A uint16 file gives bit-identical output to the int16 file it shifts, and
  reading ahead changes nothing.
"""
import ast

import numpy as np
import pytest
import torch

import kilosort_b200 as kb
from kilosort_b200 import filtered, synth
from kilosort_b200.preprocess import highpass_filter
from oracle import preprocess as op
from tests.golden import make_golden_filtered as mk
from tests.parity_util import agreement

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0")
G = np.load(mk.__file__.replace("make_golden_filtered.py", "golden_filtered.npz"))
AMP_TOL = 2e-3
TF_TOL = 2e-3


class _NoTF32:
    def __enter__(self):
        self.flags = (torch.backends.cudnn.allow_tf32, torch.backends.cuda.matmul.allow_tf32)
        torch.backends.cudnn.allow_tf32 = False
        torch.backends.cuda.matmul.allow_tf32 = False

    def __exit__(self, *a):
        torch.backends.cudnn.allow_tf32, torch.backends.cuda.matmul.allow_tf32 = self.flags


class _OracleFiltered(synth.FilteredBinary):
    """The same file read the reference's way: the padded window as float32
    on the device, then the oracle's restatement of ``BinaryFiltered.filter``
    (torch FFT high-pass, ``(M @ whiten_mat) @ X``)."""

    def padded_batch_to_torch(self, ibatch, ops=None):
        with _NoTF32():
            return op.filtered_batch(self, ibatch, ops, self.device)


def _golden_case():
    rec = synth.make_recording(**ast.literal_eval(str(G["rec_kwargs"])))
    raw = mk.make_raw(rec)
    ops = dict(Th_learned=8.0, nt=61, max_peels=100, wPCA=torch.from_numpy(rec.wPCA).to(DEV),
               nt0min=20, batch_size=int(G["NT"]), xc=G["xc"], yc=G["yc"], nblocks=2,
               yblk=G["yblk"], probe=dict(xc=G["xc"], yc=G["yc"]),
               iKxx=torch.from_numpy(G["iKxx"]).to(DEV),
               settings=dict(nearest_chans=10, position_limit=100, n_pcs=6,
                             sig_interp=float(G["sig_interp"])))
    return rec, raw, ops


def _source(raw, cls=synth.FilteredBinary):
    return cls(raw, NT=int(G["NT"]), nt=61, chan_map=G["chan_map"], hp_filter=highpass_filter(),
               whiten_mat=torch.from_numpy(G["W"]), dshift=G["dshift"], device=DEV)


def _count_device_batches(monkeypatch):
    calls = []
    orig = filtered.FilteredBatches.batch

    def batch(self, ibatch, ops=None, out=None):
        calls.append(int(ibatch))
        return orig(self, ibatch, ops, out)

    monkeypatch.setattr(filtered.FilteredBatches, "batch", batch)
    return calls


def _compare(st, tF, st_r, tF_r, what):
    # extract sorts by time with numpy's default (unstable) argsort, as the
    # reference does, so spikes at one time may come in either order; sorted by
    # (time, template, amplitude), a (time, template) pair found twice pairs
    # with its counterpart by amplitude rank
    o = np.lexsort((st[:, 2], st[:, 1], st[:, 0]))
    o_r = np.lexsort((st_r[:, 2], st_r[:, 1], st_r[:, 0]))
    st, st_r = st[o], st_r[o_r]
    a = agreement(st[:, :2], st_r[:, :2], st[:, 2], st_r[:, 2])
    assert a["n_r"] > 0 and a["agreement"] >= 0.995, (what, a)
    assert a["amp_rel_p999"] <= AMP_TOL, (what, a)
    if a["matched"] == len(st) == len(st_r):
        np.testing.assert_array_equal(st[:, :2], st_r[:, :2])
        tF_r = torch.as_tensor(tF_r)[torch.from_numpy(o_r)]
        d = (tF[torch.from_numpy(o)] - tF_r).abs().flatten(1).max(1).values
        err = d.max().item() / tF_r.abs().max().item()
        assert err <= TF_TOL, (what, err, int(d.argmax()), st[int(d.argmax())])
    return a


def test_extract_over_filtered_file_matches_reference(cuda_device, monkeypatch):
    rec, raw, ops = _golden_case()
    calls = _count_device_batches(monkeypatch)
    st, tF, ops = kb.extract(ops, _source(raw), torch.from_numpy(rec.U).to(DEV), device=DEV)
    assert sorted(calls) == list(range(int(G["n_batches"])))      # the device path ran
    _compare(st, tF, G["st"], G["tF"], "golden")
    np.testing.assert_array_equal(ops["iCC"].cpu().numpy(), G["iCC"])
    np.testing.assert_array_equal(ops["iU"].cpu().numpy(), G["iU"])


def test_uint16_file_and_read_ahead_change_nothing(cuda_device):
    rec, raw, ops = _golden_case()
    U = torch.from_numpy(rec.U).to(DEV)
    st, tF, _ = kb.extract(dict(ops), _source(raw), U, device=DEV)
    u = (raw.astype(np.int32) + 32768).astype(np.uint16)
    st_u, tF_u, _ = kb.extract(dict(ops), _source(u), U, device=DEV)
    np.testing.assert_array_equal(st, st_u)
    assert torch.equal(tF, tF_u)
    st_s, tF_s, _ = kb.extract(dict(ops, read_ahead=False), _source(raw), U, device=DEV)
    np.testing.assert_array_equal(st, st_s)
    assert torch.equal(tF, tF_s)


def test_full_size_device_filter_vs_reference_filter(cuda_device, monkeypatch):
    NT, nt = 60000, 61
    c = dict(synth.CONFIGS[2])
    c.pop("n_batches")
    rec = synth.make_recording(1002, batch_lengths=[NT, NT, 20000], **c)
    n_bin = 385
    cmap = np.arange(384)
    raw = synth.raw_recording(rec, n_bin, cmap, seed=1102)
    rng = np.random.default_rng(1103)
    W = torch.from_numpy(((np.eye(384) + 0.02 * rng.standard_normal((384, 384))) / 25.0)
                         .astype(np.float32))
    xc, yc = rec.xc.astype(np.float32), rec.yc.astype(np.float32)
    xp = torch.from_numpy(np.vstack((xc, yc)).T)
    Kxx = op.kernel2d(xp, xp, 20.0)
    iKxx = torch.linalg.inv(Kxx + 0.01 * torch.eye(384)).to(DEV)
    dshift = rng.uniform(-5.0, 5.0, (3, 1))
    ops = dict(Th_learned=8.0, nt=nt, max_peels=100, wPCA=torch.from_numpy(rec.wPCA).to(DEV),
               nt0min=20, batch_size=NT, xc=xc, yc=yc, nblocks=1, yblk=np.array([yc.mean()]),
               probe=dict(xc=xc, yc=yc), iKxx=iKxx,
               settings=dict(nearest_chans=10, position_limit=100, n_pcs=6, sig_interp=20.0))
    kw = dict(NT=NT, nt=nt, chan_map=cmap, hp_filter=highpass_filter(), whiten_mat=W,
              dshift=dshift, device=DEV)
    U = torch.from_numpy(rec.U).to(DEV)
    calls = _count_device_batches(monkeypatch)
    st, tF, _ = kb.extract(dict(ops), synth.FilteredBinary(raw, **kw), U, device=DEV)
    assert sorted(calls) == [0, 1, 2]
    src_r = _OracleFiltered(raw, **kw)
    assert src_r.n_batches == 3
    st_r, tF_r, _ = kb.extract(dict(ops, device_filter=False), src_r, U, device=DEV)
    assert len(calls) == 3                                         # the reference filter ran
    a = _compare(st, tF, st_r, tF_r, "full size")
    assert a["n_r"] > 10000


def test_grouped_extract_equals_per_batch(cuda_device):
    """extract matches groups of batches per launch (batched matcher); with
    ops['batch_group'] = 1 it matches batch by batch.  Same rows and features
    bit for bit, with a short last group (6 batches in groups of 4) and with
    groups of 2, in both projections."""
    rec, raw, ops = _golden_case()
    U = torch.from_numpy(rec.U).to(DEV)
    for proj in ("fp32", "bf16x3"):
        o = dict(ops, projection=proj)
        st1, tF1, _ = kb.extract(dict(o, batch_group=1), _source(raw), U, device=DEV)
        for g in (4, 2):
            st, tF, _ = kb.extract(dict(o, batch_group=g), _source(raw), U, device=DEV)
            np.testing.assert_array_equal(st, st1)
            assert torch.equal(tF, tF1)


@pytest.mark.parametrize("group", [1, 4])
def test_filter_error_is_reported_by_extract(cuda_device, group):
    """A channel-map entry past the file's channels: the device filter flags
    KS_ERR_ARG (and reads nothing out of bounds); extract raises it once the
    batches are consumed, per-batch and grouped."""
    from kilosort_b200 import _lib
    rec, raw, ops = _golden_case()
    cmap = np.array(G["chan_map"]).copy()
    cmap[5] = raw.shape[1]                      # one past the last file channel
    src = synth.FilteredBinary(raw, NT=int(G["NT"]), nt=61, chan_map=cmap,
                               hp_filter=highpass_filter(), whiten_mat=torch.from_numpy(G["W"]),
                               dshift=G["dshift"], device=DEV)
    with pytest.raises(_lib.KilosortB200Error) as e:
        kb.extract(dict(ops, batch_group=group), src, torch.from_numpy(rec.U).to(DEV),
                   device=DEV)
    assert e.value.status == _lib.KS_ERR_ARG
