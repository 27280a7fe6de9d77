"""Parity of the sm_100a path with the reference (through the oracle and the
golden vectors made by the reference itself).

Tolerances:
* the peel given the same score matrix and energies as the oracle is
  bit-exact in st, amps and the updated B; th_amps within 1 ulp (IEEE sqrt vs
  the CPU build's vectorised sqrt);
* full run_matching in FP32: (time, template) agreement >= 99.5 %, matched
  times exact, amplitude relative error <= 1e-4;
* the residual Xres: |diff| <= 1e-5 * (1 + |x|);
* features and ctc: relative error <= 1e-5 of the array's max magnitude.
"""
import numpy as np
import pytest
import torch

import kilosort_b200 as kb
from kilosort_b200 import _lib, synth
from oracle import matching as om
from tests import golden_util as gu
from tests.parity_util import agreement

pytestmark = pytest.mark.gpu

DEV = torch.device("cuda:0")


def _ops(g, W):
    return dict(Th_learned=float(g["Th"]), nt=int(g["nt"]), max_peels=int(g["max_peels"]),
                wPCA=W)


@pytest.mark.parametrize("name", gu.CASES)
def test_peel_bit_exact_given_same_scores(cuda_device, name):
    """Same B, nm and ctc as the oracle -> identical spikes, amplitudes, B and Xres.

    The oracle runs on this machine's CPU: its float32 projection rounds like
    the reference's on the same CPU (pinned bit for bit against the golden
    vectors on the machine that made them), but CPU libraries may sum in a
    different order on another CPU, so the expected peel output is recomputed
    here from the very B the GPU receives.
    """
    g = gu.load(name)
    rec, X, U, W = gu.case_inputs(g)
    Ut, Wt, Xt = torch.from_numpy(U), torch.from_numpy(W), torch.from_numpy(X)
    ops = _ops(g, Wt)
    nt = ops["nt"]
    ctc = om.prepare_matching(ops, Ut)
    nm = om.template_energy(Ut)
    B = om.project_scores(Xt, Ut, Wt, nt)
    Bo, Xo = B.clone(), Xt.clone()
    st_o, amps_o, th_o, _ = om.peel(Bo, Xo, Ut, Wt, ctc, nm, ops["Th_learned"], nt,
                                    ops["max_peels"])
    L = X.shape[1]
    ldb = ((L + 63) // 64) * 64
    Bd = torch.zeros((U.shape[0], ldb), dtype=torch.float32, device=DEV)
    Bd[:, :L] = B.to(DEV)
    Xres = Xt.to(DEV).clone()
    st, amps, th, iters = kb.peel(Bd[:, :L], Xres, Ut.to(DEV), Wt.to(DEV), ctc.to(DEV),
                                  nm.to(DEV), ops["Th_learned"], nt, ops["max_peels"])
    np.testing.assert_array_equal(st.cpu().numpy(), st_o.numpy())
    np.testing.assert_array_equal(amps.cpu().numpy(), amps_o.numpy())
    # th_amps = sqrt(pooled): IEEE sqrt here (as the reference on CUDA); the
    # reference's CPU build takes a vectorised sqrt that is 1 ulp off on ~0.7 %
    # of inputs, so allow one ulp
    np.testing.assert_array_max_ulp(th.cpu().numpy(), th_o.numpy(), maxulp=1)
    np.testing.assert_array_equal(Bd[:, :L].cpu().numpy(), Bo.numpy())
    np.testing.assert_allclose(Xres.cpu().numpy(), Xo.numpy(), rtol=0,
                               atol=1e-6 * (1 + np.abs(Xo.numpy()).max()))


@pytest.mark.parametrize("name", gu.CASES)
def test_run_matching_fp32_matches_reference(cuda_device, name):
    g = gu.load(name)
    rec, X, U, W = gu.case_inputs(g)
    Ut, Wt = torch.from_numpy(U), torch.from_numpy(W)
    ops = _ops(g, Wt)
    ctc = om.prepare_matching(ops, Ut)
    opsd = dict(ops, wPCA=Wt.to(DEV), projection="fp32")
    Xd = torch.from_numpy(X).to(DEV)
    X_before = Xd.clone()
    st, amps, th, Xres = kb.run_matching(opsd, Xd, Ut.to(DEV), ctc.to(DEV), device=DEV)
    assert torch.equal(Xd, X_before), "run_matching must not modify X"
    assert st.dtype == torch.int64 and st.shape[1] == 2
    assert amps.shape == (len(st), 1) and th.shape == (len(st), 1)
    a = agreement(st.cpu().numpy(), g["st"], amps.cpu().numpy(), g["amps"])
    assert a["agreement"] >= 0.995, a
    assert a["amp_rel_max"] <= 1e-4, a
    if len(g["st"]) and a["matched"] == len(g["st"]) == len(st):
        # identical spike sets: th_amps too
        np.testing.assert_allclose(th.cpu().numpy(), g["th_amps"], rtol=1e-4)
    if "xres_idx" in g and a["matched"] == len(g["st"]) == len(st):
        ref_xres = gu.xres_from_golden(g, X)
        np.testing.assert_allclose(Xres.cpu().numpy(), ref_xres, rtol=0,
                                   atol=1e-4 * (1 + np.abs(ref_xres).max()))


def test_projection_error_vs_fp64(cuda_device):
    g = gu.load("cfg1")
    rec, X, U, W = gu.case_inputs(g)
    nt = int(g["nt"])
    B64 = om.project_scores(torch.from_numpy(X).double(), torch.from_numpy(U).double(),
                            torch.from_numpy(W).double(), nt).numpy()
    B = kb.project_scores(torch.from_numpy(X).to(DEV), torch.from_numpy(U).to(DEV),
                          torch.from_numpy(W).to(DEV), nt, "fp32").cpu().numpy()
    err = np.abs(B - B64).max() / np.abs(B64).max()
    assert err < 2e-6, err


def test_template_energy(cuda_device):
    g = gu.load("small")
    rec, X, U, W = gu.case_inputs(g)
    nm = kb.template_energy(torch.from_numpy(U).to(DEV)).cpu().numpy()
    ref = om.template_energy(torch.from_numpy(U)).numpy()
    np.testing.assert_allclose(nm, ref, rtol=2e-6)


def test_prepare_matching_ctc(cuda_device):
    g = gu.load("small")
    rec, X, U, W = gu.case_inputs(g)
    ops = dict(nt=int(g["nt"]), wPCA=torch.from_numpy(W).to(DEV))
    ctc = kb.prepare_matching(ops, torch.from_numpy(U).to(DEV)).cpu().numpy()
    ref = g["ctc_full"]
    assert ctc.shape == ref.shape
    assert np.abs(ctc - ref).max() <= 1e-5 * np.abs(ref).max()


def test_prepare_extract(cuda_device):
    g = gu.load("small")
    rec, X, U, W = gu.case_inputs(g)
    iCC, mask, iU, Ucc = kb.prepare_extract(g["xc"], g["yc"], torch.from_numpy(U).to(DEV),
                                            10, 100, device=DEV)
    np.testing.assert_array_equal(iCC.cpu().numpy(), g["iCC"])
    np.testing.assert_array_equal(mask.cpu().numpy(), g["iCC_mask"])
    np.testing.assert_array_equal(iU.cpu().numpy(), g["iU"])
    np.testing.assert_array_equal(Ucc.cpu().numpy(), g["Ucc"])


def test_features_match_oracle(cuda_device):
    g = gu.load("cfg1")
    rec, X, U, W = gu.case_inputs(g)
    Ut, Wt, Xt = torch.from_numpy(U), torch.from_numpy(W), torch.from_numpy(X)
    ops = _ops(g, Wt)
    ctc = om.prepare_matching(ops, Ut)
    st, amps, th, Xres = om.run_matching(ops, Xt, Ut, ctc)
    iCC, _, iU, Ucc = om.prepare_extract(rec.xc, rec.yc, Ut, 10, 100)
    ref = om.spike_features(Xres, st, amps, Wt, iCC, iU, Ucc, ops["nt"]).transpose(0, 1)
    tF = kb.spike_features(Xres.to(DEV), st.to(DEV), amps.to(DEV), Wt.to(DEV),
                           iCC.to(DEV), iU.to(DEV), Ucc.to(DEV)).cpu()
    assert tF.shape == ref.shape
    err = (tF - ref).abs().max().item() / ref.abs().max().item()
    assert err <= 1e-5, err


def test_extract_matches_reference(cuda_device):
    import ast
    g = gu.load("extract")
    kw = ast.literal_eval(str(g["seed_kwargs"]))
    rec = synth.make_recording(**kw)
    assert gu.sha(rec.signal) == str(g["signal_sha"])
    bfile = synth.SyntheticBinary(rec, device=DEV)
    ops = dict(Th_learned=8.0, nt=61, max_peels=100, wPCA=torch.from_numpy(rec.wPCA).to(DEV),
               nt0min=20, batch_size=3000, xc=rec.xc, yc=rec.yc,
               settings=dict(nearest_chans=10, position_limit=100, n_pcs=6))
    st, tF, ops = kb.extract(ops, bfile, torch.from_numpy(rec.U).to(DEV), device=DEV)
    a = agreement(st[:, :2], g["st"][:, :2])
    assert a["agreement"] >= 0.995, a
    if a["matched"] == len(st) == len(g["st"]):
        np.testing.assert_array_equal(st[:, :2], g["st"][:, :2])
        np.testing.assert_allclose(st[:, 2], g["st"][:, 2], rtol=1e-4)
        ref = torch.from_numpy(g["tF"])
        err = (tF - ref).abs().max().item() / ref.abs().max().item()
        assert err <= 1e-4, err
    np.testing.assert_array_equal(ops["iCC"].cpu().numpy(), g["iCC"])
    np.testing.assert_array_equal(ops["iU"].cpu().numpy(), g["iU"])


def test_overflow_raises(cuda_device):
    g = gu.load("small")
    rec, X, U, W = gu.case_inputs(g)
    Ut, Wt = torch.from_numpy(U), torch.from_numpy(W)
    ops = _ops(g, Wt)
    ctc = om.prepare_matching(ops, Ut).to(DEV)
    opsd = dict(ops, wPCA=Wt.to(DEV), spike_capacity=5)
    with pytest.raises(RuntimeError, match="exceed the spike buffer"):
        kb.run_matching(opsd, torch.from_numpy(X).to(DEV), Ut.to(DEV), ctc, device=DEV)
    # the context stays usable afterwards
    opsd["spike_capacity"] = 100000
    st, *_ = kb.run_matching(opsd, torch.from_numpy(X).to(DEV), Ut.to(DEV), ctc, device=DEV)
    assert len(st) == len(g["st"])


def test_zero_iterations(cuda_device):
    g = gu.load("small")
    rec, X, U, W = gu.case_inputs(g)
    Ut, Wt = torch.from_numpy(U), torch.from_numpy(W)
    ops = _ops(g, Wt)
    ctc = om.prepare_matching(ops, Ut).to(DEV)
    opsd = dict(ops, wPCA=Wt.to(DEV), max_peels=0)
    st, amps, th, Xres = kb.run_matching(opsd, torch.from_numpy(X).to(DEV), Ut.to(DEV), ctc,
                                         device=DEV)
    assert len(st) == 0
    assert torch.equal(Xres.cpu(), torch.from_numpy(X))


def test_watchdog_wait_times_out(cuda_device):
    lib = _lib.load()
    status = torch.full((2,), -1, dtype=torch.int32, device=DEV)
    s = torch.cuda.current_stream(DEV).cuda_stream
    _lib.check(lib.ks_selftest_wait(2_000_000, status.data_ptr(), s), "ks_selftest_wait")
    torch.cuda.synchronize()
    assert int(status[0]) == _lib.KS_ERR_TIMEOUT
    # device still healthy
    assert torch.ones(4, device=DEV).sum().item() == 4


def test_cfg2_batch_fp32_vs_oracle(cuda_device):
    """One Neuropixels-scale batch (C=384, K=600, L=60122) against the oracle."""
    rec = synth.config_recording(2, n_batches=1)
    Ut, Wt = torch.from_numpy(rec.U), torch.from_numpy(rec.wPCA)
    X = np.ascontiguousarray(rec.batch(0))
    ops = dict(Th_learned=8.0, nt=61, max_peels=100, wPCA=Wt)
    torch.set_num_threads(max(1, torch.get_num_threads()))
    ctc = om.prepare_matching(ops, Ut)
    st_r, amps_r, th_r, _ = om.run_matching(ops, torch.from_numpy(X), Ut, ctc)
    opsd = dict(ops, wPCA=Wt.to(DEV), projection="fp32")
    st, amps, th, Xres = kb.run_matching(opsd, torch.from_numpy(X).to(DEV), Ut.to(DEV),
                                         ctc.to(DEV), device=DEV)
    a = agreement(st.cpu().numpy(), st_r.numpy(), amps.cpu().numpy(), amps_r.numpy())
    assert a["agreement"] >= 0.995, a
    assert a["amp_rel_max"] <= 1e-4, a


def test_tiled_scores_and_transposed_ctc(cuda_device):
    """The peel's layouts hold the same numbers as the reference layouts."""
    g = gu.load("small")
    rec, X, U, W = gu.case_inputs(g)
    Xd, Ud, Wd = (torch.from_numpy(a).to(DEV) for a in (X, U, W))
    B = kb.project_scores(Xd, Ud, Wd, 61, "fp32")
    Bt = kb.project_scores(Xd, Ud, Wd, 61, "fp32", tiled=True)
    L = X.shape[1]
    rebuilt = Bt.permute(1, 0, 2).reshape(U.shape[0], -1)[:, :L]
    assert torch.equal(rebuilt, B)
    ctc = torch.from_numpy(g["ctc_full"]).to(DEV)
    ctcT = kb.transpose_ctc(ctc, 61)
    assert torch.equal(ctcT, ctc.transpose(0, 1))


def test_transposed_ctc_cache_follows_the_tensor(cuda_device):
    """run_matching keeps the transposed ctc of the last ctc tensor it saw; a
    new ctc of the same shape that reuses the freed storage of the previous
    one (the caching allocator hands the block straight back) must not be
    taken for it.  Each result equals the oracle's for its own templates."""
    recs = [synth.make_recording(8101 + i, n_chan=48, n_templates=30, batch_lengths=[4000])
            for i in range(3)]
    for rec in recs:
        U = torch.from_numpy(rec.U)
        W = torch.from_numpy(rec.wPCA)
        X = torch.from_numpy(np.ascontiguousarray(rec.batch(0)))
        ops = dict(Th_learned=8.0, nt=rec.nt, max_peels=100, wPCA=W)
        ctc = kb.prepare_matching(dict(ops, wPCA=W.to(DEV)), U.to(DEV))
        st, amps, _, _ = kb.run_matching(dict(ops, wPCA=W.to(DEV)), X.to(DEV), U.to(DEV), ctc,
                                         device=DEV)
        st_r, amps_r, _, _ = om.run_matching(ops, X, U, ctc.cpu())
        np.testing.assert_array_equal(st.cpu().numpy(), st_r.numpy())
        del ctc                               # its storage goes back to the allocator


def test_extract_read_ahead_equals_in_order_reads(cuda_device):
    """extract reads the next batch on a worker thread and stream while the
    current one is matched; the result equals reading each batch in turn."""
    from kilosort_b200 import template_matching as tm
    rec = synth.make_recording(2101, n_chan=32, probe="np1", n_templates=24,
                               batch_lengths=[3000] * 5, rate_hz=(10.0, 30.0))
    ops = dict(Th_learned=8.0, nt=61, max_peels=100, wPCA=torch.from_numpy(rec.wPCA).to(DEV),
               nt0min=20, batch_size=3000, xc=rec.xc, yc=rec.yc,
               settings=dict(nearest_chans=10, position_limit=100, n_pcs=6))
    U = torch.from_numpy(rec.U).to(DEV)
    st, tF, ops = kb.extract(ops, synth.SyntheticBinary(rec, device=DEV), U, device=DEV)
    assert len(st) > 100
    match, features = tm._match_features(ops, ops["wPCA"].contiguous(),
                                         ops["iCC"].to(DEV).contiguous(), ops["iU"],
                                         kb.prepare_extract(rec.xc, rec.yc, U, 10, 100,
                                                            device=DEV)[3])
    st1, tF1 = tm.extract_batches(ops, synth.SyntheticBinary(rec, device=DEV), np.arange(5), U,
                                  kb.prepare_matching(ops, U), match, features,
                                  read_ahead=False)
    st1, tF1 = tm.sort_spikes(st1, tF1)
    np.testing.assert_array_equal(st, st1)
    assert torch.equal(tF, tF1)
