"""Split-BF16 tensor-core projection (tcgen05): accuracy and spike agreement.

Tolerances: the projection's max |B - B_fp64| is at most 3e-5 of max |B|
(hi/lo split: ~2^-16 per product); run_matching with it agrees with the
reference's spikes at >= 99.5 % (exact times and templates) with matched
amplitudes within 1e-3 relative.
"""
import numpy as np
import pytest
import torch

import kilosort_b200 as kb
from kilosort_b200 import synth
from oracle import matching as om
from tests import golden_util as gu
from tests.parity_util import agreement

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0")


@pytest.mark.parametrize("name", ["small", "nt41", "cfg1"])
def test_bf16x3_projection_error_vs_fp64(cuda_device, name):
    g = gu.load(name)
    rec, X, U, W = gu.case_inputs(g)
    nt = int(g["nt"])
    B64 = om.project_scores(torch.from_numpy(X).double(), torch.from_numpy(U).double(),
                            torch.from_numpy(W).double(), nt).numpy()
    Xd, Ud, Wd = (torch.from_numpy(a).to(DEV) for a in (X, U, W))
    B = kb.project_scores(Xd, Ud, Wd, nt, "bf16x3").cpu().numpy()
    err = np.abs(B - B64).max() / np.abs(B64).max()
    assert err < 3e-5, err
    # the tiled layout holds the same numbers
    Bt = kb.project_scores(Xd, Ud, Wd, nt, "bf16x3", tiled=True)
    L = X.shape[1]
    rebuilt = Bt.permute(1, 0, 2).reshape(U.shape[0], -1)[:, :L].cpu().numpy()
    np.testing.assert_array_equal(rebuilt, B)


@pytest.mark.parametrize("name", gu.CASES)
def test_run_matching_bf16x3_agreement(cuda_device, name):
    g = gu.load(name)
    rec, X, U, W = gu.case_inputs(g)
    Ut, Wt = torch.from_numpy(U), torch.from_numpy(W)
    ops = dict(Th_learned=float(g["Th"]), nt=int(g["nt"]), max_peels=int(g["max_peels"]),
               wPCA=Wt.to(DEV), projection="bf16x3")
    ctc = om.prepare_matching(dict(ops, wPCA=Wt), Ut)
    st, amps, th, Xres = kb.run_matching(ops, torch.from_numpy(X).to(DEV), Ut.to(DEV),
                                         ctc.to(DEV), device=DEV)
    a = agreement(st.cpu().numpy(), g["st"], amps.cpu().numpy(), g["amps"])
    assert a["agreement"] >= 0.995, a
    assert a["amp_rel_max"] <= 1e-3, a


def test_cfg2_batch_bf16x3_vs_oracle(cuda_device):
    rec = synth.config_recording(2, n_batches=1)
    Ut, Wt = torch.from_numpy(rec.U), torch.from_numpy(rec.wPCA)
    X = np.ascontiguousarray(rec.batch(0))
    ops = dict(Th_learned=8.0, nt=61, max_peels=100, wPCA=Wt)
    ctc = om.prepare_matching(ops, Ut)
    st_r, amps_r, _, _ = om.run_matching(ops, torch.from_numpy(X), Ut, ctc)
    opsd = dict(ops, wPCA=Wt.to(DEV), projection="bf16x3")
    st, amps, _, _ = kb.run_matching(opsd, torch.from_numpy(X).to(DEV), Ut.to(DEV),
                                     ctc.to(DEV), device=DEV)
    a = agreement(st.cpu().numpy(), st_r.numpy(), amps.cpu().numpy(), amps_r.numpy())
    assert a["agreement"] >= 0.995, a
