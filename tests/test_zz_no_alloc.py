"""ks_peel_static: the peel for callers that cannot allocate device memory.

Such callers (an acquisition loop that may not call cudaMalloc on its hot
path, a plugin that owns no device allocator) pass inputs and outputs only;
the peel's scratch is a fixed array inside the library.  This test calls the
entry point through the C ABI twice in a row and checks each result against
the workspace-based ks_peel on the same inputs (both peels are exact, so the
outputs must be identical; the tolerance of the other parity tests is met
with equality).  The second call runs with the array still holding the first
call's contents.  A batch of the longest length the array holds runs too,
and the shapes beyond the array are refused.  The file is collected last so
that a run stopping at the first failure has run every other test; it also
passes alone.
"""
import numpy as np
import pytest
import torch

import kilosort_b200 as kb
from kilosort_b200 import _lib, synth
from oracle import matching as om

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0")


def _inputs(seed, n_templates, length, n_chan=64):
    rec = synth.make_recording(seed, n_chan=n_chan, probe="np1", n_templates=n_templates,
                               batch_lengths=[length], rate_hz=(10.0, 30.0))
    U = torch.from_numpy(rec.U)
    W = torch.from_numpy(rec.wPCA)
    X = torch.from_numpy(np.ascontiguousarray(rec.batch(0)))
    ctc = om.prepare_matching(dict(nt=61, wPCA=W), U)
    Ud, Wd, Xd = U.to(DEV), W.to(DEV), X.to(DEV)
    Bt = kb.project_scores(Xd, Ud, Wd, 61, "fp32", tiled=True)
    return dict(Bt=Bt, X=Xd, U=Ud, W=Wd, ctcT=kb.transpose_ctc(ctc.to(DEV), 61),
                nm=kb.template_energy(Ud))


def _outputs(cap, dev=DEV):
    return dict(st=torch.zeros((cap, 2), dtype=torch.int64, device=dev),
                amps=torch.zeros(cap, dtype=torch.float32, device=dev),
                th=torch.zeros(cap, dtype=torch.float32, device=dev),
                info=torch.zeros(4, dtype=torch.int64, device=dev))


def _run(lib, inp, static, cap=20000):
    Bt = inp["Bt"].clone()
    Xres = inp["X"].clone()
    o = _outputs(cap)
    K, P, C = inp["U"].shape
    L = Xres.shape[1]
    s = torch.cuda.current_stream(DEV).cuda_stream
    if static:
        rc = lib.ks_peel_static(Bt.data_ptr(), Xres.data_ptr(), inp["U"].data_ptr(),
                                inp["W"].data_ptr(), inp["ctcT"].data_ptr(), inp["nm"].data_ptr(),
                                C, L, K, P, 61, 64.0, 100, cap, o["st"].data_ptr(),
                                o["amps"].data_ptr(), o["th"].data_ptr(), o["info"].data_ptr(), s)
    else:
        ws = torch.empty(lib.ks_peel_workspace_size(L, K, 61, _lib.KS_B_TILED, _lib.KS_CTC_KJL),
                         dtype=torch.uint8, device=DEV)
        rc = lib.ks_peel(Bt.data_ptr(), 0, _lib.KS_B_TILED, Xres.data_ptr(), inp["U"].data_ptr(),
                         inp["W"].data_ptr(), inp["ctcT"].data_ptr(), _lib.KS_CTC_KJL,
                         inp["nm"].data_ptr(), C, L, K, P, 61, 64.0, 100, cap,
                         o["st"].data_ptr(), o["amps"].data_ptr(), o["th"].data_ptr(),
                         o["info"].data_ptr(), ws.data_ptr(), ws.numel(), s)
    _lib.check(rc, "ks_peel_static" if static else "ks_peel")
    torch.cuda.synchronize()
    n = int(o["info"][0])
    assert int(o["info"][1]) == _lib.KS_OK
    return dict(n=n, st=o["st"][:n].cpu(), amps=o["amps"][:n].cpu(), th=o["th"][:n].cpu(),
                Bt=Bt.cpu(), Xres=Xres.cpu())


def test_static_peel_matches_workspace_peel_twice(cuda_device):
    lib = _lib.load()
    # two different batches in a row: the second call starts from the array
    # contents the first one left behind
    for seed, K, length in ((31, 48, 6000), (32, 40, 9000)):
        inp = _inputs(seed, K, length)
        ref = _run(lib, inp, static=False)
        got = _run(lib, inp, static=True)
        assert ref["n"] > 0
        assert got["n"] == ref["n"]
        for key in ("st", "amps", "th", "Bt", "Xres"):
            assert torch.equal(got[key], ref[key]), key


def test_static_peel_holds_its_longest_batch(cuda_device):
    # KS_PEEL_STATIC_MAX_L padded samples (131072) with a small template set
    lib = _lib.load()
    inp = _inputs(33, 24, 131072 - 2 * 61, n_chan=32)
    assert inp["X"].shape[1] == 131072
    ref = _run(lib, inp, static=False, cap=40000)
    got = _run(lib, inp, static=True, cap=40000)
    assert ref["n"] > 0 and got["n"] == ref["n"]
    for key in ("st", "amps", "th", "Bt", "Xres"):
        assert torch.equal(got[key], ref[key]), key


def test_static_peel_rejects_batches_beyond_the_array(cuda_device):
    lib = _lib.load()
    too_long = 131072 + 1
    rc = lib.ks_peel_static(None, None, None, None, None, None, 4, too_long, 2, 6, 61, 64.0,
                            1, 1, None, None, None, None, None)
    assert rc == _lib.KS_ERR_UNSUPPORTED
    assert b"131072" in lib.ks_last_error()
    # at the longest batch, one template more than the array holds
    rc = lib.ks_peel_static(None, None, None, None, None, None, 4, 131072, 56897, 6, 61, 64.0,
                            1, 1, None, None, None, None, None)
    assert rc == _lib.KS_ERR_UNSUPPORTED
    assert b"56896" in lib.ks_last_error()
