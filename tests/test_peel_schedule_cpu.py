"""A segment-skewed order of the greedy peel (oracle/peel_schedule.py) gives
the same spikes, amplitudes, pooled scores and final score matrix as the
oracle's iteration-by-iteration peel, bit for bit, for random orders and
several segment widths, on the golden cases (ties in `dups`, an iteration cap
in `maxpeels2`, no spikes in `empty`, a full 60122-sample batch in `cfg1`)."""
import pytest
import torch

from oracle import matching as om
from oracle.peel_schedule import peel_skewed
from tests import golden_util as gu


def _scores(name):
    g = gu.load(name)
    rec, X, U, W = gu.case_inputs(g)
    Ut, Wt, Xt = torch.from_numpy(U), torch.from_numpy(W), torch.from_numpy(X)
    nt = int(g["nt"])
    ops = dict(Th_learned=float(g["Th"]), nt=nt, max_peels=int(g["max_peels"]), wPCA=Wt)
    return (om.project_scores(Xt, Ut, Wt, nt), om.template_energy(Ut),
            om.prepare_matching(ops, Ut), ops, Xt, Ut, Wt, g)


@pytest.mark.parametrize("name", ["tiny", "small", "nt41", "maxpeels2", "empty", "dups"])
@pytest.mark.parametrize("seed,wmul", [(0, 1), (1, 2), (2, 4)])
def test_skewed_order_equals_peel(name, seed, wmul):
    B, nm, ctc, ops, Xt, Ut, Wt, g = _scores(name)
    nt = ops["nt"]
    B_ref = B.clone()
    st, amps, th, _ = om.peel(B_ref, Xt.clone(), Ut, Wt, ctc, nm, ops["Th_learned"], nt,
                              ops["max_peels"])
    assert len(st) == len(g["st"])
    B_sk = B.clone()
    st2, amps2, th2, _ = peel_skewed(B_sk, nm, ctc, ops["Th_learned"], nt, ops["max_peels"],
                                     width=nt * wmul, seed=seed)
    assert torch.equal(st, st2)
    assert torch.equal(amps, amps2)
    assert torch.equal(th, th2)
    assert torch.equal(B_ref, B_sk)


def test_skewed_order_full_batch():
    B, nm, ctc, ops, Xt, Ut, Wt, g = _scores("cfg1")
    nt = ops["nt"]
    B_ref = B.clone()
    st, amps, th, _ = om.peel(B_ref, Xt.clone(), Ut, Wt, ctc, nm, ops["Th_learned"], nt,
                              ops["max_peels"])
    B_sk = B.clone()
    st2, amps2, th2, _ = peel_skewed(B_sk, nm, ctc, ops["Th_learned"], nt, ops["max_peels"],
                                     width=256, seed=7)
    assert len(st) == len(g["st"]) > 500
    assert torch.equal(st, st2) and torch.equal(amps, amps2) and torch.equal(th, th2)
    assert torch.equal(B_ref, B_sk)
