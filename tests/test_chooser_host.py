"""CPU: the learned chooser's host logic with the shipped model.

The network is evaluated by the FP64 numpy oracle (oracle/mlp_oracle.py) in a
stand-in for the context's MLP calls, so candidate ranking, the safety margin
and the clamp of log10 N to the training range are checked without a GPU.
"""
import importlib

import numpy as np
import pytest

import mlp_oracle


class OracleMlpContext:
    """The three MLP calls LearnedChooser makes, evaluated by the oracle."""

    def mlp_create(self, n_in, n_hidden=64, n_layers=3, n_out=2, seed=0):
        self.dims = [n_in] + [n_hidden] * n_layers + [n_out]
        return mlp_oracle.layout(self.dims)[1]

    def mlp_set_params(self, p):
        self.params = np.asarray(p, np.float64)

    def mlp_forward(self, X, n_out=2):
        return mlp_oracle.forward(self.params, self.dims, X)[0].astype(np.float32)


@pytest.fixture(scope="module")
def chooser(tb):
    return importlib.import_module("tapas_reduce_b200.chooser")


def _features(chooser, log10_n, depth_bin):
    h = np.zeros(chooser.NBINS)
    h[depth_bin] = 1.0
    return np.concatenate([[log10_n], h, [0.0]])


def test_ranked_candidates_meet_the_predicted_tolerance(chooser):
    lc = chooser.LearnedChooser(OracleMlpContext())
    feats = _features(chooser, 6.0, 6)
    for tol in (1e-3, 1e-5, 1e-6):
        ranked = lc.ranked(feats, tol, precisions=(0,), k=3)
        assert 1 <= len(ranked) <= 3
        safe = ranked[-1]
        if safe["source"] == "learned":
            assert safe["pred_log10_err"] + lc.margin <= np.log10(tol) + 1e-9
        for cand in ranked[:-1]:  # unmargined candidates: faster than the safe pick
            assert cand["source"] == "learned-unmargined"
            assert cand["pred_log10_err"] <= np.log10(tol) + chooser.SHORTLIST_EXPLORE + 1e-9
            assert cand["pred_log10_ms"] < safe["pred_log10_ms"]
        times = [c["pred_log10_ms"] for c in ranked[:-1]]
        assert times == sorted(times)
        for cand in ranked:
            assert cand["P"] in chooser.P_GRID and cand["ncrit"] in chooser.NCRIT_GRID
            assert cand["precision"] == "mixed"


def test_body_count_is_clamped_to_the_training_range(chooser):
    lc = chooser.LearnedChooser(OracleMlpContext())
    top = _features(chooser, chooser.LOG10_N_MAX, 8)
    beyond = _features(chooser, chooser.LOG10_N_MAX + 2.0, 8)
    assert lc.choose(top, 1e-6, (0,)) == lc.choose(beyond, 1e-6, (0,))
    low = _features(chooser, chooser.LOG10_N_MIN, 3)
    below = _features(chooser, chooser.LOG10_N_MIN - 1.0, 3)
    assert lc.choose(low, 1e-4, (0, 1)) == lc.choose(below, 1e-4, (0, 1))
