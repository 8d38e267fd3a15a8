"""CPU: the split and hit-and-run oracles reproduce the reference's golden outputs."""

import ast

import numpy as np
import pytest

from conftest import GOLDEN
from oracle import ridge as O
from oracle import sampling as H
from oracle import split as S

SG = np.load(GOLDEN / "split_golden.npz")
HG = np.load(GOLDEN / "har_golden.npz")


@pytest.mark.parametrize("i", range(int(SG["count"])))
def test_split_oracle_matches_reference(i):
    kind, T, lam, R, iters, parent_loss = SG[f"s{i}_meta"]
    extra = ast.literal_eval(str(SG[f"s{i}_extra"]))
    p = S.Params(max_iters=int(iters), n_restarts=int(R), **extra)
    res = S.split(SG[f"s{i}_X"], SG[f"s{i}_y"], list(SG[f"s{i}_theta0"]), T, int(kind), lam, parent_loss, p)
    np.testing.assert_allclose(np.r_[res["w"], res["z"]], SG[f"s{i}_theta"], rtol=1e-9, atol=1e-11)
    assert res["stop_reason"] == str(SG[f"s{i}_stop"])
    assert res["n_iters"] == int(SG[f"s{i}_n_iters"])
    assert res["n_right"] == int(SG[f"s{i}_n_right"])
    np.testing.assert_allclose(res["losses"], SG[f"s{i}_soft_losses"], rtol=1e-9, atol=1e-13)
    np.testing.assert_allclose(res["bl"], SG[f"s{i}_beta_left"], rtol=1e-8, atol=1e-10)
    assert bool(res["fallback"]) == bool(SG[f"s{i}_fallback"])


@pytest.mark.parametrize("i", range(int(HG["batched_count"])))
def test_batched_chain_oracle_matches_reference(i):
    d, k, C, burn, thin, rounds = (int(v) for v in HG[f"b{i}_meta"])
    Ab, bb = H.box_rows(-np.ones(d), np.ones(d))
    A = np.vstack([Ab, HG[f"b{i}_Ao"]])
    b = np.concatenate([bb, HG[f"b{i}_bo"]])
    out, _ = H.chains_batched(A, b, HG[f"b{i}_x0"], HG[f"b{i}_dirs"], HG[f"b{i}_unif"], burn, thin, rounds)
    np.testing.assert_allclose(out, HG[f"b{i}_samples"], rtol=1e-13, atol=1e-13)


@pytest.mark.parametrize("i", range(int(HG["scalar_count"])))
def test_scalar_chain_oracle_matches_reference(i):
    d, k, burn, thin, n = (int(v) for v in HG[f"s{i}_meta"])
    Ab, bb = H.box_rows(-np.ones(d), np.ones(d))
    A = np.vstack([Ab, HG[f"s{i}_Ao"]])
    b = np.concatenate([bb, HG[f"s{i}_bo"]])
    out = H.chain_scalar(A, b, HG[f"s{i}_x0"], HG[f"s{i}_dirs"], HG[f"s{i}_unif"], burn, thin, n)
    np.testing.assert_allclose(out, HG[f"s{i}_samples"], rtol=1e-13, atol=1e-13)


def test_acf_oracle_matches_reference():
    out = H.autocorrelation_by_lag(HG["acf_series"], HG["acf_lags"])
    np.testing.assert_allclose(out, HG["acf"], rtol=1e-13, atol=1e-13)


def test_box_row_split_is_exact():
    from art.sampling import split_box_rows

    A = np.vstack([np.eye(3), -np.eye(3), [[0.6, 0.8, 0.0]], [[2.0, 0.0, 0.0]]])
    b = np.arange(8.0)
    lo, hi, Ao, bo = split_box_rows(A, b)
    np.testing.assert_array_equal(hi, [0, 1, 2])
    np.testing.assert_array_equal(lo, [-3, -4, -5])
    assert Ao.shape == (2, 3) and list(bo) == [6.0, 7.0]
