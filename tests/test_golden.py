"""Golden fixtures produced by the reference's own code (tests/golden/).

The fixtures were generated by tests/golden/make_golden.py with the
reference's Sparse::CholeskyDecomposition compiled from its headers; they
pin both the CPU oracle and the product's host-side symbolic analysis, and
(on a GPU) the product's factor and solve.
"""
from __future__ import annotations

import glob
import os

import numpy as np
import pytest

import oracle
from tensors_b200.cholesky import CholeskyDecomposition

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURES = sorted(glob.glob(os.path.join(HERE, "golden", "*.npz")))
STRATEGY = {"maximal": 0, "fundamental": 1, "amalgamated": 2}


def load(path):
    z = np.load(path)
    perm = z["perm"] if bool(z["has_perm"]) else None
    return z, perm


def test_fixtures_present():
    assert len(FIXTURES) >= 10


@pytest.mark.parametrize("path", FIXTURES, ids=[os.path.basename(p)[:-4] for p in FIXTURES])
def test_oracle_matches_reference_fixture(path):
    z, perm = load(path)
    o = oracle.OracleCholesky(int(z["n"]), z["outer"], z["inner"], perm, str(z["strategy"]))
    for key in oracle.ARRAYS:
        assert np.array_equal(o.array(key), z[f"arr_{key}"]), key
    assert o.factor(z["values"], float(z["reg"])) == int(z["status"])
    if int(z["status"]) != 0:
        return
    tri, rec = o.factor_values()
    scale = np.abs(z["tri"]).max()
    assert np.abs(tri - z["tri"]).max() <= 1e-12 * scale
    if len(rec):
        assert np.abs(rec - z["rec"]).max() <= 1e-12 * scale
    X = o.solve(z["B"])
    assert np.abs(X - z["X"]).max() <= 1e-10 * np.abs(z["X"]).max()
    assert abs(o.log_det() - float(z["logdet"])) <= 1e-10 * max(1.0, abs(float(z["logdet"])))


@pytest.mark.parametrize("path", FIXTURES, ids=[os.path.basename(p)[:-4] for p in FIXTURES])
def test_product_symbolic_matches_reference_fixture(path):
    z, perm = load(path)
    c = CholeskyDecomposition(z["outer"], z["inner"], perm)
    c.SetSupernodeStrategy(STRATEGY[str(z["strategy"])])
    c.SymbolicFactorization()
    for key in oracle.ARRAYS:
        assert np.array_equal(c.SymbolicArray(key), z[f"arr_{key}"]), key
    c.CheckPlan()


@pytest.mark.gpu
@pytest.mark.parametrize("path", FIXTURES, ids=[os.path.basename(p)[:-4] for p in FIXTURES])
def test_gpu_factor_and_solve_match_reference_fixture(path):
    z, perm = load(path)
    c = CholeskyDecomposition(z["outer"], z["inner"], perm)
    c.SetSupernodeStrategy(STRATEGY[str(z["strategy"])])
    assert c.NumericFactorization(z["values"], float(z["reg"])) == int(z["status"])
    if int(z["status"]) != 0:
        return
    tri, rec = c.FactorValues()
    scale = np.abs(z["tri"]).max()
    assert np.abs(tri - z["tri"]).max() <= 1e-12 * scale
    if len(rec):
        assert np.abs(rec - z["rec"]).max() <= 1e-12 * scale
    X = c.Solve(z["B"])
    assert np.abs(X - z["X"]).max() <= 1e-10 * np.abs(z["X"]).max()
    assert abs(c.LogDeterminant() - float(z["logdet"])) <= 1e-10 * max(1.0, abs(float(z["logdet"])))
