"""Pin the Gauss-Legendre rules (oracle and product) against the reference's
own tables: every gauss::container<N> of sources/HHG/thread_gauss.hpp and
the 30-point [0,1] rule of sources/HHG/Laser/gauss.hpp, committed as
tests/golden/gauss_tables.json by tests/golden/make_fixtures.py."""
import json
import os

import numpy as np
import pytest

from oracle import hhg_oracle as O

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "gauss_tables.json")))
SIZES = sorted(int(k) for k in GOLD if k.isdigit())


@pytest.mark.parametrize("n", SIZES)
def test_oracle_gauss_matches_reference_tables(n):
    x, w = O.gauss_legendre(n)
    xa = np.array(GOLD[str(n)]["abscissa"])
    wa = np.array(GOLD[str(n)]["weights"])
    assert len(xa) == n // 2
    # positive half, ascending, as the reference stores it
    assert np.max(np.abs(x[n // 2:] - xa)) <= 2e-16
    assert np.max(np.abs(w[n // 2:] - wa) / wa) <= 2e-14
    # symmetric rule
    assert np.array_equal(x[: n // 2], -x[n // 2:][::-1])


def test_oracle_gauss_matches_numpy():
    for n in (3, 7, 64, 256, 1024):
        x, w = O.gauss_legendre(n)
        xn, wn = np.polynomial.legendre.leggauss(n)
        assert np.max(np.abs(x - xn)) <= 1e-14
        assert np.max(np.abs(w - wn)) <= 5e-14  # numpy itself drifts at n = 1024
        assert abs(w.sum() - 2.0) <= 1e-13


def test_laser_magnus_rule_matches_reference():
    # gauss.hpp stores the 30-point rule on [-1, 1] (as 0.5 (x + 1), 0.5 w)
    g = GOLD["laser30"]
    x, w = O.gauss_legendre(30)
    xs = np.array(g["nodes_pm1"])
    ws = np.array(g["weights_pm1"])
    # reference order: negative nodes by increasing |x|, then positive ascending
    ref = np.concatenate([xs[:15], xs[15:]])
    mine = np.concatenate([-x[15:], x[15:]])
    assert np.max(np.abs(ref - mine)) <= 2e-17 + 1e-16
    assert np.max(np.abs(ws - np.concatenate([w[15:], w[15:]]))) <= 1e-16


def test_product_gauss_matches_oracle():
    api = pytest.importorskip("higherharmonics_b200.api")
    for n in (8, 64, 128, 512, 1024):
        x, w = api.gauss_legendre(n)
        xo, wo = O.gauss_legendre(n)
        assert np.array_equal(x, xo) and np.array_equal(w, wo)
