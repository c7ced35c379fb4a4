"""The batched GPU LU against the reference's lu_decomp / lu_solve contract (src/lu.c)."""
import numpy as np
import pytest

from openpeec_b200 import api
from oracle.pyoracle import Oracle

pytestmark = pytest.mark.gpu


def rand_c(n, seed):
    rng = np.random.default_rng(seed)
    return rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n))


def reconstruct(lu, piv):
    n = lu.shape[0]
    L = np.tril(lu, -1) + np.eye(n)
    U = np.triu(lu)
    return L @ U, piv


def apply_piv(a, piv):
    a = a.copy()
    for k, p in enumerate(piv):
        if p != k:
            a[[k, p]] = a[[p, k]]
    return a


@pytest.mark.parametrize("n", [1, 2, 7, 31, 32, 33, 65, 100, 257, 600])
def test_lu_matches_reference_rule(n):
    a = rand_c(n, n)
    info, lu, piv = api.lu_decomp(a)
    assert info == -1
    r_info, r_lu, r_piv = Oracle.lu_decomp(a)
    assert np.array_equal(piv, r_piv)                 # same pivot sequence
    assert np.max(np.abs(lu - r_lu)) <= 1e-9 * max(1.0, np.max(np.abs(r_lu)))
    prod, _ = reconstruct(lu, piv)
    assert np.max(np.abs(prod - apply_piv(a, piv))) <= 1e-11 * n * np.max(np.abs(a))


@pytest.mark.parametrize("n", [5, 64, 300])
def test_lu_solve(n):
    a = rand_c(n, 100 + n)
    b = np.random.default_rng(1).normal(size=n) + 0j
    info, lu, piv = api.lu_decomp(a)
    x = api.lu_solve(lu, piv, b)
    assert np.max(np.abs(a @ x - b)) <= 1e-10 * np.max(np.abs(b)) * n


@pytest.mark.parametrize("n", [1100, 2050])
def test_cooperative_panels_match_reference_rule(n):
    """Orders whose panels are 1024 rows or more take the cooperative panel (rows split over
    many CTAs, candidates exchanged through a bounded grid barrier): the same pivot sequence
    as the reference's rule and the same factors as the one-CTA panel would give."""
    a = rand_c(n, 7 + n)
    info, lu, piv = api.lu_decomp(a)
    assert info == -1
    r_info, r_lu, r_piv = Oracle.lu_decomp(a)
    assert np.array_equal(piv, r_piv)
    assert np.max(np.abs(lu - r_lu)) <= 1e-9 * max(1.0, np.max(np.abs(r_lu)))
    a[:, n // 2] = 0                                   # zero column: zero pivot at n // 2
    info, _, _ = api.lu_decomp(a)
    assert info == n // 2, info


def test_lu_singular_row():
    a = rand_c(6, 3)
    a[:, 2] = 0                                       # column 2 all zero -> zero pivot at k = 2
    info, _, _ = api.lu_decomp(a)
    assert info == 2
    a = np.zeros((4, 4), complex)
    assert api.lu_decomp(a)[0] == 0
