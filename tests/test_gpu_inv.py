"""Inversion on the GPU through the C-ABI: FLA_SPDinv (lower and upper),
FLA_Trinv (lower/upper x unit/non-unit), FLA_Ttmm and the LAPACK dpotri_.

Checked against outputs of the reference libflame on the same inputs
(tests/golden/reference_small.npz, keys spdinv_*, trinv_*, ttmm_*, dpotri_*)
and, at larger sizes, against the CPU oracle composed as the reference
composes it (FLA_SPDinv_internal.c:27-36: Chol, then Trinv = forward
substitution on I, then Ttmm = L^T L).  Only the named triangle is
compared; the other triangle must be left untouched.  Tolerance: relative
Frobenius 1e-12 (kappa of the inputs is O(10))."""
import numpy as np
import pytest

from conftest import rel_fro, seeded, spd, to_dev, to_host

pytestmark = pytest.mark.gpu

TOL = 1e-12
L_, U_ = 300, 301
NONUNIT, UNIT = 501, 500


def _tri(a, lower, diag=True):
    return np.tril(a, 0 if diag else -1) if lower else np.triu(a, 0 if diag else 1)


@pytest.mark.parametrize("n", [50, 140])
def test_spdinv_and_dpotri_match_reference(cuda, flame, golden, n):
    torch = cuda
    A = golden["spdinv_%d_A" % n]
    for uplo, key, lower in [(L_, "L", True), (U_, "U", False)]:
        Ad = to_dev(torch, A)
        assert flame.spdinv(Ad, uplo) == flame.FLA_SUCCESS, flame.last_error()
        got = to_host(Ad)
        ref = golden["spdinv_%d_%s" % (n, key)]
        assert rel_fro(_tri(got, lower), _tri(ref, lower)) < TOL
        assert np.array_equal(_tri(got, not lower, False), _tri(A, not lower, False))
    # dpotri_ on dpotrf_'s factor
    Ad = to_dev(torch, A)
    assert flame.chol(Ad) == flame.FLA_SUCCESS
    assert flame.dpotri("L", Ad) == 0, flame.last_error()
    assert rel_fro(np.tril(to_host(Ad)), np.tril(golden["dpotri_%d_L" % n])) < TOL


@pytest.mark.parametrize("n", [50, 140])
def test_trinv_and_ttmm_match_reference(cuda, flame, golden, n):
    torch = cuda
    M = golden["trinv_%d_M" % n]
    for uplo, ul, lower in [(L_, "l", True), (U_, "u", False)]:
        for diag, dg in [(NONUNIT, "n"), (UNIT, "u")]:
            Md = to_dev(torch, M)
            assert flame.trinv(Md, uplo, diag) == flame.FLA_SUCCESS, flame.last_error()
            got, ref = to_host(Md), golden["trinv_%d_%s%s" % (n, ul, dg)]
            assert rel_fro(_tri(got, lower), _tri(ref, lower)) < TOL, (ul, dg)
            assert np.array_equal(_tri(got, not lower, False), _tri(M, not lower, False))
            if dg == "u" and (lower or n <= 128):
                assert np.array_equal(np.diag(got), np.diag(M))
            # above order 128 the reference's blocked upper unit-diagonal
            # variant computes the non-unit inverse; the GPU matches it
            if dg == "u" and not lower and n > 128:
                assert rel_fro(np.triu(got), np.triu(golden["trinv_%d_un" % n])) < TOL
        Md = to_dev(torch, M)
        assert flame.ttmm(Md, uplo) == flame.FLA_SUCCESS, flame.last_error()
        got, ref = to_host(Md), golden["ttmm_%d_%s" % (n, ul)]
        assert rel_fro(_tri(got, lower), _tri(ref, lower)) < TOL, ul
        assert np.array_equal(_tri(got, not lower, False), _tri(M, not lower, False))


@pytest.mark.parametrize("n", [129, 513, 2000])
def test_spdinv_matches_oracle_composition(cuda, flame, oracle, n):
    torch = cuda
    A = spd(seeded(n), n)
    Ad = to_dev(torch, A)
    assert flame.spdinv(Ad) == flame.FLA_SUCCESS
    Lo, _ = oracle.chol(A)
    Li = oracle.trsm_lln(np.tril(Lo), np.eye(n))
    Ai = Li.T @ Li
    assert rel_fro(np.tril(to_host(Ad)), np.tril(Ai)) < TOL
