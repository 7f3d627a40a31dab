"""Pins the oracle (the CPU restatement used as the checker) against the reference
library's own outputs, stored as golden fixtures by tests/golden/make_golden.py."""
import numpy as np
import pytest
from cases import CASES, STRATA_CASES, inputs
from conftest import golden, rel

# gemv tolerance against the reference.  Real cases reproduce the reference's pivots and
# agree to rounding.  In the complex Helmholtz cases on the symmetric cylinder grid, a few
# leaves (4 of 940 in helmholtz_small) meet ACA+ pivot candidates that tie to the last
# bit; the reference's OpenBLAS summation order and the restatement's break those ties
# differently, giving a different but equally accurate rank-k approximation of those
# leaves (both within the compression epsilon of the exact block, checked below).
# On the 100,000-point cylinder, 43 of the 35,084 Rk leaves meet such ties (same ranks, both
# approximations within epsilon of the exact block): 1.5e-8 on the product.
GEMV_TOL = {"helmholtz_small": 2e-6, "cfg1_cylinder": 5e-8}

INFO_KEYS = ["full_count", "rk_count", "full_size", "rk_size", "compressed_size", "uncompressed_size",
             "nr_block_clusters", "largest_rk_dim_rows", "largest_rk_dim_cols", "largest_rk_mem_rows",
             "largest_rk_mem_cols", "largest_rk_mem_rank"]


def build_oracle(oracle, name):
    _, kern, tree, nrhs, seed, scalar, dump = CASES[name]
    pts, x = inputs(name)
    o = oracle.OracleHMatrix(pts, leaf=tree["leaf"], eta=tree["eta"], leaf_cols=tree.get("leaf_cols"))
    return o, pts, x, kern, tree


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_structure_matches_reference(oracle, name):
    g = golden(name)
    o, pts, x, kern, tree = build_oracle(oracle, name)
    assert np.array_equal(o.perm(), g["perm"])
    assert np.array_equal(o.perm_cols(), g["perm_cols"])
    L = o.leaves()
    assert L.shape == g["leaves"].shape
    assert np.array_equal(L[:, :5], g["leaves"][:, :5])


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_assembly_and_gemv_match_reference(oracle, name):
    g = golden(name)
    o, pts, x, kern, tree = build_oracle(oracle, name)
    o.assemble(eps=tree["eps"], min_leaf=tree.get("min_leaf", 0), **kern)
    if tree.get("retrunc"):
        o.retruncate(tree["retrunc"])
    L = o.leaves()
    assert np.array_equal(L[:, 5], g["leaves"][:, 5]), "ranks differ from the reference"
    info = o.info()
    for k in INFO_KEYS:
        assert info[k] == int(g["info_" + k]), k
    tol = GEMV_TOL.get(name, 1e-12)
    assert rel(o.gemv(x, "N"), g["y"]) < tol
    assert rel(o.gemv(x, "T"), g["y_T"]) < tol
    if "y_C" in g:
        assert rel(o.gemv(x, "C"), g["y_C"]) < tol


@pytest.mark.parametrize("name", [n for n in sorted(CASES) if CASES[n][6]])
def test_oracle_rk_factors_match_reference(oracle, name):
    g = golden(name)
    o, pts, x, kern, tree = build_oracle(oracle, name)
    o.assemble(eps=tree["eps"], **kern)
    if tree.get("retrunc"):
        o.retruncate(tree["retrunc"])
    L = o.leaves()
    pay = g["rk_payload"]
    perm = o.perm()
    off = 0
    flips = 0
    nrk = 0
    for i, (r0, m, c0, n, t, k) in enumerate(g["leaves"]):
        if t != 1 or k <= 0:
            continue
        nrk += 1
        A = pay[off:off + k * m].reshape(k, m).T
        B = pay[off + k * m:off + k * (m + n)].reshape(k, n).T
        off += k * (m + n)
        Mr = A @ B.T
        Mo = o.block(i, L)
        if rel(Mo, Mr) < 1e-11:
            continue
        # a pivot-tie flip: both must still approximate the exact block within epsilon
        flips += 1
        ex = oracle.kernel_matrix(pts[perm[r0:r0 + m]], pts[perm[c0:c0 + n]], **kern)
        tol = 10 * max(tree["eps"], tree.get("retrunc", 0.0))
        assert rel(Mr, ex) < tol and rel(Mo, ex) < tol
    assert off == len(pay)
    assert flips <= max(1, nrk // 100)


@pytest.mark.parametrize("name", sorted(STRATA_CASES))
def test_oracle_multi_strata_assembly_matches_reference(oracle, name):
    """compress() over strata (compression.cpp:745-773) and formattedAddParts
    (rk_matrix.cpp:846-1009), restated: the reference assembled these matrices through
    advanced_compute with one stratum a material; the oracle must give the same partition
    and ranks, the same products to 1e-12 and, where stored, the same Rk blocks.  The cases
    take both branches of formattedAddParts (concatenation, and the full-block sum compressed
    by SVD once the summed rank reaches min(m, n)), real and complex, one with a negative
    stratum weight."""
    g = golden(name)
    _, kern, tree, nrhs, seed, scalar, dump = STRATA_CASES[name]
    pts, x = inputs(name)
    o = oracle.OracleHMatrix(pts, leaf=tree["leaf"], eta=tree["eta"])
    o.assemble(eps=tree["eps"], **kern)
    L = o.leaves()
    assert np.array_equal(o.perm(), g["perm"])
    assert np.array_equal(L, g["leaves"]), "partition or ranks differ from the reference"
    assert rel(o.gemv(x, "N"), g["y"]) < 1e-12
    assert rel(o.gemv(x, "T"), g["y_T"]) < 1e-12
    if "y_C" in g:
        assert rel(o.gemv(x, "C"), g["y_C"]) < 1e-12
    if dump:
        pay, off = g["rk_payload"], 0
        for i, (r0, m, c0, n, t, k) in enumerate(g["leaves"]):
            if t != 1 or k <= 0:
                continue
            A = pay[off:off + k * m].reshape(k, m).T
            B = pay[off + k * m:off + k * (m + n)].reshape(k, n).T
            off += k * (m + n)
            assert rel(o.block(i, L), A @ B.T) < 1e-11, i
        assert off == len(pay)


def test_oracle_single_stratum_equals_plain_kernel(oracle):
    """One stratum of weight 1 is the plain kernel: the same leaves as the simple
    interaction callback's assembly."""
    pts, x = inputs("cube_expcov")
    a = oracle.OracleHMatrix(pts, leaf=32, eta=2.0)
    a.assemble(kind=1, eps=1e-6, ell=0.3)
    b = oracle.OracleHMatrix(pts, leaf=32, eta=2.0)
    b.assemble(kind=1, eps=1e-6, strata_param=[0.3], strata_weight=[1.0])
    assert np.array_equal(a.leaves(), b.leaves())
    assert rel(a.gemv(x), b.gemv(x)) == 0.0
