"""Multi-strata assembly on the device (hmat_b200_create_assembly_strata) against the reference's
own multi-strata matrices: the reference assembled these fixtures through advanced_compute with
prepare setting number_of_strata, one stratum a material (compress() over strata,
compression.cpp:745-773; each further stratum added by RkMatrix::formattedAddParts,
rk_matrix.cpp:846-1009, by concatenation or, once the summed rank reaches min(m, n), as a full
block compressed by SVD).  The three cases take both branches, real and complex, one with a
negative weight.

* FP64 and complex FP64 engines: permutation, partition and every rank equal the reference's;
  products 'N', 'T' (and 'C') within 1e-12 (real) / 1e-10 (complex: measured 4.6e-11 'N',
  5.9e-11 'C'); where the fixture stores them, every Rk block within 1e-11.  The full leaves,
  which hold the summed strata, agree with the oracle's entry by entry within 1e-14 (measured
  1e-16 and below), so the complex gap arises in the compression arithmetic (ACA and
  truncation in another operation order than the reference's BLAS / LAPACK calls), not in
  the kernel entries.
* Mixed engines (FP32 / complex FP32 storage, FP64 truncation): the same partition, products
  within max(10 epsilon, 1e-5) of the FP64 engine's.
* One stratum of weight 1 is the plain kernel: the same leaves and bitwise the same product.
"""
import numpy as np
import pytest
from cases import STRATA_CASES, inputs
from conftest import golden, rel

pytestmark = pytest.mark.gpu

VT = {"D": 1, "Z": 3, "S": 0, "C": 2}
LOW = {"D": "S", "Z": "C"}


def _build(hb, name, scalar):
    _, kern, tree, nrhs, seed, _, dump = STRATA_CASES[name]
    pts, x = inputs(name)
    hb.set_parameters(compressionMinLeafSize=tree.get("min_leaf", 0))
    k = hb.kernel(kern["kind"], delta=kern.get("delta", 0.01), strata_param=kern["strata_param"],
                  strata_weight=kern["strata_weight"])
    h = hb.HMatrix(pts, k, value_type=VT[scalar], leaf_size=tree["leaf"], eta=tree["eta"], epsilon=tree["eps"])
    return h, pts, x, tree


GEMV_TOL = {"D": 1e-12, "Z": 1e-10}


@pytest.mark.parametrize("name", sorted(STRATA_CASES))
def test_strata_assembly_matches_reference(hb, oracle, name):
    g = golden(name)
    _, kern, _, _, _, scalar, dump = STRATA_CASES[name]
    h, pts, x, tree = _build(hb, name, scalar)
    try:
        # the summed strata of the full leaves against the oracle's (C library arithmetic)
        o = oracle.OracleHMatrix(pts, leaf=tree["leaf"], eta=tree["eta"])
        o.assemble(eps=tree["eps"], **kern)
        L = o.leaves()
        worst = 0.0
        for i in np.nonzero(L[:, 4] == 0)[0][:200]:
            r0, m, c0, n = L[i, :4]
            F = h.leaf_payload(int(i)).reshape(n, m).T
            worst = max(worst, rel(F, o.block(int(i), L)))
        yo = o.gemv(x, "N")
        o.close()
        print(f"{name}: full-leaf entries vs the oracle {worst:.2e}, product vs the oracle "
              f"{rel(h.gemv(x, 'N'), yo):.2e}")
        assert worst < 1e-14
        tol = GEMV_TOL[scalar]
        T = h.leaf_table()
        assert np.array_equal(h.perm(), g["perm"])
        assert np.array_equal(T[:, :5], g["leaves"][:, :5])
        rk = g["leaves"][:, 4] == 1
        assert np.array_equal(T[rk, 5], g["leaves"][rk, 5]), \
            f"{int((T[rk, 5] != g['leaves'][rk, 5]).sum())} rank mismatches"
        errs = {t: rel(h.gemv(x, t), g[k]) for t, k in (("N", "y"), ("T", "y_T"), ("C", "y_C")) if k in g}
        print(f"{name}: products vs the reference {errs}")
        assert all(e < tol for e in errs.values()), errs
        if dump:
            pay, off = g["rk_payload"], 0
            for i, (r0, m, c0, n, t, k) in enumerate(g["leaves"]):
                if t != 1 or k <= 0:
                    continue
                A = pay[off:off + k * m].reshape(k, m).T
                B = pay[off + k * m:off + k * (m + n)].reshape(k, n).T
                off += k * (m + n)
                p = h.leaf_payload(i)
                Ad = p[:m * k].reshape(k, m).T
                Bd = p[m * k:].reshape(k, n).T
                assert rel(Ad @ Bd.T, A @ B.T) < 1e-11, i
    finally:
        h.close()


@pytest.mark.parametrize("name", sorted(STRATA_CASES))
def test_strata_mixed_engine_within_epsilon(hb, name):
    scalar = STRATA_CASES[name][5]
    h64, pts, x, tree = _build(hb, name, scalar)
    h32, _, _, _ = _build(hb, name, LOW[scalar])
    try:
        assert np.array_equal(h32.leaf_table()[:, :5], h64.leaf_table()[:, :5])
        tol = max(10 * tree["eps"], 1e-5)
        for trans in ("N", "T"):
            y64 = h64.gemv(x, trans)
            y32 = h32.gemv(x.astype(h32.dtype), trans).astype(y64.dtype)
            assert rel(y32, y64) < tol, trans
    finally:
        h64.close()
        h32.close()


@pytest.mark.parametrize("vt", [1, 0])
def test_single_stratum_equals_plain_kernel(hb, vt):
    pts, x = inputs("cube_expcov")
    hb.set_parameters(compressionMinLeafSize=0)
    a = hb.HMatrix(pts, hb.kernel(hb.EXP_COV, ell=0.3), value_type=vt, leaf_size=32, eta=2.0, epsilon=1e-6)
    b = hb.HMatrix(pts, hb.kernel(hb.EXP_COV, strata_param=[0.3], strata_weight=[1.0]), value_type=vt,
                   leaf_size=32, eta=2.0, epsilon=1e-6)
    try:
        assert np.array_equal(a.leaf_table(), b.leaf_table())
        xx = x.astype(a.dtype)
        assert np.array_equal(a.gemv(xx), b.gemv(xx))
    finally:
        a.close()
        b.close()
