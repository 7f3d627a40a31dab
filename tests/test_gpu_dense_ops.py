"""Dense operations on an assembled matrix in the internal (cluster) numbering:
get_block / get_values (c_wrapping.hpp:833-890), gemm_dense (c_wrapping.hpp:302-366) with
its side / transposition flag algebra, and gemm_scalar (c_wrapping.hpp:254-271).

The reference: the dense matrix assembled from the oracle's leaves (which equal the
reference library's, see test_oracle_golden), in the internal numbering."""
import numpy as np
import pytest
from cases import CASES, inputs
from conftest import rel

pytestmark = pytest.mark.gpu


def _engine_and_dense(hb, oracle, name):
    _, kern, tree, nrhs, seed, scalar, dump = CASES[name]
    pts, _ = inputs(name)
    hb.set_parameters(compressionMinLeafSize=tree.get("min_leaf", 0))
    k = hb.kernel(kern["kind"], delta=kern.get("delta", 0.01), ell=kern.get("ell", 0.3),
                  nugget=kern.get("nugget", 0.0), wavenumber=kern.get("wavenumber", 0.0))
    vt = {"D": 1, "Z": 3}[scalar]
    h = hb.HMatrix(pts, k, value_type=vt, leaf_size=tree["leaf"], eta=tree["eta"], epsilon=tree["eps"])
    o = oracle.OracleHMatrix(pts, leaf=tree["leaf"], eta=tree["eta"])
    o.assemble(eps=tree["eps"], **kern)
    n = len(pts)
    dense = np.zeros((n, n), dtype=h.dtype)
    T = o.leaves()
    for i, (r0, m, c0, nn, t, kk) in enumerate(T):
        dense[r0:r0 + m, c0:c0 + nn] = o.block(i, T)
    return h, dense, n


@pytest.mark.parametrize("name,tol", [("cube_expcov", 1e-11), ("helmholtz_small", 5e-6)])
def test_get_block_and_values(hb, oracle, name, tol):
    h, dense, n = _engine_and_dense(hb, oracle, name)
    try:
        full, rows, cols = h.get_block(0, n, 0, n)
        assert rel(full, dense) < tol
        perm, permc = h.perm(), h.perm(cols=True)
        assert np.array_equal(rows, perm) and np.array_equal(cols, permc)
        sub, r2, c2 = h.get_block(5, 37, 100, 50)
        assert np.array_equal(sub, full[5:42, 100:150])
        assert np.array_equal(r2, perm[5:42]) and np.array_equal(c2, permc[100:150])
        ren, _, _ = h.get_block(0, n, 10, 20, renumber_rows=True)
        expect = np.empty_like(ren)
        expect[perm] = full[:, 10:30]
        assert np.array_equal(ren, expect)
        # natural numbering, 1-based, unsorted and repeated
        rng = np.random.default_rng(4)
        qr = rng.integers(1, n + 1, 23)
        qc = np.concatenate([rng.integers(1, n + 1, 17), [1, n, 1]])
        rev, revc = np.argsort(perm), np.argsort(permc)
        vals = h.get_values(qr, qc)
        assert np.array_equal(vals, full[np.ix_(rev[qr - 1], revc[qc - 1])])
    finally:
        h.close()


def _op(a, t):
    return {"N": a, "T": a.T, "C": a.conj().T, "J": a.conj()}[t]


@pytest.mark.parametrize("name", ["cube_expcov", "helmholtz_small"])
def test_gemm_dense_flags(hb, oracle, name):
    h, dense, n = _engine_and_dense(hb, oracle, name)
    try:
        B, _, _ = h.get_block(0, n, 0, n)
        cplx = np.iscomplexobj(B)
        rng = np.random.default_rng(9)

        def rnd(*shape):
            v = rng.standard_normal(shape)
            return v + 1j * rng.standard_normal(shape) if cplx else v

        alpha = (0.7 - 0.2j) if cplx else 0.7
        beta = (-1.5 + 0.5j) if cplx else -1.5
        nrhs = 3
        tbs = "NTC" if cplx else "NT"
        txs = "NTCJ" if cplx else "NT"
        for side in "LR":
            for tb in tbs:
                for tx in txs:
                    if side == "L":
                        x = rnd(n, nrhs) if tx in "NJ" else rnd(nrhs, n)
                        y0 = rnd(n, nrhs)
                        want = alpha * _op(B, tb) @ _op(x, tx) + beta * y0
                    else:
                        x = rnd(nrhs, n) if tx in "NJ" else rnd(n, nrhs)
                        y0 = rnd(nrhs, n)
                        want = alpha * _op(x, tx) @ _op(B, tb) + beta * y0
                    got = h.gemm_dense(tb, tx, side, alpha, x, beta, y0)
                    assert rel(got, want) < 1e-12, (side, tb, tx, rel(got, want))
        # gemm_scalar: gemv in the internal numbering
        x = rnd(n, 2)
        assert rel(h.gemm_scalar(x), B @ x) < 1e-12
        assert rel(h.gemm_scalar(x, "T", alpha=2.0, beta=1.0, y=x), 2.0 * B.T @ x + x) < 1e-12
    finally:
        h.close()
