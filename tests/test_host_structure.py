"""The engine's host side (median clustering, bounding boxes, admissibility, block tree)
reproduces the reference's partition bit for bit: permutations, leaf lists and the
structural fields of hmat_info_t, against the golden fixtures.  Host-only."""
import numpy as np
import pytest
from cases import CASES, inputs
from conftest import golden


@pytest.mark.parametrize("name", sorted(CASES))
def test_partition_matches_reference(hb, name):
    g = golden(name)
    _, kern, tree, nrhs, seed, scalar, dump = CASES[name]
    pts, _ = inputs(name)
    vt = {"D": 1, "Z": 3}[scalar]
    h = hb.HMatrix(pts, hb.kernel(kern["kind"], wavenumber=kern.get("wavenumber", 0.0)), value_type=vt,
                   leaf_size=tree["leaf"], leaf_size_cols=tree.get("leaf_cols"), eta=tree["eta"],
                   epsilon=tree["eps"], assemble=False)
    try:
        assert np.array_equal(h.perm(), g["perm"])
        assert np.array_equal(h.perm(cols=True), g["perm_cols"])
        T = h.leaf_table()
        assert np.array_equal(T[:, :5], g["leaves"][:, :5])
        info = h.info()
        for k in ("full_count", "rk_count", "full_size", "rk_size", "uncompressed_size", "nr_block_clusters",
                  "largest_rk_dim_rows", "largest_rk_dim_cols"):
            assert info[k] == int(g["info_" + k]), k
    finally:
        h.close()


def test_partition_edge_cases(hb, oracle):
    rng = np.random.default_rng(3)
    for n, leaf in ((1, 8), (2, 1), (7, 8), (33, 4), (1000, 1000), (1001, 1000)):
        pts = rng.random((n, 3))
        h = hb.HMatrix(pts, hb.kernel(hb.LAPLACE_REG), leaf_size=leaf, assemble=False)
        o = oracle.OracleHMatrix(pts, leaf=leaf, eta=2.0)
        assert np.array_equal(h.perm(), o.perm())
        assert np.array_equal(h.leaf_table()[:, :5], o.leaves()[:, :5])
        h.close()
    # duplicated coordinates (exact ties in the stable sort)
    pts = np.repeat(rng.random((50, 3)), 4, axis=0)
    h = hb.HMatrix(pts, hb.kernel(hb.LAPLACE_REG), leaf_size=8, assemble=False)
    o = oracle.OracleHMatrix(pts, leaf=8, eta=2.0)
    assert np.array_equal(h.perm(), o.perm())
    assert np.array_equal(h.leaf_table()[:, :5], o.leaves()[:, :5])
    h.close()
