"""Batches of independent H-matrices (hmat_b200_batch_create / _assemble / _offsets): every
member's leaves come out of one assembly (one launch per phase for all members) and every
member's product out of one gemv, each as in a run of that member alone.

* Members with uneven sizes and their own correlation lengths (exponential covariance, the
  uneven-batch workload's kind of matrix at small sizes): partition and ranks equal to the
  member's own assembly, leaf payloads byte for byte, products within rounding (the batch
  splits the output blocks' work into other chunks, so sums are grouped differently), and the
  batch's product takes the launches of one matrix's product (all on the default schedule).
* A batch of two reference fixtures (an 800-point and the 20,000-point cube): each member's
  partition, ranks and products equal to the reference's.
"""
import importlib.util
import os

import numpy as np
import pytest
from cases import CASES, inputs
from conftest import ROOT, golden, rel

pytestmark = pytest.mark.gpu


def _wl():
    spec = importlib.util.spec_from_file_location("wl_batch", os.path.join(ROOT, "hmat-oss_b200", "workloads.py"))
    wl = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(wl)
    return wl


def _members(hb, count=6, seed=0):
    wl = _wl()
    rng = np.random.default_rng(seed)
    sizes = np.round(np.exp(rng.uniform(np.log(600), np.log(4000), count))).astype(int)
    ells = rng.uniform(0.1, 0.5, count)
    pts = [wl.cube(int(n), 100 + i) for i, n in enumerate(sizes)]
    kers = [hb.kernel(hb.EXP_COV, ell=float(e), nugget=1e-6) for e in ells]
    return pts, kers


@pytest.mark.parametrize("vt,tol", [(1, 1e-13), (0, 1e-6)])
def test_batch_matches_each_member_alone(hb, vt, tol, monkeypatch):
    # the default gemv schedule for all: the batch's leaves pass the size above which the gemv
    # tuner may pick other chunk sizes, its members' do not
    monkeypatch.setenv("HMAT_B200_GEMV_TUNE", "0")
    hb.set_parameters(compressionMinLeafSize=0)
    pts, kers = _members(hb)
    batch = hb.HMatrixBatch(pts, kers, value_type=vt, leaf_size=32, eta=2.0, epsilon=1e-5)
    singles = [hb.HMatrix(p, k, value_type=vt, leaf_size=32, eta=2.0, epsilon=1e-5) for p, k in zip(pts, kers)]
    try:
        rb, lb = batch.offsets()
        assert rb[-1] == sum(len(p) for p in pts)
        T = batch.leaf_table()
        rng = np.random.default_rng(9)
        for i, h in enumerate(singles):
            Ti = h.leaf_table()
            seg = T[lb[i]:lb[i + 1]].copy()
            seg[:, 0] -= rb[i]
            seg[:, 2] -= rb[i]
            assert np.array_equal(seg, Ti), f"member {i}: partition or ranks differ"
            assert np.array_equal(batch.perm()[rb[i]:rb[i + 1]] - rb[i], h.perm())
            for leaf in rng.choice(len(Ti), size=min(150, len(Ti)), replace=False):
                a = batch.leaf_payload(int(lb[i] + leaf))
                b = h.leaf_payload(int(leaf))
                assert a.tobytes() == b.tobytes(), f"member {i} leaf {leaf}"
        X = np.asfortranarray(rng.standard_normal((int(rb[-1]), 3))).astype(batch.dtype)
        for trans in ("N", "T"):
            Y = batch.gemv(X, trans)
            for i, h in enumerate(singles):
                yi = h.gemv(np.asfortranarray(X[rb[i]:rb[i + 1]]), trans)
                assert rel(Y[rb[i]:rb[i + 1]], yi) < tol, (trans, i)
        assert batch.gemv_launches(16) <= max(h.gemv_launches(16) for h in singles)
    finally:
        batch.close()
        for h in singles:
            h.close()


def test_batch_of_reference_fixtures(hb):
    names = ["cube_expcov", "cfg4_cube"]
    pts, kers, xs = [], [], []
    for nm in names:
        _, kern, tree, nrhs, seed, scalar, dump = CASES[nm]
        p, x = inputs(nm)
        pts.append(p)
        kers.append(hb.kernel(hb.EXP_COV, ell=kern["ell"], nugget=kern["nugget"]))
        xs.append(x)
    hb.set_parameters(compressionMinLeafSize=0)
    # one leaf size for the batch: both fixtures' own (32 and 64) differ, so each member is
    # built with its fixture's leaf size through its own clustering
    wl_members = []
    for nm, p, k in zip(names, pts, kers):
        tree = CASES[nm][2]
        wl_members.append(hb.HMatrix(p, k, value_type=hb.HMAT_DOUBLE_PRECISION, leaf_size=tree["leaf"],
                                     eta=tree["eta"], epsilon=tree["eps"], assemble=False))
    import ctypes as C
    lib = hb.load_library()
    arr = (C.c_void_p * 2)(*[m.m for m in wl_members])
    bm = lib.hmat_b200_batch_create(arr, 2)
    assert bm, lib.hmat_b200_last_error()
    try:
        asm = (C.c_void_p * 2)(*[m._assembly for m in wl_members])
        assert lib.hmat_b200_batch_assemble(bm, asm, wl_members[0]._comp) == 0, lib.hmat_b200_last_error()
        rb = np.zeros(3, np.int32)
        lb = np.zeros(3, np.int32)
        assert lib.hmat_b200_batch_offsets(bm, rb.ctypes.data, lb.ctypes.data) == 0
        nl = lib.hmat_b200_leaf_count(bm)
        T = np.zeros((nl, 6), np.int32)
        assert lib.hmat_b200_leaf_table(bm, T.ctypes.data) == 0
        hi = hb.HMatInterface(hb.HMAT_DOUBLE_PRECISION)
        nr = max(x.shape[1] for x in xs)
        X = np.zeros((int(rb[-1]), nr), order="F")
        for i, x in enumerate(xs):
            X[rb[i]:rb[i + 1], :x.shape[1]] = x
        for trans, key in (("N", "y"), ("T", "y_T")):
            Y = np.zeros_like(X)
            one = np.ones(1)
            zero = np.zeros(1)
            assert hi.gemv(trans.encode(), one.ctypes.data, bm, X.ctypes.data, zero.ctypes.data, Y.ctypes.data,
                           nr) == 0
            for i, nm in enumerate(names):
                g = golden(nm)
                seg = T[lb[i]:lb[i + 1]].copy()
                seg[:, 0] -= rb[i]
                seg[:, 2] -= rb[i]
                assert np.array_equal(seg, g["leaves"]), nm
                assert rel(Y[rb[i]:rb[i + 1], :xs[i].shape[1]], g[key]) < 1e-12, (nm, trans)
    finally:
        hb.HMatInterface(hb.HMAT_DOUBLE_PRECISION).destroy(bm)
        for m in wl_members:
            m.close()
