"""Parity of the B200 engine (CUDA path, through the C ABI) with the reference library's
outputs (golden fixtures) and with the oracle, on the GPU.

FP64 engines (D, Z) must reproduce the reference's partition exactly, its ranks and leaf
approximations (up to rare pivot-tie flips, which must stay within the compression
epsilon of the exact block) and its products to 1e-12 relative.  Mixed-precision
engines (S, C: FP32 bulk, FP64 truncation) are checked against the FP64 results within
the compression epsilon.
"""
import numpy as np
import pytest
from cases import CASES, inputs
from conftest import golden, rel

pytestmark = pytest.mark.gpu

VT = {"D": 1, "Z": 3}
# Complex cases on the symmetric cylinder meet exact pivot ties (see test_oracle_golden).
# On the 100,000-point cylinder 43 of the 35,084 Rk leaves meet such ties against the
# reference (the oracle shows the same 43): same ranks, a different approximation of the
# block within epsilon of it, 1.5e-8 on the product.
GEMV_TOL = {"helmholtz_small": 2e-6, "helmholtz_payload": 2e-6, "cfg1_cylinder": 5e-8}
# Rank mismatches allowed against the reference: none, except in the complex tie cases.
TIE_CASES = ("helmholtz_small", "helmholtz_payload")


def rank_mismatches_allowed(name, n_rk):
    return max(1, n_rk // 100) if name in TIE_CASES else 0


def build_engine(hb, name, value_type=None, **over):
    _, kern, tree, nrhs, seed, scalar, dump = CASES[name]
    pts, x = inputs(name)
    hb.set_parameters(compressionMinLeafSize=tree.get("min_leaf", 0))
    k = hb.kernel(kern["kind"], delta=kern.get("delta", 0.01), ell=kern.get("ell", 0.3),
                  nugget=kern.get("nugget", 0.0), wavenumber=kern.get("wavenumber", 0.0))
    vt = VT[scalar] if value_type is None else value_type
    h = hb.HMatrix(pts, k, value_type=vt, leaf_size=tree["leaf"], leaf_size_cols=tree.get("leaf_cols"),
                   eta=tree["eta"], epsilon=tree["eps"], **over)
    if tree.get("retrunc"):
        h.truncate(tree["retrunc"])  # set_low_rank_epsilon + truncate, as the reference run did
    return h, pts, x, kern, tree


@pytest.mark.parametrize("name", sorted(CASES))
def test_fp64_engine_matches_reference(hb, name):
    g = golden(name)
    h, pts, x, kern, tree = build_engine(hb, name)
    try:
        T = h.leaf_table()
        assert np.array_equal(h.perm(), g["perm"])
        assert np.array_equal(h.perm(cols=True), g["perm_cols"])
        assert np.array_equal(T[:, :5], g["leaves"][:, :5])
        rk = g["leaves"][:, 4] == 1
        mism = int((T[rk, 5] != g["leaves"][rk, 5]).sum())
        assert mism <= rank_mismatches_allowed(name, int(rk.sum())), f"{mism} rank mismatches"
        tol = GEMV_TOL.get(name, 1e-12)
        assert rel(h.gemv(x, "N"), g["y"]) < tol
        assert rel(h.gemv(x, "T"), g["y_T"]) < tol
        if "y_C" in g:
            assert rel(h.gemv(x, "C"), g["y_C"]) < tol
    finally:
        h.close()


@pytest.mark.parametrize("name", [n for n in sorted(CASES) if CASES[n][6]])
def test_fp64_engine_rk_factors_match_reference(hb, oracle, name):
    g = golden(name)
    h, pts, x, kern, tree = build_engine(hb, name)
    try:
        T = h.leaf_table()
        perm = h.perm()
        pay = g["rk_payload"]
        off = flips = nrk = 0
        for i, (r0, m, c0, n, t, k) in enumerate(g["leaves"]):
            if t != 1 or k <= 0:
                continue
            nrk += 1
            A = pay[off:off + k * m].reshape(k, m).T
            B = pay[off + k * m:off + k * (m + n)].reshape(k, n).T
            off += k * (m + n)
            Mr = A @ B.T
            Me = h.leaf_block(i)
            if rel(Me, Mr) < 1e-11:
                continue
            flips += 1
            ex = oracle.kernel_matrix(pts[perm[r0:r0 + m]], pts[perm[c0:c0 + n]], **kern)
            assert rel(Me, ex) < 10 * max(tree["eps"], tree.get("retrunc", 0.0)), (i, rel(Me, ex))
        assert flips <= max(1, nrk // 100)
        # full leaves are plain kernel entries: exact agreement with the FP64 formula
        for i in np.nonzero(T[:, 4] == 0)[0][:50]:
            r0, m, c0, n, t, k = T[i]
            ex = oracle.kernel_matrix(pts[perm[r0:r0 + m]], pts[perm[c0:c0 + n]], **kern,
                                      ids=(perm[r0:r0 + m], perm[c0:c0 + n]))
            assert rel(h.leaf_block(i), ex) < 1e-14
    finally:
        h.close()


@pytest.mark.parametrize("name", ["cfg0_laplace", "cube_expcov", "helmholtz_small"])
def test_engine_matches_oracle(hb, oracle, name):
    """Same inputs through the engine and the oracle: ranks and products."""
    h, pts, x, kern, tree = build_engine(hb, name)
    try:
        o = oracle.OracleHMatrix(pts, leaf=tree["leaf"], eta=tree["eta"])
        o.assemble(eps=tree["eps"], **kern)
        tol = GEMV_TOL.get(name, 1e-12)
        assert rel(h.gemv(x, "N"), o.gemv(x, "N")) < tol
        assert rel(h.gemv(x, "T"), o.gemv(x, "T")) < tol
    finally:
        h.close()


@pytest.mark.parametrize("name,vt", [("cfg0_laplace", 0), ("cube_expcov", 0), ("helmholtz_small", 2)])
def test_mixed_precision_within_epsilon(hb, oracle, name, vt):
    """FP32 bulk + FP64 truncation against the FP64 dense product: the error stays at
    the compression epsilon level (not above the FP64 H-matrix's own error by more than
    the FP32 rounding floor)."""
    h64, pts, x, kern, tree = build_engine(hb, name)
    h32, _, _, _, _ = build_engine(hb, name, value_type=vt)
    try:
        dense = oracle.dense_product(pts, x, **kern)
        e64 = rel(h64.gemv(x), dense)
        e32 = rel(h32.gemv(x.astype(np.complex64 if vt == 2 else np.float32)).astype(dense.dtype), dense)
        eps = max(tree["eps"], tree.get("retrunc", 0.0))
        assert e64 < 10 * eps
        assert e32 < max(2 * e64, 20 * eps) + 1e-5, (e32, e64)
        T64, T32 = h64.leaf_table(), h32.leaf_table()
        assert np.array_equal(T64[:, :5], T32[:, :5])
    finally:
        h64.close()
        h32.close()


def test_gemv_alpha_beta_and_multi_rhs(hb, oracle):
    h, pts, x, kern, tree = build_engine(hb, "cube_expcov")
    try:
        rng = np.random.default_rng(5)
        X = np.asfortranarray(rng.standard_normal((len(pts), 21)))
        Y0 = np.asfortranarray(rng.standard_normal((len(pts), 21)))
        o = oracle.OracleHMatrix(pts, leaf=tree["leaf"], eta=tree["eta"])
        o.assemble(eps=tree["eps"], **kern)
        ref = 0.5 * o.gemv(X) - 2.0 * Y0
        got = h.gemv(X, alpha=0.5, beta=-2.0, y=Y0)
        assert rel(got, ref) < 1e-12
        # one right-hand side at a time gives the same columns
        for q in (0, 7, 20):
            assert rel(h.gemv(X[:, q]), o.gemv(X[:, q])) < 1e-12
    finally:
        h.close()


@pytest.mark.parametrize("nrhs", [1, 16])
def test_mixed_gemv_accuracy_wide_leaves(hb, nrhs):
    """The FP32 product keeps FP32 accuracy on leaves thousands of columns wide: on a
    20,000-point cylinder at epsilon 1e-6 the mixed engine stays within 2e-6 of the FP64
    H-matrix product (FP32 assembly and ACA alone give about 1e-6 here)."""
    import importlib.util
    import os
    from conftest import ROOT
    spec = importlib.util.spec_from_file_location("wl_acc", os.path.join(ROOT, "hmat-oss_b200", "workloads.py"))
    wl = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(wl)
    pts = wl.cylinder(100, 200)
    hb.set_parameters(compressionMinLeafSize=0)
    k = hb.kernel(hb.LAPLACE_REG, delta=0.01)
    h64 = hb.HMatrix(pts, k, value_type=hb.HMAT_DOUBLE_PRECISION, leaf_size=64, eta=2.0, epsilon=1e-6)
    h32 = hb.HMatrix(pts, k, value_type=hb.HMAT_SIMPLE_PRECISION, leaf_size=64, eta=2.0, epsilon=1e-6)
    try:
        x = wl.rhs(len(pts), nrhs, 11)
        y64 = h64.gemv(x)
        y32 = h32.gemv(x.astype(np.float32)).astype(np.float64)
        assert rel(y32, y64) < 2e-6
    finally:
        h64.close()
        h32.close()


@pytest.mark.parametrize("nrhs", [1, 5, 16])
def test_fp32_product_error_on_stored_leaves(hb, nrhs):
    """The FP32 products' own rounding, apart from assembly and compression: the mixed
    engine's 'N' and 'T' products against the product of its stored FP32 leaves summed in
    FP64.  The tensor-core split (its dropped lo x lo term and the TF32 rounding of the lo
    parts cost up to 2^-21 a product) with round-to-nearest partial sums stays below 1e-6
    relative, within four times a float32 BLAS evaluation of the same leaves (numpy, leaf by
    leaf)."""
    import importlib.util
    import os
    from conftest import ROOT
    spec = importlib.util.spec_from_file_location("wl_rnd", os.path.join(ROOT, "hmat-oss_b200", "workloads.py"))
    wl = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(wl)
    pts = wl.cylinder(60, 120)
    hb.set_parameters(compressionMinLeafSize=0)
    h = hb.HMatrix(pts, hb.kernel(hb.LAPLACE_REG, delta=0.01), value_type=hb.HMAT_SIMPLE_PRECISION,
                   leaf_size=64, eta=2.0, epsilon=1e-6)
    try:
        n = len(pts)
        x = wl.rhs(n, nrhs, 17).astype(np.float32)
        x64 = x.astype(np.float64)
        pr, pc = h.perm(), h.perm(cols=True)
        ex = {"N": np.zeros((n, nrhs)), "T": np.zeros((n, nrhs))}
        f32 = {"N": np.zeros((n, nrhs), np.float32), "T": np.zeros((n, nrhs), np.float32)}
        for i, (r0, m, c0, nn, t, k) in enumerate(h.leaf_table()):
            rows, cols = pr[r0:r0 + m], pc[c0:c0 + nn]
            p = h.leaf_payload(i)
            if t == 0:
                F = p.reshape(nn, m).T
                ex["N"][rows] += F.astype(np.float64) @ x64[cols]
                ex["T"][cols] += F.T.astype(np.float64) @ x64[rows]
                f32["N"][rows] += F @ x[cols]
                f32["T"][cols] += F.T @ x[rows]
            elif k > 0:
                A = p[:k * m].reshape(k, m).T
                B = p[k * m:].reshape(k, nn).T
                A64, B64 = A.astype(np.float64), B.astype(np.float64)
                ex["N"][rows] += A64 @ (B64.T @ x64[cols])
                ex["T"][cols] += B64 @ (A64.T @ x64[rows])
                f32["N"][rows] += A @ (B.T @ x[cols])
                f32["T"][cols] += B @ (A.T @ x[rows])
        for trans in ("N", "T"):
            got = h.gemv(x, trans).astype(np.float64)
            e_dev = rel(got, ex[trans])
            e_np = rel(f32[trans].astype(np.float64), ex[trans])
            print(f"nrhs {nrhs} {trans}: device {e_dev:.3e}, float32 BLAS {e_np:.3e}")
            assert e_dev < 1e-6
            assert e_dev < 4 * e_np + 1e-8
    finally:
        h.close()


@pytest.mark.parametrize("name", ["cfg0_laplace", "cube_expcov", "helmholtz_small", "tall_partial"])
def test_single_rhs_transposed_products(hb, oracle, name):
    """Transposed products ('T', and 'C' for complex values) with one right-hand side agree
    with the oracle like the wider tiles do, with alpha and beta on the scattered output."""
    h, pts, x, kern, tree = build_engine(hb, name)
    try:
        o = oracle.OracleHMatrix(pts, leaf=tree["leaf"], eta=tree["eta"], leaf_cols=tree.get("leaf_cols"))
        o.assemble(eps=tree["eps"], **kern)
        tol = GEMV_TOL.get(name, 1e-12)
        x1 = np.asfortranarray(x[:, :1])
        assert rel(h.gemv(x1, "T"), o.gemv(x1, "T")) < tol
        if np.iscomplexobj(x1):
            assert rel(h.gemv(x1, "C"), o.gemv(x1, "C")) < tol
        y0 = np.asfortranarray(np.ones_like(x1) * 0.5)
        got = h.gemv(x1, "T", alpha=2.0, beta=-1.0, y=y0)
        assert rel(got, 2.0 * o.gemv(x1, "T") - y0) < tol
    finally:
        h.close()


@pytest.mark.parametrize("nrhs", [16, 5])
def test_tensor_memory_y_phase_matches_warp_level(hb, nrhs, monkeypatch):
    """The opt-in tensor-memory y-phase (tcgen05.mma with tensor-memory accumulators,
    HMAT_B200_TC_Y=1) computes the FP32 'N' product to the accuracy of the default
    warp-level tensor-core kernel: both within 2e-6 of the FP64 product, and within 1e-6
    of each other."""
    import importlib.util
    import os
    from conftest import ROOT
    spec = importlib.util.spec_from_file_location("wl_tc", os.path.join(ROOT, "hmat-oss_b200", "workloads.py"))
    wl = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(wl)
    pts = wl.cylinder(60, 120)
    hb.set_parameters(compressionMinLeafSize=0)
    k = hb.kernel(hb.LAPLACE_REG, delta=0.01)
    h64 = hb.HMatrix(pts, k, value_type=hb.HMAT_DOUBLE_PRECISION, leaf_size=64, eta=2.0, epsilon=1e-6)
    h32 = hb.HMatrix(pts, k, value_type=hb.HMAT_SIMPLE_PRECISION, leaf_size=64, eta=2.0, epsilon=1e-6)
    monkeypatch.setenv("HMAT_B200_TC_Y", "1")
    htc = hb.HMatrix(pts, k, value_type=hb.HMAT_SIMPLE_PRECISION, leaf_size=64, eta=2.0, epsilon=1e-6)
    try:
        x = wl.rhs(len(pts), nrhs, 13)
        y64 = h64.gemv(x)
        y32 = h32.gemv(x.astype(np.float32)).astype(np.float64)
        ytc = htc.gemv(x.astype(np.float32)).astype(np.float64)
        assert np.isfinite(ytc).all()
        assert rel(y32, y64) < 2e-6
        assert rel(ytc, y64) < 2e-6
        assert rel(ytc, y32) < 1e-6
        # alpha / beta through the final pass
        y0 = np.ones_like(x, dtype=np.float32)
        got = htc.gemv(x.astype(np.float32), alpha=0.5, beta=2.0, y=y0).astype(np.float64)
        assert rel(got, 0.5 * y64 + 2.0) < 2e-6
    finally:
        h64.close()
        h32.close()
        htc.close()


@pytest.mark.parametrize("name", sorted(CASES))
def test_high_rank_truncation_path_matches_reference(hb, name, monkeypatch):
    """The truncation phases for ranks above the register buckets (a CTA per row segment, per
    stack of triangles and per core) give the reference's ranks and products: with
    HMAT_B200_TS_KMAX=0 every leaf that is not a dense-SVD job takes them."""
    monkeypatch.setenv("HMAT_B200_TS_KMAX", "0")
    g = golden(name)
    h, pts, x, kern, tree = build_engine(hb, name)
    try:
        T = h.leaf_table()
        assert np.array_equal(T[:, :5], g["leaves"][:, :5])
        rk = g["leaves"][:, 4] == 1
        mism = int((T[rk, 5] != g["leaves"][rk, 5]).sum())
        assert mism <= rank_mismatches_allowed(name, int(rk.sum())), f"{mism} rank mismatches"
        tol = GEMV_TOL.get(name, 1e-12)
        assert rel(h.gemv(x, "N"), g["y"]) < tol
        assert rel(h.gemv(x, "T"), g["y_T"]) < tol
    finally:
        h.close()


def test_headline_cylinder_100k(hb, oracle):
    """The benchmark's workload (100,000-point cylinder, leaf 64, eta 2, epsilon 1e-6) pinned to
    the reference: the FP64 engine gives the reference's partition and every rank, its 'N' and
    'T' products within the tie-flip tolerance, and the oracle's product (same pivot rules)
    within 1e-12.  The mixed engine (FP32 bulk, FP64 truncation) keeps the partition and stays
    within 1e-6 of the FP64 H-matrix product on the benchmark's 16 right-hand sides."""
    import importlib.util
    import os
    from conftest import ROOT
    spec = importlib.util.spec_from_file_location("wl_cfg1", os.path.join(ROOT, "hmat-oss_b200", "workloads.py"))
    wl = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(wl)
    name = "cfg1_cylinder"
    g = golden(name)
    h64, pts, x, kern, tree = build_engine(hb, name)
    h32 = None
    try:
        T = h64.leaf_table()
        assert np.array_equal(h64.perm(), g["perm"])
        assert np.array_equal(T[:, :5], g["leaves"][:, :5])
        assert np.array_equal(T[:, 5], g["leaves"][:, 5]), "ranks differ from the reference"
        y = h64.gemv(x, "N")
        assert rel(y, g["y"]) < GEMV_TOL[name]
        assert rel(h64.gemv(x, "T"), g["y_T"]) < GEMV_TOL[name]
        o = oracle.OracleHMatrix(pts, leaf=tree["leaf"], eta=tree["eta"])
        o.assemble(eps=tree["eps"], **kern)
        assert np.array_equal(o.leaves(), T)
        assert rel(y, o.gemv(x, "N")) < 1e-12
        o.close()
        h32, _, _, _, _ = build_engine(hb, name, value_type=hb.HMAT_SIMPLE_PRECISION)
        assert np.array_equal(h32.leaf_table()[:, :5], T[:, :5])
        x16 = wl.rhs(len(pts), 16, 1)
        y64 = h64.gemv(x16)
        y32 = h32.gemv(x16.astype(np.float32)).astype(np.float64)
        err = rel(y32, y64)
        print(f"mixed vs FP64 H-matrix, 16 RHS: {err:.3e}")
        assert err <= 1e-6
        # size-independent properties at full size: repeated products bitwise identical (fixed
        # summation orders), and linearity in x within rounding
        x32 = x16.astype(np.float32)
        assert np.array_equal(h32.gemv(x32), h32.gemv(x32))
        assert np.array_equal(h64.gemv(x16), y64)
        xa, xb = x16[:, :8], x16[:, 8:]
        ylin = h64.gemv(np.asfortranarray(2.0 * xa - 0.5 * xb))
        assert rel(ylin, 2.0 * y64[:, :8] - 0.5 * y64[:, 8:]) < 1e-13
    finally:
        h64.close()
        if h32 is not None:
            h32.close()


@pytest.mark.parametrize("name", ["cfg4_cube", "cfg0_laplace", "helmholtz_small"])
def test_aca_capacity_retries_and_workspace_batches_match_reference(hb, name, monkeypatch):
    """The ACA rank-capacity retry (leaves that fill their factor slots are rerun with twice
    the capacity) and the batching of the ACA workspace give the reference's ranks and
    products: an initial capacity of 4 makes most leaves retry, some several times, and a
    64 MiB workspace budget cuts the 20,000-point cube's leaves into many batches."""
    monkeypatch.setenv("HMAT_B200_ACA_KCAP", "4")
    monkeypatch.setenv("HMAT_B200_WORKSPACE_MB", "64")
    g = golden(name)
    h, pts, x, kern, tree = build_engine(hb, name)
    try:
        T = h.leaf_table()
        assert np.array_equal(T[:, :5], g["leaves"][:, :5])
        rk = g["leaves"][:, 4] == 1
        assert int((T[rk, 5] > 4).sum()) > 0  # leaves above the initial capacity exist
        mism = int((T[rk, 5] != g["leaves"][rk, 5]).sum())
        assert mism <= rank_mismatches_allowed(name, int(rk.sum())), f"{mism} rank mismatches"
        tol = GEMV_TOL.get(name, 1e-12)
        assert rel(h.gemv(x, "N"), g["y"]) < tol
        assert rel(h.gemv(x, "T"), g["y_T"]) < tol
    finally:
        h.close()


def test_gemv_tuner_schedules_give_the_same_products(hb, oracle, monkeypatch):
    """The gemv tuner (HMAT_B200_GEMV_TUNE=2: every candidate schedule measured, whatever the
    matrix size) picks a z chunk size and a y unit width; the product with its schedule equals
    the oracle's like the default schedule's does (FP64, 1e-12), and the report names the
    measured candidates."""
    monkeypatch.setenv("HMAT_B200_GEMV_TUNE", "2")
    h, pts, x, kern, tree = build_engine(hb, "cube_expcov")
    try:
        t = h.gemv_tuning()
        assert t["how"] == "measured"
        assert t["z_chunk_units"] in (8, 16, 32) and t["y_units"] in ("widest", "half")
        assert all(t["ms"][k] > 0 for k in ("z8", "z16", "z32", "y_widest", "y_half"))
        o = oracle.OracleHMatrix(pts, leaf=tree["leaf"], eta=tree["eta"])
        o.assemble(eps=tree["eps"], **kern)
        assert rel(h.gemv(x, "N"), o.gemv(x, "N")) < 1e-12
        assert rel(h.gemv(x, "T"), o.gemv(x, "T")) < 1e-12
    finally:
        h.close()
    monkeypatch.setenv("HMAT_B200_GEMV_TUNE", "0")
    h, pts, x, kern, tree = build_engine(hb, "cube_expcov")
    try:
        assert h.gemv_tuning()["how"] == "default"
    finally:
        h.close()
