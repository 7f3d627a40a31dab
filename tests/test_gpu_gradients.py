"""Leaf gradients of L = 1/2 ||H x - b||^2 (hmat_b200_leaf_gradients), the adjoint of the
product with respect to the stored leaves.

With r = H x - b (any r here: the map is linear in r), per leaf:
    dF = r_I x_J^T                         full leaf F (m x n)
    dA = r_I (B^T x_J)^T,  dB = x_J (A^T r_I)^T   Rk leaf A B^T
summed over the right-hand sides; written in the canonical payload layout (full: m x n,
Rk: A m x k then B n x k, column-major, leaf order).  The reference has no counterpart;
it only offers the transposed product dx = H^T r (RkMatrix::gemv 'T', rk_matrix.cpp:156-206),
which the parity tests cover.

Checked against an FP64 restatement from the stored leaves (numpy), and through the
bilinear identity sum <dF, F> + sum <dA, A> = sum <dF, F> + sum <dB, B> = <r, H x>, which
holds at any size.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _setup(hb, vt, n_side=(24, 30), leaf=32, eps=1e-6):
    import importlib.util
    import os
    from conftest import ROOT
    spec = importlib.util.spec_from_file_location("wl_grad", os.path.join(ROOT, "hmat-oss_b200", "workloads.py"))
    wl = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(wl)
    pts = wl.cylinder(*n_side)
    hb.set_parameters(compressionMinLeafSize=0)
    h = hb.HMatrix(pts, hb.kernel(hb.LAPLACE_REG, delta=0.01), value_type=vt, leaf_size=leaf, eta=2.0,
                   epsilon=eps)
    return h, pts, wl


def _restated(h, x, r):
    """FP64 gradients from the stored leaves, canonical layout."""
    T = h.leaf_table()
    offs, total = h.payload_layout()
    pr, pc = h.perm(), h.perm(cols=True)
    g = np.zeros(total)
    for i, (r0, m, c0, n, t, k) in enumerate(T):
        rows, cols = pr[r0:r0 + m], pc[c0:c0 + n]
        ri, xj = r[rows].astype(np.float64), x[cols].astype(np.float64)
        p = h.leaf_payload(i).astype(np.float64)
        if t == 0:
            g[offs[i]:offs[i] + m * n] = (ri @ xj.T).T.ravel()
        elif k > 0:
            A = p[:k * m].reshape(k, m).T
            B = p[k * m:].reshape(k, n).T
            dA = ri @ (B.T @ xj).T
            dB = xj @ (A.T @ ri).T
            g[offs[i]:offs[i] + m * k] = dA.T.ravel()
            g[offs[i] + m * k:offs[i] + k * (m + n)] = dB.T.ravel()
    return g


def _device_grads(h, x, r, dtype, accumulate_twice=False):
    import torch
    n, nrhs = x.shape
    xd = torch.from_numpy(np.ascontiguousarray(x.T)).to("cuda", dtype)
    rd = torch.from_numpy(np.ascontiguousarray(r.T)).to("cuda", dtype)
    _, total = h.payload_layout()
    g = torch.full((total,), float("nan"), device="cuda", dtype=dtype)
    s = torch.cuda.Stream()
    h.leaf_gradients(xd.data_ptr(), rd.data_ptr(), nrhs, g.data_ptr(), accumulate=False, stream=s.cuda_stream)
    if accumulate_twice:
        h.leaf_gradients(xd.data_ptr(), rd.data_ptr(), nrhs, g.data_ptr(), accumulate=True, stream=s.cuda_stream)
    torch.cuda.synchronize()
    return g.cpu().numpy().astype(np.float64)


def _blocks(h, g):
    """Per-leaf <grad, leaf> split into full, A and B parts."""
    T = h.leaf_table()
    offs, _ = h.payload_layout()
    full = a_part = b_part = 0.0
    for i, (r0, m, c0, n, t, k) in enumerate(T):
        p = h.leaf_payload(i).astype(np.float64)
        if t == 0:
            full += g[offs[i]:offs[i] + m * n] @ p
        elif k > 0:
            a_part += g[offs[i]:offs[i] + m * k] @ p[:m * k]
            b_part += g[offs[i] + m * k:offs[i] + k * (m + n)] @ p[m * k:]
    return full, a_part, b_part


@pytest.mark.parametrize("vt,tol", [(1, 1e-12), (0, 2e-5)])
@pytest.mark.parametrize("nrhs", [1, 3, 16])
def test_gradients_match_fp64_restatement(hb, vt, tol, nrhs):
    import torch
    h, pts, wl = _setup(hb, vt)
    try:
        n = len(pts)
        rng = np.random.default_rng(7 + nrhs)
        x = rng.standard_normal((n, nrhs))
        r = rng.standard_normal((n, nrhs))
        dt = torch.float64 if vt == 1 else torch.float32
        if vt == 0:  # the FP32 engine sees the rounded inputs
            x, r = x.astype(np.float32).astype(np.float64), r.astype(np.float32).astype(np.float64)
        got = _device_grads(h, x, r, dt)
        want = _restated(h, x, r)
        assert np.isfinite(got).all()
        assert np.linalg.norm(got - want) / np.linalg.norm(want) <= tol
        # every leaf, not only the bulk
        T = h.leaf_table()
        offs, total = h.payload_layout()
        ends = np.append(offs[1:], total)
        worst = max(np.linalg.norm(got[a:b] - want[a:b]) / max(np.linalg.norm(want[a:b]), 1e-300)
                    for a, b in zip(offs, ends) if b > a)
        assert worst <= 50 * tol
    finally:
        h.close()


@pytest.mark.parametrize("vt,tol", [(1, 1e-11), (0, 1e-4)])
def test_gradients_bilinear_identity_and_accumulate(hb, vt, tol):
    """<grad, leaves> reproduces r^T H x (full + A parts, and full + B parts); accumulate
    adds onto the buffer."""
    import torch
    h, pts, wl = _setup(hb, vt, n_side=(40, 60))
    try:
        n = len(pts)
        rng = np.random.default_rng(3)
        x = rng.standard_normal((n, 4))
        r = rng.standard_normal((n, 4))
        dt = torch.float64 if vt == 1 else torch.float32
        if vt == 0:
            x, r = x.astype(np.float32).astype(np.float64), r.astype(np.float32).astype(np.float64)
        g = _device_grads(h, x, r, dt)
        y = h.gemv(x.astype(h.dtype)).astype(np.float64)
        rhx = float(np.sum(r * y))
        scale = float(np.sum(np.abs(r * y)))  # the sum cancels: compare to its magnitude
        full, a_part, b_part = _blocks(h, g)
        assert abs(full + a_part - rhx) <= tol * scale
        assert abs(full + b_part - rhx) <= tol * scale
        g2 = _device_grads(h, x, r, dt, accumulate_twice=True)
        assert np.linalg.norm(g2 - 2 * g) <= (1e-14 if vt == 1 else 1e-6) * np.linalg.norm(g)
    finally:
        h.close()
