"""The adjoint of the H-matrix product as a torch.autograd.Function (test harness), checked by
central finite differences and against the reference's own transposed product.

    forward:  y = H x                                   hmat_b200_gemv_device ('N')
    backward: dx = H^T r and dF, dA, dB (canonical      hmat_b200_gemv_adjoint (one pass; the same as
              payload layout)                           gemv_device 'T' + hmat_b200_leaf_gradients)
for the loss L = 1/2 ||H x - b||^2, r = H x - b.  The leaf payload enters the function as a
tensor `theta` holding the matrix's stored leaves (canonical layout: full m x n, Rk A m x k
then B n x k, column-major, leaf order), so that autograd returns dL/dtheta beside dL/dx.

Finite differences perturb one entry of x, or one stored entry of a full leaf, of A or of B,
by +-1e-6: a perturbed matrix is the original written with write_struct / write_data, the entry
changed in the data stream (the reference's data layout), and read back with read_struct /
read_data.

The reference's transposed gemv (RkMatrix::gemv 'T', rk_matrix.cpp:156-206, reached through
HMatrix::gemv and getChildForGEMM, h_matrix.cpp:772-857) is the golden y_T = H^T x_g of the
20,000-point cube (exponential covariance, l = 0.3, epsilon 1e-6, leaf 64): with b = H x - x_g
the residual is r = x_g, so dx must equal y_T.
"""
import importlib.util
import os

import numpy as np
import pytest
from cases import CASES, inputs
from conftest import ROOT, golden, rel

pytestmark = pytest.mark.gpu

FD_STEP = 1e-6


class HGemv:
    """torch.autograd.Function over the engine's device product and leaf gradients."""

    @staticmethod
    def make(torch):
        class _F(torch.autograd.Function):
            @staticmethod
            def forward(ctx, x, theta, h):
                # x: (nrhs, N) contiguous = column-major N x nrhs, client numbering
                nrhs = x.shape[0]
                y = torch.empty_like(x)
                stream = torch.cuda.current_stream().cuda_stream
                assert stream != 0, "run under a torch stream of its own (handle 0 is the matrix's own stream)"
                h.gemv_device(x.data_ptr(), y.data_ptr(), nrhs, trans="N", stream=stream)
                ctx.h = h
                ctx.save_for_backward(x)
                ctx.theta_shape = theta.shape
                return y

            @staticmethod
            def backward(ctx, gy):
                (x,) = ctx.saved_tensors
                h = ctx.h
                gy = gy.contiguous()
                nrhs = x.shape[0]
                stream = torch.cuda.current_stream().cuda_stream
                dx = torch.empty_like(x)
                dtheta = torch.empty(ctx.theta_shape, dtype=x.dtype, device=x.device)
                # dx = H^T r and the leaf gradients in one pass (hmat_b200_gemv_adjoint)
                h.gemv_adjoint(x.data_ptr(), gy.data_ptr(), nrhs, dx.data_ptr(), dtheta.data_ptr(), accumulate=False,
                               stream=stream)
                assert not h.gemv_status(stream)
                return dx, dtheta, None

        return _F


def _theta(h):
    """The stored leaves in the canonical payload layout (host, FP64 for the FP64 engine)."""
    offs, total = h.payload_layout()
    T = h.leaf_table()
    theta = np.zeros(total, dtype=h.dtype)
    for i, (r0, m, c0, n, t, k) in enumerate(T):
        size = m * n if t == 0 else max(k, 0) * (m + n)
        if size:
            theta[offs[i]:offs[i] + size] = h.leaf_payload(i)
    return theta


def _loss_and_grads(torch, h, x, b):
    # A stream of its own: torch's default stream has the handle 0, which the engine's device
    # entry points read as "the matrix's own stream" (unordered with torch's work).
    F = HGemv.make(torch)
    with torch.cuda.stream(torch.cuda.Stream()):
        theta = torch.from_numpy(_theta(h)).to("cuda").requires_grad_(True)
        xt = torch.from_numpy(np.ascontiguousarray(x.T)).to("cuda", theta.dtype).requires_grad_(True)
        bt = torch.from_numpy(np.ascontiguousarray(b.T)).to("cuda", torch.float64)
        y = F.apply(xt, theta, h)
        L = 0.5 * ((y.double() - bt) ** 2).sum()  # the residual in FP64, handed back in the engine's type
        L.backward()
        torch.cuda.current_stream().synchronize()
        return (float(L.detach()), xt.grad.T.cpu().numpy().astype(np.float64),
                theta.grad.cpu().numpy().astype(np.float64))


def _loss(hb, h, x, b):
    y = h.gemv(x.astype(h.dtype)).astype(np.float64)
    return 0.5 * float(np.sum((y - b) ** 2))


def _stream_offset(h, pos):
    """Byte offset in the data stream (the reference's layout: per leaf a header int, its
    entries, and two ints after the factors of an Rk leaf of rank > 0) of canonical payload
    entry `pos`."""
    offs, _ = h.payload_layout()
    T = h.leaf_table()
    s = np.dtype(h.dtype).itemsize
    at = 0
    for i, (r0, m, c0, n, t, k) in enumerate(T):
        size = m * n if t == 0 else max(k, 0) * (m + n)
        if offs[i] <= pos < offs[i] + size:
            return at + 4 + (pos - offs[i]) * s
        at += 4 + size * s + (8 if t == 1 and k > 0 else 0)
    raise IndexError(pos)


def _perturbed(hb, h, pos, delta):
    """The matrix with canonical payload entry `pos` changed by delta (through the streams)."""
    st, data = h.dump()
    s = np.dtype(h.dtype).itemsize
    at = _stream_offset(h, pos)
    buf = bytearray(data)
    v = np.frombuffer(bytes(buf[at:at + s]), dtype=h.dtype)[0]
    buf[at:at + s] = np.array([v + delta], dtype=h.dtype).tobytes()
    return hb.HMatrix.load(h.value_type, st, bytes(buf))


def _wl():
    spec = importlib.util.spec_from_file_location("wl_adj", os.path.join(ROOT, "hmat-oss_b200", "workloads.py"))
    wl = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(wl)
    return wl


def test_autograd_central_finite_differences(hb):
    """dL/dx and dL/d(leaves) of the autograd function against central differences (step 1e-6,
    FP64 engine) on sampled entries of x, of full leaves, and of the A and B factors."""
    import torch
    wl = _wl()
    pts = wl.cube(3000, 8)
    hb.set_parameters(compressionMinLeafSize=0)
    h = hb.HMatrix(pts, hb.kernel(hb.EXP_COV, ell=0.3, nugget=1e-6), value_type=hb.HMAT_DOUBLE_PRECISION,
                   leaf_size=32, eta=2.0, epsilon=1e-6)
    try:
        n = len(pts)
        rng = np.random.default_rng(2)
        x = rng.standard_normal((n, 2))
        # a small residual (r ~ 0.01) keeps the loss near 0.3, so that a 1e-6 step moves it far
        # above its rounding
        b = h.gemv(x) + 0.01 * rng.standard_normal((n, 2))
        L, dx, dtheta = _loss_and_grads(torch, h, x, b)
        assert abs(L - _loss(hb, h, x, b)) <= 1e-12 * abs(L)
        # x entries
        for i, q in [(0, 0), (17, 1), (n - 1, 0), (1234, 1)]:
            xp, xm = x.copy(), x.copy()
            xp[i, q] += FD_STEP
            xm[i, q] -= FD_STEP
            fd = (_loss(hb, h, xp, b) - _loss(hb, h, xm, b)) / (2 * FD_STEP)
            assert abs(fd - dx[i, q]) <= 1e-5 * abs(dx[i, q]) + 1e-7, (i, q, fd, dx[i, q])
        # leaf entries: a full leaf, and A and B of the two largest Rk leaves
        T = h.leaf_table()
        offs, _ = h.payload_layout()
        full = int(np.nonzero(T[:, 4] == 0)[0][3])
        rk = np.nonzero((T[:, 4] == 1) & (T[:, 5] > 0))[0]
        big = rk[np.argsort(-(T[rk, 1] + T[rk, 3]))[:2]]
        picks = [offs[full] + 5]
        for i in big:
            m, k = int(T[i, 1]), int(T[i, 5])
            picks += [offs[i] + (m * k) // 2, offs[i] + m * k + 3]  # one entry of A, one of B
        for pos in picks:
            hp = _perturbed(hb, h, int(pos), FD_STEP)
            hm = _perturbed(hb, h, int(pos), -FD_STEP)
            try:
                fd = (_loss(hb, hp, x, b) - _loss(hb, hm, x, b)) / (2 * FD_STEP)
            finally:
                hp.close()
                hm.close()
            g = dtheta[pos]
            assert abs(fd - g) <= 1e-5 * abs(g) + 1e-7, (pos, fd, g)
    finally:
        h.close()


@pytest.mark.parametrize("vt,tol", [(1, 1e-12), (0, 1e-5)])
def test_autograd_dx_matches_reference_transposed_gemv(hb, vt, tol):
    """With b = H x - x_g the backward pass's dx is H^T x_g: the reference's transposed product
    (golden y_T of the 20,000-point cube).  FP64 within 1e-12; the mixed engine (FP32 leaves
    and products, the residual rounded to FP32) within ten times the compression epsilon."""
    import torch
    name = "cfg4_cube"
    g = golden(name)
    _, kern, tree, nrhs, seed, scalar, dump = CASES[name]
    pts, xg = inputs(name)
    hb.set_parameters(compressionMinLeafSize=0)
    h = hb.HMatrix(pts, hb.kernel(hb.EXP_COV, ell=kern["ell"], nugget=kern["nugget"]), value_type=vt,
                   leaf_size=tree["leaf"], eta=tree["eta"], epsilon=tree["eps"])
    try:
        if vt == 1:
            assert np.array_equal(h.leaf_table(), g["leaves"])
        x = np.random.default_rng(seed).standard_normal(xg.shape)
        y = h.gemv(x.astype(h.dtype)).astype(np.float64)
        b = y - xg  # r = H x - b = x_g
        _, dx, _ = _loss_and_grads(torch, h, x, b)
        assert rel(dx, g["y_T"]) < tol
    finally:
        h.close()


@pytest.mark.parametrize("vt", [1, 0])
def test_fused_adjoint_equals_separate_calls(hb, vt):
    """hmat_b200_gemv_adjoint gives bit for bit what the transposed device product and
    hmat_b200_leaf_gradients give separately (same kernels, the transposed product's A^T r
    reused as the gradients' w), also with accumulate."""
    import torch
    wl = _wl()
    pts = wl.cube(2500, 4)
    hb.set_parameters(compressionMinLeafSize=0)
    h = hb.HMatrix(pts, hb.kernel(hb.EXP_COV, ell=0.3, nugget=1e-6), value_type=vt, leaf_size=32, eta=2.0,
                   epsilon=1e-6)
    try:
        n = len(pts)
        dt = torch.float64 if vt == 1 else torch.float32
        rng = np.random.default_rng(12)
        with torch.cuda.stream(torch.cuda.Stream()):
            st = torch.cuda.current_stream().cuda_stream
            x = torch.from_numpy(rng.standard_normal((3, n))).to("cuda", dt)
            r = torch.from_numpy(rng.standard_normal((3, n))).to("cuda", dt)
            _, total = h.payload_layout()
            dx1, dx2 = torch.empty_like(x), torch.empty_like(x)
            g1 = torch.full((total,), 0.5, device="cuda", dtype=dt)
            g2 = g1.clone()
            h.gemv_device(r.data_ptr(), dx1.data_ptr(), 3, trans="T", stream=st)
            h.leaf_gradients(x.data_ptr(), r.data_ptr(), 3, g1.data_ptr(), accumulate=True, stream=st)
            h.gemv_adjoint(x.data_ptr(), r.data_ptr(), 3, dx2.data_ptr(), g2.data_ptr(), accumulate=True, stream=st)
            torch.cuda.current_stream().synchronize()
            assert not h.gemv_status(st)
        assert torch.equal(dx1, dx2)
        assert torch.equal(g1, g2)
    finally:
        h.close()
