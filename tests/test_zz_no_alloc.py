"""The allocation-free device gemv (hmat_b200_gemv_device_noalloc), for callers that
cannot allocate GPU memory at the time they multiply (callers inside a memory pool or
caching allocator they do not own, inside callbacks where cudaMalloc / cudaFree would
synchronise or deadlock, or in loops that forbid allocation after start-up).

Its result must equal the regular device gemv's (same kernels, scratch taken from the
library's fixed device array instead of allocated buffers) on two calls in a row, since
the shared array keeps the previous call's contents.  Matrices that need more scratch
than the array holds are refused with an error, before anything is launched.  This file
is collected last so a failure here leaves every other test already run."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _matrix(hb, n_theta, n_z, vt, leaf=32):
    import importlib.util
    import os
    from conftest import ROOT
    spec = importlib.util.spec_from_file_location("wl_noalloc", os.path.join(ROOT, "hmat-oss_b200", "workloads.py"))
    wl = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(wl)
    pts = wl.cylinder(n_theta, n_z)
    hb.set_parameters(compressionMinLeafSize=0)
    h = hb.HMatrix(pts, hb.kernel(hb.LAPLACE_REG, delta=0.01), value_type=vt, leaf_size=leaf, eta=2.0, epsilon=1e-4)
    return h, pts, wl


@pytest.mark.parametrize("vt,tol", [(1, 1e-12), (0, 1e-6)])
def test_noalloc_gemv_matches_device_gemv_twice(hb, vt, tol):
    import torch
    h, pts, wl = _matrix(hb, 40, 50, vt)
    try:
        n = len(pts)
        dt = torch.float64 if vt == 1 else torch.float32
        stream = torch.cuda.Stream()
        for call, nrhs in enumerate((3, 3)):
            x = torch.from_numpy(np.ascontiguousarray(wl.rhs(n, nrhs, 40 + call).T)).to("cuda", dt)
            y_ref = torch.zeros_like(x)
            y_na = torch.full_like(x, float("nan"))
            torch.cuda.synchronize()
            h.gemv_device(x.data_ptr(), y_ref.data_ptr(), nrhs, stream=stream.cuda_stream)
            rc = h.gemv_device_noalloc(x.data_ptr(), y_na.data_ptr(), nrhs, stream=stream.cuda_stream)
            assert rc == 0, hb.load_library().hmat_b200_last_error()
            torch.cuda.synchronize()
            a = y_ref.cpu().numpy()
            b = y_na.cpu().numpy()
            assert np.isfinite(b).all()
            assert np.linalg.norm(a - b) / np.linalg.norm(a) <= tol
            # transposed product through the same scratch
            h.gemv_device(x.data_ptr(), y_ref.data_ptr(), nrhs, trans="T", stream=stream.cuda_stream)
            assert h.gemv_device_noalloc(x.data_ptr(), y_na.data_ptr(), nrhs, trans="T",
                                         stream=stream.cuda_stream) == 0
            torch.cuda.synchronize()
            a = y_ref.cpu().numpy()
            b = y_na.cpu().numpy()
            assert np.linalg.norm(a - b) / np.linalg.norm(a) <= tol
        # alpha and beta on the output, against the regular device gemv with the same y
        x = torch.from_numpy(np.ascontiguousarray(wl.rhs(n, 2, 44).T)).to("cuda", dt)
        y0 = torch.from_numpy(np.ascontiguousarray(wl.rhs(n, 2, 45).T)).to("cuda", dt)
        y_ref, y_na = y0.clone(), y0.clone()
        h.gemv_device(x.data_ptr(), y_ref.data_ptr(), 2, alpha=2.0, beta=0.5, stream=stream.cuda_stream)
        assert h.gemv_device_noalloc(x.data_ptr(), y_na.data_ptr(), 2, alpha=2.0, beta=0.5,
                                     stream=stream.cuda_stream) == 0
        assert h.gemv_status(stream.cuda_stream) == 0
        a = y_ref.cpu().numpy()
        b = y_na.cpu().numpy()
        assert np.linalg.norm(a - b) / np.linalg.norm(a) <= tol
    finally:
        h.close()


def test_noalloc_gemv_rejects_matrices_above_its_scratch(hb):
    import torch
    # 200 x 250 cylinder, FP64: x in cluster order alone is 50,000 x 16 x 8 B = 6.4 MB and the
    # z buffer is larger still, beyond the 16 MiB the entry point holds
    h, pts, wl = _matrix(hb, 200, 250, 1, leaf=64)
    try:
        x = torch.zeros((1, len(pts)), dtype=torch.float64, device="cuda")
        y = torch.zeros_like(x)
        rc = h.gemv_device_noalloc(x.data_ptr(), y.data_ptr(), 1)
        err = hb.load_library().hmat_b200_last_error().decode()
        if rc == 0:
            pytest.skip("this matrix fits the no-alloc scratch")
        assert "scratch" in err
    finally:
        h.close()
