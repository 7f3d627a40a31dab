"""Failure paths of the device engine, made to fire from the host without a GPU fault.

* The truncation's core SVD (one-sided Jacobi) stops after a capped number of sweeps and flags
  the leaf; the assembly then fails with return code 1 and a message.  HMAT_B200_JACOBI_SWEEPS=1
  lowers the cap so that the cores of rank 2 and more cannot converge; with the variable unset
  the same matrix assembles again in the same process.
* Every wait of the gemv kernels for a bulk copy is bounded; a kernel whose wait gives up sets
  the matrix's status flag, lets the copies it has in flight land, and stops.
  HMAT_B200_GEMV_WAIT_LIMIT=-1 (read when a matrix's engine is created) makes every such wait
  give up at once.  The device entry points report it through hmat_b200_gemv_status, the C
  table's gemv through its return code; a matrix created without the variable multiplies
  correctly afterwards.
"""
import importlib.util
import os

import numpy as np
import pytest
from conftest import ROOT, rel

pytestmark = pytest.mark.gpu


def _wl():
    spec = importlib.util.spec_from_file_location("wl_fail", os.path.join(ROOT, "hmat-oss_b200", "workloads.py"))
    wl = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(wl)
    return wl


def _cylinder(hb, vt, assemble=True):
    wl = _wl()
    pts = wl.cylinder(40, 50)
    hb.set_parameters(compressionMinLeafSize=0)
    h = hb.HMatrix(pts, hb.kernel(hb.LAPLACE_REG, delta=0.01), value_type=vt, leaf_size=32, eta=2.0, epsilon=1e-4,
                   assemble=assemble)
    return h, pts, wl


def test_jacobi_sweep_cap_fails_the_assembly_then_it_recovers(hb, oracle, monkeypatch):
    h, pts, wl = _cylinder(hb, hb.HMAT_DOUBLE_PRECISION, assemble=False)
    try:
        monkeypatch.setenv("HMAT_B200_JACOBI_SWEEPS", "1")
        with pytest.raises(hb.HMatError, match="did not converge within 1 sweeps"):
            h.assemble()
        monkeypatch.delenv("HMAT_B200_JACOBI_SWEEPS")
        h.assemble()  # the same matrix, same process
        x = wl.rhs(len(pts), 2, 3)
        o = oracle.OracleHMatrix(pts, leaf=32, eta=2.0)
        o.assemble(0, 1e-4, delta=0.01)
        assert np.array_equal(h.leaf_table(), o.leaves())
        assert rel(h.gemv(x), o.gemv(x)) < 1e-12
    finally:
        h.close()


@pytest.mark.parametrize("vt,trans", [(1, "N"), (1, "T"), (0, "N"), (0, "T")])
def test_gemv_wait_give_up_is_reported(hb, oracle, monkeypatch, vt, trans):
    import torch
    monkeypatch.setenv("HMAT_B200_GEMV_WAIT_LIMIT", "-1")
    h, pts, wl = _cylinder(hb, vt)
    monkeypatch.delenv("HMAT_B200_GEMV_WAIT_LIMIT")
    good = None
    try:
        n = len(pts)
        dt = torch.float64 if vt == 1 else torch.float32
        x = torch.from_numpy(np.ascontiguousarray(wl.rhs(n, 3, 5).T)).to("cuda", dt)
        y = torch.zeros_like(x)
        stream = torch.cuda.Stream()
        assert h.gemv_status(stream.cuda_stream) == 0
        h.gemv_device(x.data_ptr(), y.data_ptr(), 3, trans=trans, stream=stream.cuda_stream)
        assert h.gemv_status(stream.cuda_stream) == 1
        assert h.gemv_status(stream.cuda_stream) == 0  # the query clears the flag
        assert h.gemv_device_noalloc(x.data_ptr(), y.data_ptr(), 3, trans=trans, stream=stream.cuda_stream) == 0
        assert h.gemv_status(stream.cuda_stream) == 1
        with pytest.raises(hb.HMatError, match="gave up"):
            h.gemv(wl.rhs(n, 1, 6).astype(np.float64 if vt == 1 else np.float32), trans)
        assert h.gemv_status() == 0
        # a matrix created without the hook multiplies correctly on the same device
        good, _, _ = _cylinder(hb, vt)
        xh = wl.rhs(n, 2, 7)
        o = oracle.OracleHMatrix(pts, leaf=32, eta=2.0)
        o.assemble(0, 1e-4, delta=0.01)
        tol = 1e-12 if vt == 1 else 1e-5
        assert rel(good.gemv(xh.astype(np.float64 if vt == 1 else np.float32), trans), o.gemv(xh, trans)) < tol
        assert good.gemv_status() == 0
    finally:
        h.close()
        if good is not None:
            good.close()
