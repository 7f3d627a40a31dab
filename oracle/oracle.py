"""Python side of the oracle (TEST INFRASTRUCTURE ONLY).

Binds the C restatement (liboracle.so, see hmat_oracle.h) and runs the reference library's
own build (oracle/_ref/ref_driver, compiled from the reference sources by Makefile.ref)
when it is present.  Only the tests, the smoke check and the benchmark's CPU-baseline leg
use this module; the product never does.
"""
from __future__ import annotations

import ctypes as C
import json
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
REF_DRIVER = os.path.join(HERE, "_ref", "ref_driver")


class Kernel(C.Structure):
    _fields_ = [("kind", C.c_int), ("delta", C.c_double), ("ell", C.c_double), ("nugget", C.c_double),
                ("wavenumber", C.c_double), ("nstrata", C.c_int), ("sparam", C.c_double * 8),
                ("sweight", C.c_double * 8)]


def make_kernel(kind, delta=0.01, ell=0.3, nugget=0.0, wavenumber=0.0, strata_param=None, strata_weight=None):
    """Kernel descriptor; strata_param / strata_weight give a multi-strata kernel (stratum s =
    w_s times the kernel with parameter a_s: ell, delta or wavenumber)."""
    k = Kernel(kind, delta, ell, nugget, wavenumber)
    if strata_param is not None:
        if len(strata_param) != len(strata_weight) or not 1 <= len(strata_param) <= 8:
            raise ValueError("strata_param and strata_weight: same length, 1 to 8 strata")
        k.nstrata = len(strata_param)
        for s, (a, w) in enumerate(zip(strata_param, strata_weight)):
            k.sparam[s] = a
            k.sweight[s] = w
    return k


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            subprocess.run(["make", "-C", HERE, "liboracle.so"], check=True, capture_output=True)
        L = C.CDLL(LIB)
        P = C.c_void_p
        L.oracle_create.restype = P
        L.oracle_create.argtypes = [P, C.c_int, C.c_int, C.c_double]
        L.oracle_create2.restype = P
        L.oracle_create2.argtypes = [P, C.c_int, C.c_int, C.c_int, C.c_double]
        L.oracle_perm_cols.argtypes = [P, P]
        L.oracle_destroy.argtypes = [P]
        for f in ("oracle_perm", "oracle_leaves", "oracle_info", "oracle_nodes"):
            getattr(L, f).argtypes = [P, P]
        L.oracle_num_leaves.argtypes = [P]
        L.oracle_num_nodes.argtypes = [P]
        L.oracle_assemble.argtypes = [P, C.POINTER(Kernel), C.c_double, C.c_int]
        L.oracle_assemble2.argtypes = [P, C.POINTER(Kernel), C.c_double, C.c_int, C.c_int]
        L.oracle_retruncate.argtypes = [P, C.c_double]
        L.oracle_leaf_payload_size.restype = C.c_longlong
        L.oracle_leaf_payload_size.argtypes = [P, C.c_int]
        L.oracle_leaf_payload.argtypes = [P, C.c_int, P]
        L.oracle_gemv.argtypes = [P, C.c_char, C.c_int, P, P]
        L.oracle_kernel_eval.argtypes = [P, C.POINTER(Kernel), C.c_int, C.c_int, P]
        _lib = L
    return _lib


class OracleHMatrix:
    """FP64 oracle H-matrix (cluster tree, block tree, ACA+ + truncation, gemv)."""

    def __init__(self, points, leaf=64, eta=2.0, leaf_cols=None):
        self.points = np.ascontiguousarray(points, dtype=np.float64)
        self.n = len(self.points)
        self.h = lib().oracle_create2(self.points.ctypes.data, self.n, leaf, leaf_cols or leaf, eta)
        self.is_complex = False

    def perm(self):
        p = np.zeros(self.n, np.int32)
        lib().oracle_perm(self.h, p.ctypes.data)
        return p

    def perm_cols(self):
        p = np.zeros(self.n, np.int32)
        lib().oracle_perm_cols(self.h, p.ctypes.data)
        return p

    def leaves(self):
        nl = lib().oracle_num_leaves(self.h)
        out = np.zeros((nl, 6), np.int32)
        lib().oracle_leaves(self.h, out.ctypes.data)
        return out

    def info(self):
        out = np.zeros(12, np.int64)
        lib().oracle_info(self.h, out.ctypes.data)
        keys = ["full_count", "rk_count", "full_size", "rk_size", "compressed_size", "uncompressed_size",
                "nr_block_clusters", "largest_rk_dim_rows", "largest_rk_dim_cols", "largest_rk_mem_rows",
                "largest_rk_mem_cols", "largest_rk_mem_rank"]
        return dict(zip(keys, [int(v) for v in out]))

    def assemble(self, kind, eps, delta=0.01, ell=0.3, nugget=0.0, wavenumber=0.0, min_leaf=0, strata_param=None,
                 strata_weight=None):
        self.kernel = make_kernel(kind, delta, ell, nugget, wavenumber, strata_param, strata_weight)
        self.is_complex = kind == 2
        rc = lib().oracle_assemble2(self.h, C.byref(self.kernel), eps, int(self.is_complex), min_leaf)
        assert rc == 0

    def retruncate(self, eps):
        """Re-truncates every Rk leaf at eps (HMatrix::truncate, h_matrix.cpp:2107-2123)."""
        assert lib().oracle_retruncate(self.h, eps) == 0

    def payload(self, i):
        s = lib().oracle_leaf_payload_size(self.h, i)
        w = 2 if self.is_complex else 1
        out = np.zeros(max(1, s * w), np.float64)
        lib().oracle_leaf_payload(self.h, i, out.ctypes.data)
        out = out[:s * w]
        return out.view(np.complex128) if self.is_complex else out

    def block(self, i, table=None):
        t = self.leaves() if table is None else table
        r0, m, c0, n, typ, k = t[i]
        p = self.payload(i)
        if typ == 0:
            return p.reshape(n, m).T
        if k <= 0:
            return np.zeros((m, n), p.dtype)
        return p[:k * m].reshape(k, m).T @ p[k * m:].reshape(k, n).T.T

    def gemv(self, x, trans="N"):
        dt = np.complex128 if self.is_complex else np.float64
        x = np.asfortranarray(x, dtype=dt)
        nrhs = 1 if x.ndim == 1 else x.shape[1]
        y = np.zeros_like(x)
        lib().oracle_gemv(self.h, trans.encode(), nrhs, x.ctypes.data, y.ctypes.data)
        return y

    def close(self):
        if self.h:
            lib().oracle_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def kernel_matrix(points_rows, points_cols, kind, delta=0.01, ell=0.3, nugget=0.0, wavenumber=0.0, ids=None):
    """Dense kernel block in FP64 (numpy), same formulas as the oracle's callbacks."""
    d = points_rows[:, None, :] - points_cols[None, :, :]
    r = np.sqrt((d * d).sum(-1))
    if kind == 0:
        return 1.0 / (4.0 * np.pi * (r + delta))
    if kind == 1:
        K = np.exp(-r / ell)
        if ids is not None:
            K[ids[0][:, None] == ids[1][None, :]] += nugget
        return K
    return np.exp(1j * wavenumber * r) / (4.0 * np.pi * (r + delta))


def dense_product(points, x, kind, chunk=2048, **kw):
    """y = K x with the exact dense kernel matrix, FP64 (the ground truth of the path)."""
    n = len(points)
    x2 = x.reshape(n, -1)
    y = np.zeros(x2.shape, dtype=np.complex128 if (kind == 2 or np.iscomplexobj(x)) else np.float64)
    idx = np.arange(n)
    for s in range(0, n, chunk):
        K = kernel_matrix(points[s:s + chunk], points, kind, ids=(idx[s:s + chunk], idx), **kw)
        y[s:s + chunk] = K @ x2
    return y.reshape(x.shape)


def have_reference():
    return os.path.exists(REF_DRIVER)


def run_reference(points, kind, eps, leaf=64, eta=2.0, delta=0.01, ell=0.3, nugget=0.0, wavenumber=0.0, x=None,
                  nrhs=1, trans="N", scalar="D", dump_factors=False, gemv_reps=1, min_leaf=0, leaf_cols=0,
                  gemv_warmup=0, retrunc=0.0, strata_param=None, strata_weight=None, read_data=None,
                  write_data=None):
    """Runs the reference library (oracle/_ref/ref_driver) and returns its outputs.  With
    strata_param / strata_weight, the matrix is assembled through advanced_compute with one
    stratum per entry (w_s times the kernel with parameter a_s: ell, delta or wavenumber).
    read_data (bytes): the leaves are read from that data stream (hmat_interface_t.read_data)
    into the matrix built on the points instead of being assembled; write_data=True returns the
    assembled matrix's data stream (hmat_interface_t.write_data) as out["data"]."""
    if not have_reference():
        raise FileNotFoundError(REF_DRIVER)
    kname = {0: "laplace", 1: "expcov", 2: "helmholtz"}[kind]
    with tempfile.TemporaryDirectory() as d:
        pts = os.path.join(d, "pts.bin")
        np.ascontiguousarray(points, dtype=np.float64).tofile(pts)
        lines = [f"points={pts}", f"n={len(points)}", f"kernel={kname}", f"delta={delta!r}", f"ell={ell!r}",
                 f"nugget={nugget!r}", f"wavenumber={wavenumber!r}", f"leaf={leaf}", f"eta={eta!r}", f"eps={eps!r}",
                 f"nrhs={nrhs}", f"trans={trans}", f"scalar={scalar}", f"dump_factors={int(dump_factors)}",
                 f"gemv_reps={gemv_reps}", f"gemv_warmup={gemv_warmup}", f"min_leaf={min_leaf}",
                 f"leaf_cols={leaf_cols}", f"retrunc={retrunc!r}",
                 f"out={os.path.join(d, 'out')}"]
        if read_data is not None:
            rp = os.path.join(d, "data_in.bin")
            with open(rp, "wb") as f:
                f.write(read_data)
            lines.append(f"read_data={rp}")
        if write_data:
            lines.append(f"write_data={os.path.join(d, 'data_out.bin')}")
        if strata_param is not None:
            lines.append("strata_param=" + ",".join(repr(float(a)) for a in strata_param))
            lines.append("strata_weight=" + ",".join(repr(float(w)) for w in strata_weight))
        dt = {"D": np.float64, "S": np.float32, "Z": np.complex128, "C": np.complex64}[scalar]
        if x is not None:
            xp = os.path.join(d, "x.bin")
            np.asfortranarray(x, dtype=dt).ravel(order="F").tofile(xp)
            lines.append(f"x={xp}")
        pf = os.path.join(d, "p.txt")
        with open(pf, "w") as f:
            f.write("\n".join(lines) + "\n")
        env = dict(os.environ, OPENBLAS_NUM_THREADS="1")
        r = subprocess.run([REF_DRIVER, pf], capture_output=True, text=True, env=env)
        if r.returncode != 0:
            raise RuntimeError(f"ref_driver failed ({r.returncode}): {r.stderr[-2000:]}")
        out = {"json": json.load(open(os.path.join(d, "out.json")))}
        out["perm"] = np.fromfile(os.path.join(d, "out.perm"), np.int32)
        out["perm_cols"] = np.fromfile(os.path.join(d, "out.permc"), np.int32)
        out["leaves"] = np.fromfile(os.path.join(d, "out.leaves"), np.int32).reshape(-1, 6)
        if x is not None:
            out["y"] = np.fromfile(os.path.join(d, "out.y"), dt).reshape(x.shape, order="F")
        if dump_factors:
            out["payload"] = np.fromfile(os.path.join(d, "out.payload"), dt)
        if write_data:
            with open(os.path.join(d, "data_out.bin"), "rb") as f:
                out["data"] = f.read()
        return out
