"""Python mirror of the hmat-oss C interface, backed by the B200 engine.

The product is ``libhmat_b200.so`` (C ABI declared in ``include/hmat_b200.h``); this
module binds it with ctypes and mirrors the reference's C entry points with the same
names and argument meaning (``hmat_init_default_interface``, ``create_empty_hmatrix_admissibility``,
``set_low_rank_epsilon``, ``assemble_generic``, ``gemv``, ``get_info``, ``destroy``, ...), so
that host programs and tests read like the reference's own examples
(examples/c-simple-cylinder.c, examples/c-simple-kriging.c).  There is no CPU fallback: if
the shared library is missing, importing the bindings raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libhmat_b200.so")

HMAT_SIMPLE_PRECISION = 0
HMAT_DOUBLE_PRECISION = 1
HMAT_SIMPLE_COMPLEX = 2
HMAT_DOUBLE_COMPLEX = 3

DTYPES = {
    HMAT_SIMPLE_PRECISION: np.float32,
    HMAT_DOUBLE_PRECISION: np.float64,
    HMAT_SIMPLE_COMPLEX: np.complex64,
    HMAT_DOUBLE_COMPLEX: np.complex128,
}

LAPLACE_REG = 0
EXP_COV = 1
HELMHOLTZ_REG = 2

hmat_factorization_none = -1


class KernelDesc(C.Structure):
    _fields_ = [("kind", C.c_int), ("delta", C.c_double), ("ell", C.c_double), ("nugget", C.c_double),
                ("wavenumber", C.c_double)]


class AssembleContext(C.Structure):
    """hmat_assemble_context_t (reference: include/hmat/hmat.h:516-622)."""
    _fields_ = [("assembly", C.c_void_p), ("simple_compute", C.c_void_p), ("block_compute", C.c_void_p),
                ("advanced_compute", C.c_void_p), ("user_context", C.c_void_p), ("prepare", C.c_void_p),
                ("compression", C.c_void_p), ("lower_symmetric", C.c_int), ("factorization", C.c_int),
                ("progress", C.c_void_p)]


class GetValuesContext(C.Structure):
    """hmat_get_values_context_t (hmat.h:637-656)."""
    _fields_ = [("matrix", C.c_void_p), ("values", C.c_void_p), ("row_offset", C.c_int), ("col_offset", C.c_int),
                ("row_size", C.c_int), ("col_size", C.c_int), ("row_indices", C.POINTER(C.c_int)),
                ("col_indices", C.POINTER(C.c_int)), ("renumber_rows", C.c_int, 1)]


class ClusterInfo(C.Structure):
    _fields_ = [("spatial_dimension", C.c_int), ("dimension", C.c_int), ("nr_tree_nodes", C.c_size_t)]


class Info(C.Structure):
    """hmat_info_t (reference: include/hmat/hmat.h:404-439)."""
    _fields_ = [("full_zeros", C.c_int), ("full_size", C.c_size_t), ("rk_size", C.c_size_t),
                ("full_count", C.c_size_t), ("rk_count", C.c_size_t), ("compressed_size", C.c_size_t),
                ("uncompressed_size", C.c_size_t), ("nr_block_clusters", C.c_int),
                ("largest_rk_dim_rows", C.c_int), ("largest_rk_dim_cols", C.c_int),
                ("largest_rk_mem_rows", C.c_int), ("largest_rk_mem_cols", C.c_int),
                ("largest_rk_mem_rank", C.c_int)]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


class Settings(C.Structure):
    """hmat_settings_t (reference: include/hmat/hmat.h:1107-1131)."""
    _fields_ = [("compressionMinLeafSize", C.c_int), ("coarseningEpsilon", C.c_double), ("maxLeafSize", C.c_int),
                ("coarsening", C.c_int), ("validateNullRowCol", C.c_int), ("validateCompression", C.c_int),
                ("validateRecompression", C.c_int), ("dumpTrace", C.c_int), ("validationReRun", C.c_int),
                ("validationDump", C.c_int), ("validationErrorThreshold", C.c_double)]


# Slot order of hmat_interface_t (reference: include/hmat/hmat.h:717-1103).
_SLOTS = ["create_empty_hmatrix_admissibility", "own_cluster_trees", "set_low_rank_epsilon", "assemble_generic",
          "copy", "copy_struct", "norm", "logdet", "inverse", "factorize_generic", "destroy", "get_child",
          "destroy_child", "solve_generic", "solve_mat", "solve_systems", "solve_dense", "transpose", "scale",
          "truncate", "vector_reorder", "vector_restore", "gemm", "axpy", "trsm", "gemv", "gemm_scalar",
          "full_gemm", "gemm_dense", "add_identity", "init", "finalize", "get_info", "get_profile", "get_ratio",
          "FPcompress", "FPdecompress", "GetFPCompressionSettings", "SetFPCompressionSettings",
          "SetFPCompressionSettingsParams", "dump_info", "get_cluster_trees", "set_cluster_trees",
          "extract_diagonal", "solve_lower_triangular", "solve_lower_triangular_dense", "get_block",
          "get_values", "walk", "apply_on_leaf", "value_type", "internal", "read_struct", "write_struct",
          "read_data", "write_data", "set_progressbar", "extract_diagonal_block"]


class InterfaceTable(C.Structure):
    _fields_ = [(s, C.c_int if s == "value_type" else C.c_void_p) for s in _SLOTS]


_P = C.c_void_p
_IOSTREAM = C.CFUNCTYPE(None, C.c_void_p, C.c_size_t, C.c_void_p)
_PROTOS = {
    "create_empty_hmatrix_admissibility": C.CFUNCTYPE(_P, _P, _P, C.c_int, _P),
    "own_cluster_trees": C.CFUNCTYPE(None, _P, C.c_int, C.c_int),
    "set_low_rank_epsilon": C.CFUNCTYPE(None, _P, C.c_double),
    "assemble_generic": C.CFUNCTYPE(C.c_int, _P, C.POINTER(AssembleContext)),
    "destroy": C.CFUNCTYPE(C.c_int, _P),
    "gemv": C.CFUNCTYPE(C.c_int, C.c_char, _P, _P, _P, _P, _P, C.c_int),
    "get_info": C.CFUNCTYPE(C.c_int, _P, C.POINTER(Info)),
    "vector_reorder": C.CFUNCTYPE(C.c_int, _P, _P, C.c_int, _P, C.c_int),
    "vector_restore": C.CFUNCTYPE(C.c_int, _P, _P, C.c_int, _P, C.c_int),
    "truncate": C.CFUNCTYPE(C.c_int, _P),
    "gemm_dense": C.CFUNCTYPE(C.c_int, C.c_char, C.c_char, C.c_char, _P, _P, _P, _P, _P, C.c_int),
    "gemm_scalar": C.CFUNCTYPE(C.c_int, C.c_char, _P, _P, _P, _P, _P, C.c_int),
    "get_block": C.CFUNCTYPE(C.c_int, C.POINTER(GetValuesContext)),
    "write_struct": C.CFUNCTYPE(None, _P, _IOSTREAM, _P),
    "write_data": C.CFUNCTYPE(None, _P, _IOSTREAM, _P),
    "read_struct": C.CFUNCTYPE(_P, _IOSTREAM, _P),
    "read_data": C.CFUNCTYPE(None, _P, _IOSTREAM, _P),
    "get_cluster_trees": C.CFUNCTYPE(C.c_int, _P, C.POINTER(_P), C.POINTER(_P)),
    "get_values": C.CFUNCTYPE(C.c_int, C.POINTER(GetValuesContext)),
    "solve_systems": C.CFUNCTYPE(C.c_int, _P, _P, C.c_int),
    "init": C.CFUNCTYPE(C.c_int),
    "finalize": C.CFUNCTYPE(C.c_int),
}

_lib = None

# Entry points declared in include/hmat_b200.h; the tests check that every one is exported.
EXPORTED = [
    "hmat_create_clustering_median", "hmat_create_clustering_max_dof", "hmat_delete_clustering",
    "hmat_set_clustering_divider", "hmat_create_cluster_tree", "hmat_delete_cluster_tree", "hmat_tree_nodes_count",
    "hmat_cluster_get_info", "hmat_cluster_get_indices", "hmat_init_admissibility_param",
    "hmat_create_admissibility", "hmat_update_admissibility", "hmat_create_admissibility_standard",
    "hmat_delete_admissibility", "hmat_create_compression_aca_plus", "hmat_create_compression_aca_partial",
    "hmat_create_compression_svd", "hmat_create_compression_aca_full", "hmat_create_compression_aca_random",
    "hmat_create_compression_rrqr", "hmat_delete_compression", "hmat_default_progress",
    "hmat_assemble_context_init", "hmat_factorization_context_init", "hmat_solve_context_init",
    "hmat_init_default_interface", "hmat_get_parameters", "hmat_set_parameters", "hmat_get_version",
    "hmat_b200_create_assembly", "hmat_b200_create_assembly_strata", "hmat_b200_delete_assembly", "hmat_b200_gemv_device", "hmat_b200_gemv_device_noalloc", "hmat_b200_gemv_status",
    "hmat_b200_batch_create", "hmat_b200_batch_offsets", "hmat_b200_batch_assemble",
    "hmat_b200_leaf_count",
    "hmat_b200_leaf_table", "hmat_b200_leaf_payload", "hmat_b200_payload_layout", "hmat_b200_leaf_gradients",
    "hmat_b200_gemv_adjoint", "hmat_b200_phase_times", "hmat_b200_gemv_profile", "hmat_b200_gemv_launches", "hmat_b200_aca_shapes",
    "hmat_b200_gemv_tuning", "hmat_b200_last_error",
    "hmat_b200_clear_last_error",
]


def load_library(path: str = LIB_PATH) -> C.CDLL:
    """Loads libhmat_b200.so (built in-tree by `make -C hmat-oss_b200`).  Raises if absent."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(f"{path} is missing: build it with `make -C hmat-oss_b200` (no CPU fallback exists)")
    lib = C.CDLL(path)
    sig = {
        "hmat_create_clustering_median": (_P, []),
        "hmat_create_clustering_max_dof": (_P, [_P, C.c_int]),
        "hmat_delete_clustering": (None, [_P]),
        "hmat_create_cluster_tree": (_P, [_P, C.c_int, C.c_int, _P]),
        "hmat_delete_cluster_tree": (None, [_P]),
        "hmat_tree_nodes_count": (C.c_int, [_P]),
        "hmat_cluster_get_indices": (C.POINTER(C.c_int), [_P]),
        "hmat_create_admissibility_standard": (_P, [C.c_double]),
        "hmat_delete_admissibility": (None, [_P]),
        "hmat_create_compression_aca_plus": (_P, [C.c_double]),
        "hmat_create_compression_aca_partial": (_P, [C.c_double]),
        "hmat_create_compression_svd": (_P, [C.c_double]),
        "hmat_delete_compression": (None, [_P]),
        "hmat_assemble_context_init": (None, [C.POINTER(AssembleContext)]),
        "hmat_init_default_interface": (None, [C.POINTER(InterfaceTable), C.c_int]),
        "hmat_get_parameters": (None, [C.POINTER(Settings)]),
        "hmat_set_parameters": (C.c_int, [C.POINTER(Settings)]),
        "hmat_get_version": (C.c_char_p, []),
        "hmat_b200_create_assembly": (_P, [C.POINTER(KernelDesc), _P, C.c_int]),
        "hmat_b200_create_assembly_strata": (_P, [C.POINTER(KernelDesc), _P, C.c_int, C.c_int, _P, _P]),
        "hmat_b200_delete_assembly": (None, [_P]),
        "hmat_b200_gemv_device": (C.c_int, [_P, C.c_char, _P, _P, _P, _P, C.c_int, _P]),
        "hmat_b200_gemv_device_noalloc": (C.c_int, [_P, C.c_char, _P, _P, _P, _P, C.c_int, _P]),
        "hmat_b200_gemv_status": (C.c_int, [_P, _P, C.POINTER(C.c_int)]),
        "hmat_b200_batch_create": (_P, [_P, C.c_int]),
        "hmat_b200_batch_offsets": (C.c_int, [_P, _P, _P]),
        "hmat_b200_batch_assemble": (C.c_int, [_P, _P, _P]),
        "hmat_b200_leaf_count": (C.c_int, [_P]),
        "hmat_b200_leaf_table": (C.c_int, [_P, _P]),
        "hmat_b200_leaf_payload": (C.c_longlong, [_P, C.c_int, _P]),
        "hmat_b200_payload_layout": (C.c_int, [_P, _P, C.POINTER(C.c_longlong)]),
        "hmat_b200_leaf_gradients": (C.c_int, [_P, _P, _P, C.c_int, _P, C.c_int, _P]),
        "hmat_b200_gemv_adjoint": (C.c_int, [_P, _P, _P, C.c_int, _P, _P, C.c_int, _P]),
        "hmat_b200_phase_times": (C.c_int, [_P, _P]),
        "hmat_b200_gemv_profile": (C.c_int, [_P, C.c_char, _P, _P, C.c_int, _P, _P]),
        "hmat_b200_gemv_launches": (C.c_int, [_P, C.c_char, C.c_int]),
        "hmat_b200_aca_shapes": (C.c_int, [_P, _P, _P, _P]),
        "hmat_b200_gemv_tuning": (C.c_int, [_P, _P, _P, _P]),
        "hmat_b200_last_error": (C.c_char_p, []),
        "hmat_b200_clear_last_error": (None, []),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


class HMatError(RuntimeError):
    pass


def _check(rc: int, what: str):
    if rc != 0:
        msg = load_library().hmat_b200_last_error().decode()
        raise HMatError(f"{what} failed: {msg}")


def get_parameters() -> Settings:
    s = Settings()
    load_library().hmat_get_parameters(C.byref(s))
    return s


def set_parameters(**kw):
    s = get_parameters()
    for k, v in kw.items():
        setattr(s, k, v)
    _check(load_library().hmat_set_parameters(C.byref(s)), "hmat_set_parameters")


class HMatInterface:
    """The function table of one value type (hmat_init_default_interface)."""

    def __init__(self, value_type: int):
        lib = load_library()
        self.value_type = value_type
        self.table = InterfaceTable()
        lib.hmat_init_default_interface(C.byref(self.table), value_type)
        self._fns = {}

    def fn(self, slot: str):
        if slot not in self._fns:
            self._fns[slot] = _PROTOS[slot](getattr(self.table, slot))
        return self._fns[slot]

    def create_empty_hmatrix_admissibility(self, rows_tree, cols_tree, lower_symmetric, cond):
        return self.fn("create_empty_hmatrix_admissibility")(rows_tree, cols_tree, lower_symmetric, cond)

    def set_low_rank_epsilon(self, m, eps):
        self.fn("set_low_rank_epsilon")(m, eps)

    def assemble_generic(self, m, ctx: AssembleContext) -> int:
        return self.fn("assemble_generic")(m, C.byref(ctx))

    def gemv(self, trans, alpha, m, x, beta, y, nrhs) -> int:
        return self.fn("gemv")(trans, alpha, m, x, beta, y, nrhs)

    def get_info(self, m) -> Info:
        info = Info()
        _check(self.fn("get_info")(m, C.byref(info)), "get_info")
        return info

    def destroy(self, m) -> int:
        return self.fn("destroy")(m)


class HMatrix:
    """One H-matrix on the B200 engine, built the way the reference's examples build theirs:
    median clustering with a maximum leaf size, standard admissibility, ACA+ compression at
    `epsilon`, low-rank epsilon `low_rank_epsilon` (defaults to `epsilon`)."""

    def __init__(self, points: np.ndarray, kernel: KernelDesc, *, value_type: int = HMAT_DOUBLE_PRECISION,
                 leaf_size: int = 64, eta: float = 2.0, epsilon: float = 1e-4, low_rank_epsilon: float | None = None,
                 compression: str = "aca_plus", assemble: bool = True, leaf_size_cols: int | None = None):
        lib = load_library()
        self.lib = lib
        self.points = np.ascontiguousarray(points, dtype=np.float64)
        self.n = int(self.points.shape[0])
        self.value_type = value_type
        self.dtype = DTYPES[value_type]
        self.hi = HMatInterface(value_type)
        self._median = lib.hmat_create_clustering_median()
        self._algo = lib.hmat_create_clustering_max_dof(self._median, leaf_size)
        self.tree = lib.hmat_create_cluster_tree(self.points.ctypes.data, 3, self.n, self._algo)
        if not self.tree:
            raise HMatError("hmat_create_cluster_tree failed: " + lib.hmat_b200_last_error().decode())
        self._algo_c = self.tree_cols = None
        if leaf_size_cols:
            self._algo_c = lib.hmat_create_clustering_max_dof(self._median, leaf_size_cols)
            self.tree_cols = lib.hmat_create_cluster_tree(self.points.ctypes.data, 3, self.n, self._algo_c)
        self._adm = lib.hmat_create_admissibility_standard(eta)
        self.m = self.hi.create_empty_hmatrix_admissibility(self.tree, self.tree_cols or self.tree, 0, self._adm)
        if not self.m:
            raise HMatError("create_empty_hmatrix_admissibility failed: " + lib.hmat_b200_last_error().decode())
        self.hi.set_low_rank_epsilon(self.m, epsilon if low_rank_epsilon is None else low_rank_epsilon)
        make = {"aca_plus": lib.hmat_create_compression_aca_plus,
                "aca_partial": lib.hmat_create_compression_aca_partial,
                "svd": lib.hmat_create_compression_svd}[compression]
        self._comp = make(epsilon)
        self._kernel = kernel
        strata = getattr(kernel, "strata", None)
        if strata is not None:
            sp = np.ascontiguousarray(strata[0], dtype=np.float64)
            sw = np.ascontiguousarray(strata[1], dtype=np.float64)
            self._assembly = lib.hmat_b200_create_assembly_strata(C.byref(kernel), self.points.ctypes.data, self.n,
                                                                  len(sp), sp.ctypes.data, sw.ctypes.data)
        else:
            self._assembly = lib.hmat_b200_create_assembly(C.byref(kernel), self.points.ctypes.data, self.n)
        if not self._assembly:
            raise HMatError("hmat_b200_create_assembly failed: " + lib.hmat_b200_last_error().decode())
        if assemble:
            self.assemble()

    # -- reference-shaped operations --
    def assemble(self):
        ctx = AssembleContext()
        self.lib.hmat_assemble_context_init(C.byref(ctx))
        ctx.assembly = self._assembly
        ctx.compression = self._comp
        ctx.factorization = hmat_factorization_none
        _check(self.hi.assemble_generic(self.m, ctx), "assemble_generic")

    def gemv(self, x: np.ndarray, trans: str = "N", alpha=1.0, beta=0.0, y: np.ndarray | None = None) -> np.ndarray:
        """y = alpha op(H) x + beta y through the C table's gemv (host buffers)."""
        x = np.asfortranarray(x, dtype=self.dtype)
        nrhs = 1 if x.ndim == 1 else x.shape[1]
        if y is None:
            y = np.zeros_like(x)
        else:
            y = np.array(y, dtype=self.dtype, order="F", copy=True)
        a = np.array([alpha], dtype=self.dtype)
        b = np.array([beta], dtype=self.dtype)
        _check(self.hi.gemv(trans.encode(), a.ctypes.data, self.m, x.ctypes.data, b.ctypes.data, y.ctypes.data,
                            nrhs), "gemv")
        return y

    def gemv_device(self, x_ptr: int, y_ptr: int, nrhs: int, trans: str = "N", alpha=1.0, beta=0.0, stream=0):
        a = np.array([alpha], dtype=self.dtype)
        b = np.array([beta], dtype=self.dtype)
        _check(self.lib.hmat_b200_gemv_device(self.m, trans.encode(), a.ctypes.data, C.c_void_p(x_ptr),
                                              b.ctypes.data, C.c_void_p(y_ptr), nrhs, C.c_void_p(stream)),
               "hmat_b200_gemv_device")

    def gemv_device_noalloc(self, x_ptr: int, y_ptr: int, nrhs: int, trans: str = "N", alpha=1.0, beta=0.0,
                            stream=0) -> int:
        """The allocation-free device gemv; returns the C return code (0 on success)."""
        a = np.array([alpha], dtype=self.dtype)
        b = np.array([beta], dtype=self.dtype)
        return self.lib.hmat_b200_gemv_device_noalloc(self.m, trans.encode(), a.ctypes.data, C.c_void_p(x_ptr),
                                                      b.ctypes.data, C.c_void_p(y_ptr), nrhs, C.c_void_p(stream))

    def gemv_status(self, stream=0) -> int:
        """Non-zero if a device product of this matrix failed since the last query
        (hmat_b200_gemv_status; clears the flag): 1 a kernel's wait for a bulk copy gave up, 2 a
        unit failed the kernels' checks of its copies.  0 when all went well."""
        failed = C.c_int(0)
        _check(self.lib.hmat_b200_gemv_status(self.m, C.c_void_p(stream), C.byref(failed)), "hmat_b200_gemv_status")
        return int(failed.value)

    def info(self) -> dict:
        return self.hi.get_info(self.m).as_dict()

    def perm(self, cols: bool = False) -> np.ndarray:
        if getattr(self, "_borrowed_trees", None):  # a matrix read from a stream owns its trees
            rt, ct = self._borrowed_trees
            p = self.lib.hmat_cluster_get_indices(ct if cols else rt)
        else:
            p = self.lib.hmat_cluster_get_indices(self.tree_cols if (cols and self.tree_cols) else self.tree)
        return np.ctypeslib.as_array(p, shape=(self.n,)).copy()

    # -- write_struct / write_data / read_struct / read_data --
    def dump(self) -> tuple:
        """(struct, data) streams of this matrix, through the C table's write_struct and
        write_data."""
        chunks = []
        cb = _IOSTREAM(lambda buf, n, ud: chunks.append(C.string_at(buf, n)) if n else None)
        self.lib.hmat_b200_clear_last_error()
        self.hi.fn("write_struct")(self.m, cb, None)
        st = b"".join(chunks)
        chunks.clear()
        self.hi.fn("write_data")(self.m, cb, None)
        err = self.lib.hmat_b200_last_error()
        if err:
            raise HMatError(err.decode())
        return st, b"".join(chunks)

    def read_data(self, data_stream: bytes):
        """The leaves of a data stream (hmat_interface_t.write_data of this library or of the
        reference: both write the reference's data format) into this matrix, which must have
        the writer's partition: hmat_interface_t.read_data.  The matrix is then assembled."""
        pos, short = [0], []

        def rd(buf, n, ud):
            if n == 0:
                return
            take = data_stream[pos[0]:pos[0] + n]
            pos[0] += n
            if len(take) < n:
                short.append(n)
                take = take + bytes(n - len(take))
            C.memmove(buf, take, n)
        self.lib.hmat_b200_clear_last_error()
        self.hi.fn("read_data")(self.m, _IOSTREAM(rd), None)
        err = self.lib.hmat_b200_last_error()
        if err or short or pos[0] != len(data_stream):
            raise HMatError((err.decode() if err else "") + (" (stream too short)" if short else "") +
                            (" (stream longer than the matrix's leaves)" if pos[0] < len(data_stream) else ""))

    @classmethod
    def load(cls, value_type: int, struct_stream: bytes, data_stream: bytes) -> "HMatrix":
        """A matrix read back with read_struct and read_data (no clustering, no assembly)."""
        lib = load_library()
        hi = HMatInterface(value_type)
        short = []

        def reader(data):
            pos = [0]

            def rd(buf, n, ud):
                if n == 0:
                    return
                take = data[pos[0]:pos[0] + n]
                pos[0] += n
                if len(take) < n:  # past the end: zeros, reported after the call
                    short.append(n)
                    take = take + bytes(n - len(take))
                C.memmove(buf, take, n)
            return _IOSTREAM(rd)

        lib.hmat_b200_clear_last_error()
        rs, rdd = reader(struct_stream), reader(data_stream)
        m = hi.fn("read_struct")(rs, None)
        if not m:
            raise HMatError("read_struct failed: " + lib.hmat_b200_last_error().decode())
        hi.fn("read_data")(m, rdd, None)
        err = lib.hmat_b200_last_error()
        if err or short:
            hi.destroy(m)
            raise HMatError((err.decode() if err else "") + (" (stream too short)" if short else ""))
        obj = cls.__new__(cls)
        obj.lib, obj.hi, obj.m = lib, hi, m
        obj.value_type, obj.dtype = value_type, DTYPES[value_type]
        rt, ct = C.c_void_p(), C.c_void_p()
        hi.fn("get_cluster_trees")(m, C.byref(rt), C.byref(ct))
        obj._borrowed_trees = (rt.value, ct.value)
        obj.tree = obj.tree_cols = None
        info = ClusterInfo()
        lib.hmat_cluster_get_info(rt, C.byref(info))
        obj.n = int(info.dimension)
        return obj

    def leaf_table(self) -> np.ndarray:
        n = self.lib.hmat_b200_leaf_count(self.m)
        out = np.zeros((n, 6), dtype=np.int32)
        _check(self.lib.hmat_b200_leaf_table(self.m, out.ctypes.data), "hmat_b200_leaf_table")
        return out

    def leaf_payload(self, i: int) -> np.ndarray:
        r0, m, c0, n, t, k = self.leaf_table()[i]
        size = m * n if t == 0 else max(k, 0) * (m + n)
        out = np.zeros(max(size, 1), dtype=self.dtype)
        got = self.lib.hmat_b200_leaf_payload(self.m, i, out.ctypes.data)
        if got < 0:
            raise HMatError("hmat_b200_leaf_payload failed")
        return out[:got]

    def leaf_block(self, i: int) -> np.ndarray:
        """The dense block of leaf i (F, or A B^T), in cluster numbering."""
        r0, m, c0, n, t, k = self.leaf_table()[i]
        p = self.leaf_payload(i)
        if t == 0:
            return p.reshape(n, m).T
        if k <= 0:
            return np.zeros((m, n), dtype=self.dtype)
        A = p[:k * m].reshape(k, m).T
        B = p[k * m:].reshape(k, n).T
        return A @ B.T

    def payload_layout(self):
        """Canonical payload offsets per leaf and the total number of scalars."""
        n = self.lib.hmat_b200_leaf_count(self.m)
        offs = np.zeros(n, dtype=np.int64)
        tot = C.c_longlong()
        _check(self.lib.hmat_b200_payload_layout(self.m, offs.ctypes.data, C.byref(tot)), "hmat_b200_payload_layout")
        return offs, tot.value

    def leaf_gradients(self, x_ptr, r_ptr, nrhs, grad_ptr, accumulate=False, stream=0):
        _check(self.lib.hmat_b200_leaf_gradients(self.m, C.c_void_p(x_ptr), C.c_void_p(r_ptr), nrhs,
                                                 C.c_void_p(grad_ptr), int(accumulate), C.c_void_p(stream)),
               "hmat_b200_leaf_gradients")

    def gemv_adjoint(self, x_ptr, r_ptr, nrhs, dx_ptr, grad_ptr, accumulate=False, stream=0):
        """dx = H^T r and the leaf gradients in one pass (hmat_b200_gemv_adjoint)."""
        _check(self.lib.hmat_b200_gemv_adjoint(self.m, C.c_void_p(x_ptr), C.c_void_p(r_ptr), nrhs, C.c_void_p(dx_ptr),
                                               C.c_void_p(grad_ptr), int(accumulate), C.c_void_p(stream)),
               "hmat_b200_gemv_adjoint")

    def gemv_profile(self, x_ptr: int, y_ptr: int, nrhs: int, trans: str = "N"):
        ms = np.zeros(3)
        by = np.zeros(3)
        _check(self.lib.hmat_b200_gemv_profile(self.m, trans.encode(), C.c_void_p(x_ptr), C.c_void_p(y_ptr), nrhs,
                                               ms.ctypes.data, by.ctypes.data), "hmat_b200_gemv_profile")
        return {"ms": dict(zip(("gather", "zphase", "yphase"), ms)),
                "bytes": dict(zip(("gather", "zphase", "yphase"), by))}

    def gemm_dense(self, trans_b: str, trans_x: str, side: str, alpha, x: np.ndarray, beta, y: np.ndarray) -> np.ndarray:
        """op(Y) <- alpha op(B) op(X) + beta op(Y) (side 'L') or Y <- alpha op(X) op(B) + beta Y
        (side 'R') in the internal numbering, through the C table's gemm_dense.  x and y are
        column-major arrays whose shapes follow the flags; returns the new y."""
        xf = np.array(x, dtype=self.dtype, order="F", copy=True)
        yf = np.array(y, dtype=self.dtype, order="F", copy=True)
        if yf.ndim != 2:
            raise ValueError("y must be 2-D (n x nrhs for side 'L', nrhs x n for side 'R')")
        nrhs = yf.shape[0] if side == "R" else yf.shape[1]
        a = np.array([alpha], dtype=self.dtype)
        b = np.array([beta], dtype=self.dtype)
        _check(self.hi.fn("gemm_dense")(trans_b.encode(), trans_x.encode(), side.encode(), a.ctypes.data, self.m,
                                        xf.ctypes.data, b.ctypes.data, yf.ctypes.data, int(nrhs)), "gemm_dense")
        return yf

    def gemm_scalar(self, x: np.ndarray, trans: str = "N", alpha=1.0, beta=0.0, y: np.ndarray | None = None):
        """gemv in the internal numbering (the C table's gemm_scalar)."""
        xf = np.asfortranarray(x, dtype=self.dtype)
        nrhs = 1 if xf.ndim == 1 else xf.shape[1]
        yf = np.zeros_like(xf) if y is None else np.array(y, dtype=self.dtype, order="F", copy=True)
        a = np.array([alpha], dtype=self.dtype)
        b = np.array([beta], dtype=self.dtype)
        _check(self.hi.fn("gemm_scalar")(trans.encode(), a.ctypes.data, self.m, xf.ctypes.data, b.ctypes.data,
                                         yf.ctypes.data, nrhs), "gemm_scalar")
        return yf

    def get_block(self, row_offset: int, row_size: int, col_offset: int, col_size: int, renumber_rows=False):
        """Dense block (internal numbering) and its row / column numbering (get_block)."""
        out = np.zeros((row_size, col_size), dtype=self.dtype, order="F")
        ctx = GetValuesContext(self.m, out.ctypes.data, row_offset, col_offset, row_size, col_size, None, None,
                               int(bool(renumber_rows)))
        _check(self.hi.fn("get_block")(C.byref(ctx)), "get_block")
        rows = np.ctypeslib.as_array(ctx.row_indices, shape=(row_size,)).copy() if row_size else np.zeros(0, int)
        cols = np.ctypeslib.as_array(ctx.col_indices, shape=(col_size,)).copy() if col_size else np.zeros(0, int)
        return out, rows, cols

    def get_values(self, rows, cols) -> np.ndarray:
        """Entries for rows x cols given in natural numbering 1..n (get_values)."""
        r = np.ascontiguousarray(rows, dtype=np.int32)
        c = np.ascontiguousarray(cols, dtype=np.int32)
        out = np.zeros((len(r), len(c)), dtype=self.dtype, order="F")
        ctx = GetValuesContext(self.m, out.ctypes.data, 0, 0, len(r), len(c),
                               r.ctypes.data_as(C.POINTER(C.c_int)), c.ctypes.data_as(C.POINTER(C.c_int)), 0)
        _check(self.hi.fn("get_values")(C.byref(ctx)), "get_values")
        return out

    def set_low_rank_epsilon(self, eps: float) -> None:
        self.hi.fn("set_low_rank_epsilon")(self.m, eps)

    def truncate(self, eps: float | None = None) -> None:
        """Re-truncates every Rk leaf at the low-rank epsilon (set first when `eps` is given),
        through the C table's truncate."""
        if eps is not None:
            self.set_low_rank_epsilon(eps)
        _check(self.hi.fn("truncate")(self.m), "truncate")

    def gemv_launches(self, nrhs: int, trans: str = "N") -> int:
        """Kernel launches one product with nrhs right-hand sides makes."""
        n = self.lib.hmat_b200_gemv_launches(self.m, trans.encode(), nrhs)
        if n < 0:
            raise HMatError("hmat_b200_gemv_launches failed: " + self.lib.hmat_b200_last_error().decode())
        return n

    def phase_times(self) -> dict:
        out = np.zeros(4, dtype=np.float64)
        _check(self.lib.hmat_b200_phase_times(self.m, out.ctypes.data), "hmat_b200_phase_times")
        return {"full_ms": out[0], "aca_ms": out[1], "truncate_ms": out[2], "gemv_ms": out[3]}

    def aca_tuning(self) -> dict:
        """ACA kernel shape per leaf-size bucket of the last assembly: bucket name ->
        {"threads": 0 (warp per leaf) / 64 / 128 / 512, "how": "default" / "measured" /
        "cached", "rates": leaf cost per ms of each sampled shape}; empty buckets omitted."""
        shape = np.zeros(4, dtype=np.int32)
        tuned = np.zeros(4, dtype=np.int32)
        rate = np.zeros(20, dtype=np.float64)
        _check(self.lib.hmat_b200_aca_shapes(self.m, shape.ctypes.data, tuned.ctypes.data, rate.ctypes.data),
               "hmat_b200_aca_shapes")
        names = ("m,n<=64", "m+n<2048", "m+n<8192", "m+n>=8192")
        shapes = ("warp", "64", "128", "256", "512")
        out = {}
        for b in range(4):
            if shape[b] < 0:
                continue
            out[names[b]] = {"threads": int(shape[b]), "how": ("default", "measured", "cached")[int(tuned[b])],
                             "rates": {shapes[s]: float(rate[5 * b + s]) for s in range(5) if rate[5 * b + s] > 0}}
        return out

    def gemv_tuning(self) -> dict:
        """The gemv tuner's choice for this matrix's 'N' schedule (hmat_b200_gemv_tuning)."""
        ch = np.zeros(2, np.int32)
        how = C.c_int()
        ms = np.zeros(5)
        _check(self.lib.hmat_b200_gemv_tuning(self.m, ch.ctypes.data, C.byref(how), ms.ctypes.data),
               "hmat_b200_gemv_tuning")
        return {"z_chunk_units": int(ch[0]), "y_units": ("widest", "half")[int(ch[1])],
                "how": ("default", "measured", "cached")[how.value],
                "ms": {"z8": ms[0], "z16": ms[1], "z32": ms[2], "y_widest": ms[3], "y_half": ms[4]}}

    def gemv_bytes(self, nrhs: int) -> int:
        """Algorithmic bytes of one product: every stored leaf scalar read once, x read and
        y written once."""
        t = self.leaf_table()
        s = np.dtype(self.dtype).itemsize
        full = t[t[:, 4] == 0]
        rk = t[(t[:, 4] == 1) & (t[:, 5] > 0)]
        stored = int((full[:, 1].astype(np.int64) * full[:, 3]).sum() +
                     (rk[:, 5].astype(np.int64) * (rk[:, 1] + rk[:, 3])).sum())
        return stored * s + 2 * self.n * nrhs * s

    def close(self):
        lib = self.lib
        if getattr(self, "m", None):
            self.hi.destroy(self.m)
            self.m = None
        for attr, fn in (("_assembly", lib.hmat_b200_delete_assembly), ("_comp", lib.hmat_delete_compression),
                         ("_adm", lib.hmat_delete_admissibility), ("tree", lib.hmat_delete_cluster_tree),
                         ("tree_cols", lib.hmat_delete_cluster_tree), ("_algo", lib.hmat_delete_clustering),
                         ("_algo_c", lib.hmat_delete_clustering), ("_median", lib.hmat_delete_clustering)):
            v = getattr(self, attr, None)
            if v:
                fn(v)
                setattr(self, attr, None)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class HMatrixBatch(HMatrix):
    """Independent H-matrices assembled and multiplied together (hmat_b200_batch_*): member i
    is built on points[i] with kernels[i] (one kernel kind and nugget; each its own correlation
    length, regularisation or wavenumber), all with the same value type, leaf size, eta and
    epsilon.  The object is the block-diagonal matrix of the members: gemv takes the members'
    vectors stacked (offsets()[0] gives each member's first row), leaf_table() lists the
    members' leaves in order (offsets()[1])."""

    def __init__(self, points: list, kernels: list, *, value_type: int = HMAT_DOUBLE_PRECISION, leaf_size: int = 64,
                 eta: float = 2.0, epsilon: float = 1e-4, compression: str = "aca_plus", assemble: bool = True):
        if len(points) != len(kernels) or not points:
            raise ValueError("one kernel per member matrix")
        lib = load_library()
        self.lib = lib
        self.value_type = value_type
        self.dtype = DTYPES[value_type]
        self.hi = HMatInterface(value_type)
        self.members = [HMatrix(p, k, value_type=value_type, leaf_size=leaf_size, eta=eta, epsilon=epsilon,
                                compression=compression, assemble=False) for p, k in zip(points, kernels)]
        arr = (C.c_void_p * len(self.members))(*[mm.m for mm in self.members])
        self.m = lib.hmat_b200_batch_create(arr, len(self.members))
        if not self.m:
            raise HMatError("hmat_b200_batch_create failed: " + lib.hmat_b200_last_error().decode())
        self.n = int(sum(len(p) for p in points))
        self.tree = self.tree_cols = None
        self._borrowed_trees = None
        self._comp = self.members[0]._comp
        if assemble:
            self.assemble()

    def assemble(self):
        arr = (C.c_void_p * len(self.members))(*[mm._assembly for mm in self.members])
        _check(self.lib.hmat_b200_batch_assemble(self.m, arr, self._comp), "hmat_b200_batch_assemble")

    def offsets(self):
        """(first row of each member, first leaf of each member), count + 1 entries each."""
        rb = np.zeros(len(self.members) + 1, np.int32)
        lb = np.zeros(len(self.members) + 1, np.int32)
        _check(self.lib.hmat_b200_batch_offsets(self.m, rb.ctypes.data, lb.ctypes.data), "hmat_b200_batch_offsets")
        return rb, lb

    def perm(self, cols: bool = False) -> np.ndarray:
        rt, ct = C.c_void_p(), C.c_void_p()
        self.hi.fn("get_cluster_trees")(self.m, C.byref(rt), C.byref(ct))
        p = self.lib.hmat_cluster_get_indices(ct if cols else rt)
        return np.ctypeslib.as_array(p, shape=(self.n,)).copy()

    def close(self):
        if getattr(self, "m", None):
            self.hi.destroy(self.m)
            self.m = None
        for mm in getattr(self, "members", []):
            mm.close()
        self.members = []


def kernel(kind: int, delta: float = 0.01, ell: float = 0.3, nugget: float = 0.0, wavenumber: float = 0.0,
           strata_param=None, strata_weight=None):
    """Kernel descriptor.  With strata_param / strata_weight (same length, 1 to 8), a multi-strata
    kernel: stratum q is strata_weight[q] times the kernel with its parameter (ell, delta or
    wavenumber by kind) set to strata_param[q] (hmat_b200_create_assembly_strata)."""
    k = KernelDesc(kind, delta, ell, nugget, wavenumber)
    if strata_param is not None or strata_weight is not None:
        if strata_param is None or strata_weight is None or len(strata_param) != len(strata_weight):
            raise ValueError("strata_param and strata_weight: both, same length")
        k.strata = (list(map(float, strata_param)), list(map(float, strata_weight)))
    return k
