"""write_struct / read_struct / write_data / read_data (the reference's checkpoint entries,
c_wrapping.hpp:921-946): a matrix written and read back has the same cluster trees, leaves and
products, without re-assembly.  The structure stream is this library's own format; the data
stream is the reference's (MatrixDataMarshaller, serialization.cpp:248-309): the non-empty
leaves in depth-first order, an Rk leaf as its rank, A, B and two orthogonality ints, a full
leaf as a header int and its entries."""
import ctypes as C

import numpy as np
import pytest
from cases import CASES, inputs


def _build(hb, name, vt, assemble=True):
    _, kern, tree, nrhs, seed, scalar, dump = CASES[name]
    pts, x = inputs(name)
    hb.set_parameters(compressionMinLeafSize=tree.get("min_leaf", 0))
    k = hb.kernel(kern["kind"], delta=kern.get("delta", 0.01), ell=kern.get("ell", 0.3),
                  nugget=kern.get("nugget", 0.0), wavenumber=kern.get("wavenumber", 0.0))
    h = hb.HMatrix(pts, k, value_type=vt, leaf_size=tree["leaf"], eta=tree["eta"], epsilon=tree["eps"],
                   assemble=assemble)
    return h, x


def _struct_bytes(hb, h):
    chunks = []
    cb = hb._IOSTREAM(lambda buf, n, ud: chunks.append(C.string_at(buf, n)) if n else None)
    h.hi.fn("write_struct")(h.m, cb, None)
    return b"".join(chunks)


def _read_struct(hb, hi, data):
    pos = [0]

    def rd(buf, n, ud):
        take = data[pos[0]:pos[0] + n]
        pos[0] += n
        C.memmove(buf, take + bytes(n - len(take)), n)
    return hi.fn("read_struct")(hb._IOSTREAM(rd), None)


def test_struct_round_trip_host_only(hb):
    """Cluster trees and leaves survive write_struct / read_struct (no GPU needed)."""
    h, _ = _build(hb, "cube_expcov", hb.HMAT_DOUBLE_PRECISION, assemble=False)
    try:
        st = _struct_bytes(hb, h)
        assert st[:4] == b"HB2S"
        m2 = _read_struct(hb, h.hi, st)
        assert m2
        try:
            rt, ct = C.c_void_p(), C.c_void_p()
            assert h.hi.fn("get_cluster_trees")(m2, C.byref(rt), C.byref(ct)) == 0
            p = np.ctypeslib.as_array(h.lib.hmat_cluster_get_indices(rt), shape=(h.n,))
            assert np.array_equal(p, h.perm())
            n = h.lib.hmat_b200_leaf_count(m2)
            t2 = np.zeros((n, 6), dtype=np.int32)
            assert h.lib.hmat_b200_leaf_table(m2, t2.ctypes.data) == 0
            assert np.array_equal(t2[:, :5], h.leaf_table()[:, :5])
        finally:
            h.hi.destroy(m2)
        # a stream cut short, or read by another value type, is refused
        assert not _read_struct(hb, h.hi, st[:len(st) // 2])
        assert not _read_struct(hb, hb.HMatInterface(hb.HMAT_SIMPLE_PRECISION), st)
    finally:
        h.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name,vt", [("cube_expcov", 1), ("cube_expcov", 0), ("helmholtz_small", 3)])
def test_checkpoint_round_trip(hb, name, vt):
    h, x = _build(hb, name, vt)
    try:
        st, data = h.dump()
        # the reference's data layout, leaf by leaf
        T = h.leaf_table()
        sz = np.dtype(h.dtype).itemsize
        full = T[:, 4] == 0
        rk = (T[:, 4] == 1) & (T[:, 5] > 0)
        want = 4 * len(T) + sz * int((T[full, 1].astype(np.int64) * T[full, 3]).sum() +
                                     (T[rk, 5].astype(np.int64) * (T[rk, 1] + T[rk, 3])).sum()) + 8 * int(rk.sum())
        assert len(data) == want
        first = int(np.frombuffer(data[:4], np.int32)[0])
        assert first == (0 if T[0, 4] == 0 else T[0, 5])
        g = hb.HMatrix.load(vt, st, data)
        try:
            assert np.array_equal(g.perm(), h.perm())
            assert np.array_equal(g.leaf_table(), h.leaf_table())
            xs = x.astype(h.dtype)
            assert np.array_equal(g.gemv(xs), h.gemv(xs))
            assert np.array_equal(g.gemv(xs, "T"), h.gemv(xs, "T"))
            # writing the loaded matrix gives the same streams
            st2, data2 = g.dump()
            assert st2 == st and data2 == data
        finally:
            g.close()
        with pytest.raises(hb.HMatError):
            hb.HMatrix.load(vt, st, data[:len(data) - 8])
    finally:
        h.close()
