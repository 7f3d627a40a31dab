"""Checkpoints exchanged with the reference library: write_data / read_data of both libraries
use the reference's data stream (MatrixDataMarshaller / MatrixDataUnmarshaller,
serialization.cpp:248-394), so the leaves of a matrix written by one load into a matrix of the
same partition built by the other.

* reference -> B200: the reference (oracle/_ref, built from its own sources) assembles a fixture
  and writes its data stream; a B200 matrix built on the same points and parameters, not
  assembled, reads it and multiplies: partition and ranks are the reference's, and the product
  equals the reference's own within rounding (1e-13), real and complex.
* B200 -> reference: the B200 engine assembles, writes its data stream, and the reference reads
  it into the matrix it builds and multiplies: its product equals the B200 product within
  rounding, and the whole stream is consumed.
"""
import numpy as np
import pytest
from cases import CASES, inputs
from conftest import rel

pytestmark = pytest.mark.gpu

VT = {"D": 1, "S": 0, "Z": 3, "C": 2}
NAMES = ["cube_expcov", "helmholtz_small", "tall_partial"]


def _ref_kwargs(name):
    _, kern, tree, nrhs, seed, scalar, dump = CASES[name]
    return dict(kind=kern["kind"], eps=tree["eps"], leaf=tree["leaf"], eta=tree["eta"], delta=kern.get("delta", 0.01),
                ell=kern.get("ell", 0.3), nugget=kern.get("nugget", 0.0), wavenumber=kern.get("wavenumber", 0.0),
                leaf_cols=tree.get("leaf_cols") or 0, min_leaf=tree.get("min_leaf", 0))


def _b200(hb, name, scalar, assemble):
    _, kern, tree, nrhs, seed, _, dump = CASES[name]
    pts, x = inputs(name)
    hb.set_parameters(compressionMinLeafSize=tree.get("min_leaf", 0))
    k = hb.kernel(kern["kind"], delta=kern.get("delta", 0.01), ell=kern.get("ell", 0.3),
                  nugget=kern.get("nugget", 0.0), wavenumber=kern.get("wavenumber", 0.0))
    h = hb.HMatrix(pts, k, value_type=VT[scalar], leaf_size=tree["leaf"], leaf_size_cols=tree.get("leaf_cols"),
                   eta=tree["eta"], epsilon=tree["eps"], assemble=assemble)
    return h, pts, x


@pytest.mark.parametrize("name", NAMES)
def test_reference_checkpoint_loads_into_b200(hb, oracle, name):
    if not oracle.have_reference():
        pytest.skip("the reference build (oracle/_ref) is absent")
    scalar = CASES[name][5]
    h, pts, x = _b200(hb, name, scalar, assemble=False)
    try:
        ref = oracle.run_reference(pts, x=x, nrhs=x.shape[1], scalar=scalar, write_data=True, **_ref_kwargs(name))
        h.read_data(ref["data"])
        assert np.array_equal(h.leaf_table(), ref["leaves"])
        assert rel(h.gemv(x), ref["y"]) < 1e-13
    finally:
        h.close()


@pytest.mark.parametrize("name,scalar", [(n, CASES[n][5]) for n in NAMES] + [("cube_expcov", "S")])
def test_b200_checkpoint_loads_into_reference(hb, oracle, name, scalar):
    if not oracle.have_reference():
        pytest.skip("the reference build (oracle/_ref) is absent")
    h, pts, x = _b200(hb, name, scalar, assemble=True)
    try:
        _, data = h.dump()
        xs = x.astype(h.dtype)
        ref = oracle.run_reference(pts, x=xs, nrhs=x.shape[1], scalar=scalar, read_data=data, **_ref_kwargs(name))
        assert np.array_equal(ref["leaves"], h.leaf_table())
        tol = 1e-13 if scalar in ("D", "Z") else 1e-5
        assert rel(ref["y"], h.gemv(xs)) < tol
    finally:
        h.close()
