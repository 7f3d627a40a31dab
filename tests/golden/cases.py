"""Inputs of the golden fixtures: seeded point clouds, kernels, tree parameters and
right-hand sides (shared by make_golden.py and the tests that replay the cases)."""
import importlib.util
import os

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))

spec = importlib.util.spec_from_file_location("workloads", os.path.join(ROOT, "hmat-oss_b200", "workloads.py"))
wl = importlib.util.module_from_spec(spec)
spec.loader.exec_module(wl)

# name -> (points builder, kernel kwargs, tree/compression kwargs, nrhs, rhs seed, scalar, dump payload)
CASES = {
    "cfg0_laplace": (lambda: wl.cylinder(80, 100), dict(kind=0, delta=0.01), dict(leaf=64, eta=2.0, eps=1e-4), 1, 0,
                     "D", False),
    "cube_expcov": (lambda: wl.cube(800, 11), dict(kind=1, ell=0.3, nugget=1e-6), dict(leaf=32, eta=2.0, eps=1e-6), 3,
                    12, "D", False),
    "cube_expcov_payload": (lambda: wl.cube(300, 21), dict(kind=1, ell=0.2, nugget=1e-6),
                            dict(leaf=16, eta=2.0, eps=1e-5), 1, 22, "D", True),
    "helmholtz_small": (lambda: wl.cylinder(30, 40), dict(kind=2, delta=0.01, wavenumber=wl.helmholtz_wavenumber(1200)),
                        dict(leaf=32, eta=3.0, eps=1e-4), 2, 13, "Z", False),
    "helmholtz_payload": (lambda: wl.cylinder(15, 20), dict(kind=2, delta=0.01, wavenumber=wl.helmholtz_wavenumber(300)),
                          dict(leaf=16, eta=3.0, eps=1e-4), 1, 23, "Z", True),
    "tall_partial": (lambda: wl.cube(6000, 5), dict(kind=1, ell=0.3, nugget=1e-6),
                     dict(leaf=2048, leaf_cols=16, eta=2.0, eps=1e-5), 1, 3, "D", False),
    "svd_small": (lambda: wl.cylinder(40, 50), dict(kind=0, delta=0.01), dict(leaf=32, eta=2.0, eps=1e-4, min_leaf=100),
                  2, 14, "D", False),
    # the headline workload: 100,000-point cylinder (250 x 400 grid), eps 1e-6, 2 of its 16 RHS
    "cfg1_cylinder": (lambda: wl.cylinder(250, 400), dict(kind=0, delta=0.01), dict(leaf=64, eta=2.0, eps=1e-6), 2, 1,
                      "D", False),
    # the adjoint workload's shape at 20,000 points: uniform cube, exponential covariance l=0.3
    "cfg4_cube": (lambda: wl.cube(20000, 2), dict(kind=1, ell=0.3, nugget=1e-6), dict(leaf=64, eta=2.0, eps=1e-6), 2,
                  2, "D", False),
    # assembled at 1e-6, then set_low_rank_epsilon(1e-3) + truncate
    "retrunc_expcov": (lambda: wl.cube(800, 31), dict(kind=1, ell=0.3, nugget=1e-6),
                       dict(leaf=32, eta=2.0, eps=1e-6, retrunc=1e-3), 2, 32, "D", True),
}


# Multi-strata kernels assembled through advanced_compute (one stratum a material: w_s times the
# kernel with parameter a_s).  Kept apart from CASES: the device engine does not assemble them;
# they pin the oracle's restatement of compress() over strata (compression.cpp:745-773) and of
# formattedAddParts (rk_matrix.cpp:846-1009).
STRATA_CASES = {
    "strata_expcov": (lambda: wl.cube(800, 41),
                      dict(kind=1, strata_param=[0.1, 0.3, 1.0], strata_weight=[1.0, 0.5, 0.25]),
                      dict(leaf=32, eta=2.0, eps=1e-6), 2, 42, "D", True),
    "strata_laplace_signed": (lambda: wl.cylinder(20, 30),
                              dict(kind=0, strata_param=[0.01, 0.2], strata_weight=[1.0, -0.5]),
                              dict(leaf=16, eta=2.0, eps=1e-10), 1, 44, "D", False),
    "strata_helmholtz": (lambda: wl.cylinder(15, 20),
                         dict(kind=2, delta=0.01, strata_param=[5.0, 12.0], strata_weight=[1.0, 0.5]),
                         dict(leaf=16, eta=3.0, eps=1e-6), 1, 45, "Z", False),
}


def inputs(name):
    build, kern, tree, nrhs, seed, scalar, dump = CASES[name] if name in CASES else STRATA_CASES[name]
    pts = build()
    x = wl.rhs(len(pts), nrhs, seed, complex_=scalar in ("Z", "C"))
    return pts, x
