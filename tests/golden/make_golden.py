"""Generates the golden fixtures of tests/golden/ by running the reference library itself.

The reference hmat-oss is compiled from its own sources by oracle/Makefile.ref into
oracle/_ref/ (libhmat_ref.so + ref_driver, a driver over the reference's public C API).
This script runs that driver on small seeded inputs and stores what the parity tests
compare against: cluster permutations, leaf lists (offsets, sizes, type, rank), gemv
results for 'N' and 'T', hmat_info_t fields and, for the smallest cases, the leaf
payloads.  The multi-strata cases assemble through advanced_compute with one stratum a
material.  Inputs are regenerated from their seeds by the tests, so only outputs are
stored.

Usage (where the reference tree and oracle/_ref exist):  python tests/golden/make_golden.py
"""
import importlib.util
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, HERE)
import oracle as O  # noqa: E402

from cases import CASES, STRATA_CASES, inputs  # noqa: E402


def make(name):
    _, kern, tree, nrhs, _, scalar, dump = CASES[name] if name in CASES else STRATA_CASES[name]
    pts, x = inputs(name)
    out = {}
    rn = O.run_reference(pts, x=x, nrhs=nrhs, trans="N", scalar=scalar, dump_factors=dump, **kern, **tree)
    out["perm"] = rn["perm"]
    out["perm_cols"] = rn["perm_cols"]
    out["leaves"] = rn["leaves"]
    out["y"] = rn["y"]
    info = rn["json"]
    for k in ("full_count", "rk_count", "full_size", "rk_size", "compressed_size", "uncompressed_size",
              "nr_block_clusters", "largest_rk_dim_rows", "largest_rk_dim_cols", "largest_rk_mem_rows",
              "largest_rk_mem_cols", "largest_rk_mem_rank"):
        out["info_" + k] = np.int64(info[k])
    if dump:
        # keep the Rk factors only (full leaves are plain kernel entries)
        pay, off, keep = rn["payload"], 0, []
        for r0, m, c0, n, t, k in rn["leaves"]:
            size = m * n if t == 0 else max(k, 0) * (m + n)
            if t == 1:
                keep.append(pay[off:off + size])
            off += size
        out["rk_payload"] = np.concatenate(keep) if keep else np.zeros(0, pay.dtype)
    rt = O.run_reference(pts, x=x, nrhs=nrhs, trans="T", scalar=scalar, **kern, **tree)
    out["y_T"] = rt["y"]
    if scalar in ("Z", "C"):
        rc = O.run_reference(pts, x=x, nrhs=nrhs, trans="C", scalar=scalar, **kern, **tree)
        out["y_C"] = rc["y"]
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    print(name, {k: getattr(v, "shape", v) for k, v in out.items() if not k.startswith("info_")})


if __name__ == "__main__":
    for n in (sys.argv[1:] or list(CASES) + list(STRATA_CASES)):
        make(n)
