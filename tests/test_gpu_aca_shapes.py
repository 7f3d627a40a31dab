"""ACA autotuner: the warp-per-leaf kernel and the CTA kernels of 64, 128, 256 and 512
threads build the same factors (Gram terms summed a warp per term, pivot ties broken by first
index), so the shape the autotuner picks per leaf-size bucket only moves time.  Each shape
forced on every leaf it can take, and the autotuner's own sample runs, must give bit-identical
leaves."""
import importlib.util
import os

import numpy as np
import pytest
from conftest import ROOT

pytestmark = pytest.mark.gpu

ENVS = [{"HMAT_B200_ACA_SHAPE": "64"}, {"HMAT_B200_ACA_SHAPE": "128"}, {"HMAT_B200_ACA_SHAPE": "256"},
        {"HMAT_B200_ACA_SHAPE": "512"}, {"HMAT_B200_ACA_SHAPE": "warp"}, {"HMAT_B200_ACA_TUNE": "2"}]


def _workloads():
    spec = importlib.util.spec_from_file_location("wl_shapes", os.path.join(ROOT, "hmat-oss_b200", "workloads.py"))
    wl = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(wl)
    return wl


def _build(hb, monkeypatch, env, vt, kern, pts):
    for k in ("HMAT_B200_ACA_SHAPE", "HMAT_B200_ACA_TUNE"):
        monkeypatch.delenv(k, raising=False)
    for k, v in env.items():
        monkeypatch.setenv(k, v)
    hb.set_parameters(compressionMinLeafSize=0)
    return hb.HMatrix(pts, kern, value_type=vt, leaf_size=64, eta=2.0, epsilon=1e-5)


@pytest.mark.parametrize("vt,kind", [(0, "laplace"), (1, "laplace"), (2, "helmholtz")])
def test_every_aca_shape_builds_the_same_leaves(hb, monkeypatch, vt, kind):
    wl = _workloads()
    pts = wl.cylinder(80, 250)  # 4,352 / 3,904 / 96 Rk leaves in the first three buckets
    kern = hb.kernel(hb.HELMHOLTZ_REG, wavenumber=8.0) if kind == "helmholtz" else hb.kernel(hb.LAPLACE_REG)
    ref = _build(hb, monkeypatch, {"HMAT_B200_ACA_TUNE": "0"}, vt, kern, pts)
    try:
        T = ref.leaf_table()
        want = ref.dump()  # the leaves' factors, serialised in leaf order
        base = ref.aca_tuning()
        assert set(base) >= {"m,n<=64", "m+n<2048", "m+n<8192"}
        assert all(v["how"] == "default" for v in base.values())
    finally:
        ref.close()
    for env in ENVS:
        h = _build(hb, monkeypatch, env, vt, kern, pts)
        try:
            assert np.array_equal(h.leaf_table(), T), env
            got = h.dump()
            assert got[0] == want[0] and got[1] == want[1], env
            tun = h.aca_tuning()
            shape = env.get("HMAT_B200_ACA_SHAPE")
            for name, v in tun.items():
                if shape == "warp":
                    assert v["threads"] == (0 if name == "m,n<=64" else base[name]["threads"])
                elif shape:
                    assert v["threads"] == int(shape)
                else:
                    # sampled: the faster candidate of the two took the rest of the bucket
                    assert v["how"] == "measured", (name, v)
                    assert v["rates"] and all(r > 0 for r in v["rates"].values())
                    best = max(v["rates"], key=v["rates"].get)
                    assert v["threads"] == (0 if best == "warp" else int(best))
        finally:
            h.close()
