"""A C program compiled against the reference's own header (hmat/hmat.h of hmat-oss) and linked
against libhmat_b200.so runs unchanged (tests/c/dropin.c): clustering, block tree, get_info and
the refusal of a host callback without a GPU; the same through the table forwarder of
INTEGRATION.md (HMAT_ENGINE=b200); and, on the GPU, assembly and gemv 'N' / 'T' in FP64 and in
the mixed engine against the dense kernel product.

The program is built by tests/c/Makefile (REF = the reference source tree) into tests/c/_bin/;
where the reference tree is absent the prebuilt binary is used."""
import os
import subprocess

import pytest
from conftest import ROOT

BIN = os.path.join(ROOT, "tests", "c", "_bin", "dropin")


def _binary():
    ref = os.environ.get("HMAT_REFERENCE_SRC")
    if ref and os.path.isdir(os.path.join(ref, "include", "hmat")):
        subprocess.run(["make", "-C", os.path.join(ROOT, "tests", "c"), f"REF={ref}"], check=True,
                       capture_output=True)
    if not os.path.exists(BIN):
        pytest.skip("tests/c/_bin/dropin is not built (set HMAT_REFERENCE_SRC to build it)")
    return BIN


def _run(mode, **env):
    r = subprocess.run([_binary(), mode], capture_output=True, text=True, env=dict(os.environ, **env), timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert f"dropin {mode} ok" in r.stdout
    return r.stdout


def test_reference_header_program_host_part():
    _run("host")


def test_reference_header_program_through_the_forwarder():
    _run("forward", HMAT_ENGINE="b200")


@pytest.mark.gpu
def test_reference_header_program_assembles_and_multiplies():
    out = _run("gpu")
    assert "FP64 gemv 'N'" in out and "mixed gemv 'T'" in out
