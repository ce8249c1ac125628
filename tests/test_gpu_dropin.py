"""The C++ drop-in header against the reference itself: the reference's
GradientPhiGaussDolfyn / FluxMassDolfynFaceLoop templates and
cupcfd::fvm::gpu's, called with identical argument lists on the reference's
own EuclideanVector arrays, must agree bit for bit (tests/cpp/dropin_demo.cpp,
built by `make -C oracle dropin` where the reference sources exist)."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "oracle", "_ref", "dropin_demo")

pytestmark = pytest.mark.gpu


@pytest.mark.skipif(not os.path.exists(BIN), reason="drop-in demo not built (needs the reference sources)")
@pytest.mark.parametrize("n", [3, 12, 33])
def test_dropin_matches_reference_kernels(gpu, n):
    r = subprocess.run([BIN, str(n)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.startswith("OK dropin")
