"""The reference's own phase test program, run on the GPU path.

oracle/_ref/test_eutectic_b200 is the reference's src/phase/test/test_eutectic.cpp
compiled unmodified against this library's C++ host layer
(include/mantle/phase/eutectic_rescaled.h over libmantlepar_b200), so its
known-answer, boundary-ownership, 10 000 seeded-state, derivative, scale and
exception checks run against the GPU kernels. The binary is built by
`make -C oracle ref-tests` where the reference sources are mounted.
"""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "oracle", "_ref", "test_eutectic_b200")

pytestmark = pytest.mark.gpu


@pytest.mark.skipif(not os.path.exists(BIN), reason="reference test program not built (make -C oracle ref-tests)")
def test_reference_phase_program_passes_on_gpu(cuda_lib):
    r = subprocess.run([BIN], capture_output=True, text=True, timeout=900)
    print(r.stdout)
    assert r.returncode == 0, (r.stdout[-2000:], r.stderr[-4000:])
    assert "FAIL" not in r.stderr
    assert r.stdout.count("PASS ") >= 5
