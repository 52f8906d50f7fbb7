"""The mixed policy's FP64 reciprocal (Newton-Raphson refinement of rcp.approx.ftz.f64,
grhd::rcp_mixed in physics.cuh) against CUDA's correctly rounded 1.0 / x.

tests/rcp_probe.cu includes the shipped header, so the function checked is the one the
mixed cell update runs.  The bound is one unit in the last place over 1.3e8 seeded
positive normal x in two exponent ranges.
"""
import os
import re
import subprocess
import tempfile

import pytest

from grhd_b200 import build

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "rcp_probe.cu")
INC = os.path.join(os.path.dirname(HERE), "grhd_b200", "csrc", "gpu")


def test_rcp_mixed_within_one_ulp():
    with tempfile.TemporaryDirectory() as d:
        exe = os.path.join(d, "rcp_probe")
        subprocess.run([build._nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-std=c++17",
                        "-I", INC, "-o", exe, SRC], check=True, capture_output=True, text=True)
        out = subprocess.run([exe], check=True, capture_output=True, text=True, timeout=120).stdout
    rows = re.findall(r"range (\d) emax (\d+) samples (\d+) max_ulp (\d+) max_rel (\S+)", out)
    assert len(rows) == 2, out
    for _, emax, _, ulp, rel in rows:
        assert int(ulp) <= 1, f"exponents within +-{emax}: {ulp} ulp ({out.strip()})"
        assert float(rel) <= 2.3e-16, out
