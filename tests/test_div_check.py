"""FastDiv (hormone_b200/csrc/hmn_div.cuh) against IEEE division on the GPU.

tests/div_check.cu, compiled here with the library's FP64 flags, draws 2^24
operand pairs in each of six families (random over the checked exponent
range, the range limits, significands with long runs of ones or zeros, b a
power of two, a = +-0, nearly equal operands) and requires every reciprocal
and quotient that FastDiv does not flag to equal IEEE division bit for bit.
The stage kernels recompute a slope, face or cell with IEEE division
wherever a flag is raised, so this is the property their bitwise parity
rests on."""
import os
import subprocess

import pytest

from hormone_b200 import build

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))


def test_fastdiv_equals_ieee_division(tmp_path):
    exe = str(tmp_path / "div_check")
    subprocess.run([build.nvcc(), *build.ARCH, "-O3", "-std=c++17", "--fmad=false", "-I", build.CSRC,
                    os.path.join(HERE, "div_check.cu"), "-o", exe], check=True)
    r = subprocess.run([exe, str(1 << 24), "20261203"], capture_output=True, text=True)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    lines = [l for l in r.stdout.splitlines() if "pairs=" in l]
    assert len(lines) == 6
    stats = {l.split()[0]: dict(kv.split("=") for kv in l.split()[1:]) for l in lines}
    for fam, st in stats.items():
        assert int(st["mismatches"]) == 0, (fam, st)
    # the flag is rare where operands lie inside the checked range
    for fam in ("random", "runs_of_ones_or_zeros", "b_power_of_two", "a_zero", "nearly_equal"):
        assert int(stats[fam]["flagged"]) < int(stats[fam]["pairs"]) // 10, (fam, stats[fam])
