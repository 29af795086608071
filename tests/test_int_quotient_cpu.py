"""The integer time-axis evaluation (T = arange) takes the segment quotients
A = (x1-t)/h and B = (t-x0)/h as RN(a*y) plus one Markstein correction, with
y = RN(1/h) from a table.  That equals the IEEE division for every integer
pair 0 <= a <= h <= 65536 (spacings of traces up to 32768 samples): checked
here exhaustively, bit for bit, on the host's IEEE double arithmetic (the
same correctly rounded mul / fma / div as the GPU's)."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs gcc")
def test_one_markstein_step_is_exact_for_integer_quotients(tmp_path):
    exe = str(tmp_path / "int_quotient")
    subprocess.run(["gcc", "-O2", "-ffp-contract=off", "-o", exe,
                    os.path.join(HERE, "c", "int_quotient.c"), "-lm"], check=True)
    out = subprocess.run([exe, "65536"], check=True, capture_output=True, text=True).stdout.split()
    n, pairs, bad1, bad0 = (int(v) for v in out)
    assert n == 65536 and pairs == 65537 * 65538 // 2 - 1
    assert bad1 == 0
    assert bad0 > 0          # the bare product is not enough: the correction matters
