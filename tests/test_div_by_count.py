"""The two-term-reciprocal division of the Welford kernel
(WelfordAcc::step_recip in frost_b200/csrc/rfi_kernels.cu) restated in C and
compared bit for bit with IEEE double division on 30 M random operands and
counts up to 262 144 (and up to 2^32 for one operand in eleven); the GPU RFI
parity tests check the kernel itself."""

import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_division_by_count_is_correctly_rounded(tmp_path):
    exe = str(tmp_path / "div_by_count_test")
    subprocess.run(["gcc", "-O2", "-ffp-contract=off", os.path.join(ROOT, "tests", "cpp", "div_by_count_test.c"),
                    "-lm", "-o", exe], check=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout
    assert "bad 0" in r.stdout
