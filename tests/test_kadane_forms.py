"""The reduced Kadane forms the RFI scan kernels run (KadaneState32 and
KadanePair32, the states of u and -u together, in the time scan,
KadaneBest in the frequency scan; frost_b200/csrc/rfi_types.hpp,
host-compiled) agree with the full KadaneState append field for field on
200 000 random sequences (exact zero sums, ties, gaps in the positions); the
GPU RFI parity tests check the kernels against frost's own cleaner."""

import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reduced_kadane_forms_match_the_full_state(tmp_path):
    exe = str(tmp_path / "kadane_forms_test")
    subprocess.run(["g++", "-O2", "-std=c++20", "-ffp-contract=off",
                    "-I" + os.path.join(ROOT, "frost_b200", "csrc"), "-I" + os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "kadane_forms_test.cpp"), "-o", exe], check=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout
    assert "bad 0" in r.stdout
