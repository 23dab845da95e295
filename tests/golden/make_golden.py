"""Regenerates the committed golden fixtures in tests/golden/.

Run here, where the reference sources are present:
    python tests/golden/make_golden.py [--reference /root/reference]

* iqrm_golden.json — the IQRM known-answer vector and expected flag lists,
  read as text from the reference's own test
  (tests/cpp/api/rfi_test.cpp:213-257).
* dm_lists.npz — generate_dm_list of the reference (lib/dedisp/dedisp.cpp)
  for the benchmark observing setups and the reference's dedisp test setup.
* rfi_cases.json — for small seeded blocks (frost_b200.synth), SHA-256
  digests of the reference cleaner's execute_normalized output and channel
  mask, plus its report, from oracle/_ref/libfrost_ref.so (strict IEEE
  build). The GPU parity tests regenerate the same inputs from the seeds.
"""

from __future__ import annotations

import argparse
import hashlib
import json
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from frost_b200.config import DedispPlanConfig  # noqa: E402
from tests.rfi_cases import CASES, make_case  # noqa: E402


def iqrm_from_reference(ref_root: str) -> dict:
    text = open(os.path.join(ref_root, "tests/cpp/api/rfi_test.cpp")).read()
    start = text.index('TEST_CASE("iqrm_mask matches Morello')
    body = text[start:start + 6000]
    vec = body[body.index("std::vector<float> x = {") : body.index("};")]
    values = [float(v.rstrip("F")) for v in re.findall(r"-?\d+\.\d+F", vec)]
    cases = []
    pat = re.compile(
        r"CHECK\(flagged\(iqrm_mask\(x, (\d+), ([\d.]+)F(?:, ignore_of\(\{([\d, ]+)\}\))?\)\) ==\s*"
        r"std::vector<SizeType>\{([\d, ]+)\}\);")
    for m in pat.finditer(body):
        ignore = [int(v) for v in m.group(3).split(",")] if m.group(3) else []
        expected = [int(v) for v in m.group(4).split(",")]
        cases.append({"radius": int(m.group(1)), "threshold": float(m.group(2)),
                      "ignore": ignore, "expected": expected})
    assert len(values) == 64 and len(cases) == 4, (len(values), len(cases))
    return {"source": "tests/cpp/api/rfi_test.cpp:213-257", "x": values, "cases": cases}


DM_SETUPS = {
    # name: (nchans, dt, f0, df, dm_min, dm_max, pulse_width_us)
    "config1": (1024, 64e-6, 1500.0, -0.29296875, 0.0, 500.0, 40.0),
    "config2": (4096, 64e-6, 1535.958984375, -0.08203125, 0.0, 2000.0, 40.0),
    "dedisp_test": (16, 1e-3, 1400.0, -1.0, 0.0, 50.0, 1000.0),
    "calibration": (32, 1e-3, 800.0, 8.0, 0.0, 100.0, 1000.0),
}


def digest(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default="/root/reference")
    args = ap.parse_args()
    from oracle import ref

    with open(os.path.join(HERE, "iqrm_golden.json"), "w") as f:
        json.dump(iqrm_from_reference(args.reference), f, indent=1)

    lists = {}
    for name, (n, dt, f0, df, lo, hi, pw) in DM_SETUPS.items():
        cfg = DedispPlanConfig(nchans=n, dt=dt, f0=f0, df=df, dm_min=lo, dm_max=hi,
                               dm_pulse_width=pw, dm_tol=1.25)
        lists[name] = ref.generate_dm_list(cfg)
    np.savez(os.path.join(HERE, "dm_lists.npz"), **lists)

    cases = {}
    for name in CASES:
        cfg, layout, baseline, blocks = make_case(name)
        cleaner = ref.RefRFICleaner(cfg, layout, baseline)
        steps = []
        for block, nsamps in blocks:
            out = cleaner.execute_normalized(block, nsamps)
            steps.append({"out_sha256": digest(out), "mask_sha256": digest(cleaner.channel_mask()),
                          "report": {k: v for k, v in cleaner.report().items()
                                     if not k.startswith("t_")}})
        cases[name] = steps
    with open(os.path.join(HERE, "rfi_cases.json"), "w") as f:
        json.dump(cases, f, indent=1, sort_keys=True)
    print("wrote", sorted(os.listdir(HERE)))


if __name__ == "__main__":
    main()
