"""Regenerate tests/golden/diffraction_ref.json from the reference's fixture.

The reference (physwkim/xrt-rs) pins its Kirchhoff integral with one fixture,
validation/fixtures/diffraction_ref.json: 5 rays x 3 pixels at 10 keV and
z = 1000 mm, with expected (Es, Ep) per pixel. Its Rust test
tests/golden_diffraction.rs:119-188 and Python test
validation/test_diffraction.py:36-59 compare against it at abs 1e-10.

This script copies the numeric content (inputs and expected outputs, nothing
else) into tests/golden/ so the suite does not need the reference checkout at
run time.

    python tests/golden/make_golden.py path/to/xrt-rs/validation/fixtures/diffraction_ref.json
"""
import json
import os
import sys

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "diffraction_ref.json")


def main(src: str) -> None:
    with open(src) as f:
        fix = json.load(f)
    cases = []
    for tc in fix["test_cases"]:
        cases.append({
            "id": tc["id"],
            "rays": tc["rays"],
            "pixels": tc["pixels"],
            "expected": tc["expected"],
        })
    out = {
        "source": "physwkim/xrt-rs validation/fixtures/diffraction_ref.json",
        "tolerance_abs": 1e-10,
        "tolerance_source": "tests/golden_diffraction.rs:119-188",
        "test_cases": cases,
    }
    with open(OUT, "w") as f:
        json.dump(out, f, indent=1)
    print(f"wrote {OUT} ({len(cases)} case(s))")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_golden.py path/to/validation/fixtures/diffraction_ref.json")
    main(sys.argv[1])
