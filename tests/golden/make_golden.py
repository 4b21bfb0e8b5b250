"""Regenerates the golden fixtures of tests/golden/ from the reference source text.

    python tests/golden/make_golden.py REFERENCE_ROOT

The reference cannot be compiled in this environment (its third-party dependencies are
absent), so the only fixtures that can be taken from it are numbers written in its source:
the binned-spectrum tables (src/spectral.cxx:14-34), the sun spectrum (src/light.hxx:260),
the wavelength bin centres (src/spectral.hxx:37-41), the PCG32 default state and stream
constants the reference seeds with, and the known answers asserted by its unit tests
(src/tests.cxx).  The fixtures are committed; the tests never read the reference tree.
"""
from __future__ import annotations

import json
import re
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent


def numbers(text: str):
    return [float(x) for x in re.findall(r"-?\d+\.\d+(?:[eE][-+]?\d+)?", text)]


def block(text: str, start_pat: str) -> str:
    m = re.search(start_pat, text)
    if not m:
        raise SystemExit(f"pattern not found: {start_pat}")
    i = text.index("{", m.end() - 1)
    depth = 0
    for j in range(i, len(text)):
        if text[j] == "{":
            depth += 1
        elif text[j] == "}":
            depth -= 1
            if depth == 0:
                return text[i:j + 1]
    raise SystemExit("unbalanced braces")


def main(root: str) -> int:
    src = Path(root) / "src"
    spectral = (src / "spectral.cxx").read_text()
    spectral_h = (src / "spectral.hxx").read_text()
    light_h = (src / "light.hxx").read_text()
    tests = (src / "tests.cxx").read_text()
    smits = numbers(block(spectral, r"static const double spectra\[7\]\[NBINS\]\s*="))
    m = numbers(block(spectral, r"static const double mat_spectrum_to_rgb\[3\]\[NBINS\]\s*="))
    wl = numbers(block(spectral_h, r"static const Scalar wavelengths\[NBINS\]\s*="))
    sun_line = re.search(r"emission_spectrum <<(.*?);", light_h, re.S).group(1)
    sun = numbers(sun_line)
    assert len(smits) == 7 * 36 and len(m) == 3 * 36 and len(wl) == 36 and len(sun) == 36
    # Known answers of the spectral unit tests (tests.cxx:255-327).
    trials = re.findall(r"\{\s*([0-9.]+)_rgb,\s*([0-9.]+)_rgb,\s*([0-9.]+)_rgb\s*\}", tests)
    rgb_trials = [[float(a), float(b), float(c)] for a, b, c in trials[:10]]
    out = {
        "source": "reference src/spectral.cxx, src/spectral.hxx, src/light.hxx, src/tests.cxx",
        "smits_basis": [smits[36 * i:36 * (i + 1)] for i in range(7)],
        "spectrum_to_rgb": [m[36 * i:36 * (i + 1)] for i in range(3)],
        "wavelengths": wl,
        "sun_spectrum": sun,
        "rgb_round_trip_trials": rgb_trials,
        "rgb_round_trip_tolerance": 1.3e-2,
        "pcg32_default_state": "0x853c49e6748fea9b",
        "pcg32_default_stream": "0xda3e39cb94b95bdb",
    }
    (HERE / "spectral_tables.json").write_text(json.dumps(out, indent=1))
    print("wrote", HERE / "spectral_tables.json")
    return 0


if __name__ == "__main__":
    if len(sys.argv) != 2:
        print("usage: python make_golden.py REFERENCE_ROOT")
        sys.exit(2)
    sys.exit(main(sys.argv[1]))
