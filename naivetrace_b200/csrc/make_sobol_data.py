"""Writes tt_sobol_data.h: the two tables of the quasi-random sampler of the null-path tracer.

- Sobol direction-number parameters for dimensions 1..4095: the lines d = 2..4096 of the
  Joe-Kuo table the reference ships (misc/new-joe-kuo-5.21201; columns d, s, a, m_1..m_s).
  Dimension 0 is the van der Corput sequence.  The generator matrices are built from these
  at run time (tt_capi.cu, and separately in the oracle).  4096 dimensions cover every
  subsequence the tracer addresses: subsequence ids below 64, 64 dimensions each.
- The per-pixel Cranley-Patterson rotations, rotation_offsets[128 * 128][2] of the
  reference's src/sampler_tables.cxx, written with the same decimal literals so that they
  round to the same floats.

Usage: python make_sobol_data.py REFERENCE_ROOT   (the root of the reference's source tree)
"""
import re
import sys
from pathlib import Path

NUM_DIMS = 4096
BLOCK = 128


def main(argv):
    if len(argv) != 2:
        print(__doc__)
        return 2
    ref = Path(argv[1])
    lines = (ref / "misc" / "new-joe-kuo-5.21201").read_text().split("\n")
    sam = []
    for row in lines[1:NUM_DIMS]:
        f = [int(x) for x in row.split()]
        d, s, a, m = f[0], f[1], f[2], f[3:]
        assert len(m) == s and all(1 <= v < (1 << (i + 1)) and v % 2 == 1 for i, v in enumerate(m)), d
        sam.append([s, a] + m)
    assert len(sam) == NUM_DIMS - 1
    text = (ref / "src" / "sampler_tables.cxx").read_text()
    body = text[text.index("= //"):]
    pairs = re.findall(r"\{\s*([-+0-9.eE]+)\s*,\s*([-+0-9.eE]+)\s*\}", body)
    assert len(pairs) == BLOCK * BLOCK, len(pairs)
    out = [
        "// Generated by make_sobol_data.py; do not edit.",
        "// Sobol direction-number parameters of dimensions 1..4095 (Joe and Kuo, new-joe-kuo-5.21201,",
        "// lines d = 2..4096) and the per-pixel Cranley-Patterson rotations of the quasi-random",
        "// sampler (sampler_tables.cxx rotation_offsets).",
        "#pragma once",
        "#include <stdint.h>",
        "",
        f"#define TT_SOBOL_DIMS {NUM_DIMS}",
        f"#define TT_ROTATION_BLOCK {BLOCK}",
        "",
        "// Per dimension d = 1, 2, ...: s, a, m_1 .. m_s.",
        "static const uint16_t tt_sobol_sam[] = {",
    ]
    flat = [v for row in sam for v in row]
    for i in range(0, len(flat), 24):
        out.append("  " + ",".join(str(v) for v in flat[i:i + 24]) + ",")
    out.append("};")
    out.append("")
    out.append("// [128 * 128][2]: rotation of pixel (x % 128) + 128 * (y % 128).")
    out.append("static const float tt_rotation_offsets[] = {")
    for i in range(0, len(pairs), 8):
        out.append("  " + ",".join(f"{x}f,{y}f" for x, y in pairs[i:i + 8]) + ",")
    out.append("};")
    dst = Path(__file__).with_name("tt_sobol_data.h")
    dst.write_text("\n".join(out) + "\n")
    print(f"wrote {dst} ({len(flat)} direction-number entries, {len(pairs)} rotations)")
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv))
