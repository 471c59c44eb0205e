#!/usr/bin/env python3
"""Writes joe_kuo_params.inc: the primitive-polynomial parameters (d, s, a, m_1..m_s) of the first
255 rows of the Joe & Kuo Sobol direction-number file (new-joe-kuo-6.21201, dimensions d = 2..256).

The reference builds its 256 x 32 direction-vector table from exactly these rows
(scripts/generate_luts_sobol.py:20-32 reads num_lines - 1 = 255 data rows; the table's last row
stays zero, corelib/internal/common/math/CMakeLists.txt:71-88 passes -d 256 -s 32).  The rows are
published third-party data; this script only re-formats them as a C initialiser so the device
sampler and the host code can expand them with their own recurrence.

Usage: python gen_joe_kuo_params.py <path to joe_kuo.txt>   (the reference ships it as
scripts/joe_kuo.txt).  The output is committed, so the build never needs the input file.
"""
import os
import sys

ROWS = 255


def main() -> None:
    if len(sys.argv) != 2:
        sys.exit("usage: gen_joe_kuo_params.py <path to joe_kuo.txt>")
    src = sys.argv[1]
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "joe_kuo_params.inc")
    lines = []
    with open(src) as f:
        f.readline()  # header
        for _ in range(ROWS):
            parts = f.readline().split()
            d, s, a = int(parts[0]), int(parts[1]), int(parts[2])
            m = [int(x) for x in parts[3:3 + s]]
            assert len(m) == s and s <= 12
            lines.append("  {%d, %d, %d, {%s}}," % (d, s, a, ", ".join(str(x) for x in m)))
    with open(out, "w") as f:
        f.write("/* Generated by gen_joe_kuo_params.py: Joe & Kuo (2008) primitive polynomials and initial\n"
                " * direction numbers, dimensions 2..256.  Fields: d, s (degree), a (coefficients), m_1..m_s. */\n")
        f.write("\n".join(lines) + "\n")
    print("wrote", out, len(lines), "rows")


if __name__ == "__main__":
    main()
