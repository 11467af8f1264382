"""Writes pow5_table.inc: the 128-bit truncated powers of five that the CSV
reader's decimal -> binary float conversion multiplies by (the Eisel-Lemire
method: D. Lemire, "Number parsing at a gigabyte per second", Software:
Practice and Experience 51(8), 2021; the table with 128-bit entries needs no
slow path for decimals of up to 19 significant digits: N. Mushtak and
D. Lemire, "Fast number parsing without fallback", 2023).

Entry q (q in [-342, 308]) is 5^q scaled by a power of two to 128 bits with
its top bit set: 5^q truncated for q >= 0; for q < 0, floor(2^b / 5^-q) + 1
with b = bits(5^-q) + 127 (q >= -27) or 2 * bits(5^-q) + 128, then truncated
to its top 128 bits.  Exact integer arithmetic, run by build.py.

Usage: python pow5_table.py OUT.inc
"""

import sys

SMALLEST, LARGEST = -342, 308


def entries():
    out = []
    for q in range(SMALLEST, 0):
        p5 = 5 ** -q
        z = p5.bit_length()
        if q >= -27:
            c = (1 << (z + 127)) // p5 + 1
        else:
            c = (1 << (2 * z + 128)) // p5 + 1
            while c >= (1 << 128):
                c >>= 1
        out.append(c)
    for q in range(0, LARGEST + 1):
        p5 = 5 ** q
        while p5 < (1 << 127):
            p5 <<= 1
        while p5 >= (1 << 128):
            p5 >>= 1
        out.append(p5)
    return out


def main(path):
    mask = (1 << 64) - 1
    lines = [
        "// Generated by pow5_table.py: 128-bit powers of five for q in [%d, %d]," % (SMALLEST, LARGEST),
        "// two words per entry (high, low).",
        "constexpr int kPow5Smallest = %d;" % SMALLEST,
        "constexpr int kPow5Largest  = %d;" % LARGEST,
        "__device__ const unsigned long long kPow5Table[%d] = {" % (2 * (LARGEST - SMALLEST + 1)),
    ]
    for c in entries():
        lines.append("  0x%016xull, 0x%016xull," % (c >> 64, c & mask))
    lines.append("};")
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


if __name__ == "__main__":
    main(sys.argv[1])
