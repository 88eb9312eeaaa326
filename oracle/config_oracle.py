"""Python restatement of the reference's canonical configuration text.

TEST INFRASTRUCTURE ONLY.  ``Lattice4::to_canonical_config`` (reference
crate QSOLKCB/YANG-MILLS, reference/rust/src/lib.rs:587-616) written with
Python string formatting, plus the same layout for SU(3) links
(18 words per link, the 3x3 matrix row-major, real then imaginary part).
The test-suite checks the engine's encoder against it byte for byte.
"""
import struct

SU2_CONFIG_FORMAT_ID = "YM-SU2-CONFIG-V1"   # lib.rs:23
SU3_CONFIG_FORMAT_ID = "YM-SU3-CONFIG-V1"


def _word(x: float) -> str:
    return "%016x" % struct.unpack("<Q", struct.pack("<d", float(x)))[0]


def to_canonical_config(format_id: str, extents, rows) -> str:
    """rows: one sequence of binary64 words per link, in link order."""
    out = [format_id, "extents=" + ",".join(str(int(e)) for e in extents), "link_count=%d" % len(rows)]
    out += [",".join(_word(w) for w in row) for row in rows]
    return "\n".join(out) + "\n"


def su2_rows(links):
    return [list(map(float, l)) for l in links]


def su3_rows(links):
    rows = []
    for m in links:
        row = []
        for r in range(3):
            for c in range(3):
                row += [float(m[r][c].real), float(m[r][c].imag)]
        rows.append(row)
    return rows
