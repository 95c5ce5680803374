"""Generate coag_tables.inc: Whitby/CMAQ coagulation correction factors.

The three tables are published data (Whitby et al. 1991, as tabulated in
CMAQ v4.6) that the microphysics step indexes at run time:
  bm0ij[10][10][10]  0th-moment intermodal free-molecular correction
  bm3i[10][10][10]   3rd-moment intermodal free-molecular correction
  bm0[10]            0th-moment intramodal correction
The numbers must be identical to the ones mam4xx uses
(src/mam4xx/coagulation.hpp:81-285, 330-537, 588-591), so this script reads
them from the mam4xx source text and writes them as C initialisers with
round-trip precision. Run in a container that has the reference tree:
    python mam4xx_b200/csrc/gen_coag_tables.py /path/to/mam4xx
The generated file is committed; builds never read the reference tree.
"""

import os
import re
import sys


def _block(text, decl):
    i = text.index(decl)
    start = text.index("{", i)
    depth = 0
    for j in range(start, len(text)):
        if text[j] == "{":
            depth += 1
        elif text[j] == "}":
            depth -= 1
            if depth == 0:
                return text[start:j + 1]
    raise ValueError(decl)


def _numbers(block):
    return [float(t) for t in re.findall(r"[-+]?(?:\d+\.?\d*|\.\d+)(?:[eE][-+]?\d+)?", block)]


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"
    text = open(os.path.join(ref, "src/mam4xx/coagulation.hpp")).read()
    bm0ij = _numbers(_block(text, "const Real bm0ij[10][10][10]"))
    bm3i = _numbers(_block(text, "const Real bm3i[10][10][10]"))
    bm0 = _numbers(_block(text, "const Real bm0[10]"))
    assert len(bm0ij) == 1000 and len(bm3i) == 1000 and len(bm0) == 10
    here = os.path.dirname(os.path.abspath(__file__))
    out = os.path.join(here, "coag_tables.inc")

    def fmt(vals, per=6):
        lines = []
        for k in range(0, len(vals), per):
            lines.append("    " + ", ".join(repr(v) for v in vals[k:k + per]) + ",")
        return "\n".join(lines)

    with open(out, "w") as f:
        f.write("/* Generated by gen_coag_tables.py -- Whitby/CMAQ coagulation\n"
                " * correction factors, flattened [n1][n2a][n2n] (index\n"
                " * n1*100 + n2a*10 + n2n) and the 10 intramodal factors.\n"
                " * Define COAG_TABLE_QUALIFIER before including. */\n")
        f.write("#ifndef COAG_TABLE_QUALIFIER\n#define COAG_TABLE_QUALIFIER static const\n#endif\n")
        f.write("COAG_TABLE_QUALIFIER double kCoagBm0ij[1000] = {\n%s\n};\n" % fmt(bm0ij))
        f.write("COAG_TABLE_QUALIFIER double kCoagBm3i[1000] = {\n%s\n};\n" % fmt(bm3i))
        f.write("COAG_TABLE_QUALIFIER double kCoagBm0[10] = {\n%s\n};\n" % fmt(bm0))
    print("wrote", out)


if __name__ == "__main__":
    main()
