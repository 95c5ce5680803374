"""Extract the known-answer vectors of mam4xx's own unit tests into JSON.

Reads the reference C++ test sources as text (they cannot be built here) and
writes small fixtures next to this script:

  gasaerexch_h2so4.json  30 vectors of the H2SO4 quasi-analytic update
                         (src/tests/mam4_gasaerexch_unit_tests.cpp:40-171)
  coag_tables.json       spot values of the bm0ij / bm3i correction tables
                         checked against Fortran
                         (src/tests/mam4_coagulation_unit_tests.cpp:22-59)

Run once in a container that has the reference tree:
    python tests/golden/extract_golden.py /path/to/mam4xx
The fixtures are committed; tests never read the reference tree.
"""

import json
import os
import re
import sys


def _array_block(text, name):
    """Return the brace-enclosed initialiser of `const Real name[...] = {...};`."""
    m = re.search(r"const Real %s(\[[^\]]*\])+\s*=\s*\{" % re.escape(name), text)
    if not m:
        raise KeyError(name)
    start = m.end() - 1
    depth = 0
    for i in range(start, len(text)):
        if text[i] == "{":
            depth += 1
        elif text[i] == "}":
            depth -= 1
            if depth == 0:
                return text[start : i + 1]
    raise ValueError("unbalanced braces for %s" % name)


def _nested(block):
    """Parse a C brace initialiser of numbers into nested Python lists."""
    tokens = re.findall(r"\{|\}|[-+]?(?:\d+\.?\d*|\.\d+)(?:[eE][-+]?\d+)?", block)
    stack = [[]]
    for t in tokens:
        if t == "{":
            stack.append([])
        elif t == "}":
            top = stack.pop()
            stack[-1].append(top)
        else:
            stack[-1].append(float(t))
    return stack[0][0]


def _scalar(text, name):
    m = re.search(r"const Real %s\s*=\s*([-+0-9.eE]+)\s*;" % re.escape(name), text)
    return float(m.group(1))


def extract_gasaerexch(ref):
    path = os.path.join(ref, "src/tests/mam4_gasaerexch_unit_tests.cpp")
    text = open(path).read()
    out = {"source": "src/tests/mam4_gasaerexch_unit_tests.cpp"}
    out["dts"] = _nested(_array_block(text, "dts"))
    out["qgas_netprod_otrproc"] = _scalar(text, "qgas_netprod_otrproc")
    for name in ["uptkaer", "in_qaer_cur", "out_qaer_cur", "out_qgas_avg",
                 "in_qgas_cur", "out_qgas_cur"]:
        out[name] = _nested(_array_block(text, name))
    # Catch2 Approx epsilon used there: 100 * FLT_EPSILON in double builds.
    out["rel_tol"] = 100 * 1.1920928955078125e-07
    return out


def extract_coag(ref):
    path = os.path.join(ref, "src/tests/mam4_coagulation_unit_tests.cpp")
    text = open(path).read()
    cases = []
    # blocks: n1 = ..; n2a = ..; n2n = ..; Real bm0ij_f = ..;  (or bm3i_f)
    pat = re.compile(
        r"n1\s*=\s*(\d+);\s*(?:int\s+)?n2a\s*=\s*(\d+);\s*(?:int\s+)?n2n\s*=\s*(\d+);"
        r"\s*(?:Real\s+)?(bm0ij|bm3i)_f\s*=\s*([-+0-9.eE]+);")
    for m in pat.finditer(re.sub(r"int\s+(n1|n2a|n2n)", r"\1", text)):
        cases.append({"table": m.group(4), "n1": int(m.group(1)),
                      "n2a": int(m.group(2)), "n2n": int(m.group(3)),
                      "value": float(m.group(5))})
    return {"source": "src/tests/mam4_coagulation_unit_tests.cpp",
            "abs_tol": 1.1920928955078125e-07, "cases": cases}


def main():
    # the mam4xx tree: first argument, else MAM4XX_REFERENCE, else the default checkout
    ref = (sys.argv[1] if len(sys.argv) > 1 else
           os.environ.get("MAM4XX_REFERENCE", "/root/reference"))
    here = os.path.dirname(os.path.abspath(__file__))
    g = extract_gasaerexch(ref)
    assert len(g["in_qgas_cur"]) == 3 and len(g["in_qgas_cur"][0]) == 10
    with open(os.path.join(here, "gasaerexch_h2so4.json"), "w") as f:
        json.dump(g, f, indent=1)
    c = extract_coag(ref)
    assert len(c["cases"]) == 4, c
    with open(os.path.join(here, "coag_tables.json"), "w") as f:
        json.dump(c, f, indent=1)
    print("wrote", len(g["in_qgas_cur"]) * 10, "gasaerexch vectors and",
          len(c["cases"]), "coag table cases")


if __name__ == "__main__":
    main()
