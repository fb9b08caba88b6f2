"""ORACLE build recipe — test infrastructure only.

Extracts the literal Chebyshev coefficients of the reference's Rys tables
(crates/integral/src/math/rys_tables.rs, read where it lies under the mounted
reference tree) into oracle/_ref/rys_tables.inc, a C include that the oracle
compiles in when present so its Rys interpolation uses exactly the numbers the
reference uses at run time.  The output is a build product: oracle/_ref/ is
git-ignored and never committed.

Usage: python oracle/extract_rys_tables.py [reference_root] [out_path]
"""
import os
import re
import sys


def parse(src, name):
    m = re.search(r"static %s: \[\[f64; NC\]; (\d+)\] = \[(.*?)\];" % name, src, re.S)
    if m is None:
        raise SystemExit("table %s not found" % name)
    rows = re.findall(r"\[([^\[\]]+)\]", m.group(2))
    return [[x.strip() for x in r.split(",") if x.strip()] for r in rows]


def main():
    if len(sys.argv) < 2:
        raise SystemExit("usage: extract_rys_tables.py <reference root> [<output .inc>]")
    root = sys.argv[1]
    here = os.path.dirname(os.path.abspath(__file__))
    out = sys.argv[2] if len(sys.argv) > 2 else os.path.join(here, "_ref", "rys_tables.inc")
    path = os.path.join(root, "crates", "integral", "src", "math", "rys_tables.rs")
    if not os.path.exists(path):
        print("reference Rys tables not found; the oracle will use its regenerated tables")
        return 0
    src = open(path).read()
    os.makedirs(os.path.dirname(out), exist_ok=True)
    lines = ["// generated from the reference's rys_tables.rs by extract_rys_tables.py"]
    nsubs = []
    for n in range(1, 14):
        R = parse(src, "ROOT_N%d" % n)
        W = parse(src, "WEIGHT_N%d" % n)
        assert len(R) == len(W) and len(R) % n == 0 and all(len(r) == 17 for r in R + W)
        nsubs.append(len(R) // n)
        lines.append("static const double REF_ROOT_N%d[] = {%s};" % (n, ",".join(v for r in R for v in r)))
        lines.append("static const double REF_WEIGHT_N%d[] = {%s};" % (n, ",".join(v for r in W for v in r)))
    lines.append("static const int REF_NSUB[13] = {%s};" % ",".join(map(str, nsubs)))
    lines.append("static const double* const REF_ROOT[13] = {%s};" % ",".join("REF_ROOT_N%d" % n for n in range(1, 14)))
    lines.append("static const double* const REF_WEIGHT[13] = {%s};" % ",".join("REF_WEIGHT_N%d" % n for n in range(1, 14)))
    with open(out, "w") as f:
        f.write("\n".join(lines) + "\n")
    print("wrote", out)
    return 0


if __name__ == "__main__":
    sys.exit(main())
