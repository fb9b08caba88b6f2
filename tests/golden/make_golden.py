"""Regenerate the golden fixtures of tests/golden from the reference tree.

Reads, as text, the reference's own committed test data and generated
tables (the Rust crate cannot be built here):

* crates/integral/tests/c2s_independent_reference.rs — the signed 60-digit
  mpmath c2s rows (C2S_SIGNED_REF) -> c2s_signed.json (l <= 4);
* crates/integral/src/math/rys_tables.rs — the Chebyshev Rys tables the
  reference interpolates at run time -> rys_tables.json: per n the number of
  subintervals, a SHA-256 of the coefficients (float64, little endian) and
  the first and last series of roots and weights.

Usage: python tests/golden/make_golden.py [reference_root]
"""
import hashlib
import json
import os
import re
import struct
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def parse_c2s(root):
    src = open(os.path.join(root, "crates/integral/tests/c2s_independent_reference.rs")).read()
    body = src[src.index("pub const C2S_SIGNED_REF"):]
    body = body[body.index("= &[") + 4:]
    rows = re.findall(r"&\[([^\[\]]*)\]", body)
    vals = [[float(x) for x in r.split(",") if x.strip()] for r in rows]
    out = {}
    k = 0
    for l in range(0, 7):
        n = 2 * l + 1
        if l <= 4:
            out[str(l)] = vals[k:k + n]
        k += n
    return out


def parse_rys(root):
    src = open(os.path.join(root, "crates/integral/src/math/rys_tables.rs")).read()
    out = {}
    for n in range(1, 14):
        ent = {}
        for kind in ("ROOT", "WEIGHT"):
            m = re.search(r"static %s_N%d: \[\[f64; NC\]; (\d+)\] = \[(.*?)\];" % (kind, n), src, re.S)
            series = [[float(x) for x in r.split(",") if x.strip()] for r in re.findall(r"\[([^\[\]]+)\]", m.group(2))]
            flat = [v for s in series for v in s]
            ent[kind.lower() + "_sha256"] = hashlib.sha256(struct.pack("<%dd" % len(flat), *flat)).hexdigest()
            ent[kind.lower() + "_first"] = series[0]
            ent[kind.lower() + "_last"] = series[-1]
            ent["n_sub"] = len(series) // n
        out[str(n)] = ent
    return out


def main():
    if len(sys.argv) < 2:
        raise SystemExit("usage: make_golden.py <reference root>")
    root = sys.argv[1]
    with open(os.path.join(HERE, "c2s_signed.json"), "w") as f:
        json.dump({"source": "crates/integral/tests/c2s_independent_reference.rs (C2S_SIGNED_REF)",
                   "rows": parse_c2s(root)}, f, indent=1)
    with open(os.path.join(HERE, "rys_tables.json"), "w") as f:
        json.dump({"source": "crates/integral/src/math/rys_tables.rs", "tables": parse_rys(root)}, f, indent=1)
    print("wrote c2s_signed.json, rys_tables.json")


if __name__ == "__main__":
    main()
