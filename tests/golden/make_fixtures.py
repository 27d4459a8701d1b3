"""Regenerate the golden fixtures in this folder from the reference tree.

Run once in a checkout that has the reference mounted (default
``/root/reference``); the outputs are committed so that tests never read the
reference at run time.

* ``bench_<name>.test.gz`` -- the reference's golden product files
  (benchmark/*.test): three lines a, b, c = a*b of decimal coefficients, as
  read by benchmark/bench_two_convolution_poly_mul.cpp:128-160.  Copied
  byte-for-byte, gzip-compressed.
* ``unit_kats.json`` -- the known-answer cases written inline in
  unit_tests/test_two_convolution_poly_mul.cpp: bit widths (:9-54), limb
  splits (:56-78), x-argument scaling (:80-109) and the exact signed products
  (:112-193), parsed from the C++ text (commented-out cases are skipped).
"""
from __future__ import annotations

import gzip
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def _strip_comments(src: str) -> str:
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return "\n".join(line.split("//", 1)[0] for line in src.splitlines())


def _int_lists(s: str):
    return [[int(v) for v in re.findall(r"-?\d+", body)] for body in re.findall(r"\{([^{}]*)\}", s)]


def parse_unit_kats(path: str) -> dict:
    src = _strip_comments(open(path).read())
    out = {"bit_width": [], "limb_split": [], "scale_x": [], "products": []}

    def section(name):
        i = src.index(f"TEST(TwoConvolutionPolyMul, {name})")
        j = src.find("TEST(", i + 5)
        return src[i: j if j > 0 else len(src)]

    # bit widths: run_test(a, b, expected); hex and mpz_class literals included
    for m in re.finditer(r"UnivariateMPZPolynomial a = \{(.*?)\};\s*UnivariateMPZPolynomial b = \{(.*?)\};\s*run_test\(a, b, (\d+)\)",
                         section("FindLargestBitWidthOfCoefficients"), re.S):
        def vals(t):
            r = []
            for h, lit in re.findall(r'mpz_class\("([0-9a-fA-F]+)",\s*16\)|(-?0x[0-9a-fA-F]+|-?\d+)', t):
                r.append(int(h, 16) if h else int(lit, 0))
            return r
        out["bit_width"].append({"a": vals(m.group(1)), "b": vals(m.group(2)), "expected": int(m.group(3))})

    for m in re.finditer(r"UnivariateMPZPolynomial a = \{(.*?)\};\s*BivariateBase base = \{\.N = (\d+), \.K = (\d+), \.M = (\d+)\};\s*"
                         r"EXPECT_EQ\(convert_to_modular_bivariate\(a, base, (\d+)\), BivariateMPZPolynomial\(\{(.*?)\}\)\)",
                         section("ConvertToModularBivariate"), re.S):
        a = [int(t.strip(), 0) for t in m.group(1).split(",")]
        exp = [int(t.strip(), 0) for t in m.group(6).split(",")]
        out["limb_split"].append({"a": a, "N": int(m.group(2)), "K": int(m.group(3)), "M": int(m.group(4)),
                                  "prime": int(m.group(5)), "expected": exp})

    for m in re.finditer(r"BivariateMPZPolynomial A = \{(.*?)\};\s*BivariateBase base = \{\.N = (\d+), \.K = (\d+), \.M = (\d+)\};\s*"
                         r"sfixn theta = (\d+);\s*sfixn prime = (\d+);\s*EXPECT_EQ\(run_test\(A, base, theta, prime\), \(BivariateMPZPolynomial\{(.*?)\}\)\)",
                         section("ScaleXArgumentDev"), re.S):
        out["scale_x"].append({"A": [int(t) for t in m.group(1).split(",")], "K": int(m.group(3)),
                               "theta": int(m.group(5)), "prime": int(m.group(6)),
                               "expected": [int(t) for t in m.group(7).split(",")]})

    body = section("TwoConvolutionPolyMul")
    for m in re.finditer(r"run_test\(\s*(\{.*?\})\s*,\s*(\{.*?\})\s*,\s*(\{.*?\})\s*\);", body, re.S):
        a, b, c = (_int_lists(g)[0] for g in m.groups())
        out["products"].append({"a": a, "b": b, "c": c})
    return out


def main(ref_root: str = "/root/reference") -> None:
    bench = os.path.join(ref_root, "benchmark")
    names = sorted(f for f in os.listdir(bench) if f.endswith(".test"))
    # every fixed-width golden file and every big-coefficient file (n32 ... n1024:
    # 32 ... 1024 terms of as many bits; n1024 is 1.9 MB of text, 0.9 MB gzipped)
    keep = [f for f in names if "_p" in f or f in ("n32.test", "n64.test", "n128.test", "n256.test", "n512.test",
                                                   "n1024.test")]
    for f in keep:
        data = open(os.path.join(bench, f), "rb").read()
        with gzip.GzipFile(os.path.join(HERE, f"bench_{f}.gz"), "wb", mtime=0) as g:
            g.write(data)
    kats = parse_unit_kats(os.path.join(ref_root, "unit_tests", "test_two_convolution_poly_mul.cpp"))
    with open(os.path.join(HERE, "unit_kats.json"), "w") as fh:
        json.dump(kats, fh)
    print(f"{len(keep)} golden files; KATs: " + ", ".join(f"{k}={len(v)}" for k, v in kats.items()))


if __name__ == "__main__":
    main(*sys.argv[1:])
