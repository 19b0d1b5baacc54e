"""Regenerate tests/golden/p1_constants.json from the reference's P1 known-answer
constants (hardware/u55c/hls/include/par1_ckks_hls_constants.hpp and
par1_bfv_hls_constants.hpp).  Those headers are the only in-tree values that
Lattigo v2.3.0 itself produced for this path (exported by
software/mkf/mkf_cpu/fpga_constants_test.go:114-240).  Run from the repository
root with the path of a checkout of the reference:

    python tests/golden/make_golden.py REFERENCE
"""
import json
import os
import re
import sys



def header_dir(ref):
    return os.path.join(ref, "hardware", "u55c", "hls", "include")


def parse(path):
    text = open(path).read()
    out = {}
    for m in re.finditer(r"static const ap_uint<64>\s+(\w+)((?:\[[^\]]+\])+)\s*=\s*(\{.*?\});", text, re.S):
        name, body = m.group(1), m.group(3)
        nums = [int(x) for x in re.findall(r"(\d+)ULL", body)]
        dims = re.findall(r"\[([^\]]+)\]", m.group(2))
        out[name] = {"dims": dims, "values": nums}
    for m in re.finditer(r"static constexpr unsigned(?: long long)?\s+(\w+)\s*=\s*(\d+)", text):
        out[m.group(1)] = int(m.group(2))
    return out


def main():
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py REFERENCE")
    hdr = header_dir(sys.argv[1])
    ckks = parse(os.path.join(hdr, "par1_ckks_hls_constants.hpp"))
    bfv = parse(os.path.join(hdr, "par1_bfv_hls_constants.hpp"))
    doc = {
        "source": "hardware/u55c/hls/include/par1_{ckks,bfv}_hls_constants.hpp",
        "ckks": ckks,
        "bfv": bfv,
    }
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "p1_constants.json")
    with open(dst, "w") as f:
        json.dump(doc, f, indent=1, sort_keys=True)
    print("wrote", dst)


if __name__ == "__main__":
    main()
