"""Extract the CUDA source held in the `krnl` string of a reference Python
module (cpab/gpu/expm/expm_affine_by_series_{2D,3D}.py) into a file, so that
oracle/ref_expm.cpp can compile it as host code.

TEST INFRASTRUCTURE ONLY.  Usage: python extract_krnl.py <src.py> <out.inc>
"""
import re
import sys


def extract(src_path: str) -> str:
    text = open(src_path, encoding="latin-1").read()
    m = re.search(r'^krnl\s*=\s*"""(.*?)"""', text, re.S | re.M)
    if m is None:
        raise SystemExit(f"no krnl string in {src_path}")
    return m.group(1)


if __name__ == "__main__":
    body = extract(sys.argv[1])
    with open(sys.argv[2], "w") as f:
        f.write(body)
