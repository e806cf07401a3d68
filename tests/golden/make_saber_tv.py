"""Generate tests/golden/saber_l3_tv.npz from the reference's only known-answer fixture.

The reference (DPCrypto) ships one fixture, SABER-GPU/include/tv.h: a Saber (l=3)
keypair with GenMatrix output, encaps coins, the message and the encaps secret.
This script parses those C array initialisers as data and stores them as numpy
arrays, so the tests never need the reference tree at run time.

Run where the reference tree is present, giving the path of its tv.h:
    python tests/golden/make_saber_tv.py <reference>/SABER-GPU/include/tv.h
"""
import os
import re
import sys

import numpy as np


def parse(path: str) -> dict:
    text = open(path).read()
    out = {}
    for m in re.finditer(r"(uint8_t|uint16_t)\s+(\w+)\s*\[[^\]]*\]\s*=\s*\{([^}]*)\}", text):
        ctype, name, body = m.groups()
        vals = [int(v, 0) for v in body.replace("\n", " ").split(",") if v.strip()]
        out[name] = np.array(vals, dtype=np.uint8 if ctype == "uint8_t" else np.uint16)
    return out


def main() -> None:
    if len(sys.argv) != 2:
        sys.exit("usage: make_saber_tv.py <path of SABER-GPU/include/tv.h>")
    src = sys.argv[1]
    arrays = parse(src)
    expected = {"A": 2304, "sp": 768, "pk": 992, "m_tv": 32, "sk_tv": 2304, "buf_tv": 64}
    for k, n in expected.items():
        assert k in arrays and arrays[k].size == n, (k, arrays.get(k, np.zeros(0)).size)
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "saber_l3_tv.npz")
    np.savez_compressed(dst, A=arrays["A"], sp=arrays["sp"], pk=arrays["pk"],
                        m=arrays["m_tv"].astype(np.uint8), sk=arrays["sk_tv"], buf=arrays["buf_tv"])
    print("wrote", dst)


if __name__ == "__main__":
    main()
