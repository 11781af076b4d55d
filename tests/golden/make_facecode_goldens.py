"""Extract the known-answer table of ``decode(facecode)`` into ``facecode_goldens.json``.

Run once, in a container that has the Raven.jl source tree; the output is committed.
It reads ``test/facecode.jl`` as text (nothing from the reference is executed).  That
file lists ``(code, value)`` pairs: UInt8 codes (two hex digits) decode to 4
hanging-face values, UInt16 codes (four hex digits) to 6 hanging-face and 12
hanging-edge values.

Usage: ``python tests/golden/make_facecode_goldens.py /path/to/Raven.jl``
"""

import json
import os
import re
import sys


def extract(root):
    path = os.path.join(root, "test", "facecode.jl")
    with open(path) as f:
        text = f.read()
    body = text[text.index("Any["):]
    tokens = re.findall(r"0x[0-9a-fA-F]+", body)
    out8, out16 = [], []
    i = 0
    while i < len(tokens):
        code = tokens[i]
        width = len(code) - 2
        if width == 2:
            vals = [int(v, 16) for v in tokens[i + 1:i + 5]]
            out8.append([int(code, 16), vals])
            i += 5
        elif width == 4:
            vals = [int(v, 16) for v in tokens[i + 1:i + 19]]
            out16.append([int(code, 16), vals[:6], vals[6:]])
            i += 19
        else:
            raise ValueError(f"unexpected literal {code} at token {i}")
    return {"source": "test/facecode.jl", "uint8": out8, "uint16": out16}


def main():
    if len(sys.argv) != 2:
        sys.exit(f"usage: python {os.path.basename(__file__)} <path of a Raven.jl checkout>")
    root = sys.argv[1]
    data = extract(root)
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "facecode_goldens.json")
    with open(dst, "w") as f:
        json.dump(data, f, separators=(",", ":"))
    print(f"{len(data['uint8'])} UInt8 and {len(data['uint16'])} UInt16 codes -> {dst}")


if __name__ == "__main__":
    main()
