"""Extract the unstructured coarse grids of the reference's grid tests into
``coarse_grid_fixtures.json``.

Run once, in a container that has the Raven.jl source tree; the output is committed.
It reads two test files as text (nothing from the reference is executed):
  * ``test/gridnumbering.jl``: the two-cell meshes whose second cell is listed in
    another vertex order, so that the shared face meets rotated (2 quadrilateral
    and 8 hexahedral orders), with the cell size N of each block;
  * ``test/grids.jl``: the two-cell meshes of the `generate` tests (one 2-D, one 3-D).
Each record holds the vertices, the list of cell tuples (1-based vertex ids) and N.

Usage: ``python tests/golden/make_coarse_goldens.py /path/to/Raven.jl``
"""

import json
import os
import re
import sys

SVEC = re.compile(r"SVector\{(\d),FT\}\(([^)]*)\)")
TUPLE = re.compile(r"\(([\d,\s]+)\)")


def _vertices(block):
    out = []
    for dim, args in SVEC.findall(block):
        vals = [float(v) for v in args.split(",")]
        if len(vals) != int(dim):
            raise ValueError(f"bad vertex {args}")
        out.append(vals)
    return out


def _tuples(block):
    return [[int(v) for v in t.split(",")] for t in TUPLE.findall(block)]


def _bracket(text, start):
    """The text of the bracketed list opening at text[start] == '['."""
    depth = 0
    for i in range(start, len(text)):
        if text[i] == "[":
            depth += 1
        elif text[i] == "]":
            depth -= 1
            if depth == 0:
                return text[start:i + 1]
    raise ValueError("unbalanced brackets")


def _strip_comments(text):
    return "\n".join(line.split("#", 1)[0] for line in text.splitlines())


def extract(root):
    records = []
    path = os.path.join(root, "test", "gridnumbering.jl")
    with open(path) as f:
        text = _strip_comments(f.read())
    for m in re.finditer(r"for cells in \[", text):
        cells_block = _bracket(text, m.end() - 1)
        head = text[:m.start()]
        v0 = head.rindex("vertices = [")
        verts = _vertices(_bracket(head, v0 + len("vertices = [") - 1))
        n = int(re.findall(r"\bN = (\d+)", head)[-1])
        for group in re.findall(r"\[(\([^\[\]]*\))\]", cells_block):
            records.append({"source": "test/gridnumbering.jl", "N": n, "vertices": verts, "cells": _tuples(group)})
    path = os.path.join(root, "test", "grids.jl")
    with open(path) as f:
        text = _strip_comments(f.read())
    for m in re.finditer(r"cells = \[", text):
        head = text[:m.start()]
        v0 = head.rindex("vertices = [")
        vblock = _bracket(head, v0 + len("vertices = [") - 1)
        if "SVector{" not in vblock:
            continue
        cm = re.findall(r"LobattoCell\{FT,AT\}\(([\d,\s]+)\)", head)[-1]
        n = int(cm.split(",")[0])
        records.append({"source": "test/grids.jl", "N": n, "vertices": _vertices(vblock),
                        "cells": _tuples(_bracket(text, m.end() - 1))})
    return records


def main(argv):
    if len(argv) != 2:
        print(__doc__.strip().splitlines()[-1], file=sys.stderr)
        return 2
    recs = extract(argv[1])
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "coarse_grid_fixtures.json")
    with open(out, "w") as f:
        json.dump({"records": recs}, f, indent=1)
    print(f"wrote {len(recs)} meshes to {out}")
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv))
