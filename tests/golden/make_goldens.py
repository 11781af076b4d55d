"""Extract the reference's own known-answer values into ``reference_goldens.json``.

This script is run once, in a container that has the Raven.jl source tree, and its
output is committed.  It reads the reference's test files as text (nothing from the
reference is executed) and records:

* every ``expected_error[<form>, <level>] = <value>`` entry of the balance-law
  convergence tests (``test/balancelaws/{advection,euler}/*.jl``), with the
  file, line and relative tolerance the reference test applies (``≈`` defaults to
  ``rtol = sqrt(eps)``; some files pass ``rtol = 10sqrt(eps(FT))``);
* the two golden ``vmapP`` vectors of the 1-element periodic bricks in
  ``test/gridnumbering.jl``.

Usage: ``python tests/golden/make_goldens.py /path/to/Raven.jl``
"""

import json
import os
import re
import sys

EPS = 2.0 ** -52


def _form_key(text):
    text = text.strip()
    if text.startswith("WeakForm"):
        return "weak"
    m = re.match(r"FluxDifferencingForm\((\w+)\(\)\)", text)
    if not m:
        raise ValueError(f"unknown volume form {text!r}")
    return {
        "CentralFlux": "fd_central",
        "EntropyConservativeFlux": "fd_ec",
        "KennedyGruberFlux": "fd_kg",
    }[m.group(1)]


def extract_errors(root):
    out = []
    for law in ("advection", "euler"):
        d = os.path.join(root, "test", "balancelaws", law)
        for fname in sorted(os.listdir(d)):
            if not fname.endswith(".jl"):
                continue
            path = os.path.join(d, fname)
            with open(path) as f:
                lines = f.read().split("\n")
            text = "\n".join(lines)
            rtol = 10.0 * EPS ** 0.5 if "rtol = 10sqrt(eps(FT))" in text else EPS ** 0.5
            i = 0
            while i < len(lines):
                line = lines[i]
                m = re.match(r"\s*expected_error\[(.*),\s*(\d+)\]\s*=\s*(\S*)\s*$", line)
                if m:
                    value = m.group(3)
                    lineno = i + 1
                    if value == "":
                        i += 1
                        value = lines[i].strip()
                    out.append(
                        {
                            "law": law,
                            "test": fname[:-3],
                            "form": _form_key(m.group(1)),
                            "level": int(m.group(2)),
                            "expected": float(value),
                            "rtol": rtol,
                            "source": f"test/balancelaws/{law}/{fname}:{lineno}",
                        }
                    )
                i += 1
    return out


def extract_vmapP(root):
    path = os.path.join(root, "test", "gridnumbering.jl")
    with open(path) as f:
        lines = f.read().split("\n")
    out = []
    for i, line in enumerate(lines):
        m = re.search(r"LobattoCell\(([\d, ]+)\)", line)
        if not m or "cell = " not in line:
            continue
        nq = [int(x) for x in m.group(1).split(",")]
        # the brick call and the vmapP literal follow within a few lines
        for j in range(i + 1, min(i + 10, len(lines))):
            if "fm.vmapP ==" in lines[j]:
                lit = lines[j].split("==", 1)[1]
                k = j
                while ";;]" not in lit:
                    k += 1
                    lit += lines[k]
                nums = [int(x) for x in re.findall(r"-?\d+", lit.split(";;]")[0])]
                brick = re.search(r"brick\(\(([\d, ]+)\),\s*\(([^)]*)\)\)", " ".join(lines[i:j]))
                out.append(
                    {
                        "dim": len(nq),
                        "nq": nq[0],
                        "elements_per_side": [int(x) for x in brick.group(1).split(",")],
                        "periodic": [x.strip() == "true" for x in brick.group(2).split(",")],
                        "vmapP": nums,
                        "source": f"test/gridnumbering.jl:{j + 1}",
                    }
                )
                break
    return out


def main():
    if len(sys.argv) != 2:
        sys.exit(f"usage: python {os.path.basename(__file__)} <path of a Raven.jl checkout>")
    root = sys.argv[1]
    data = {
        "generator": "tests/golden/make_goldens.py",
        "errors": extract_errors(root),
        "vmapP": extract_vmapP(root),
    }
    here = os.path.dirname(os.path.abspath(__file__))
    with open(os.path.join(here, "reference_goldens.json"), "w") as f:
        json.dump(data, f, indent=1)
    print(f"{len(data['errors'])} error goldens, {len(data['vmapP'])} vmapP goldens")


if __name__ == "__main__":
    main()
