"""Extract the twisted-bilayer eigenvalue pins from the reference's own test file.

Reads LatticeQM.jl's ``test/test_tbg.jl`` (its path is the required argument,
``python extract_reference_pins.py <LatticeQM.jl checkout>/test/test_tbg.jl``) and writes ``reference_pins.json`` beside this
script: for every ``@test isapprox(ev[...], value; atol=...)`` line in the
spectrum fixtures, the lattice, the k-point, the 1-based index expression, the
value, the tolerance and the source line.  Run once where the reference is
mounted; the JSON is committed so the tests need no reference checkout.
"""
import json
import os
import re
import sys

# (first line, last line) of each fixture block -> (lattice builder, N, k)
BLOCKS = [
    ((66, 80), ("honeycomb_twisted", 1, [0.0, 0.0])),
    ((83, 89), ("honeycomb_twisted", 1, [1 / 3, -1 / 3])),
    ((218, 220), ("honeycomb_twisted", 2, [0.0, 0.0])),
    ((221, 223), ("honeycomb_twisted", 2, [1 / 3, -1 / 3])),
    ((229, 231), ("honeycomb_twisted", 3, [0.0, 0.0])),
    ((245, 247), ("honeycomb_twisted_ABBA", 1, [0.0, 0.0])),
    ((253, 255), ("honeycomb_twisted_ABAB", 1, [0.0, 0.0])),
]
PAT = re.compile(r"isapprox\(\s*ev\w*\[([^\]]+)\]\s*,\s*([-+0-9.eE]+)\s*;\s*atol\s*=\s*([0-9.eE+-]+)\)")


def main(path):
    lines = open(path, encoding="utf-8").read().splitlines()
    pins = []
    for (a, b), (builder, N, k) in BLOCKS:
        for ln in range(a, b + 1):
            m = PAT.search(lines[ln - 1])
            if m:
                pins.append({"builder": builder, "N": N, "k": k, "index": m.group(1).strip(),
                             "value": float(m.group(2)), "atol": float(m.group(3)),
                             "source": f"test/test_tbg.jl:{ln}"})
    out = {"hopping": "Operators.graphene(lat; format=:dense, mode=:nospin, tz=0.32)", "pins": pins}
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_pins.json")
    with open(dst, "w") as f:
        json.dump(out, f, indent=1)
    print(f"{len(pins)} pins -> {dst}")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python extract_reference_pins.py <path to LatticeQM.jl>/test/test_tbg.jl")
    main(sys.argv[1])
