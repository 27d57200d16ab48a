"""Generate tests/golden/lattice.json from the reference's own lattice definition.

Reads src/solver/lattice.ts of the reference checkout (its root given by the REFERENCE_ROOT
environment variable, which is required), extracts the D2Q9 and D3Q19 velocity sets and weights from the `build(...)`
calls (lattice.ts:39-60), and derives opp / mirrorY / mirrorZ / mirrorYZ exactly as the
reference's `build` does (lattice.ts:20-37): index of the reflected velocity in the same list.

The JSON is committed; the tests read only the JSON, never the reference tree.
Run:  REFERENCE_ROOT=<reference checkout> python tests/golden/make_lattice_golden.py
"""
import json
import os
import re
from fractions import Fraction

REF = os.environ.get("REFERENCE_ROOT", "")
SRC = os.path.join(REF, "src", "solver", "lattice.ts") if REF else ""
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lattice.json")


def _eval_weights(expr: str):
    """Evaluate the TS weight array literal: fractions and `...Array(k).fill(a / b)` spreads."""
    out = []
    for item in [s.strip() for s in expr.split(",") if s.strip()]:
        m = re.fullmatch(r"\.\.\.Array\((\d+)\)\.fill\((\d+)\s*/\s*(\d+)\)", item)
        if m:
            out += [Fraction(int(m.group(2)), int(m.group(3)))] * int(m.group(1))
            continue
        m = re.fullmatch(r"(\d+)\s*/\s*(\d+)", item)
        if m:
            out.append(Fraction(int(m.group(1)), int(m.group(2))))
            continue
        raise ValueError(f"unparsed weight item {item!r}")
    return out


def parse(text: str, name: str):
    m = re.search(r"export const %s = build\((.*?)\n\);" % name, text, re.S)
    if not m:
        raise ValueError(f"{name} not found")
    body = m.group(1)
    vel = re.search(r"\[\s*(\[[-\d, \[\]\s]*\])\s*,\s*\]", body, re.S)
    c = [tuple(int(v) for v in t) for t in re.findall(r"\[(-?\d+),\s*(-?\d+),\s*(-?\d+)\]", vel.group(1))]
    wexpr = body[vel.end():]
    wm = re.search(r"\[(.*)\]", wexpr, re.S)
    w = _eval_weights(wm.group(1))
    assert len(c) == len(w), (name, len(c), len(w))

    def find(v):
        return c.index(tuple(v))

    return {
        "name": name,
        "q": len(c),
        "c": [list(t) for t in c],
        "w_num": [x.numerator for x in w],
        "w_den": [x.denominator for x in w],
        "opp": [find((-a, -b, -d)) for a, b, d in c],
        "mirrorY": [find((a, -b, d)) for a, b, d in c],
        "mirrorZ": [find((a, b, -d)) for a, b, d in c],
        "mirrorYZ": [find((a, -b, -d)) for a, b, d in c],
    }


def main():
    if not REF:
        raise SystemExit("set REFERENCE_ROOT to the root of the reference checkout")
    with open(SRC, encoding="utf-8") as fh:
        text = fh.read()
    data = {"source": "src/solver/lattice.ts:39-60", "D2Q9": parse(text, "D2Q9"), "D3Q19": parse(text, "D3Q19")}
    with open(OUT, "w", encoding="utf-8") as fh:
        json.dump(data, fh, indent=1)
    print("wrote", OUT)


if __name__ == "__main__":
    main()
