"""Extract the reference's golden Box-union-Plane fixture.

Reads tests/BooleanOperationExactZero/result.hpp of ViennaLS 5.8.3 (the only
golden fixture of the reference) and writes boolean_exact_zero.json: the HRLE
run list (start index, value) of Union(Plane, Box) after the boolean
operation's two Prune passes.  Run once where the reference is checked
out, with its root directory as the only argument; the JSON is committed.

    python make_boolean_exact_zero.py <path of the ViennaLS checkout>
"""
import json
import os
import re
import sys

if len(sys.argv) != 2:
    sys.exit("usage: make_boolean_exact_zero.py <path of the ViennaLS checkout>")
SRC = os.path.join(sys.argv[1], "tests", "BooleanOperationExactZero", "result.hpp")
text = open(SRC).read()
idx = re.findall(r"VectorType<double, 2>\{(-?\d+), (-?\d+)\}", text)
vals = [v.strip() for v in text.split("resultValues[] = {")[1].split("}")[0].split(",") if v.strip()]
assert len(idx) == len(vals)
runs = [{"index": [int(a), int(b)], "value": float(v)} for (a, b), v in zip(idx, vals)]
out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "boolean_exact_zero.json")
json.dump({"source": "tests/BooleanOperationExactZero/result.hpp", "runs": runs}, open(out, "w"), indent=0)
print("wrote", out, len(runs))
