"""Extract the reference's golden Box-union-Plane fixture.

Reads tests/BooleanOperationExactZero/result.hpp of ViennaLS 5.8.3 (the only
golden fixture of the reference) and writes boolean_exact_zero.json: the HRLE
run list (start index, value) of Union(Plane, Box) after the boolean
operation's two Prune passes.  Run once in a container that has the
reference checked out; the JSON is committed.
"""
import json
import os
import re
import sys

SRC = os.path.join(sys.argv[1] if len(sys.argv) > 1 else "/root/reference",
                   "tests", "BooleanOperationExactZero", "result.hpp")
text = open(SRC).read()
idx = re.findall(r"VectorType<double, 2>\{(-?\d+), (-?\d+)\}", text)
vals = [v.strip() for v in text.split("resultValues[] = {")[1].split("}")[0].split(",") if v.strip()]
assert len(idx) == len(vals)
runs = [{"index": [int(a), int(b)], "value": float(v)} for (a, b), v in zip(idx, vals)]
out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "boolean_exact_zero.json")
json.dump({"source": "tests/BooleanOperationExactZero/result.hpp", "runs": runs}, open(out, "w"), indent=0)
print("wrote", out, len(runs))
