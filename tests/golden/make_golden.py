"""Regenerate tests/golden/validation_golden.json from the reference's own results.

Reads the CSV files written by the reference's physics validation suite
(ChannelFlow.jl validation/results/{decay,ts_convergence,ts_history,waleffe}.csv,
produced by validation/viscous_decay.jl, validation/tollmien_schlichting.jl
and validation/waleffe_equilibrium.jl) and stores them as a small JSON
fixture, so that the tests can pin the oracle without the reference checkout.
Run from the repository root with the path of a ChannelFlow.jl checkout:

    python tests/golden/make_golden.py /path/to/ChannelFlow.jl
"""
import csv
import json
import os
import sys

if len(sys.argv) != 2:
    sys.exit("usage: make_golden.py /path/to/ChannelFlow.jl")
src = sys.argv[1]
out = {"source": "ChannelFlow.jl validation/results (reference run outputs)"}
for name in ("decay", "ts_convergence", "ts_history", "waleffe"):
    with open(os.path.join(src, "validation", "results", name + ".csv")) as f:
        rows = list(csv.DictReader(f))
    conv = []
    for r in rows:
        conv.append({k: (v if k in ("flow", "branch") else float(v)) for k, v in r.items()})
    out[name] = conv
dest = os.path.join(os.path.dirname(os.path.abspath(__file__)), "validation_golden.json")
with open(dest, "w") as f:
    json.dump(out, f, indent=1)
print("wrote", dest)
