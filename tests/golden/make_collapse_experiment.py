"""Writes collapse_2d_experiment.json: the laboratory free surface and failure
line of the 2D granular column collapse that MaterialPointSolver.jl ships with
its validation case (docs/assets/data/2d_collapse_experiments/surface.csv and
failure.csv of the reference repository; x, y in metres).  Run from the
repository root with the reference checked out at the directory that the
environment variable REFERENCE names (required)."""
import csv
import json
import os
import sys

REF = os.environ.get("REFERENCE")
if not REF:
    sys.exit("set REFERENCE to the MaterialPointSolver.jl checkout to read its data files from")
SRC = os.path.join(REF, "docs", "assets", "data", "2d_collapse_experiments")


def read(name):
    with open(os.path.join(SRC, name)) as fh:
        return [[float(v) for v in row] for row in csv.reader(fh) if row]


def main(out=os.path.join(os.path.dirname(os.path.abspath(__file__)), "collapse_2d_experiment.json")):
    data = {"source": "MaterialPointSolver.jl docs/assets/data/2d_collapse_experiments/{surface,failure}.csv",
            "surface": read("surface.csv"), "failure": read("failure.csv")}
    with open(out, "w") as fh:
        json.dump(data, fh, indent=1)
    print(out, len(data["surface"]), len(data["failure"]))


if __name__ == "__main__":
    main(*sys.argv[1:])
