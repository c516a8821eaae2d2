"""Writes cantilever_2d_curves.json: the tip deflection against time of the 2D
cantilever beam that MaterialPointSolver.jl plots in its accuracy test
(test/c1_accuracy/t1_cantilever_beam/2d_cantilever_beam.jl), as shipped in
docs/assets/data/2d_cantileverbeam_data/ of the reference repository: the FEM
solution (FEM_cantilever_beam.csv) and the published uGIMP and CPDI MPM curves
(MPM_uGIMP.csv, MPM_CPDI.csv); time in s, vertical displacement of the bottom
corner particle at the free end in m, each curve sorted by time.  Run from the
repository root with the reference checked out at the directory that the
environment variable REFERENCE names (required)."""
import csv
import json
import os
import sys

REF = os.environ.get("REFERENCE")
if not REF:
    sys.exit("set REFERENCE to the MaterialPointSolver.jl checkout to read its data files from")
SRC = os.path.join(REF, "docs", "assets", "data", "2d_cantileverbeam_data")


def read(name):
    with open(os.path.join(SRC, name)) as fh:
        rows = [[float(v) for v in row] for row in csv.reader(fh) if row]
    return sorted(rows)


def main(out=os.path.join(os.path.dirname(os.path.abspath(__file__)), "cantilever_2d_curves.json")):
    data = {"source": "MaterialPointSolver.jl docs/assets/data/2d_cantileverbeam_data/"
                      "{FEM_cantilever_beam,MPM_uGIMP,MPM_CPDI}.csv",
            "fem": read("FEM_cantilever_beam.csv"), "ugimp": read("MPM_uGIMP.csv"), "cpdi": read("MPM_CPDI.csv")}
    with open(out, "w") as fh:
        json.dump(data, fh, indent=1)
    print(out, len(data["fem"]), len(data["ugimp"]), len(data["cpdi"]))


if __name__ == "__main__":
    main(*sys.argv[1:])
