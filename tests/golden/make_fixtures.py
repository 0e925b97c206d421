"""Regenerates the golden fixtures under tests/golden/ from the reference
project's shipped data (run in a container where the reference is mounted).

makegrid_ny200.json: y(200), yh(201) written by output_grids
(PFC/setup.f90:1331-1359) for ny=200 with STRETCH=2.75, as printed in
PFC/makegrid.m (format f16.8).
"""
import json
import os
import re
import sys

REF = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"
HERE = os.path.dirname(os.path.abspath(__file__))


def main():
    txt = open(os.path.join(REF, "ParallelFortran-Code", "makegrid.m")).read()

    def block(name):
        m = re.search(r"\b" + name + r" = \[(.*?)\];", txt, re.S)
        return [float(v) for v in m.group(1).split()]

    out = {"source": "ParallelFortran-Code/makegrid.m", "ny": 200, "stretch": 2.75,
           "decimals": 8, "y": block("y"), "yh": block("yh")}
    with open(os.path.join(HERE, "makegrid_ny200.json"), "w") as f:
        json.dump(out, f)
    print("wrote makegrid_ny200.json", len(out["y"]), len(out["yh"]))


if __name__ == "__main__":
    main()
