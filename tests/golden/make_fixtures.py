"""Regenerates the golden fixtures under tests/golden/ from the reference
project's shipped data.  The reference checkout's root is the first argument
or the REFERENCE_ROOT environment variable:

    python tests/golden/make_fixtures.py <reference checkout>

makegrid_ny200.json: y(200), yh(201) written by output_grids
(PFC/setup.f90:1331-1359) for ny=200 with STRETCH=2.75, as printed in
PFC/makegrid.m (format f16.8).

flow_ref.dat: the reference's own run-parameter file
(ParallelFortran-Code/flow.dat), copied as the flow.dat reader's fixture.

partition_nproc24.json: the partition table distribute_data
(PFC/setup.f90:298-437) printed for Nx=128, Nz=64 (Nz2=96) on 24 ranks in
PFC/diagnostics.txt (the leftover line and the per-rank nx_proc, x_start,
nz_proc, z_start, nz_small, z_small columns).
"""
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def reference_root():
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("REFERENCE_ROOT")
    if not ref:
        sys.exit("usage: make_fixtures.py <reference checkout> (or set REFERENCE_ROOT)")
    return ref


def main():
    REF = reference_root()
    txt = open(os.path.join(REF, "ParallelFortran-Code", "makegrid.m")).read()

    def block(name):
        m = re.search(r"\b" + name + r" = \[(.*?)\];", txt, re.S)
        return [float(v) for v in m.group(1).split()]

    out = {"source": "ParallelFortran-Code/makegrid.m", "ny": 200, "stretch": 2.75,
           "decimals": 8, "y": block("y"), "yh": block("yh")}
    with open(os.path.join(HERE, "makegrid_ny200.json"), "w") as f:
        json.dump(out, f)
    print("wrote makegrid_ny200.json", len(out["y"]), len(out["yh"]))

    lines = open(os.path.join(REF, "ParallelFortran-Code", "diagnostics.txt")).read().splitlines()
    head = next(i for i, l in enumerate(lines) if l.strip().startswith("Proc   nx_proc"))
    left = [int(v) for v in lines[head - 1].split()]
    rows = []
    for l in lines[head + 1:]:
        f = l.split()
        if len(f) != 7:
            break
        rows.append([int(v) for v in f])
    cols = ["proc", "nx_proc", "x_start", "nz_proc", "z_start", "nz_small_proc", "z_small_start"]
    part = {"source": "ParallelFortran-Code/diagnostics.txt", "nx": 128, "nz": 64, "nz2": 96, "nproc": len(rows),
            "xleft_zleft_zsmallleft": left}
    for k, name in enumerate(cols):
        part[name] = [r[k] for r in rows]
    with open(os.path.join(HERE, "partition_nproc24.json"), "w") as f:
        json.dump(part, f)
    print("wrote partition_nproc24.json", len(rows))

    src = open(os.path.join(REF, "ParallelFortran-Code", "flow.dat")).read()
    with open(os.path.join(HERE, "flow_ref.dat"), "w") as f:
        f.write(src)
    print("wrote flow_ref.dat", len(src.splitlines()), "lines")


if __name__ == "__main__":
    main()
