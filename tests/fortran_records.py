"""Readers for the reference's output files, written independently of the
library for the tests: Fortran unformatted sequential records (4-byte
lengths around each record, native byte order) and the legacy binary VTK
snapshot of output_hdf_dfsd (PFC/read_write.f90:296-500)."""
import numpy as np


def read_records(path):
    recs = []
    with open(path, "rb") as f:
        b = f.read()
    i = 0
    while i < len(b):
        n = int(np.frombuffer(b, np.int32, 1, i)[0])
        rec = b[i + 4:i + 4 + n]
        n2 = int(np.frombuffer(b, np.int32, 1, i + 4 + n)[0])
        assert n2 == n, "record markers disagree"
        recs.append(rec)
        i += n + 8
    return recs


def parse_restart(path, nx, ny, nz):
    """-> header dict, data1 (nz, nx/2+1, ny+1, 3), tail record ints"""
    recs = read_records(path)
    h = recs[0]
    assert len(h) == 52
    ints = np.frombuffer(h, np.int32, 3, 0)
    reals = np.frombuffer(h, np.float64, 5, 12)
    head = dict(nx=int(ints[0]), ny=int(ints[1]), nz=int(ints[2]), lx=reals[0], lz=reals[1], re=reals[2],
                dt=reals[3], t_total=reals[4])
    nxh = nx // 2 + 1
    assert len(recs) == 1 + nxh + 1
    d1 = np.zeros((nz, nxh, ny + 1, 3), np.complex128, order="F")
    for x in range(nxh):
        sl = np.frombuffer(recs[1 + x], np.complex128).reshape((nz, ny + 1, 3), order="F")
        d1[:, x, :, :] = sl
    tail = np.frombuffer(recs[-1], np.int32)
    return head, d1, tail


def parse_vtk(path):
    """-> dict(lines=[header lines], x, y, z (float32), vel (nx, ny+1, nz, 3) float32)"""
    b = open(path, "rb").read()
    out = {"lines": []}
    i = 0

    def line():
        nonlocal i
        j = b.index(b"\n", i)
        s = b[i:j].decode()
        i = j + 1
        out["lines"].append(s)
        return s

    for _ in range(5):
        line()
    dims = [int(v) for v in out["lines"][4].split()[1:4]]
    nx, n1, nz = dims
    for key, n in (("x", nx), ("y", n1), ("z", nz)):
        line()
        out[key] = np.frombuffer(b, ">f4", n, i).astype(np.float32)
        i += 4 * n
        assert b[i:i + 1] == b"\n"
        i += 1
    line()
    line()
    npts = nx * n1 * nz
    v = np.frombuffer(b, ">f4", 3 * npts, i).astype(np.float32)
    i += 12 * npts
    assert b[i:i + 1] == b"\n"
    i += 1
    # (c, x, plane, z) with c fastest
    out["vel"] = v.reshape((3, nx, n1, nz), order="F").transpose(1, 2, 3, 0)
    out["dims"] = dims
    # optional further sections: VECTORS name float / SCALARS name float 1
    while i < len(b):
        kind, name = line().split()[:2]
        if kind == "SCALARS":
            line()   # LOOKUP_TABLE default
            n = npts
        else:
            n = 3 * npts
        a = np.frombuffer(b, ">f4", n, i).astype(np.float32)
        i += 4 * n
        assert b[i:i + 1] == b"\n"
        i += 1
        if kind == "SCALARS":
            out[name] = a.reshape((nx, n1, nz), order="F")
        else:
            out[name] = a.reshape((3, nx, n1, nz), order="F").transpose(1, 2, 3, 0)
    return out
