"""Builds tests/golden/ref_cloudload.json from the reference's own regression
tests (tests/test_01, tests/test_02 of the Ash3d source tree): the control
parameters this restatement needs, read from the control file and the 1-D
wind sounding, and the golden output grids of the reference binary (ESRI
ASCII): CloudLoad, CloudHeight and CloudConcentration at 2 h and 4 h and
CloudArrivalTime, each kept as its nonzero cells (fill values included).

    python tests/golden/make_ref_cloudload.py [path/to/Ash3d/source/tree]

Only this script reads the reference tree; the test reads the fixture.
"""
import json
import pathlib
import sys

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent


def _data_lines(path):
    """Non-comment, non-separator lines of a control file, split on '#'."""
    out = []
    for ln in path.read_text().splitlines():
        if not ln.strip() or ln.startswith("#") or ln.startswith("*"):
            continue
        out.append(ln.split("#")[0].split())
    return out


def control(path):
    """Block 1-3 values of an Ash3d control file (projected grid, one pulse)."""
    d = _data_lines(path)
    # block 1: name, projection, LL corner, width/height, vent, dx dy, dz,
    # diffusivity + Suzuki constant, number of pulses; block 2: the pulse
    xll, yll = (float(v) for v in d[2][:2])
    width, height = (float(v) for v in d[3][:2])
    xv, yv = (float(v) for v in d[4][:2])
    dx, dy = (float(v) for v in d[5][:2])
    dz = float(d[6][0])
    diff, suzuki = (float(v) for v in d[7][:2])
    pulse = d[9]
    # block 3: iwind iwindformat, iHeightHandler, simulation time
    simtime = float(d[12][0])
    return dict(nx=int(round(width / dx)), ny=int(round(height / dy)), dx=dx, dy=dy, dz=dz,
                ivent=int((xv - xll) / dx) + 1, jvent=int((yv - yll) / dy) + 1,
                diffusivity_m2s=diff, suzuki_a=suzuki, duration_h=float(pulse[4]),
                plume_km=float(pulse[5]), volume_km3=float(pulse[6]), sim_hours=simtime)


def sounding(path):
    """(z_m, u_mps, v_mps) of the levels of a 1-D ASCII wind file."""
    lines = path.read_text().splitlines()
    nlev = int(lines[1].split()[1])
    return [[float(v) for v in lines[3 + i].split()[:3]] for i in range(nlev)]


def cloudload(path):
    """A 2-D output grid as [i][j] (j from the south), nonzero cells only."""
    head = dict(ln.split()[:2] for ln in path.read_text().splitlines()[:2])
    nx, ny = int(head["NCOLS"]), int(head["NROWS"])
    g = np.loadtxt(path, skiprows=6).reshape(ny, nx)[::-1, :].T
    nz = np.argwhere(g != 0.0)
    return [[int(i), int(j), float(g[i, j])] for i, j in nz]


def main(root):
    root = pathlib.Path(root)
    out = {}
    for test, inp in (("test_01", "TC1_XY_MSH.inp"), ("test_02", "TC2_XY_MSH.inp")):
        t = root / "tests" / test
        out[test] = {"control": control(t / inp), "sounding": sounding(t / "Hanford_Ncol_N.txt"),
                     "cloudload": {h: cloudload(t / "output" / f"CloudLoad_{float(h):06.2f}hrs.dat")
                                   for h in ("2.0", "4.0")},
                     "cloudheight": {h: cloudload(t / "output" / f"CloudHeight_{float(h):06.2f}hrs.dat")
                                     for h in ("2.0", "4.0")},
                     "cloudconc": {h: cloudload(t / "output" / f"CloudConcentration_{float(h):06.2f}hrs.dat")
                                   for h in ("2.0", "4.0")},
                     "cloudarrival": cloudload(t / "output" / "CloudArrivalTime.dat")}
    (HERE / "ref_cloudload.json").write_text(json.dumps(out, separators=(",", ":")))


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_ref_cloudload.py <path of the Ash3d source tree>")
    main(sys.argv[1])
