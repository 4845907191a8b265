"""Extract the reference's MHD jump states (experiment/CorrugationShock/data/*.mat) into
corrugation_jumps.json beside this script.

Each file holds one stationary-shock solution of the reference's MHDJumpSolver (pre- and
post-shock density, pressure, velocity and magnetic field, in the shock frame) for a sonic Mach
number, Alfven Mach number, field angle and gamma; the values are copied as they are.  Usage:

    python tests/golden/make_corrugation_fixture.py <root of the reference tree>

The JSON is committed so the tests do not need the reference at run time."""
import glob
import json
import os
import sys

import numpy as np
import scipy.io

HERE = os.path.dirname(os.path.abspath(__file__))


def main(root):
    out = []
    paths = sorted(glob.glob(os.path.join(root, "experiment", "CorrugationShock", "data", "ics-*.mat")))
    if not paths:
        raise SystemExit(f"no experiment/CorrugationShock/data/ics-*.mat under {root}")
    for path in paths:
        r = scipy.io.loadmat(path)["result"][0, 0]
        names = r.dtype.names
        base = os.path.basename(path)
        rec = {"file": "experiment/CorrugationShock/data/" + base}
        # gamma is part of the name when it is not 5/3 (..._g1_4.mat -> 1.4)
        rec["gamma"] = float(base.split("-g")[1][:-4].replace("_", ".")) if "-g" in base else 5.0 / 3.0
        imag = 0.0
        for k in names:
            v = np.asarray(r[k])
            if np.iscomplexobj(v):
                imag = max(imag, float(np.abs(v.imag).max()))
            rec[k] = np.real(v).astype(float).tolist()
        rec["max_imag"] = imag   # a few solver outputs carry complex parts; the tests skip those
        out.append(rec)
    with open(os.path.join(HERE, "corrugation_jumps.json"), "w") as f:
        json.dump(out, f, indent=1)
    print(f"{len(out)} jump solutions, fields {names}")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        raise SystemExit("usage: make_corrugation_fixture.py <root of the reference tree>")
    main(sys.argv[1])
