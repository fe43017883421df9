"""Regenerate tests/golden/continua/: a small restart file set (WriteFlowField.F90 layout, final
write with the refined salinity) written by the oracle's version-0 HDF5 writer
(oracle/afid_h5.py write_v0), independently of the library's native writer.  The test checks
that the native writer produces the same bytes from the same arrays and that both readers read
them back.

    python tests/golden/make_continua_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

OUT = os.path.join(HERE, "continua")
# coarse 4 x 3 x 2 (nxm, nym, nzm), refined 8 x 6 x 4, tanh grids, time 0.625
GRID = dict(nxm=4, nym=3, nzm=2, nxmr=8, nymr=6, nzmr=4, ylen=1.0, zlen=1.0, istr3=4, str3=2.0, istr3r=4,
            time=0.625)


def arrays(seed: int = 2026):
    g = GRID
    rng = np.random.default_rng(seed)
    nx = g["nxm"] + 1
    f = {k: rng.standard_normal((g["nzm"], g["nym"], nx)) for k in ("temp", "vx", "vy", "vz", "pr")}
    for k in ("temp", "vy", "vz", "pr"):
        f[k][..., -1] = 0.0          # the upper wall node of the cell-centred fields
    sal = np.zeros((g["nzmr"], g["nymr"], g["nxmr"] + 1))
    sal[..., :g["nxmr"]] = rng.standard_normal((g["nzmr"], g["nymr"], g["nxmr"]))
    f["sal"] = sal                   # extra refined x node zero, as the reference leaves it
    return f


def master():
    g = GRID
    i4 = lambda v: np.array([v], dtype="<i4")  # noqa: E731
    f8 = lambda v: np.array([v], dtype="<f8")  # noqa: E731
    return {"nx": i4(g["nxm"] + 1), "ny": i4(g["nym"] + 1), "nz": i4(g["nzm"] + 1), "ylen": f8(g["ylen"]),
            "zlen": f8(g["zlen"]), "time": f8(g["time"]), "istr3": i4(g["istr3"]), "str3": f8(g["str3"]),
            "nxr": i4(g["nxmr"] + 1), "nyr": i4(g["nymr"] + 1), "nzr": i4(g["nzmr"] + 1), "istr3r": i4(g["istr3r"])}


def main():
    from oracle import afid_h5 as h5
    os.makedirs(OUT, exist_ok=True)
    for k, a in arrays().items():
        h5.write_v0(os.path.join(OUT, f"continua_{k}.h5"), {"var": a})
    h5.write_v0(os.path.join(OUT, "continua_master.h5"), master())
    print("wrote", sorted(os.listdir(OUT)))


if __name__ == "__main__":
    main()
