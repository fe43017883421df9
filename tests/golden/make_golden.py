"""Regenerate the golden fixtures of tests/golden/ from the FP64 NumPy oracle.

Each fixture is a small seeded case (bou.in text + initial state seed + random-velocity
amplitude) and the oracle state after 1 and 3 RK3 steps; tests/golden/salinity/ holds the same
for the multi-resolution salinity path (coarse fields and refined salinity).  The reference itself cannot run
here (Fortran/MPI/FFTW/HDF5 absent), so these pin the oracle's own behaviour against later
changes; the reference-anchored pins are the published 1-D diffusion errors and the
divergence-free invariant (tests/test_oracle.py).

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "afid-murphfi_b200"))  # tests/helpers.py imports the binding

CASES = {
    "rbc3d_16x12x8_rv": dict(shape=(16, 12, 8), kw=dict(rayt=1e6, dt=2e-3), seed=11, rv=0.2),
    "rbc3d_40x10x6_rv": dict(shape=(40, 10, 6), kw=dict(rayt=1e5, dt=1e-3, istr3=6, str3=4.0), seed=12, rv=0.3),
    "rbc2d_32x48x1": dict(shape=(32, 48, 1), kw=dict(rayt=1e7, dt=2e-3, ylen=2.0, zlen=0.01), seed=13, rv=0.0),
}


def make(name: str, spec: dict) -> dict:
    from helpers import bou_text
    from oracle import afid_oracle as o
    text = bou_text(*spec["shape"], **spec["kw"])
    p = o.parse_bou_in(text)
    g = o.create_grid(p)
    s = o.initial_state(g, spec["seed"])
    if spec["rv"]:
        rng = np.random.default_rng(spec["seed"])
        for f in ("vx", "vy", "vz", "pr"):
            getattr(s, f)[...] = spec["rv"] * rng.standard_normal(s.vx.shape)
        s.vx[..., 0] = 0.0
        s.vx[..., -1] = 0.0
        for f in ("vy", "vz", "temp", "pr"):
            getattr(s, f)[..., -1] = 0.0
    out = {"bou_in": np.array(text), "dt": np.array(p.dt)}
    for f in ("vx", "vy", "vz", "temp", "pr"):
        out["init_" + f] = getattr(s, f).copy()
    for n in range(3):
        o.time_marcher(g, s, p.dt)
        if n in (0, 2):
            for f in ("vx", "vy", "vz", "temp", "pr"):
                out[f"step{n + 1}_{f}"] = getattr(s, f).copy()
    out["step3_cfl"] = np.array(o.calc_max_cfl(g, s))
    out["step3_nu"] = np.array(o.nusselt_volume(g, s))
    return out


# Multi-resolution salinity (MULTIRES = FLAGSAL = 1): the coarse flow state and the refined
# salinity after 1 and 3 steps of oracle/afid_salinity.py, in tests/golden/salinity/.
SAL_CASES = {
    "ddc3d_12x8x4_r24x16x8": dict(shape=(12, 8, 4), kw=dict(rayt=1e6, dt=1e-3, multires=1, nxmr=24, nymr=16,
                                                            nzmr=8, flagsal=1, istr3r=4, rays=1e6, pras=10.0,
                                                            active_s=1), seed=21, rv=0.05),
    "ddc2d_16x24x1_r36x48x1": dict(shape=(16, 24, 1), kw=dict(rayt=1e6, dt=1e-3, ylen=2.0, zlen=0.01, multires=1,
                                                              nxmr=36, nymr=48, nzmr=1, flagsal=1, istr3r=0,
                                                              rays=-1e6, pras=7.0, active_s=1, sfixn=0),
                                   seed=22, rv=0.05),
}


def make_sal(name: str, spec: dict) -> dict:
    from helpers import bou_text
    from oracle import afid_oracle as o
    from oracle import afid_salinity as sa
    text = bou_text(*spec["shape"], **spec["kw"])
    p = o.parse_bou_in(text)
    g = o.create_grid(p)
    m = sa.create_mgrd(g)
    s = o.initial_state(g, spec["seed"])
    rng = np.random.default_rng(spec["seed"])
    for f in ("vx", "vy", "vz"):
        getattr(s, f)[...] = spec["rv"] * rng.standard_normal(s.vx.shape)
    s.vx[..., 0] = 0.0
    s.vx[..., -1] = 0.0
    for f in ("vy", "vz", "temp", "pr"):
        getattr(s, f)[..., -1] = 0.0
    sal = np.clip(sa.initial_salinity(m, g, spec["seed"]) + 0.01 * rng.standard_normal((m.nzmr, m.nymr, m.nxmr)),
                  -0.5, 0.5)
    ss = sa.new_sal_state(m, g, sal)
    sa.interp_vel_mgrd(m, g, s, ss)
    sa.interp_sal_multigrid(m, g, ss)
    out = {"bou_in": np.array(text), "dt": np.array(p.dt), "init_sal": sal.copy()}
    for f in ("vx", "vy", "vz", "temp", "pr"):
        out["init_" + f] = getattr(s, f).copy()
    for n in range(3):
        sa.time_marcher(g, s, m, ss, p.dt)
        if n in (0, 2):
            for f in ("vx", "vy", "vz", "temp", "pr"):
                out[f"step{n + 1}_{f}"] = getattr(s, f).copy()
            out[f"step{n + 1}_sal"] = ss.sal.copy()
    out["step3_cflmr"] = np.array(sa.calc_max_cfl_refined(m, ss))
    return out


if __name__ == "__main__":
    for name, spec in CASES.items():
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **make(name, spec))
    os.makedirs(os.path.join(HERE, "salinity"), exist_ok=True)
    for name, spec in SAL_CASES.items():
        np.savez_compressed(os.path.join(HERE, "salinity", name + ".npz"), **make_sal(name, spec))
        print("wrote", name)
