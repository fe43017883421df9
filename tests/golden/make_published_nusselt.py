"""Digitise the Nusselt time series that the reference publishes for its Rayleigh-Benard example
(docs/figures/Nusselt.svg, drawn by tools/plot_time_series.py from a run with Ra = 1e8, Pr = 10,
128^3 coarse and 384^3 refined cells, the scalar on the refined grid; docs/examples/rbc.md) into
tests/golden/published_nusselt_rbc_ra1e8_pr10.json.

The SVG is matplotlib output: every curve is a polyline in plot coordinates, and the grid lines
give the axis mapping (t = 0 .. 200 on x, Nu = 0 .. 100 on y).  The script maps the five curves
back to (t, Nu) and stores them with their time averages (trapezoidal, over the polyline, from
t = 75 and t = 100 to the end).  Run it where the reference checkout is present:

    python tests/golden/make_published_nusselt.py [reference_root]
"""
import json
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "published_nusselt_rbc_ra1e8_pr10.json")
# legend order of plot_time_series.py: Nu_pl, Nu_pu, Nu_chi, Nu_eps, Nu_vol
NAMES = ("nu_pl", "nu_pu", "nu_chi", "nu_eps", "nu_vol")


def digitise(svg_text: str) -> dict:
    paths = re.findall(r'<g id="(line2d_\d+)">\s*<path d="([^"]+)"', svg_text)
    pts = lambda d: np.array([[float(a), float(b)] for a, b in re.findall(r"[ML] ([\d.]+) ([\d.]+)", d)])  # noqa: E731
    grid = [pts(d) for _, d in paths if len(pts(d)) == 2]
    verticals = sorted({round(p[0, 0], 6) for p in grid if abs(p[0, 0] - p[1, 0]) < 1e-9})
    horizontals = sorted({round(p[0, 1], 6) for p in grid if abs(p[0, 1] - p[1, 1]) < 1e-9})
    x0, x1 = verticals[0], verticals[-1]          # t = 0 and t = 200 (nine grid lines, 25 apart)
    yb, yt = horizontals[-1], horizontals[0]       # Nu = 0 (bottom) and Nu = 100 (top)
    curves = [pts(d) for _, d in paths if len(pts(d)) > 50]
    if len(curves) != 5 or len(verticals) != 9 or len(horizontals) != 6:
        raise ValueError("unexpected figure structure")
    out = {"source": "docs/figures/Nusselt.svg (tools/plot_time_series.py; docs/examples/rbc.md)",
           "case": {"rays": 1e8, "pras": 10.0, "coarse": [128, 128, 128], "refined": [384, 384, 384],
                    "t_end": 200.0},
           "series": {}, "mean_from_75": {}, "mean_from_100": {}}
    for name, c in zip(NAMES, curves):
        t = (c[:, 0] - x0) / (x1 - x0) * 200.0
        nu = (yb - c[:, 1]) / (yb - yt) * 100.0
        out["series"][name] = {"t": [round(v, 4) for v in t], "nu": [round(v, 4) for v in nu]}
        for t0, key in ((75.0, "mean_from_75"), (100.0, "mean_from_100")):
            m = t >= t0
            out[key][name] = round(float(np.trapezoid(nu[m], t[m]) / (t[m][-1] - t[m][0])), 3)
    return out


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"
    with open(os.path.join(root, "docs", "figures", "Nusselt.svg")) as f:
        data = digitise(f.read())
    with open(OUT, "w") as f:
        json.dump(data, f, indent=1)
    print(json.dumps({k: data[k] for k in ("mean_from_75", "mean_from_100")}))
