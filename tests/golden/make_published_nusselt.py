"""Digitise the time series that the reference publishes for its Rayleigh-Benard example
(docs/examples/rbc.md: Ra = 1e8, Pr = 10, 128^3 coarse and 384^3 refined cells, the scalar on
the refined grid) into tests/golden/published_rbc_ra1e8_pr10.json:

* docs/figures/Nusselt.svg (tools/plot_time_series.py:17-45): Nu_pl, Nu_pu, Nu_chi, Nu_eps,
  Nu_vol over t = 0 .. 200, y axis 0 .. 100;
* docs/figures/Reynolds.svg (tools/plot_time_series.py:47-76): the vertical, horizontal and total
  Reynolds numbers, y axis 0 .. 800.

The SVGs are matplotlib output: every curve is a polyline in plot coordinates, and the grid lines
give the axis mapping.  The script maps the curves back to data and stores them with their time
averages (trapezoidal, over the polyline, from t = 75 and t = 100 to the end).  Run it where the
reference checkout is present:

    python tests/golden/make_published_nusselt.py [reference_root]
"""
import json
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "published_rbc_ra1e8_pr10.json")
FIGURES = {  # file, legend order of plot_time_series.py, top of the y axis, horizontal grid lines
    "nusselt": ("Nusselt.svg", ("nu_pl", "nu_pu", "nu_chi", "nu_eps", "nu_vol"), 100.0, 6),
    "reynolds": ("Reynolds.svg", ("re_v", "re_h", "re_t"), 800.0, 5),
}


def digitise(svg_text: str, names, ymax: float, nhoriz: int) -> dict:
    paths = re.findall(r'<g id="(line2d_\d+)">\s*<path d="([^"]+)"', svg_text)
    pts = lambda d: np.array([[float(a), float(b)] for a, b in re.findall(r"[ML] ([\d.]+) ([\d.]+)", d)])  # noqa: E731
    grid = [pts(d) for _, d in paths if len(pts(d)) == 2]
    verticals = sorted({round(p[0, 0], 6) for p in grid if abs(p[0, 0] - p[1, 0]) < 1e-9})
    horizontals = sorted({round(p[0, 1], 6) for p in grid if abs(p[0, 1] - p[1, 1]) < 1e-9})
    curves = [pts(d) for _, d in paths if len(pts(d)) > 50]
    if len(curves) != len(names) or len(verticals) != 9 or len(horizontals) != nhoriz:
        raise ValueError("unexpected figure structure")
    x0, x1 = verticals[0], verticals[-1]          # t = 0 and t = 200 (nine grid lines, 25 apart)
    yb, yt = horizontals[-1], horizontals[0]       # y = 0 (bottom) and y = ymax (top)
    out = {"series": {}, "mean_from_75": {}, "mean_from_100": {}}
    for name, c in zip(names, curves):
        t = (c[:, 0] - x0) / (x1 - x0) * 200.0
        y = (yb - c[:, 1]) / (yb - yt) * ymax
        out["series"][name] = {"t": [round(v, 4) for v in t], "value": [round(v, 4) for v in y]}
        for t0, key in ((75.0, "mean_from_75"), (100.0, "mean_from_100")):
            m = t >= t0
            out[key][name] = round(float(np.trapezoid(y[m], t[m]) / (t[m][-1] - t[m][0])), 3)
    return out


def digitise_all(root: str) -> dict:
    data = {"source": "docs/figures/Nusselt.svg, docs/figures/Reynolds.svg (tools/plot_time_series.py; "
                      "docs/examples/rbc.md)",
            "case": {"rays": 1e8, "pras": 10.0, "coarse": [128, 128, 128], "refined": [384, 384, 384],
                     "t_end": 200.0}}
    for key, (fname, names, ymax, nh) in FIGURES.items():
        with open(os.path.join(root, "docs", "figures", fname)) as f:
            data[key] = digitise(f.read(), names, ymax, nh)
    return data


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"
    data = digitise_all(root)
    with open(OUT, "w") as f:
        json.dump(data, f, indent=1)
    print(json.dumps({k: data[k]["mean_from_75"] for k in FIGURES}))
