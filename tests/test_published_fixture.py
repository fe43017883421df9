"""The digitised Nusselt series of the reference's published Rayleigh-Benard example
(tests/golden/published_nusselt_rbc_ra1e8_pr10.json, made by tests/golden/make_published_nusselt.py)
is what the figure in the reference checkout holds, and its five definitions agree with each other
as a statistically steady run's must (within 1.5% over t >= 75).  The figure check runs only where
the reference checkout is present; AFID_REFERENCE_ROOT overrides its location."""
import json
import os
import sys

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURE = os.path.join(HERE, "golden", "published_nusselt_rbc_ra1e8_pr10.json")
REF = os.environ.get("AFID_REFERENCE_ROOT", "/root/reference")


def test_published_nusselt_definitions_agree():
    d = json.load(open(FIXTURE))
    means = d["mean_from_75"]
    assert set(means) == {"nu_pl", "nu_pu", "nu_chi", "nu_eps", "nu_vol"}
    mid = sum(means.values()) / 5
    assert 25.0 < mid < 40.0
    assert all(abs(v - mid) / mid < 0.015 for v in means.values()), means


@pytest.mark.skipif(not os.path.exists(os.path.join(REF, "docs", "figures", "Nusselt.svg")),
                    reason="reference checkout not present")
def test_fixture_is_the_digitised_figure():
    sys.path.insert(0, os.path.join(HERE, "golden"))
    from make_published_nusselt import digitise
    with open(os.path.join(REF, "docs", "figures", "Nusselt.svg")) as f:
        fresh = digitise(f.read())
    assert json.loads(json.dumps(fresh)) == json.load(open(FIXTURE))
