"""The digitised series of the reference's published Rayleigh-Benard example
(tests/golden/published_rbc_ra1e8_pr10.json, made by tests/golden/make_published_nusselt.py) are
what the figures in the reference checkout hold, and the five Nusselt definitions agree with each
other as a statistically steady run's must (within 1.5% over t >= 75), as do the Reynolds numbers
(total = sqrt(vertical^2 + horizontal^2) within the digitisation error).  The figure check runs
only where the reference checkout is present; AFID_REFERENCE_ROOT overrides its location."""
import json
import os
import sys

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURE = os.path.join(HERE, "golden", "published_rbc_ra1e8_pr10.json")
REF = os.environ.get("AFID_REFERENCE_ROOT", "/root/reference")


def test_published_definitions_agree():
    d = json.load(open(FIXTURE))
    nu = d["nusselt"]["mean_from_75"]
    assert set(nu) == {"nu_pl", "nu_pu", "nu_chi", "nu_eps", "nu_vol"}
    mid = sum(nu.values()) / 5
    assert 25.0 < mid < 40.0
    assert all(abs(v - mid) / mid < 0.015 for v in nu.values()), nu
    s = d["reynolds"]["series"]
    assert len(s["re_t"]["t"]) > 100
    re = d["reynolds"]["mean_from_75"]
    assert re["re_t"] > re["re_v"] > 0.0 and re["re_t"] > re["re_h"] > 0.0


@pytest.mark.skipif(not os.path.exists(os.path.join(REF, "docs", "figures", "Nusselt.svg")),
                    reason="reference checkout not present")
def test_fixture_is_the_digitised_figures():
    sys.path.insert(0, os.path.join(HERE, "golden"))
    from make_published_nusselt import digitise_all
    fresh = digitise_all(REF)
    assert json.loads(json.dumps(fresh)) == json.load(open(FIXTURE))
