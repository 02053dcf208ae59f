"""The CPU oracle against fixtures produced by the reference's own hourly step.

The fixtures (tests/golden/*.npz) come from tests/golden/make_golden.py, which
runs the reference's ``timestep_body`` and ``_run_day_inner`` unmodified in
float64.  The oracle must reproduce them (it does so bit for bit).
"""
import warnings

import numpy as np
import pytest

import oracle
from goldens import CASES, Case, compare

warnings.filterwarnings("ignore", category=RuntimeWarning)


@pytest.mark.parametrize("name", CASES)
def test_oracle_matches_reference_steps(name):
    c = Case(name)
    prog = {k: v.copy() for k, v in c.prog.items()}
    acc = oracle.new_acc(c.ncell)
    checked = 0
    with np.errstate(all="ignore"):
        for h in range(c.nhour):
            prog, D, acc = oracle.step(prog, c.stat, c.forcing_at(h), c.params, acc)
            if (h + 1) in c.record:
                bad = compare(prog, c.out(h + 1, "prog"), 1e-12) + compare(D, c.out(h + 1, "diag"), 1e-12)
                assert not bad, bad[:5]
                checked += 1
    assert checked == len(c.record)


def test_oracle_matches_reference_day_accumulators():
    c = Case("day_mixed")
    assert c.has_day
    prog = {k: v.copy() for k, v in c.prog.items()}
    acc = oracle.new_acc(c.ncell)
    with np.errstate(all="ignore"):
        for h in range(c.nhour):
            prog, D, acc = oracle.step(prog, c.stat, c.forcing_at(h), c.params, acc)
    # the reference casts each step's CH4 flux to float32 before accumulating it
    assert not compare(acc, c.day("acc"), 1e-6)
    assert not compare(prog, c.day("prog"), 1e-12)


def test_golden_cases_cover_the_edge_regimes():
    c = Case("day_mixed")
    fi = c.out(24, "prog")["fi"]
    assert fi[1] > 0.5                       # snowpack cell keeps snow
    assert c.stat["fu"][0] == 0.0            # bare cell present
    assert np.any(c.prog["wisoi"] > 0.5)     # frozen cell present
    assert c.prog["wpud"][3] > 0.0           # flooded cell present


def test_oracle_matches_reference_et_and_nee_parts():
    """The optional ET and NEE components (loops_gswp3.py:263-281) against the
    reference's day with those modules attached (tests/golden/day_parts.npz)."""
    import os
    from ibis_b200.params import FLAG_ETPARTS, FLAG_NEEPARTS
    c = Case("day_mixed")
    z = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "day_parts.npz"))
    want = {k[8:]: z[k] for k in z.files if k.startswith("day.acc.")}
    P = c.params.copy()
    P.flags |= FLAG_ETPARTS | FLAG_NEEPARTS
    prog = {k: v.copy() for k, v in c.prog.items()}
    acc = oracle.new_acc(c.ncell)
    with np.errstate(all="ignore"):
        for h in range(c.nhour):
            prog, D, acc = oracle.step(prog, c.stat, c.forcing_at(h), P, acc)
    parts = ("et_trans", "et_interc", "et_soilev", "et_snowsub", "nee_night", "nee_day")
    assert not compare({k: acc[k] for k in parts}, {k: want[k] for k in parts}, 1e-9)
    assert not compare(acc, {k: v for k, v in want.items() if k not in parts}, 1e-6)   # the rest unchanged
    np.testing.assert_allclose(acc["et_trans"] + acc["et_interc"] + acc["et_soilev"] + acc["et_snowsub"],
                               acc["adaet"], rtol=1e-12, atol=1e-12)
    assert np.any(acc["nee_night"] != 0) and np.any(acc["nee_day"] != 0) and np.any(acc["et_snowsub"] != 0)
