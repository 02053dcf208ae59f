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
