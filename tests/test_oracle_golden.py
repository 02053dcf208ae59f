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


X3_CASES = ("release", "switches")


@pytest.mark.parametrize("name", X3_CASES)
def test_oracle_matches_reference_ibis3_steps(name):
    """The IBIS 3.0 extensions of the step (vmax and slope mixing, capacity split,
    acclimation with per-PFT constants, light-rate factor, frost ramp, canopy-level
    capacity scaling, leaf-only light scaling, cropland grass capacity, organic
    soil solids) against the reference run with its own switches on: the release
    parameter file's stomata, respiration and methane sections, and the switches
    that file leaves off (make_golden.py build_x3_case)."""
    c = Case(name)
    prog = {k: v.copy() for k, v in c.prog.items()}
    acc = oracle.new_acc(c.ncell)
    checked = 0
    with np.errstate(all="ignore"):
        for h in range(c.nhour):
            prog, D, acc = oracle.step(prog, c.stat, c.forcing_at(h), c.params, acc)
            if (h + 1) in c.record:
                bad = compare(prog, c.out(h + 1, "prog"), 1e-12) + compare(D, c.out(h + 1, "diag"), 1e-12)
                assert not bad, (h + 1, bad[:5])
                checked += 1
    assert checked == len(c.record)


def test_oracle_matches_reference_release_day_accumulators():
    """_run_day_inner's sums under the release switches: the NPP split by capacity,
    the ET components of the modules the seasonal state brings, CH4 and soil means."""
    c = Case("release")
    prog = {k: v.copy() for k, v in c.prog.items()}
    acc = oracle.new_acc(c.ncell)
    with np.errstate(all="ignore"):
        for h in range(c.nhour):
            prog, D, acc = oracle.step(prog, c.stat, c.forcing_at(h), c.params, acc)
    want = c.day("acc")
    assert "et_trans" in want and "aynpp" in want
    assert not compare(acc, want, 1e-6)                       # CH4 cast to float32 per step by the reference
    assert not compare({k: acc[k] for k in ("aynpp", "aynpptot", "aygpptot", "et_trans")},
                       {k: want[k] for k in ("aynpp", "aynpptot", "aygpptot", "et_trans")}, 1e-12)
    assert not compare(prog, c.day("prog"), 1e-12)


def test_release_case_exercises_the_switches():
    """The fixtures reach the switched branches: acclimation factors strictly
    between 0 and 1 and at both clips, mixed big leaves, capacity shares that
    differ from the leaf-area shares, crop and organic inputs present."""
    from oracle.canopy import capacity_factor, big_leaves
    from oracle.step import gpp_shares
    c = Case("release")
    vf = capacity_factor(c.stat, c.params)
    acc_pfts = vf[:, [3, 5, 8]]
    assert np.any(acc_pfts == 0.0) and np.any(acc_pfts == 1.0) and np.any((acc_pfts > 0) & (acc_pfts < 1))
    sh = gpp_shares(c.stat["frac"], c.params)
    assert np.max(np.abs(sh - c.stat["frac"])) > 1e-3
    (vub, *_), _, (mub, *_) = big_leaves(c.stat, c.params)
    assert np.unique(np.round(mub, 9)).size > 3
    s = Case("switches")
    assert s.stat["cropfrac"].max() > 0.5 and s.stat["forganic"].max() > 0.3
    _, je, _ = big_leaves(s.stat, s.params)
    assert all(j is not None for j in je) and np.any(je[4] != 1.0)
