"""The IBIS 3.0 extensions of the hourly step on the GPU.

The fixtures ``tests/golden/release.npz`` and ``tests/golden/switches.npz`` are
the reference's own ``timestep_body`` (and, for ``release``, its
``_run_day_inner``) run with its stomata switches on: the release parameter
file's stomata, respiration and methane sections (vmax and slope mixing by
displayed leaf area, the NPP split by capacity, temperature acclimation with
per-PFT constants, sunlit/shaded canopies, consistent soil-water weights), and
the switches that file leaves off (canopy-level capacity scaling, leaf-only
light scaling, acclimation with its light-rate factor and frost ramp, the
cropland share's grass capacity, organic soil solids).

Tolerances (as for the F77 step in test_gpu_parity.py):
* float64 kernels vs the reference's outputs and vs the float64 oracle:
  relative 1e-9 per field at every recorded hour (absolute floors for
  near-zero fields, tests/goldens.py:FLOORS); day accumulators 1e-6 (the
  reference casts each step's CH4 flux to float32).
* FP32 kernels vs the float64 oracle after one hour: the bounds of the F77
  step's FP32 test (test_gpu_parity.FP32_ONE_HOUR); conductances and
  intercellular CO2 within 1e-4.
"""
import types
import warnings

import numpy as np
import pytest
import torch

import oracle
from goldens import Case, compare
from ibis_b200 import dropin
from ibis_b200 import layout as L
from ibis_b200.columns import Columns
from ibis_b200.params import FLAG_KAHAN

warnings.filterwarnings("ignore", category=RuntimeWarning)
pytestmark = pytest.mark.gpu

X3_CASES = ("release", "switches")


def _run(c, dtype, nstep, mode="fused", diag=True):
    cols = Columns.from_host(c.prog, c.stat, dtype=dtype, diag=diag, acc=True, mode=mode)
    P = c.params.copy()
    if dtype == torch.float64:
        P.flags &= ~FLAG_KAHAN
    cols.run(cols.forcing(c.forc, 0, nstep), P)
    torch.cuda.synchronize()
    return cols


def _oracle(c, nstep):
    prog = {k: v.copy() for k, v in c.prog.items()}
    acc = oracle.new_acc(c.ncell)
    with np.errstate(all="ignore"):
        for h in range(nstep):
            prog, D, acc = oracle.step(prog, c.stat, c.forcing_at(h), c.params, acc)
    return prog, D, acc


@pytest.mark.parametrize("name", X3_CASES)
def test_f64_kernel_matches_reference_at_every_recorded_hour(cuda_lib, name):
    c = Case(name)
    for h in c.record:
        cols = _run(c, torch.float64, h)
        bad = compare({**cols.prog_host(), **cols.diag_host()}, {**c.out(h, "prog"), **c.out(h, "diag")}, 1e-9)
        assert not bad, (h, bad[:6])
        assert not cols.nonfinite()[0]


@pytest.mark.parametrize("name", X3_CASES)
@pytest.mark.parametrize("nstep", [1, 6])
def test_f64_kernel_matches_oracle(cuda_lib, name, nstep):
    c = Case(name)
    cols = _run(c, torch.float64, nstep)
    prog, D, _ = _oracle(c, nstep)
    bad = compare({**cols.prog_host(), **cols.diag_host()}, {**prog, **D}, 1e-9)
    assert not bad, bad[:6]


def test_f64_release_day_accumulators_match_reference(cuda_lib):
    """The day's sums under the release switches: NPP split by capacity, ET
    components, CH4 and soil means, against _run_day_inner."""
    c = Case("release")
    cols = _run(c, torch.float64, 24, diag=False)
    got, want = cols.acc_host(compensated=False), c.day("acc")
    assert "et_trans" in want
    assert not compare(got, want, 1e-6)
    assert not compare(cols.prog_host(), c.day("prog"), 1e-9)


@pytest.mark.parametrize("name", X3_CASES)
def test_f32_kernel_close_to_oracle(cuda_lib, name):
    c = Case(name)
    cols = _run(c, torch.float32, 1)
    prog, _, _ = _oracle(c, 1)
    got = cols.prog_host()
    from test_gpu_parity import FP32_ONE_HOUR
    for k, bound in FP32_ONE_HOUR.items():
        g = np.asarray(got[k], np.float64).reshape(prog[k].shape)
        assert float(np.max(np.abs(g - prog[k]))) <= bound, k
    for k in ("gs_upper", "gs_lower", "ci_upper", "ci_lower"):
        g, w = np.asarray(got[k], np.float64).reshape(prog[k].shape), prog[k]
        np.testing.assert_allclose(g, w, rtol=1e-4, atol=1e-8, err_msg=k)


def test_f32_release_day_close_to_reference(cuda_lib):
    """The FP32 fused day under the release switches (the long fused
    configuration with accumulators on chip) against the reference's float64
    day: every accumulator within 1e-3 of its plane's largest magnitude on 90 %
    of the cells, and the annual GPP and NPP totals within 1e-3."""
    c = Case("release")
    cols = _run(c, torch.float32, 24, diag=False)
    got, want = cols.acc_host(), c.day("acc")
    for k, w in want.items():
        g = np.asarray(got[k], np.float64).reshape(w.shape)
        scale = max(float(np.abs(w).max()), 1e-30)
        cells = np.abs(g - w).reshape(w.shape[0], -1).max(axis=1) <= 1e-3 * scale
        assert cells.mean() >= 0.9, (k, float(cells.mean()))
    for k in ("aygpptot", "aynpptot"):
        assert abs(got[k].sum() - want[k].sum()) <= 1e-3 * np.abs(want[k]).sum(), k


def test_split_form_matches_fused_form(cuda_lib):
    c = Case("release")
    a = _run(c, torch.float32, 6)
    b = _run(c, torch.float32, 6, mode="split")
    pa, pb = a.prog_host(), b.prog_host()
    for k in ("tsoi", "tg", "tu", "tl", "ti"):
        np.testing.assert_allclose(pb[k], pa[k], rtol=1e-4, atol=0.05, err_msg=k)
    for k in ("gs_upper", "gs_lower"):
        np.testing.assert_allclose(pb[k], pa[k], rtol=1e-3, atol=1e-6, err_msg=k)


def test_switches_change_the_result(cuda_lib):
    """Each case's switches move the step: the same columns without them give
    different stomatal conductances (so the extended kernels are not silently
    running the F77 step)."""
    from ibis_b200.params import X3_FLAGS
    for name in X3_CASES:
        c = Case(name)
        on = _run(c, torch.float64, 1).prog_host()
        c.params.flags &= ~X3_FLAGS
        off = _run(c, torch.float64, 1).prog_host()
        assert np.max(np.abs(on["gs_upper"] - off["gs_upper"]) + np.abs(on["gs_lower"] - off["gs_lower"]).max()) > 1e-6


def _ns(d):
    root = types.SimpleNamespace()
    for path, v in d.items():
        obj = root
        *head, last = path.split(".")
        for h in head:
            if not hasattr(obj, h):
                setattr(obj, h, types.SimpleNamespace())
            obj = getattr(obj, h)
        setattr(obj, last, v)
    return root


def _mock_x3(c):
    """State, constants and parameters with the reference's attribute paths, the
    switches of the case's flags set as the reference's StomataParams fields."""
    from ibis_b200 import params as prm
    P = c.params
    leaves = {}
    for f in L.PROG + L.STAT:
        if f.leaf.startswith(("methane.", "sim.")):
            continue
        src = c.prog if f in L.PROG else c.stat
        if f.name in src:
            leaves["state." + f.leaf] = np.asarray(src[f.name], dtype=np.float64).copy()
    leaves["state.vegetation.nytimes"] = np.float64(c.prog["nytimes"][0])
    for f in L.FORC:
        leaves["state." + f.leaf] = np.asarray(c.forc[f.name][0], dtype=np.float64)
    for f in L.DIAG:
        leaves.setdefault("state." + f.leaf, np.zeros((c.ncell, f.k)) if f.k > 1 else np.zeros(c.ncell))
    for name, path in dropin.PARAM_PATHS.items():
        v = np.asarray(getattr(P, name), dtype=np.float64)
        if name == "hsoi":
            v = np.concatenate([v, [0.0]])
        if name == "froot":
            v = v.reshape(6, 2)
        leaves[path] = v if v.size > 1 else float(v)
    sp = "params.stomata_params."
    for name, flag in dropin.SWITCH_FLAGS.items():
        leaves[sp + name] = bool(P.flags & flag)
    leaves[sp + "acclim_on"] = bool(P.flags & prm.FLAG_ACCLIM)
    leaves[sp + "frost_on"] = bool(P.flags & prm.FLAG_FROST)
    leaves[sp + "acclim_pfts"] = tuple(int(k) for k in np.flatnonzero(P.acclim_mask))
    leaves[sp + "acclim_per_pft"] = True
    leaves[sp + "acclim_s0_pft"] = np.asarray(P.acclim_s0_pft)
    leaves[sp + "acclim_smax_pft"] = np.asarray(P.acclim_smax_pft)
    leaves["params.h2o_consistent_weights"] = bool(P.flags & prm.FLAG_H2O_CONSISTENT)
    for f in L.STAT:
        if f.leaf.startswith("sim.") and f.name in c.stat:
            leaves["params." + f.leaf[4:]] = np.asarray(c.stat[f.name], dtype=np.float64)
    tree = _ns(leaves)
    if not P.flags & prm.FLAG_CROP:
        tree.params.cropfrac = None
    return tree.state, tree.consts, tree.params


@pytest.mark.parametrize("name", X3_CASES)
def test_dropin_step_matches_reference_with_switches(cuda_lib, name):
    """The drop-in ``timestep_body`` over reference-shaped objects carrying the
    switches (and the seasonal state, td, cropland share and organic fraction
    as the reference holds them) equals the reference's step."""
    c = Case(name)
    state, consts, params = _mock_x3(c)
    P = dropin.step_params(state, consts, params, c.params.dtime)
    assert P.flags == c.params.flags & ~(prm_run_flags()), (bin(P.flags), bin(c.params.flags))
    for h in range(c.record[1] if len(c.record) > 1 else 1):
        for f in L.FORC:
            state = dropin.tree_set(state, f.leaf, np.asarray(c.forc[f.name][h], dtype=np.float64))
        state = dropin.timestep_body(state, consts, params, c.params.dtime)
        if h + 1 in c.record:
            got = {f.name: np.asarray(dropin._get({"s": state}, "s." + f.leaf)) for f in L.PROG}
            got["nytimes"] = np.full(c.ncell, float(got["nytimes"]))
            assert not compare(got, c.out(h + 1, "prog"), 1e-9), h + 1


def prm_run_flags():
    from ibis_b200 import params as prm
    return prm.FLAG_ACC | prm.FLAG_CH4 | prm.FLAG_SOIL_MEANS | prm.FLAG_KAHAN | prm.FLAG_ETPARTS
