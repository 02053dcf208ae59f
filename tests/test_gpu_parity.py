"""CUDA hourly step against the CPU oracle and the reference's golden fixtures.

Tolerances:
* float64 kernels vs the float64 oracle: relative 1e-9 per field after 1 and
  6 steps on every golden case, with absolute floors for near-zero fields
  (tests/goldens.py:FLOORS).  Cells may differ only where a threshold branch of
  the reference flips on last-bit differences; none does on these cases.
* FP32 kernels (FP64 canopy and soil-water solves) vs the float64 oracle
  after one step, every cell: temperatures within 5 mK, soil water and ice
  within 1e-5, snow and puddle stores within their own small bounds -- a small
  multiple of the measured departure (at most 1.1 mK on the realistic
  restart_1996 state, 0.2 mK on the synthetic cases; the reference's own
  float32 run departs from its float64 run by up to 1.6 K hourly in canopy
  temperature over a year, docs/technote/17_numerics_verification.md:367-383).
* After several hours, cells sitting on a phase-change threshold in the
  realistic restart_1996 state are exempt (tests/goldens.py:THRESHOLD_CELLS).
"""
import warnings

import numpy as np
import pytest
import torch

import oracle
from goldens import CASES, MULTI_HOUR_RTOL, THRESHOLD_CELLS, Case, compare, compare_cells
from ibis_b200 import layout as L
from ibis_b200.columns import Columns

warnings.filterwarnings("ignore", category=RuntimeWarning)
pytestmark = pytest.mark.gpu


def _run_gpu(c: Case, dtype, nstep, diag=True):
    cols = Columns.from_host(c.prog, c.stat, dtype=dtype, diag=diag, acc=True)
    P = c.params.copy()
    if dtype == torch.float64:
        P.flags = P.flags & ~(1 << 8)   # plain summation in float64
    forc = cols.forcing(c.forc, 0, nstep)
    cols.run(forc, P)
    torch.cuda.synchronize()
    return cols


def _run_oracle(c: Case, nstep):
    prog = {k: v.copy() for k, v in c.prog.items()}
    acc = oracle.new_acc(c.ncell)
    with np.errstate(all="ignore"):
        for h in range(nstep):
            prog, D, acc = oracle.step(prog, c.stat, c.forcing_at(h), c.params, acc)
    return prog, D, acc


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("nstep", [1, 6])
def test_f64_kernel_matches_oracle(cuda_lib, name, nstep):
    c = Case(name)
    cols = _run_gpu(c, torch.float64, nstep)
    prog, D, acc = _run_oracle(c, nstep)
    n_ex = THRESHOLD_CELLS.get(name, 0) if nstep > 1 else 0
    rtol = MULTI_HOUR_RTOL.get(name, 1e-9) if nstep > 1 else 1e-9
    bad, ex = compare_cells({**cols.prog_host(), **cols.diag_host()}, {**prog, **D}, rtol, n_ex)
    assert not bad, bad[:6]
    assert not cols.nonfinite()[0]


@pytest.mark.parametrize("name", CASES)
def test_f64_kernel_matches_reference_golden(cuda_lib, name):
    c = Case(name)
    h = c.record[-1]
    cols = _run_gpu(c, torch.float64, h)
    bad, ex = compare_cells({**cols.prog_host(), **cols.diag_host()}, {**c.out(h, "prog"), **c.out(h, "diag")},
                            MULTI_HOUR_RTOL.get(name, 1e-9), THRESHOLD_CELLS.get(name, 0))
    assert not bad, bad[:6]


def test_f64_kernel_day_accumulators_match_reference(cuda_lib):
    c = Case("day_mixed")
    cols = _run_gpu(c, torch.float64, 24, diag=False)
    got = cols.acc_host(compensated=False)
    assert not compare(got, c.day("acc"), 1e-6)


@pytest.mark.parametrize("name", CASES)
def test_f32_kernel_close_to_oracle(cuda_lib, name):
    c = Case(name)
    cols = _run_gpu(c, torch.float32, 1)
    prog, D, acc = _run_oracle(c, 1)
    got = cols.prog_host()
    for k, bound in FP32_ONE_HOUR.items():
        g = np.asarray(got[k], np.float64).reshape(prog[k].shape)
        err = float(np.max(np.abs(g - prog[k])))
        assert err <= bound, (k, err, bound)


# FP32 vs float64 after one hour, absolute, every cell: about 5x the largest
# departure measured over the golden cases (temperatures K, stores kg m-2 or
# fractions)
FP32_ONE_HOUR = {
    **{k: 5e-3 for k in ("tsoi", "tg", "tu", "ts", "tl", "t12", "t34", "tsno", "ti", "tsoi_deep")},
    "wsoi": 1e-5, "wisoi": 1e-5, "fi": 2e-6, "hsno": 3e-5, "wpud": 5e-4, "wipud": 2e-5, "q12": 2e-6, "q34": 2e-6,
}


@pytest.mark.parametrize("name", ["day_mixed", "sunshade"])
def test_split_form_matches_fused_form(cuda_lib, name):
    """The two-kernel form runs the same phases; FP32 results agree to rounding."""
    c = Case(name)
    out = {}
    for mode in ("fused", "split"):
        cols = Columns.from_host(c.prog, c.stat, dtype=torch.float32, diag=True, acc=True, mode=mode)
        cols.run(cols.forcing(c.forc), c.params)
        torch.cuda.synchronize()
        out[mode] = (cols.prog_host(), cols.acc_host())
    for k in ("tsoi", "tg", "tu", "tl", "tsno", "ti"):
        np.testing.assert_allclose(out["split"][0][k], out["fused"][0][k], rtol=1e-4, atol=0.05, err_msg=k)
    for k in ("wsoi", "wisoi", "fi"):
        np.testing.assert_allclose(out["split"][0][k], out["fused"][0][k], rtol=1e-3, atol=1e-4, err_msg=k)


@pytest.mark.parametrize("chunk", [1, 5, 24, "auto"])
def test_run_from_host_matches_device_run(cuda_lib, chunk):
    """Forcing streamed from pinned host memory in chunks gives the same bits as
    the same hours from device memory (the same kernel per hour; state and
    Kahan terms are stored and reloaded exactly between chunks)."""
    c = Case("day_mixed")
    a = Columns.from_host(c.prog, c.stat, dtype=torch.float32, acc=True)
    b = Columns.from_host(c.prog, c.stat, dtype=torch.float32, acc=True)
    forc = a.forcing(c.forc)
    a.run(forc, c.params)
    b.run_from_host(forc.cpu().pin_memory(), c.params, chunk=chunk)
    torch.cuda.synchronize()
    assert torch.equal(a.prog, b.prog) and torch.equal(a.acc, b.acc)


@pytest.mark.parametrize("nstep", [1, 24])
def test_plain_entry_matches_its_configuration(cuda_lib, nstep):
    """ibis_step_f32 (no configuration argument) gives the same bits as
    ibis_step_config_f32 with the configuration it takes for that launch
    length: block 224 with on-chip accumulators for a day, the default
    configuration for one hour."""
    import ctypes
    from ibis_b200 import lib
    c = Case("day_mixed")
    so = lib.load()
    out = []
    for how in ("plain", "config"):
        cols = Columns.from_host(c.prog, c.stat, dtype=torch.float32, acc=True)
        forc = cols.forcing(c.forc, 0, nstep)
        p = ctypes.byref(c.params.to_c())
        ptr = lambda t: ctypes.c_void_p(t.data_ptr())
        s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        if how == "plain":
            rc = so.ibis_step_f32(ptr(cols.prog), ptr(cols.stat), ptr(forc), ctypes.c_void_p(0), ptr(cols.acc),
                                  cols.ncell, cols.ld, nstep, p, ptr(cols.status), s)
        else:
            rc = so.ibis_step_config_f32(ptr(cols.prog), ptr(cols.stat), ptr(forc), ctypes.c_void_p(0),
                                         ptr(cols.acc), ctypes.c_void_p(0), cols.ncell, cols.ld, nstep, p,
                                         ptr(cols.status), s, 6 if nstep >= 4 else 0)
        assert rc == 0
        torch.cuda.synchronize()
        out.append((cols.prog.clone(), cols.acc.clone()))
    assert torch.equal(out[0][0], out[1][0]) and torch.equal(out[0][1], out[1][1])


def test_f32_day_accumulators_close_to_reference(cuda_lib):
    """The FP32 fused day (24 hours in one launch, accumulators and their Kahan
    terms on chip) against the reference's float64 day: every accumulator the
    day loop keeps (daily sums, annual sums, hourly CH4, soil means) within
    1e-3 of its plane's largest magnitude on 90 % of the cells, and the soil
    means within 1e-4 relative everywhere (the FP32 step's own departure in soil
    water is ~2e-5 after a day)."""
    c = Case("day_mixed")
    cols = _run_gpu(c, torch.float32, 24, diag=False)
    got, want = cols.acc_host(), c.day("acc")
    for k, w in want.items():
        g = np.asarray(got[k], np.float64).reshape(w.shape)
        scale = max(float(np.abs(w).max()), 1e-30)
        cells = np.abs(g - w).reshape(w.shape[0], -1).max(axis=1) <= 1e-3 * scale
        assert cells.mean() >= 0.9, (k, float(cells.mean()))
    for k in ("tsoi_mean", "wsoi_mean", "tg_mean"):
        w = want[k]
        np.testing.assert_allclose(np.asarray(got[k]).reshape(w.shape), w, rtol=1e-4, atol=1e-5, err_msg=k)


def test_et_and_nee_parts_match_reference(cuda_lib):
    """The optional ET and NEE components summed by the step (FLAG_ETPARTS,
    FLAG_NEEPARTS) against the reference's day with those modules attached:
    float64 kernel within 1e-6 (as the other accumulators); the FP32 fused day
    (on-chip accumulators) within 1e-3 of each plane's largest magnitude on 90 %
    of the cells, its four ET parts summing to its AET."""
    import os
    from ibis_b200.params import FLAG_ETPARTS, FLAG_NEEPARTS
    c = Case("day_mixed")
    z = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "day_parts.npz"))
    parts = ("et_trans", "et_interc", "et_soilev", "et_snowsub", "nee_night", "nee_day")
    want = {k: z["day.acc." + k] for k in parts}
    for dtype in (torch.float64, torch.float32):
        P = c.params.copy()
        P.flags |= FLAG_ETPARTS | FLAG_NEEPARTS
        if dtype == torch.float64:
            P.flags &= ~(1 << 8)
        cols = Columns.from_host(c.prog, c.stat, dtype=dtype, acc=True)
        cols.run(cols.forcing(c.forc), P)
        torch.cuda.synchronize()
        got = cols.acc_host()
        if dtype == torch.float64:
            assert not compare({k: got[k] for k in parts}, want, 1e-6)
            continue
        for k in parts:
            scale = max(float(np.abs(want[k]).max()), 1e-30)
            assert np.mean(np.abs(got[k] - want[k]) <= 1e-3 * scale) >= 0.9, k
        et = got["et_trans"] + got["et_interc"] + got["et_soilev"] + got["et_snowsub"]
        np.testing.assert_allclose(et, got["adaet"], rtol=1e-5, atol=1e-5)
