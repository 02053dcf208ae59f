"""Argument checks of the C entry points, on the host: a bad size, stride,
flag or missing buffer returns -EINVAL before anything reaches a GPU, so these
run without one.  The device pointers passed are never dereferenced on the
host; every call here is rejected before a launch."""
import ctypes

import pytest

from ibis_b200 import lib
from ibis_b200.params import DayParams, IbisParamsC, StepParams

EINVAL = -22
DEV = ctypes.c_void_p(256)          # a stand-in device address (never touched)
NUL = ctypes.c_void_p(0)


@pytest.fixture(scope="module")
def so():
    return lib.load()


def _p(**kw):
    P = StepParams()
    for k, v in kw.items():
        setattr(P, k, v)
    return ctypes.byref(P.to_c())


def test_step_rejects_bad_shapes(so):
    p = _p()
    for ncell, ld, nstep in ((-1, 32, 1), (40, 32, 1), (30, 33, 1), (30, 32, -1)):
        assert so.ibis_step_f32(DEV, DEV, DEV, NUL, DEV, ncell, ld, nstep, p, NUL, NUL) == EINVAL
    assert so.ibis_step_f32(NUL, DEV, DEV, NUL, DEV, 30, 32, 1, p, NUL, NUL) == EINVAL
    bad = StepParams().to_c()
    bad.flags = 1 << 30                      # no such variant
    assert so.ibis_step_f32(DEV, DEV, DEV, NUL, DEV, 30, 32, 1, ctypes.byref(bad), NUL, NUL) == EINVAL


def test_host_step_rejects_bad_arguments(so):
    p = _p()
    args = (DEV, DEV, DEV, DEV, NUL, DEV, NUL)
    f = so.ibis_step_host_f32
    assert f(*args, 30, 33, 1, p, NUL, 0, 0, -1, NUL) == EINVAL      # ld not a multiple of 32
    assert f(*args, 40, 32, 1, p, NUL, 0, 0, -1, NUL) == EINVAL      # ncell > ld
    assert f(*args, 30, 32, 1, p, NUL, 48, 0, -1, NUL) == EINVAL     # group not a multiple of 32
    assert f(*args, 30, 32, 1, p, NUL, -32, 0, -1, NUL) == EINVAL
    assert f(*args, 30, 32, 1, p, NUL, 0, -2 ** 31, -1, NUL) == EINVAL   # no such first chunk
    split = next(c["id"] for c in lib.configs() if c["form"] == "split")
    assert f(*args, 30, 32, 1, p, NUL, 0, 0, split, NUL) == EINVAL   # needs scratch
    assert f(*args, 30, 32, 1, p, NUL, 0, 0, 99, NUL) == EINVAL
    assert f(DEV, DEV, NUL, DEV, NUL, DEV, NUL, 30, 32, 1, p, NUL, 0, 0, -1, NUL) == EINVAL
    assert f(DEV, DEV, DEV, NUL, NUL, DEV, NUL, 30, 32, 1, p, NUL, 0, 0, -1, NUL) == EINVAL
    assert f(*args, 0, 32, 1, p, NUL, 0, 0, -1, NUL) == 0             # nothing to do


def test_day_host_rejects_bad_arguments(so):
    p = _p()
    f = so.ibis_day_host_f32
    a = (DEV, DEV, DEV, DEV, DEV, DEV, NUL, DEV, NUL)
    assert f(*a, 30, 33, 1, 1, 0, 0, 0, p, NUL, 0, -1, NUL) == EINVAL          # ld not a multiple of 32
    assert f(*a, 30, 32, 1, 0, 0, 0, 0, p, NUL, 0, -1, NUL) == EINVAL          # day of year 0
    assert f(*a, 30, 32, 1, 1, 0, 0, 4, p, NUL, 0, -1, NUL) == EINVAL          # unknown generator flag
    assert f(*a, 30, 32, 1, 1, 0, 0, 0, _p(dtime=7000.0), NUL, 0, -1, NUL) == EINVAL   # not a whole day of steps
    assert f(DEV, DEV, NUL, DEV, DEV, DEV, NUL, DEV, NUL, 30, 32, 1, 1, 0, 0, 0, p, NUL, 0, -1, NUL) == EINVAL
    assert f(*a, 0, 32, 1, 1, 0, 0, 0, p, NUL, 0, -1, NUL) == 0                # nothing to do


def test_day_kernels_reject_bad_arguments(so):
    p, dp = _p(), ctypes.byref(DayParams().to_c())
    for f in (so.ibis_day_begin_f32, so.ibis_day_begin_f64):
        assert f(DEV, DEV, DEV, DEV, 30, 33, p, dp, NUL) == EINVAL          # ld not a multiple of 32
        assert f(DEV, NUL, DEV, DEV, 30, 32, p, dp, NUL) == EINVAL          # no day-state planes
        assert f(DEV, DEV, DEV, DEV, 64, 32, p, dp, NUL) == EINVAL          # ncell > ld
    for f in (so.ibis_day_end_f32, so.ibis_day_end_f64):
        assert f(NUL, DEV, DEV, DEV, DEV, 30, 32, p, dp, NUL) == EINVAL     # no prognostic planes
        assert f(DEV, DEV, DEV, DEV, DEV, 30, 32, _p(ndaypy=0.0), dp, NUL) == EINVAL
        assert f(DEV, DEV, DEV, DEV, DEV, 30, 32, p, ctypes.byref(DayParams(ddays=0.0).to_c()), NUL) == EINVAL
    assert so.ibis_day_begin_f32(DEV, DEV, DEV, DEV, 0, 32, p, dp, NUL) == 0   # nothing to do


def test_month_kernels_reject_bad_arguments(so):
    p = _p()
    assert so.ibis_month_begin_f32(DEV, DEV, NUL, 30, 32, 8, NUL) == EINVAL           # unknown flag
    assert so.ibis_month_begin_f64(NUL, DEV, NUL, 30, 32, 0, NUL) == EINVAL
    for f in (so.ibis_month_end_f32, so.ibis_month_end_f64):
        assert f(DEV, DEV, DEV, DEV, DEV, NUL, 30, 32, 0, p, 0, NUL) == EINVAL        # ndays < 1
        assert f(DEV, DEV, NUL, DEV, DEV, NUL, 30, 32, 30, p, 2, NUL) == EINVAL       # mean without accumulators
        assert f(DEV, DEV, DEV, DEV, NUL, NUL, 30, 32, 30, p, 4, NUL) == EINVAL       # partition without ayco2mic
        assert f(DEV, DEV, DEV, DEV, DEV, NUL, 30, 32, 30, p, 16, NUL) == EINVAL      # unknown flag


def test_forcing_generator_rejects_bad_arguments(so):
    args = (DEV, DEV, DEV, 30, 32, 2)
    assert so.ibis_diurnal_f32(*args, 0, 0, 3600.0, 1, 0, NUL) == EINVAL            # day of year 0
    assert so.ibis_diurnal_f32(*args, 10, 0, 7000.0, 1, 0, NUL) == EINVAL           # not a whole day of steps
    assert so.ibis_diurnal_f32(*args, 10, 0, 3600.0, 1, 4, NUL) == EINVAL           # unknown flag
    assert so.ibis_diurnal_sw_f32(DEV, DEV, NUL, DEV, DEV, 30, 32, 2, 10, 0, 3600.0, 1, 0, NUL) == EINVAL
    assert so.ibis_diurnal_sw_f32(DEV, DEV, DEV, NUL, DEV, 30, 32, 2, 10, 0, 3600.0, 1, 0, NUL) == EINVAL


def test_ensemble_entries_reject_bad_descriptors(so):
    e = lib.IbisEnsembleC(prog=256, acc=256, stat=256, forc=256, run_params=256, run_site=256, run_forc=256,
                          run_nstep=256, run_pos=None, order=None, yearly=None, forc_len=10, nrun=40, ld_run=32,
                          nsite=1, ld_site=32, nyear=0, year_steps=24, norder=0, queue=256, status=256)
    p = _p()
    assert so.ibis_ensemble_f32(ctypes.byref(e), p, 0, NUL) == EINVAL               # nrun > ld_run
    d = lib.IbisEnsembleDailyC(records=260, site_lat=256, len=4, seed=1, flags=0)    # records not 16-byte aligned
    e.nrun = 20
    assert so.ibis_ensemble_daily_f32(ctypes.byref(e), ctypes.byref(d), p, 0, NUL) == EINVAL
    d.records, d.flags = 256, 2                                                       # unknown flag
    assert so.ibis_ensemble_daily_f32(ctypes.byref(e), ctypes.byref(d), p, 0, NUL) == EINVAL
    d.flags = 0
    assert so.ibis_ensemble_daily_f32(ctypes.byref(e), ctypes.byref(d), _p(dtime=7000.0), 0, NUL) == EINVAL
