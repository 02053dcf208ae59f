"""The step from host buffers (``ibis_step_host_f32`` through
``Columns.run_host``): the columns cut into groups and the hours into chunks,
each piece's forcing copied in, stepped and copied out on the library's streams.

The groups and chunks of hours run the same kernels on the same columns as
one launch over every column and hour, so the state, the accumulators and the
state copied to the host equal that launch's bit for bit, whatever the group
size (several groups per compute stream included) and chunk length (the
caller's Columns fix the launch configuration for all of them).  A column
made non-finite in a late group is reported in the caller's numbering of the
columns.  Every loop of the step has a fixed trip count and its two
float-to-int conversions read static soil inputs, so a NaN in the forcing
stays data: it propagates into that column and is flagged.
"""
import numpy as np
import pytest
import torch

from ibis_b200 import synth
from ibis_b200.columns import Columns
from ibis_b200.params import StepParams, FLAG_ACC, FLAG_CH4, FLAG_KAHAN

pytestmark = pytest.mark.gpu

NCELL, HOURS = 5000, 6


def _workload(seed=3):
    rng = np.random.Generator(np.random.PCG64(seed))
    stat = synth.make_columns(rng, NCELL)
    forc = synth.make_forcing(rng, rng.uniform(-40.0, 70.0, NCELL), HOURS, start_doy=172)
    prog = synth.make_initial(rng, stat, {k: v[0] for k, v in forc.items()})
    P = StepParams(co2conc=390.0e-6)
    P.flags |= FLAG_ACC | FLAG_CH4 | FLAG_KAHAN
    return prog, stat, forc, P


def _columns(prog, stat):
    return Columns.from_host(prog, stat, dtype=torch.float32, acc=True)


@pytest.mark.parametrize("group,chunk", [(0, 0), (256, 0), (640, 0), (4992, 0), (5024, 2), (640, 3), (0, 1)])
def test_host_groups_equal_one_launch(cuda_lib, group, chunk):
    prog, stat, forc, P = _workload()
    ref = _columns(prog, stat)
    ref.run(ref.forcing(forc), P)
    cols = _columns(prog, stat)
    h_forc = torch.from_numpy(synth.forcing_planes(forc, cols.ld)).pin_memory()
    h_prog = torch.zeros_like(cols.prog, device="cpu").pin_memory()
    stream = torch.cuda.Stream()
    cols.run_host(h_forc, P, host_prog=h_prog, group=group, chunk=chunk, stream=stream)
    stream.synchronize()
    torch.cuda.synchronize()
    np.testing.assert_array_equal(cols.prog.cpu().numpy(), ref.prog.cpu().numpy())
    np.testing.assert_array_equal(cols.acc.cpu().numpy(), ref.acc.cpu().numpy())
    np.testing.assert_array_equal(h_prog.numpy()[:, :NCELL], ref.prog.cpu().numpy()[:, :NCELL])
    assert not cols.nonfinite()[0]


def test_host_step_reports_cells_in_caller_numbering(cuda_lib):
    prog, stat, forc, P = _workload()
    bad = 3301                                         # in the sixth group of 640 cells
    forc = {k: v.copy() for k, v in forc.items()}
    forc["ta"][2, bad] = np.nan
    cols = _columns(prog, stat)
    h_forc = torch.from_numpy(synth.forcing_planes(forc, cols.ld)).pin_memory()
    cols.run_host(h_forc, P, group=640)
    torch.cuda.synchronize()
    flagged, first = cols.nonfinite()
    assert flagged and first == bad


@pytest.mark.parametrize("group,fira", [(0, False), (640, True), (4992, False)])
def test_host_days_from_daily_weather_equal_the_device_path(cuda_lib, group, fira):
    """``ibis_day_host_f32`` (``Columns.run_host_daily``): per group the daily
    weather in, the forcing generated (variates keyed by the caller's cell
    numbers), the days stepped and the state out -- equal to generating the
    forcing over every cell (``forcing.hourly_forcing``) and one step launch,
    bit for bit."""
    from ibis_b200 import forcing as _forcing
    prog, stat, forc, P = _workload()
    rng = np.random.default_rng(4)
    nday = 2
    lat = rng.uniform(-60.0, 80.0, NCELL)
    w = synth.make_daily_weather(rng, lat, nday)
    ref = _columns(prog, stat)
    lat_d = torch.zeros(ref.ld, dtype=torch.float32, device="cuda")
    lat_d[:NCELL] = torch.from_numpy(lat.astype(np.float32)).cuda()
    planes = _forcing.daily_planes(w, ref.ld)
    f = _forcing.hourly_forcing(torch.from_numpy(planes).cuda(), lat_d, NCELL, jday0=100, day0=7, seed=11,
                                observed_fira=fira)
    ref.run(f, P)
    cols = _columns(prog, stat)
    h_prog = torch.zeros_like(cols.prog, device="cpu").pin_memory()
    stream = torch.cuda.Stream()
    cols.run_host_daily(torch.from_numpy(planes).pin_memory(), lat_d, P, 100, day0=7, seed=11, observed_fira=fira,
                        host_prog=h_prog, group=group, stream=stream)
    stream.synchronize()
    torch.cuda.synchronize()
    np.testing.assert_array_equal(cols.prog.cpu().numpy(), ref.prog.cpu().numpy())
    np.testing.assert_array_equal(cols.acc.cpu().numpy(), ref.acc.cpu().numpy())
    np.testing.assert_array_equal(h_prog.numpy()[:, :NCELL], ref.prog.cpu().numpy()[:, :NCELL])
