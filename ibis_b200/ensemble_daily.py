"""Calibration ensembles with the daily cadence: runs whose vegetation and soil
carbon evolve (phenology, 10-day means, decomposition, soil C/N) as in the
reference's day loop, all on the GPU.

The reference calibrates a site by scanning its day loop (``_run_month_scan``,
python-port/ibis/timestepping/loops_gswp3.py:346-612) with the candidate's
parameters (verify/calibration/site_fit.py:375-436).  :class:`EnsembleDayLoop`
does that for every (site, parameter vector) run at once, one day at a time:

* the day's hourly forcing of every site from its daily weather
  (``ibis_diurnal_f32``), written as the ensemble's 48-byte hourly records;
* ``ibis_day_begin`` on the run planes (phenology rewrites each run's canopy
  structure, so every run carries its own static planes);
* the day's 24 hours of every run in one persistent launch
  (``ibis_ensemble_f32``: run r's statics are column r, its records the
  site's 24);
* ``ibis_day_end`` on the run planes.

Runs at one site share the site's weather and variates; each run keeps its own
state, accumulators, daily-cadence state and calibration vector.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import layout as L
from . import lib as _lib
from . import synth
from .forcing import daily_planes, hourly_forcing
from .lib import IbisEnsembleC
from .params import FLAG_ACC, DayParams, StepParams

_TD = L.OFF["DAILY"]["td"][0]


def _p(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


class EnsembleDayLoop:
    """``nsite`` sites x ``nparam`` calibration vectors with the daily cadence.

    ``stat``, ``prog`` and ``dayst`` are per-site dicts (layout fields, (nsite, ...)
    arrays), ``daily`` the sites' daily weather (dict of (nday, nsite) arrays
    named as ``layout.DAILY``), ``vectors`` (nparam, N_RUN) calibration vectors
    applied on top of ``params``.  Runs are site-major: run = site * nparam + p."""

    def __init__(self, stat: dict, prog: dict, dayst: dict, daily: dict, lat, vectors, params: StepParams,
                 day_params: DayParams | None = None, seed: int = 0, jday: int = 1, device="cuda"):
        self.device = torch.device(device)
        if self.device.index is None:
            self.device = torch.device("cuda", torch.cuda.current_device())
        dev, f32 = self.device, dict(dtype=torch.float32, device=self.device)
        vectors = np.asarray(vectors, dtype=np.float32)
        self.nsite = int(np.shape(lat)[0])
        self.nparam = vectors.shape[0]
        self.nrun = self.nsite * self.nparam
        self.ld_site = L.leading_dim(self.nsite)
        self.ld_run = L.leading_dim(self.nrun)
        self.site_of_run = np.repeat(np.arange(self.nsite), self.nparam)
        pick = lambda planes: np.ascontiguousarray(planes[:, self.site_of_run])
        run_planes = lambda group, values: np.pad(pick(synth.to_planes(group, values, self.ld_site)),
                                                  ((0, 0), (0, self.ld_run - self.nrun)))
        self.prog = torch.from_numpy(run_planes("PROG", prog)).to(dev)
        self.stat = torch.from_numpy(run_planes("STAT", stat)).to(dev)
        dayst = dict(dayst, latitude=np.deg2rad(np.asarray(lat, np.float64)))    # the seasonal states' day length
        self.dayst = torch.from_numpy(run_planes("DAYST", dayst)).to(dev)
        self.acc = torch.zeros((2 * L.N_ACC, self.ld_run), **f32)
        rp = np.zeros((L.N_RUN, self.ld_run), dtype=np.float32)
        rp[:, :self.nrun] = vectors[np.tile(np.arange(self.nparam), self.nsite)].T
        self.run_params = torch.from_numpy(rp).to(dev)
        self.run_stat = torch.arange(self.nrun, dtype=torch.int32, device=dev)       # statics: each run's own column
        self.run_forc = torch.from_numpy((self.site_of_run * 24).astype(np.int64)).to(dev)
        self.run_nstep = torch.full((self.nrun,), 24, dtype=torch.int32, device=dev)
        self.run_pos = torch.zeros(self.nrun, dtype=torch.int32, device=dev)
        self.queue = torch.zeros(1, dtype=torch.int32, device=dev)
        self.status = torch.tensor([0, 2 ** 31 - 1], dtype=torch.int32, device=dev)
        self.records = torch.zeros((self.nsite * 24, L.N_FORC), **f32)
        self.params = params.copy()
        self.params.flags = (self.params.flags | FLAG_ACC)
        if float(self.params.dtime) != 3600.0:
            raise ValueError("the ensemble day loop runs hourly steps")
        self.day_params = day_params or DayParams()
        self._pc = self.params.to_c()
        self._dpc = self.day_params.to_c()
        self.daily = torch.from_numpy(daily_planes(daily, self.ld_site)).to(dev)
        self.hourly = torch.empty((24, L.N_FORC, self.ld_site), **f32)
        lat_planes = np.zeros(self.ld_site, dtype=np.float32)
        lat_planes[:self.nsite] = lat
        self.lat = torch.from_numpy(lat_planes).to(dev)
        self.site_index = torch.from_numpy(self.site_of_run.astype(np.int64)).to(dev)
        self.td = torch.zeros(self.ld_run, **f32)
        self.seed, self.jday, self.day = int(seed), int(jday), 0
        self.lib = _lib.load()
        self._c = IbisEnsembleC(prog=_p(self.prog), acc=_p(self.acc), stat=_p(self.stat), forc=_p(self.records),
                                run_params=_p(self.run_params), run_site=_p(self.run_stat),
                                run_forc=_p(self.run_forc), run_nstep=_p(self.run_nstep), run_pos=_p(self.run_pos),
                                order=None, yearly=None, forc_len=int(self.records.shape[0]), nrun=self.nrun,
                                ld_run=self.ld_run, nsite=self.nrun, ld_site=self.ld_run, nyear=0, year_steps=24,
                                norder=self.nrun, queue=_p(self.queue), status=_p(self.status))

    @property
    def ndays(self) -> int:
        return int(self.daily.shape[0])

    def run_day(self, stream=None):
        """The next day of every run."""
        d = self.day
        if d >= self.ndays:
            raise ValueError("no daily weather left")
        stream = stream or torch.cuda.current_stream(self.device)
        s = ctypes.c_void_p(stream.cuda_stream)
        with torch.cuda.stream(stream):
            hourly_forcing(self.daily[d:d + 1], self.lat, self.nsite, jday0=self.jday, day0=d, seed=self.seed,
                           observed_fira=True, out=self.hourly, stream=stream)           # (24, N_FORC, ld_site)
            self.records.view(self.nsite, 24, L.N_FORC).copy_(self.hourly[:, :, :self.nsite].permute(2, 0, 1))
            self.td[:self.nrun] = self.daily[d, _TD][self.site_index]
        n, ld = self.nrun, self.ld_run
        self._dpc.jday = float(self.jday)                   # the day length of the seasonal states
        _lib.check(self.lib.ibis_day_begin_f32(_p(self.stat), _p(self.dayst), _p(self.acc), _p(self.td), n, ld,
                                               ctypes.byref(self._pc), ctypes.byref(self._dpc), s), "ibis_day_begin")
        _lib.check(self.lib.ibis_ensemble_f32(ctypes.byref(self._c), ctypes.byref(self._pc), 0, s),
                   "ibis_ensemble_f32")
        _lib.check(self.lib.ibis_day_end_f32(_p(self.prog), _p(self.stat), _p(self.dayst), _p(self.acc), _p(self.td),
                                             n, ld, ctypes.byref(self._pc), ctypes.byref(self._dpc), s),
                   "ibis_day_end")
        with torch.cuda.stream(stream):
            self.run_pos += 24
        self.jday = self.jday % 365 + 1
        self.day += 1
        return self

    def run(self, ndays: int | None = None, stream=None):
        for _ in range(self.ndays - self.day if ndays is None else int(ndays)):
            self.run_day(stream)
        return self

    # ------------------------------------------------------------------ results
    def prog_host(self) -> dict:
        return synth.from_planes("PROG", self.prog.cpu().numpy(), self.nrun)

    def dayst_host(self) -> dict:
        return synth.from_planes("DAYST", self.dayst.cpu().numpy(), self.nrun)

    def acc_host(self) -> dict:
        a = self.acc.cpu().numpy().astype(np.float64)
        return synth.from_planes("ACC", a[:L.N_ACC] - a[L.N_ACC:], self.nrun)

    def nonfinite(self):
        s = self.status.cpu().numpy()
        return bool(s[0] & 1), bool(s[0] & 2), int(s[1])

    def cell_steps(self) -> int:
        return self.nrun * 24 * self.day

