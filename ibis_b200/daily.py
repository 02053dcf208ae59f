"""The day loop on the device: daily cadence around the hourly steps.

The reference's GSWP3 driver advances the state one day at a time
(``_run_month_scan._day_body``, python-port/ibis/timestepping/loops_gswp3.py:382-608):
phenology and the zeroing of the daily sums, the day's 24 hourly steps with
their accumulators, then the 10-day means, annual sums, decomposition factors
and one day of soil C/N.  :class:`DayLoop` keeps that whole day on the GPU:

    ibis_day_begin  ->  ibis_diurnal_f32 (24 hours of forcing from the day's
    weather)  ->  ibis_step (24 hours, accumulators on)  ->  ibis_day_end

four launches per day with no host round trip, the daily-cadence state
(``layout.DAYST``: phenology, 10-day means, annual sums, litter and soil
carbon) resident beside the columns.  Seasonal formulations, the stress
accumulator, crop and slot types are off, as in the reference's defaults.

:meth:`DayLoop.run_month` adds the month's wetland methane
(``ibis_month_begin`` / ``ibis_month_end``: ``methane_step`` or
``methane_step_from_mean``, optionally ``scale_month`` and the carbon
partition, python-port/ibis/bgc/methane.py:431-496) over the ``layout.WET``
planes.
"""
from __future__ import annotations

import copy
import ctypes

import numpy as np
import torch

from . import layout as L
from . import lib as _lib
from . import restart as _restart
from . import synth
from .columns import Columns
from .forcing import OBSERVED_FIRA, hourly_forcing
from .params import FLAG_ACC, FLAG_CH4, FLAG_ETPARTS, FLAG_NEEPARTS, DayParams, StepParams

_TD = L.OFF["DAILY"]["td"][0]
MONTH_NEW_YEAR, MONTH_FROM_MEAN, MONTH_PARTITION = 1, 2, 4


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


class DayLoop:
    """Days of the reference's day loop on ``cols``.

    ``params`` is the hourly step's record (accumulators are switched on),
    ``day_params`` the phenology and soil-biogeochemistry constants, ``dayst``
    the daily-cadence state as a dict of per-cell arrays named as
    ``layout.DAYST`` (a checkpoint supplies it; see :meth:`from_restart`).
    ``lat`` (degrees), ``seed``, ``jday`` (day of year of the next day) and
    ``day`` (its counter for the variates) drive the forcing generator; ``lat``
    and ``jday`` also give the day length of the seasonal states, which advance
    with ``day_params.seasonal_on`` (the growing-season stress sums with
    ``day_params.stress_on``)."""

    def __init__(self, cols: Columns, params: StepParams, day_params: DayParams, dayst: dict, lat=None,
                 seed: int = 0, jday: int = 1, day: int = 0, dtime: float = 3600.0, observed_fira: bool = True):
        if cols.acc is None:
            raise ValueError("the day loop needs the columns' accumulators")
        self.cols = cols
        self.params = params.copy()
        self.params.flags |= FLAG_ACC
        self.day_params = copy.deepcopy(day_params)
        n, ld = cols.ncell, cols.ld
        if self.day_params.seasonal_on and lat is None:
            raise ValueError("the seasonal states need the cells' latitudes (lat=)")
        lat = np.zeros(n) if lat is None else np.asarray(lat, dtype=np.float64)
        dayst = dict(dayst, latitude=np.deg2rad(lat))
        self.dayst = torch.from_numpy(synth.to_planes("DAYST", dayst, ld, cols._np_dtype)).to(cols.device)
        # the hourly steps read the acclimation state from their own STAT plane
        # (IBIS_FLAG_ACCLIM); ibis_day_begin refreshes it each day it advances
        if "acclim_x" in dayst:
            p_ax = L.OFF["STAT"]["acclim_x"][0]
            cols.stat[p_ax] = self.dayst[L.OFF["DAYST"]["acclim_x"][0]]
        lat_planes = np.zeros(ld, dtype=np.float32)
        lat_planes[:n] = lat
        self.lat = torch.from_numpy(lat_planes).to(cols.device)
        self.seed, self.jday, self.day, self.dtime = int(seed), int(jday), int(day), float(dtime)
        self.observed_fira = bool(observed_fira)
        self.nh = int(round(86400.0 / self.dtime))
        self._forc = None
        self._td = torch.zeros(ld, dtype=cols.dtype, device=cols.device)
        lib = _lib.load()
        f32 = cols.dtype == torch.float32
        self._begin = lib.ibis_day_begin_f32 if f32 else lib.ibis_day_begin_f64
        self._end = lib.ibis_day_end_f32 if f32 else lib.ibis_day_end_f64
        self._mbegin = lib.ibis_month_begin_f32 if f32 else lib.ibis_month_begin_f64
        self._mend = lib.ibis_month_end_f32 if f32 else lib.ibis_month_end_f64
        self.wet = torch.zeros((L.N_WET, ld), dtype=cols.dtype, device=cols.device)
        self.checkpoint = None          # (leaves, meta, extra) of the checkpoint the loop started from

    @classmethod
    def from_restart(cls, path: str, dtype=torch.float32, device="cuda", params: StepParams | None = None,
                     day_params: DayParams | None = None, **kw):
        """A day loop seeded from a reference checkpoint: the columns, the
        daily-cadence state, the running sums, and the last hour's soil-water
        stress the next day's phenology reads, and the optional modules the
        checkpoint carries -- wetland CH4 state, stress sums, ET and NEE parts,
        seasonal states -- which then keep advancing (:meth:`save` writes them
        all back)."""
        cols, P, leaves, meta, extra = _restart.columns_from_restart(path, dtype=dtype, device=device,
                                                                     params=params, acc=True)
        n = cols.ncell
        # the annual sums and the last hour's stress carry on from the file; the
        # a10anc* leaves hold 10-day means between days (DAYST), not sums
        acc0 = _restart.group_from_leaves(leaves, "ACC", n)
        cols.set_acc({k: v for k, v in acc0.items() if not k.startswith("a10anc")})
        dayst = _restart.group_from_leaves(leaves, "DAYST", n)
        # the optional modules the checkpoint carries keep advancing
        DP = copy.deepcopy(day_params or DayParams())
        DP.seasonal_on = float("seasonal.acclim_x" in leaves)
        DP.stress_on = float("stress.nday" in leaves)
        P.flags |= (FLAG_ETPARTS if "etparts.trans" in leaves else 0) | \
            (FLAG_NEEPARTS if "neeparts.night" in leaves else 0)
        loop = cls(cols, P, DP, dayst, **kw)
        if "wetland.flux" in leaves:
            loop.set_wet(_restart.group_from_leaves(leaves, "WET", n))
        loop.checkpoint = (leaves, meta, extra)
        return loop

    # the STAT fields the daily cadence rewrites
    _STAT_WRITTEN = ("frac", "lai", "ztop", "zbot", "tco2mic")

    def save(self, path: str, leaves: dict | None = None, meta=None, extra=None):
        """Write the state after the last day as a reference checkpoint: the
        prognostic state, the canopy structure and respiration the cadence
        rewrites, the daily and annual sums and the last hour's stress, and the
        daily-cadence state (phenology, 10-day means, carbon pools), into the
        leaves of ``leaves`` (default: the checkpoint the loop started from);
        every other leaf is carried over."""
        if leaves is None:
            if getattr(self, "checkpoint", None) is None:
                raise ValueError("no checkpoint leaves to write into: pass leaves=")
            leaves, meta0, extra0 = self.checkpoint
            if meta is None:
                meta = meta0
            elif _restart.TREEDEF_KEY in meta0:      # keep the checkpoint's tree structure with the caller's meta
                meta = {**meta, _restart.TREEDEF_KEY: meta0[_restart.TREEDEF_KEY]}
            extra = extra0 if extra is None else extra
        c = self.cols
        stat = synth.from_planes("STAT", c.stat.cpu().numpy(), c.ncell)
        acc = c.acc_host()
        # between days the reference keeps the 10-day means in the leaves the
        # step uses for daily sums: the DAYST values go last and win
        acc = {k: v for k, v in acc.items() if not k.startswith("a10anc")}
        wet = self.wet_host() if "wetland.flux" in leaves else {}
        groups = [("PROG", c.prog_host()), ("STAT", {k: stat[k] for k in self._STAT_WRITTEN}), ("ACC", acc),
                  ("WET", {k: v for k, v in wet.items() if k != "rh0"}),
                  ("DAYST", self.dayst_host())]
        _restart.write_state(path, leaves, groups, meta, extra)

    # ------------------------------------------------------------------ state
    def dayst_host(self) -> dict:
        return synth.from_planes("DAYST", self.dayst.cpu().numpy(), self.cols.ncell)

    def set_dayst(self, dayst: dict):
        """Replace the daily-cadence state; the latitude plane is kept unless given."""
        a = synth.to_planes("DAYST", {"latitude": self.dayst_host()["latitude"], **dayst}, self.cols.ld,
                            self.cols._np_dtype)
        self.dayst.copy_(torch.from_numpy(a))

    def wet_host(self) -> dict:
        return synth.from_planes("WET", self.wet.cpu().numpy(), self.cols.ncell)

    def set_wet(self, wet: dict):
        a = synth.to_planes("WET", wet, self.cols.ld, self.cols._np_dtype)
        self.wet.copy_(torch.from_numpy(a))

    # ------------------------------------------------------------------ steps
    def begin(self, td: torch.Tensor, stream=None):
        """Phenology and the zeroing of the daily sums (``td``: the day's mean air temperature plane)."""
        c = self.cols
        stream = stream or torch.cuda.current_stream(c.device)
        self.day_params.jday = float(self.jday)
        rc = self._begin(_ptr(c.stat), _ptr(self.dayst), _ptr(c.acc), _ptr(td), c.ncell, c.ld,
                         ctypes.byref(self.params.to_c()), ctypes.byref(self.day_params.to_c()),
                         ctypes.c_void_p(stream.cuda_stream))
        _lib.check(rc, "ibis_day_begin")

    def end(self, td: torch.Tensor, stream=None):
        """10-day means, annual sums, decomposition factors, soil C/N and respiration sums."""
        c = self.cols
        stream = stream or torch.cuda.current_stream(c.device)
        rc = self._end(_ptr(c.prog), _ptr(c.stat), _ptr(self.dayst), _ptr(c.acc), _ptr(td), c.ncell, c.ld,
                       ctypes.byref(self.params.to_c()), ctypes.byref(self.day_params.to_c()),
                       ctypes.c_void_p(stream.cuda_stream))
        _lib.check(rc, "ibis_day_end")

    def run_day(self, daily: torch.Tensor, forc: torch.Tensor | None = None, td: torch.Tensor | None = None,
                stream=None, sw_obs: torch.Tensor | None = None, use: torch.Tensor | None = None):
        """One day: ``daily`` is the day's weather ``(N_DAILY, ld)`` float32 on
        the device.  The hourly forcing is generated from it unless ``forc``
        (``(24, N_FORC, ld)`` in the columns' dtype) is given; the day's mean
        temperature is its ``td`` plane unless ``td`` (``(ld,)`` in the
        columns' dtype) is given.  ``sw_obs`` ``(24, ld)`` and ``use``
        ``(ld,)``: the day's observed hourly shortwave and the cells that use it."""
        c = self.cols
        stream = stream or torch.cuda.current_stream(c.device)
        if daily.shape != (L.N_DAILY, c.ld) or daily.dtype != torch.float32 or daily.device != c.device:
            raise ValueError(f"daily weather must be a ({L.N_DAILY}, {c.ld}) float32 tensor on the columns' device")
        with torch.cuda.stream(stream):
            self._td.copy_(daily[_TD] if td is None else td)
            self.begin(self._td, stream)
            if forc is None:
                if self._forc is None:
                    self._forc = torch.empty((self.nh, L.N_FORC, c.ld), dtype=torch.float32, device=c.device)
                hourly_forcing(daily[None], self.lat, c.ncell, jday0=self.jday, day0=self.day, seed=self.seed,
                               dtime=self.dtime, observed_fira=self.observed_fira, out=self._forc, stream=stream,
                               sw_obs=None if sw_obs is None else sw_obs[None],
                               use=None if use is None else use[None])
                forc = self._forc if c.dtype == torch.float32 else self._forc.to(c.dtype)
            c.run(forc, self.params, stream=stream)
            self.end(self._td, stream)
        self.jday = self.jday % 365 + 1
        self.day += 1
        return self

    def begin_month(self, new_year: bool = False, stream=None):
        """Zero the CH4 accumulator and keep ayco2mic for the carbon partition;
        ``new_year`` clears the annual sums first (reset_annual)."""
        c = self.cols
        stream = stream or torch.cuda.current_stream(c.device)
        rc = self._mbegin(_ptr(c.acc), _ptr(self.wet), _ptr(self.dayst), c.ncell, c.ld,
                          MONTH_NEW_YEAR if new_year else 0, ctypes.c_void_p(stream.cuda_stream))
        _lib.check(rc, "ibis_month_begin")

    def end_month(self, ndays: int, from_mean: bool = True, scale: torch.Tensor | None = None,
                  partition: bool = False, stream=None):
        """The month's methane step; ``scale`` is an optional ``(ld,)`` inundated
        fraction in the columns' dtype (scale_month)."""
        c = self.cols
        stream = stream or torch.cuda.current_stream(c.device)
        if from_mean and not self.params.flags & FLAG_CH4:
            raise ValueError("the month's mean flux needs the hourly CH4 accumulator (FLAG_CH4)")
        if scale is not None and (scale.shape != (c.ld,) or scale.dtype != c.dtype or scale.device != c.device):
            raise ValueError(f"scale must be a ({c.ld},) tensor of the columns' dtype and device")
        flags = (MONTH_FROM_MEAN if from_mean else 0) | (MONTH_PARTITION if partition else 0)
        rc = self._mend(_ptr(c.prog), _ptr(c.stat), _ptr(c.acc), _ptr(self.wet), _ptr(self.dayst),
                        ctypes.c_void_p(0) if scale is None else _ptr(scale), c.ncell, c.ld, int(ndays),
                        ctypes.byref(self.params.to_c()), flags, ctypes.c_void_p(stream.cuda_stream))
        _lib.check(rc, "ibis_month_end")

    def run_month(self, daily: torch.Tensor, from_mean: bool = True, scale: torch.Tensor | None = None,
                  partition: bool = False, new_year: bool = False, stream=None):
        """A calendar month (``daily``: ``(ndays, N_DAILY, ld)``) and its wetland methane."""
        self.begin_month(new_year, stream)
        self.run(daily, stream)
        self.end_month(daily.shape[0], from_mean, scale, partition, stream)
        return self

    def run(self, daily: torch.Tensor, stream=None):
        """``daily``: ``(nday, N_DAILY, ld)`` float32 on the device, one day after another."""
        for d in range(daily.shape[0]):
            self.run_day(daily[d], stream=stream)
        return self


__all__ = ["DayLoop", "OBSERVED_FIRA"]
