"""Calibration ensembles on the GPU: many (site x parameter vector) runs at once.

The reference calibrates one tower site at a time: a CMA-ES loop hands
candidate parameter vectors to host worker processes, each of which applies
the vector to ``SimParams`` (verify/calibration/fit_carbon.py:253-381, 438)
and scans the day loop over the site's record
(verify/calibration/site_fit.py:375-436).  :class:`Ensemble` runs every
candidate at every site in one launch instead:

* a run is one (site, parameter vector) pair with a record of its own length;
* runs at one site share the site's static planes and forcing records;
* each run's 31 calibrated parameters (``layout.RUN``) are a column of the
  ``run_params`` planes; everything else comes from one :class:`StepParams`;
* :meth:`Ensemble.run` is the persistent form (``ibis_ensemble_f32``): warps
  take 32 runs at a time from a device counter, longest records first;
* :meth:`Ensemble.run_hourly` is the plain form: one launch per hour
  (``ibis_ensemble_hours_f32``), optionally captured in a CUDA graph of
  ``chunk`` hours and replayed until the longest record ends;
* with day records (``make_ensemble(..., daily=True)``) the persistent form
  generates each run's hours from its site's daily weather as it steps
  (``ibis_ensemble_daily_f32``: the reference's diurnal algorithm), so the
  forcing held and read is 48 bytes per site-day instead of per site-hour.

Runs are numbered site-major (run = site * nparam + p), so with 32 or 64
parameter vectors every warp's runs share one site and one record length.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import numpy as np
import torch

from . import layout as L
from . import lib as _lib
from . import synth
from .lib import IbisEnsembleC, IbisEnsembleDailyC
from .params import FLAG_ACC, FLAG_CH4, StepParams

YEAR_HOURS = 8760

# StepParams attribute behind each RUN field; rwood/rroot/rgrowth are scalars
# in the calibration vector and fill all 12 plant-type entries.
_SOURCES = {"vmax": "vmax_pft", "coefm": "coefm", "stressfac": "stressfac", "soil_beta_power": "soil_beta_power",
            "wliqumax": "wliqumax", "wliqsmax": "wliqsmax", "wliqlmax": "wliqlmax", "fmax": "fmax",
            "r_ch4": "r_ch4", "q10p": "q10p", "z_tau": "z_tau", "tau_oxid": "tau_oxid", "z_wt_max": "z_wt_max",
            "rwood": "rwood", "rroot": "rroot", "rgrowth": "rgrowth"}
_SCALAR_TABLES = ("rwood", "rroot", "rgrowth")


def default_vector(params: StepParams | None = None) -> np.ndarray:
    """The 31-value calibration vector of ``params`` (float32, ``layout.RUN`` order)."""
    params = StepParams() if params is None else params
    out = []
    for f in L.RUN:
        v = np.asarray(getattr(params, _SOURCES[f.name]), dtype=np.float64).reshape(-1)
        out.extend(v[:1] if f.name in _SCALAR_TABLES else v[:f.k])
    v = np.array(out, dtype=np.float32)
    assert v.size == L.N_RUN
    return v


def draw_vectors(rng, n: int, params: StepParams | None = None, spread: float = 0.5) -> np.ndarray:
    """``n`` vectors, each value log-uniform within +-``spread`` of the default
    (magnitude drawn in [(1-spread)|d|, (1+spread)|d|], sign kept)."""
    d = default_vector(params).astype(np.float64)
    lo, hi = np.log((1.0 - spread) * np.abs(d)), np.log((1.0 + spread) * np.abs(d))
    u = rng.uniform(size=(n, d.size))
    return (np.sign(d) * np.exp(lo + u * (hi - lo))).astype(np.float32)


def apply_vector(params: StepParams, v) -> StepParams:
    """A copy of ``params`` carrying calibration vector ``v`` (the uniform-parameter
    equivalent of one ensemble run)."""
    out = params.copy()
    v = np.asarray(v, dtype=np.float32).astype(np.float64)
    for f in L.RUN:
        p0, k = L.OFF["RUN"][f.name]
        name = _SOURCES[f.name]
        if f.name in _SCALAR_TABLES:
            setattr(out, name, np.full(12, v[p0]))
        elif k > 1:
            setattr(out, name, v[p0:p0 + k])
        else:
            setattr(out, name, float(v[p0]))
    return out


@dataclass
class EnsembleSpec:
    """Host description of an ensemble: per-site inputs and per-run vectors."""
    nsite: int
    nparam: int
    site_hours: np.ndarray            # (nsite,) record length of each site (hours)
    stat: dict                        # per-site static fields (nsite, ...)
    prog: dict                        # per-site initial state (nsite, ...)
    forc: np.ndarray | None           # (total_hours, N_FORC) float32 records, site after site (None: day records)
    site_first: np.ndarray            # (nsite,) first record of each site in ``forc``
    vectors: np.ndarray               # (nparam, N_RUN) float32
    params: StepParams
    latitude: np.ndarray
    meta: dict = field(default_factory=dict)
    daily: np.ndarray | None = None   # (total_days, DAILY_WORDS) day records; then site_first counts days
    weather_seed: int = 0             # key of the daily form's counter-based variates

    @property
    def nrun(self) -> int:
        return self.nsite * self.nparam


def forcing_records(forc: dict) -> np.ndarray:
    """(nhour, N_FORC) float32 records of one cell from a make_forcing dict of (nhour, 1[, k]) arrays."""
    nh = forc["ta"].shape[0]
    out = np.zeros((nh, L.N_FORC), dtype=np.float32)
    for f in L.FORC:
        p0, k = L.OFF["FORC"][f.name]
        v = np.asarray(forc[f.name])
        out[:, p0:p0 + k] = v.reshape(nh, k)
    return out


DAILY_WORDS = 12      # IBIS_DAILY_* words, day of year, two padding words (48 bytes)


def daily_records(daily: dict, jday0: int = 1) -> np.ndarray:
    """(nday, DAILY_WORDS) float32 day records of one site from a dict of (nday,)
    arrays named as ``layout.DAILY``; day d is day of year ((jday0 - 1 + d) mod 365) + 1."""
    nday = np.shape(daily["tmax"])[0]
    out = np.zeros((nday, DAILY_WORDS), dtype=np.float32)
    for f in L.DAILY:
        if f.name in daily:
            out[:, L.OFF["DAILY"][f.name][0]] = np.asarray(daily[f.name]).reshape(nday)
    out[:, L.N_DAILY] = (jday0 - 1 + np.arange(nday)) % 365 + 1
    return out


def make_ensemble(nsite: int, nparam: int, years=(1, 15), seed: int = 0, lat_range=(-40.0, 70.0),
                  year_hours: int = YEAR_HOURS, site_hours=None, alpha: float = 1.0,
                  params: StepParams | None = None, include_default: bool = True,
                  daily: bool = False) -> EnsembleSpec:
    """Seeded synthetic ensemble: ``nsite`` towers with records of U{years} whole
    years (or the explicit ``site_hours``) of hourly forcing, ``nparam``
    calibration vectors drawn log-uniform within +-50% of the defaults (vector 0
    is the default itself when ``include_default``).  With ``daily`` the
    records are days of weather (``synth.make_daily_weather``) for the
    daily form, and ``site_hours`` must be whole days."""
    rng = np.random.Generator(np.random.PCG64(seed))
    params = StepParams(co2conc=390.0e-6) if params is None else params
    lat = rng.uniform(lat_range[0], lat_range[1], size=nsite)
    if site_hours is None:
        site_hours = rng.integers(years[0], years[1] + 1, size=nsite) * year_hours
    site_hours = np.asarray(site_hours, dtype=np.int64).reshape(nsite)
    stat = synth.make_columns(rng, nsite, alpha)
    recs, first, f0 = [], np.zeros(nsite, dtype=np.int64), []
    pos = 0
    if daily and np.any(site_hours % 24):
        raise ValueError("daily records need whole days")
    for s in range(nsite):
        if daily:
            nday = int(site_hours[s]) // 24
            dw = synth.make_daily_weather(rng, lat[s:s + 1], nday)
            recs.append(daily_records({k: v[:, 0] for k, v in dw.items()}, jday0=1))
            fs = synth.make_forcing(rng, lat[s:s + 1], 1, start_doy=1)
            pos_next = pos + nday
        else:
            fs = synth.make_forcing(rng, lat[s:s + 1], int(site_hours[s]), start_doy=1)
            recs.append(forcing_records(fs))
            pos_next = pos + int(site_hours[s])
        f0.append({k: v[0] for k, v in fs.items()})
        first[s] = pos
        pos = pos_next
    F0 = {k: np.concatenate([d[k] for d in f0], axis=0) for k in f0[0]}
    prog = synth.make_initial(rng, stat, F0)
    vec = draw_vectors(rng, nparam, params)
    if include_default and nparam > 0:
        vec[0] = default_vector(params)
    width = DAILY_WORDS if daily else L.N_FORC
    table = np.concatenate(recs, axis=0) if recs else np.zeros((0, width), np.float32)
    return EnsembleSpec(nsite=nsite, nparam=nparam, site_hours=site_hours, stat=stat, prog=prog,
                        forc=None if daily else table, site_first=first, vectors=vec, params=params, latitude=lat,
                        meta=dict(seed=seed, years=years, year_hours=year_hours),
                        daily=table if daily else None, weather_seed=seed)


class Ensemble:
    """Device buffers and launches of one ensemble (FP32 kernels)."""

    def __init__(self, spec: EnsembleSpec, device="cuda", year_steps: int = YEAR_HOURS, acc: bool = True):
        self.spec = spec
        self.device = torch.device(device)
        if self.device.type == "cuda" and self.device.index is None:
            self.device = torch.device("cuda", torch.cuda.current_device())
        self.lib = _lib.load()
        self.nsite, self.nparam, self.nrun = spec.nsite, spec.nparam, spec.nrun
        self.ld_site = L.leading_dim(self.nsite)
        self.ld_run = L.leading_dim(self.nrun)
        self.year_steps = int(year_steps)
        dev, f32 = self.device, torch.float32
        site_of_run = np.repeat(np.arange(self.nsite), self.nparam)
        param_of_run = np.tile(np.arange(self.nparam), self.nsite)
        nstep = spec.site_hours[site_of_run].astype(np.int32)
        self.run_nstep_host = nstep
        self.nyear = int(-(-int(nstep.max(initial=0)) // self.year_steps))
        prog_site = synth.to_planes("PROG", spec.prog, self.ld_site)
        prog0 = np.zeros((L.N_PROG, self.ld_run), dtype=np.float32)
        prog0[:, :self.nrun] = prog_site[:, site_of_run]
        rp = np.zeros((L.N_RUN, self.ld_run), dtype=np.float32)
        rp[:, :self.nrun] = spec.vectors[param_of_run].T
        self.prog0 = torch.from_numpy(prog0).to(dev)
        self.prog = self.prog0.clone()
        self.stat = torch.from_numpy(synth.to_planes("STAT", spec.stat, self.ld_site)).to(dev)
        self.daily = spec.daily is not None
        if self.daily:
            self.forc = None
            self.day_records = torch.from_numpy(np.ascontiguousarray(spec.daily, dtype=np.float32)).to(dev)
            self.site_lat = torch.from_numpy(np.asarray(spec.latitude, dtype=np.float32)).to(dev)
            self._dc = IbisEnsembleDailyC(records=self.day_records.data_ptr(), site_lat=self.site_lat.data_ptr(),
                                          len=int(self.day_records.shape[0]), seed=int(spec.weather_seed) & 0xFFFFFFFF,
                                          flags=1)
        else:
            self.forc = torch.from_numpy(np.ascontiguousarray(spec.forc, dtype=np.float32)).to(dev)
        self.run_params = torch.from_numpy(rp).to(dev)
        self.run_site = torch.from_numpy(site_of_run.astype(np.int32)).to(dev)
        self.run_forc = torch.from_numpy(spec.site_first[site_of_run].astype(np.int64)).to(dev)
        self.run_nstep = torch.from_numpy(nstep).to(dev)
        # queue order: longest records first, site-major within a length
        order = np.argsort(-nstep.astype(np.int64), kind="stable").astype(np.int32)
        self.order = torch.from_numpy(order).to(dev)
        self.acc = torch.zeros((2 * L.N_ACC, self.ld_run), dtype=f32, device=dev) if acc else None
        self.yearly = (torch.zeros((max(self.nyear, 1), L.N_YEARLY, self.ld_run), dtype=f32, device=dev)
                       if acc else None)
        self.queue = torch.zeros(1, dtype=torch.int32, device=dev)
        self.hour = torch.zeros(1, dtype=torch.int32, device=dev)
        self.status = torch.tensor([0, 2 ** 31 - 1], dtype=torch.int32, device=dev)
        self.params = spec.params.copy()
        if not acc:
            self.params.flags = self.params.flags & ~(FLAG_ACC | FLAG_CH4)
        self._pc = self.params.to_c()
        self._c = self._describe()
        self._graph = None

    def _describe(self) -> IbisEnsembleC:
        p = lambda t: ctypes.c_void_p(t.data_ptr()) if t is not None else None
        return IbisEnsembleC(prog=p(self.prog), acc=p(self.acc), stat=p(self.stat), forc=p(self.forc),
                             run_params=p(self.run_params), run_site=p(self.run_site), run_forc=p(self.run_forc),
                             run_nstep=p(self.run_nstep), run_pos=None, order=p(self.order),
                             yearly=p(self.yearly), forc_len=0 if self.forc is None else int(self.forc.shape[0]),
                             nrun=self.nrun,
                             ld_run=self.ld_run, nsite=self.nsite, ld_site=self.ld_site, nyear=self.nyear,
                             year_steps=self.year_steps, norder=self.nrun, queue=p(self.queue), status=p(self.status))

    # ------------------------------------------------------------------ runs
    def reset(self):
        """Back to the initial state (accumulators, yearly totals, status cleared)."""
        self.prog.copy_(self.prog0)
        if self.acc is not None:
            self.acc.zero_()
            self.yearly.zero_()
        self.status.copy_(torch.tensor([0, 2 ** 31 - 1], dtype=torch.int32))
        self.hour.zero_()

    def _stream(self, stream):
        return (stream or torch.cuda.current_stream(self.device)).cuda_stream

    def run(self, block: int = 0, stream=None):
        """Every run, whole record, in one persistent launch (``block`` 0 = automatic)."""
        if self.daily:
            _lib.check(self.lib.ibis_ensemble_daily_f32(ctypes.byref(self._c), ctypes.byref(self._dc),
                                                        ctypes.byref(self._pc), int(block),
                                                        ctypes.c_void_p(self._stream(stream))),
                       "ibis_ensemble_daily_f32")
            return
        _lib.check(self.lib.ibis_ensemble_f32(ctypes.byref(self._c), ctypes.byref(self._pc), int(block),
                                              ctypes.c_void_p(self._stream(stream))), "ibis_ensemble_f32")

    def run_hours(self, nhour: int, stream=None):
        """``nhour`` one-hour launches from the device hour counter (which they advance)."""
        if self.daily:
            raise ValueError("the one-launch-per-hour form reads hourly records; this ensemble has day records")
        _lib.check(self.lib.ibis_ensemble_hours_f32(ctypes.byref(self._c), ctypes.byref(self._pc),
                                                    ctypes.c_void_p(self.hour.data_ptr()), int(nhour),
                                                    ctypes.c_void_p(self._stream(stream))),
                   "ibis_ensemble_hours_f32")

    def run_hourly(self, chunk: int = 24, graph: bool = True):
        """Every run to the end of its record with one launch per hour: the first
        ``chunk`` hours eagerly, the rest by replaying a CUDA graph of ``chunk``
        launches (or eagerly, ``graph=False``)."""
        total = int(self.run_nstep_host.max(initial=0))
        nchunk = -(-total // chunk)
        if nchunk == 0:
            return
        self.run_hours(chunk)
        if nchunk == 1:
            return
        if not graph:
            for _ in range(nchunk - 1):
                self.run_hours(chunk)
            return
        if self._graph is None or self._graph[0] != chunk:
            g = torch.cuda.CUDAGraph()
            s = torch.cuda.Stream(self.device)
            s.wait_stream(torch.cuda.current_stream(self.device))
            with torch.cuda.stream(s):
                with torch.cuda.graph(g, stream=s, capture_error_mode="relaxed"):
                    self.run_hours(chunk, stream=s)
            torch.cuda.current_stream(self.device).wait_stream(s)
            self._graph = (chunk, g)
        g = self._graph[1]
        for _ in range(nchunk - 1):
            g.replay()

    def occupancy(self, block: int) -> int:
        return int(self.lib.ibis_ensemble_occupancy(ctypes.byref(self._pc), int(block)))

    def tune(self, blocks=None, reps: int = 1) -> dict:
        """Time the persistent launch at each block size (multiples of 32 up to 256);
        returns ``{"best": block, "ms": {block: ms}}``.  Restores the initial state."""
        blocks = list(range(32, 257, 32)) if blocks is None else list(blocks)
        ms = {}
        st = torch.cuda.current_stream(self.device)
        for b in blocks:
            if self.occupancy(b) <= 0:
                continue
            t = []
            for _ in range(reps):
                self.reset()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(st)
                self.run(block=b)
                e1.record(st)
                e1.synchronize()
                t.append(e0.elapsed_time(e1))
            ms[b] = min(t)
        self.reset()
        return {"best": min(ms, key=ms.get), "ms": ms}

    # --------------------------------------------------------------- results
    def cell_steps(self) -> int:
        return int(self.run_nstep_host.astype(np.int64).sum())

    def nonfinite(self):
        s = self.status.cpu().numpy()
        return bool(s[0] & 1), bool(s[0] & 2), int(s[1])

    def prog_host(self) -> dict:
        return synth.from_planes("PROG", self.prog.cpu().numpy(), self.nrun)

    def acc_host(self, compensated: bool = True) -> dict:
        a = self.acc.cpu().numpy().astype(np.float64)
        v = a[:L.N_ACC] - (a[L.N_ACC:] if compensated else 0.0)
        return synth.from_planes("ACC", v, self.nrun)

    def yearly_sums(self) -> np.ndarray:
        """(nrun, nyear, N_YEARLY) per-year sums (NaN past the end of a run's record)."""
        y = self.yearly.cpu().numpy().astype(np.float64)[:, :, :self.nrun]      # (nyear, K, nrun)
        tot = np.transpose(y, (2, 0, 1))
        out = np.diff(np.concatenate([np.zeros_like(tot[:, :1]), tot], axis=1), axis=1)
        years = self.run_nstep_host // self.year_steps
        mask = np.arange(self.nyear)[None, :] >= years[:, None]
        out[mask] = np.nan
        return out
