"""Serving loop: evaluation requests batched continuously into one resident ensemble.

A request names tower sites from a resident :class:`SiteLibrary`, a number of
years and one 31-value calibration vector (``layout.RUN``); it is answered
with the per-year sums of the ``layout.YEARLY`` fluxes of every site.  The
reference has no serving layer: its calibration harness evaluates one
candidate at one site per host worker process
(verify/calibration/site_fit.py:375-436).

:class:`Server` keeps a fixed set of run *slots* on the GPU (prognostic state,
accumulators, parameter vector and yearly totals of one run each; the slot
count is what the memory budget allows) and advances every occupied slot in
*epochs* of ``epoch_hours`` hours, one persistent ensemble launch
(``ibis_ensemble_f32``) per epoch:

* before each epoch, requests that have arrived are admitted, first come first
  served, while their runs fit in free slots; their slots are initialised on
  the device and join the runs already in flight (continuous batching: new
  work shares the launch with old work instead of waiting for it);
* after the epoch in which a request's last run ends, its yearly totals are
  gathered into pinned host memory and its slots are freed at once (the copy is
  ordered before any re-use of the slots on the stream);
* the host prepares and enqueues up to ``lookahead`` epochs ahead of the GPU,
  each with its own descriptor arrays, so the GPU does not wait on it.

A run's result does not depend on what else is in flight: each slot's state
is advanced by the same step code, and splitting a record into epochs stores
and reloads the state exactly.  ``tests/test_serve.py`` checks that a request
answered alone and in a mix gives the same bits.
"""
from __future__ import annotations

import collections
import ctypes
import time
from dataclasses import dataclass

import numpy as np
import torch

from . import ensemble as E
from . import layout as L
from . import lib as _lib
from . import synth
from .lib import IbisEnsembleC, IbisEnsembleDailyC
from .params import StepParams

INT_MAX = 2 ** 31 - 1


@dataclass
class Request:
    rid: int
    sites: np.ndarray            # site ids in the library
    years: int
    vector: np.ndarray           # (N_RUN,) float32 calibration vector
    arrival: float = 0.0         # seconds after the start of the loop


@dataclass
class Result:
    rid: int
    yearly: np.ndarray           # (nsite, years, N_YEARLY) per-year sums
    nonfinite: bool
    arrival: float
    admitted: float
    done: float                  # GPU-clock seconds after the start of the loop

    @property
    def latency(self) -> float:
        return self.done - self.arrival


class SiteLibrary:
    """Static planes, initial state and forcing records of the sites requests may
    name, resident on the device (``years`` whole years of records per site).
    With ``daily`` the records are days of weather (48 bytes per site-day
    instead of 48 per site-hour) and the runs generate their hours in the
    kernel (``ibis_ensemble_daily_f32``); epochs are then whole days."""

    def __init__(self, nsite: int, years: int, seed: int = 0, year_hours: int = E.YEAR_HOURS, device="cuda",
                 lat_range=(-40.0, 70.0), params: StepParams | None = None, daily: bool = False):
        spec = E.make_ensemble(nsite, 1, site_hours=np.full(nsite, years * year_hours), seed=seed,
                               lat_range=lat_range, year_hours=year_hours, params=params, daily=daily)
        self.daily = bool(daily)
        self.spec = spec
        self.nsite, self.years, self.year_hours = nsite, years, year_hours
        self.device = torch.device(device)
        if self.device.index is None:
            self.device = torch.device("cuda", torch.cuda.current_device())
        self.ld_site = L.leading_dim(nsite)
        self.stat = torch.from_numpy(synth.to_planes("STAT", spec.stat, self.ld_site)).to(self.device)
        self.prog = torch.from_numpy(synth.to_planes("PROG", spec.prog, self.ld_site)).to(self.device)
        self.forc = torch.from_numpy(spec.daily if daily else spec.forc).to(self.device)
        self.first = spec.site_first.astype(np.int64)       # first record: an hour, or with ``daily`` a day
        self.params = spec.params
        if daily:
            self.lat = torch.from_numpy(np.asarray(spec.latitude, dtype=np.float32)).to(self.device)
            self.daily_desc = IbisEnsembleDailyC(records=self.forc.data_ptr(), site_lat=self.lat.data_ptr(),
                                                 len=int(self.forc.shape[0]),
                                                 seed=int(spec.weather_seed) & 0xFFFFFFFF, flags=1)

    @property
    def nbytes(self) -> int:
        return sum(t.numel() * t.element_size() for t in (self.stat, self.prog, self.forc))


# device bytes one slot holds: state, accumulators + compensation, parameter
# vector, yearly totals, descriptors
def slot_bytes(max_years: int) -> int:
    return 4 * (L.N_PROG + 2 * L.N_ACC + L.N_RUN + max_years * L.N_YEARLY) + 8 + 4 * 5


class Server:
    """Continuous-batching request loop over one :class:`SiteLibrary`."""

    def __init__(self, library: SiteLibrary, budget_bytes: float = 150e9, max_slots: int = 1 << 16,
                 epoch_hours: int = 168, lookahead: int = 2, block: int = 0):
        self.lib = library
        self.dev = library.device
        self.max_years = library.years
        self.epoch_hours = int(epoch_hours)
        self.lookahead = max(1, int(lookahead))
        if library.daily and self.epoch_hours % 24:
            raise ValueError("a library of day records needs epochs of whole days")
        self.block = int(block)
        free_bytes = budget_bytes - library.nbytes
        if free_bytes <= 0:
            raise ValueError("the memory budget does not hold the site library")
        self.nslot = int(min(max_slots, free_bytes // slot_bytes(self.max_years)))
        if self.nslot < 32:
            raise ValueError("the memory budget holds fewer than 32 run slots")
        self.nslot -= self.nslot % 32
        C, dev = self.nslot, self.dev
        self.ld = C
        f32 = dict(dtype=torch.float32, device=dev)
        self.prog = torch.zeros((L.N_PROG, C), **f32)
        self.acc = torch.zeros((2 * L.N_ACC, C), **f32)
        self.run_params = torch.zeros((L.N_RUN, C), **f32)
        self.yearly = torch.zeros((self.max_years, L.N_YEARLY, C), **f32)
        self.run_site = torch.zeros(C, dtype=torch.int32, device=dev)
        self.queue = torch.zeros(1, dtype=torch.int32, device=dev)
        self.status = torch.tensor([0, INT_MAX], dtype=torch.int32, device=dev)
        # per-epoch descriptors, one set per epoch that may be in flight: device
        # arrays and the pinned host arrays they are copied from
        self._desc = []
        for _ in range(self.lookahead):
            d = dict(forc=torch.zeros(C, dtype=torch.int64, device=dev),
                     nstep=torch.zeros(C, dtype=torch.int32, device=dev),
                     pos=torch.zeros(C, dtype=torch.int32, device=dev),
                     order=torch.zeros(C, dtype=torch.int32, device=dev))
            h = {k: torch.zeros(v.shape, dtype=v.dtype).pin_memory() for k, v in d.items()}
            self._desc.append((d, h))
        self._pc = library.params.to_c()
        self._so = _lib.load()
        self.stream = torch.cuda.Stream(dev)
        # host view of the slots
        self.slot_site = np.zeros(C, dtype=np.int64)
        self.slot_len = np.zeros(C, dtype=np.int64)
        self.slot_pos = np.zeros(C, dtype=np.int64)
        self.slot_req = np.full(C, -1, dtype=np.int64)
        self.free = collections.deque(range(C))

    # ----------------------------------------------------------- descriptors
    def _launch(self, buf: int, active: np.ndarray, n: np.ndarray):
        """Enqueue one epoch: the runs in slots ``active`` advance ``n`` hours each."""
        d, h = self._desc[buf]
        k = active.size
        hf, hn, hp, ho = (h[x].numpy() for x in ("forc", "nstep", "pos", "order"))
        pos = self.slot_pos[active] // 24 if self.lib.daily else self.slot_pos[active]
        hf[active] = self.lib.first[self.slot_site[active]] + pos
        hn[active] = n
        hp[active] = self.slot_pos[active]
        ho[:k] = active[np.argsort(-n, kind="stable")]          # longest first
        with torch.cuda.stream(self.stream):
            for x in ("forc", "nstep", "pos", "order"):
                d[x].copy_(h[x], non_blocking=True)
        e = IbisEnsembleC(prog=self.prog.data_ptr(), acc=self.acc.data_ptr(), stat=self.lib.stat.data_ptr(),
                          forc=self.lib.forc.data_ptr(), run_params=self.run_params.data_ptr(),
                          run_site=self.run_site.data_ptr(), run_forc=d["forc"].data_ptr(),
                          run_nstep=d["nstep"].data_ptr(), run_pos=d["pos"].data_ptr(), order=d["order"].data_ptr(),
                          yearly=self.yearly.data_ptr(), forc_len=0 if self.lib.daily else int(self.lib.forc.shape[0]),
                          nrun=self.nslot,
                          ld_run=self.ld, nsite=self.lib.nsite, ld_site=self.lib.ld_site, nyear=self.max_years,
                          year_steps=self.lib.year_hours, norder=k, queue=self.queue.data_ptr(),
                          status=self.status.data_ptr())
        if self.lib.daily:
            _lib.check(self._so.ibis_ensemble_daily_f32(ctypes.byref(e), ctypes.byref(self.lib.daily_desc),
                                                        ctypes.byref(self._pc), self.block,
                                                        ctypes.c_void_p(self.stream.cuda_stream)),
                       "ibis_ensemble_daily_f32")
            return
        _lib.check(self._so.ibis_ensemble_f32(ctypes.byref(e), ctypes.byref(self._pc), self.block,
                                              ctypes.c_void_p(self.stream.cuda_stream)), "ibis_ensemble_f32")

    def _admit(self, req: Request, now: float):
        """Place ``req``'s runs in free slots and initialise them on the device."""
        nrun = len(req.sites)
        slots = np.array([self.free.popleft() for _ in range(nrun)], dtype=np.int64)
        sites = np.asarray(req.sites, dtype=np.int64)
        self.slot_site[slots] = sites
        self.slot_len[slots] = req.years * self.lib.year_hours
        self.slot_pos[slots] = 0
        self.slot_req[slots] = req.rid
        with torch.cuda.stream(self.stream):
            si = torch.from_numpy(slots).to(self.dev, non_blocking=True)
            ti = torch.from_numpy(sites).to(self.dev, non_blocking=True)
            self.prog[:, si] = self.lib.prog[:, ti]
            self.acc[:, si] = 0.0
            self.yearly[:, :, si] = 0.0
            v = torch.from_numpy(np.asarray(req.vector, dtype=np.float32)).to(self.dev, non_blocking=True)
            self.run_params[:, si] = v[:, None].expand(L.N_RUN, nrun)
            self.run_site[si] = ti.to(torch.int32)
        self._active[req.rid] = dict(req=req, slots=slots, admitted=now)

    def _retire(self, rid: int):
        """Gather a finished request's yearly totals (asynchronously) and free its slots."""
        info = self._active.pop(rid)
        req, slots = info["req"], info["slots"]
        with torch.cuda.stream(self.stream):
            si = torch.from_numpy(slots).to(self.dev, non_blocking=True)
            y = self.yearly[:req.years, :, si]                       # (years, K, nrun)
            p = self.prog[:, si]
            host_y = torch.empty(y.shape, dtype=y.dtype).pin_memory()
            host_p = torch.empty(p.shape, dtype=p.dtype).pin_memory()
            host_y.copy_(y, non_blocking=True)
            host_p.copy_(p, non_blocking=True)
            ev = torch.cuda.Event(enable_timing=True)
            ev.record(self.stream)
        self.slot_req[slots] = -1
        self.free.extend(slots.tolist())
        self._gathering.append(dict(info, host_y=host_y, host_p=host_p, event=ev))

    def _collect(self, block: bool = False):
        keep = []
        for g in self._gathering:
            if block:
                g["event"].synchronize()
            if not g["event"].query():
                keep.append(g)
                continue
            tot = g["host_y"].numpy().astype(np.float64)                 # running totals at year ends
            tot = np.transpose(tot, (2, 0, 1))                            # (nrun, years, K)
            yearly = np.diff(np.concatenate([np.zeros_like(tot[:, :1]), tot], axis=1), axis=1)
            nonfinite = not np.isfinite(g["host_p"].numpy()).all()
            done = self._t0_event.elapsed_time(g["event"]) / 1e3
            r = g["req"]
            self.results[r.rid] = Result(rid=r.rid, yearly=yearly, nonfinite=nonfinite, arrival=r.arrival,
                                         admitted=g["admitted"], done=done)
        self._gathering = keep

    # ------------------------------------------------------------------ loop
    def serve(self, requests, realtime: bool = True, epoch_seconds: float | None = None) -> dict:
        """Answer ``requests`` (sorted by arrival).  With ``realtime`` a request is
        admitted once the wall clock passes its arrival; otherwise the clock
        advances ``epoch_seconds`` per epoch (arrival order and epoch boundaries
        only change when a run starts, never its result)."""
        requests = sorted(requests, key=lambda r: r.arrival)
        for r in requests:
            if r.years < 1 or r.years > self.max_years:
                raise ValueError(f"request {r.rid}: years must be in 1..{self.max_years}")
            if len(r.sites) == 0 or len(r.sites) > self.nslot:
                raise ValueError(f"request {r.rid}: 1..{self.nslot} sites")
            if np.any(np.asarray(r.sites) < 0) or np.any(np.asarray(r.sites) >= self.lib.nsite):
                raise ValueError(f"request {r.rid}: site id outside the library")
        self.results = {}
        self._active = {}
        self._gathering = []
        pending = collections.deque()
        inflight = collections.deque()
        self.status.copy_(torch.tensor([0, INT_MAX], dtype=torch.int32))
        torch.cuda.synchronize(self.dev)
        self._t0_event = torch.cuda.Event(enable_timing=True)
        self._t0_event.record(self.stream)
        t0 = time.perf_counter()
        vclock = 0.0
        clock = (lambda: time.perf_counter() - t0) if realtime else (lambda: vclock)
        i, epochs, cell_steps, buf = 0, 0, 0, 0
        busy = 0.0
        depths = []
        while i < len(requests) or pending or self._active or self._gathering:
            now = clock()
            while i < len(requests) and requests[i].arrival <= now:
                pending.append(requests[i])
                i += 1
            while pending and len(pending[0].sites) <= len(self.free):
                self._admit(pending.popleft(), now)
            occ = np.flatnonzero(self.slot_req >= 0)
            if occ.size == 0:
                self._collect(block=not pending and i >= len(requests))
                if i < len(requests) and not pending:
                    if realtime:
                        time.sleep(max(0.0, min(requests[i].arrival - clock(), 0.01)))
                    else:
                        vclock = max(vclock, requests[i].arrival)
                continue
            # keep at most `lookahead` epochs in flight (and the descriptor buffer free)
            while len(inflight) >= self.lookahead:
                inflight.popleft().synchronize()
            n = np.minimum(self.epoch_hours, self.slot_len[occ] - self.slot_pos[occ])
            depths.append(len(pending))
            self._launch(buf, occ, n)
            ev = torch.cuda.Event()
            ev.record(self.stream)
            inflight.append(ev)
            buf = (buf + 1) % self.lookahead
            epochs += 1
            cell_steps += int(n.sum())
            self.slot_pos[occ] += n
            finished = set(self.slot_req[occ[self.slot_pos[occ] >= self.slot_len[occ]]].tolist())
            for rid in finished:
                info = self._active[rid]
                if np.all(self.slot_pos[info["slots"]] >= self.slot_len[info["slots"]]):
                    self._retire(rid)
            self._collect()
            if not realtime:
                vclock += epoch_seconds if epoch_seconds is not None else 0.0
        torch.cuda.synchronize(self.dev)
        t_end = time.perf_counter() - t0
        self._collect(block=True)
        lat = np.array([r.latency for r in self.results.values()])
        span = max((r.done for r in self.results.values()), default=0.0)
        return {"requests": len(self.results), "epochs": epochs, "cell_steps": cell_steps,
                "wall_s": t_end, "gpu_span_s": span,
                "cell_steps_per_s": cell_steps / span if span > 0 else 0.0,
                "p50_s": float(np.percentile(lat, 50)) if lat.size else None,
                "p99_s": float(np.percentile(lat, 99)) if lat.size else None,
                "mean_s": float(lat.mean()) if lat.size else None,
                "slots": self.nslot, "epoch_hours": self.epoch_hours,
                "queue_depth_max": int(max(depths, default=0)),
                "queue_depth_mean": float(np.mean(depths)) if depths else 0.0,
                "hbm_gb": self.nbytes / 1e9,
                "status": self.status.cpu().numpy().tolist()}

    @property
    def nbytes(self) -> int:
        """Device bytes of the site library and the run slots."""
        ts = [self.prog, self.acc, self.run_params, self.yearly, self.run_site]
        ts += [t for d, _ in self._desc for t in d.values()]
        return self.lib.nbytes + sum(t.numel() * t.element_size() for t in ts)


def poisson_requests(rng, rate: float, duration: float, nsite_lib: int, max_sites: int = 64, max_years: int = 10,
                     params: StepParams | None = None, start_id: int = 0):
    """Requests arriving as a Poisson process of ``rate`` per second for ``duration``
    seconds: U{1..max_sites} distinct library sites, U{1..max_years} years, and a
    calibration vector drawn log-uniform within +-50% of the defaults."""
    out, t, rid = [], 0.0, start_id
    while True:
        t += rng.exponential(1.0 / rate)
        if t > duration:
            break
        ns = int(rng.integers(1, max_sites + 1))
        sites = rng.choice(nsite_lib, size=min(ns, nsite_lib), replace=False)
        years = int(rng.integers(1, max_years + 1))
        vec = E.draw_vectors(rng, 1, params)[0]
        out.append(Request(rid=rid, sites=np.sort(sites), years=years, vector=vec, arrival=t))
        rid += 1
    return out


def serve_plain(library: SiteLibrary, requests, block: int = 0) -> dict:
    """The plain form of the request loop, for comparison: requests answered one
    at a time in arrival order, each as its own persistent ensemble launch over
    its runs' whole records (buffers allocated per request, no batching with
    other requests).  Latency from arrival to the GPU-clock end of its launch."""
    if library.daily:
        raise ValueError("the plain form reads hourly records")
    dev = library.device
    so = _lib.load()
    pc = library.params.to_c()
    requests = sorted(requests, key=lambda r: r.arrival)
    stream = torch.cuda.Stream(dev)
    t0_ev = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize(dev)
    t0_ev.record(stream)
    t0 = time.perf_counter()
    lat = []
    cell_steps = 0
    for r in requests:
        wait = r.arrival - (time.perf_counter() - t0)
        if wait > 0:
            time.sleep(wait)
        nrun, ld = len(r.sites), L.leading_dim(len(r.sites))
        sites = torch.from_numpy(np.asarray(r.sites, dtype=np.int64)).to(dev)
        f32 = dict(dtype=torch.float32, device=dev)
        with torch.cuda.stream(stream):
            prog = torch.zeros((L.N_PROG, ld), **f32)
            prog[:, :nrun] = library.prog[:, sites]
            acc = torch.zeros((2 * L.N_ACC, ld), **f32)
            rp = torch.zeros((L.N_RUN, ld), **f32)
            rp[:, :nrun] = torch.from_numpy(np.asarray(r.vector, dtype=np.float32)).to(dev)[:, None]
            yearly = torch.zeros((r.years, L.N_YEARLY, ld), **f32)
            run_site = sites.to(torch.int32)
            run_forc = torch.from_numpy(library.first[np.asarray(r.sites)]).to(dev)
            run_nstep = torch.full((nrun,), r.years * library.year_hours, dtype=torch.int32, device=dev)
            queue = torch.zeros(1, dtype=torch.int32, device=dev)
            status = torch.tensor([0, INT_MAX], dtype=torch.int32, device=dev)
        e = IbisEnsembleC(prog=prog.data_ptr(), acc=acc.data_ptr(), stat=library.stat.data_ptr(),
                          forc=library.forc.data_ptr(), run_params=rp.data_ptr(), run_site=run_site.data_ptr(),
                          run_forc=run_forc.data_ptr(), run_nstep=run_nstep.data_ptr(), run_pos=None, order=None,
                          yearly=yearly.data_ptr(), forc_len=int(library.forc.shape[0]), nrun=nrun, ld_run=ld,
                          nsite=library.nsite, ld_site=library.ld_site, nyear=r.years,
                          year_steps=library.year_hours, norder=nrun, queue=queue.data_ptr(),
                          status=status.data_ptr())
        _lib.check(so.ibis_ensemble_f32(ctypes.byref(e), ctypes.byref(pc), int(block),
                                        ctypes.c_void_p(stream.cuda_stream)), "ibis_ensemble_f32")
        done = torch.cuda.Event(enable_timing=True)
        done.record(stream)
        done.synchronize()
        lat.append(t0_ev.elapsed_time(done) / 1e3 - r.arrival)
        cell_steps += nrun * r.years * library.year_hours
    lat = np.asarray(lat)
    return {"requests": len(lat), "p50_s": float(np.percentile(lat, 50)) if lat.size else None,
            "p99_s": float(np.percentile(lat, 99)) if lat.size else None, "cell_steps": cell_steps}
