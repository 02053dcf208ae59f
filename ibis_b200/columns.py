"""Device-resident column state and the launch of the hourly-step kernels.

A :class:`Columns` owns the structure-of-arrays buffers of ``ncell`` columns on
one GPU (torch tensors are used only as device allocations) and advances them
through the C ABI of ``include/ibis_b200.h``.  Forcing for ``nstep`` hours is a
``(nstep, IBIS_FORC_COUNT, ld)`` device tensor; the whole run executes in one
launch, so prognostic state and accumulators stay on chip across the hours.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import layout as L
from . import lib as _lib
from . import synth
from .params import StepParams, FLAG_DIAG, FLAG_ACC, FLAG_CH4, FLAG_SOIL_MEANS

INT_MAX = 2 ** 31 - 1
AUTO_FUSED = 6          # fused, block 224, accumulators on chip
AUTO_MIN_HOURS = 4      # shorter launches keep the accumulators in global memory (configuration 0)
_ACC_FLAGS = FLAG_ACC | FLAG_CH4 | FLAG_SOIL_MEANS


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else ctypes.c_void_p(0)


class Columns:
    """``ncell`` IBIS columns resident on ``device`` in FP32 (default) or FP64."""

    def __init__(self, ncell: int, dtype=torch.float32, device="cuda", diag: bool = False, acc: bool = True,
                 mode: str = "fused"):
        if dtype not in (torch.float32, torch.float64):
            raise ValueError("dtype must be torch.float32 or torch.float64")
        self.ncell = int(ncell)
        self.ld = L.leading_dim(self.ncell)
        self.dtype = dtype
        dev = torch.device(device)
        if dev.type != "cuda":
            raise ValueError("Columns live on a CUDA device; there is no host implementation")
        if dev.index is None:
            dev = torch.device("cuda", torch.cuda.current_device())
        self.device = dev
        kw = dict(dtype=dtype, device=self.device)
        self.prog = torch.zeros((L.N_PROG, self.ld), **kw)
        self.stat = torch.zeros((L.N_STAT, self.ld), **kw)
        self.diag = torch.zeros((L.N_DIAG, self.ld), **kw) if diag else None
        self.acc = torch.zeros((2 * L.N_ACC, self.ld), **kw) if acc else None
        self.status = torch.tensor([0, INT_MAX], dtype=torch.int32, device=self.device)
        self._np_dtype = np.float32 if dtype == torch.float32 else np.float64
        lib = _lib.load()
        self._fn = lib.ibis_step_f32 if dtype == torch.float32 else lib.ibis_step_f64
        self._cfg_fn = lib.ibis_step_config_f32
        self.scratch = None
        self.config = None
        self.set_mode(mode)

    def set_mode(self, mode: str):
        """``fused`` (one kernel per launch), ``split`` (surface + ground kernels per hour),
        or an integer launch configuration (see ``lib.configs()``).

        ``fused`` picks the configuration per call in FP32: block 224 with the
        accumulators on chip (configuration 6, the fastest at 95,333 cells)
        for launches of ``AUTO_MIN_HOURS`` hours or more, the default
        configuration 0 (global accumulators) for shorter ones; ``tune.tune``
        times every configuration on the caller's own batch instead."""
        if mode is None:
            mode = "fused"
        if isinstance(mode, (int, np.integer)) and not isinstance(mode, bool):
            cfgs = _lib.configs()
            if not 0 <= int(mode) < len(cfgs):
                raise ValueError(f"launch configuration {mode} out of range")
            cfg = int(mode)
            form = cfgs[cfg]["form"]
        elif mode in ("fused", "split"):
            form = mode
            cfg = (None if self.dtype == torch.float32 else 0) if mode == "fused" else 8
        else:
            raise ValueError("mode must be 'fused', 'split' or a configuration index")
        if self.dtype != torch.float32 and (form == "split" or cfg not in (0, None)):
            raise ValueError("only the default fused form exists in float64")
        if form == "split" and self.scratch is None:
            self.scratch = torch.zeros((_lib.load().ibis_mid_planes(), self.ld), dtype=self.dtype,
                                       device=self.device)
        self.mode = form
        self.config = cfg

    # -------------------------------------------------------------- transfer
    @classmethod
    def from_host(cls, prog: dict, stat: dict, dtype=torch.float32, device="cuda", diag=False, acc=True,
                  mode="fused"):
        n = prog["tg"].shape[0]
        c = cls(n, dtype=dtype, device=device, diag=diag, acc=acc, mode=mode)
        c.set_prog(prog)
        c.set_stat(stat)
        return c

    def set_prog(self, prog: dict):
        a = synth.to_planes("PROG", prog, self.ld, self._np_dtype)
        self.prog.copy_(torch.from_numpy(a))

    def set_stat(self, stat: dict):
        a = synth.to_planes("STAT", stat, self.ld, self._np_dtype)
        self.stat.copy_(torch.from_numpy(a))

    def forcing(self, forc: dict, h0: int = 0, h1: int | None = None) -> torch.Tensor:
        """Device forcing tensor (nstep, IBIS_FORC_COUNT, ld) for hours [h0, h1)."""
        a = synth.forcing_planes(forc, self.ld, h0, h1, self._np_dtype)
        return torch.from_numpy(a).to(self.device)

    def prog_host(self) -> dict:
        return synth.from_planes("PROG", self.prog.cpu().numpy(), self.ncell)

    def diag_host(self) -> dict:
        if self.diag is None:
            raise ValueError("diagnostics were not allocated")
        return synth.from_planes("DIAG", self.diag.cpu().numpy(), self.ncell)

    def acc_host(self, compensated: bool = True) -> dict:
        """Accumulators; with ``compensated`` the Kahan terms are folded in."""
        if self.acc is None:
            raise ValueError("accumulators were not allocated")
        a = self.acc.cpu().numpy().astype(np.float64)
        v = a[:L.N_ACC]
        if compensated:
            v = v - a[L.N_ACC:]
        return synth.from_planes("ACC", v, self.ncell)

    def set_acc(self, values: dict):
        """Set accumulator planes (per-cell arrays named as ``layout.ACC``);
        their compensation planes are zeroed, the other planes kept."""
        if self.acc is None:
            raise ValueError("accumulators were not allocated")
        for name, v in values.items():
            p0, k = L.OFF["ACC"][name]
            a = np.asarray(v, dtype=np.float64).reshape(self.ncell, -1) if k > 1 else \
                np.asarray(v, dtype=np.float64).reshape(1, self.ncell)
            t = torch.from_numpy(np.ascontiguousarray(a.T if k > 1 else a)).to(self.acc)
            self.acc[p0:p0 + k, :self.ncell] = t
            self.acc[L.N_ACC + p0:L.N_ACC + p0 + k].zero_()

    def reset_acc(self):
        if self.acc is not None:
            self.acc.zero_()

    def reset_status(self):
        self.status.copy_(torch.tensor([0, INT_MAX], dtype=torch.int32))

    def nonfinite(self):
        """(flag, first cell) of the non-finite detector."""
        s = self.status.cpu().numpy()
        return bool(s[0] & 1), int(s[1])

    # -------------------------------------------------------------- compute
    def launch_config(self, nstep: int) -> int:
        """The launch configuration a call of ``nstep`` hours uses."""
        if self.config is not None:
            return self.config
        return AUTO_FUSED if nstep >= AUTO_MIN_HOURS else 0

    def run(self, forc: torch.Tensor, params: StepParams, nstep: int | None = None, stream=None):
        """Advance the columns ``nstep`` hours with forcing ``forc`` (asynchronous)."""
        if forc.dtype != self.dtype or forc.device != self.device:
            raise ValueError("forcing must have the Columns' dtype and device")
        if forc.dim() != 3 or forc.shape[1] != L.N_FORC or forc.shape[2] != self.ld:
            raise ValueError(f"forcing must be (nstep, {L.N_FORC}, {self.ld})")
        if not forc.is_contiguous():
            raise ValueError("forcing must be contiguous")
        nstep = forc.shape[0] if nstep is None else int(nstep)
        if nstep > forc.shape[0]:
            raise ValueError("nstep exceeds the forcing provided")
        flags = params.flags
        if self.diag is None:
            flags &= ~FLAG_DIAG
        else:
            flags |= FLAG_DIAG
        if self.acc is None:
            flags &= ~_ACC_FLAGS
        p = params.to_c()
        p.flags = flags
        if stream is None:
            stream = torch.cuda.current_stream(self.device)
        if self.dtype == torch.float32:
            rc = self._cfg_fn(_ptr(self.prog), _ptr(self.stat), _ptr(forc), _ptr(self.diag), _ptr(self.acc),
                              _ptr(self.scratch), self.ncell, self.ld, nstep, ctypes.byref(p), _ptr(self.status),
                              ctypes.c_void_p(stream.cuda_stream), self.launch_config(nstep))
        else:
            rc = self._fn(_ptr(self.prog), _ptr(self.stat), _ptr(forc), _ptr(self.diag), _ptr(self.acc), self.ncell,
                          self.ld, nstep, ctypes.byref(p), _ptr(self.status), ctypes.c_void_p(stream.cuda_stream))
        _lib.check(rc, "ibis_step")
        return self

    def run_host(self, host_forc: torch.Tensor, params: StepParams, host_prog: torch.Tensor | None = None,
                 group: int = 0, chunk: int = 0, stream=None):
        """Advance the columns through ``host_forc`` (a pinned host tensor
        ``(nstep, IBIS_FORC_COUNT, ld)``) and, with ``host_prog`` (a pinned host
        tensor shaped like ``prog``), copy the state after the last hour out:
        ``ibis_step_host_f32``, which overlaps the copies with the steps -- in
        groups of ``group`` columns for batches of several waves (0: sixteen
        groups), each group's hours in chunks (``chunk`` hours each, ``-c``:
        ``c`` hours then the rest; 0: a third of the hours then the rest, or for
        a batch of about one wave 4 hours growing by 1.75).  Asynchronous on
        ``stream``; read ``host_prog`` after synchronising it.  FP32 columns
        only; a two-kernel launch mode runs the library's fused choice."""
        if self.dtype != torch.float32:
            raise ValueError("run_host runs FP32 columns")
        if host_forc.device.type != "cpu" or host_forc.dtype != self.dtype or not host_forc.is_pinned():
            raise ValueError("host forcing must be a pinned CPU tensor of the Columns' dtype")
        if host_forc.dim() != 3 or host_forc.shape[1] != L.N_FORC or host_forc.shape[2] != self.ld:
            raise ValueError(f"host forcing must be (nstep, {L.N_FORC}, {self.ld})")
        if not host_forc.is_contiguous():
            raise ValueError("host forcing must be contiguous")
        if host_prog is not None and (host_prog.device.type != "cpu" or not host_prog.is_pinned()
                                      or host_prog.shape != self.prog.shape or host_prog.dtype != self.dtype
                                      or not host_prog.is_contiguous()):
            raise ValueError("host_prog must be a pinned contiguous CPU tensor shaped like prog")
        nstep = host_forc.shape[0]
        if getattr(self, "_host_forc", None) is None or self._host_forc.shape[0] < nstep:
            self._host_forc = torch.empty((nstep, L.N_FORC, self.ld), dtype=self.dtype, device=self.device)
        cfg = self.launch_config(nstep)
        if _lib.configs()[cfg]["form"] != "fused":
            cfg = -1                       # a two-kernel configuration needs scratch: the library's own choice
        flags = params.flags & ~FLAG_DIAG if self.diag is None else params.flags | FLAG_DIAG
        if self.acc is None:
            flags &= ~_ACC_FLAGS
        p = params.to_c()
        p.flags = flags
        if stream is None:
            stream = torch.cuda.current_stream(self.device)
        rc = _lib.load().ibis_step_host_f32(_ptr(self.prog), _ptr(self.stat), _ptr(host_forc),
                                            _ptr(self._host_forc), _ptr(self.diag), _ptr(self.acc), _ptr(host_prog),
                                            self.ncell, self.ld, nstep, ctypes.byref(p), _ptr(self.status),
                                            int(group), int(chunk), int(cfg),
                                            ctypes.c_void_p(stream.cuda_stream))
        _lib.check(rc, "ibis_step_host_f32")
        return self

    def run_host_daily(self, host_daily: torch.Tensor, lat: torch.Tensor, params: StepParams, jday0: int,
                       day0: int = 0, seed: int = 0, observed_fira: bool = False,
                       host_prog: torch.Tensor | None = None, group: int = 0, stream=None):
        """Advance the columns through the days of ``host_daily`` (a pinned host
        tensor ``(nday, IBIS_DAILY_COUNT, ld)`` of daily weather), the hourly
        forcing generated on the device as ``forcing.hourly_forcing`` generates
        it (``lat``: ``(ld,)`` float32 degrees on the device), and copy the state
        after the last hour to ``host_prog``: ``ibis_day_host_f32``, in groups of
        columns whose copies and generation overlap the other groups' hours.
        Asynchronous on ``stream``.  FP32 columns only."""
        if self.dtype != torch.float32:
            raise ValueError("run_host_daily runs FP32 columns")
        if (host_daily.device.type != "cpu" or host_daily.dtype != torch.float32 or not host_daily.is_pinned()
                or host_daily.dim() != 3 or host_daily.shape[1:] != (L.N_DAILY, self.ld)
                or not host_daily.is_contiguous()):
            raise ValueError(f"host daily weather must be a pinned contiguous (nday, {L.N_DAILY}, {self.ld}) float32 "
                             "CPU tensor")
        if lat.shape != (self.ld,) or lat.dtype != torch.float32 or lat.device != self.device:
            raise ValueError(f"lat must be a ({self.ld},) float32 tensor on the columns' device")
        if host_prog is not None and (host_prog.device.type != "cpu" or not host_prog.is_pinned()
                                      or host_prog.shape != self.prog.shape or host_prog.dtype != self.dtype
                                      or not host_prog.is_contiguous()):
            raise ValueError("host_prog must be a pinned contiguous CPU tensor shaped like prog")
        nday = host_daily.shape[0]
        nh = int(round(86400.0 / params.dtime))
        if getattr(self, "_host_daily", None) is None or self._host_daily.shape[0] < nday:
            self._host_daily = torch.empty((nday, L.N_DAILY, self.ld), dtype=torch.float32, device=self.device)
        if getattr(self, "_host_forc", None) is None or self._host_forc.shape[0] < nday * nh:
            self._host_forc = torch.empty((nday * nh, L.N_FORC, self.ld), dtype=self.dtype, device=self.device)
        cfg = self.launch_config(nday * nh)
        if _lib.configs()[cfg]["form"] != "fused":
            cfg = -1
        flags = params.flags & ~FLAG_DIAG if self.diag is None else params.flags | FLAG_DIAG
        if self.acc is None:
            flags &= ~_ACC_FLAGS
        p = params.to_c()
        p.flags = flags
        if stream is None:
            stream = torch.cuda.current_stream(self.device)
        rc = _lib.load().ibis_day_host_f32(_ptr(self.prog), _ptr(self.stat), _ptr(host_daily), _ptr(self._host_daily),
                                           _ptr(lat), _ptr(self._host_forc), _ptr(self.diag), _ptr(self.acc),
                                           _ptr(host_prog), self.ncell, self.ld, nday, int(jday0), int(day0),
                                           int(seed) & 0xFFFFFFFF, 1 if observed_fira else 0, ctypes.byref(p),
                                           _ptr(self.status), int(group), int(cfg), ctypes.c_void_p(stream.cuda_stream))
        _lib.check(rc, "ibis_day_host_f32")
        return self

    @staticmethod
    def chunk_schedule(nstep: int, chunk="auto"):
        """Hours per host-to-device chunk.  An integer gives equal chunks;
        ``"auto"`` starts with 4 hours and grows each chunk by 1.75, the last
        chunk taking a remainder under half its size.  At 95,333 cells a
        forcing hour copies in ~0.08 ms over PCIe and computes in ~0.13 ms, so
        each copy stays about within the computation of the chunk before it and
        only the first, small copy is exposed; each extra launch costs ~0.15 ms
        (measured), so few chunks ([4, 7, 13] for a day) beat many small ones
        ([2, 3, 4, 6, 9]: 0.3 ms slower)."""
        if chunk == "auto":
            out, c = [], 4.0
            while sum(out) < nstep:
                rem = nstep - sum(out)
                n = min(int(c), rem)
                if rem - n < n / 2:
                    n = rem
                out.append(n)
                c *= 1.75
            return out
        c = max(1, min(int(chunk), nstep))
        return [min(c, nstep - h0) for h0 in range(0, nstep, c)]

    def run_from_host(self, host_forc: torch.Tensor, params: StepParams, chunk="auto", stream=None):
        """Advance the columns through ``host_forc`` (a pinned host tensor
        ``(nstep, IBIS_FORC_COUNT, ld)``), copying the forcing in chunks
        (:meth:`chunk_schedule`) on a second stream so the copy of chunk k+1
        overlaps the computation of chunk k.  Asynchronous on ``stream``: work
        queued on it afterwards (a read-back of the state) runs after the last hour."""
        if host_forc.device.type != "cpu" or host_forc.dtype != self.dtype or not host_forc.is_pinned():
            raise ValueError("host forcing must be a pinned CPU tensor of the Columns' dtype")
        if host_forc.dim() != 3 or host_forc.shape[1] != L.N_FORC or host_forc.shape[2] != self.ld:
            raise ValueError(f"host forcing must be (nstep, {L.N_FORC}, {self.ld})")
        nstep = host_forc.shape[0]
        sched = self.chunk_schedule(nstep, chunk)
        chunk = max(sched)
        stream = stream or torch.cuda.current_stream(self.device)
        key = (chunk, host_forc.dtype)
        if getattr(self, "_staging", None) is None or self._staging[0] != key:
            bufs = [torch.empty((chunk, L.N_FORC, self.ld), dtype=self.dtype, device=self.device) for _ in range(2)]
            self._staging = (key, bufs, torch.cuda.Stream(self.device),
                             [torch.cuda.Event() for _ in range(2)], [torch.cuda.Event() for _ in range(2)])
        _, bufs, copy_stream, copied, used = self._staging
        start = torch.cuda.Event()
        start.record(stream)
        copy_stream.wait_event(start)
        h0 = 0
        for k, n in enumerate(sched):
            slot = k % 2
            with torch.cuda.stream(copy_stream):
                if k >= 2:
                    copy_stream.wait_event(used[slot])        # the computation of chunk k-2 has read this buffer
                bufs[slot][:n].copy_(host_forc[h0:h0 + n], non_blocking=True)
                copied[slot].record(copy_stream)
            stream.wait_event(copied[slot])
            self.run(bufs[slot][:n], params, stream=stream)
            used[slot].record(stream)
            h0 += n
        return self
