"""Autotuner for the launch configuration of the FP32 hourly-step kernels.

A launch configuration fixes the form (one fused kernel per launch, the same
with each hour's forcing tile staged into shared memory by bulk copies, or a
surface kernel and a ground kernel per hour), the block size and the register
budget (minimum resident blocks per SM).  Which is fastest depends on the batch:
the number of columns sets how many waves of blocks fill the 148 SMs, and the
hours per launch set how much the fused form's register-resident state saves.
:func:`tune` times every configuration on the caller's own columns and forcing
(restoring the state after each trial) and records the winner per
(cells, hours, flags) key for the process.
"""
from __future__ import annotations

import torch

from . import lib as _lib

_CACHE: dict = {}


def _key(cols, nstep, params):
    return (cols.ncell, int(nstep), int(params.flags), str(cols.device))


def tune(cols, forc: torch.Tensor, params, nstep: int | None = None, reps: int = 3, configs=None,
         apply: bool = True) -> dict:
    """Time each configuration for ``nstep`` hours of ``forc`` on ``cols``.

    Returns ``{"best": id, "ms": {id: median ms}, "configs": [...]}`` and, with
    ``apply``, switches ``cols`` to the fastest configuration.  The columns'
    prognostic state, accumulators and status word are restored after every
    trial, so tuning leaves the run where it was.
    """
    if cols.dtype != torch.float32:
        return {"best": 0, "ms": {}, "configs": []}
    nstep = forc.shape[0] if nstep is None else int(nstep)
    key = _key(cols, nstep, params)
    if key in _CACHE and configs is None:
        res = _CACHE[key]
        if apply:
            cols.set_mode(res["best"])
        return res
    all_cfgs = _lib.configs()
    ids = [c["id"] for c in all_cfgs] if configs is None else list(configs)
    prog0 = cols.prog.clone()
    acc0 = cols.acc.clone() if cols.acc is not None else None
    status0 = cols.status.clone()
    mode0 = cols.config
    stream = torch.cuda.current_stream(cols.device)
    ms = {}
    for cid in ids:
        cols.set_mode(cid)
        times = []
        for r in range(reps + 1):
            cols.prog.copy_(prog0)
            if acc0 is not None:
                cols.acc.copy_(acc0)
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            cols.run(forc, params, nstep=nstep, stream=stream)
            b.record(stream)
            b.synchronize()
            if r > 0:
                times.append(a.elapsed_time(b))
        times.sort()
        ms[cid] = times[len(times) // 2]
    cols.prog.copy_(prog0)
    if acc0 is not None:
        cols.acc.copy_(acc0)
    cols.status.copy_(status0)
    best = min(ms, key=ms.get)
    res = {"best": best, "ms": ms, "configs": [c for c in all_cfgs if c["id"] in ids]}
    if configs is None:
        _CACHE[key] = res
    cols.set_mode(best if apply else ("fused" if mode0 is None else mode0))
    return res
