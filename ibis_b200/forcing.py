"""Hourly forcing generated on the GPU from daily weather.

The reference turns each day's weather (``DailyWeather``: max/min temperature,
cloud, precipitation, pressure, humidity, wind) into hourly forcing with
``compute_precip_timing`` and ``diurnal``
(python-port/ibis/physics/weather.py:395-601), one call per hour of the day
loop.  :func:`hourly_forcing` does it for every cell, day and hour in one
launch (``ibis_diurnal_f32``): a run can keep 32 bytes of daily weather per
cell-day on the device, or ship only those from the host, instead of 48 bytes
per cell-hour.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import layout as L
from . import lib as _lib

OBSERVED_FIRA = 1


def daily_planes(daily: dict, ld: int, dtype=np.float32):
    """(nday, N_DAILY, ld) array from a dict of (nday, ncell) arrays named as ``layout.DAILY``."""
    nday, n = np.shape(daily["tmax"])
    out = np.zeros((nday, L.N_DAILY, ld), dtype=dtype)
    for f in L.DAILY:
        p0, _ = L.OFF["DAILY"][f.name]
        if f.name in daily:
            out[:, p0, :n] = daily[f.name]
    return out


def hourly_forcing(daily: torch.Tensor, lat: torch.Tensor, ncell: int, jday0: int = 1, day0: int = 0,
                   seed: int = 0, dtime: float = 3600.0, observed_fira: bool = False, out: torch.Tensor | None = None,
                   stream=None, sw_obs: torch.Tensor | None = None, use: torch.Tensor | None = None) -> torch.Tensor:
    """Hourly FORC planes ``(nday * 86400/dtime, N_FORC, ld)`` for ``daily``
    ``(nday, N_DAILY, ld)`` (float32, on the GPU) at latitudes ``lat`` (degrees).

    ``sw_obs`` ``(nday, 86400/dtime, ld)`` float32 and ``use`` ``(nday, ld)``
    bool/uint8: an observed hourly shortwave total for the cell-days ``use``
    marks (``observed_shortwave``, weather.py:458-481)."""
    if daily.dtype != torch.float32 or daily.device.type != "cuda" or daily.dim() != 3:
        raise ValueError("daily must be a (nday, N_DAILY, ld) float32 CUDA tensor")
    nday, npl, ld = daily.shape
    if npl != L.N_DAILY or lat.shape[0] < ld or lat.dtype != torch.float32 or lat.device != daily.device:
        raise ValueError("lat must be a float32 tensor of ld latitudes on the same device")
    nh = int(round(86400.0 / dtime))
    if out is None:
        out = torch.empty((nday * nh, L.N_FORC, ld), dtype=torch.float32, device=daily.device)
    if not (daily.is_contiguous() and out.is_contiguous() and lat.is_contiguous()):
        raise ValueError("buffers must be contiguous")
    stream = stream or torch.cuda.current_stream(daily.device)
    if sw_obs is not None:
        if use is None or sw_obs.shape != (nday, nh, ld) or sw_obs.dtype != torch.float32 or use.shape != (nday, ld):
            raise ValueError(f"sw_obs must be ({nday}, {nh}, {ld}) float32 and use ({nday}, {ld})")
        if sw_obs.device != daily.device or use.device != daily.device:
            raise ValueError("sw_obs and use must be on the daily weather's device")
        use8 = use.to(torch.uint8).contiguous()
        sw_obs = sw_obs.contiguous()
        for t in (use8, sw_obs):               # temporaries the kernel reads on `stream`
            t.record_stream(stream)
        rc = _lib.load().ibis_diurnal_sw_f32(ctypes.c_void_p(daily.data_ptr()), ctypes.c_void_p(lat.data_ptr()),
                                             ctypes.c_void_p(sw_obs.data_ptr()), ctypes.c_void_p(use8.data_ptr()),
                                             ctypes.c_void_p(out.data_ptr()), int(ncell), int(ld), int(nday),
                                             int(jday0), int(day0), float(dtime), int(seed) & 0xFFFFFFFF,
                                             OBSERVED_FIRA if observed_fira else 0,
                                             ctypes.c_void_p(stream.cuda_stream))
        _lib.check(rc, "ibis_diurnal_sw_f32")
        return out
    rc = _lib.load().ibis_diurnal_f32(ctypes.c_void_p(daily.data_ptr()), ctypes.c_void_p(lat.data_ptr()),
                                      ctypes.c_void_p(out.data_ptr()), int(ncell), int(ld), int(nday), int(jday0),
                                      int(day0), float(dtime), int(seed) & 0xFFFFFFFF,
                                      OBSERVED_FIRA if observed_fira else 0, ctypes.c_void_p(stream.cuda_stream))
    _lib.check(rc, "ibis_diurnal_f32")
    return out
