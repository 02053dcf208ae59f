"""Wetland (inundated) area of the monthly methane on the device.

The reference has two optional sources of the month's inundated fraction
besides the WAD2M climatology, both host-side numpy there:

* the dynamic wetland area (``python-port/ibis/bgc/wetland_area.py``): the
  climatology scaled by the standardised anomaly of the top metre's liquid
  water -- :func:`dynamic_fraction` (``ibis_wetland_dynamic_f32``);
* the learned wetland area (``python-port/ibis/bgc/wetland_learned.py``): one
  gradient-boosted tree model per wetland band, fed the month's predictors from
  its mean soil state and water totals -- :class:`FeatureBuilder`
  (``ibis_wetland_grid`` / ``ibis_wetland_features``), :class:`LearnedWetland`
  (``ibis_wetland_learned``), and :func:`run_month_learned`, the global
  driver's learned month on a :class:`~ibis_b200.daily.DayLoop`
  (``scripts/run_global.py:786-831``): the month at unit inundated fraction,
  then its flux and annual total scaled by the learned fraction.

The trained file is the reference's (``verify/methane/wetland_learned_train.py
--save``): an ``.npz`` of the predictor names, the file's cells, their bands,
climatologies and bounds, and one XGBoost booster per band saved as JSON.  The
boosters are read here without xgboost (the JSON model format: each tree's
children, split predictors, thresholds / leaf values and default directions)
into flat node arrays the kernel walks.
"""
from __future__ import annotations

import ctypes
import json

import numpy as np
import torch

from . import layout as L
from . import lib as _lib
from .params import FLAG_SOIL_MEANS

ROOT_LAYERS = 4
NFEAT = 33                 # IBIS_WETLAND_NFEAT
NSTAT = 12
NBUF = 28                  # IBIS_WFB_COUNT
DYN_FEATS = ('W', 'Wice', 'ws1', 'ws2', 'ws3', 'ws4', 'ws5', 'ws6', 'wi1', 'wi2', 't1', 't14', 'tg', 'frz1', 'prcp',
             'aet', 'runoff', 'W_l1', 'W_l2', 'W_l3', 'W_3mo', 'prcp_3mo', 'prcp_3mo_l1', 'prcp_3mo_l3', 'runoff_3mo',
             'runoff_3mo_l1', 'runoff_3mo_l3', 'nb_prcp_3mo', 'nb_prcp_3mo_l1', 'nb_prcp_3mo_l2', 'nb_runoff_3mo',
             'nb_runoff_3mo_l1', 'nb_runoff_3mo_l2')
STAT_FEATS = ('FMAX_clm', 'SLOPE', 'STD_ELEV', 'TOPO', 'PCT_WETLAND', 'PCT_LAKE', 'binfl', 'sand', 'clay', 'lat',
              'fmin_w', 'fmax_w')
_TRANSFORM = {"reg:squarederror": 0, "reg:linear": 0, "reg:logistic": 1, "binary:logistic": 1}


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else ctypes.c_void_p(0)


def _stream(device, stream):
    return stream if stream is not None else torch.cuda.current_stream(device)


def dynamic_fraction(cols, area: torch.Tensor, out: torch.Tensor | None = None, params=None, stream=None):
    """The dynamic wetland area of the month for FP32 ``cols``' current state:
    ``area`` ``(6, ld)`` float64 on the device (fclim, mu, sd, beta, fmin, fmax
    of the month); returns ``out`` ``(ld,)`` float32 (e.g. ``cols.stat[IBIS_STAT_F_INUND]``)."""
    from .params import StepParams
    if cols.dtype != torch.float32:
        raise ValueError("the wetland kernels read FP32 columns")
    if area.shape != (6, cols.ld) or area.dtype != torch.float64 or area.device != cols.device:
        raise ValueError(f"area must be a (6, {cols.ld}) float64 tensor on the columns' device")
    out = torch.empty(cols.ld, dtype=torch.float32, device=cols.device) if out is None else out
    p = (params or StepParams()).to_c()
    s = _stream(cols.device, stream)
    rc = _lib.load().ibis_wetland_dynamic_f32(_ptr(cols.prog), _ptr(cols.stat), _ptr(area), _ptr(out), cols.ncell,
                                              cols.ld, ctypes.byref(p), ctypes.c_void_p(s.cuda_stream))
    _lib.check(rc, "ibis_wetland_dynamic_f32")
    return out


class FeatureBuilder:
    """The learned wetland's monthly predictors on the device for ``npoi`` land
    points at grid rows ``I`` and columns ``J`` of an ``nlat`` x ``nlon`` grid;
    ``poros`` ``(npoi, nlayer)`` and ``hsoi`` ``(nlayer,)`` as the model's soil.
    :meth:`step` once per month, in calendar order."""

    def __init__(self, I, J, poros, hsoi, nlat: int = 360, nlon: int = 720, ld: int | None = None, device="cuda"):
        self.device = torch.device(device)
        if self.device.index is None:
            self.device = torch.device("cuda", torch.cuda.current_device())
        I, J = np.asarray(I, np.int64), np.asarray(J, np.int64)
        self.npoi = len(I)
        if len(J) != self.npoi or (self.npoi and (I.min() < 0 or I.max() >= nlat or J.min() < 0 or J.max() >= nlon)):
            raise ValueError("land points must lie on the grid")
        self.ld = L.leading_dim(self.npoi) if ld is None else int(ld)
        self.nlat, self.nlon = int(nlat), int(nlon)
        dev = self.device
        self.cell_i = torch.from_numpy(I.astype(np.int32)).to(dev)
        self.cell_j = torch.from_numpy(J.astype(np.int32)).to(dev)
        por = np.zeros((ROOT_LAYERS, self.ld))
        por[:, :self.npoi] = np.asarray(poros, np.float64)[:, :ROOT_LAYERS].T
        self.poros = torch.from_numpy(por).to(dev)
        self.hsoi = [float(x) for x in np.asarray(hsoi, np.float64)[:ROOT_LAYERS]]
        self.lf = torch.zeros(self.nlat * self.nlon, dtype=torch.float64, device=dev)
        self.buf = torch.zeros((NBUF, self.ld), dtype=torch.float64, device=dev)
        self.work = torch.zeros((4, self.nlat * self.nlon), dtype=torch.float64, device=dev)
        self.nmonth = 0
        _lib.check(_lib.load().ibis_wetland_grid(ctypes.byref(self._c()), ctypes.c_void_p(
            torch.cuda.current_stream(dev).cuda_stream)), "ibis_wetland_grid")

    def _c(self):
        c = _lib.IbisWetlandBuilderC(npoi=self.npoi, ld=self.ld, nlat=self.nlat, nlon=self.nlon,
                                     cell_i=self.cell_i.data_ptr(), cell_j=self.cell_j.data_ptr(),
                                     poros=self.poros.data_ptr(), lf=self.lf.data_ptr(), buf=self.buf.data_ptr(),
                                     work=self.work.data_ptr(), nmonth=self.nmonth)
        for k in range(ROOT_LAYERS):
            c.hsoi[k] = self.hsoi[k]
        return c

    def step(self, means: torch.Tensor, totals: torch.Tensor, out: torch.Tensor | None = None, stream=None):
        """``means`` ``(19, ld)`` float32 (tsoi 6, wsoi 6, wisoi 6, tg: the month's
        means), ``totals`` ``(3, ld)`` float32 (precipitation, AET, runoff +
        drainage of the month), on the device; returns ``(33, ld)`` float64
        predictors in the model's order (``DYN_FEATS``)."""
        for t, k in ((means, 19), (totals, 3)):
            if t.shape != (k, self.ld) or t.dtype != torch.float32 or t.device != self.device or not t.is_contiguous():
                raise ValueError(f"expected a contiguous ({k}, {self.ld}) float32 tensor on {self.device}")
        out = torch.empty((NFEAT, self.ld), dtype=torch.float64, device=self.device) if out is None else out
        s = _stream(self.device, stream)
        rc = _lib.load().ibis_wetland_features(ctypes.byref(self._c()), _ptr(means), _ptr(totals), _ptr(out),
                                               ctypes.c_void_p(s.cuda_stream))
        _lib.check(rc, "ibis_wetland_features")
        self.nmonth += 1
        return out

    def step_host(self, tsoi_mean, wsoi_mean, wisoi_mean, tg_mean, prcp, aet, runoff) -> dict:
        """:meth:`step` with the reference's arguments as host arrays
        (``FeatureBuilder.step``): returns ``{name: (npoi,) array}``."""
        m = np.zeros((19, self.ld), np.float32)
        n = self.npoi
        m[0:6, :n] = np.asarray(tsoi_mean, np.float32).T
        m[6:12, :n] = np.asarray(wsoi_mean, np.float32).T
        m[12:18, :n] = np.asarray(wisoi_mean, np.float32).T
        m[18, :n] = np.asarray(tg_mean, np.float32)
        t = np.zeros((3, self.ld), np.float32)
        for k, v in enumerate((prcp, aet, runoff)):
            t[k, :n] = np.asarray(v, np.float32)
        f = self.step(torch.from_numpy(m).to(self.device), torch.from_numpy(t).to(self.device)).cpu().numpy()
        return {name: f[k, :n] for k, name in enumerate(DYN_FEATS)}


def _base_score(s) -> float:
    s = str(s).strip()
    if s.startswith("["):
        vals = [float(v) for v in s.strip("[]").split(",") if v.strip()]
        if len(vals) != 1:
            raise ValueError("only single-target boosters are supported")
        return vals[0]
    return float(s)


def forest_arrays(models, nfeat: int = NFEAT + NSTAT) -> dict:
    """Flat node arrays of boosters given as XGBoost JSON texts, one per band;
    every child index, split predictor and tree is checked."""
    tree_first, node_first = [0], [0]
    left, right, feat, value, dleft, base, trans = [], [], [], [], [], [], []
    for text in models:
        doc = json.loads(str(text))
        learner = doc["learner"]
        obj = learner["objective"]["name"]
        if obj not in _TRANSFORM:
            raise ValueError(f"booster objective {obj!r} is not supported")
        mp = learner["learner_model_param"]
        if int(mp.get("num_class", "0")) > 1 or int(mp.get("num_target", "1")) != 1:
            raise ValueError("only single-target boosters are supported")
        if int(mp["num_feature"]) > nfeat:
            raise ValueError(f"booster has {mp['num_feature']} predictors, the file {nfeat}")
        b = _base_score(mp["base_score"])
        if _TRANSFORM[obj] == 1:
            b = float(np.log(b / (1.0 - b)))
        base.append(np.float32(b))
        trans.append(_TRANSFORM[obj])
        for t in learner["gradient_booster"]["model"]["trees"]:
            lc, rc = np.asarray(t["left_children"], np.int64), np.asarray(t["right_children"], np.int64)
            si = np.asarray(t["split_indices"], np.int64)
            n = len(lc)
            if n == 0 or len(rc) != n or len(si) != n or len(t["split_conditions"]) != n or len(t["default_left"]) != n:
                raise ValueError("malformed tree")
            if any(int(x) != 0 for x in t.get("split_type", [])):
                raise ValueError("categorical splits are not supported")
            inner = lc >= 0
            if np.any((lc >= n) | (rc >= n) | (inner & ((rc < 0) | (lc == 0) | (rc == 0))) |
                      (inner & ((si < 0) | (si >= nfeat)))):
                raise ValueError("malformed tree")
            left += lc.tolist()
            right += rc.tolist()
            feat += np.where(inner, si, 0).tolist()
            value += np.asarray(t["split_conditions"], np.float64).astype(np.float32).tolist()
            dleft += [int(bool(x)) for x in t["default_left"]]
            node_first.append(node_first[-1] + n)
        tree_first.append(len(node_first) - 1)
    return dict(tree_first=np.asarray(tree_first, np.int32), node_first=np.asarray(node_first, np.int32),
                left=np.asarray(left, np.int32), right=np.asarray(right, np.int32), feature=np.asarray(feat, np.int32),
                value=np.asarray(value, np.float32), default_left=np.asarray(dleft, np.uint8),
                base_margin=np.asarray(base, np.float32), transform=np.asarray(trans, np.int32))


class LearnedWetland:
    """The trained file applied to a run's ``npoi`` land points at grid rows
    ``I`` and columns ``J`` (the reference's ``LearnedWetland``): the file's
    cells that are not land points of the run are dropped (``n_dropped``)."""

    def __init__(self, path_or_arrays, I, J, ld: int | None = None, device="cuda"):
        z = np.load(path_or_arrays, allow_pickle=False) if isinstance(path_or_arrays, str) else path_or_arrays
        dyn = tuple(str(x) for x in z['dyn_feats'])
        stat = tuple(str(x) for x in z['stat_feats'])
        if dyn != DYN_FEATS or stat != STAT_FEATS:
            raise ValueError(f'feature list differs from the model order (file {dyn + stat})')
        self.device = torch.device(device)
        if self.device.index is None:
            self.device = torch.device("cuda", torch.cuda.current_device())
        self.npoi = len(I)
        self.ld = L.leading_dim(self.npoi) if ld is None else int(ld)
        pos = {(int(i), int(j)): p for p, (i, j) in enumerate(zip(np.asarray(I), np.asarray(J)))}
        keep = np.array([(int(i), int(j)) in pos for i, j in zip(z['cells_I'], z['cells_J'])], bool)
        self.pts = np.array([pos[(int(i), int(j))] for i, j, k in zip(z['cells_I'], z['cells_J'], keep) if k],
                            np.int64)
        self.band = np.asarray(z['band'], np.int64)[keep]
        self.n_dropped = int((~keep).sum())
        models = [str(js) for js in z['models']]
        if self.band.size and (self.band.min() < 0 or self.band.max() >= len(models)):
            raise ValueError("a cell's band has no model")
        arrays = forest_arrays(models)
        dev = self.device
        self._arrays = {k: torch.from_numpy(v).to(dev) for k, v in arrays.items()}
        self.nband = len(models)
        self.pbar = torch.from_numpy(np.ascontiguousarray(np.asarray(z['pbar'], np.float64)[:, keep])).to(dev)
        self.fclim = torch.from_numpy(np.ascontiguousarray(np.asarray(z['fclim'], np.float64)[:, keep])).to(dev)
        self.fmax = torch.from_numpy(np.asarray(z['fmax'], np.float64)[keep].copy()).to(dev)
        lam = np.asarray(z['lam'], np.float64)
        if lam.shape != (self.nband,):
            raise ValueError(f"the file has {lam.size} band inflations for {self.nband} models")
        self.lam = torch.from_numpy(lam.copy()).to(dev)
        self.stat = torch.from_numpy(np.ascontiguousarray(np.asarray(z['stat'], np.float64)[keep])).to(dev)
        self._pts = torch.from_numpy(self.pts.astype(np.int32)).to(dev)
        self._band = torch.from_numpy(self.band.astype(np.int32)).to(dev)

    def _forest(self):
        a = self._arrays
        return _lib.IbisForestC(nband=self.nband, nfeat=NFEAT + NSTAT, **{k: a[k].data_ptr() for k in (
            "tree_first", "node_first", "left", "right", "feature", "value", "default_left", "base_margin",
            "transform")})

    def fraction(self, imonth: int, feats: torch.Tensor, f_base: torch.Tensor, out: torch.Tensor | None = None,
                 stream=None) -> torch.Tensor:
        """The month's inundated fraction ``(ld,)`` float32 over the land points:
        the file's cells from the hybrid of the climatology and the learned
        anomaly, every other point ``f_base`` (the month's climatology)."""
        if feats.shape != (NFEAT, self.ld) or feats.dtype != torch.float64 or feats.device != self.device:
            raise ValueError(f"feats must be ({NFEAT}, {self.ld}) float64 on {self.device}")
        if f_base.shape != (self.ld,) or f_base.dtype != torch.float32 or f_base.device != self.device:
            raise ValueError(f"f_base must be ({self.ld},) float32 on {self.device}")
        out = torch.empty(self.ld, dtype=torch.float32, device=self.device) if out is None else out
        m = int(imonth)
        s = _stream(self.device, stream)
        rc = _lib.load().ibis_wetland_learned(ctypes.byref(self._forest()), _ptr(feats), self.npoi, self.ld,
                                              _ptr(self._pts), _ptr(self._band), _ptr(self.fclim[m]),
                                              _ptr(self.pbar[m]), _ptr(self.fmax), _ptr(self.stat), _ptr(self.lam),
                                              len(self.pts), _ptr(f_base), _ptr(out), ctypes.c_void_p(s.cuda_stream))
        _lib.check(rc, "ibis_wetland_learned")
        return out

    def fraction_host(self, imonth: int, feats: dict, f_base) -> np.ndarray:
        """:meth:`fraction` with the reference's arguments (``LearnedWetland.fraction``):
        ``feats`` ``{name: (npoi,) array}``, ``f_base`` ``(npoi,)``; returns the
        ``(npoi,)`` float32 fraction."""
        fd = np.zeros((NFEAT, self.ld))
        for k, name in enumerate(DYN_FEATS):
            fd[k, :self.npoi] = np.asarray(feats[name], np.float64)
        fb = np.zeros(self.ld, np.float32)
        fb[:self.npoi] = np.asarray(f_base, np.float32)
        out = self.fraction(imonth, torch.from_numpy(fd).to(self.device), torch.from_numpy(fb).to(self.device))
        return out.cpu().numpy()[:self.npoi]


def run_month_learned(loop, daily: torch.Tensor, fb: FeatureBuilder, lw: LearnedWetland, imonth: int,
                      f_base: torch.Tensor, from_mean: bool = True, partition: bool = False, new_year: bool = False,
                      stream=None) -> torch.Tensor:
    """The global driver's month under the learned wetland area
    (scripts/run_global.py:786-831) on a DayLoop whose step parameters carry
    FLAG_SOIL_MEANS and FLAG_CH4: the month at unit inundated fraction, then the
    predictors from its mean soil state and water totals (precipitation, AET,
    runoff + drainage), the learned fraction, and the month's methane step with
    the flux and its share of the annual total scaled by it (scale_month).
    Returns the fraction ``(ld,)``; the STAT f_inund plane is left at 1."""
    cols = loop.cols
    if not loop.params.flags & FLAG_SOIL_MEANS:
        raise ValueError("the learned wetland needs the month's soil means: set FLAG_SOIL_MEANS in the loop's params")
    if fb.ld != cols.ld or lw.ld != cols.ld or cols.dtype != torch.float32:
        raise ValueError("the builder, the file and the FP32 columns must share the leading dimension")
    s = _stream(cols.device, stream)
    nacc = L.N_ACC
    # the month-mean planes in the builder's order (tsoi 6, wsoi 6, wisoi 6, tg), then runoff and drainage
    mean_planes = [L.OFF["ACC"][k][0] + j for k in ("tsoi_mean", "wsoi_mean", "wisoi_mean", "tg_mean")
                   for j in range(L.OFF["ACC"][k][1])]
    acc_planes = torch.tensor(mean_planes + [L.OFF["ACC"]["aytrunof"][0], L.OFF["ACC"]["aytdrain"][0]],
                              device=cols.device)
    day_planes = torch.tensor([L.OFF["DAYST"]["ayprcp"][0], L.OFF["DAYST"]["ayaet"][0]], device=cols.device)
    f_in = L.OFF["STAT"]["f_inund"][0]
    with torch.cuda.stream(s):
        loop.begin_month(new_year, s)
        acc0 = cols.acc[acc_planes] - cols.acc[acc_planes + nacc]
        day0 = loop.dayst[day_planes].clone()
        cols.stat[f_in].fill_(1.0)
        loop.run(daily, s)
        ndays = daily.shape[0]
        d_acc = (cols.acc[acc_planes] - cols.acc[acc_planes + nacc]) - acc0
        d_day = loop.dayst[day_planes] - day0
        means = (d_acc[:19] / ndays).to(torch.float32).contiguous()
        totals = torch.stack([d_day[0], d_day[1], d_acc[19] + d_acc[20]]).to(torch.float32).contiguous()
        feats = fb.step(means, totals, stream=s)
        f = lw.fraction(imonth, feats, f_base, stream=s)
        loop.end_month(ndays, from_mean, f, partition, s)
    return f


__all__ = ["dynamic_fraction", "FeatureBuilder", "LearnedWetland", "forest_arrays", "run_month_learned",
           "DYN_FEATS", "STAT_FEATS"]
