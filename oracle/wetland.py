"""Wetland (inundated) area of the monthly methane in float64 -- TEST INFRASTRUCTURE ONLY.

Restates the reference's two optional sources of the month's inundated
fraction:

* the dynamic wetland area, ``root_zone_water`` and ``dynamic_fraction``
  (``python-port/ibis/bgc/wetland_area.py:22-39``);
* the learned wetland area (``python-port/ibis/bgc/wetland_learned.py``): the
  month-by-month predictors of ``FeatureBuilder`` (:49-104), ``hybrid_fraction``
  (:107-110) and ``LearnedWetland`` (:113-160), the last applying one
  gradient-boosted tree model per wetland band.

Two third-party pieces sit under the learned path and are restated here:

* the 5 x 5 neighbourhood means use scipy's ``uniform_filter(g, 5,
  mode='wrap')`` (scipy >= 1.10, the reference's ``wetland`` extra,
  ``python-port/pyproject.toml:23``): per axis in order (rows' axis first), each
  line extended periodically, a running sum started from the first window's
  sequential sum and moved by ``+= entering - leaving``, each output the sum
  divided by the width.  Checked bit for bit against scipy's own output on the
  committed fixture (``tests/test_wetland.py``).
* the tree models are XGBoost boosters (``xgboost >= 3.0``, same extra) saved as
  JSON (``save_raw('json')``, ``verify/methane/wetland_learned_train.py:124``).
  xgboost is not installed here, so their evaluation is restated from the
  published JSON model format: ``learner.gradient_booster.model.trees``, each
  tree's ``left_children`` / ``right_children`` (-1 at a leaf),
  ``split_indices``, ``split_conditions`` (the threshold of a split node, the
  value of a leaf) and ``default_left``; a row goes left when its feature is
  below the threshold (float32 comparison), and where the feature is missing
  (NaN) the way ``default_left`` says; the prediction is the float32 sum, tree
  by tree, of the leaves reached, started from the margin of
  ``learner_model_param.base_score``, then the objective's transform (identity
  for ``reg:squarederror``, the training script's objective).  That part is
  parity-unpinned: no xgboost output exists here to check it against.
"""
from __future__ import annotations

import json

import numpy as np

ROOT_LAYERS = 4          # wetland_learned.py:36, wetland_area.py:18
NB = 5                   # wetland_learned.py:37
T_FREEZE = 273.16        # wetland_area.py:19
DYN_FEATS = ('W', 'Wice', 'ws1', 'ws2', 'ws3', 'ws4', 'ws5', 'ws6', 'wi1', 'wi2', 't1', 't14', 'tg', 'frz1', 'prcp',
             'aet', 'runoff', 'W_l1', 'W_l2', 'W_l3', 'W_3mo', 'prcp_3mo', 'prcp_3mo_l1', 'prcp_3mo_l3', 'runoff_3mo',
             'runoff_3mo_l1', 'runoff_3mo_l3', 'nb_prcp_3mo', 'nb_prcp_3mo_l1', 'nb_prcp_3mo_l2', 'nb_runoff_3mo',
             'nb_runoff_3mo_l1', 'nb_runoff_3mo_l2')          # wetland_learned.py:26-29, model order
STAT_FEATS = ('FMAX_clm', 'SLOPE', 'STD_ELEV', 'TOPO', 'PCT_WETLAND', 'PCT_LAKE', 'binfl', 'sand', 'clay', 'lat',
              'fmin_w', 'fmax_w')                             # wetland_learned.py:30


# ---------------------------------------------------------------------------
# dynamic wetland area (wetland_area.py:22-39)
# ---------------------------------------------------------------------------
def root_zone_water(wsoi, poros, hsoi, tsoi=None, nlay=ROOT_LAYERS):
    """sum over the top ``nlay`` layers of wsoi * poros * hsoi, a frozen layer (tsoi <= 273.16 K) counting 0."""
    w = np.asarray(wsoi, np.float64)[:, :nlay] * np.asarray(poros, np.float64)[:, :nlay] * \
        np.asarray(hsoi, np.float64)[None, :nlay]
    if tsoi is not None:
        w = np.where(np.asarray(tsoi, np.float64)[:, :nlay] > T_FREEZE, w, 0.0)
    return w.sum(axis=1)


def dynamic_fraction(f_clim, W, mu, sd, beta, f_min, f_max, frozen=None):
    """clip(f_clim (1 + beta A), f_min, f_max) clipped to [0, 1]; A = (W - mu)/sd (0 where sd <= 1e-9 or frozen)."""
    f_clim, W, mu, sd = (np.asarray(x, np.float64) for x in (f_clim, W, mu, sd))
    A = np.where(sd > 1e-9, (W - mu) / np.maximum(sd, 1e-9), 0.0)
    if frozen is not None:
        A = np.where(np.asarray(frozen, bool), 0.0, A)
    f = np.clip(f_clim * (1.0 + np.asarray(beta, np.float64) * A), np.asarray(f_min, np.float64),
                np.asarray(f_max, np.float64))
    return np.clip(f, 0.0, 1.0)


# ---------------------------------------------------------------------------
# learned wetland area (wetland_learned.py)
# ---------------------------------------------------------------------------
def box_filter_wrap(g, size=NB):
    """scipy.ndimage.uniform_filter(g, size, mode='wrap') on a 2-D grid, restated (module docstring)."""
    out = np.asarray(g, np.float64)
    s1 = size // 2
    s2 = size - s1 - 1
    for axis in (0, 1):
        x = np.moveaxis(out, axis, 0)
        n = x.shape[0]
        ext = x[np.arange(-s1, n + s2) % n]
        res = np.empty_like(x)
        tmp = ext[0].copy()
        for k in range(1, size):
            tmp = tmp + ext[k]
        res[0] = tmp / size
        for l in range(1, n):
            tmp = tmp + (ext[l + size - 1] - ext[l - 1])
            res[l] = tmp / size
        out = np.moveaxis(res, 0, axis)
    return out


def _mean3(lst):
    return np.mean(lst[-3:], axis=0)


def _lag(lst, L):
    return lst[-1 - L] if len(lst) > L else lst[-1]


class FeatureBuilder:
    """The month's predictors from its MEAN soil state and its water totals
    (wetland_learned.py:40-104): buffers of the last months for the lags, the
    3-month means and the 5 x 5 neighbourhood means on the (nlat, nlon) grid."""

    def __init__(self, I, J, poros, hsoi, nlat=360, nlon=720):
        self.I = np.asarray(I, int)
        self.J = np.asarray(J, int)
        self.nlat, self.nlon = nlat, nlon
        self.p4 = np.asarray(poros, np.float64)[:, :ROOT_LAYERS]
        self.h4 = np.asarray(hsoi, np.float64)[:ROOT_LAYERS]
        lm = np.zeros((nlat, nlon))
        lm[self.I, self.J] = 1.0
        self.lf = box_filter_wrap(lm)
        self.buf = {k: [] for k in ('W', 'prcp', 'runoff', 'W3', 'P3', 'R3', 'NP3', 'NR3')}

    def _nb(self, v):
        g = np.zeros((self.nlat, self.nlon))
        g[self.I, self.J] = v
        return (box_filter_wrap(g) / np.maximum(self.lf, 1e-6))[self.I, self.J]

    def _push(self, k, v, keep=4):
        self.buf[k].append(v)
        if len(self.buf[k]) > keep:
            self.buf[k].pop(0)

    def step(self, tsoi_mean, wsoi_mean, wisoi_mean, tg_mean, prcp, aet, runoff):
        ws = np.asarray(wsoi_mean, np.float64)
        wi = np.asarray(wisoi_mean, np.float64)
        ts = np.asarray(tsoi_mean, np.float64)
        W = (ws[:, :ROOT_LAYERS] * self.p4 * self.h4[None, :]).sum(1)
        Wice = (wi[:, :ROOT_LAYERS] * self.p4 * self.h4[None, :]).sum(1)
        prcp = np.asarray(prcp, np.float64)
        runoff = np.asarray(runoff, np.float64)
        f = {'W': W, 'Wice': Wice}
        for l in range(6):
            f[f'ws{l + 1}'] = ws[:, l]
        f.update({'wi1': wi[:, 0], 'wi2': wi[:, 1], 't1': ts[:, 0],
                  't14': (ts[:, :ROOT_LAYERS] * self.h4[None, :]).sum(1) / self.h4.sum(),
                  'tg': np.asarray(tg_mean, np.float64),
                  'frz1': wi[:, 0] / np.maximum(ws[:, 0] + wi[:, 0], 1e-6), 'prcp': prcp,
                  'aet': np.asarray(aet, np.float64), 'runoff': runoff})
        b = self.buf
        self._push('W', W)
        self._push('prcp', prcp, 3)
        self._push('runoff', runoff, 3)
        self._push('W3', _mean3(b['W']))
        self._push('P3', _mean3(b['prcp']))
        self._push('R3', _mean3(b['runoff']))
        # the mean of the last grids of prcp / runoff is the grid of the mean of
        # their last values (land points only, zero elsewhere): filter that
        self._push('NP3', self._nb(b['P3'][-1]), 3)
        self._push('NR3', self._nb(b['R3'][-1]), 3)
        f.update({'W_l1': _lag(b['W'], 1), 'W_l2': _lag(b['W'], 2), 'W_l3': _lag(b['W'], 3), 'W_3mo': b['W3'][-1],
                  'prcp_3mo': b['P3'][-1], 'prcp_3mo_l1': _lag(b['P3'], 1), 'prcp_3mo_l3': _lag(b['P3'], 3),
                  'runoff_3mo': b['R3'][-1], 'runoff_3mo_l1': _lag(b['R3'], 1), 'runoff_3mo_l3': _lag(b['R3'], 3),
                  'nb_prcp_3mo': b['NP3'][-1], 'nb_prcp_3mo_l1': _lag(b['NP3'], 1),
                  'nb_prcp_3mo_l2': _lag(b['NP3'], 2), 'nb_runoff_3mo': b['NR3'][-1],
                  'nb_runoff_3mo_l1': _lag(b['NR3'], 1), 'nb_runoff_3mo_l2': _lag(b['NR3'], 2)})
        return f


def hybrid_fraction(fclim_m, P, Pbar_m, lam, fmax):
    """clip(fclim + lam (P - Pbar), 0, fmax) (wetland_learned.py:107-110)."""
    return np.clip(np.asarray(fclim_m, np.float64) + np.asarray(lam, np.float64) *
                   (np.asarray(P, np.float64) - np.asarray(Pbar_m, np.float64)), 0.0, np.asarray(fmax, np.float64))


# ---------------------------------------------------------------------------
# gradient-boosted tree models (XGBoost JSON format, restated; module docstring)
# ---------------------------------------------------------------------------
_TRANSFORMS = {"reg:squarederror": None, "reg:linear": None, "reg:logistic": "sigmoid",
               "binary:logistic": "sigmoid"}


def _base_score(s):
    s = str(s).strip()
    if s.startswith("["):
        vals = [float(v) for v in s.strip("[]").split(",") if v.strip()]
        if len(vals) != 1:
            raise ValueError("only single-target boosters are supported")
        return vals[0]
    return float(s)


class Forest:
    """One booster: its trees as flat arrays, its base margin and transform."""

    def __init__(self, text):
        doc = json.loads(text)
        learner = doc["learner"]
        obj = learner["objective"]["name"]
        if obj not in _TRANSFORMS:
            raise ValueError(f"objective {obj!r} is not supported")
        mp = learner["learner_model_param"]
        if int(mp.get("num_class", "0")) > 1 or int(mp.get("num_target", "1")) != 1:
            raise ValueError("only single-target boosters are supported")
        self.num_feature = int(mp["num_feature"])
        base = _base_score(mp["base_score"])
        self.transform = _TRANSFORMS[obj]
        if self.transform == "sigmoid":
            base = float(np.log(base / (1.0 - base)))      # the margin of the base probability
        self.base_margin = np.float32(base)
        model = learner["gradient_booster"]["model"]
        self.trees = []
        for t in model["trees"]:
            if any(int(x) != 0 for x in t.get("split_type", [])):
                raise ValueError("categorical splits are not supported")
            self.trees.append((np.asarray(t["left_children"], np.int64), np.asarray(t["right_children"], np.int64),
                               np.asarray(t["split_indices"], np.int64),
                               np.asarray(t["split_conditions"], np.float64).astype(np.float32),
                               np.asarray(t["default_left"], np.int64).astype(bool)))

    def predict(self, X):
        X = np.asarray(X, np.float32)
        out = np.full(X.shape[0], self.base_margin, np.float32)
        rows = np.arange(X.shape[0])
        for left, right, feat, cond, dleft in self.trees:
            node = np.zeros(X.shape[0], np.int64)
            while True:
                inner = left[node] >= 0
                if not inner.any():
                    break
                v = X[rows, feat[node]]
                go_left = np.where(np.isnan(v), dleft[node], v < cond[node])
                node = np.where(inner, np.where(go_left, left[node], right[node]), node)
            out = (out + cond[node]).astype(np.float32)
        if self.transform == "sigmoid":
            out = (np.float32(1.0) / (np.float32(1.0) + np.exp(-out))).astype(np.float32)
        return out


class LearnedWetland:
    """The trained file applied to a run's land points (wetland_learned.py:113-160):
    ``I``, ``J`` the run's land points on the grid; the file's cells that are
    not land points of the run are dropped."""

    def __init__(self, path_or_dict, I, J):
        z = np.load(path_or_dict, allow_pickle=False) if isinstance(path_or_dict, str) else path_or_dict
        dyn = tuple(str(x) for x in z['dyn_feats'])
        stat = tuple(str(x) for x in z['stat_feats'])
        if dyn != DYN_FEATS or stat != STAT_FEATS:
            raise ValueError(f'feature list differs from the model order (file {dyn + stat})')
        pos = {(int(i), int(j)): p for p, (i, j) in enumerate(zip(np.asarray(I), np.asarray(J)))}
        keep = np.array([(int(i), int(j)) in pos for i, j in zip(z['cells_I'], z['cells_J'])])
        self.pts = np.array([pos[(int(i), int(j))] for i, j, k in zip(z['cells_I'], z['cells_J'], keep) if k], int)
        self.band = np.asarray(z['band'])[keep]
        self.pbar = np.asarray(z['pbar'], np.float64)[:, keep]
        self.fclim = np.asarray(z['fclim'], np.float64)[:, keep]
        self.fmax = np.asarray(z['fmax'], np.float64)[keep]
        self.lam = np.asarray(z['lam'], np.float64)
        self.stat = np.asarray(z['stat'], np.float64)[keep]
        self.models = [Forest(str(js)) for js in z['models']]
        self.n_dropped = int((~keep).sum())

    def features(self, feats):
        X = np.empty((len(self.pts), len(DYN_FEATS) + len(STAT_FEATS)), np.float32)
        for c, k in enumerate(DYN_FEATS):
            X[:, c] = feats[k][self.pts]
        X[:, len(DYN_FEATS):] = self.stat
        return X

    def predict(self, feats):
        X = self.features(feats)
        P = np.full(len(self.pts), np.nan)
        for b, m in enumerate(self.models):
            sel = self.band == b
            if sel.any():
                P[sel] = np.clip(m.predict(X[sel]), 0.0, 1.0)
        return P

    def fraction(self, imonth, feats, f_base):
        P = self.predict(feats)
        f = np.array(f_base, np.float64, copy=True)
        f[self.pts] = hybrid_fraction(self.fclim[imonth], P, self.pbar[imonth], self.lam[self.band], self.fmax)
        return np.clip(f, 0.0, 1.0)
