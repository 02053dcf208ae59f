"""Wetland area of the monthly methane: the oracle against the reference.

``tests/golden/wetland_area.npz`` holds the reference's own functions
(``tests/golden/make_golden.py:write_wetland_case``): the learned wetland's
feature builder over 9 months on a 12 x 20 grid (bgc/wetland_learned.py:40-104),
``hybrid_fraction`` (:107-110), and the dynamic area's ``root_zone_water`` /
``dynamic_fraction`` (bgc/wetland_area.py:22-39).  The oracle reproduces every
value bit for bit, scipy's 5 x 5 wrap-around box filter included (checked
against scipy itself on larger grids too).  The tree models are restated from
XGBoost's JSON format (xgboost is not installed, so that part is checked on
models with known answers, not against xgboost), and ``LearnedWetland`` keeps
the reference's cell mapping (tests/test_wetland_learned.py of the reference).
"""
import os

import numpy as np
import pytest

from oracle import wetland as W
from wetland_models import booster_json, random_booster

GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "wetland_area.npz"))


def test_feature_builder_equals_reference():
    z = GOLD
    assert tuple(str(x) for x in z["dyn_feats"]) == W.DYN_FEATS
    assert tuple(str(x) for x in z["stat_feats"]) == W.STAT_FEATS
    fb = W.FeatureBuilder(z["in.I"], z["in.J"], z["in.poros"], z["in.hsoi"], int(z["in.nlat"]), int(z["in.nlon"]))
    for t in range(z["in.ws"].shape[0]):
        f = fb.step(z["in.ts"][t], z["in.ws"][t], z["in.wi"][t], z["in.tg"][t], z["in.prcp"][t], z["in.aet"][t],
                    z["in.runoff"][t])
        for k, name in enumerate(W.DYN_FEATS):
            np.testing.assert_array_equal(f[name], z["out.feats"][t, k], err_msg=f"month {t} {name}")


def test_hybrid_and_dynamic_area_equal_reference():
    z = GOLD
    np.testing.assert_array_equal(W.hybrid_fraction(z["in.fclim"], z["in.P"], z["in.pbar"], z["in.lam"],
                                                    z["in.fmax"]), z["out.hybrid"])
    Wz = W.root_zone_water(z["in.ws"][0], z["in.poros"], z["in.hsoi"], z["in.ts"][0])
    np.testing.assert_array_equal(Wz, z["out.W"])
    frozen = np.asarray(z["in.ts"][0][:, 0], np.float64) <= W.T_FREEZE
    f = W.dynamic_fraction(z["in.fclim"], Wz, z["in.mu"], z["in.sd"], z["in.beta"], z["in.fmin"], z["in.fmax"],
                           frozen=frozen)
    np.testing.assert_array_equal(f, z["out.dynamic"])
    assert frozen.any() and (~frozen).any()


@pytest.mark.parametrize("shape", [(4, 3), (12, 20), (90, 180)])
def test_box_filter_equals_scipy(shape):
    scipy_ndimage = pytest.importorskip("scipy.ndimage")
    rng = np.random.default_rng(sum(shape))
    g = rng.uniform(0.0, 200.0, shape) * (rng.random(shape) < 0.6)
    np.testing.assert_array_equal(W.box_filter_wrap(g), scipy_ndimage.uniform_filter(g, 5, mode="wrap"))


def test_forest_known_answers():
    # tree 0: x0 < 0.5 -> 0.125 ; else (x2 < 3, missing -> left) -> 0.25 / -0.5
    # tree 1: (x1 < -1, missing -> right) -> 0.0625 / 0.03125
    t0 = [("split", 0, 0.5, 1, 2, False), ("leaf", 0.125), ("split", 2, 3.0, 3, 4, True), ("leaf", 0.25),
          ("leaf", -0.5)]
    t1 = [("split", 1, -1.0, 1, 2, False), ("leaf", 0.0625), ("leaf", 0.03125)]
    m = W.Forest(booster_json([t0, t1], base_score="[5E-1]", nfeat=3))
    X = np.array([[0.4, 0.0, 0.0], [0.5, -2.0, 2.0], [0.7, 0.0, 3.0], [0.7, np.nan, np.nan], [np.nan, -1.0, 9.0]],
                 np.float32)
    want = np.float32(0.5) + np.array([0.125 + 0.03125, 0.25 + 0.0625, -0.5 + 0.03125, 0.25 + 0.03125,
                                       -0.5 + 0.03125], np.float32)
    np.testing.assert_array_equal(m.predict(X), want)
    lg = W.Forest(booster_json([t1], base_score="2.5E-1", objective="binary:logistic", nfeat=3))
    margin = np.float32(np.log(0.25 / 0.75)) + np.float32(0.03125)
    np.testing.assert_allclose(lg.predict(X[:1]), 1.0 / (1.0 + np.exp(-margin)), rtol=1e-6)
    with pytest.raises(ValueError):
        W.Forest(booster_json([t1], objective="reg:gamma", nfeat=3))


def _trained_file(tmp_path, rng):
    nf = len(W.DYN_FEATS) + len(W.STAT_FEATS)
    models = [random_booster(rng, ntree=5, depth=2, nfeat=nf) for _ in range(3)]
    cI = np.array([1, 2, 9])
    cJ = np.array([3, 4, 9])                       # (9, 9) is not a land point of the run below
    path = tmp_path / "f.npz"
    np.savez(path, dyn_feats=np.array(W.DYN_FEATS), stat_feats=np.array(W.STAT_FEATS), cells_I=cI, cells_J=cJ,
             band=np.array([0, 1, 2]), pbar=np.full((12, 3), 0.2), fclim=np.full((12, 3), 0.3),
             fmax=np.array([0.5, 0.5, 0.5]), lam=np.array([2.0, 1.0, 1.5]), stat=rng.random((3, len(W.STAT_FEATS))),
             models=np.array(models))
    return path


def test_learned_file_applies_to_its_own_cells_only(tmp_path):
    rng = np.random.default_rng(2)
    path = _trained_file(tmp_path, rng)
    I = np.array([0, 1, 2, 5])
    J = np.array([0, 3, 4, 6])                     # land points; cells (1,3) -> 1, (2,4) -> 2
    lw = W.LearnedWetland(str(path), I, J)
    assert list(lw.pts) == [1, 2] and lw.n_dropped == 1
    feats = {k: rng.random(4) for k in W.DYN_FEATS}
    base = np.array([0.01, 0.02, 0.03, 0.04])
    f = lw.fraction(5, feats, base)
    assert f[0] == base[0] and f[3] == base[3]    # other land points keep the base fraction
    assert np.all((f[1:3] >= 0) & (f[1:3] <= 0.5))
    bad = dict(np.load(path))
    bad["dyn_feats"] = np.array(list(W.DYN_FEATS)[::-1])
    np.savez(tmp_path / "g.npz", **bad)
    with pytest.raises(ValueError):
        W.LearnedWetland(str(tmp_path / "g.npz"), I, J)


def test_forest_arrays_check_the_trees():
    """The host reads boosters into flat node arrays and refuses malformed or
    unsupported ones before anything reaches a GPU."""
    import json
    from ibis_b200.wetland import forest_arrays
    t0 = [("split", 0, 0.5, 1, 2, False), ("leaf", 0.125), ("leaf", -0.5)]
    a = forest_arrays([booster_json([t0], base_score="[5E-1]", nfeat=45)])
    assert a["tree_first"].tolist() == [0, 1] and a["node_first"].tolist() == [0, 3]
    assert a["left"].tolist() == [1, -1, -1] and a["value"].tolist() == [0.5, 0.125, -0.5]
    assert a["base_margin"].tolist() == [0.5] and a["transform"].tolist() == [0]
    bad_child = json.loads(booster_json([t0], nfeat=45))
    bad_child["learner"]["gradient_booster"]["model"]["trees"][0]["right_children"][0] = 7
    bad_feat = json.loads(booster_json([[("split", 60, 0.5, 1, 2, False), ("leaf", 0.1), ("leaf", 0.2)]], nfeat=45))
    for doc in (bad_child, bad_feat):
        with pytest.raises(ValueError):
            forest_arrays([json.dumps(doc)])
    with pytest.raises(ValueError):
        forest_arrays([booster_json([t0], objective="reg:gamma", nfeat=45)])
