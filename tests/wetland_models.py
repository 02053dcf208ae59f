"""Boosters in XGBoost's JSON model format for the learned-wetland tests.

xgboost is not installed here, so the models the tests evaluate are written
directly in the format ``Booster.save_raw('json')`` produces (the fields the
evaluation reads, with the values a real file carries for the rest): a
hand-made model with known answers, and seeded random forests shaped like the
reference's trained ones (depth-limited trees over the 45 predictors).
"""
import json

import numpy as np

NFEAT = 45


def tree_json(nodes, tid=0):
    """``nodes``: list of ("split", feature, threshold, left, right, default_left) or ("leaf", value)."""
    n = len(nodes)
    left, right, feat, cond, dleft, parents = [], [], [], [], [], [-1] * n
    for i, nd in enumerate(nodes):
        if nd[0] == "split":
            _, f, t, l, r, d = nd
            left.append(l); right.append(r); feat.append(f); cond.append(float(t)); dleft.append(int(d))
            parents[l] = i
            parents[r] = i
        else:
            left.append(-1); right.append(-1); feat.append(0); cond.append(float(nd[1])); dleft.append(0)
    return {"base_weights": [0.0] * n, "categories": [], "categories_nodes": [], "categories_segments": [],
            "categories_sizes": [], "default_left": dleft, "id": tid, "left_children": left,
            "loss_changes": [0.0] * n, "parents": [2147483647 if p < 0 else p for p in parents],
            "right_children": right, "split_conditions": cond, "split_indices": feat, "split_type": [0] * n,
            "sum_hessian": [1.0] * n,
            "tree_param": {"num_deleted": "0", "num_feature": str(NFEAT), "num_nodes": str(n), "size_leaf_vector": "1"}}


def booster_json(trees, base_score="5E-1", objective="reg:squarederror", nfeat=NFEAT):
    return json.dumps({
        "learner": {
            "attributes": {}, "feature_names": [], "feature_types": [],
            "gradient_booster": {"model": {
                "gbtree_model_param": {"num_parallel_tree": "1", "num_trees": str(len(trees))},
                "iteration_indptr": list(range(len(trees) + 1)), "tree_info": [0] * len(trees),
                "trees": [tree_json(t, k) for k, t in enumerate(trees)]}, "name": "gbtree"},
            "learner_model_param": {"base_score": base_score, "boost_from_average": "1", "num_class": "0",
                                    "num_feature": str(nfeat), "num_target": "1"},
            "objective": {"name": objective, "reg_loss_param": {"scale_pos_weight": "1"}}},
        "version": [3, 0, 0]})


def random_booster(rng, ntree=20, depth=4, nfeat=NFEAT, lo=None, hi=None):
    """A forest of complete trees of ``depth`` splits on random predictors at
    thresholds drawn inside each predictor's range [lo, hi); random default
    directions; small leaf values (as boosted trees' shrunken leaves)."""
    lo = np.zeros(nfeat) if lo is None else np.asarray(lo, float)
    hi = np.ones(nfeat) if hi is None else np.asarray(hi, float)
    trees = []
    for _ in range(ntree):
        nodes = []
        nsplit = 2 ** depth - 1
        for i in range(nsplit):
            f = int(rng.integers(nfeat))
            t = float(np.float32(rng.uniform(lo[f], hi[f])))
            nodes.append(("split", f, t, 2 * i + 1, 2 * i + 2, bool(rng.integers(2))))
        for _ in range(nsplit + 1):
            nodes.append(("leaf", float(np.float32(rng.normal(0.0, 0.05)))))
        trees.append(nodes)
    return booster_json(trees, base_score=f"{rng.uniform(0.1, 0.4):.6E}")
