"""The reference's restart (checkpoint) files, read and written without JAX.

The reference saves an ``IBISState`` as one ``.npz``: every leaf of
``jax.tree.flatten(state)`` as ``leaf_{i}`` in flatten order (the Equinox
field order of the state modules), ``num_leaves``, ``treedef_repr`` and
``meta_*`` entries (python-port/ibis/io/restart.py:19-52), and loads it into a
template state of the same structure (restart.py:63-193).  This module keeps
that order as data (:data:`LEAVES`, the 258 leaves of the base state with
bedrock, generated from the reference's own state classes) so a checkpoint can
seed device columns, and device columns can be written back as a checkpoint,
with no JAX present:

* :func:`load` -> ``{leaf path: array}`` and the metadata;
* :func:`columns_from_restart` -> :class:`~ibis_b200.columns.Columns` plus the
  parameter record the state implies (soil layer thicknesses, root profile,
  CO2);
* :func:`write_columns` / :func:`save` -> a checkpoint the reference's
  ``load_state`` reads, with the prognostic (and, if kept, diagnostic) leaves
  taken from the columns and every other leaf carried over.

After the base leaves a checkpoint can carry optional modules, in the
state's field order (state/model_state.py:40-63).  Those the day loop uses are
named by their count, as the reference's loader identifies them
(io/restart.py:60-62, 94-133): the wetland CH4 state (3 leaves; a saved tree
structure naming ``MethaneState`` settles it, else the count), then the chain
of calibration modules, each implying the ones before it -- StressAccum (4
leaves; 3 in files written before its smoothed-stress leaf), ETParts,
SeasonalState, NEEParts (0, 4, 8, 11 or 13 leaves; 3, 7, 10 or 12 in the old
form).  Trailing leaves that no such count explains (permafrost, fire, BVOC
modules) are kept untouched and copied through by position.
"""
from __future__ import annotations

import re
import types

import numpy as np

from . import layout as L
from .restart_leaves import LEAVES

BEDROCK_LEAF = "soil.tsoi_deep"


WETLAND_LEAVES = ("wetland.flux", "wetland.annual", "wetland.zwt")
CHAIN = (("stress.aystressu", "stress.aystressl", "stress.nday", "stress.u_smooth"),
         ("etparts.trans", "etparts.interc", "etparts.soilev", "etparts.snowsub"),
         ("seasonal.acclim_x", "seasonal.ssen_u", "seasonal.ssen_l"),
         ("neeparts.night", "neeparts.day"))
TRAILING = WETLAND_LEAVES + tuple(p for mod in CHAIN for p in mod)
OLD_STRESS_LEAVES = 3


def _chain_names(n: int, old: bool):
    """Leaf names of a chain of ``n`` leaves (``old``: the 3-leaf StressAccum), or None."""
    names = []
    for k, mod in enumerate(CHAIN):
        if len(names) >= n:
            break
        names += list(mod[:OLD_STRESS_LEAVES] if old and k == 0 else mod)
    return names if len(names) == n else None


def trailing_names(n: int, treedef_repr: str | None = None):
    """Names of the ``n`` leaves after the base state, or None when the count
    (and the saved tree structure) does not identify them."""
    chain = lambda m: m >= 0 and (_chain_names(m, False) is not None or _chain_names(m, True) is not None)
    wet = ("MethaneState" in treedef_repr) if treedef_repr is not None else (not chain(n) and chain(n - 3))
    rest = n - (len(WETLAND_LEAVES) if wet else 0)
    if rest < 0:
        return None
    names = _chain_names(rest, False) or _chain_names(rest, True)
    if names is None:
        return None
    return (list(WETLAND_LEAVES) if wet else []) + names


def _soil_leaf_count(treedef_repr: str):
    """Children of the SoilState node in a saved tree structure, or None."""
    m = re.search(r"SoilState\[[^\]]*\], \[([^\]]*)\]", treedef_repr)
    return None if m is None else m.group(1).count("*")


def base_leaves(bedrock: bool):
    """Leaf paths of the base state in checkpoint order."""
    return [p for p in LEAVES if bedrock or p != BEDROCK_LEAF]


def _bedrock_from_shapes(arrays):
    """Whether a checkpoint without a saved tree structure carries the bedrock
    leaf: its position holds ``soil.tsoi_deep`` (npoi, nbedrock) with bedrock
    and ``snow.fi`` (npoi,) without."""
    i = LEAVES.index(BEDROCK_LEAF)
    a = arrays[i] if i < len(arrays) else None
    return a is not None and np.ndim(a) == 2


def load_full(path: str):
    """Read a checkpoint.  Returns ``(leaves, meta, extra, treedef_repr)``: the
    base leaves and the named optional modules (:func:`trailing_names`) by path,
    the ``meta_*`` entries, trailing leaves no count identifies (a list, by
    position), and the saved tree structure (None when the file has none)."""
    z = np.load(path, allow_pickle=False)
    n = int(z["num_leaves"])
    arrays = [None if f"leaf_{i}_is_none" in z.files else z[f"leaf_{i}"] for i in range(n)]
    nsoil_all = sum(1 for p in LEAVES if p.startswith("soil."))
    tree = str(z["treedef_repr"]) if "treedef_repr" in z.files else None
    if tree is not None:
        k = _soil_leaf_count(tree)
        if k is None:
            raise ValueError(f"{path}: no SoilState in the saved tree structure")
        bedrock = k == nsoil_all
    else:
        bedrock = _bedrock_from_shapes(arrays)
    names = base_leaves(bedrock)
    if n < len(names):
        raise ValueError(f"{path}: {n} leaves, the base state has {len(names)}")
    leaves = dict(zip(names, arrays[:len(names)]))
    meta = {k[5:]: (z[k].item() if z[k].ndim == 0 else z[k]) for k in z.files if k.startswith("meta_")}
    trail = arrays[len(names):]
    tnames = trailing_names(len(trail), tree)
    if tnames is None:
        return leaves, meta, trail, tree
    leaves.update(zip(tnames, trail))
    return leaves, meta, [], tree


def load(path: str):
    """Read a checkpoint: ``(leaves, meta, extra)`` of :func:`load_full`."""
    leaves, meta, extra, _ = load_full(path)
    return leaves, meta, extra


# Class names of the state modules in the reference's saved tree structures
# (state/model_state.py:28-63 and the module classes), by leaf-path prefix.
_MODULE_CLASS = {"soil": "SoilState", "snow": "SnowState", "canopy": "CanopyState", "atm": "AtmState",
                 "vegetation": "VegetationState", "carbon": "CarbonState", "hydrology": "HydrologyDiag",
                 "summary": "SummaryState", "wetland": "MethaneState", "stress": "StressAccum",
                 "etparts": "ETParts", "seasonal": "SeasonalState", "neeparts": "NEEParts"}


def treedef_for(names, n_extra: int = 0) -> str:
    """A tree structure in the form of the reference's ``repr(treedef)`` for a
    state with the leaves ``names`` (checkpoint order) and ``n_extra``
    unnamed trailing leaves: one node per module, named by its class, with one
    ``*`` per leaf.  It carries what loaders read from it -- the soil module's
    leaf count (bedrock) and whether ``MethaneState`` is present."""
    nodes, counts = [], {}
    for p in names:
        mod = p.split(".")[0]
        if mod not in counts:
            nodes.append(mod)
            counts[mod] = 0
        counts[mod] += 1
    parts = [f"CustomNode({_MODULE_CLASS.get(m, m)}[(Missing,)], [{', '.join(['*'] * counts[m])}])" for m in nodes]
    if n_extra:
        parts.append(f"[{', '.join(['*'] * n_extra)}]")
    return f"PyTreeDef(CustomNode(IBISState[(Missing,)], [{', '.join(parts)}]))"


def _treedef_agrees(tree: str, names) -> bool:
    """Whether a saved tree structure still describes a state with the leaves
    ``names``: the same soil leaf count and the same optional modules."""
    k = _soil_leaf_count(tree)
    if k is None or k != sum(1 for p in names if p.startswith("soil.")):
        return False
    mods = {p.split(".")[0] for p in names}
    return all((_MODULE_CLASS[m] in tree) == (m in mods) for m in ("wetland", "stress", "etparts", "seasonal",
                                                                   "neeparts"))


def save(path: str, leaves: dict, meta: dict | None = None, extra=None, treedef_repr: str | None = None):
    """Write ``leaves`` (base state by path, bedrock leaf optional, then the
    named optional modules present, in the state's order) and ``extra`` in the
    reference's checkpoint format.  The file always carries a tree structure:
    ``treedef_repr`` (the structure of the file the leaves came from) while it
    still describes the leaves written, else one made by :func:`treedef_for`,
    so a loader never has to tell the optional modules apart by leaf count."""
    bedrock = leaves.get(BEDROCK_LEAF) is not None
    names = base_leaves(bedrock)
    missing = [p for p in names if p not in leaves]
    if missing:
        raise ValueError(f"leaves missing from the state: {missing[:5]}")
    names = names + [p for p in TRAILING if p in leaves]
    arrays = [leaves[p] for p in names] + list(extra or [])
    out = {"num_leaves": np.asarray(len(arrays))}
    if treedef_repr is None or not _treedef_agrees(treedef_repr, names):
        treedef_repr = treedef_for(names, len(extra or []))
    out["treedef_repr"] = np.asarray(treedef_repr)
    for i, a in enumerate(arrays):
        if a is None:
            out[f"leaf_{i}_is_none"] = np.asarray(True)
        else:
            out[f"leaf_{i}"] = np.asarray(a)
    for k, v in (meta or {}).items():
        out[f"meta_{k}"] = np.asarray(v)
    np.savez_compressed(path, **out)


def as_tree(leaves: dict):
    """The flat leaves as nested attribute objects (``tree.soil.tsoi`` ...), the
    shape :mod:`ibis_b200.dropin` reads."""
    root = types.SimpleNamespace()
    for path, v in leaves.items():
        obj = root
        *head, last = path.split(".")
        for h in head:
            if not hasattr(obj, h):
                setattr(obj, h, types.SimpleNamespace())
            obj = getattr(obj, h)
        setattr(obj, last, v)
    if not hasattr(root.soil, "tsoi_deep"):
        root.soil.tsoi_deep = None
    return root


def params_from_leaves(leaves: dict, params=None):
    """The parameter record a checkpoint implies: ``params`` (defaults otherwise)
    with the soil layer thicknesses, root profile and CO2 of the state, and the
    bedrock flag set when the state carries bedrock."""
    from .params import FLAG_BEDROCK, StepParams
    P = (params or StepParams()).copy()
    for name, leaf in (("hsoi", "soil.hsoi"), ("froot", "vegetation.froot"), ("co2conc", "atm.co2conc")):
        v = leaves.get(leaf)
        if v is not None:
            v = np.asarray(v, dtype=np.float64).reshape(-1)
            setattr(P, name, v[:L.NSOILAY] if name == "hsoi" else (v if name == "froot" else float(v[0])))
    # the snow constants stay the record's: the reference's load_state takes them
    # from its template, not from the file (older files carry outdated values,
    # io/restart.py:174-183)
    P.flags = (P.flags | FLAG_BEDROCK) if leaves.get(BEDROCK_LEAF) is not None else (P.flags & ~FLAG_BEDROCK)
    return P


def group_from_leaves(leaves: dict, group: str, ncell: int) -> dict:
    """The fields of a plane group (``layout.GROUPS``) the checkpoint holds, as
    per-cell float64 arrays (scalars broadcast)."""
    out = {}
    for f in L.GROUPS[group]:
        v = leaves.get(f.leaf)
        if v is None:
            continue
        a = np.asarray(v, dtype=np.float64)
        out[f.name] = np.full(ncell, float(a)) if a.ndim == 0 else a
    return out


def columns_from_restart(path: str, dtype=None, device="cuda", params=None, diag=False, acc=True):
    """Device columns holding a checkpoint's state, and the parameter record.

    ``params`` supplies everything a checkpoint does not hold (a
    :class:`~ibis_b200.params.StepParams`; defaults otherwise); the soil layer
    thicknesses, root profile and CO2 come from the state.
    Returns ``(columns, params, leaves, meta, extra)``."""
    import torch

    from . import dropin
    from .columns import Columns

    leaves, meta, extra, treedef = load_full(path)
    tree = as_tree(leaves)
    ncell = int(np.asarray(tree.soil.tg).shape[0])
    prog = dropin._leaf_dict(tree, "PROG", ncell)
    stat = dropin._leaf_dict(tree, "STAT", ncell)
    P = params_from_leaves(leaves, params)
    if dtype is None:
        dtype = torch.float32 if np.asarray(tree.soil.tg).dtype == np.float32 else torch.float64
    cols = Columns.from_host(prog, stat, dtype=dtype, device=device, diag=diag, acc=acc)
    meta = dict(meta)
    if treedef is not None:
        meta[TREEDEF_KEY] = treedef
    return cols, P, leaves, meta, extra


# A checkpoint's saved tree structure rides with its metadata dict between
# columns_from_restart and write_state under this key; it is never written as
# a meta_ entry.
TREEDEF_KEY = "__treedef_repr__"


def write_state(path: str, leaves: dict, groups, meta=None, extra=None):
    """Save ``leaves`` with the values of ``groups`` -- a sequence of
    (layout group, {field: per-cell array}) pairs, later pairs taking precedence
    where two fields share a leaf -- written into the leaves they mirror, in the
    leaves' own dtypes.  Leaves no group names are carried over unchanged; the
    tree structure of the file they came from (in ``meta`` from
    :func:`columns_from_restart`) is written back while it still fits."""
    out = dict(leaves)
    for group, values in groups:
        for f in L.GROUPS[group]:
            old = out.get(f.leaf)
            if old is None or f.name not in values:
                continue
            v = np.asarray(values[f.name]).astype(np.asarray(old).dtype)
            out[f.leaf] = v.reshape(-1)[0] if np.ndim(old) == 0 else v.reshape(np.shape(old))
    meta = dict(meta or {})
    treedef = meta.pop(TREEDEF_KEY, None)
    save(path, out, meta, extra, treedef)


def write_columns(path: str, cols, leaves: dict, meta=None, extra=None):
    """Save ``cols``' prognostic state (and diagnostics, if the columns keep them)
    into the checkpoint ``leaves`` came from, in the leaves' own dtypes."""
    groups = [("PROG", cols.prog_host())]
    if cols.diag is not None:
        groups.append(("DIAG", cols.diag_host()))
    write_state(path, leaves, groups, meta, extra)
