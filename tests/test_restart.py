"""Reading and writing the reference's checkpoint files (ibis_b200/restart.py).

CPU: the leaf order, a save/load round trip, and -- where the reference tree is
present -- every leaf this loader reads from the reference's own checkpoint
against the reference's own ``load_state``.  GPU: a checkpoint seeds device
columns whose steps match the reference's steps of the same checkpoint
(tests/golden/restart_1996.npz, float64, 1e-9), and the columns write back a
checkpoint that reads back exactly.
"""
import os
import subprocess
import sys

import numpy as np
import pytest

from ibis_b200 import layout as L
from ibis_b200 import restart

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURE = os.path.join(HERE, "golden", "restart_16cells.npz")
from goldens import HAVE_REF, REF_PORT, REF_ROOT  # noqa: E402
REF_CKPT = os.path.join(REF_ROOT, "verify_out_stage1", "site_transient_1996.npz") if REF_ROOT else ""


def test_leaf_order_covers_the_layout():
    assert len(restart.LEAVES) == 258 and len(set(restart.LEAVES)) == 258
    assert restart.LEAVES[:4] == ("soil.tsoi", "soil.wsoi", "soil.wisoi", "soil.tg")
    for f in L.PROG + L.STAT:
        if not f.leaf.startswith(L.OPTIONAL_LEAF_PREFIXES):
            assert f.leaf in restart.LEAVES, f.leaf
    assert len(restart.base_leaves(False)) == 257


def test_fixture_loads():
    leaves, meta, extra = restart.load(FIXTURE)
    assert meta == {"year": 1996} and extra == []
    assert leaves["soil.tsoi"].shape == (16, 6) and leaves["soil.tsoi_deep"].shape == (16, 3)
    assert leaves["soil.hsoi"].shape == (7,)
    assert np.all(leaves["soil.tsoi"] > 200.0) and np.all(leaves["soil.poros"] > 0.0)


def test_save_load_round_trip(tmp_path):
    leaves, meta, extra = restart.load(FIXTURE)
    leaves["soil.tg"] = leaves["soil.tg"] + 1.0
    p = tmp_path / "ck.npz"
    restart.save(str(p), leaves, meta, extra=[np.arange(3.0)])      # one trailing leaf: no module count
    back, meta2, extra2 = restart.load(str(p))
    assert meta2 == meta and len(extra2) == 1 and np.array_equal(extra2[0], np.arange(3.0))
    for k in restart.LEAVES:
        assert np.array_equal(np.asarray(back[k]), np.asarray(leaves[k])), k
    nobed = {k: v for k, v in leaves.items() if k != restart.BEDROCK_LEAF}
    restart.save(str(p), nobed, meta)
    back, _, _ = restart.load(str(p))
    assert restart.BEDROCK_LEAF not in back and len(back) == 257


MODULES = os.path.join(HERE, "golden", "restart_modules_16cells.npz")
MODULE_VALUES = os.path.join(HERE, "golden", "restart_modules_values.npz")


def test_trailing_names_follow_the_module_chain():
    """The optional modules after the base leaves are named by their count as
    the reference's loader identifies them: the calibration chain (stress, ET
    parts, seasonal, NEE parts; the old 3-leaf stress form), with the wetland
    state before it where the saved tree structure names it or the count
    leaves no other reading."""
    chain = [p for mod in restart.CHAIN for p in mod]
    old = chain[:3] + chain[4:]
    for n in (0, 4, 8, 11, 13):
        assert restart.trailing_names(n) == chain[:n]
    for n in (3, 7, 10, 12):
        assert restart.trailing_names(n) == old[:n]
    wet = list(restart.WETLAND_LEAVES)
    assert restart.trailing_names(16) == wet + chain and restart.trailing_names(11 + 3) == wet + chain[:11]
    assert restart.trailing_names(7, "CustomNode(MethaneState[()], [*, *, *])") == wet + chain[:4]
    assert restart.trailing_names(7) == old[:7]            # without the structure: the old chain, as the reference
    assert restart.trailing_names(6) == wet + old[:3]
    for n in (1, 2, 5, 9, 20):
        assert restart.trailing_names(n) is None, n


def test_modules_checkpoint_round_trip(tmp_path):
    """The reference's own checkpoint with the wetland state and the four
    calibration modules attached: every module leaf read by name with the
    values the reference saved, and written back in the same order."""
    leaves, meta, extra = restart.load(MODULES)
    want = np.load(MODULE_VALUES)
    assert extra == [] and len(leaves) == 258 + 16
    for k in want.files:
        assert np.array_equal(np.asarray(leaves[k[len("value."):]]), want[k]), k
    leaves["seasonal.ssen_u"] = leaves["seasonal.ssen_u"] + 1.0
    p = tmp_path / "ck.npz"
    restart.save(str(p), leaves, meta)
    z = np.load(str(p))
    ref = np.load(MODULES)
    assert int(z["num_leaves"]) == int(ref["num_leaves"])
    i = restart.LEAVES.index("soil.tg")
    assert np.array_equal(z[f"leaf_{i}"], ref[f"leaf_{i}"])
    back, _, _ = restart.load(str(p))
    assert np.array_equal(back["seasonal.ssen_u"], want["value.seasonal.ssen_u"] + 1.0)


_MODULES_REF_CHECK = r"""
import sys, numpy as np
sys.path.insert(0, "{golden}/jaxshim"); sys.path.insert(0, "{ref}"); sys.path.insert(0, "{repo}")
from ibis.dimensions import GridConfig
from ibis.state.model_state import create_ibis_state
from ibis.io.restart import load_state
from ibis_b200 import restart
leaves, meta, extra = restart.load("{src}")
for k in [k for k in leaves if k.split(".")[0] in ("wetland", "stress", "etparts", "seasonal", "neeparts")]:
    leaves[k] = (np.asarray(leaves[k]) * 2.0 + 1.0).astype(np.float32)
restart.save("{dst}", leaves, meta)
st, m = load_state("{dst}", create_ibis_state(GridConfig(nlon=1, nlat=1, npoi=16, nbedrock=3), with_neeparts=True))
n = 0
for k, v in leaves.items():
    mod, leaf = k.split(".")
    if mod in ("wetland", "stress", "etparts", "seasonal", "neeparts"):
        assert np.array_equal(np.asarray(getattr(getattr(st, mod), leaf)), v), k
        n += 1
print("modules ok", n)
"""


@pytest.mark.skipif(not HAVE_REF, reason="reference sources not present (IBIS_REFERENCE)")
def test_saved_modules_load_in_the_reference(tmp_path):
    """A checkpoint with the modules written here loads in the reference's own
    ``load_state`` (wetland state attached by it from the count) with every
    module leaf as written."""
    code = _MODULES_REF_CHECK.format(golden=os.path.join(HERE, "golden"), ref=REF_PORT,
                                     repo=os.path.dirname(HERE), src=MODULES, dst=str(tmp_path / "ck.npz"))
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0 and "modules ok 16" in r.stdout, r.stderr[-3000:]


_REF_CHECK = r"""
import sys, numpy as np
sys.path.insert(0, "{golden}/jaxshim"); sys.path.insert(0, "{ref}"); sys.path.insert(0, "{repo}")
from ibis.dimensions import GridConfig
from ibis.state.model_state import create_ibis_state
from ibis.io.restart import load_state
from ibis_b200 import restart
leaves, meta, extra = restart.load("{ckpt}")
n = leaves["soil.tg"].shape[0]
st, m = load_state("{ckpt}", create_ibis_state(GridConfig(nlon=1, nlat=1, npoi=n, nbedrock=3)))
static = ("z0sno", "rhos", "consno", "hsnotop", "hsnomin", "fimin", "fimax")
for path, v in leaves.items():
    mod, leaf = path.split(".")
    if mod == "snow" and leaf in static:
        continue                                   # the reference takes these from its template
    r = np.asarray(getattr(getattr(st, mod), leaf))
    assert np.array_equal(r.astype(np.float64), np.asarray(v).astype(np.float64)), path
print("leaves ok", len(leaves))
"""


@pytest.mark.skipif(not REF_CKPT or not os.path.exists(REF_CKPT), reason="reference checkpoint not present (IBIS_REFERENCE)")
def test_loader_agrees_with_the_reference_loader():
    code = _REF_CHECK.format(golden=os.path.join(HERE, "golden"), ref=REF_PORT,
                             repo=os.path.dirname(HERE), ckpt=REF_CKPT)
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0 and "leaves ok 258" in r.stdout, r.stderr[-3000:]


@pytest.mark.gpu
def test_checkpoint_columns_step_like_the_reference(cuda_lib, tmp_path):
    import torch
    from goldens import Case, compare
    c = Case("restart_1996")
    cols, P, leaves, meta, extra = restart.columns_from_restart(FIXTURE, dtype=torch.float64, diag=True, acc=False)
    n = cols.ncell
    forc = {k: v[:, :n] for k, v in c.forc.items()}
    cols.run(cols.forcing(forc, 0, 6), c.params)
    torch.cuda.synchronize()
    want = {k: v[:n] for k, v in c.out(6, "prog").items()}
    got = cols.prog_host()
    bad = compare(got, want, 1e-9)
    assert not bad, bad[:5]
    p = tmp_path / "after.npz"
    restart.write_columns(str(p), cols, leaves, meta, extra)
    back, meta2, _ = restart.load(str(p))
    prog = cols.prog_host()
    for f in L.PROG:
        v = np.asarray(back[f.leaf], dtype=np.float64)
        ref = prog[f.name][0] if v.ndim == 0 else prog[f.name]
        assert np.array_equal(v, np.asarray(ref).astype(np.float32).astype(np.float64).reshape(v.shape)), f.name
    # the metadata round-trips; the file's own tree structure rides beside it and is written back
    assert meta2 == {k: v for k, v in meta.items() if k != restart.TREEDEF_KEY}
    assert str(np.load(str(p))["treedef_repr"]) == meta[restart.TREEDEF_KEY]


def _with_modules(leaves, mods, n):
    out = dict(leaves)
    rng = np.random.default_rng(3)
    for m in mods:
        for p in (restart.WETLAND_LEAVES if m == "wetland" else next(c for c in restart.CHAIN if c[0].startswith(m))):
            out[p] = rng.random(n)
    return out


def test_written_modules_read_back_by_name(tmp_path):
    """Every file this module writes carries a tree structure, so the optional
    modules come back by name where their leaf counts alone are ambiguous: the
    wetland state plus a 4-leaf StressAccum (7 trailing leaves, also the old
    3-leaf StressAccum plus ETParts) and wetland + StressAccum + ETParts (11, also
    StressAccum + ETParts + SeasonalState); with and without bedrock."""
    leaves, meta, _ = restart.load(FIXTURE)
    n = leaves["soil.tg"].shape[0]
    for bed in (True, False):
        base = leaves if bed else {k: v for k, v in leaves.items() if k != restart.BEDROCK_LEAF}
        for mods in (("wetland", "stress"), ("wetland", "stress", "etparts"), ("stress",),
                     ("stress", "etparts", "seasonal")):
            state = _with_modules(base, mods, n)
            p = str(tmp_path / "m.npz")
            restart.write_state(p, state, [], meta)
            back, _, extra = restart.load(p)
            assert extra == [] and set(back) == set(state), (bed, mods)
            for k, v in state.items():
                assert np.array_equal(np.asarray(back[k]), np.asarray(v)), (bed, mods, k)


def test_bedrock_without_tree_structure_from_shapes(tmp_path):
    """A file without a saved tree structure: bedrock is read from the array at
    the bedrock leaf's position (soil.tsoi_deep is (npoi, 3), snow.fi (npoi,)),
    so a no-bedrock state carrying a module is not taken for a bedrock state."""
    leaves, meta, _ = restart.load(FIXTURE)
    n = leaves["soil.tg"].shape[0]
    nobed = _with_modules({k: v for k, v in leaves.items() if k != restart.BEDROCK_LEAF}, ("stress",), n)
    p = str(tmp_path / "nt.npz")
    restart.save(p, nobed, meta)
    z = dict(np.load(p))
    z.pop("treedef_repr")
    np.savez(p, **z)
    back, _, extra = restart.load(p)
    assert restart.BEDROCK_LEAF not in back and extra == []
    assert all(np.array_equal(np.asarray(back[k]), np.asarray(v)) for k, v in nobed.items())


def test_loaded_tree_structure_is_written_back(tmp_path):
    """A checkpoint's own tree structure is written back when the module set is
    unchanged, and replaced by one naming the modules when it is not."""
    leaves, meta, extra = restart.load(MODULES)
    p = str(tmp_path / "w.npz")
    restart.save(p, leaves, meta, extra)
    leaves, meta, extra, tree = restart.load_full(p)
    assert tree is not None and "MethaneState" in tree
    restart.save(p, leaves, meta, extra, tree)
    assert str(np.load(p)["treedef_repr"]) == tree
    fewer = {k: v for k, v in leaves.items() if not k.startswith("wetland.")}
    restart.save(p, fewer, meta, extra, tree)
    t2 = str(np.load(p)["treedef_repr"])
    assert "MethaneState" not in t2 and "SoilState" in t2
    back, _, _ = restart.load(p)
    assert set(back) == set(fewer)
