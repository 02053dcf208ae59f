"""The drop-in ``timestep_body(state, consts, params, dtime)`` over pytree-like
objects: parameter mapping against the reference's own objects (CPU, where the
reference sources exist), leaf replacement (CPU), and the step through the
drop-in against the reference's golden outputs (GPU, float64, 1e-9)."""
import dataclasses
import os
import subprocess
import sys
import types
from typing import NamedTuple

import numpy as np
import pytest

from ibis_b200 import dropin
from ibis_b200 import layout as L
from ibis_b200.params import PARAM_FIELDS, FLAG_BEDROCK, FLAG_H2O_CONSISTENT, FLAG_SUNSHADE_L, FLAG_SUNSHADE_U

HERE = os.path.dirname(os.path.abspath(__file__))
from goldens import REF_PORT as REF  # noqa: E402


@dataclasses.dataclass(frozen=True)
class _DC:
    a: float
    b: object


class _NT(NamedTuple):
    x: float
    y: float


def test_tree_set_on_dataclass_namedtuple_namespace():
    root = _DC(a=1.0, b=types.SimpleNamespace(c=_NT(2.0, 3.0), d=4.0))
    new = dropin.tree_set(root, "b.c.y", 9.0)
    assert new.b.c.y == 9.0 and new.b.c.x == 2.0 and new.a == 1.0
    assert root.b.c.y == 3.0                       # the original is untouched
    new2 = dropin.tree_set(new, "a", 5.0)
    assert new2.a == 5.0 and new2.b is new.b


@pytest.mark.parametrize("switch", dropin.UNSUPPORTED_SWITCHES)
def test_unimplemented_stomata_switch_is_refused(switch):
    """A stomata formulation the step does not carry raises instead of running
    the default formulation in its place; the implemented switches pass."""
    state = types.SimpleNamespace(soil=types.SimpleNamespace(tsoi_deep=None))
    sp = types.SimpleNamespace(sunshade_u=True, sunshade_l=False, **{switch: True})
    with pytest.raises(NotImplementedError, match=switch):
        dropin.step_params(state, types.SimpleNamespace(), types.SimpleNamespace(stomata_params=sp), 3600.0)
    setattr(sp, switch, False)
    P = dropin.step_params(state, types.SimpleNamespace(), types.SimpleNamespace(stomata_params=sp), 3600.0)
    assert P.flags & FLAG_SUNSHADE_U and not P.flags & FLAG_BEDROCK


_MAP_CHECK = r"""
import sys, numpy as np
sys.path.insert(0, "{golden}/jaxshim"); sys.path.insert(0, "{ref}"); sys.path.insert(0, "{golden}"); sys.path.insert(0, "{repo}")
import make_golden as mg
from ibis.constants import get_constants
from ibis_b200 import dropin, synth
from ibis_b200.params import PARAM_FIELDS
for name, spec in mg.CASES.items():
    wl = mg.build_case(name, spec)
    st, sp = mg.reference_state(wl), mg.reference_params(wl)
    got = dropin.step_params(st, get_constants(), sp, wl.params.dtime)
    for f, n, _ in PARAM_FIELDS:
        if f in ("omegasno", "flux_max", "t_max_dev", "ndaypy"):
            continue
        a, b = np.asarray(getattr(got, f), float), np.asarray(getattr(wl.params, f), float)
        assert np.allclose(a, b, rtol=1e-12, atol=0), (name, f, a, b)
    assert got.flags == wl.params.flags & 0xF, (name, got.flags, wl.params.flags)
print("mapping ok")
"""


@pytest.mark.skipif(not REF or not os.path.isdir(REF), reason="reference sources not present (IBIS_REFERENCE)")
def test_param_mapping_against_reference_objects():
    code = _MAP_CHECK.format(golden=os.path.join(HERE, "golden"), ref=REF, repo=os.path.dirname(HERE))
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0 and "mapping ok" in r.stdout, r.stderr[-3000:]


# ---------------------------------------------------------------- GPU

def _ns(d):
    """Nested SimpleNamespace from {"a.b.c": value}."""
    root = types.SimpleNamespace()
    for path, v in d.items():
        obj = root
        *head, last = path.split(".")
        for h in head:
            if not hasattr(obj, h):
                setattr(obj, h, types.SimpleNamespace())
            obj = getattr(obj, h)
        setattr(obj, last, v)
    return root


def _mock(case, h=0):
    """State, constants and parameters as attribute trees with the reference's paths."""
    P = case.params
    bed = bool(P.flags & FLAG_BEDROCK)
    leaves = {}
    for f in L.PROG + L.STAT:
        if f.leaf.startswith(L.OPTIONAL_LEAF_PREFIXES) or (f.name == "tsoi_deep" and not bed):
            continue
        src = case.prog if f in L.PROG else case.stat
        if f.name not in src:          # inputs of switched-off extensions the fixture does not carry
            continue
        leaves["state." + f.leaf] = np.asarray(src[f.name], dtype=np.float64).copy()
    leaves["state.vegetation.nytimes"] = np.float64(case.prog["nytimes"][0])
    for f in L.FORC:
        leaves["state." + f.leaf] = np.asarray(case.forc[f.name][h], dtype=np.float64)
    for f in L.DIAG:
        k = f.k
        leaves.setdefault("state." + f.leaf, np.zeros((case.ncell, k)) if k > 1 else np.zeros(case.ncell))
    if not bed:
        leaves["state.soil.tsoi_deep"] = None
    for name, path in dropin.PARAM_PATHS.items():
        if path.startswith("params.bedrock.") and not bed:
            continue
        v = np.asarray(getattr(P, name), dtype=np.float64)
        if name == "hsoi":
            v = np.concatenate([v, [0.0]])
        if name == "froot":
            v = v.reshape(6, 2)
        leaves[path] = v if v.size > 1 else float(v)
    if not bed:
        leaves["params.bedrock"] = None
    leaves["params.h2o_consistent_weights"] = bool(P.flags & FLAG_H2O_CONSISTENT)
    leaves["params.stomata_params.sunshade_u"] = bool(P.flags & FLAG_SUNSHADE_U)
    leaves["params.stomata_params.sunshade_l"] = bool(P.flags & FLAG_SUNSHADE_L)
    tree = _ns(leaves)
    return tree.state, tree.consts, tree.params


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["day_mixed", "nobedrock", "sunshade", "perturbed"])
def test_dropin_step_matches_reference_golden(cuda_lib, name):
    from goldens import Case, compare
    c = Case(name)
    state, consts, params = _mock(c)
    last = max(c.record)
    for h in range(last):
        for f in L.FORC:
            state = dropin.tree_set(state, f.leaf, np.asarray(c.forc[f.name][h], dtype=np.float64))
        state = dropin.timestep_body(state, consts, params, c.params.dtime)
        if h + 1 in c.record:
            got = {f.name: np.asarray(dropin._get({"s": state}, "s." + f.leaf)) for f in L.PROG
                   if dropin._get({"s": state}, "s." + f.leaf) is not None}
            got["nytimes"] = np.full(c.ncell, float(got["nytimes"]))
            bad = compare(got, c.out(h + 1, "prog"), 1e-9)
            dg = {f.name: np.asarray(dropin._get({"s": state}, "s." + f.leaf)) for f in L.DIAG}
            bad += compare(dg, c.out(h + 1, "diag"), 1e-9)
            assert not bad, (h + 1, bad[:5])


@pytest.mark.gpu
def test_run_hours_sums_attached_et_and_nee_parts(cuda_lib):
    """A state carrying the reference's optional ``etparts`` / ``neeparts``
    modules gets them summed over the hours and written back (float64 state:
    the reference's day with both modules within 1e-6, as the other
    accumulators); a state without them is left without them."""
    from goldens import Case, compare
    c = Case("day_mixed")
    z = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "day_parts.npz"))
    state, consts, params = _mock(c)
    zero = np.zeros(c.ncell)
    state.etparts = types.SimpleNamespace(trans=zero, interc=zero, soilev=zero, snowsub=zero)
    state.neeparts = types.SimpleNamespace(night=zero, day=zero)
    assert dropin.parts_flags(state) != 0
    out, acc = dropin.run_hours(state, consts, params, c.forc, c.params.dtime)
    got = {f.name: np.asarray(dropin._get({"s": out}, "s." + f.leaf)) for f in L.ACC
           if f.leaf.startswith(("etparts.", "neeparts."))}
    assert len(got) == 6
    assert not compare(got, {k: z["day.acc." + k] for k in got}, 1e-6)
    plain, _ = dropin.run_hours(_mock(c)[0], consts, params, c.forc, c.params.dtime)
    assert getattr(plain, "etparts", None) is None and dropin.parts_flags(plain) == 0
