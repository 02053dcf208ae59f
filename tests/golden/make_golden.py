"""Generate golden fixtures by running the REFERENCE's own hourly step.

The reference (UW-GCRL/ibis, ``python-port/``) is JAX + Equinox code and
neither is installed here, so this script puts a small NumPy-backed stand-in
for ``jax``/``jax.numpy``/``equinox`` (``tests/golden/jaxshim``) first on
``sys.path`` and imports the reference package unmodified from
``$IBIS_REFERENCE/python-port`` (default ``/root/reference``).  It then runs, in float64:

* ``ibis.timestepping.loops.timestep_body`` hour by hour, recording the state
  it returns (prognostic and diagnostic leaves), and
* ``ibis.timestepping.loops_gswp3._run_day_inner`` for one day with the
  wetland-CH4 and soil-mean accumulators on, with its weather generator
  ``diurnal`` replaced by the synthetic forcing and its per-step float32 cast
  replaced by the identity (the float64 reference run),

on seeded synthetic columns from ``ibis_b200.synth``, and writes the inputs
and outputs to ``tests/golden/<case>.npz``.  The fixtures travel with the
repository; this script only runs where the reference tree exists.

It also writes ``ibis_b200/restart_leaves.py`` (the leaf order of the
reference's checkpoint files, from its state classes) and the
``restart_1996`` case: the reference's own checkpoint of a 171-cell transient
run, stepped by its own ``timestep_body``.

Usage:  python tests/golden/make_golden.py [--only CASE|restart_leaves]
"""
from __future__ import annotations

import argparse
import dataclasses
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
# the reference project's root (holding python-port/); this script reads it there
REF_ROOT = os.environ.get("IBIS_REFERENCE", "/root/reference")
REF = os.path.join(REF_ROOT, "python-port")

os.environ.pop("IBIS_FLUX_MAX", None)
os.environ.pop("IBIS_T_MAX_DEV", None)
sys.path.insert(0, os.path.join(HERE, "jaxshim"))
sys.path.insert(0, REF)
sys.path.insert(0, REPO)

import jax.numpy as jnp  # noqa: E402  (the NumPy stand-in)
import equinox as eqx  # noqa: E402
from ibis.constants import get_constants  # noqa: E402
from ibis.dimensions import GridConfig  # noqa: E402
from ibis.state.model_state import create_ibis_state  # noqa: E402
from ibis.timestepping import loops, loops_gswp3  # noqa: E402
from ibis.physics.bedrock import BedrockParams  # noqa: E402
from ibis.bgc.methane import MethaneParams  # noqa: E402

from ibis_b200 import layout as L  # noqa: E402
from ibis_b200 import synth  # noqa: E402
from ibis_b200.params import (StepParams, FLAG_BEDROCK, FLAG_H2O_CONSISTENT, FLAG_SUNSHADE_U,  # noqa: E402
                              FLAG_SUNSHADE_L, FLAG_ACC, FLAG_CH4, FLAG_SOIL_MEANS)


def _a(x):
    return jnp.asarray(np.asarray(x, dtype=np.float64))


def reference_state(wl, parts=False, seasonal=False):
    """IBISState (float64) holding the workload's prognostic and static fields
    (with ``parts`` also the optional ET/NEE component modules, with ``seasonal``
    the seasonal module -- and the stress and ET-part modules it brings -- holding
    the workload's acclimation state, and the day's mean air temperature)."""
    n = wl.ncell
    bed = bool(wl.params.flags & FLAG_BEDROCK)
    st = create_ibis_state(GridConfig(nlon=2, nlat=1, npoi=n, nbedrock=3 if bed else 0), with_neeparts=parts,
                           with_seasonal=seasonal)
    if seasonal:
        st = dataclasses.replace(st, seasonal=dataclasses.replace(st.seasonal, acclim_x=_a(wl.stat["acclim_x"])))
    if "td" in wl.stat:
        st = dataclasses.replace(st, atm=dataclasses.replace(st.atm, td=_a(wl.stat["td"])))
    P, S = wl.prog, wl.stat
    hsoi = np.zeros(L.NSOILAY + 1)
    hsoi[:L.NSOILAY] = wl.params.hsoi
    soil_fields = {f.leaf.split(".")[1]: f.name for f in L.PROG + L.STAT if f.leaf.startswith("soil.")}
    if not bed:
        soil_fields.pop("tsoi_deep")
    src = {**S, **P}
    soil = st.soil
    for leaf, name in soil_fields.items():
        soil = dataclasses.replace(soil, **{leaf: _a(src[name])})
    soil = dataclasses.replace(soil, hsoi=_a(hsoi))
    snow = st.snow
    for f in L.PROG:
        if f.leaf.startswith("snow."):
            snow = dataclasses.replace(snow, **{f.leaf.split(".")[1]: _a(P[f.name])})
    can = st.canopy
    for f in L.PROG:
        if f.leaf.startswith("canopy."):
            can = dataclasses.replace(can, **{f.leaf.split(".")[1]: _a(P[f.name])})
    veg = st.vegetation
    for f in L.PROG + L.STAT:
        if f.leaf.startswith("vegetation.") and f.name != "nytimes":
            veg = dataclasses.replace(veg, **{f.leaf.split(".")[1]: _a(src[f.name])})
    veg = dataclasses.replace(veg, nytimes=_a(P["nytimes"][0]), froot=_a(wl.params.froot2))
    atm = dataclasses.replace(st.atm, co2conc=float(wl.params.co2conc))
    return dataclasses.replace(st, soil=soil, snow=snow, canopy=can, vegetation=veg, atm=atm)


def reference_params(wl):
    p = wl.params
    sp = loops.default_sim_params(wl.ncell)
    stom = dataclasses.replace(
        sp.stomata_params, coefm=_a(p.coefm), coefb=_a(p.coefb), gamma=_a(p.gamma), gsmin=_a(p.gsmin),
        vmax_pft=_a(p.vmax_pft), stressfac=float(p.stressfac),
        sunshade_u=bool(p.flags & FLAG_SUNSHADE_U), sunshade_l=bool(p.flags & FLAG_SUNSHADE_L))
    canp = sp.canopy._replace(soil_beta_power=float(p.soil_beta_power))
    ip = sp.interception._replace(wliqumax=float(p.wliqumax), wliqsmax=float(p.wliqsmax),
                                  wliqlmax=float(p.wliqlmax), fmax=float(p.fmax))
    meth = MethaneParams(r_ch4=float(p.r_ch4), q10p=float(p.q10p), z_tau=float(p.z_tau),
                         tau_oxid=float(p.tau_oxid), z_wt_max=float(p.z_wt_max))
    bgc = dataclasses.replace(sp.bgc_params, rwood=_a(p.rwood), rroot=_a(p.rroot), rgrowth=_a(p.rgrowth))
    return dataclasses.replace(
        sp, stomata_params=stom, canopy=canp, interception=ip, methane=meth, bgc_params=bgc,
        latitude=_a(np.deg2rad(wl.latitude)),
        bedrock=BedrockParams() if p.flags & FLAG_BEDROCK else None,
        h2o_consistent_weights=bool(p.flags & FLAG_H2O_CONSISTENT))


def set_forcing(st, F):
    atm = st.atm
    for f in L.FORC:
        atm = dataclasses.replace(atm, **{f.leaf.split(".")[1]: _a(F[f.name])})
    return dataclasses.replace(st, atm=atm)


def get(obj, path):
    for part in path.split("."):
        obj = getattr(obj, part)
    return np.asarray(obj, dtype=np.float64)


def snapshot(st):
    out = {}
    for f in L.PROG:
        if f.name == "tsoi_deep" and st.soil.tsoi_deep is None:
            continue
        v = get(st, f.leaf)
        out["prog." + f.name] = np.broadcast_to(v, (st.soil.tg.shape[0],) + v.shape[1:]) if f.name == "nytimes" else v
    for f in L.DIAG:
        mod, leaf = f.leaf.split(".")
        if hasattr(getattr(st, mod), leaf):      # diagnostics this build adds have no reference leaf
            out["diag." + f.name] = get(st, f.leaf)
    return out


def run_steps(wl, record, ref=None):
    """timestep_body hour by hour; ``ref`` = (params, state) built by the caller."""
    consts = get_constants()
    params, st = ref if ref is not None else (reference_params(wl), reference_state(wl))
    snaps = {}
    for h in range(wl.nhour):
        st = set_forcing(st, wl.forcing_at(h))
        st = loops.timestep_body(st, consts, params, float(wl.params.dtime))
        if (h + 1) in record:
            snaps[h + 1] = snapshot(st)
    return snaps


def run_day_accumulators(wl, parts=False, ref=None):
    """_run_day_inner over 24 hourly steps with CH4 and soil means on (and with
    ``parts`` the ET/NEE component modules attached; ``ref`` = (params, state)
    built by the caller, whose ET/NEE modules are recorded when present)."""
    assert wl.nhour == 24
    consts = get_constants()
    if ref is not None:
        params, st = ref
        parts = st.etparts is not None
    else:
        params = reference_params(wl)
        st = reference_state(wl, parts)
    F = wl.forc

    def fake_diurnal(time, jday, dw, lat, plens, startp, endp, key, dtime, nband=2):
        h = int(round(float(time) / float(dtime)))
        hw = types.SimpleNamespace(coszen=_a(F["coszen"][h]), ta=_a(F["ta"][h]), qa=_a(F["qa"][h]),
                                   ua=_a(F["ua"][h]), solad=_a(F["solad"][h]), solai=_a(F["solai"][h]),
                                   raina=_a(F["raina"][h]), snowa=_a(F["snowa"][h]), fira=_a(F["fira"][h]))
        return key, hw

    saved = (loops_gswp3.diurnal, loops_gswp3._cast_tree_f32)
    loops_gswp3.diurnal = fake_diurnal
    loops_gswp3._cast_tree_f32 = lambda tree: tree
    try:
        dw = types.SimpleNamespace(psurf=_a(F["psurf"][0]))
        n = wl.ncell
        z = _a(np.zeros(n))
        key = jnp.asarray(np.array([0, 1], dtype=np.uint32))
        st_out, _, acc = loops_gswp3._run_day_inner(
            st, consts, params, dw, _a(F["fira"][0]), z, z, z, jnp.asarray(np.int32(wl.start_doy)), key,
            float(wl.params.dtime), ch4=(_a(wl.stat["f_inund"]), params.methane, None), soil_means=True)
    finally:
        loops_gswp3.diurnal, loops_gswp3._cast_tree_f32 = saved
    out = snapshot(st_out)
    for f in L.ACC:
        if f.leaf.startswith("summary."):
            out["acc." + f.name] = get(st_out, f.leaf)
    out["acc.ch4"] = np.asarray(acc[0], dtype=np.float64)
    out["acc.tsoi_mean"] = np.asarray(acc[1], dtype=np.float64)
    out["acc.wsoi_mean"] = np.asarray(acc[2], dtype=np.float64)
    out["acc.wisoi_mean"] = np.asarray(acc[3], dtype=np.float64)
    out["acc.tg_mean"] = np.asarray(acc[4], dtype=np.float64)
    if parts:
        for f in L.ACC:
            if f.leaf.startswith(("etparts.", "neeparts.")) and getattr(st_out, f.leaf.split(".")[0]) is not None:
                out["acc." + f.name] = get(st_out, f.leaf)
    return out


def write_parts_case():
    """tests/golden/day_parts.npz: the day_mixed day of _run_day_inner again,
    with the optional ET and NEE component modules attached
    (state/et_parts.py, state/nee_parts.py; summed in loops_gswp3.py:263-281)."""
    wl = build_case("day_mixed", CASES["day_mixed"])
    out = {f"day.{k}": v for k, v in run_day_accumulators(wl, parts=True).items()}
    path = os.path.join(HERE, "day_parts.npz")
    np.savez_compressed(path, **out)
    print(f"wrote {path}: {len(out)} arrays, {os.path.getsize(path)} bytes")


def pack_inputs(wl):
    d = {}
    for k, v in wl.prog.items():
        d["in.prog." + k] = v
    for k, v in wl.stat.items():
        d["in.stat." + k] = v
    for k, v in wl.forc.items():
        d["in.forc." + k] = v
    from ibis_b200.params import PARAM_FIELDS
    for name, _, _ in PARAM_FIELDS:
        d["in.param." + name] = np.asarray(getattr(wl.params, name), dtype=np.float64)
    d["in.param.flags"] = np.asarray(wl.params.flags, dtype=np.int64)
    d["in.latitude"] = wl.latitude
    d["in.start_doy"] = np.asarray(wl.start_doy)
    return d


CASES = {
    # 16 cells incl. bare/snowpack/frozen/flooded/polar-night/desert columns, bedrock, one day with accumulators
    "day_mixed": dict(ncell=16, nhour=24, seed=11, edge_cases=True, record=(1, 2, 6, 24), day=True),
    # soil column without bedrock, consistent soil-water weights
    "nobedrock": dict(ncell=8, nhour=6, seed=12, edge_cases=True, record=(1, 6), bedrock=False,
                      flags_on=FLAG_H2O_CONSISTENT),
    # sunlit/shaded two-big-leaf canopies on both stories
    "sunshade": dict(ncell=8, nhour=6, seed=13, edge_cases=True, record=(1, 6),
                     flags_on=FLAG_SUNSHADE_U | FLAG_SUNSHADE_L),
    # perturbed calibration parameters (the 31-parameter vector) and a soil-evaporation exponent
    "perturbed": dict(ncell=8, nhour=6, seed=14, edge_cases=False, record=(1, 6), perturb=True),
}


def build_case(name, spec):
    wl = synth.make_workload(spec["ncell"], spec["nhour"], seed=spec["seed"], edge_cases=spec["edge_cases"],
                             bedrock=spec.get("bedrock", True))
    wl.params.flags = wl.params.flags | spec.get("flags_on", 0)
    if spec.get("day"):
        wl.params.flags = wl.params.flags | FLAG_ACC | FLAG_CH4 | FLAG_SOIL_MEANS
        # the day loop takes one longwave value per day (GSWP3 rlds): make the forcing match
        wl.forc["fira"][:] = wl.forc["fira"][0][None, :]
    if spec.get("perturb"):
        rng = np.random.Generator(np.random.PCG64(spec["seed"] + 1000))
        f = lambda v: np.asarray(v) * np.exp(rng.uniform(np.log(0.5), np.log(1.5), size=np.shape(v)))
        p = wl.params
        p.vmax_pft, p.coefm = f(p.vmax_pft), f(p.coefm)
        p.stressfac, p.soil_beta_power = f(p.stressfac), 2.0
        p.wliqumax, p.wliqsmax, p.wliqlmax, p.fmax = f(p.wliqumax), f(p.wliqsmax), f(p.wliqlmax), f(p.fmax)
        p.r_ch4, p.q10p, p.z_tau, p.tau_oxid, p.z_wt_max = (f(p.r_ch4), f(p.q10p), f(p.z_tau), f(p.tau_oxid),
                                                            f(p.z_wt_max))
        p.rwood, p.rroot, p.rgrowth = (np.full(12, f(p.rwood[0])), np.full(12, f(p.rroot[0])),
                                        np.full(12, f(p.rgrowth[0])))
    return wl


# The IBIS 3.0 extensions of the step, run by the reference with its own switches:
# "release" takes the stomata, soil-BGC respiration and methane sections of the
# release parameter file (loaded by the reference's own loaders) on 16 columns for
# a day with the accumulators and a seasonal state; "switches" turns on the
# switches that file leaves off (canopy-level capacity scaling on both stories,
# leaf-only light scaling, acclimation of four PFTs with the light-rate factor and
# the frost ramp, the cropland share's grass capacity, organic soil solids).
X3_CASES = {
    "release": dict(ncell=16, nhour=24, seed=41, record=(1, 6, 24), day=True,
                    yaml="configs/params/params_31s_ch4h.yaml"),
    "switches": dict(ncell=12, nhour=6, seed=42, record=(1, 6),
                     stomata=dict(cap_scale_u=True, cap_scale_l=True, scale_leaf_only=True, acclim_on=True,
                                  acclim_pfts=(3, 5, 8, 10), acclim_light=True, frost_on=True, frost_t0=-8.0,
                                  frost_t1=8.0, cap_kn=0.2),
                     crop=dict(vmax_scale_c3=0.33, vmax_scale_c4=1.16, c4_share=-1.0), forganic=True),
}


def build_x3_case(name, spec):
    """Workload, reference parameters and reference state of an IBIS 3.0 case; the
    workload's flat parameters come from the drop-in's mapping of the reference
    objects (so the case also pins that mapping)."""
    from ibis.io.physics_params import (load_physics_params, build_stomata_params, build_bgc_params,
                                        build_methane_params)
    from ibis.io.parameters import CropParams
    from ibis_b200 import dropin
    from ibis_b200.params import FLAG_KAHAN, FLAG_ETPARTS
    wl = synth.make_workload(spec["ncell"], spec["nhour"], seed=spec["seed"], edge_cases=True, bedrock=True)
    n = wl.ncell
    rng = np.random.Generator(np.random.PCG64(spec["seed"] + 2000))
    wl.stat["acclim_x"] = rng.uniform(-12.0, 28.0, n)
    wl.stat["td"] = rng.uniform(262.0, 290.0, n)
    run_flags = FLAG_KAHAN
    if spec.get("day"):
        run_flags |= FLAG_ACC | FLAG_CH4 | FLAG_SOIL_MEANS
        wl.forc["fira"][:] = wl.forc["fira"][0][None, :]
    params = reference_params(wl)
    if "yaml" in spec:
        d = load_physics_params(os.path.join(REF, spec["yaml"]))
        params = dataclasses.replace(params, stomata_params=build_stomata_params(d), bgc_params=build_bgc_params(d),
                                     methane=build_methane_params(d),
                                     h2o_consistent_weights=bool(d.get("soil", {}).get("h2o_consistent_weights")))
    else:
        params = dataclasses.replace(params, stomata_params=dataclasses.replace(params.stomata_params,
                                                                              **spec["stomata"]))
    if "crop" in spec:
        wl.stat["cropfrac"] = rng.uniform(0.0, 1.0, n)
        params = dataclasses.replace(params, crop=CropParams(**spec["crop"]), cropfrac=_a(wl.stat["cropfrac"]))
    if spec.get("forganic"):
        wl.stat["forganic"] = rng.uniform(0.0, 0.6, (n, L.NSOILAY))
        params = dataclasses.replace(params, forganic=_a(wl.stat["forganic"]))
    st = reference_state(wl, seasonal=True)
    P = dropin.step_params(st, get_constants(), params, float(wl.params.dtime))
    P.flags |= run_flags | (FLAG_ETPARTS if spec.get("day") else 0)
    wl.params = P
    return wl, params, st


def write_x3_case(name):
    spec = X3_CASES[name]
    wl, params, st = build_x3_case(name, spec)
    out = pack_inputs(wl)
    for h, snap in run_steps(wl, set(spec["record"]), ref=(params, st)).items():
        for k, v in snap.items():
            out[f"out.{h}.{k}"] = v
    if spec.get("day"):
        for k, v in run_day_accumulators(wl, ref=(params, st)).items():
            out[f"day.{k}"] = v
    out["meta.record"] = np.asarray(spec["record"])
    path = os.path.join(HERE, f"{name}.npz")
    np.savez_compressed(path, **out)
    print(f"wrote {path}: {len(out)} arrays, {os.path.getsize(path)} bytes")


RESTART = os.path.join(REF_ROOT, "verify_out_stage1", "site_transient_1996.npz")
LEAVES_PY = os.path.join(REPO, "ibis_b200", "restart_leaves.py")


def leaf_paths(x, pre=""):
    """Leaf paths of a state in jax.tree.flatten order (the stand-in's flatten)."""
    from jax import _tree
    c = _tree._children(x)
    if c is None:
        return [pre]
    kind, ch, _ = c
    if kind == "none":
        return []
    if kind == "dc":
        names = [f.name for f in dataclasses.fields(x) if not f.metadata.get("static", False)]
        return [p for n, v in zip(names, ch) for p in leaf_paths(v, f"{pre}.{n}" if pre else n)]
    return [p for i, v in enumerate(ch) for p in leaf_paths(v, f"{pre}[{i}]")]


def write_restart_leaves():
    """ibis_b200/restart_leaves.py: the checkpoint leaf order of the reference's base IBISState."""
    import jax
    t = create_ibis_state(GridConfig(nlon=1, nlat=1, npoi=2, nbedrock=3))
    paths = leaf_paths(t)
    assert len(paths) == len(jax.tree.flatten(t)[0])
    lines = ['"""Leaf order of the reference\'s base ``IBISState`` with bedrock: the order',
             "``jax.tree.flatten`` gives and the restart files store (``leaf_{i}``).",
             "",
             "Generated by tests/golden/make_golden.py from the reference's own state",
             "classes (python-port/ibis/state/*.py, model_state.py:35-63); do not edit.",
             '"""', "", "LEAVES = ("]
    lines += [f'    "{p}",' for p in paths] + [")", ""]
    with open(LEAVES_PY, "w") as f:
        f.write("\n".join(lines))
    print(f"wrote {LEAVES_PY}: {len(paths)} leaves")


def build_restart_case(nhour=6, record=(1, 2, 6), seed=15):
    """A realistic state: the reference's checkpoint of a 171-cell transient run
    (1996), loaded by the reference's own load_state, stepped by its own
    timestep_body under default SimParams and synthetic forcing.  The inputs the
    fixture stores come from ibis_b200.restart (this repository's loader), so the
    case also checks that the loader and the leaf mapping carry every leaf the
    step reads."""
    from ibis.io.restart import load_state
    from ibis_b200 import dropin, restart
    leaves, meta, extra = restart.load(RESTART)
    n = int(np.asarray(leaves["soil.tg"]).shape[0])
    st, _ = load_state(RESTART, create_ibis_state(GridConfig(nlon=1, nlat=1, npoi=n, nbedrock=3)))
    consts = get_constants()
    rng = np.random.Generator(np.random.PCG64(seed))
    lat = rng.uniform(-40.0, 70.0, size=n)
    forc = synth.make_forcing(rng, lat, nhour, start_doy=172)
    sp = dataclasses.replace(loops.default_sim_params(n), latitude=_a(np.deg2rad(lat)), bedrock=BedrockParams())
    P = dropin.step_params(st, consts, sp, 3600.0)
    tree = restart.as_tree(leaves)
    prog = dropin._leaf_dict(tree, "PROG", n)
    stat = dropin._leaf_dict(tree, "STAT", n)
    stat["f_inund"] = np.zeros(n)
    wl = synth.Workload(ncell=n, nhour=nhour, prog=prog, stat=stat, forc=forc, params=P, latitude=lat,
                        start_doy=172, meta=dict(source="site_transient_1996"))
    out = pack_inputs(wl)
    for h in range(nhour):
        st = set_forcing(st, wl.forcing_at(h))
        st = loops.timestep_body(st, consts, sp, 3600.0)
        if h + 1 in record:
            for k, v in snapshot(st).items():
                out[f"out.{h + 1}.{k}"] = v
    out["meta.record"] = np.asarray(record)
    path = os.path.join(HERE, "restart_1996.npz")
    np.savez_compressed(path, **out)
    print(f"wrote {path}: {len(out)} arrays, {os.path.getsize(path)} bytes")


def write_restart_subset(ncell=16):
    """tests/golden/restart_16cells.npz: the reference's checkpoint cut to its
    first cells (every per-cell leaf sliced, the rest as stored), for tests that
    load a checkpoint where the reference tree is absent."""
    z = np.load(RESTART, allow_pickle=False)
    n = int(np.asarray(z["leaf_3"]).shape[0])            # soil.tg
    out = {}
    for k in z.files:
        v = z[k]
        if k.startswith("leaf_") and not k.endswith("_is_none") and v.ndim >= 1 and v.shape[0] == n:
            v = v[:ncell]
        out[k] = v
    path = os.path.join(HERE, f"restart_{ncell}cells.npz")
    np.savez_compressed(path, **out)
    print(f"wrote {path}: {os.path.getsize(path)} bytes")


def write_restart_modules_case(seed=31):
    """tests/golden/restart_modules_16cells.npz: the reference's own
    ``save_state`` (io/restart.py:19-52) of the 16-cell checkpoint's state with
    the wetland CH4 state and the four calibration modules (stress, ET parts,
    seasonal, NEE parts) attached, every module leaf filled with distinct
    seeded values, recorded by leaf path in restart_modules_values.npz.  The
    NumPy stand-in for ``jax`` has no JAX tree-structure text, so that entry
    is dropped: readers identify the modules by their leaf count, as the
    reference's ``load_state`` does for files without it (io/restart.py:109-115)."""
    from ibis.io.restart import load_state, save_state
    from ibis.bgc.methane import create_methane_state
    n = 16
    st, _ = load_state(os.path.join(HERE, "restart_16cells.npz"),
                       create_ibis_state(GridConfig(nlon=1, nlat=1, npoi=n, nbedrock=3), with_neeparts=True))
    st = eqx.tree_at(lambda s: s.wetland, st, create_methane_state(n), is_leaf=lambda x: x is None)
    rng = np.random.Generator(np.random.PCG64(seed))
    values = {}
    modules = (("wetland", ("flux", "annual", "zwt")), ("stress", ("aystressu", "aystressl", "nday", "u_smooth")),
               ("etparts", ("trans", "interc", "soilev", "snowsub")), ("seasonal", ("acclim_x", "ssen_u", "ssen_l")),
               ("neeparts", ("night", "day")))
    for mod, names in modules:
        vals = tuple(rng.uniform(0.1, 10.0, n).astype(np.float32) for _ in names)
        st = eqx.tree_at(lambda s, mod=mod, names=names: tuple(getattr(getattr(s, mod), k) for k in names), st,
                         tuple(jnp.asarray(v) for v in vals))
        values.update({f"value.{mod}.{k}": v for k, v in zip(names, vals)})
    path = os.path.join(HERE, "restart_modules_16cells.npz")
    tmp = path[:-4] + "_tmp.npz"
    save_state(st, tmp, metadata={"year": 1996})
    z = np.load(tmp, allow_pickle=False)
    out = {k: z[k] for k in z.files if k != "treedef_repr"}
    os.remove(tmp)
    np.savez_compressed(path, **out)
    np.savez_compressed(os.path.join(HERE, "restart_modules_values.npz"), **values)
    print(f"wrote {path}: {int(out['num_leaves'])} leaves, {os.path.getsize(path)} bytes")


def daily_inputs(ncell=12, seed=16):
    """Seeded daily weather for the diurnal fixture: warm and cold days, dry,
    wet and very wet days (an event longer than the random length), humidity
    above saturation at tmin, and latitudes from the polar night to the
    midnight sun."""
    rng = np.random.Generator(np.random.PCG64(seed))
    tmin = rng.uniform(250.0, 295.0, ncell)
    tmax = tmin + rng.uniform(2.0, 15.0, ncell)
    d = dict(tmax=tmax, tmin=tmin, cloud=rng.uniform(0.0, 1.0, ncell),
             precip=np.where(rng.uniform(size=ncell) < 0.4, 0.0, rng.gamma(0.8, 8.0, ncell)),
             psurf=rng.uniform(70000.0, 103000.0, ncell), qd=rng.uniform(0.001, 0.02, ncell),
             ud=rng.uniform(0.5, 8.0, ncell), fira=rng.uniform(200.0, 420.0, ncell))
    d["precip"][0] = 400.0
    d["precip"][1] = 0.0
    lat = rng.uniform(-60.0, 70.0, ncell)
    lat[2], lat[3] = 80.0, -80.0
    return d, lat


def write_diurnal_case(days=(15, 172), seed=7, dtime=3600.0):
    """tests/golden/diurnal.npz: the reference's compute_precip_timing and
    diurnal (weather.py:395-601) for 24 hours of two days, with their uniform
    variates supplied from the counter-based generator the device uses."""
    import jax
    from ibis.physics import weather
    from oracle.weather import uniform24
    daily, lat = daily_inputs()
    n = lat.size
    queue = []

    def uniform(key, shape, *a, **k):
        return jnp.asarray(queue.pop(0).reshape(shape))

    saved = getattr(jax.random, "uniform", None)
    jax.random.uniform = uniform
    out = {f"in.daily.{k}": v for k, v in daily.items()}
    out["in.lat"] = lat
    out["in.days"] = np.asarray(days)
    out["in.seed"] = np.asarray(seed)
    out["in.dtime"] = np.asarray(dtime)
    key = jnp.asarray(np.array([0, 1], dtype=np.uint32))
    try:
        for di, jday in enumerate(days):
            cells = np.arange(n)
            queue[:] = [uniform24(seed, cells, di, 0), uniform24(seed, cells, di, 1)]
            _, plens, startp, endp = weather.compute_precip_timing(key, _a(daily["precip"]), dtime)
            for k, v in (("plens", plens), ("startp", startp), ("endp", endp)):
                out[f"out.{di}.{k}"] = np.asarray(v, dtype=np.float64)
            dw = weather.DailyWeather(td=_a(0.5 * (daily["tmax"] + daily["tmin"])), tmax=_a(daily["tmax"]),
                                      tmin=_a(daily["tmin"]), cloud=_a(daily["cloud"]), precip=_a(daily["precip"]),
                                      psurf=_a(daily["psurf"]), qd=_a(daily["qd"]), ud=_a(daily["ud"]),
                                      iwet=_a(np.zeros(n)), xstore=_a(np.zeros((n, 3))))
            for h in range(int(86400.0 / dtime)):
                queue[:] = [uniform24(seed, cells, di, 2 + h)]
                _, hw = weather.diurnal(h * dtime, jday, dw, _a(lat), plens, startp, endp, key, dtime)
                for k in ("coszen", "ta", "qa", "ua", "fira", "raina", "snowa", "solad", "solai"):
                    out[f"out.{di}.{h}.{k}"] = np.asarray(getattr(hw, k), dtype=np.float64)
    finally:
        if saved is None:
            del jax.random.uniform
        else:
            jax.random.uniform = saved
    path = os.path.join(HERE, "diurnal.npz")
    np.savez_compressed(path, **out)
    print(f"wrote {path}: {len(out)} arrays, {os.path.getsize(path)} bytes")


def write_days_case(ndays=3, jday0=172, seed=9, modules=False, release=False):
    """tests/golden/days_16cells.npz: the reference's own GSWP3 day loop
    (_run_month_scan, loops_gswp3.py:334-612) for ``ndays`` days on the 16-cell
    checkpoint: phenology, 24 hourly steps with accumulators, 10-day means,
    decomposition factors and soil BGC, every leaf recorded after each day.
    Its variates (event timing, hourly wind) come from the counter-based
    generator of the device forcing code; the float32 cast of each day is the
    identity (the float64 run).

    With ``modules`` (tests/golden/days_modules_16cells.npz) the state carries
    the optional stress, ET-parts, seasonal and NEE-parts modules, seeded with
    random seasonal and stress states, under photoperiod-gated senescence of
    both canopies with low critical sums and a growing-season threshold of
    12 C, so the senescence triggers and the growing-season mask both split
    the cells.  With ``release`` as well (tests/golden/days_release_16cells.npz)
    the stomata section of the release parameter file
    (configs/params/params_31s_ch4h.yaml, by the reference's own loader: vmax and
    slope mixing, the NPP split by capacity, acclimation with per-PFT constants,
    sunlit/shaded canopies) and its consistent soil-water weights apply, so the
    acclimation the seasonal state drives reaches the hourly steps."""
    import jax
    from ibis.io.restart import load_state
    from oracle.weather import uniform24
    fix = os.path.join(HERE, "restart_16cells.npz")
    n = 16
    grid = GridConfig(nlon=1, nlat=1, npoi=n, nbedrock=3)
    st, _ = load_state(fix, create_ibis_state(grid, with_neeparts=modules))
    consts = get_constants()
    rng = np.random.Generator(np.random.PCG64(seed))
    lat = rng.uniform(-40.0, 70.0, size=n)
    sp = dataclasses.replace(loops.default_sim_params(n), latitude=_a(np.deg2rad(lat)), bedrock=BedrockParams())
    if modules:
        mrng = np.random.Generator(np.random.PCG64(seed + 1))
        st = eqx.tree_at(lambda s: (s.seasonal.acclim_x, s.seasonal.ssen_u, s.seasonal.ssen_l), st,
                         (_a(mrng.uniform(-5.0, 25.0, n)), _a(mrng.uniform(0.0, 40.0, n)),
                          _a(mrng.uniform(0.0, 40.0, n))))
        st = eqx.tree_at(lambda s: (s.stress.aystressu, s.stress.aystressl, s.stress.nday), st,
                         (_a(mrng.uniform(0.0, 50.0, n)), _a(mrng.uniform(0.0, 50.0, n)),
                          _a(np.floor(mrng.uniform(0.0, 60.0, n)))))
        sp = dataclasses.replace(sp, pheno=dataclasses.replace(
            sp.pheno, sen_photoperiod_u=True, sen_photoperiod_l=True, sen_ycrit_u=25.0, sen_ycrit_l=40.0,
            stress_accum_tmin=12.0))
    if release:
        from ibis.io.physics_params import load_physics_params, build_stomata_params
        d = load_physics_params(os.path.join(REF, "configs/params/params_31s_ch4h.yaml"))
        sp = dataclasses.replace(sp, stomata_params=build_stomata_params(d), h2o_consistent_weights=True)
    days = []
    for d in range(ndays):
        dd, _ = daily_inputs(n, seed=seed + 10 + d)
        dd["td"] = 0.5 * (dd["tmax"] + dd["tmin"]) + rng.uniform(-1.0, 1.0, n)
        days.append(dd)
    queue = []

    def uniform(key, shape, *a, **k):
        return jnp.asarray(queue.pop(0).reshape(shape))

    saved = (getattr(jax.random, "uniform", None), loops_gswp3._cast_tree_f32)
    jax.random.uniform = uniform
    loops_gswp3._cast_tree_f32 = lambda tree: tree
    out = {"in.lat": lat, "in.jday0": np.asarray(jday0), "in.seed": np.asarray(seed), "in.ndays": np.asarray(ndays),
           "in.modules": np.asarray(int(modules))}
    if modules:
        for leaf in ("seasonal.acclim_x", "seasonal.ssen_u", "seasonal.ssen_l", "stress.aystressu",
                     "stress.aystressl", "stress.nday"):
            mod, name = leaf.split(".")
            out["in." + leaf] = np.asarray(getattr(getattr(st, mod), name), dtype=np.float64)
    from ibis_b200 import dropin
    from ibis_b200.params import PARAM_FIELDS
    P = dropin.step_params(st, consts, sp, 3600.0)
    P.flags |= dropin.parts_flags(st)
    for name, _, _ in PARAM_FIELDS:
        out["in.param." + name] = np.asarray(getattr(P, name), dtype=np.float64)
    out["in.param.flags"] = np.asarray(P.flags, dtype=np.int64)
    DP = dropin.day_params(sp)
    for name in dropin.DAY_PARAM_PATHS:
        out["in.dparam." + name] = np.asarray(getattr(DP, name), dtype=np.float64)
    for d, dd in enumerate(days):
        for k, v in dd.items():
            out[f"in.daily.{d}.{k}"] = np.asarray(v)
    key = jnp.asarray(np.array([0, 1], dtype=np.uint32))
    try:
        for d, dd in enumerate(days):
            cells = np.arange(n)
            queue[:] = [uniform24(seed, cells, d, s) for s in range(26)]
            xs = tuple(_a(np.asarray(dd[k])[None]) for k in ("td", "tmax", "tmin", "cloud", "precip", "psurf", "qd",
                                                             "ud")) + (_a(np.zeros((1, n))), _a(dd["fira"][None]),
                                                                       jnp.asarray(np.array([jday0 + d], np.int32)))
            st, key, _ = loops_gswp3._run_month_scan(st, key, consts, sp, xs, 1, 365, 3600.0, 2)
            assert not queue
            for pth, v in zip(leaf_paths(st), jax.tree.flatten(st)[0]):
                out[f"out.{d}.{pth}"] = np.asarray(v, dtype=np.float64)
    finally:
        if saved[0] is None:
            del jax.random.uniform
        else:
            jax.random.uniform = saved[0]
        loops_gswp3._cast_tree_f32 = saved[1]
    path = os.path.join(HERE, "days_release_16cells.npz" if release else
                        "days_modules_16cells.npz" if modules else "days_16cells.npz")
    np.savez_compressed(path, **out)
    print(f"wrote {path}: {len(out)} arrays, {os.path.getsize(path)} bytes")


def write_observed_sw_case(seed=23, n=64):
    """tests/golden/observed_sw.npz: the reference's ``observed_shortwave``
    (physics/weather.py:458-481) on random observed totals (negative, zero and
    above-clear-sky included), sun heights (below the horizon included), masks
    and generator values, on four days of the year."""
    from ibis.physics.weather import observed_shortwave
    rng = np.random.Generator(np.random.PCG64(seed))
    out = {}
    for d, jday in enumerate((1, 80, 172, 300)):
        sw = rng.uniform(-50.0, 1300.0, n)
        sw[:4] = (0.0, 1e-3, 1500.0, -1.0)
        cz = rng.uniform(-0.3, 1.0, n)
        cz[4:8] = (0.0, 1e-4, 1.0, -1e-4)
        use = rng.uniform(size=n) < 0.7
        sd, si = rng.uniform(0.0, 500.0, (n, 2)), rng.uniform(0.0, 200.0, (n, 2))
        a, b = observed_shortwave(_a(sw), jnp.asarray(use), _a(cz), jday, _a(sd), _a(si))
        out.update({f"{d}.sw": sw, f"{d}.coszen": cz, f"{d}.use": use, f"{d}.solad_gen": sd, f"{d}.solai_gen": si,
                    f"{d}.jday": np.asarray(jday), f"{d}.solad": np.asarray(a, np.float64),
                    f"{d}.solai": np.asarray(b, np.float64)})
    path = os.path.join(HERE, "observed_sw.npz")
    np.savez_compressed(path, **out)
    print(f"wrote {path}: {len(out)} arrays, {os.path.getsize(path)} bytes")


def write_wetland_case(seed=41, nlat=12, nlon=20, nmonth=9):
    """tests/golden/wetland_area.npz: the reference's wetland-area functions on
    seeded inputs -- the learned wetland's month-by-month feature builder
    (bgc/wetland_learned.py:49-104) over ``nmonth`` months on a ``nlat`` x
    ``nlon`` grid with about 60 % land (its lags, 3-month means and 5 x 5
    neighbourhood means wrapping at every edge), ``hybrid_fraction`` (:107-110),
    and the dynamic wetland area's ``root_zone_water`` / ``dynamic_fraction``
    (bgc/wetland_area.py:22-39), frozen layers and zero spreads included."""
    from ibis.bgc import wetland_learned as WL
    from ibis.bgc import wetland_area as WA
    rng = np.random.Generator(np.random.PCG64(seed))
    I, J = np.where(rng.random((nlat, nlon)) < 0.6)
    n, nl = len(I), 6
    poros = rng.uniform(0.3, 0.6, (n, nl))
    hsoi = np.array([0.10, 0.15, 0.25, 0.50, 1.0, 2.0])
    ws = rng.uniform(0.0, 1.0, (nmonth, n, nl)).astype(np.float32)
    wi = rng.uniform(0.0, 0.3, (nmonth, n, nl)).astype(np.float32)
    ts = rng.uniform(250.0, 300.0, (nmonth, n, nl)).astype(np.float32)
    tg = rng.uniform(250.0, 300.0, (nmonth, n)).astype(np.float32)
    pr = rng.uniform(0.0, 200.0, (nmonth, n)).astype(np.float32)
    et = rng.uniform(0.0, 100.0, (nmonth, n)).astype(np.float32)
    ro = rng.uniform(0.0, 80.0, (nmonth, n)).astype(np.float32)
    fb = WL.FeatureBuilder(I, J, poros, hsoi, nlat, nlon)
    out = {"in.I": I, "in.J": J, "in.poros": poros, "in.hsoi": hsoi, "in.ws": ws, "in.wi": wi, "in.ts": ts,
           "in.tg": tg, "in.prcp": pr, "in.aet": et, "in.runoff": ro, "in.nlat": np.asarray(nlat),
           "in.nlon": np.asarray(nlon), "dyn_feats": np.array(WL.DYN_FEATS), "stat_feats": np.array(WL.STAT_FEATS)}
    feats = np.zeros((nmonth, len(WL.DYN_FEATS), n))
    for t in range(nmonth):
        f = fb.step(ts[t], ws[t], wi[t], tg[t], pr[t], et[t], ro[t])
        for k, name in enumerate(WL.DYN_FEATS):
            feats[t, k] = f[name]
    out["out.feats"] = feats
    # hybrid fraction: anomalies of both signs, bounds hit from above and below
    fclim = rng.uniform(0.0, 0.5, n); fmax = rng.uniform(0.05, 0.9, n); P = rng.uniform(0.0, 1.0, n)
    pbar = rng.uniform(0.0, 1.0, n); lam = rng.uniform(0.0, 3.0, n)
    fclim[:3] = (0.0, 0.9, 0.2)
    out.update({"in.fclim": fclim, "in.fmax": fmax, "in.P": P, "in.pbar": pbar, "in.lam": lam,
                "out.hybrid": np.asarray(WL.hybrid_fraction(fclim, P, pbar, lam, fmax), np.float64)})
    # dynamic area: root-zone water (frozen layers count 0) and the bounded anomaly fraction
    W = WA.root_zone_water(ws[0], poros, hsoi, ts[0])
    mu = rng.uniform(0.05, 0.3, n); sd = rng.uniform(0.0, 0.1, n)
    sd[:4] = (0.0, 1e-10, 1e-9, 2e-9)
    beta = rng.uniform(0.0, 0.2, n); fmin = rng.uniform(0.0, 0.05, n)
    frozen = np.asarray(ts[0][:, 0], np.float64) <= WA.T_FREEZE
    out.update({"in.mu": mu, "in.sd": sd, "in.beta": beta, "in.fmin": fmin, "out.W": np.asarray(W, np.float64),
                "out.dynamic": np.asarray(WA.dynamic_fraction(fclim, W, mu, sd, beta, fmin, fmax, frozen=frozen),
                                          np.float64),
                "meta.t_freeze": np.asarray(WA.T_FREEZE), "meta.root_layers": np.asarray(WA.ROOT_LAYERS),
                "meta.nb": np.asarray(WL.NB)})
    path = os.path.join(HERE, "wetland_area.npz")
    np.savez_compressed(path, **out)
    print(f"wrote {path}: {len(out)} arrays, {os.path.getsize(path)} bytes")


def write_methane_case(seed=21, ndays=31):
    """tests/golden/methane_month.npz: the reference's monthly wetland methane
    functions (bgc/methane.py:233-496) on the 16-cell checkpoint's soil state:
    the water table with and without an observed depth (NaN, negative and
    beyond-z_max entries included), the flux, ``methane_step``,
    ``methane_step_from_mean``, ``scale_month``, ``ch4_carbon_from_rh`` and
    ``reset_annual``, under the default and one non-default MethaneParams."""
    from ibis.bgc import methane as M
    from ibis.io.restart import load_state
    n = 16
    st, _ = load_state(os.path.join(HERE, "restart_16cells.npz"),
                       create_ibis_state(GridConfig(nlon=1, nlat=1, npoi=n, nbedrock=3)))
    so = st.soil
    tsoi, wsoi, wisoi = (np.asarray(x, np.float64) for x in (so.tsoi, so.wsoi, so.wisoi))
    hsoi = np.asarray(so.hsoi, np.float64)[:tsoi.shape[1]]
    rng = np.random.Generator(np.random.PCG64(seed))
    wisoi = wisoi.copy()
    wisoi[:4] = rng.uniform(0.0, 0.9, (4, tsoi.shape[1]))        # frozen soil in a few cells
    tsoi = tsoi.copy()
    tsoi[4:7] = 270.0 + rng.uniform(0.0, 6.0, (3, tsoi.shape[1]))  # thawed/frozen layers around tmelt
    f_inund = rng.uniform(-0.1, 1.1, n)
    rh = rng.uniform(0.0, 5e-3, n)
    rh[0] = -1e-4
    zwt_obs = rng.uniform(-0.3, 5.0, n)
    zwt_obs[rng.uniform(size=n) < 0.4] = np.nan
    flux_month = rng.uniform(0.0, 1e-4, n)
    annual0 = rng.uniform(0.0, 1e-2, n)
    scale = rng.uniform(0.0, 1.2, n)
    rh_now, rh_before = rng.uniform(0.2, 0.4, n), rng.uniform(0.0, 0.3, n)
    out = {"in.tsoi": tsoi, "in.wsoi": wsoi, "in.wisoi": wisoi, "in.hsoi": hsoi, "in.f_inund": f_inund, "in.rh": rh,
           "in.zwt_obs": zwt_obs, "in.flux_month": flux_month, "in.annual0": annual0, "in.scale": scale,
           "in.rh_now": rh_now, "in.rh_before": rh_before, "in.ndays": np.asarray(ndays)}
    variants = {"default": M.MethaneParams(),
                "custom": M.MethaneParams(z_wt_max=0.45, sat_crit=0.85, q10p=2.1, r_ch4=0.31, z_tau=0.35,
                                          tau_oxid=0.2, t_ref=290.0, z_max=3.0)}
    a = lambda x: np.asarray(x, np.float64)
    for tag, p in variants.items():
        for f in ("sat_crit", "z_max", "r_ch4", "q10p", "t_ref", "z_wt_max", "z_wt_ref", "z_tau", "tau_oxid"):
            out[f"param.{tag}.{f}"] = np.asarray(float(getattr(p, f)))
        out[f"{tag}.zwt"] = a(M.wetland_water_table(_a(wsoi), _a(wisoi), _a(hsoi), p))
        out[f"{tag}.flux"] = a(M.methane_flux(_a(f_inund), _a(rh), _a(tsoi), _a(wsoi), _a(wisoi), _a(hsoi), p))
        out[f"{tag}.flux_obs"] = a(M.methane_flux(_a(f_inund), _a(rh), _a(tsoi), _a(wsoi), _a(wisoi), _a(hsoi), p,
                                                  zwt_obs=_a(zwt_obs)))
        m0 = M.MethaneState(flux=_a(np.zeros(n)), annual=_a(annual0), zwt=_a(np.zeros(n)))
        for obs in (False, True):
            zo = _a(zwt_obs) if obs else None
            sfx = "_obs" if obs else ""
            ms = M.methane_step(m0, _a(f_inund), _a(rh), _a(tsoi), _a(wsoi), _a(wisoi), _a(hsoi), ndays, p, zwt_obs=zo)
            mm = M.methane_step_from_mean(m0, _a(flux_month), _a(wsoi), _a(wisoi), _a(hsoi), ndays, p, zwt_obs=zo)
            for name, st_ in (("step", ms), ("mean", mm)):
                for leaf in ("flux", "annual", "zwt"):
                    out[f"{tag}.{name}{sfx}.{leaf}"] = a(getattr(st_, leaf))
            sc = M.scale_month(mm, _a(annual0), _a(scale))
            for leaf in ("flux", "annual", "zwt"):
                out[f"{tag}.scaled{sfx}.{leaf}"] = a(getattr(sc, leaf))
            out[f"{tag}.take{sfx}"] = a(M.ch4_carbon_from_rh(sc.annual, _a(annual0), _a(rh_now), _a(rh_before)))
        out[f"{tag}.reset.annual"] = a(M.reset_annual(m0).annual)
    path = os.path.join(HERE, "methane_month.npz")
    np.savez_compressed(path, **out)
    print(f"wrote {path}: {len(out)} arrays, {os.path.getsize(path)} bytes")


def write_methane_bands_case(seed=21, ndays=31):
    """tests/golden/methane_bands.npz: the reference's wetland methane with
    per-cell parameters by biome (``biome_methane_params``,
    bgc/methane.py:521-563) on the 16-cell checkpoint's soil state: the
    latitude rule alone (the validated production constants), with Koeppen
    wetland types overriding it in some cells, and the release parameter
    file's methane section and ``methane_bands`` (loaded by the reference's own
    loader) -- the per-cell parameters, water table, flux (with and without an
    observed depth) and ``methane_step``."""
    import json
    from ibis.bgc import methane as M
    from ibis.io.physics_params import load_physics_params, build_methane_params
    from ibis.io.restart import load_state
    n = 16
    st, _ = load_state(os.path.join(HERE, "restart_16cells.npz"),
                       create_ibis_state(GridConfig(nlon=1, nlat=1, npoi=n, nbedrock=3)))
    so = st.soil
    tsoi, wsoi, wisoi = (np.asarray(x, np.float64) for x in (so.tsoi, so.wsoi, so.wisoi))
    hsoi = np.asarray(so.hsoi, np.float64)[:tsoi.shape[1]]
    rng = np.random.Generator(np.random.PCG64(seed))
    tsoi = tsoi.copy()
    tsoi[4:7] = 270.0 + rng.uniform(0.0, 6.0, (3, tsoi.shape[1]))
    f_inund = rng.uniform(0.0, 1.0, n)
    rh = rng.uniform(0.0, 5e-3, n)
    zwt_obs = rng.uniform(-0.3, 5.0, n)
    zwt_obs[rng.uniform(size=n) < 0.4] = np.nan
    annual0 = rng.uniform(0.0, 1e-2, n)
    # latitudes on and around the biome edges; Koeppen types (-1: the latitude rule)
    lat = np.array([-60.0, -30.0, -29.999, -10.0, 0.0, 10.0, 29.999, 30.0, 45.0, 59.999, 60.0, 65.0, 70.0, 75.0,
                    -45.0, 20.0])
    band_index = np.array([-1, 0, 1, -1, 2, -1, -1, 0, 2, -1, 1, -1, 0, -1, 2, -1])
    d = load_physics_params(os.path.join(REF, "configs/params/params_31s_ch4h.yaml"))
    base, bands = build_methane_params(d), d["methane_bands"]
    out = {"in.tsoi": tsoi, "in.wsoi": wsoi, "in.wisoi": wisoi, "in.hsoi": hsoi, "in.f_inund": f_inund, "in.rh": rh,
           "in.zwt_obs": zwt_obs, "in.annual0": annual0, "in.ndays": np.asarray(ndays), "in.lat": lat,
           "in.band_index": band_index, "in.bands": np.asarray(json.dumps(bands))}
    fields = ("sat_crit", "z_max", "r_ch4", "q10p", "t_ref", "z_wt_max", "z_wt_ref", "z_tau", "tau_oxid")
    for f in fields:
        out[f"base.default.{f}"] = np.asarray(float(getattr(M.MethaneParams(), f)))
        out[f"base.release.{f}"] = np.asarray(float(getattr(base, f)))
    variants = {"biome": (M.biome_methane_params(_a(lat)), "default", False, False),
                "biome_koppen": (M.biome_methane_params(_a(lat), band_index=band_index), "default", True, False),
                "release": (M.biome_methane_params(_a(lat), base=base, bands=bands, band_index=band_index),
                            "release", True, True)}
    a = lambda x: np.asarray(x, np.float64)
    for tag, (p, b, koppen, with_bands) in variants.items():
        out[f"meta.{tag}"] = np.asarray([b, str(int(koppen)), str(int(with_bands))])
        for f in fields:
            out[f"param.{tag}.{f}"] = np.broadcast_to(a(getattr(p, f)), (n,)).copy()
        out[f"{tag}.zwt"] = a(M.wetland_water_table(_a(wsoi), _a(wisoi), _a(hsoi), p))
        out[f"{tag}.flux"] = a(M.methane_flux(_a(f_inund), _a(rh), _a(tsoi), _a(wsoi), _a(wisoi), _a(hsoi), p))
        out[f"{tag}.flux_obs"] = a(M.methane_flux(_a(f_inund), _a(rh), _a(tsoi), _a(wsoi), _a(wisoi), _a(hsoi), p,
                                                  zwt_obs=_a(zwt_obs)))
        m0 = M.MethaneState(flux=_a(np.zeros(n)), annual=_a(annual0), zwt=_a(np.zeros(n)))
        ms = M.methane_step(m0, _a(f_inund), _a(rh), _a(tsoi), _a(wsoi), _a(wisoi), _a(hsoi), ndays, p)
        for leaf in ("flux", "annual", "zwt"):
            out[f"{tag}.step.{leaf}"] = a(getattr(ms, leaf))
    path = os.path.join(HERE, "methane_bands.npz")
    np.savez_compressed(path, **out)
    print(f"wrote {path}: {len(out)} arrays, {os.path.getsize(path)} bytes")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--only", default=None)
    args = ap.parse_args()
    if args.only in (None, "restart_leaves"):
        write_restart_leaves()
    if args.only in (None, "restart_1996"):
        build_restart_case()
        write_restart_subset()
    if args.only in (None, "diurnal"):
        write_diurnal_case()
    if args.only in (None, "days"):
        write_days_case()
    if args.only in (None, "methane_month"):
        write_methane_case()
    if args.only in (None, "observed_sw"):
        write_observed_sw_case()
    if args.only in (None, "wetland_area"):
        write_wetland_case()
    if args.only in (None, "methane_bands"):
        write_methane_bands_case()
    if args.only in (None, "day_parts"):
        write_parts_case()
    if args.only in (None, "days_modules"):
        write_days_case(jday0=250, modules=True)
    if args.only in (None, "days_release"):
        write_days_case(jday0=250, modules=True, release=True)
    if args.only in (None, "restart_modules"):
        write_restart_modules_case()
    for name in X3_CASES:
        if args.only in (None, name):
            write_x3_case(name)
    if args.only in ("restart_leaves", "restart_1996", "diurnal", "days", "methane_month", "observed_sw", "wetland_area", "methane_bands",
                     "day_parts", "days_modules", "days_release", "restart_modules") + tuple(X3_CASES):
        return
    for name, spec in CASES.items():
        if args.only and name != args.only:
            continue
        wl = build_case(name, spec)
        out = pack_inputs(wl)
        snaps = run_steps(wl, set(spec["record"]))
        for h, s in snaps.items():
            for k, v in s.items():
                out[f"out.{h}.{k}"] = v
        if spec.get("day"):
            for k, v in run_day_accumulators(wl).items():
                out[f"day.{k}"] = v
        out["meta.record"] = np.asarray(spec["record"])
        path = os.path.join(HERE, f"{name}.npz")
        np.savez_compressed(path, **out)
        print(f"wrote {path}: {len(out)} arrays, {os.path.getsize(path)} bytes")


if __name__ == "__main__":
    main()
