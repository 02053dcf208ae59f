"""FP32 production kernels against the FP64 kernels over a year, and the FP64
kernels against the oracle over a week (last-bit differences between CUDA's
and the host's arithmetic grow slowly through the snow and soil-water
coupling; after 6 steps they are below 1e-9, tests/test_gpu_parity.py).

Bounds (relative error of the all-cell annual total, 1,000 cells x 8,760 h):
GPP, NPP, ET, canopy sensible heat and the annual-mean soil temperature of
every layer within 1e-4; runoff and drainage within 1e-3 and wetland CH4
within 2e-3, which follow soil moisture, whose FP32 trajectory departs further
from the FP64 one.  Integer-valued counters stay integers; the fire-season
counters are threshold counts of FP state and agree in at least 98% of cells.
The reference's own float32 run differs from its float64 run by more than this
(docs/technote/17_numerics_verification.md:367-383).
"""
import warnings

import numpy as np
import pytest
import torch

import oracle
from ibis_b200 import precision, synth
from ibis_b200.columns import Columns
from goldens import compare

pytestmark = pytest.mark.gpu
warnings.filterwarnings("ignore", category=RuntimeWarning)


@pytest.fixture(scope="module")
def year_report(cuda_lib):
    return precision.report(1000, 8760)


def test_no_nonfinite(year_report):
    assert not year_report["nonfinite"]["f32"] and not year_report["nonfinite"]["f64"]


@pytest.mark.parametrize("flux,bound", [("gpp", 1e-4), ("npp", 1e-4), ("et", 1e-4), ("sensible_heat", 1e-4),
                                        ("runoff", 1e-3), ("drainage", 1e-3), ("ch4", 2e-3)])
def test_annual_flux_totals(year_report, flux, bound):
    assert year_report["fluxes"][flux]["total_rel"] < bound, year_report["fluxes"][flux]


def test_soil_temperature_by_layer(year_report):
    for k, v in year_report["soil_t"].items():
        assert v["total_rel"] < 1e-4 and v["max_rel"] < 1e-3, (k, v)


def test_counters(year_report):
    c = year_report["counters"]
    assert all(v["integer_valued"] for v in c.values())
    assert c["nytimes"]["equal_frac"] == 1.0
    assert c["nfirestep"]["equal_frac"] >= 0.98 and c["nfirestep_vpd"]["equal_frac"] >= 0.98


def test_f64_kernel_tracks_oracle_for_a_week(cuda_lib):
    """168 hours on 16 ordinary columns: temperatures within 1e-6 relative,
    every other field and accumulator within 1e-3 (thresholds such as puddle
    freezing amplify last-bit differences over a week; after 6 steps every field
    agrees to 1e-9, tests/test_gpu_parity.py)."""
    w = synth.make_workload(16, 168, seed=21, edge_cases=False)
    P = w.params.copy()
    P.flags = P.flags & ~(1 << 8)
    cols = Columns.from_host(w.prog, w.stat, dtype=torch.float64, acc=True)
    cols.run(cols.forcing(w.forc), P)
    torch.cuda.synchronize()
    prog = {k: v.copy() for k, v in w.prog.items()}
    acc = oracle.new_acc(16)
    with np.errstate(all="ignore"):
        for h in range(168):
            prog, D, acc = oracle.step(prog, w.stat, w.forcing_at(h), P, acc)
    temps = ("tsoi", "tg", "tu", "ts", "tl", "t12", "t34", "tsno", "ti", "tlsub", "tsoi_deep")
    got = cols.prog_host()
    bad = compare({k: got[k] for k in temps}, prog, 1e-6)
    assert not bad, bad[:6]
    bad = compare(got, prog, 1e-3) + compare(cols.acc_host(compensated=False), acc, 1e-3)
    assert not bad, bad[:6]
