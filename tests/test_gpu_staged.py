"""The staged fused configuration (form 2: each hour's forcing tile brought into
shared memory by bulk copies while the hour before it runs) against the
unstaged fused kernel of the same block size (configuration 6).

Both run the same step code on the same forcing values; only where the values
come from differs, so the day agrees to the FP32 rounding the two separately
compiled kernels may differ by (the tolerances of the fused-vs-split test),
a forcing buffer the copies cannot address falls back to configuration 6's
own kernel (the same bits), and no launch reports a wait that gave up
(status[0] bit 2).
"""
import ctypes

import numpy as np
import pytest
import torch

from ibis_b200 import lib, replicas, synth
from ibis_b200.columns import Columns

pytestmark = pytest.mark.gpu

STAGED = 11
UNSTAGED = 6


def _ptr(t, offset_bytes=0):
    return ctypes.c_void_p(t.data_ptr() + offset_bytes)


def _run(wl, cfg, nstep, forc_offset=0):
    cols = Columns.from_host(wl.prog, wl.stat, dtype=torch.float32, acc=True)
    forc = cols.forcing(wl.forc, 0, nstep)
    if forc_offset:
        # the same values one float further on: the start is no longer 16-byte aligned
        buf = torch.zeros(forc.numel() + 4, dtype=torch.float32, device=forc.device)
        buf[forc_offset:forc_offset + forc.numel()].copy_(forc.reshape(-1))
        fptr = _ptr(buf, 4 * forc_offset)
    else:
        fptr = _ptr(forc)
    so = lib.load()
    rc = so.ibis_step_config_f32(_ptr(cols.prog), _ptr(cols.stat), fptr, ctypes.c_void_p(0), _ptr(cols.acc),
                                 ctypes.c_void_p(0), cols.ncell, cols.ld, nstep, ctypes.byref(wl.params.to_c()),
                                 _ptr(cols.status), ctypes.c_void_p(torch.cuda.current_stream().cuda_stream), cfg)
    assert rc == 0, rc
    torch.cuda.synchronize()
    st = cols.status.cpu().numpy()
    return cols, int(st[0])


def _close(a, b):
    pa, pb = a.prog_host(), b.prog_host()
    for k in ("tsoi", "tg", "tu", "tl", "tsno", "ti"):
        np.testing.assert_allclose(pa[k], pb[k], rtol=1e-4, atol=0.05, err_msg=k)
    for k in ("wsoi", "wisoi", "fi"):
        np.testing.assert_allclose(pa[k], pb[k], rtol=1e-3, atol=1e-4, err_msg=k)
    aa, ab = a.acc_host(), b.acc_host()
    for k, w in ab.items():
        g = np.asarray(aa[k], np.float64)
        scale = max(float(np.abs(w).max()), 1e-30)
        assert float(np.abs(g - w).max()) <= 1e-3 * scale, k


def test_staged_is_listed_as_a_fused_configuration(cuda_lib):
    c = lib.configs()[STAGED]
    assert c["form"] == "fused" and c["staged"] and c["block"] == 224 and c["min_blocks"] == 1
    assert not lib.configs()[UNSTAGED]["staged"]


@pytest.mark.parametrize("ncell,nstep", [(1001, 24), (224 * 3, 5), (37, 1), (4480, 2)])
def test_staged_day_matches_unstaged(cuda_lib, ncell, nstep):
    """Ragged last blocks (1001 and 37 cells: the last tile rounds up to 4
    cells), whole blocks, one hour and a day."""
    wl = synth.make_workload(ncell, 24, seed=replicas.replica_seed(1000, 0))
    a, sa = _run(wl, STAGED, nstep)
    b, sb = _run(wl, UNSTAGED, nstep)
    assert sa == 0 and sb == 0
    _close(a, b)


def test_unaligned_forcing_falls_back_to_the_unstaged_kernel(cuda_lib):
    wl = synth.make_workload(1001, 24, seed=replicas.replica_seed(1000, 0))
    a, sa = _run(wl, STAGED, 24, forc_offset=1)
    b, sb = _run(wl, UNSTAGED, 24)
    assert sa == 0 and sb == 0
    assert torch.equal(a.prog, b.prog) and torch.equal(a.acc, b.acc)


def test_staged_through_the_host_pipeline(cuda_lib):
    """ibis_step_host_f32 with the staged configuration: groups of two
    blocks, each reading its forcing at its own offset, against the same
    configuration from device memory."""
    wl = synth.make_workload(224 * 40 + 17, 24, seed=replicas.replica_seed(1000, 0))
    a = Columns.from_host(wl.prog, wl.stat, dtype=torch.float32, acc=True, mode=STAGED)
    b = Columns.from_host(wl.prog, wl.stat, dtype=torch.float32, acc=True, mode=STAGED)
    forc = a.forcing(wl.forc)
    a.run(forc, wl.params)
    b.run_host(forc.cpu().pin_memory(), wl.params, group=224 * 2)
    torch.cuda.synchronize()
    assert int(a.status[0]) == 0 and int(b.status[0]) == 0
    assert torch.equal(a.prog, b.prog) and torch.equal(a.acc, b.acc)
