"""The allocation-free two-kernel entry point against the ordinary one.

``ibis_step_split_noalloc_f32`` serves callers that cannot allocate device
memory while they run the step (XLA custom-call handlers, which must not
allocate behind XLA's allocator; serving loops that reserved all memory up
front): its hand-off scratch is a fixed array inside the library.  It must give the same results as
``ibis_step_split_f32`` with a caller-allocated scratch buffer, on two calls in
a row (the second call reuses the array the first one left behind).  This file
is collected last so that a failure here stops nothing else.
"""
import ctypes

import numpy as np
import pytest
import torch

from ibis_b200 import layout as L
from ibis_b200 import lib as ilib
from ibis_b200 import synth

pytestmark = pytest.mark.gpu


def _buffers(wl, ld, dev):
    prog = torch.from_numpy(synth.to_planes("PROG", wl.prog, ld)).to(dev)
    stat = torch.from_numpy(synth.to_planes("STAT", wl.stat, ld)).to(dev)
    acc = torch.zeros((2 * L.N_ACC, ld), device=dev)
    return prog, stat, acc


def test_noalloc_split_matches_allocated_split_twice():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    lib = ilib.load()
    dev = torch.device("cuda", torch.cuda.current_device())
    wl = synth.make_workload(3000, 6, seed=21, edge_cases=True)
    ld = L.leading_dim(wl.ncell)
    forc = torch.from_numpy(synth.forcing_planes(wl.forc, ld)).to(dev)
    params = wl.params.to_c()
    ptr = lambda t: ctypes.c_void_p(t.data_ptr()) if t is not None else ctypes.c_void_p(0)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    p_ref, s_ref, a_ref = _buffers(wl, ld, dev)
    p_new, s_new, a_new = _buffers(wl, ld, dev)
    scratch = torch.zeros((lib.ibis_mid_planes(), ld), device=dev)
    st_ref = torch.tensor([0, 2 ** 31 - 1], dtype=torch.int32, device=dev)
    st_new = torch.tensor([0, 2 ** 31 - 1], dtype=torch.int32, device=dev)
    for call in range(2):
        h0, h1 = 3 * call, 3 * call + 3
        f = forc[h0:h1].contiguous()
        rc = lib.ibis_step_split_f32(ptr(p_ref), ptr(s_ref), ptr(f), None, ptr(a_ref), ptr(scratch), wl.ncell, ld,
                                     3, ctypes.byref(params), ptr(st_ref), stream)
        assert rc == 0
        rc = lib.ibis_step_split_noalloc_f32(ptr(p_new), ptr(s_new), ptr(f), None, ptr(a_new), wl.ncell, ld, 3,
                                             ctypes.byref(params), ptr(st_new), stream)
        assert rc == 0
        torch.cuda.synchronize()
        # the same kernels on the same inputs, only the scratch differs: the
        # results must be the same bits (a stale or aliased plane would show)
        np.testing.assert_array_equal(p_new.cpu().numpy(), p_ref.cpu().numpy())
        np.testing.assert_array_equal(a_new.cpu().numpy(), a_ref.cpu().numpy())
    assert st_new.cpu().tolist() == st_ref.cpu().tolist()


def test_noalloc_rejects_oversized_batches():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    lib = ilib.load()
    params = synth.make_workload(1, 1).params.to_c()
    # ld beyond the built-in scratch: refused before any pointer is touched
    rc = lib.ibis_step_split_noalloc_f32(ctypes.c_void_p(8), ctypes.c_void_p(8), ctypes.c_void_p(8), None,
                                         ctypes.c_void_p(8), 40000, 40000 + 32 - 40000 % 32, 1,
                                         ctypes.byref(params), None, None)
    assert rc == -22
