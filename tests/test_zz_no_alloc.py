"""fs_edc_noalloc: the EDC step with its flag-scan scratch in a static device
array, for callers that may not allocate device memory (a host whose own
allocator owns the GPU's memory, or a loop that cannot take cudaMalloc's
synchronisation).  Its results must equal fs_edc's, also on a second call
that finds the first call's scratch contents.

Collected last on purpose: it must pass in a fresh process and after the
other GPU tests.
"""
import gc

import numpy as np
import pytest
import torch

from firewebapp_b200 import _lib
from firewebapp_b200._lib import ptr

pytestmark = pytest.mark.gpu

MAX_CELLS = 1 << 27   # FS_EDC_NOALLOC_MAX_CELLS in include/firestep.h


def _inputs(n, seed):
    rng = np.random.default_rng(seed)
    d = dict(
        rho=rng.uniform(0.3, 1.2, n), k=rng.uniform(1e-3, 1.0, n), e=rng.uniform(1e-3, 1.0, n),
        Tg=rng.uniform(300.0, 1800.0, n),
        Yf=np.where(rng.random(n) < 3e-4, rng.uniform(0.0, 0.2, n), 0.0),
        YO=rng.uniform(0.0, 0.232, n), YH=rng.uniform(0.0, 0.2, n))
    return {k: torch.tensor(v, dtype=torch.float64, device="cuda") for k, v in d.items()}


def _run(entry, n, t, scratch=None):
    """One call on copies of the inputs; returns the outputs and the torch
    allocator's (allocated, reserved) bytes just before and just after it."""
    L = _lib.lib()
    Tg, Yf, YO = t["Tg"].clone(), t["Yf"].clone(), t["YO"].clone()
    om = torch.zeros_like(Tg)
    s = torch.cuda.current_stream().cuda_stream
    args = [n, ptr(t["rho"]), ptr(Tg), ptr(Yf), ptr(YO), ptr(t["k"]), ptr(t["e"]), ptr(t["YH"]),
            ptr(om), 0.34, 1100.0, 2e-3, 1, 1.3, 17e6, 0]
    torch.cuda.synchronize()
    # tensors left unreachable by earlier tests are freed now, and no
    # collection runs between the two readings, so any change between them is
    # the call's own
    gc.collect()
    gc.disable()
    try:
        before = (torch.cuda.memory_allocated(), torch.cuda.memory_reserved())
        if entry == "fs_edc":
            st = L.fs_edc(*args, ptr(scratch), s)
        else:
            st = L.fs_edc_noalloc(*args, s)
        torch.cuda.synchronize()
        after = (torch.cuda.memory_allocated(), torch.cuda.memory_reserved())
    finally:
        gc.enable()
    _lib.check(st, entry)
    return (Tg, Yf, YO, om), before, after


def test_noalloc_equals_fs_edc_on_two_calls():
    L = _lib.lib()
    for n, seed in ((1_234_567, 1), (700_001, 2)):
        t = _inputs(n, seed)
        scratch = torch.zeros(int(L.fs_edc_scratch_bytes(n)) + 16, dtype=torch.uint8,
                              device="cuda")
        want, _, _ = _run("fs_edc", n, t, scratch)
        got, before, after = _run("fs_edc_noalloc", n, t)
        assert before == after          # nothing asked of torch's allocator
        for a, b in zip(got, want):
            assert torch.equal(a, b)


def test_noalloc_rejects_sizes_beyond_the_limit():
    L = _lib.lib()
    t = torch.zeros(8, dtype=torch.float64, device="cuda")
    p = ptr(t)
    st = L.fs_edc_noalloc(MAX_CELLS + 1, p, p, p, p, p, p, p, p, 0.34, 1100.0, 1e-3, 1, 1.3,
                          17e6, 0, torch.cuda.current_stream().cuda_stream)
    assert st == 1
    msg = L.fs_last_error().decode()
    assert "static scratch limit" in msg and str(MAX_CELLS) in msg


def test_zero_cells_is_a_no_op_for_both_entries():
    """n == 0 returns FS_OK from both EDC entry points and touches nothing."""
    L = _lib.lib()
    t = torch.full((8,), 7.0, dtype=torch.float64, device="cuda")
    p = ptr(t)
    s = torch.cuda.current_stream().cuda_stream
    scratch = torch.zeros(64, dtype=torch.uint8, device="cuda")
    assert L.fs_edc(0, p, p, p, p, p, p, p, p, 0.34, 1100.0, 1e-3, 1, 1.3, 17e6, 0,
                    ptr(scratch), s) == 0
    assert L.fs_edc_noalloc(0, p, p, p, p, p, p, p, p, 0.34, 1100.0, 1e-3, 1, 1.3, 17e6, 0,
                            s) == 0
    torch.cuda.synchronize()
    assert torch.all(t == 7.0)
