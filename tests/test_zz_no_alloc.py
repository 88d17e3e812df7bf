"""The allocation-free RHS entry point (hw_rhs_noalloc) against the regular one.

hw_rhs_noalloc serves callers that cannot allocate device memory when they call
the RHS; its scratch is a static device array shared by every call.  This file
runs last so that, if it fails, every other test has already run.  Each case
makes two calls in a row (the array keeps the previous call's contents) and
compares them with hw_rhs on the same inputs, within the RHS tolerance of the
parity tests (relative L2 1e-12).
"""
import os

import numpy as np
import pytest

from decks_util import random_state, rel_l2, small_deck

pytestmark = pytest.mark.gpu

hw = pytest.importorskip("hawassi_c_b200")


# (grid, model, varying bottom, CTAs per member, points per CTA); slice 256 runs the
# smallest slice template, the varying bottom the general (HSS) branch of the RHS
CASES = [(1024, "HS2", False, 1, 0), (2048, "HS2", False, 2, 0), (2048, "HS3", False, 1, 0),
         (4096, "HS2", False, 4, 0), (2048, "HS2", True, 2, 0), (1024, "HS2", False, 0, 256)]


@pytest.mark.parametrize("nx,model,varying,cluster,slice_", CASES)
def test_rhs_noalloc_matches_rhs(tmp_path, nx, model, varying, cluster, slice_):
    torch = pytest.importorskip("torch")
    deck = small_deck(tmp_path, f"na_{nx}_{model}_{int(varying)}", nx=nx, model=model, varying=varying)
    e = hw.Engine(deck, cluster=cluster, slice=slice_)
    stream = torch.cuda.current_stream().cuda_stream
    calls0 = e.stats()["rhs_calls"]
    for i, t in enumerate([0.5, 1.7]):
        y = random_state(nx, 40 + i)
        ref = e.rhs(t, y)
        yd = torch.from_numpy(y).cuda()
        dd = torch.full_like(yd, float("nan"))
        torch.cuda.synchronize()
        e.rhs_noalloc(t, yd.data_ptr(), dd.data_ptr(), stream=stream)
        torch.cuda.synchronize()
        got = dd.cpu().numpy()
        assert np.all(np.isfinite(got))
        assert rel_l2(got, ref) < 1e-12
    # both entry points count their calls on the member
    assert e.stats()["rhs_calls"] == calls0 + 4
    e.close()


def test_rhs_noalloc_breaking_state(golden_dir):
    """On a breaking deck the allocation-free RHS advances the member's breaking
    state like hw_rhs: from a mid-break state of the reference's 1dFBr005Bor deck
    (Nx = 4096, two CTAs), two calls in a row on each entry point give the same
    dydt (eddy-viscosity force included) and the same breaking.dat records."""
    torch = pytest.importorskip("torch")
    deck = os.path.join(golden_dir, "fbr005")
    run = hw.Engine(deck, cluster=2)
    run.run_to_time(12.62)
    t0, _, y = run.state()
    run.close()
    a, b = hw.Engine(deck, cluster=2), hw.Engine(deck, cluster=2)
    stream = torch.cuda.current_stream().cuda_stream
    yd = torch.from_numpy(y).cuda()
    for dt_ in (0.0, 0.004):
        ref = a.rhs(t0 + dt_, y)
        dd = torch.full_like(yd, float("nan"))
        torch.cuda.synchronize()
        b.rhs_noalloc(t0 + dt_, yd.data_ptr(), dd.data_ptr(), stream=stream)
        torch.cuda.synchronize()
        assert rel_l2(dd.cpu().numpy(), ref) < 1e-12
    log_a, log_b = a.breaking_log(), b.breaking_log()
    assert log_a and log_a == log_b
    assert a.stats()["rhs_calls"] == b.stats()["rhs_calls"] == 2
    a.close()
    b.close()


def test_rhs_noalloc_rejects_large_grid(tmp_path):
    torch = pytest.importorskip("torch")
    deck = small_deck(tmp_path, "na_big", nx=8192, model="HS2")
    e = hw.Engine(deck)
    yd = torch.zeros(4 * 8192, dtype=torch.float64, device="cuda")
    dd = torch.zeros_like(yd)
    with pytest.raises(hw.EngineError, match="exceeds"):
        e.rhs_noalloc(0.0, yd.data_ptr(), dd.data_ptr())
    e.close()
