"""The allocation-free RHS entry point (hw_rhs_noalloc) against the regular one.

hw_rhs_noalloc serves callers that cannot allocate device memory when they call
the RHS; its scratch is a static device array shared by every call.  This file
runs last so that, if it fails, every other test has already run.  Each case
makes two calls in a row (the array keeps the previous call's contents) and
compares them with hw_rhs on the same inputs, within the RHS tolerance of the
parity tests (relative L2 1e-12).
"""
import numpy as np
import pytest

from decks_util import random_state, rel_l2, small_deck

pytestmark = pytest.mark.gpu

hw = pytest.importorskip("hawassi_c_b200")


@pytest.mark.parametrize("nx,model,cluster", [(1024, "HS2", 1), (2048, "HS2", 2), (2048, "HS3", 1), (4096, "HS2", 4)])
def test_rhs_noalloc_matches_rhs(tmp_path, nx, model, cluster):
    torch = pytest.importorskip("torch")
    deck = small_deck(tmp_path, f"na_{nx}_{model}", nx=nx, model=model)
    e = hw.Engine(deck, cluster=cluster)
    stream = torch.cuda.current_stream().cuda_stream
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
    e.close()


def test_rhs_noalloc_rejects_large_grid(tmp_path):
    torch = pytest.importorskip("torch")
    deck = small_deck(tmp_path, "na_big", nx=8192, model="HS2")
    e = hw.Engine(deck)
    yd = torch.zeros(4 * 8192, dtype=torch.float64, device="cuda")
    dd = torch.zeros_like(yd)
    with pytest.raises(hw.EngineError, match="exceeds"):
        e.rhs_noalloc(0.0, yd.data_ptr(), dd.data_ptr())
    e.close()
