"""Autotuner of the batched ragged runner: per grid size, the slice (grid points per
CTA, i.e. the thread-block-cluster size C = Nx / slice of a member) that gives the
whole ensemble the highest RHS throughput, measured on the device.

    slices, trials = autotune_slices(decks)
    eng = Engine(decks, slices=slices)

The grid-size classes run concurrently and share the GPU, so a class's best shape
depends on the others: the tuner does coordinate descent on the whole ensemble,
starting from the default shape (2048-point slices), changing one class's slice at a
time and keeping a change only when the ensemble's throughput over the same simulated
interval (`warm` windows, then a timed window of `window` output samples) improves.
"""
import time

from .engine import Engine, EngineError, deck_table


def _valid(nx, s):
    c = nx // s
    return 256 <= s <= 2048 and nx % s == 0 and 1 <= c <= 16 and (c & (c - 1)) == 0


def _measure(decks, nxs, slices, window, warm, device, eps_abs, eps_rel):
    eng = Engine(decks, eps_abs=eps_abs, eps_rel=eps_rel, device=device, slices=slices)
    try:
        i_stop = 0
        for _ in range(warm):
            i_stop += window
            eng.run(i_stop, sync=True)
        p0 = sum(eng.stats(m)["rhs_calls"] * nxs[m] for m in range(eng.members))
        t0 = time.perf_counter()
        i_stop += window
        eng.run(i_stop, sync=True)
        dt = time.perf_counter() - t0
        p1 = sum(eng.stats(m)["rhs_calls"] * nxs[m] for m in range(eng.members))
        return (p1 - p0) / max(dt, 1e-12)
    finally:
        eng.close()


def autotune_slices(decks, candidates=(2048, 1024, 512), window=5, warm=2, device=0, eps_abs=1e-8,
                    eps_rel=1e-6, log=None):
    """Returns ({Nx: slice}, [(slices tried, RHS grid points / s), ...])."""
    nxs = [int(deck_table(d, "Nx")[0]) for d in decks]
    classes = sorted(set(nxs), reverse=True)
    cur = {nx: next(s for s in (2048, 1024, 512, 256) if _valid(nx, s)) for nx in classes}
    trials = []
    best = _measure(decks, nxs, dict(cur), window, warm, device, eps_abs, eps_rel)
    trials.append((dict(cur), best))
    if log:
        log(f"autotune start {cur}: {best:.3e} RHS-pt/s")
    for nx in classes:
        for s in candidates:
            if s == cur[nx] or not _valid(nx, s):
                continue
            trial = dict(cur)
            trial[nx] = s
            try:
                v = _measure(decks, nxs, trial, window, warm, device, eps_abs, eps_rel)
            except EngineError:
                continue
            trials.append((dict(trial), v))
            if log:
                log(f"autotune {trial}: {v:.3e} RHS-pt/s")
            if v > best:
                best, cur = v, trial
    return cur, trials
