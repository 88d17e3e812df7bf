"""Sharding one fixed ensemble of independent members over the ranks of a job.

The members of an ensemble never exchange data while they step, so a job of N
GPUs (one process per GPU) splits ONE ensemble into N shards that run with no
collective in the data path, each as its own ragged ensemble on its GPU.  The
split balances the expected device time of the shards:

    cost(member) = Nx log2 Nx          (transforms per RHS grid sweep)
                 x (t_end - t0) * w    (expected steps: the RKF45 step of these
                                        stiff spectral systems scales with the
                                        period of the fastest resolved mode,
                                        w = sqrt(g k_cut tanh(k_cut h)))

and the members are assigned largest first to the least-loaded rank (the LPT
rule, within 4/3 of the optimal makespan).  After the run, one gather of a few
scalars per member (simulated time, RHS calls, accepted / rejected steps,
status, energy) brings the whole ensemble's summary to every rank: a single
collective off the hot loop (NCCL on the GPUs, gloo on the CPU).
"""
import math

import numpy as np

G = 9.80665


def expected_steps(nx, length, depth, t_span, cutfrac=4.0):
    """Relative step count of a member: simulated span times the angular frequency
    of the largest wavenumber its spectral cut-off keeps (k_cut = k_Nyquist /
    cutfrac * 2, the alias mask's edge)."""
    dx = length / (nx - 1)
    k_cut = (math.pi / dx) * 2.0 / cutfrac
    w = math.sqrt(G * k_cut * math.tanh(k_cut * depth))
    return t_span * w


def member_cost(nx, length, depth, t_span, cutfrac=4.0):
    return nx * math.log2(nx) * expected_steps(nx, length, depth, t_span, cutfrac)


def greedy_partition(costs, n_ranks):
    """LPT assignment: members sorted by decreasing cost (ties by index), each to the
    rank with the smallest load so far (ties to the lowest rank).  Returns one
    ascending list of member indices per rank; every rank gets the same answer
    from the same costs, so no communication is needed to agree on it."""
    if n_ranks < 1:
        raise ValueError("n_ranks must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    loads = [0.0] * n_ranks
    shards = [[] for _ in range(n_ranks)]
    for i in order:
        r = min(range(n_ranks), key=lambda q: (loads[q], q))
        shards[r].append(i)
        loads[r] += float(costs[i])
    return [sorted(s) for s in shards]


def shard_loads(costs, shards):
    return [sum(float(costs[i]) for i in s) for s in shards]


def deck_costs(paths, t_span=None):
    """Cost of each deck directory from its set-up tables (host only, no GPU)."""
    from .engine import deck_table
    out = []
    for p in paths:
        nx = int(deck_table(p, "Nx")[0])
        x = deck_table(p, "x")
        depth = float(np.max(deck_table(p, "depth")))
        tt = deck_table(p, "ttrace")
        span = float(tt[-1] - tt[0]) if t_span is None else float(t_span)
        cut = float(deck_table(p, "cutfracwn")[0]) if nx else 4.0
        out.append(member_cost(nx, float(x[-1] - x[0]), depth, span, cut if cut > 0 else 4.0))
    return out


SCALARS = ("t", "rhs_calls", "accepted", "rejected", "status", "energy")


def gather_member_scalars(local_members, local_rows, n_members, device="cpu"):
    """One end-of-run exchange: every rank contributes the rows of the members it ran
    (local_rows[j] = the SCALARS of member local_members[j]) and receives the
    [n_members, len(SCALARS)] table of the whole ensemble, in member order.  Rows
    are placed into a zero table and summed over ranks (one SUM all-reduce, FP64:
    the integer counters stay exact below 2^53)."""
    import torch
    import torch.distributed as dist
    tab = torch.zeros((n_members, len(SCALARS)), dtype=torch.float64, device=device)
    for m, row in zip(local_members, local_rows):
        tab[int(m)] = torch.tensor([float(v) for v in row], dtype=torch.float64, device=device)
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(tab, op=dist.ReduceOp.SUM)
    return tab.cpu().numpy()
