"""Split one ensemble of independent chains over several GPUs (one process and
one context per GPU) and gather the per-chain trajectory records.

The chains do not interact, so the data path has no collective: every rank
advances its share of the chains, and at the end one all-gather of a few
scalars per chain and trajectory (Delta H, accept, plaquette, ...) gives every
rank the whole ensemble's records.  Each rank's context sets the chains'
Philox stream indices to their positions in the whole ensemble
(``Chmc.set_stream_index``), so a chain draws the same hot start, momenta and
Metropolis uniforms on any number of GPUs.
"""
from __future__ import annotations

from typing import Sequence

RECORD_KEYS = ("delta_h", "accept", "avg_plaquette", "h_old", "h_new", "uniform", "reunit_maxdev")


def chain_cost(dims: Sequence[int], n_steps: int = 1) -> int:
    """Work of one trajectory of a chain, in site-force-evaluations (V x steps)."""
    v = 1
    for d in dims:
        v *= int(d)
    return v * int(n_steps)


def partition(costs: Sequence[float], world: int) -> list[list[int]]:
    """Longest-processing-time split: chains by decreasing cost, each to the rank with
    the least work so far (ties to the lower rank and the lower chain index).  Every
    rank gets the same answer; each rank's list is in ascending chain order."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    loads = [0.0] * world
    parts: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (loads[k], k))
        parts[r].append(i)
        loads[r] += costs[i]
    return [sorted(p) for p in parts]


def imbalance(costs: Sequence[float], parts: Sequence[Sequence[int]]) -> float:
    """max rank load / mean rank load."""
    loads = [sum(costs[i] for i in p) for p in parts]
    mean = sum(loads) / len(loads)
    return max(loads) / mean if mean else 1.0


def gather_records(recs, parts, rank: int, dist, device: str = "cpu"):
    """recs[t][j]: record dict of trajectory t of this rank's j-th chain (parts[rank][j]).
    Returns out[t][c] for every chain c of the ensemble (dicts with RECORD_KEYS) on every
    rank.  One all_gather of a (trajectories x max chains per rank x keys) float64 tensor;
    every rank takes this step with the same shapes."""
    import torch

    nt = len(recs)
    nmax = max(len(p) for p in parts)
    buf = torch.full((nt, nmax, len(RECORD_KEYS)), float("nan"), dtype=torch.float64, device=device)
    for t in range(nt):
        for j in range(len(parts[rank])):
            for k, key in enumerate(RECORD_KEYS):
                buf[t, j, k] = float(recs[t][j][key])
    if dist is None:
        bufs = [buf]
    else:
        bufs = [torch.empty_like(buf) for _ in parts]
        dist.all_gather(bufs, buf)
    n_total = sum(len(p) for p in parts)
    out = [[None] * n_total for _ in range(nt)]
    for r, p in enumerate(parts):
        b = bufs[r].cpu()
        for t in range(nt):
            for j, c in enumerate(p):
                d = {key: float(b[t, j, k]) for k, key in enumerate(RECORD_KEYS)}
                d["accept"] = int(d["accept"])
                out[t][c] = d
    return out
