"""Matvec over several processes, one per GPU, split by right-hand-side
columns.

The reference's only parallelism is OpenMP over cells inside one process
(include/compute.hpp:408); its right-hand sides (nCols) share the tree and
are otherwise independent.  Here every rank builds the same tree on its own
GPU and computes a contiguous block of the columns with the single-GPU entry
point; the blocks are then exchanged with one all-gather, so that every rank
ends with the full ``output``.  The column blocks need no other exchange: no
collective sits on the data path of a matvec.
"""
from __future__ import annotations

import numpy as np

from . import H2_3D_Compute, H2_3D_Tree


def column_blocks(nCols: int, world: int):
    """[(c0, c1)] per rank: contiguous, sizes differing by at most one, the
    larger blocks first."""
    if nCols < 0 or world < 1:
        raise ValueError("need nCols >= 0 and world >= 1")
    base, extra = divmod(nCols, world)
    out, c = [], 0
    for r in range(world):
        n = base + (1 if r < extra else 0)
        out.append((c, c + n))
        c += n
    return out


def H2_3D_Compute_columns(tree: H2_3D_Tree, target, source, weight, nCols: int, output,
                          group=None) -> np.ndarray:
    """``output += K(target, source) @ weight`` (the reference's layouts:
    weight column-major Ns x nCols, output column-major Nf x nCols), with the
    columns split over the ranks of ``group`` (torch.distributed, already
    initialised; every rank passes the same arguments and its own tree).
    gloo exchanges host tensors, nccl device tensors on the tree's GPU."""
    import torch
    import torch.distributed as dist

    rank, world = dist.get_rank(group), dist.get_world_size(group)
    t = np.ascontiguousarray(target, dtype=np.float64).reshape(-1, 3)
    s = t if source is target else np.ascontiguousarray(source, dtype=np.float64).reshape(-1, 3)
    w = np.ascontiguousarray(weight, dtype=np.float64).ravel()
    Nf, Ns = t.shape[0], s.shape[0]
    if w.size != Ns * nCols or output.size != Nf * nCols:
        raise ValueError("weight must hold Ns*nCols and output Nf*nCols values")
    blocks = column_blocks(nCols, world)
    c0, c1 = blocks[rank]
    width = max(b - a for a, b in blocks)
    mine = np.zeros(Nf * width)
    if c1 > c0:
        H2_3D_Compute(tree, t, s, w[c0 * Ns:c1 * Ns], c1 - c0, mine[:Nf * (c1 - c0)])
    dev = "cpu"
    if dist.get_backend(group) == "nccl":
        dev = torch.device("cuda", tree.device)
    local = torch.from_numpy(mine).to(dev)
    parts = [torch.empty_like(local) for _ in range(world)]
    dist.all_gather(parts, local, group=group)
    for r, (a, b) in enumerate(blocks):
        if b > a:
            output[a * Nf:b * Nf] += parts[r][:Nf * (b - a)].cpu().numpy()
    return output
