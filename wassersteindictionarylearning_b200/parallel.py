"""Data parallelism over histograms.

Each rank evaluates the objective for its own histograms (`evaluate_both` on
its shard).  Barycenters, losses and weight gradients need no exchange; the
atom part of the gradient and the loss are sums over all histograms, so one
all-reduce of K*N + 1 values per evaluation completes them.  The simplex
projection and the chain rule applied to the atom gradient
(cpp/inverseWasserstein.h:1103-1108, :1125-1128) are linear with the same atoms
on every rank, so they commute with the sum and are applied per rank first.
"""
from __future__ import annotations


def allreduce_atoms_and_loss(g, f, PK: int, dist, group=None):
    """Sum g[PK:] (the atom gradient) and the scalar loss f over ranks in place.

    g, f are torch tensors on the communication device (CPU for gloo, the rank's
    GPU for NCCL); f has one element.  One collective per call.
    """
    import torch
    buf = torch.cat([g[PK:], f.reshape(1)])
    dist.all_reduce(buf, group=group)
    g[PK:].copy_(buf[:-1])
    f.copy_(buf[-1:].reshape(f.shape))
    return g, f
