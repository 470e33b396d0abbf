"""torch.autograd.Function bindings over the C ABI.

KnnDistances: squared distances to the k nearest neighbours, differentiable
with respect to query and point coordinates with the neighbour ids held
fixed (selection is integer-exact and not differentiated).

BarnesHutPlummer: accelerations and potentials of the Plummer-law
Barnes-Hut walk, differentiable with respect to positions and masses
through the same tree walk (decisions held fixed).  With recompute=True
the tree is released after the forward and rebuilt in the backward, so
nothing of the tree is held between the two passes.
"""
from __future__ import annotations

import torch

from ._capi import BH_LAW_PLUMMER, default_bh_params, default_schedule
from .api import Index, knn_backward
from .bh import BarnesHut


class KnnDistances(torch.autograd.Function):
    @staticmethod
    def forward(ctx, queries, points, k: int, schedule=None):
        s = schedule if schedule is not None else default_schedule()
        ix = Index().build(points.detach().contiguous(), s)
        ids, d2 = ix.knn(queries.detach().contiguous(), k, s)
        ctx.save_for_backward(queries, points, ids)
        ctx.mark_non_differentiable(ids)
        return d2, ids

    @staticmethod
    def backward(ctx, g_d2, g_ids):
        queries, points, ids = ctx.saved_tensors
        if g_d2 is None:
            return None, None, None, None
        gq, gp = knn_backward(queries.detach().contiguous(), points.detach().contiguous(), ids,
                              g_d2.contiguous())
        return (gq if ctx.needs_input_grad[0] else None,
                gp if ctx.needs_input_grad[1] else None, None, None)


def knn_distances(queries, points, k: int, schedule=None):
    """(d2 [Q, k], ids [Q, k]); d2 carries gradients to queries and points."""
    return KnnDistances.apply(queries, points, k, schedule)


class BarnesHutPlummer(torch.autograd.Function):
    @staticmethod
    def forward(ctx, pos, mass, theta: float, eps: float, G: float, quadrupole: bool,
                bucket: int, recompute: bool):
        p = default_bh_params(law=BH_LAW_PLUMMER, theta=theta, eps=eps, G=G,
                              quadrupole=int(quadrupole), bucket=bucket)
        bh = BarnesHut().build(pos.detach().contiguous(), mass.detach().contiguous(), p)
        acc, phi = bh.forward(p)
        if recompute:
            bh.release()
        ctx.bh = bh
        ctx.params = p
        ctx.recompute = recompute
        ctx.save_for_backward(pos, mass)
        return acc, phi

    @staticmethod
    def backward(ctx, g_acc, g_phi):
        pos, mass = ctx.saved_tensors
        bh = ctx.bh
        if ctx.recompute:
            bh.build(pos.detach().contiguous(), mass.detach().contiguous(), ctx.params)
        if g_acc is None:
            g_acc = torch.zeros_like(pos)
        g_pos, g_mass = bh.backward(g_acc.contiguous(), g_phi, ctx.params)
        ctx.bh = None
        return g_pos, g_mass, None, None, None, None, None, None


def barnes_hut_plummer(pos, mass, theta: float = 0.5, eps: float = 1e-3, G: float = 1.0,
                       quadrupole: bool = True, bucket: int = 16, recompute: bool = False):
    """(acc [N, 3], phi [N]) with gradients to pos and mass."""
    return BarnesHutPlummer.apply(pos, mass, theta, eps, G, quadrupole, bucket, recompute)
