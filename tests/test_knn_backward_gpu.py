"""kNN distance backward against a plain PyTorch fp32 reference (indices
held fixed)."""
import numpy as np
import pytest
import torch

from rtdsl import workloads

pytestmark = pytest.mark.gpu


def test_knn_backward_matches_torch(rtd, cuda):
    pts, q = workloads.clustered(n=20_000, nq=3_000, seed=31, n_clusters=8, box=4.0)
    P = torch.from_numpy(pts).cuda()
    Q = torch.from_numpy(q).cuda()
    s = rtd.default_schedule()
    ix = rtd.Index().build(P, s)
    ids, d2 = ix.knn(Q, 7, s)
    g = torch.rand_like(d2)
    gq, gp = rtd.knn_backward(Q, P, ids, g)
    # torch reference
    Pr = P.clone().requires_grad_(True)
    Qr = Q.clone().requires_grad_(True)
    nb = Pr[ids.long()]
    d2r = ((Qr[:, None, :] - nb) ** 2).sum(-1)
    torch.testing.assert_close(d2r.detach(), d2, rtol=1e-5, atol=1e-6)
    (d2r * g).sum().backward()
    torch.testing.assert_close(gq, Qr.grad, rtol=1e-4, atol=1e-5)
    torch.testing.assert_close(gp, Pr.grad, rtol=1e-4, atol=1e-5)


def test_knn_backward_skips_empty_slots(rtd, cuda):
    P = torch.rand((3, 3), device="cuda")
    Q = torch.rand((10, 3), device="cuda")
    s = rtd.default_schedule()
    ids, d2 = rtd.Index().build(P, s).knn(Q, 5, s)
    g = torch.ones_like(d2)
    gq, gp = rtd.knn_backward(Q, P, ids, g)
    exp = 2.0 * (Q[:, None, :] - P[None, :, :]).sum(1)
    torch.testing.assert_close(gq, exp, rtol=1e-5, atol=1e-5)
    assert torch.isfinite(gp).all()


@pytest.mark.parametrize("k", [1, 5, 40, 300])
def test_knn_distances_autograd_function(rtd, cuda, k):
    """The torch.autograd.Function (rtdsl.torch_ops.knn_distances) through
    torch.autograd.grad: forward distances and gradients w.r.t. queries and
    points equal a plain PyTorch fp32 reference over the same (fixed) ids,
    for the loss sum_q mean_j w_qj * d2_qj; the ids are not differentiable.
    Tolerance: rtol 1e-4, atol 1e-5 (fp32 sums in another order)."""
    from rtdsl.torch_ops import knn_distances
    pts, q = workloads.clustered(n=12_000, nq=2_000, seed=33, n_clusters=6, box=3.0)
    P = torch.from_numpy(pts).cuda().requires_grad_(True)
    Q = torch.from_numpy(q).cuda().requires_grad_(True)
    w = torch.rand((len(q), k), device="cuda")
    d2, ids = knn_distances(Q, P, k)
    assert not ids.requires_grad and d2.requires_grad
    loss = (w * d2).mean(dim=1).sum()
    gq, gp = torch.autograd.grad(loss, (Q, P))
    # reference: the same loss over the same ids in plain PyTorch
    Pr = P.detach().clone().requires_grad_(True)
    Qr = Q.detach().clone().requires_grad_(True)
    d2r = ((Qr[:, None, :] - Pr[ids.long()]) ** 2).sum(-1)
    torch.testing.assert_close(d2.detach(), d2r.detach(), rtol=1e-5, atol=1e-6)
    gqr, gpr = torch.autograd.grad((w * d2r).mean(dim=1).sum(), (Qr, Pr))
    torch.testing.assert_close(gq, gqr, rtol=1e-4, atol=1e-5)
    torch.testing.assert_close(gp, gpr, rtol=1e-4, atol=1e-5)
    # only one input needing a gradient
    d2b, _ = knn_distances(Q.detach(), P, k)
    (gp_only,) = torch.autograd.grad((w * d2b).mean(dim=1).sum(), (P,))
    torch.testing.assert_close(gp_only, gpr, rtol=1e-4, atol=1e-5)
