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
