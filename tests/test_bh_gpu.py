"""Barnes-Hut parity.

Reference law: the GPU tree must equal the CPU restatement of
BarnesHutTree::build node for node (bitwise), and the walk's forces must be
bit-identical to the restated reference walk.

Plummer law (monopole + quadrupole, group MAC): forces / potentials against
an FP64 evaluation with the same decisions, against the FP64 direct sum,
and the adjoint against FP64 central differences (decisions frozen) and the
FP64 direct-sum gradient.
"""
import os

import numpy as np
import pytest
import torch

from conftest import GOLDEN
from rtdsl import workloads

pytestmark = pytest.mark.gpu


def gpu_tree(pos, mass, **kw):
    from rtdsl.bh import BarnesHut
    from rtdsl._capi import default_bh_params
    p = default_bh_params(**kw)
    bh = BarnesHut().build(torch.from_numpy(pos).cuda(), torch.from_numpy(mass).cuda(), p)
    return bh, p


def assert_tree_equal(orc_nodes, orc_order, nodes, order):
    assert len(nodes) == len(orc_nodes), (len(nodes), len(orc_nodes))
    np.testing.assert_array_equal(order, orc_order)
    for f in ("is_leaf", "next_idx", "autorope", "bucket_start", "num_particles"):
        np.testing.assert_array_equal(nodes[f], orc_nodes[f], err_msg=f)
    for f in ("com", "mass", "width"):
        np.testing.assert_array_equal(nodes[f].view(np.uint32), orc_nodes[f].view(np.uint32), err_msg=f)


def cases():
    g = np.load(os.path.join(GOLDEN, "bh_physics.npz"))
    rng = np.random.default_rng(8)
    out = [("physics2000", g["pos"], g["mass"], 128)]
    p, m = workloads.plummer(20_000, seed=3)
    out.append(("plummer20k_b128", p, m, 128))
    out.append(("plummer20k_b16", p, m, 16))
    c, _ = workloads.clustered(n=30_000, nq=10, seed=4, n_clusters=5, box=3.0)
    out.append(("clustered30k_b32", c, rng.uniform(0.5, 1.5, len(c)).astype(np.float32), 32))
    dup = np.repeat(rng.random((40, 3)).astype(np.float32), 50, axis=0)   # width-stop leaves
    out.append(("duplicates2000_b8", dup, np.ones(len(dup), np.float32), 8))
    out.append(("tiny1", np.array([[1., 2., 3.]], np.float32), np.ones(1, np.float32), 128))
    t = rng.random((129, 3)).astype(np.float32)
    out.append(("n129", t, np.ones(129, np.float32), 128))
    out.append(("n128", t[:128], np.ones(128, np.float32), 128))
    return out


@pytest.mark.parametrize("case", cases(), ids=lambda c: c[0])
def test_reference_tree_and_forces_bitwise(orc, cuda, case):
    name, pos, mass, bucket = case
    pos = np.ascontiguousarray(pos, dtype=np.float32)
    mass = np.ascontiguousarray(mass, dtype=np.float32)
    on, oo, _ = orc.bh_build(pos, mass, bucket=bucket)
    bh, p = gpu_tree(pos, mass, bucket=bucket)
    nodes, order = bh.export()
    assert_tree_equal(on, oo, nodes, order)
    for theta in (0.5, 0.0, 1.2):
        p.theta = theta
        f, _ = bh.forward(p)
        torch.cuda.synchronize()
        of = orc.bh_ref_forces(pos, mass, on, oo, theta)
        np.testing.assert_array_equal(f.cpu().numpy().view(np.uint32), of.view(np.uint32))


@pytest.mark.slow
@pytest.mark.parametrize("bucket", [128, 32])
def test_reference_tree_and_forces_1m_bitwise(orc, cuda, bucket):
    """The 1M-body Plummer sphere (the Barnes-Hut workload's bodies) with the
    reference law: the GPU tree node for node against the restated
    BarnesHutTree::build, and the forces of 4,096 sampled bodies bit for bit
    against the restated reference walk at theta 0.5."""
    pos, mass = workloads.plummer(1_000_000, seed=7)
    on, oo, _ = orc.bh_build(pos, mass, bucket=bucket)
    bh, p = gpu_tree(pos, mass, bucket=bucket)
    nodes, order = bh.export()
    assert_tree_equal(on, oo, nodes, order)
    p.theta = 0.5
    f, _ = bh.forward(p)
    f = f.cpu().numpy()
    sel = np.sort(np.random.default_rng(bucket).choice(len(pos), 4096, replace=False))
    of = orc.bh_ref_forces_at(pos, mass, on, oo, sel, 0.5)
    np.testing.assert_array_equal(f[sel].view(np.uint32), of.view(np.uint32))


def test_host_barnes_hut_physics_check(orc, cuda):
    """barnes_hut!(bodies, 0.5, G, out) on verify_physics.py's data: the sum
    of force magnitudes within 2% of the FP64 direct sum (verify_physics.py:45)
    and within 1e-5 of the restated reference walk."""
    from rtdsl.bh import barnes_hut
    g = np.load(os.path.join(GOLDEN, "bh_physics.npz"))
    bodies = np.concatenate([g["pos"], g["mass"][:, None]], axis=1)
    f = barnes_hut(bodies, 0.5, 6.674e-11)
    mag = np.sum(np.linalg.norm(f.astype(np.float64), axis=1))
    assert abs(mag - float(g["mag_sum"])) / float(g["mag_sum"]) < 0.02
    on, oo, _ = orc.bh_build(g["pos"], g["mass"])
    of = orc.bh_ref_forces(g["pos"], g["mass"], on, oo, 0.5)
    rel = np.linalg.norm(f - of) / np.linalg.norm(of)
    assert rel <= 1e-5


def test_reference_law_vs_fp64_direct(orc, cuda):
    pos, mass = workloads.plummer(50_000, seed=11)
    bh, p = gpu_tree(pos, mass)
    f, _ = bh.forward(p)
    f = f.cpu().numpy().astype(np.float64)
    tg = np.random.default_rng(0).choice(len(pos), 512, replace=False)
    ref = orc.direct_ref_f64(pos, mass, tg)
    err = np.linalg.norm(f[tg] - ref, axis=1) / np.linalg.norm(ref, axis=1)
    assert np.median(err) < 5e-2   # BH approximation error at theta = 0.5, monopole


def test_plummer_forward_matches_frozen_fp64(orc, cuda):
    pos, mass = workloads.plummer(16_384, seed=7)
    for quad in (1, 0):
        bh, p = gpu_tree(pos, mass, law=1, theta=0.5, eps=1e-3, G=1.0, bucket=16, quadrupole=quad)
        acc, phi = bh.forward(p)
        frozen = orc.PlummerFrozen(pos, mass, theta=0.5, bucket=16)
        L, ophi, oacc = frozen.eval(pos, mass, eps=1e-3, G=1.0, quad=bool(quad))
        a = acc.cpu().numpy().astype(np.float64)
        ph = phi.cpu().numpy().astype(np.float64)
        rel_a = np.linalg.norm(a - oacc) / np.linalg.norm(oacc)
        rel_p = np.linalg.norm(ph - ophi) / np.linalg.norm(ophi)
        assert rel_a < 2e-5 and rel_p < 2e-5, (quad, rel_a, rel_p)


def test_plummer_theta0_is_direct_sum(orc, cuda):
    pos, mass = workloads.plummer(4_096, seed=5)
    bh, p = gpu_tree(pos, mass, law=1, theta=0.0, eps=1e-2, G=1.0, bucket=16)
    acc, phi = bh.forward(p)
    L, dphi, dacc = orc.direct_plummer_f64(pos, mass, eps=1e-2, G=1.0)
    np.testing.assert_allclose(acc.cpu().numpy(), dacc, rtol=1e-4, atol=1e-4 * np.abs(dacc).max())
    np.testing.assert_allclose(phi.cpu().numpy(), dphi, rtol=1e-5, atol=1e-6 * np.abs(dphi).max())


def test_plummer_accuracy_vs_direct_sum(orc, cuda):
    pos, mass = workloads.plummer(16_384, seed=7)
    bh, p = gpu_tree(pos, mass, law=1, theta=0.5, eps=1e-3, G=1.0, bucket=16)
    acc, phi = bh.forward(p)
    L, dphi, dacc = orc.direct_plummer_f64(pos, mass, eps=1e-3, G=1.0)
    a = acc.cpu().numpy().astype(np.float64)
    err = np.linalg.norm(a - dacc, axis=1) / np.linalg.norm(dacc, axis=1)
    assert np.median(err) < 1e-3 and np.percentile(err, 99) < 1e-2
    perr = np.abs(phi.cpu().numpy() - dphi) / np.abs(dphi)
    assert np.median(perr) < 1e-4


def _loss_grads(bh, p, pos_t, mass_t):
    acc, phi = bh.forward(p)
    g_pos, g_mass = bh.backward(acc, torch.ones_like(phi), p)
    torch.cuda.synchronize()
    return acc, phi, g_pos.cpu().numpy().astype(np.float64), g_mass.cpu().numpy().astype(np.float64)


@pytest.mark.parametrize("quad", [1, 0])
def test_plummer_adjoint_vs_frozen_fd(orc, cuda, quad):
    """Central differences (h = 1e-4) of the FP64 frozen-decision loss
    L = sum(phi) + 0.5 sum|a|^2 on 32 sampled coordinates and 16 masses."""
    n = 16_384
    pos, mass = workloads.plummer(n, seed=7)
    bh, p = gpu_tree(pos, mass, law=1, theta=0.5, eps=1e-3, G=1.0, bucket=16, quadrupole=quad)
    _, _, gp, gm = _loss_grads(bh, p, None, None)
    frozen = orc.PlummerFrozen(pos, mass, theta=0.5, bucket=16)
    rng = np.random.default_rng(1)
    h = 1e-4
    p64 = pos.astype(np.float64)
    m64 = mass.astype(np.float64)
    errs = []
    for idx in rng.choice(n * 3, 32, replace=False):
        b, a = divmod(int(idx), 3)
        pp = p64.copy(); pp[b, a] += h
        pm = p64.copy(); pm[b, a] -= h
        fd = (frozen.eval(pp, m64, 1e-3, 1.0, bool(quad))[0] -
              frozen.eval(pm, m64, 1e-3, 1.0, bool(quad))[0]) / (2 * h)
        errs.append(abs(fd - gp[b, a]) / max(abs(fd), 1e-3 * np.abs(gp).max()))
    for b in rng.choice(n, 16, replace=False):
        hm = 1e-4 * m64[b]
        mp = m64.copy(); mp[b] += hm
        mm = m64.copy(); mm[b] -= hm
        fd = (frozen.eval(p64, mp, 1e-3, 1.0, bool(quad))[0] -
              frozen.eval(p64, mm, 1e-3, 1.0, bool(quad))[0]) / (2 * hm)
        errs.append(abs(fd - gm[b]) / max(abs(fd), 1e-3 * np.abs(gm).max()))
    errs = np.array(errs)
    assert np.median(errs) < 1e-3 and errs.max() < 2e-2, errs


def test_plummer_adjoint_vs_direct_sum_gradient(orc, cuda):
    """GPU BH adjoint vs the FP64 direct-sum gradient at N = 16,384: they
    differ by the BH approximation (theta 0.5, quadrupole)."""
    n = 16_384
    pos, mass = workloads.plummer(n, seed=9)
    bh, p = gpu_tree(pos, mass, law=1, theta=0.5, eps=1e-3, G=1.0, bucket=16)
    _, _, gp, gm = _loss_grads(bh, p, None, None)
    L, phi, acc, dgp, dgm = orc.direct_plummer_f64(pos, mass, 1e-3, 1.0, grad=True)
    rel_p = np.linalg.norm(gp - dgp) / np.linalg.norm(dgp)
    rel_m = np.linalg.norm(gm - dgm) / np.linalg.norm(dgm)
    assert rel_p < 2e-2 and rel_m < 1e-2, (rel_p, rel_m)


def test_autograd_function_matches_backward(orc, cuda):
    from rtdsl.torch_ops import barnes_hut_plummer
    pos, mass = workloads.plummer(8_192, seed=2)
    P = torch.from_numpy(pos).cuda().requires_grad_(True)
    M = torch.from_numpy(mass).cuda().requires_grad_(True)
    for recompute in (False, True):
        acc, phi = barnes_hut_plummer(P, M, theta=0.5, eps=1e-3, G=1.0, bucket=16,
                                      recompute=recompute)
        L = phi.sum() + 0.5 * (acc ** 2).sum()
        gP, gM = torch.autograd.grad(L, (P, M))
        bh, p = gpu_tree(pos, mass, law=1, theta=0.5, eps=1e-3, G=1.0, bucket=16)
        _, _, gp, gm = _loss_grads(bh, p, None, None)
        np.testing.assert_allclose(gP.cpu().numpy(), gp, rtol=1e-4, atol=1e-6 * np.abs(gp).max())
        np.testing.assert_allclose(gM.cpu().numpy(), gm, rtol=1e-4, atol=1e-6 * np.abs(gm).max())


def test_bh_errors_and_empty(cuda):
    from rtdsl import RtdError
    from rtdsl.bh import BarnesHut
    from rtdsl._capi import default_bh_params
    bh = BarnesHut().build(torch.zeros((0, 3), device="cuda"), torch.zeros((0,), device="cuda"))
    f, _ = bh.forward()
    assert f.shape == (0, 3)
    bh2 = BarnesHut().build(torch.rand((100, 3), device="cuda"), torch.rand(100, device="cuda"))
    with pytest.raises(RtdError):
        bh2.backward(torch.zeros((100, 3), device="cuda"), None, default_bh_params(law=0))


def test_plummer_interaction_counts(cuda):
    """The walk's interaction counts: at theta = 0 no cell is accepted and
    every body meets all n bodies; at theta = 0.5 the counts equal an FP32
    numpy walk of the exported tree with the same per-body MAC
    (width^2 < theta^2 |COM - x|^2, each operation rounded)."""
    pos, mass = workloads.plummer(6_000, seed=4)
    bh, p = gpu_tree(pos, mass, law=1, theta=0.5, eps=1e-3, G=1.0, bucket=16)
    c0 = bh.interaction_counts(0.0, stride=1)
    assert c0["sampled"] == 6000 and c0["cells_per_body"] == 0 and c0["bodies_per_body"] == 6000
    stride = 97
    c = bh.interaction_counts(0.5, stride=stride)
    nodes, order = bh.export()
    fpos = pos[order].astype(np.float32)
    th2 = np.float32(0.25)
    cells = bodies = 0
    for i in range(0, len(fpos), stride):
        x = fpos[i]
        q = 0
        while q < len(nodes):
            nd = nodes[q]
            d = (nd["com"].astype(np.float32) - x).astype(np.float32)
            d2 = np.float32(np.float32(np.float32(d[0] * d[0]) + np.float32(d[1] * d[1])) + np.float32(d[2] * d[2]))
            w = np.float32(nd["width"])
            if np.float32(w * w) < np.float32(th2 * d2):
                cells += 1
                q = int(nd["autorope"])
            else:
                if nd["is_leaf"]:
                    bodies += int(nd["num_particles"])
                q += 1
    ns = (len(fpos) + stride - 1) // stride
    assert c["sampled"] == ns
    assert round(c["cells_per_body"] * ns) == cells and round(c["bodies_per_body"] * ns) == bodies


def test_leapfrog_matches_fp64_direct_sum(orc, cuda):
    """theta = 0 makes every interaction direct, so a few leapfrog steps must
    follow an FP64 leapfrog driven by the FP64 direct sum (FP32 rounding)."""
    from rtdsl.bh import BarnesHut
    from rtdsl._capi import default_bh_params
    pos, mass = workloads.plummer(2_000, seed=12)
    rng = np.random.default_rng(1)
    vel = (rng.normal(size=pos.shape) * 0.3).astype(np.float32)
    p = default_bh_params(law=1, theta=0.0, eps=0.05, G=1.0, bucket=16)
    P = torch.from_numpy(pos).cuda()
    V = torch.from_numpy(vel).cuda()
    M = torch.from_numpy(mass).cuda()
    dt, steps = 1e-3, 5
    BarnesHut().leapfrog(P, V, M, dt, steps, p)
    x = pos.astype(np.float64)
    v = vel.astype(np.float64)
    m = mass.astype(np.float64)
    a = orc.direct_plummer_f64(x, m, 0.05, 1.0)[2]
    for _ in range(steps):
        v += 0.5 * dt * a
        x += dt * v
        a = orc.direct_plummer_f64(x, m, 0.05, 1.0)[2]
        v += 0.5 * dt * a
    np.testing.assert_allclose(P.cpu().numpy(), x, rtol=2e-6, atol=2e-5)
    np.testing.assert_allclose(V.cpu().numpy(), v, rtol=0, atol=2e-4 * np.abs(v).max())


def test_leapfrog_energy_and_chaining(orc, cuda):
    """Energy of a Plummer sphere in virial equilibrium is conserved to
    1e-3 over 40 steps at theta 0.5, and two calls of 20 steps chained
    through the returned accelerations equal one call of 40."""
    from rtdsl.bh import BarnesHut
    from rtdsl._capi import default_bh_params
    n = 8_192
    pos, mass = workloads.plummer(n, seed=5)
    r = np.linalg.norm(pos.astype(np.float64), axis=1)
    rng = np.random.default_rng(2)
    # isotropic velocities with the local Plummer dispersion sigma^2 = 1/(6 sqrt(1+r^2))
    sig = np.sqrt(1.0 / (6.0 * np.sqrt(1.0 + r * r)))
    vel = (rng.normal(size=pos.shape) * sig[:, None]).astype(np.float32)
    p = default_bh_params(law=1, theta=0.5, eps=0.01, G=1.0, bucket=16)

    def energy(P, V, M):
        x = P.cpu().numpy().astype(np.float64)
        v = V.cpu().numpy().astype(np.float64)
        m = M.cpu().numpy().astype(np.float64)
        _, phi, _ = orc.direct_plummer_f64(x, m, 0.01, 1.0)
        return 0.5 * np.sum(m * np.sum(v * v, axis=1)) + 0.5 * np.sum(m * phi)

    M = torch.from_numpy(mass).cuda()
    P1, V1 = torch.from_numpy(pos).cuda(), torch.from_numpy(vel).cuda()
    e0 = energy(P1, V1, M)
    bh = BarnesHut()
    acc = bh.leapfrog(P1, V1, M, 2e-3, 20, p)
    bh.leapfrog(P1, V1, M, 2e-3, 20, p, acc=acc)
    e1 = energy(P1, V1, M)
    assert abs(e1 - e0) / abs(e0) < 1e-3, (e0, e1)
    P2, V2 = torch.from_numpy(pos).cuda(), torch.from_numpy(vel).cuda()
    BarnesHut().leapfrog(P2, V2, M, 2e-3, 40, p)
    assert torch.equal(P1, P2) and torch.equal(V1, V2)


@pytest.mark.parametrize("quad", [True, False])
def test_plummer_adjoint_replays_the_forward_log(cuda, quad):
    """After a first backward, forwards record their interaction tiles and
    the next backward replays them instead of walking: the gradients equal
    the walking adjoint's (first iteration) up to the order of the FP32
    atomic sums over warps (relative norm difference below 1e-5, which the
    walking adjoint shows between two runs too).  With another theta the
    handle's gradients equal a fresh handle's to the same tolerance."""
    pos, mass = workloads.plummer(60_000, seed=12)
    bh, p = gpu_tree(pos, mass, law=1, theta=0.5, eps=1e-3, G=1.0, bucket=16,
                     quadrupole=int(quad))
    ones = torch.ones((len(pos),), device="cuda")
    outs = []
    for it in range(4):
        acc, _ = bh.forward(p)
        gp, gm = bh.backward(acc, ones, p)
        outs.append((gp.cpu().numpy(), gm.cpu().numpy()))
        info = bh.info()
        if it == 0:
            assert info["log_pages"] == 0          # no backward had run before this forward
        if it >= 2:
            assert info["log_pages"] > 0           # the pool was sized by the forward before
    rel = lambda a, b: float(np.linalg.norm((a - b).astype(np.float64)) /   # noqa: E731
                             np.linalg.norm(b.astype(np.float64)))
    for gp, gm in outs[1:]:
        assert rel(gp, outs[0][0]) < 1e-5 and rel(gm, outs[0][1]) < 1e-5
    # another theta
    p2 = type(p).from_buffer_copy(p)
    p2.theta = 0.7
    gp_w, _ = bh.backward(bh.forward(p2)[0], ones, p2)
    fresh, _ = gpu_tree(pos, mass, law=1, theta=0.7, eps=1e-3, G=1.0, bucket=16,
                        quadrupole=int(quad))
    gp_f, _ = fresh.backward(fresh.forward(p2)[0], ones, p2)
    assert rel(gp_w.cpu().numpy(), gp_f.cpu().numpy()) < 1e-5
