"""GPU tests of the batched multi-system solver (kq_batch_*): systems of different lattices, gauge fields, masses
and shift sets solved in one set of persistent launches; every system checked against the oracle and against the
single-system solver."""
import numpy as np
import pytest
import torch

import kuqcd_b200 as K
from oracle import oracle as O

SYSTEMS = [  # dims, eps, mass, shifts, parity, seed
    ((4, 4, 4, 4), 0.2, 0.1, 8, 0, 11),
    ((6, 6, 6, 6), 0.35, 0.03, 12, 1, 12),
    ((8, 4, 4, 8), 0.4, 0.05, 16, 0, 13),
    ((4, 4, 4, 1), 0.3, 0.07, 3, 1, 14),
]


def build(dims, eps, seed, parity):
    fat, lng = O.make_links(dims, eps, seed)
    ctx = K.Context(dims)
    ctx.load_links(K.KUQCD_FAT_LINK, fat)
    ctx.load_links(K.KUQCD_LONG_LINK, lng)
    b = O.make_source(dims, parity, seed)
    vb = ctx.spinor_bytes(K.KUQCD_DOUBLE)
    d_b = torch.zeros(vb, dtype=torch.uint8, device="cuda")
    ctx.upload(K.KUQCD_DOUBLE, b, d_b)
    return ctx, fat, lng, b, d_b, vb


@pytest.mark.gpu
@pytest.mark.parametrize("solver,prec", [(K.KQ_SOLVER_MIXED, K.KUQCD_HALF), (K.KQ_SOLVER_MIXED, K.KUQCD_SINGLE),
                                         (K.KQ_SOLVER_CGM_WINDOWED, K.KUQCD_DOUBLE)])
def test_batch_solves_every_system(cuda, tmp_path, monkeypatch, solver, prec):
    monkeypatch.setenv("KUQCD_TUNE_CACHE", str(tmp_path / "tune.txt"))
    batch = K.Batch()
    keep = []
    for dims, eps, mass, ns, parity, seed in SYSTEMS:
        ctx, fat, lng, b, d_b, vb = build(dims, eps, seed, parity)
        sig = list(mass * mass + np.logspace(-4, 0, ns))
        d_x = torch.zeros(vb * ns, dtype=torch.uint8, device="cuda")
        tol = (1e-10) ** 2 * float(b @ b)
        batch.add(ctx, d_b, d_x, sig, parity=parity, solver=solver, prec=prec, rel_residual=1e-10, tol=tol)
        keep.append((ctx, fat, lng, b, d_x, vb, sig, parity, dims))
    info = batch.solve()
    # the first solve of a signature measures the launch shape (unless this process already tuned it)
    assert info.num_systems == len(SYSTEMS) and info.tile in (128, 256) and info.ctas_per_sm >= 1
    for i, (ctx, fat, lng, b, d_x, vb, sig, parity, dims) in enumerate(keep):
        si = batch.system_info(i)
        assert si.status == 0, i
        for k, s in enumerate(sig):
            xk = ctx.download(K.KUQCD_DOUBLE, d_x[k * vb:(k + 1) * vb])
            r = O.true_residual(dims, fat, lng, parity, s, b, xk)
            assert r <= (1.2e-10 if solver == K.KQ_SOLVER_MIXED else 1.5e-10), (i, k, r)
    # same batch again: the launch shape now comes from the cache
    info2 = batch.solve()
    assert info2.tuned_now == 0 and info2.tile == info.tile and info2.ctas_per_sm == info.ctas_per_sm
    batch.close()


@pytest.mark.gpu
def test_batch_matches_single_system_solver(cuda, tmp_path, monkeypatch):
    """KQ_SOLVER_CGM_WINDOWED in a batch runs the same recurrences as the single-system solver: same iteration
    count, same solutions up to reduction order."""
    monkeypatch.setenv("KUQCD_TUNE_CACHE", str(tmp_path / "tune.txt"))
    dims, eps, mass, ns, parity, seed = SYSTEMS[1]
    ctx, fat, lng, b, d_b, vb = build(dims, eps, seed, parity)
    sig = list(mass * mass + np.logspace(-4, 0, ns))
    tol = (1e-10) ** 2 * float(b @ b)
    xs, single = ctx.solve(b, sig, parity=parity, solver=K.KQ_SOLVER_CGM_WINDOWED, tol=tol)
    # a second, smaller system shares the launches
    ctx2, _, _, b2, d_b2, vb2 = build((4, 4, 4, 4), 0.3, 99, 0)
    batch = K.Batch()
    d_x = torch.zeros(vb * ns, dtype=torch.uint8, device="cuda")
    d_x2 = torch.zeros(vb2 * 4, dtype=torch.uint8, device="cuda")
    batch.add(ctx, d_b, d_x, sig, parity=parity, solver=K.KQ_SOLVER_CGM_WINDOWED, tol=tol)
    batch.add(ctx2, d_b2, d_x2, [0.01, 0.1, 0.5, 1.0], solver=K.KQ_SOLVER_CGM_WINDOWED,
              tol=(1e-10) ** 2 * float(b2 @ b2))
    batch.solve()
    assert abs(batch.system_info(0).iter - single.iter) <= 1
    for k in range(ns):
        xb = ctx.download(K.KUQCD_DOUBLE, d_x[k * vb:(k + 1) * vb])
        assert np.abs(xb - xs[k]).max() <= 1e-9 * np.abs(xs[k]).max(), k
    batch.close()


@pytest.mark.gpu
def test_batch_argument_checks(cuda):
    batch = K.Batch()
    with pytest.raises(K.KuQCDError):
        batch.solve()  # empty
    ctx = K.Context((4, 4, 4, 4))  # no links
    d = torch.zeros(16, dtype=torch.uint8, device="cuda")
    with pytest.raises(K.KuQCDError):
        batch.add(ctx, d, d, [0.1])
    batch.close()


@pytest.mark.gpu
@pytest.mark.parametrize("large_sites,threads", [(256, 2), (1, 1), (1, 3)])
def test_batch_with_large_systems_on_the_single_system_solver(cuda, tmp_path, monkeypatch, large_sites, threads):
    """Systems of at least KUQCD_BATCH_LARGE_SITES sites per parity go through the single-system solver, on
    KUQCD_BATCH_LARGE_THREADS host threads at once, while the rest are batched (256: two of each kind, overlapping on
    the GPU; 1: every system on its own); each system still reaches its target and reports its own status and
    iterations."""
    monkeypatch.setenv("KUQCD_TUNE_CACHE", str(tmp_path / "tune.txt"))
    monkeypatch.setenv("KUQCD_BATCH_LARGE_SITES", str(large_sites))
    monkeypatch.setenv("KUQCD_BATCH_LARGE_THREADS", str(threads))
    batch = K.Batch()
    keep = []
    for dims, eps, mass, ns, parity, seed in SYSTEMS:
        ctx, fat, lng, b, d_b, vb = build(dims, eps, seed, parity)
        sig = list(mass * mass + np.logspace(-4, 0, ns))
        d_x = torch.zeros(vb * ns, dtype=torch.uint8, device="cuda")
        batch.add(ctx, d_b, d_x, sig, parity=parity, solver=K.KQ_SOLVER_MIXED, prec=K.KUQCD_HALF,
                  rel_residual=1e-10, tol=(1e-10) ** 2 * float(b @ b))
        keep.append((ctx, fat, lng, b, d_x, vb, sig, parity, dims))
    info = batch.solve()
    assert info.num_systems == len(SYSTEMS) and info.iterations > 0
    for i, (ctx, fat, lng, b, d_x, vb, sig, parity, dims) in enumerate(keep):
        si = batch.system_info(i)
        assert si.status == 0 and si.iter > 0, i
        for k, s in enumerate(sig):
            xk = ctx.download(K.KUQCD_DOUBLE, d_x[k * vb:(k + 1) * vb])
            r = O.true_residual(dims, fat, lng, parity, s, b, xk)
            assert r <= 1.2e-10, (i, k, r)
    batch.close()


def sources_on_one_field(dims, eps, seed, n, parity=0):
    """n systems on one gauge field: own Gaussian source and own mass each (one context, so the batch groups them
    and its dslash loads every link once for all members)."""
    fat, lng = O.make_links(dims, eps, seed)
    ctx = K.Context(dims)
    ctx.load_links(K.KUQCD_FAT_LINK, fat)
    ctx.load_links(K.KUQCD_LONG_LINK, lng)
    vb = ctx.spinor_bytes(K.KUQCD_DOUBLE)
    rng = np.random.default_rng(seed)
    out = []
    for j in range(n):
        b = O.make_source(dims, parity, seed * 100 + j)
        d_b = torch.zeros(vb, dtype=torch.uint8, device="cuda")
        ctx.upload(K.KUQCD_DOUBLE, b, d_b)
        mass = float(rng.uniform(0.01, 0.1))
        ns = int(rng.integers(4, 13))
        out.append((b, d_b, list(mass * mass + np.logspace(-4, 0, ns))))
    return ctx, fat, lng, vb, out


@pytest.mark.gpu
@pytest.mark.parametrize("solver,prec", [(K.KQ_SOLVER_MIXED, K.KUQCD_HALF),
                                         (K.KQ_SOLVER_CGM_WINDOWED, K.KUQCD_DOUBLE)])
def test_batch_many_sources_on_one_field_match_single_system(cuda, tmp_path, monkeypatch, solver, prec):
    """8 sources (own masses and shift sets) on one 16^4 gauge field, batched with the grouped multi-RHS dslash,
    against the single-system solver on each: solutions within 1e-9, true residuals within target; the tuner
    searched the right-hand sides per CTA and the sites per thread."""
    monkeypatch.setenv("KUQCD_TUNE_CACHE", str(tmp_path / "tune.txt"))
    dims = (16, 16, 16, 16)
    ctx, fat, lng, vb, systems = sources_on_one_field(dims, 0.3, 21, 8)
    batch = K.Batch()
    xs = []
    for b, d_b, sig in systems:
        d_x = torch.zeros(vb * len(sig), dtype=torch.uint8, device="cuda")
        batch.add(ctx, d_b, d_x, sig, solver=solver, prec=prec, rel_residual=1e-10,
                  tol=(1e-10) ** 2 * float(b @ b))
        xs.append(d_x)
    info = batch.solve()
    assert info.num_systems == 8 and info.rhs_per_cta in (1, 2, 4, 8) and info.sites_per_thread in (1, 2)
    assert info.groups == (8 + info.rhs_per_cta - 1) // info.rhs_per_cta
    for j, (b, d_b, sig) in enumerate(systems):
        assert batch.system_info(j).status == 0, j
        ref, single = ctx.solve(b, sig, parity=0, solver=solver, prec=prec, rel_residual=1e-10,
                                tol=(1e-10) ** 2 * float(b @ b))
        if solver == K.KQ_SOLVER_CGM_WINDOWED:
            assert abs(batch.system_info(j).iter - single.iter) <= 1, j
        for k, s in enumerate(sig):
            xb = ctx.download(K.KUQCD_DOUBLE, xs[j][k * vb:(k + 1) * vb])
            r = O.true_residual(dims, fat, lng, 0, s, b, xb)
            assert r <= (1.2e-10 if solver == K.KQ_SOLVER_MIXED else 1.5e-10), (j, k, r)
            assert np.abs(xb - ref[k]).max() <= 1e-9 * np.abs(ref[k]).max(), (j, k)
    # the tuned shape, whichever FP64 pass mode it has, comes back from the cache
    info2 = batch.solve()
    assert info2.tuned_now == 0
    assert (info2.rhs_per_cta, info2.sites_per_thread, info2.fp64_rhs_per_pass) == \
        (info.rhs_per_cta, info.sites_per_thread, info.fp64_rhs_per_pass)
    batch.close()


@pytest.mark.gpu
@pytest.mark.parametrize("rhs,spt,p64", [(1, 1, 1), (2, 2, 2), (4, 1, 4), (4, 2, 1), (8, 2, 2), (8, 1, 4),
                                         (2, 1, 0), (4, 2, 0), (8, 1, 0)])
def test_batch_groups_of_every_width(cuda, monkeypatch, rhs, spt, p64):
    """Every right-hand-sides-per-CTA width and FP64 pass size (0: the staged FP64 kernels, members spread over the
    warps and links shared through shared memory), set through KUQCD_BATCH_SHAPE, on groups that do not fill them:
    3 sources on one field (odd parity), 2 on another lattice, one system alone, lattices whose half volume is not
    a multiple of the staged round; all reach their targets."""
    monkeypatch.setenv("KUQCD_BATCH_SHAPE", f"256,2,{rhs},{spt},{p64}")
    batch = K.Batch()
    keep = []
    for dims, eps, seed, n, parity in [((8, 8, 8, 8), 0.3, 31, 3, 1), ((8, 4, 4, 8), 0.35, 32, 2, 0),
                                       ((6, 6, 6, 6), 0.25, 33, 1, 0)]:
        ctx, fat, lng, vb, systems = sources_on_one_field(dims, eps, seed, n, parity)
        for b, d_b, sig in systems:
            d_x = torch.zeros(vb * len(sig), dtype=torch.uint8, device="cuda")
            batch.add(ctx, d_b, d_x, sig, parity=parity, solver=K.KQ_SOLVER_MIXED, prec=K.KUQCD_HALF,
                      rel_residual=1e-10)
            keep.append((ctx, fat, lng, vb, b, d_x, sig, parity, dims))
    info = batch.solve()
    assert info.tuned_now == 0 and info.rhs_per_cta == rhs and info.sites_per_thread == spt
    assert info.fp64_rhs_per_pass == p64
    assert info.groups == sum((n + rhs - 1) // rhs for n in (3, 2, 1))
    for i, (ctx, fat, lng, vb, b, d_x, sig, parity, dims) in enumerate(keep):
        assert batch.system_info(i).status == 0, i
        for k, s in enumerate(sig):
            xk = ctx.download(K.KUQCD_DOUBLE, d_x[k * vb:(k + 1) * vb])
            r = O.true_residual(dims, fat, lng, parity, s, b, xk)
            assert r <= 1.2e-10, (i, k, r)
    batch.close()
