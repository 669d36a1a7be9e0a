"""One reconstruction split by views (tomo_context_create_views, tomo_solver_phase): view
ranges against the whole acquisition on one GPU, and two ranks emulated in lockstep in one
process (their kernels never wait on each other; the sums are done between phases)."""
import numpy as np
import pytest

from conftest import rel_l2

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _problem(n=32, views=24, seed=0):
    import oracle
    from tomogpi_b200 import ConfigCT, phantoms

    cfg = ConfigCT.cone_beam(n, views)
    truth = oracle.phantom(phantoms.config_phantom(seed, n), n, n, n)
    g = oracle.project(cfg, oracle.SIDDON, truth)
    g = (g + np.random.default_rng(seed).normal(0, 0.01 * g.max(), g.shape)).astype(np.float32)
    return cfg, truth, g


@pytest.mark.parametrize("begin,count", [(0, 10), (7, 11), (13, 11)])
def test_view_range_context_equals_whole(begin, count):
    """Projection of a view range = those views of the whole projection (bit for bit); its
    backprojection = the whole backprojection of a sinogram zero outside the range (bit for
    bit: the whole one adds exact zeros first, and only acquisition view 0 takes the
    double-precision A of backprojection3D_kernel_16reg.cuh:404)."""
    import tomogpi_b200 as t

    cfg, truth, g = _problem()
    vol = torch.from_numpy(truth).cuda()
    with t.Context(cfg) as full, t.Context(cfg, views=(begin, count)) as part:
        assert part.sinogram_shape == (count, 32, 32)
        for kind in ("RS", "RS_UM", "SIDDON_REF"):
            assert torch.equal(part.project(kind, vol), full.project(kind, vol)[begin:begin + count]), kind
        gz = np.zeros_like(g)
        gz[begin:begin + count] = g[begin:begin + count]
        gpart = torch.from_numpy(np.ascontiguousarray(g[begin:begin + count])).cuda()
        for kind in ("VI", "VI_UM", "FDK"):
            a = part.backproject(kind, gpart)
            b = full.backproject(kind, torch.from_numpy(gz).cuda())
            assert torch.equal(a, b), kind


def test_view_range_arguments():
    import tomogpi_b200 as t
    from tomogpi_b200._lib import TomoError

    cfg, truth, g = _problem(n=16, views=8)
    for bad in ((-1, 4), (0, 0), (5, 4), (8, 1)):
        with pytest.raises(TomoError):
            t.Context(cfg, views=bad)


@pytest.mark.parametrize("huber,weighted", [(None, False), (0.05, False), (None, True)])
def test_two_ranks_in_lockstep_match_one(huber, weighted):
    """Two ranks, each on half of the views, summing dJ and the view norms between phases
    as iterate_exchange does, against the one-GPU solver; with the weighted gradient each
    rank holds the weights of its own views."""
    import tomogpi_b200 as t
    from tomogpi_b200.sharded import PHASE_GRADIENT, PHASE_NORMS, PHASE_UPDATE, ShardedSolver

    cfg, truth, g = _problem()
    iters, opt_nb = 6, 4
    prm = t.GradientParams(gradient_iteration_nb=iters, optimal_step_iteration_nb=opt_nb,
                           regularization_parameter=0.05)
    reg = None if huber is None else ("huber", huber)
    w = np.random.default_rng(9).uniform(0.5, 1.5, g.shape).astype(np.float32) if weighted else None
    gd = torch.from_numpy(g).cuda()
    with t.Context(cfg) as ctx:
        one = t.Solver(ctx, prm)
        if reg:
            one.set_regularizer(*reg)
        if weighted:
            one.set_weights(w)
        ref = torch.zeros(cfg.volume_shape, device="cuda:0")
        one.iterate(ref, gd)
        ref_alpha = one.alphas()
        one.close()
    ranks = [ShardedSolver(cfg, prm, device=0, rank=r, world=2, regularizer=reg, weights=w) for r in range(2)]
    vols = [torch.zeros(cfg.volume_shape, device="cuda:0") for _ in ranks]
    parts = [s.real_part(gd) for s in ranks]
    for it in range(1, iters + 1):
        for s, v, gp in zip(ranks, vols, parts):
            s.solver.phase(v, gp, it, PHASE_GRADIENT)
        total = ranks[0].dJ + ranks[1].dJ
        for s in ranks:
            s.dJ.copy_(total)
        for s, v in zip(ranks, vols):
            s.solver.phase(v, None, it, PHASE_NORMS)
        if it < opt_nb:  # as iterate_exchange: rank 0's norms of the summed dJ, the sum of ||H_k dJ||^2
            ranks[1].norms[[0, 2, 4]] = 0.0
            n = ranks[0].norms[0:5] + ranks[1].norms[0:5]
            for s in ranks:
                s.norms[0:3].copy_(n[0:3])
                s.norms[4:5].copy_(n[4:5])
        for s, v in zip(ranks, vols):
            s.solver.phase(v, None, it, PHASE_UPDATE)
    assert torch.equal(vols[0], vols[1])                       # every rank holds the same iterate
    assert np.array_equal(ranks[0].alphas(), ranks[1].alphas())
    assert np.allclose(ranks[0].alphas(), ref_alpha, rtol=1e-5, atol=0)
    assert rel_l2(vols[0].cpu().numpy(), ref.cpu().numpy()) <= 1e-5
    for s in ranks:
        s.close()


def test_single_rank_sharded_equals_solver():
    """world = 1: the phase loop is the solver's own iteration, bit for bit."""
    import tomogpi_b200 as t
    from tomogpi_b200.sharded import ShardedSolver

    cfg, truth, g = _problem(n=24, views=16)
    prm = t.GradientParams(gradient_iteration_nb=5, optimal_step_iteration_nb=3, regularization_parameter=0.01)
    gd = torch.from_numpy(g).cuda()
    with t.Context(cfg) as ctx:
        one = t.Solver(ctx, prm)
        a = torch.zeros(cfg.volume_shape, device="cuda:0")
        one.iterate(a, gd)
        one.close()
    s = ShardedSolver(cfg, prm, device=0, rank=0, world=1)
    b = torch.zeros(cfg.volume_shape, device="cuda:0")
    s.iterate(b, s.real_part(gd))
    s.close()
    assert torch.equal(a, b)


def test_single_rank_sharded_weighted_beta_equals_solver():
    """world = 1 with the weighted gradient and the generalised Gaussian of shape 1.5: the
    phase loop is the solver's own iteration, bit for bit."""
    import tomogpi_b200 as t
    from tomogpi_b200.sharded import ShardedSolver

    cfg, truth, g = _problem(n=24, views=16)
    w = np.random.default_rng(6).uniform(0.5, 1.5, g.shape).astype(np.float32)
    prm = t.GradientParams(gradient_iteration_nb=5, optimal_step_iteration_nb=3, regularization_parameter=0.01)
    gd = torch.from_numpy(g).cuda()
    with t.Context(cfg) as ctx:
        one = t.Solver(ctx, prm)
        one.set_regularizer("gg", beta=1.5)
        one.set_weights(w)
        a = torch.zeros(cfg.volume_shape, device="cuda:0")
        one.iterate(a, gd)
        one.close()
    s = ShardedSolver(cfg, prm, device=0, rank=0, world=1, regularizer=("gg", 0.0, 1.5), weights=w)
    b = torch.zeros(cfg.volume_shape, device="cuda:0")
    s.iterate(b, s.real_part(gd))
    s.close()
    assert torch.equal(a, b)
