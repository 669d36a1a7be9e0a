"""The device-resident gradient loops (Iter3D::doSimpleGradient and
Iter3D::doWeightedGradient, with the generalised-Gaussian or the Huber regulariser) against
the oracle's restatement of the same loops."""
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
    g = g + np.random.default_rng(seed).normal(0, 0.01 * g.max(), g.shape).astype(np.float32)
    return cfg, truth, g.astype(np.float32)


@pytest.mark.parametrize("layout", ["plain", "cell8", "tex", "hybrid", "hybrid+tma", "march", "march+tma"])
@pytest.mark.parametrize("opt_nb", [21, 3])
def test_gradient_fp32_matches_oracle(opt_nb, layout):
    import oracle
    import tomogpi_b200 as t

    cfg, truth, g = _problem()
    iters = 6
    ref, ref_alpha = oracle.simple_gradient(cfg, oracle.RS, np.zeros(cfg.volume_shape, np.float32), g, iters, 0.01,
                                            opt_nb)
    with t.Context(cfg) as ctx:
        ctx.set_tuning(rs_layout=layout.split("+")[0], vi_layout="tma" if layout.endswith("+tma") else "padded")
        solver = t.Solver(ctx, t.GradientParams(gradient_iteration_nb=iters, optimal_step_iteration_nb=opt_nb,
                                                regularization_parameter=0.01))
        vol = torch.zeros(cfg.volume_shape, device="cuda:0")
        solver.iterate(vol, torch.from_numpy(g).cuda())
        got = vol.cpu().numpy()
        alphas = solver.alphas()
        solver.close()
    assert np.allclose(alphas, ref_alpha, rtol=1e-4, atol=0)
    assert rel_l2(got, ref) <= 1e-4


def test_gradient_resume_equals_straight_run():
    import tomogpi_b200 as t

    cfg, truth, g = _problem(n=24, views=16)
    gd = torch.from_numpy(g).cuda()
    p = t.GradientParams(gradient_iteration_nb=6, optimal_step_iteration_nb=4)
    with t.Context(cfg) as ctx:
        s1 = t.Solver(ctx, p)
        a = torch.zeros(cfg.volume_shape, device="cuda:0")
        s1.iterate(a, gd)
        s2 = t.Solver(ctx, p)
        b = torch.zeros(cfg.volume_shape, device="cuda:0")
        s2.iterate(b, gd, first=1, count=3)
        state = s2.get_state()
        ckpt = b.clone()
        s3 = t.Solver(ctx, p)
        s3.set_state(*state)
        s3.iterate(ckpt, gd, first=state[1], count=3)
        assert torch.equal(a, ckpt)


@pytest.mark.parametrize("n", [32, 64])
@pytest.mark.parametrize("storage", ["bf16", "f16"])
def test_gradient_mixed_precision_error(storage, n):
    """16-bit operator storage with an FP32 master iterate: error against the FP64 oracle
    and against the FP32 run, after 20 iterations."""
    import oracle
    import tomogpi_b200 as t

    cfg, truth, g = _problem(n=n, views=n)
    iters = 20
    tdt = {"bf16": torch.bfloat16, "f16": torch.float16}[storage]
    # the measured data is the 16-bit sinogram: every run (and the oracle) starts from it
    g = torch.from_numpy(g).to(tdt).float().numpy()
    ref64, _ = oracle.simple_gradient(cfg, oracle.RS, np.zeros(cfg.volume_shape), g.astype(np.float64), iters, 0.01,
                                      21, fp64=True)
    out = {}
    with t.Context(cfg) as ctx:
        for st in ("f32", storage):
            gd = torch.from_numpy(g).cuda().to({"f32": torch.float32, "bf16": torch.bfloat16, "f16": torch.float16}[st])
            s = t.Solver(ctx, t.GradientParams(gradient_iteration_nb=iters, optimal_step_iteration_nb=21,
                                               regularization_parameter=0.01, storage=st))
            v = torch.zeros(cfg.volume_shape, device="cuda:0")
            s.iterate(v, gd)
            out[st] = v.cpu().numpy()
            s.close()
    e32 = rel_l2(out["f32"], ref64)
    emp = rel_l2(out[storage], ref64)
    print(f"n={n} rel L2 vs FP64 oracle: f32 {e32:.2e}, {storage} {emp:.2e}; "
          f"{storage} vs f32 {rel_l2(out[storage], out['f32']):.2e}")
    assert e32 <= 1e-3
    assert emp <= 1e-3


@pytest.mark.parametrize("storage", ["bf16", "f16"])
def test_mixed_precision_against_fp64_on_fp32_data(storage):
    """The measured data in FP32: the FP64 oracle runs on the FP32 sinogram, and the 16-bit
    runs are stated both with the sinogram stored in 16 bits (the data's own rounding, 2^-9
    relative per ray sum in BF16, then dominates) and kept in FP32 (real_f32: only the
    operators' 16-bit storage remains), after 20 iterations. The target is <= 1e-3 relative
    L2 against FP64; BF16-rounded data misses it at these sizes (about 3e-3 at 64^3), which
    is why real_f32 exists."""
    import oracle
    import tomogpi_b200 as t

    cfg, truth, g = _problem(n=64, views=64)
    iters = 20
    tdt = {"bf16": torch.bfloat16, "f16": torch.float16}[storage]
    ref64, _ = oracle.simple_gradient(cfg, oracle.RS, np.zeros(cfg.volume_shape), g.astype(np.float64), iters, 0.01,
                                      21, fp64=True)
    out = {}
    with t.Context(cfg) as ctx:
        for name, st, real_f32, gd in (("f32", "f32", False, torch.from_numpy(g).cuda()),
                                       ("rounded", storage, False, torch.from_numpy(g).cuda().to(tdt)),
                                       ("real_f32", storage, True, torch.from_numpy(g).cuda())):
            s = t.Solver(ctx, t.GradientParams(gradient_iteration_nb=iters, optimal_step_iteration_nb=21,
                                               regularization_parameter=0.01, storage=st, real_f32=real_f32))
            v = torch.zeros(cfg.volume_shape, device="cuda:0")
            s.iterate(v, gd)
            out[name] = v.cpu().numpy()
            s.close()
    errs = {k: rel_l2(v, ref64) for k, v in out.items()}
    print(f"64^3 {storage} rel L2 vs FP64 oracle on FP32 data: FP32 {errs['f32']:.2e}, "
          f"{storage} data {errs['rounded']:.2e}, FP32 data {errs['real_f32']:.2e}")
    assert errs["f32"] <= 1e-4
    assert errs["real_f32"] <= 1e-3
    if storage == "f16":
        assert errs["rounded"] <= 1e-3


@pytest.mark.parametrize("storage", ["bf16", "f16"])
def test_half_solver_texture_equals_cells(storage):
    """16-bit storage: the solver's texture layout, filled from the FP32 iterate by the
    rounding conversion kernel, gives the same iterates and steps as the cell layout."""
    import tomogpi_b200 as t

    cfg, _, g = _problem(n=40, views=20, seed=3)
    tdt = {"bf16": torch.bfloat16, "f16": torch.float16}[storage]
    res = {}
    with t.Context(cfg) as ctx:
        for lay in ("cell8", "tex", "hybrid"):
            ctx.set_tuning(rs_layout=lay)
            s = t.Solver(ctx, t.GradientParams(gradient_iteration_nb=4, optimal_step_iteration_nb=3,
                                               regularization_parameter=0.01, storage=storage))
            vol = torch.zeros(cfg.volume_shape, device="cuda:0")
            s.iterate(vol, torch.from_numpy(g).cuda().to(tdt))
            res[lay] = (vol.cpu().numpy(), s.alphas())
            s.close()
    for lay in ("tex", "hybrid"):
        assert np.array_equal(res["cell8"][0], res[lay][0]), lay
        # the single-job solver sums ||H dJ||^2 with double atomics, whose order varies between
        # runs: the steps agree to the last few bits (and round to the same float step)
        assert np.allclose(res["cell8"][1], res[lay][1], rtol=1e-12, atol=0), lay


def test_fp16_range_guard():
    """FP16 storage where dJ = -2 H^T r exceeds FP16's range (65504): the gradient is scaled
    by a power of two before it is stored, and the step's norm scaled back. The solver and
    the batch stay finite and match the FP32 runs on the same FP16-rounded data."""
    import tomogpi_b200 as t

    cfg, _, g = _problem(n=32, views=48, seed=5)
    g = g * (8000.0 / g.max())                     # ray sums up to 8000: FP16 holds them
    g16 = torch.from_numpy(g).cuda().half()
    p16 = t.GradientParams(gradient_iteration_nb=5, optimal_step_iteration_nb=6, regularization_parameter=0.01,
                           storage="f16")
    p32 = t.GradientParams(gradient_iteration_nb=5, optimal_step_iteration_nb=6, regularization_parameter=0.01)
    out = {}
    with t.Context(cfg) as ctx:
        dj = ctx.backproject("VI", g16.float())
        assert float(dj.abs().max()) * 2 > 65504   # the unguarded dJ would overflow
        for name, prm, gg in (("f16", p16, g16), ("f32", p32, g16.float())):
            s = t.Solver(ctx, prm)
            v = torch.zeros(cfg.volume_shape, device="cuda:0")
            s.iterate(v, gg)
            out[name] = v.cpu().numpy()
            out[name + "_alpha"] = s.alphas()
            s.close()
    for name, prm, gg in (("bf16", p16, g16), ("b32", p32, g16.float())):
        b = t.Batch(prm)
        v = torch.zeros(cfg.volume_shape, device="cuda:0")
        b.add(cfg, v, gg, rs_layout="tex")
        b.iterate(5)
        out[name] = v.cpu().numpy()
        b.close()
    for k in ("f16", "bf16"):
        assert np.isfinite(out[k]).all()
    assert np.isfinite(out["f16_alpha"]).all() and (out["f16_alpha"] < 0).all()
    assert rel_l2(out["f16"], out["f32"]) <= 2e-3, rel_l2(out["f16"], out["f32"])
    assert rel_l2(out["bf16"], out["b32"]) <= 2e-3, rel_l2(out["bf16"], out["b32"])


@pytest.mark.parametrize("storage", ["f32", "bf16"])
def test_solver_vi_texture_equals_padded(storage):
    """The solver's VI reading the residual from a layered texture (copied from the padded
    residual each iteration) gives the same iterates as reading the padded residual."""
    import tomogpi_b200 as t

    cfg, _, g = _problem(n=32, views=24, seed=8)
    tdt = {"f32": torch.float32, "bf16": torch.bfloat16}[storage]
    res = {}
    with t.Context(cfg) as ctx:
        for lay in ("padded", "tex"):
            ctx.set_tuning(vi_layout=lay)
            s = t.Solver(ctx, t.GradientParams(gradient_iteration_nb=4, optimal_step_iteration_nb=5,
                                               regularization_parameter=0.01, storage=storage))
            vol = torch.zeros(cfg.volume_shape, device="cuda:0")
            s.iterate(vol, torch.from_numpy(g).cuda().to(tdt))
            res[lay] = vol.cpu().numpy()
            s.close()
    assert np.array_equal(res["padded"], res["tex"])


@pytest.mark.parametrize("thr", [0.002, 0.05, 1e9])
@pytest.mark.parametrize("opt_nb", [21, 3])
def test_huber_gradient_matches_oracle(thr, opt_nb):
    """The Huber regulariser (HuberRegularizer_CPU.cu:206-253) in the simple gradient: the
    FP32 loop against the oracle's FP32 restatement (steps to 1e-4 relative, iterate 1e-4
    relative L2), and against the FP64 oracle after 20 iterations (1e-3). Thresholds below,
    inside and above the range of L f, so every branch of psi' and psi'' is taken."""
    import oracle
    import tomogpi_b200 as t

    cfg, truth, g = _problem()
    iters = 6
    ref, ref_alpha = oracle.simple_gradient(cfg, oracle.RS, np.zeros(cfg.volume_shape, np.float32), g, iters, 0.05,
                                            opt_nb, huber_threshold=thr)
    with t.Context(cfg) as ctx:
        solver = t.Solver(ctx, t.GradientParams(gradient_iteration_nb=iters, optimal_step_iteration_nb=opt_nb,
                                                regularization_parameter=0.05))
        solver.set_regularizer("huber", thr)
        vol = torch.zeros(cfg.volume_shape, device="cuda:0")
        solver.iterate(vol, torch.from_numpy(g).cuda())
        got = vol.cpu().numpy()
        alphas = solver.alphas()
        solver.close()
    assert np.allclose(alphas, ref_alpha, rtol=1e-4, atol=0)
    assert rel_l2(got, ref) <= 1e-4
    # the Huber and GG loops differ once the iterate has structure
    gg, _ = oracle.simple_gradient(cfg, oracle.RS, np.zeros(cfg.volume_shape, np.float32), g, iters, 0.05, opt_nb)
    if thr < 1.0:
        assert rel_l2(gg, ref) > 1e-6


def test_huber_gradient_fp64_error():
    import oracle
    import tomogpi_b200 as t

    cfg, truth, g = _problem()
    iters = 20
    ref64, _ = oracle.simple_gradient(cfg, oracle.RS, np.zeros(cfg.volume_shape), g.astype(np.float64), iters, 0.05,
                                      21, fp64=True, huber_threshold=0.05)
    with t.Context(cfg) as ctx:
        s = t.Solver(ctx, t.GradientParams(gradient_iteration_nb=iters, optimal_step_iteration_nb=21,
                                           regularization_parameter=0.05))
        s.set_regularizer("huber", 0.05)
        v = torch.zeros(cfg.volume_shape, device="cuda:0")
        s.iterate(v, torch.from_numpy(g).cuda())
        got = v.cpu().numpy()
        s.close()
    err = rel_l2(got, ref64)
    print(f"Huber, 20 iterations: rel L2 vs FP64 oracle {err:.2e}")
    assert err <= 1e-3


def test_regularizer_argument_checks():
    import tomogpi_b200 as t
    from tomogpi_b200._lib import TomoError

    cfg, truth, g = _problem(n=16, views=8)
    with t.Context(cfg) as ctx:
        s = t.Solver(ctx, t.GradientParams(gradient_iteration_nb=1))
        with pytest.raises(ValueError):
            s.set_regularizer("tv")
        with pytest.raises(TomoError):
            s.set_regularizer("huber", -1.0)
        with pytest.raises(TomoError):
            s.set_regularizer("huber", float("nan"))
        s.set_regularizer("gg")
        s.close()


@pytest.mark.parametrize("beta", [1.2, 1.5, 2.5])
@pytest.mark.parametrize("opt_nb", [21, 3])
def test_gg_beta_gradient_matches_oracle(beta, opt_nb):
    """The generalised Gaussian of shape beta != 2 in the simple gradient
    (GeneralizedGaussianRegularizer_GPU.cu:161-225: dJ += beta*lambda L(sign(f) |f|^(beta-1)),
    normdJProjReg = beta sum |L dJ|^beta): the FP32 loop against the oracle's FP32 loop (pinned
    bit for bit to the reference's own loop and regulariser built for the host), steps to
    1e-4 relative, iterate 1e-4 relative L2; and against the FP64 oracle after 20
    iterations (1e-3)."""
    import oracle
    import tomogpi_b200 as t

    cfg, truth, g = _problem()
    lam = 0.05
    for iters, fp64 in ((6, False), (20, True)):
        dt = np.float64 if fp64 else np.float32
        ref, ref_alpha = oracle.simple_gradient(cfg, oracle.RS, np.zeros(cfg.volume_shape, dt), g.astype(dt), iters,
                                                lam, opt_nb, beta=beta, fp64=fp64)
        with t.Context(cfg) as ctx:
            s = t.Solver(ctx, t.GradientParams(gradient_iteration_nb=iters, optimal_step_iteration_nb=opt_nb,
                                               regularization_parameter=lam))
            s.set_regularizer("gg", beta=beta)
            vol = torch.zeros(cfg.volume_shape, device="cuda:0")
            s.iterate(vol, torch.from_numpy(g).cuda())
            got = vol.cpu().numpy()
            alphas = s.alphas()
            s.close()
        err = rel_l2(got, ref)
        print(f"GG beta {beta}, opt {opt_nb}, {iters} iterations: rel L2 vs {'FP64' if fp64 else 'FP32'} oracle "
              f"{err:.2e}")
        if fp64:
            assert err <= 1e-3
        else:
            assert np.allclose(alphas, ref_alpha, rtol=1e-4, atol=0)
            assert err <= 1e-4
    b2, _ = oracle.simple_gradient(cfg, oracle.RS, np.zeros(cfg.volume_shape, np.float32), g, 20, lam, opt_nb)
    assert rel_l2(b2, got) > 1e-6  # not the beta = 2 loop


@pytest.mark.parametrize("beta", [1.0, 1.3, 2.0, 3.0])
@pytest.mark.parametrize("total,optimal", [(1, 4), (4, 4)])
def test_gg_beta_regularization_matches_oracle(beta, total, optimal):
    """tomo_gg_regularization_beta (the MEX ApplyLaplacianRegularization_to_dJ with
    configIteration beta) against the oracle's criterion: dJ 1e-6 relative L2, jReg and
    normdJProjReg 1e-6 relative. The volume holds exact zeros (sign(0) = 0)."""
    import oracle
    import tomogpi_b200 as t

    rng = np.random.default_rng(int(beta * 10) + total)
    vol = rng.normal(0, 0.3, (20, 24, 28)).astype(np.float32)
    vol[rng.random(vol.shape) < 0.1] = 0.0
    dJ = rng.normal(0, 1.0, vol.shape).astype(np.float32)
    d_ref, j_ref, n_ref = oracle.regularizer_criterion(vol, dJ, 0.037, total, optimal, beta=beta)
    d = torch.from_numpy(dJ).cuda()
    j, n = t.gg_regularization(torch.from_numpy(vol).cuda(), d, 0.037, total, optimal, beta=beta)
    assert rel_l2(d.cpu().numpy(), d_ref) <= 1e-6
    assert abs(j - j_ref) <= 1e-6 * abs(j_ref)
    if total < optimal:
        assert abs(n - n_ref) <= 1e-6 * abs(n_ref)
    else:
        assert n is None and n_ref is None


@pytest.mark.parametrize("layout", ["tex", "hybrid", "march+tma"])
@pytest.mark.parametrize("beta", [2.0, 1.5])
def test_weighted_gradient_matches_oracle(layout, beta):
    """Iter3D::doWeightedGradient (Iter3D_Algo_Gradient.cu:227-373): the residual times the
    weight sinogram before each backprojection, alpha_min from -999999999999. FP32 loop
    against the oracle's loop (pinned bit for bit to the reference's own weighted loop built
    for the host): steps 1e-4 relative, iterate 1e-4 relative L2. Weights given as a device
    tensor and as a host array give the same iterate; optimal_step_iteration_nb 4 < 6
    iterations, so the last steps take alpha_min."""
    import oracle
    import tomogpi_b200 as t

    cfg, truth, g = _problem()
    rng = np.random.default_rng(7)
    w = rng.uniform(0.25, 1.75, g.shape).astype(np.float32)
    w[rng.random(g.shape) < 0.05] = 0.0
    iters, opt_nb, lam = 6, 4, 0.02
    ref, ref_alpha = oracle.simple_gradient(cfg, oracle.RS, np.zeros(cfg.volume_shape, np.float32), g, iters, lam,
                                            opt_nb, beta=beta, weights=w)
    plain, _ = oracle.simple_gradient(cfg, oracle.RS, np.zeros(cfg.volume_shape, np.float32), g, iters, lam, opt_nb,
                                      beta=beta)
    assert rel_l2(plain, ref) > 1e-3  # the weights matter
    res = []
    with t.Context(cfg) as ctx:
        ctx.set_tuning(rs_layout=layout.split("+")[0], vi_layout="tma" if layout.endswith("+tma") else "padded")
        for host in (False, True):
            s = t.Solver(ctx, t.GradientParams(gradient_iteration_nb=iters, optimal_step_iteration_nb=opt_nb,
                                               regularization_parameter=lam))
            s.set_regularizer("gg", beta=beta)
            s.set_weights(w if host else torch.from_numpy(w).cuda())
            vol = torch.zeros(cfg.volume_shape, device="cuda:0")
            s.iterate(vol, torch.from_numpy(g).cuda())
            res.append((vol.cpu().numpy(), s.alphas()))
            s.close()
    assert np.array_equal(res[0][0], res[1][0])
    got, alphas = res[0]
    assert np.allclose(alphas, ref_alpha, rtol=1e-4, atol=0)
    assert rel_l2(got, ref) <= 1e-4


def test_weights_and_beta_argument_checks():
    import tomogpi_b200 as t
    from tomogpi_b200._lib import TomoError

    cfg, truth, g = _problem(n=16, views=8)
    with t.Context(cfg) as ctx:
        s = t.Solver(ctx, t.GradientParams(gradient_iteration_nb=2))
        for beta in (0.5, float("nan")):
            with pytest.raises(TomoError):
                s.set_regularizer("gg", beta=beta)
        with pytest.raises(TypeError):
            s.set_weights(torch.ones(3, 4, 5, device="cuda:0"))
        with pytest.raises(ValueError):
            s.set_weights(np.ones((3, 4, 5), np.float32))
        vol = torch.zeros(cfg.volume_shape, device="cuda:0")
        s.iterate(vol, torch.from_numpy(g).cuda(), count=1)
        with pytest.raises(TomoError):  # only before the first iteration
            s.set_weights(np.ones(g.shape, np.float32))
        s.close()


@pytest.mark.parametrize("storage,real_f32,projector,layout", [("f32", False, "RS", "hybrid"),
                                                               ("bf16", True, "RS", "tex"),
                                                               ("f16", False, "RS_UM", "cell8"),
                                                               ("f32", False, "SIDDON", "tex")])
def test_host_buffer_solver_equals_device_solver(storage, real_f32, projector, layout):
    """tomo_solver_iterate_host (host iterate and measured sinogram, copied in and out; the
    sinogram's copy overlaps the first projection, and the residual is then formed in a
    pass of its own) against tomo_solver_iterate on device buffers: the same iterate and
    steps bit for bit, over two calls of three iterations."""
    import tomogpi_b200 as t

    cfg, truth, g = _problem(n=32, views=24)
    rdt = {"f32": np.float32, "f16": np.float16, "bf16": np.float32}[storage if not real_f32 else "f32"]
    tdt = {"f32": torch.float32, "f16": torch.float16, "bf16": torch.float32}[storage if not real_f32 else "f32"]
    g_real = g.astype(rdt)
    prm = t.GradientParams(gradient_iteration_nb=6, optimal_step_iteration_nb=4, regularization_parameter=0.01,
                           storage=storage, real_f32=real_f32, projector=projector)
    with t.Context(cfg) as ctx:
        ctx.set_tuning(rs_layout=layout)
        a = t.Solver(ctx, prm)
        va = torch.zeros(cfg.volume_shape, device="cuda:0")
        gd = torch.from_numpy(g_real).cuda().to(tdt)
        a.iterate(va, gd, first=1, count=3)
        a.iterate(va, gd, first=4, count=3)
        b = t.Solver(ctx, prm)
        vb = np.zeros(cfg.volume_shape, np.float32)
        b.iterate_host(vb, g_real, first=1, count=3)
        b.iterate_host(vb, g_real, first=4, count=3)
        assert np.array_equal(va.cpu().numpy(), vb)
        assert np.array_equal(a.alphas(), b.alphas())
        assert np.abs(vb).max() > 0
        a.close()
        b.close()
