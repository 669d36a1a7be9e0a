"""Batched reconstructions (tomo_batch): persistent work-queue kernels over many uneven jobs.

* a job's iterate is bit-identical alone and in any mix, added late or early, with or
  without the CUDA graph (deterministic per-item norms);
* a one-job batch matches the single-job solver (same arithmetic; the norms' summation
  order differs, so within 1e-6);
* mixed precision: BF16 storage with FP32 master iterate against the FP64 oracle.
"""
import numpy as np
import pytest

from conftest import rel_l2

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _job(n, views, seed, mag=2.0, det=None, storage=torch.float32):
    import oracle
    from tomogpi_b200 import ConfigCT, phantoms

    cfg = ConfigCT.cone_beam(n, views, det=det or n, magnification=mag)
    truth = oracle.phantom(phantoms.config_phantom(seed, n), n, n, n)
    g = oracle.project(cfg, oracle.SIDDON, truth)
    g = g + np.random.default_rng(seed).normal(0, 0.01 * g.max(), g.shape).astype(np.float32)
    return cfg, torch.from_numpy(g.astype(np.float32)).cuda().to(storage)


def _params(**kw):
    import tomogpi_b200 as t

    base = dict(gradient_iteration_nb=4, optimal_step_iteration_nb=5, regularization_parameter=0.01)
    base.update(kw)
    return t.GradientParams(**base)


def _run_batch(jobs, params, iters, graph=True, layout="tex", late=None):
    """jobs: list of (cfg, g); returns the final iterates (numpy) in job order."""
    import tomogpi_b200 as t

    b = t.Batch(params, graph=graph)
    vols, ids = [], []
    late = late or {}
    for k, (cfg, g) in enumerate(jobs):
        vols.append(torch.zeros(cfg.volume_shape, device="cuda:0"))
        if k not in late:
            ids.append(b.add(cfg, vols[k], g, rs_layout=layout))
        else:
            ids.append(None)
    done = 0
    while done < iters + max(late.values(), default=0):
        for k, at in late.items():
            if at == done and ids[k] is None:
                ids[k] = b.add(jobs[k][0], vols[k], jobs[k][1], rs_layout=layout)
        b.iterate(1)
        done += 1
    torch.cuda.synchronize()
    out = [v.cpu().numpy() for v in vols]
    alphas = [b.alphas(i) for i in ids]
    stats = b.stats()
    b.close()
    return out, alphas, stats


def test_batch_alone_vs_mix_is_bit_identical():
    a = _job(32, 24, 1)
    mix = [a, _job(24, 40, 2, mag=1.6), _job(40, 30, 3, mag=2.4), _job(16, 60, 4)]
    p = _params()
    alone, al_a, _ = _run_batch([a], p, 4)
    inmix, al_m, st = _run_batch(mix, p, 4)
    assert np.array_equal(alone[0], inmix[0])
    assert np.array_equal(al_a[0], al_m[0])
    assert st["live_jobs"] == 4 and st["work_items"] > 0


def test_batch_late_join_and_graph_off_are_bit_identical():
    a, c = _job(32, 24, 1), _job(24, 20, 5, mag=1.8)
    p = _params()
    ref, _, _ = _run_batch([a, c], p, 4)
    late, _, _ = _run_batch([a, c], p, 4, late={1: 2})  # job 1 admitted after two iterations
    nog, _, _ = _run_batch([a, c], p, 4, graph=False)
    for k in range(2):
        assert np.array_equal(ref[k], late[k])
        assert np.array_equal(ref[k], nog[k])


@pytest.mark.parametrize("layout", ["tex", "cell8", "plain"])
def test_batch_single_job_matches_solver(layout):
    import tomogpi_b200 as t

    cfg, g = _job(32, 24, 7)
    p = _params()
    out, al, _ = _run_batch([(cfg, g)], p, 4, layout=layout)
    with t.Context(cfg) as ctx:
        ctx.set_tuning(rs_layout=layout)
        s = t.Solver(ctx, p)
        v = torch.zeros(cfg.volume_shape, device="cuda:0")
        s.iterate(v, g)
        ref = v.cpu().numpy()
        ref_al = s.alphas()
    assert rel_l2(out[0], ref) <= 1e-6
    assert np.allclose(al[0], ref_al, rtol=1e-9, atol=0)


def test_batch_bf16_storage_error_against_fp64_oracle():
    """BF16 operator storage, FP32 master iterate, 20 iterations, cells layout (the 16-bit
    path): error against the FP64 oracle of the same loop."""
    import oracle

    cfg, g32 = _job(32, 32, 9)
    g16 = g32.to(torch.bfloat16)
    p = _params(gradient_iteration_nb=20, optimal_step_iteration_nb=21, storage="bf16")
    out, _, _ = _run_batch([(cfg, g16)], p, 20, layout="cell8")
    # the oracle reconstructs from the same measured data (the BF16 sinogram)
    ref64, _ = oracle.simple_gradient(cfg, oracle.RS, np.zeros(cfg.volume_shape),
                                      g16.float().cpu().numpy().astype(np.float64), 20, 0.01, 21, fp64=True)
    err = rel_l2(out[0], ref64)
    print(f"bf16 batch rel L2 vs FP64 oracle after 20 iterations: {err:.2e}")
    assert err <= 1e-3


def test_batch_remove_and_finished_jobs_are_skipped():
    import tomogpi_b200 as t

    a, c = _job(24, 16, 11), _job(16, 16, 12)
    p = _params(gradient_iteration_nb=3, optimal_step_iteration_nb=4)
    b = t.Batch(p)
    va = torch.zeros(a[0].volume_shape, device="cuda:0")
    vc = torch.zeros(c[0].volume_shape, device="cuda:0")
    ja = b.add(a[0], va, a[1])
    jc = b.add(c[0], vc, c[1])
    b.iterate(5)  # two more than the jobs' iteration count
    assert b.status(ja)[0] == 3 and b.status(jc)[0] == 3
    snap = va.clone()
    b.iterate(1)
    assert torch.equal(va, snap)  # finished jobs are left alone
    b.remove(jc)
    assert b.stats()["live_jobs"] == 1
    b.close()


def test_batch_bf16_texture_equals_cells():
    """BF16 storage in the batch: the texture layout (filled from the FP32 iterate by the
    conversion kernel) and the cell layout give identical iterates, alone and mixed."""
    mix = [_job(32, 24, 1, storage=torch.bfloat16), _job(24, 40, 2, mag=1.6, storage=torch.bfloat16)]
    p = _params(storage="bf16")
    a, al_a, _ = _run_batch(mix, p, 4, layout="cell8")
    b, al_b, _ = _run_batch(mix, p, 4, layout="tex")
    for k in range(2):
        assert np.array_equal(a[k], b[k])
        assert np.array_equal(al_a[k], al_b[k])


def test_batch_real_f32_matches_solver_and_mix():
    """BF16 storage with the measured sinogram kept in FP32 (real_f32): a job's iterate is
    bit-identical alone and in a mix, equals the single-job solver's to 1e-6, and differs
    from the run on the BF16-rounded sinogram."""
    import tomogpi_b200 as t

    a = _job(32, 24, 1)
    mix = [a, _job(24, 40, 2, mag=1.6), _job(40, 30, 3, mag=2.4)]
    p = _params(storage="bf16", real_f32=True)
    alone, _, _ = _run_batch([a], p, 4)
    inmix, _, _ = _run_batch(mix, p, 4)
    assert np.array_equal(alone[0], inmix[0])
    cfg, g = a
    with t.Context(cfg) as ctx:
        s = t.Solver(ctx, p)
        v = torch.zeros(cfg.volume_shape, device="cuda:0")
        s.iterate(v, g)
        solo = v.cpu().numpy()
        s.close()
    assert rel_l2(alone[0], solo) <= 1e-6
    rounded, _, _ = _run_batch([(cfg, g.to(torch.bfloat16))], _params(storage="bf16"), 4)
    assert not np.array_equal(rounded[0], alone[0])
