"""relMSE against an FP64 high-spp converged oracle.

The converged reference is the oracle (the C++ restatement of the reference's
integrators) instantiated in FP64 -- geometry, traversal, shading and film all
in double -- at high spp.  Each image is scored by

    relMSE = mean over pixels and channels of (x - ref)^2 / (ref^2 + 1e-2).

The GPU (FP32 transport) must reach the same relMSE as the FP32 oracle at the
same spp: on the same sample streams the two relMSEs agree to 2% (the images
agree pixel by pixel), and on independent seeds the ratio of replicate means
stays within [0.6, 1.65] -- relMSE is heavy-tailed (a single 16-spp BDPT
replicate ranges over 3x), so this second bar is loose.  Equal relMSE at equal
spp is the bar under which batched and plain GPU throughput are compared.  The
measured values print with `pytest -s`.
"""
import ctypes as C

import numpy as np
import pytest

import agentray
import agentray.scenes as S
import oracle as O
from agentray import _abi as A
from agentray.scene_data import integrator_cfg

pytestmark = pytest.mark.gpu


def relmse(x, ref):
    return float(np.mean((x - ref) ** 2 / (ref ** 2 + 1e-2)))


def _render_gpu(ctx, scene, cam, cfg, w, h):
    out = np.empty(w * h * 3, np.float32)
    agentray.check(agentray.lib().ar_render(ctx.handle, scene.handle, C.byref(cam.desc()), C.byref(cfg), w, h,
                                            out.ctypes.data, 0))
    return out.reshape(h, w, 3).astype(np.float64)


def _compare(ctx, sc, cam, kind, ref_cfg, w, h, spp, reps=8, **kw):
    """Mean relMSE of GPU and FP32-oracle replicates: GPU seeds 1000+k, oracle
    seeds 1000+k (same streams) and 2000+k (independent)."""
    ref = O.OracleScene(sc, precision=64).render(cam, ref_cfg, w, h, sampler=O.SAMPLER_COUNTER)
    g = agentray.Scene(ctx, sc)
    osc = O.OracleScene(sc)
    gpu = [relmse(_render_gpu(ctx, g, cam, integrator_cfg(kind, spp=spp, seed=1000 + k, **kw), w, h), ref)
           for k in range(reps)]
    same = [relmse(osc.render(cam, integrator_cfg(kind, spp=spp, seed=1000 + k, **kw), w, h,
                              sampler=O.SAMPLER_COUNTER), ref) for k in range(reps)]
    indep = [relmse(osc.render(cam, integrator_cfg(kind, spp=spp, seed=2000 + k, **kw), w, h,
                               sampler=O.SAMPLER_COUNTER), ref) for k in range(reps)]
    return float(np.mean(gpu)), float(np.mean(same)), float(np.mean(indep)), ref, g


def _check(gpu, same, indep):
    assert abs(gpu / same - 1.0) <= 0.02, (gpu, same)
    assert 0.6 <= gpu / indep <= 1.65, (gpu, indep)


def test_pt_relmse_equals_oracle(ctx):
    sc, cam = S.cornell_box(1)
    w = h = 48
    ref_cfg = integrator_cfg(A.INTEGRATOR_PT, spp=4096, max_depth=8, rr_depth=3, seed=7)
    gpu, same, indep, ref, g = _compare(ctx, sc, cam, A.INTEGRATOR_PT, ref_cfg, w, h, spp=16, max_depth=8,
                                        rr_depth=3)
    print(f"\nPT Cornell {w}x{h} 16 spp: relMSE GPU {gpu:.5f}  FP32 oracle same seeds {same:.5f}, "
          f"independent {indep:.5f}  (ref: FP64 oracle 4096 spp)")
    _check(gpu, same, indep)
    # high spp: the FP64-film GPU image converges on the FP64 oracle
    hi = relmse(_render_gpu(ctx, g, cam, integrator_cfg(A.INTEGRATOR_PT, spp=1024, seed=3,
                                                        film_precision=A.FILM_F64), w, h), ref)
    print(f"PT Cornell {w}x{h} 1024 spp, FP64 film: relMSE {hi:.6f}")
    assert hi < gpu / 32


def test_bdpt_relmse_equals_oracle(ctx):
    sc, cam = S.cornell_box(1)
    w = h = 32
    ref_cfg = integrator_cfg(A.INTEGRATOR_BDPT, spp=2048, max_depth=6, rr_depth=3, seed=7)
    gpu, same, indep, _, _ = _compare(ctx, sc, cam, A.INTEGRATOR_BDPT, ref_cfg, w, h, spp=16, max_depth=6,
                                      rr_depth=3)
    print(f"\nBDPT Cornell {w}x{h} 16 spp: relMSE GPU {gpu:.5f}  FP32 oracle same seeds {same:.5f}, "
          f"independent {indep:.5f}  (ref: FP64 oracle 2048 spp)")
    _check(gpu, same, indep)


def test_gdpt_relmse_equals_oracle(ctx):
    sc, cam = S.cornell_box(1)
    w, h = 48, 40
    # Scored against FP64 PT, where a consistent reconstruction converges.  The
    # reference's +div G right-hand side does not (relMSE ~40); the GPU
    # reproduces it exactly (same seeds) -- see the consistent-sign test below.
    ref_cfg = integrator_cfg(A.INTEGRATOR_PT, spp=4096, max_depth=6, rr_depth=3, seed=7)
    gpu, same, indep, ref, g = _compare(ctx, sc, cam, A.INTEGRATOR_GDPT, ref_cfg, w, h, spp=16, max_depth=6,
                                        rr_depth=3)
    print(f"\nGDPT (SOR) Cornell {w}x{h} 16 spp: relMSE GPU {gpu:.5f}  FP32 oracle same seeds {same:.5f}, "
          f"independent {indep:.5f}  (ref: FP64 oracle PT 4096 spp)")
    _check(gpu, same, indep)
    cg = np.mean([relmse(_render_gpu(ctx, g, cam, integrator_cfg(
        A.INTEGRATOR_GDPT, spp=16, max_depth=6, rr_depth=3, seed=1000 + k, poisson_solver=A.POISSON_CG,
        poisson_tolerance=1e-6), w, h), ref) for k in range(8)])
    print(f"GDPT (CG + FP64 refinement, 1e-6) Cornell {w}x{h} 16 spp: relMSE GPU {cg:.5f}")
    assert 0.6 <= cg / gpu <= 1.65, (cg, gpu)


def test_gdpt_consistent_divergence_converges_to_pt(ctx):
    """Extension: with AR_GDPT_CONSISTENT_DIVERGENCE the reconstruction uses
    -div G, the sign consistent with its stencil, and lands on the PT image
    (the reference's +div G does not: its relMSE above is ~40)."""
    sc, cam = S.cornell_box(1)
    w, h = 48, 40
    ref_cfg = integrator_cfg(A.INTEGRATOR_PT, spp=4096, max_depth=6, rr_depth=3, seed=7)
    flags = A.GDPT_CONSISTENT_DIVERGENCE
    gpu, same, indep, _, _ = _compare(ctx, sc, cam, A.INTEGRATOR_GDPT, ref_cfg, w, h, spp=16, max_depth=6,
                                      rr_depth=3, gdpt_flags=flags)
    print(f"\nGDPT consistent divergence, Cornell {w}x{h} 16 spp: relMSE GPU {gpu:.5f}  FP32 oracle same seeds "
          f"{same:.5f}, independent {indep:.5f}")
    _check(gpu, same, indep)
    # unbiased, but heavy-tailed: gradients across the light's edge spike
    # (16-spp replicates range 0.04..1.4 on the oracle); far from ~40 either way
    assert gpu < 1.0


def test_consistent_divergence_recovers_exact_gradients(ctx):
    # primal = truth + noise, gradients exact: the consistent solve removes
    # most of the noise and equals the exact FP64 solution of the system with
    # -div G (the oracle's +div G solve fed negated gradients); the reference
    # sign leaves four times the error.
    rng = np.random.default_rng(4)
    h, w = 40, 56
    yy, xx = np.mgrid[0:h, 0:w]
    truth = np.stack([np.sin(xx / 7.0) + 2, np.cos(yy / 5.0) + 2, (xx + yy) / 50.0 + 1], -1).astype(np.float32)
    gx = np.zeros_like(truth)
    gy = np.zeros_like(truth)
    gx[:, :-1] = truth[:, 1:] - truth[:, :-1]
    gy[:-1, :] = truth[1:, :] - truth[:-1, :]
    primal = (truth + rng.normal(scale=0.3, size=truth.shape)).astype(np.float32)
    fixed, res = agentray.poisson_reconstruct(ctx, primal, gx, gy, 0.2, A.POISSON_CG, 2000, 1.6, 1e-6,
                                              gdpt_flags=A.GDPT_CONSISTENT_DIVERGENCE)
    refsign, _ = agentray.poisson_reconstruct(ctx, primal, gx, gy, 0.2, A.POISSON_CG, 2000, 1.6, 1e-6)
    exact, _ = O.poisson_exact_f64(primal, -gx, -gy, 0.2)
    np.testing.assert_allclose(fixed, np.maximum(exact, 0), atol=5e-5 * np.abs(exact).max())
    err = lambda x: float(np.sqrt(np.mean((x - truth) ** 2)))
    assert err(fixed) < 0.25 * err(primal), (err(fixed), err(primal))
    assert err(refsign) > 3 * err(fixed), (err(refsign), err(fixed))

