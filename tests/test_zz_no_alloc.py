"""ar_poisson_sor_static: the scratch-free Poisson solve for callers that must
not allocate device memory while they run (a frame loop, or a plugin whose
host application owns the whole device pool).  It must give the same image as
the allocating entry point, ar_poisson_reconstruct with the SOR solver, call
after call: its scratch is one static device array shared by all calls, so a
second call with another size must not see anything of the first.

Collected last (file name) so that a failure here comes after every other test
in a run that stops at the first failure."""
import ctypes as C

import numpy as np
import pytest

import agentray
from agentray import _abi as A
from agentray.scene_data import integrator_cfg

pytestmark = pytest.mark.gpu


def _films(h, w, seed):
    rng = np.random.default_rng(seed)
    primal = rng.uniform(0.0, 2.0, (h, w, 3)).astype(np.float32)
    gx = (rng.normal(size=(h, w, 3)) * 0.2).astype(np.float32)
    gy = (rng.normal(size=(h, w, 3)) * 0.2).astype(np.float32)
    gx[:, -1] = 0
    gy[-1, :] = 0
    return primal, gx, gy


def _static_sor(primal, gx, gy, alpha=0.2, iters=200, omega=1.6):
    import torch
    h, w, _ = primal.shape
    dev = [torch.from_numpy(a).cuda() for a in (primal, gx, gy)]
    out = torch.full((h, w, 3), -1.0, dtype=torch.float32, device="cuda")
    cfg = integrator_cfg(A.INTEGRATOR_GDPT, alpha=alpha, poisson_iterations=iters, sor_omega=omega,
                         poisson_solver=A.POISSON_SOR)
    stream = torch.cuda.current_stream()
    rc = agentray.lib().ar_poisson_sor_static(C.byref(cfg), w, h, dev[0].data_ptr(), dev[1].data_ptr(),
                                              dev[2].data_ptr(), out.data_ptr(), C.c_void_p(stream.cuda_stream))
    agentray.check(rc)
    torch.cuda.synchronize()
    return out.cpu().numpy()


def test_static_sor_matches_allocating_entry_point(ctx):
    # Two calls in a row with different sizes and data: each must equal the
    # allocating solver's output bit for bit (red-black SOR is order independent).
    for (h, w, seed) in ((200, 300, 11), (96, 128, 12)):
        primal, gx, gy = _films(h, w, seed)
        ref, _ = agentray.poisson_reconstruct(ctx, primal, gx, gy, 0.2, A.POISSON_SOR, 200, 1.6)
        got = _static_sor(primal, gx, gy)
        np.testing.assert_array_equal(got, ref)


def test_static_sor_rejects_images_beyond_its_scratch(ctx):
    import torch
    w, h = 1024, 512  # 2x the AR_STATIC_SOR_MAX_PIXELS limit of 512*512
    buf = torch.zeros(8, dtype=torch.float32, device="cuda")
    cfg = integrator_cfg(A.INTEGRATOR_GDPT, poisson_solver=A.POISSON_SOR)
    rc = agentray.lib().ar_poisson_sor_static(C.byref(cfg), w, h, buf.data_ptr(), buf.data_ptr(), buf.data_ptr(),
                                              buf.data_ptr(), None)
    assert rc == A.AR_ERR_INVALID_ARGUMENT
    assert b"exceeds the static scratch" in agentray.lib().ar_last_error()


def test_static_sor_rejects_other_solvers_and_host_pointers(ctx):
    # It solves with SOR only: a CG request is refused, not silently served by
    # SOR.  Host arrays are refused before any kernel could touch them.
    import torch
    buf = torch.zeros(16 * 16 * 3, dtype=torch.float32, device="cuda")
    p = buf.data_ptr()
    cg = integrator_cfg(A.INTEGRATOR_GDPT, poisson_solver=A.POISSON_CG)
    rc = agentray.lib().ar_poisson_sor_static(C.byref(cg), 16, 16, p, p, p, p, None)
    assert rc == A.AR_ERR_UNSUPPORTED
    host = np.zeros(16 * 16 * 3, np.float32)
    sor = integrator_cfg(A.INTEGRATOR_GDPT, poisson_solver=A.POISSON_SOR)
    rc = agentray.lib().ar_poisson_sor_static(C.byref(sor), 16, 16, p, p, p, host.ctypes.data, None)
    assert rc == A.AR_ERR_INVALID_ARGUMENT
    assert b"not device memory" in agentray.lib().ar_last_error()
