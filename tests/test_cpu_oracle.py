"""CPU tests: the oracle against known answers and analytic cases, and the
C-ABI library surface.  No GPU needed."""
import math
import re
import os

import numpy as np
import pytest

import oracle as O
import agentray.scenes as S
from agentray import _abi as A
from agentray.scene_data import integrator_cfg

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_splitmix64_known_answers():
    # Published SplitMix64 sequence for seed 1234567 (Vigna); the oracle seeds
    # its xoshiro256++ state with this generator.
    def splitmix(state):
        out = []
        for _ in range(5):
            state = (state + 0x9E3779B97F4A7C15) & (2**64 - 1)
            z = state
            z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & (2**64 - 1)
            z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & (2**64 - 1)
            out.append(z ^ (z >> 31))
        return out
    assert splitmix(1234567) == [6457827717110365317, 3203168211198807973, 9817491932198370423,
                                 4593380528125082431, 16408922859458223821]


def test_xoshiro_stream_matches_python_restatement():
    # Pixel (3, 5) of IndependentSampler::seeded_for_pixel (src/sampler.rs:79-83).
    M = 2**64 - 1
    seed = ((5 * 2654435761) ^ (3 * 805459861)) & M
    s = []
    st = seed
    for _ in range(4):
        st = (st + 0x9E3779B97F4A7C15) & M
        z = st
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M
        s.append(z ^ (z >> 31))
    rotl = lambda x, k: ((x << k) | (x >> (64 - k))) & M
    vals = []
    for _ in range(8):
        r = (rotl((s[0] + s[3]) & M, 23) + s[0]) & M
        t = (s[1] << 17) & M
        s[2] ^= s[0]; s[3] ^= s[1]; s[1] ^= s[2]; s[0] ^= s[3]; s[2] ^= t; s[3] = rotl(s[3], 45)
        vals.append(np.float32((r >> 32) >> 8) * np.float32(1.0 / 16777216.0))
    np.testing.assert_array_equal(O.xoshiro_f32(3, 5, 8), np.array(vals, np.float32))


def test_sampling_sincos_accuracy():
    # ar_trig.h (shared by the FP32 oracle and the kernels): every sampling
    # angle 2*pi*u, u in [0, 1), within 1.5e-7 of float64 sin/cos; exact at
    # the quadrant points; |s|, |c| <= 1.
    rng = np.random.default_rng(5)
    u = np.concatenate([rng.uniform(0, 1, 2_000_000), np.arange(1 << 16) / (1 << 16)]).astype(np.float32)
    x = (np.float32(2 * math.pi) * u).astype(np.float32)
    s, c = O.sincos_f32(x)
    xd = x.astype(np.float64)
    assert np.abs(s - np.sin(xd)).max() < 1.5e-7
    assert np.abs(c - np.cos(xd)).max() < 1.5e-7
    assert np.abs(s).max() <= 1.0 and np.abs(c).max() <= 1.0
    s0, c0 = O.sincos_f32(np.zeros(1, np.float32))
    assert s0[0] == 0.0 and c0[0] == 1.0


def test_counter_sampler_range_and_independence():
    u = O.counter_u01(7, 12345, 3, 0, 100000)
    assert u.min() >= 0.0 and u.max() < 1.0
    assert abs(u.mean() - 0.5) < 0.005
    v = O.counter_u01(7, 12346, 3, 0, 100000)
    assert abs(np.corrcoef(u, v)[0, 1]) < 0.02


def _brute_force(pos, idx, o, d, tmin, tmax):
    v0 = pos[idx[:, 0]].astype(np.float64)
    e1 = pos[idx[:, 1]].astype(np.float64) - v0
    e2 = pos[idx[:, 2]].astype(np.float64) - v0
    dn = d / np.linalg.norm(d)
    h = np.cross(dn, e2)
    a = np.einsum("ij,ij->i", e1, h)
    ok = np.abs(a) >= 1e-8
    f = np.where(ok, 1.0 / np.where(ok, a, 1.0), 0.0)
    s = o - v0
    u = f * np.einsum("ij,ij->i", s, h)
    q = np.cross(s, e1)
    v = f * (q @ dn)
    t = f * np.einsum("ij,ij->i", e2, q)
    hit = ok & (u >= 0) & (u <= 1) & (v >= 0) & (u + v <= 1) & (t >= tmin) & (t <= tmax)
    if not hit.any():
        return 0xFFFFFFFF, np.inf
    k = np.argmin(np.where(hit, t, np.inf))
    return k, t[k]


def test_oracle_bvh_matches_brute_force():
    sc = S.triangle_soup(3000, seed=11)
    osc = O.OracleScene(sc)
    ot, dt = S.soup_rays(400, seed=12)
    r = osc.trace_closest(ot, dt)
    pos, idx = sc.meshes[0].positions, sc.meshes[0].indices
    agree = 0
    for i in range(ot.shape[0]):
        k, t = _brute_force(pos, idx, ot[i, :3].astype(np.float64), dt[i, :3].astype(np.float64), 1e-4, np.inf)
        if k == r["prim"][i] or (k != 0xFFFFFFFF and abs(t - r["t"][i]) <= 1e-5 * max(1, t)):
            agree += 1
    assert agree == ot.shape[0]


def test_oracle_any_hit_consistent_with_closest():
    sc = S.triangle_soup(5000, seed=5)
    osc = O.OracleScene(sc)
    ot, dt = S.soup_rays(2000, seed=6, tmax=0.25)
    occ = osc.trace_any(ot, dt)
    r = osc.trace_closest(ot, dt)
    np.testing.assert_array_equal(occ.astype(bool), r["prim"] != 0xFFFFFFFF)


def test_oracle_furnace_direct_lighting():
    # Point light at the centre of a closed Lambertian sphere: one bounce gives
    # L = albedo / pi * I / r^2 (r ~ 1 for the icosphere facets).
    sc, cam = S.furnace(albedo=0.5)
    osc = O.OracleScene(sc, precision=64)
    img = osc.render(cam, integrator_cfg(A.INTEGRATOR_PT, spp=2, max_depth=1), 16, 16)
    expect = 0.5 / math.pi
    assert np.allclose(img, expect, rtol=0.02)


def test_oracle_furnace_multibounce():
    # With D bounces the interior radiance is albedo/pi * I/r^2 * sum_{k<D} albedo^k.
    sc, cam = S.furnace(albedo=0.5)
    osc = O.OracleScene(sc, precision=64)
    img = osc.render(cam, integrator_cfg(A.INTEGRATOR_PT, spp=64, max_depth=4, rr_depth=10), 16, 16)
    expect = 0.5 / math.pi * sum(0.5 ** k for k in range(4))
    assert abs(img.mean() - expect) / expect < 0.03


def test_oracle_poisson_sor_converges_to_exact_solution():
    rng = np.random.default_rng(0)
    h, w = 24, 32
    primal = rng.uniform(0.0, 1.0, (h, w, 3)).astype(np.float32)
    gx = (rng.normal(size=(h, w, 3)) * 0.1).astype(np.float32)
    gy = (rng.normal(size=(h, w, 3)) * 0.1).astype(np.float32)
    gx[:, -1] = 0
    gy[-1, :] = 0
    exact, res = O.poisson_exact_f64(primal, gx, gy, 0.2)
    assert res < 1e-10
    sor = O.poisson_sor_f32(primal, gx, gy, 0.2, 400, 1.6)
    np.testing.assert_allclose(sor, np.maximum(exact, 0), atol=2e-4)


def test_oracle_gdpt_gradients_are_zero_on_border():
    sc, cam = S.cornell_box(1)
    osc = O.OracleScene(sc)
    img, primal, dx, dy = osc.render(cam, integrator_cfg(A.INTEGRATOR_GDPT, spp=2), 16, 12, gdpt_films=True)
    assert np.all(dx[:, -1] == 0) and np.all(dy[-1, :] == 0)
    assert np.all(img >= 0)


def test_oracle_gdpt_divergence_sign():
    """The reference's Poisson right-hand side (+div G) pulls the GDPT image
    away from the PT image; the consistent sign (-div G, an opt-in extension)
    lands on it."""
    sc, cam = S.cornell_box(1)
    w, h = 24, 20
    osc = O.OracleScene(sc)
    pt = osc.render(cam, integrator_cfg(A.INTEGRATOR_PT, spp=256, max_depth=6, seed=1), w, h)
    ref_sign = osc.render(cam, integrator_cfg(A.INTEGRATOR_GDPT, spp=32, max_depth=6, seed=2), w, h)
    fixed = osc.render(cam, integrator_cfg(A.INTEGRATOR_GDPT, spp=32, max_depth=6, seed=2,
                                           gdpt_flags=A.GDPT_CONSISTENT_DIVERGENCE), w, h)
    err = lambda x: float(np.mean(np.abs(x - pt)))
    assert err(fixed) < 0.2 * err(ref_sign), (err(fixed), err(ref_sign))


def test_header_symbols_exported():
    import ctypes
    from agentray import _lib
    header = open(os.path.join(ROOT, "include", "agentray.h")).read()
    decls = set(re.findall(r"^\s*(?:const\s+)?\w+\*?\s+\**(ar_\w+)\s*\(", header, re.M))
    assert decls, "no declarations parsed"
    lb = ctypes.CDLL(_lib.LIB_PATH)
    for name in decls:
        assert hasattr(lb, name), name
    assert decls == set(_lib.SIGNATURES), decls ^ set(_lib.SIGNATURES)
    assert lb.ar_abi_version() == 1


def test_oracle_dielectric_scene_is_finite_and_transmits():
    # The glass Cornell box renders finite values, and the glass lets light
    # through: pixels behind the glass sphere are not black.
    sc, cam = S.cornell_box(1, glass=True)
    osc = O.OracleScene(sc)
    img = osc.render(cam, integrator_cfg(A.INTEGRATOR_PT, spp=32, max_depth=8, seed=3), 24, 24)
    assert np.isfinite(img).all()
    assert img.mean() > 0.05
    # swapping the glass for an opaque black-free Lambertian changes the image
    plain, _ = S.cornell_box(1)
    other = O.OracleScene(plain).render(cam, integrator_cfg(A.INTEGRATOR_PT, spp=32, max_depth=8, seed=3), 24, 24)
    assert np.abs(img - other).mean() > 1e-3


def test_header_is_plain_c_with_ctypes_layouts(tmp_path):
    # The boundary header compiles as strict C99 (what cgo / bindgen / a C
    # caller sees), and its struct sizes equal the Python mirror's.
    import subprocess
    from agentray import _abi as A
    structs = {"ar_mesh_desc": A.MeshDesc, "ar_object_desc": A.ObjectDesc, "ar_material_desc": A.MaterialDesc,
               "ar_texture_desc": A.TextureDesc, "ar_light_desc": A.LightDesc, "ar_scene_desc": A.SceneDesc,
               "ar_camera_desc": A.CameraDesc, "ar_integrator_cfg": A.IntegratorCfg, "ar_ray_batch": A.RayBatch,
               "ar_hit": A.Hit, "ar_accel_opts": A.AccelOpts, "ar_scene_stats": A.SceneStats,
               "ar_tuning": A.Tuning, "ar_tune_opts": A.TuneOpts, "ar_tune_result": A.TuneResult,
               "ar_server_opts": A.ServerOpts, "ar_job_info": A.JobInfo, "ar_server_stats": A.ServerStats,
               "ar_render_stats": A.RenderStats}
    src = tmp_path / "h.c"
    src.write_text('#include <stdio.h>\n#include "agentray.h"\nint main(void) {\n' +
                   "".join(f'    printf("%zu\\n", sizeof({n}));\n' for n in structs) + "    return 0;\n}\n")
    exe = tmp_path / "h"
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Wextra", "-Werror", "-pedantic",
                    "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    sizes = [int(x) for x in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()]
    import ctypes
    assert sizes == [ctypes.sizeof(t) for t in structs.values()], dict(zip(structs, sizes))
