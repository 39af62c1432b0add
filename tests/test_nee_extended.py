"""The extended light sampling (PT_FLAG_NEE_EXTENDED), beyond the reference,
whose known limits it lifts (README.md:453-456): emissive triangles join the
sphere lights, and rough metal samples the lights too, weighted against its
own scattered ray by the power heuristic. CPU checks of the oracle's
restatement: the metal lobe's density against the scatter itself, and the
estimator against plain path tracing. GPU parity is in
tests/test_gpu_nee_extended.py, GPU convergence in tests/test_gpu_converge.py."""
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest


@pytest.mark.parametrize("fuzz", [0.05, 0.25, 0.7, 1.0])
def test_metal_lobe_density_matches_the_scatter(built, fuzz):
    """metal::scatter sends mirror + fuzz * (a point uniform in the unit ball)
    (include/material.hpp:85-91). The density the estimator uses for it,
    checked against the fraction of 400,000 such scatters that land in small
    cones around probe directions."""
    from oracle.oracle import oracle_metal_lobe_pdf
    rng = np.random.default_rng(7)
    r = np.array([0.3, 0.8, -0.2])
    r = (r / np.linalg.norm(r)).astype(np.float32)
    n = 400000
    u = rng.normal(size=(n, 3))
    u *= (rng.random(n) ** (1 / 3) / np.linalg.norm(u, axis=1))[:, None]
    x = r + fuzz * u
    w = x / np.linalg.norm(x, axis=1)[:, None]
    half = 0.1 * fuzz
    cap = 1 - np.cos(half)
    for probe in w[:6]:
        frac = float((w @ probe > 1 - cap).mean())
        pdf = oracle_metal_lobe_pdf(r, fuzz, probe.astype(np.float32))
        est = frac / (2 * np.pi * cap)
        hits = frac * n
        assert abs(est - pdf) <= 5 * est / np.sqrt(max(hits, 1)) + 0.02 * pdf, (fuzz, est, pdf, hits)
    assert oracle_metal_lobe_pdf(r, fuzz, (-r).astype(np.float32)) == 0.0


def image_mean(built, nee, flags, seed, spp, w=64, h=36):
    from oracle.oracle import Oracle
    from photon_tracer_b200 import abi
    g = built.Generated(abi.PT_GEN_MESH_LIGHT)
    g.desc.sample_lights = nee
    o = Oracle(g.desc)
    o.render(g.camera, w, h, 1, 10, seed=seed, rows=1)  # the sampler's tables, once

    def rows(j0):
        return o.render(g.camera, w, h, spp, 10, seed=seed, row0=j0, rows=4, flags=flags)[0]
    with ThreadPoolExecutor(8) as ex:
        img = sum(ex.map(rows, range(0, h, 4)))
    return img.reshape(-1, 3).mean(axis=0, dtype=np.float64)


def test_extended_estimator_converges_to_plain_path_tracing(built):
    """The room lit by emissive triangle meshes, rough metal and a mirror:
    the oracle's extended estimate and plain path tracing (no light
    sampling) agree in the image mean per channel within 1% and within the
    noise (|z| <= 5); the extended estimate is the less noisy one."""
    ext = np.array([image_mean(built, 1, 1, 100 + k, 512) for k in range(4)])
    plain = np.array([image_mean(built, 0, 0, 200 + k, 512) for k in range(4)])
    me, mp = ext.mean(axis=0), plain.mean(axis=0)
    se = np.sqrt(ext.var(axis=0, ddof=1) / 4 + plain.var(axis=0, ddof=1) / 4)
    assert np.all(np.abs(me - mp) <= 1e-2 * mp), (me, mp)
    assert np.all(np.abs(me - mp) <= 5 * se), ((me - mp) / se)
    assert ext.std(axis=0).sum() < plain.std(axis=0).sum()


def test_flags_zero_renders_the_reference_estimator(built):
    """flags 0 is the reference's estimator: the oracle with flags 0 and its
    plain entry point give the same bytes."""
    from oracle.oracle import Oracle
    from photon_tracer_b200 import abi
    g = built.Generated(abi.PT_GEN_MESH_LIGHT)
    o = Oracle(g.desc)
    a = o.render(g.camera, 24, 16, 2, 10, seed=3, aux=True, flags=0)
    import ctypes as C
    out = np.zeros((16, 24, 3), np.float32)
    ax = np.zeros((16, 24, 7), np.float32)
    rays = C.c_uint64()
    o.lib.po_render(o.h, C.byref(g.camera), 24, 16, 2, 10, 3, 0, 0, None, 0, 16, out.ctypes.data_as(C.c_void_p),
                    ax.ctypes.data_as(C.c_void_p), C.byref(rays), None)
    assert a[0].tobytes() == out.tobytes() and a[1].tobytes() == ax.tobytes() and a[2] == rays.value
