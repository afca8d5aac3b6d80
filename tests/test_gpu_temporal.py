"""GPU parity of the temporal passes through the C ABI (RenderTemporalScene):
the primary-surface metadata and ReSTIR DI passes against the oracle's
restatement (bit for bit), reprojection and SVGF against the reference's own
CPU code (temporal.cpp) at the reference's published GPU tolerances."""

import numpy as np
import pytest

from hydra_lotus_b200 import abi, scenes
from oracle import oracle, ref

from parity import PathParity

pytestmark = pytest.mark.gpu

SIZE = 64
# The reference's GPU-vs-CPU tolerances for the SVGF passes
# (docs/reports/2026-10-18-svgf-filter.md): composite max relative error
# 1.2e-5 and variance max absolute error 9.3e-5 (for variances near 1; a
# relative 4e-6, 32 float ulps, covers large ones, such as the variance of
# 1000 a pixel of the disk-neighbour case reaches).
COMPOSITE_RTOL = 1.2e-5
VARIANCE_ATOL = 9.3e-5
VARIANCE_RTOL = 4e-6


def restir_room_lit():
    """The ReSTIR room with analytic lights besides its emissive triangles:
    a sphere, a small sphere, a rect, a disk, a distant and a parallel light
    (each a reservoir candidate; spheres by their whole area)."""
    s = scenes.restir_room(seed=0, size=SIZE, emitters=120)
    for light in scenes.lit_room(seed=0, size=SIZE).lights:
        s.lights.append(light)
    return s


def temporal_frames(integrator, spatial=True, frames=3, filter_iterations=5, cap=5, lit=False, neighbours=0,
                    radius=2):
    scene = restir_room_lit() if lit else scenes.restir_room(seed=0, size=SIZE, emitters=300)
    settings = abi.default_settings(integrator=integrator,
                                    light_sampling=abi.LIGHT_SAMPLING_RESTIR_INITIAL,
                                    max_bounces=4, sample_index=100, restir_candidates=8,
                                    restir_temporal=1, restir_max_history_candidates=20,
                                    restir_spatial=1 if spatial else 0, restir_spatial_radius=radius,
                                    restir_spatial_neighbours=neighbours)
    descs = []
    previous = None
    for k in range(frames):
        view, w2c = scenes.orbit_camera(k, frames=24)
        frame = abi.make_frame(w2c, SIZE, SIZE, settings, 1)
        d = abi.temporal_desc(frame, view, previous[0] if previous else None,
                              previous[1] if previous else None, history_available=k > 0,
                              accumulate_radiance=True, max_history_samples=cap,
                              filter_iterations=filter_iterations)
        descs.append(d)
        previous = (view, w2c)
    return scene, descs


def products(r, h, w, names):
    return {n: r.read_product(getattr(abi, "PRODUCT_" + n.upper()), h, w) for n in names}


def exact(a, b):
    return np.array_equal(np.frombuffer(a.tobytes(), np.uint8), np.frombuffer(b.tobytes(), np.uint8))


@pytest.mark.parametrize("integrator,lit,neighbours,radius", [
    (abi.INTEGRATOR_WAVEFRONT, False, 0, 2), (abi.INTEGRATOR_REFERENCE, False, 0, 2),
    (abi.INTEGRATOR_WAVEFRONT, True, 0, 2),
    # The disk mode: five neighbours drawn from a 30-pixel disk.
    (abi.INTEGRATOR_WAVEFRONT, False, 5, 30)])
def test_temporal_passes_match_checkers(cuda, integrator, lit, neighbours, radius):
    scene, descs = temporal_frames(integrator, lit=lit, neighbours=neighbours, radius=radius)
    o = oracle.OracleTemporalScene(scene)
    with cuda.CudaOffscreenRenderer(0) as r:
        cuda.check(r.update_scene(scene), "update_scene")
        for k, d in enumerate(descs):
            res, color = r.render_temporal(d)
            cuda.check(res, f"render_temporal frame {k}")
            p = products(r, SIZE, SIZE, ["surface", "previous_surface", "validity", "radiance",
                                         "previous_radiance", "batch", "restir_initial",
                                         "restir_temporal", "restir_previous", "restir_spatial",
                                         "restir_sources", "restir_surfaces",
                                         "restir_previous_surfaces"])
            tc = oracle.oracle_temporal(d)
            frame = d.frame
            si = frame.settings.sample_index + k  # the stream's batch sample index
            # Primary-surface metadata: bit for bit.
            want = o.temporal_surface(frame, tc)
            assert exact(p["surface"], want), f"frame {k}: temporal surface differs"
            # Reprojection: the reference's own ReprojectTemporalHistory.
            prev = p["previous_surface"] if k > 0 else np.zeros(0, dtype=abi.TEMPORAL_PIXEL)
            v = ref.reproject(p["surface"], prev, d.validation)
            assert exact(p["validity"], v), f"frame {k}: validity differs from the reference's"
            # ReSTIR passes, each from the GPU's own inputs: bit for bit.
            init = o.restir_initial(frame, tc, si)
            assert exact(p["restir_initial"], init), f"frame {k}: initial reservoirs differ"
            reuse, surf = o.restir_temporal(frame, tc, si, p["restir_initial"], p["validity"], p["surface"],
                                            p["restir_previous"], p["restir_previous_surfaces"])
            assert exact(p["restir_temporal"], reuse), f"frame {k}: temporal reservoirs differ"
            assert exact(p["restir_surfaces"], surf), f"frame {k}: reservoir surfaces differ"
            spatial, sources = o.restir_spatial(frame, tc, si, p["restir_temporal"], p["restir_surfaces"])
            assert exact(p["restir_spatial"], spatial), f"frame {k}: spatial reservoirs differ"
            assert np.array_equal(p["restir_sources"], sources)
            if k > 0:
                used = (reuse["previous_index"] != 0xFFFFFFFF).mean()
                assert used > 0.3, f"temporal reuse found history at only {used:.2f} of pixels"
            # The fresh batch: the path tracer with the final reservoirs at
            # its primary vertex.
            batch, _ = o.sample_restir(frame, si, p["restir_spatial"])
            pp = PathParity(p["batch"], batch)
            print(k, pp)
            pp.assert_ok()
            assert pp.exact > 0.99, pp
            # SVGF against the reference's CPU oracles.
            var = ref.estimate_variance(p["surface"], p["radiance"], 1, d.max_history_samples)
            np.testing.assert_allclose(p["radiance"]["variance"], var, rtol=VARIANCE_RTOL, atol=VARIANCE_ATOL)
            comp = ref.filter_composite(p["surface"], p["radiance"], 1, d.max_history_samples,
                                        d.filter_iterations)
            scale = np.maximum(np.abs(comp), 1e-3)
            rel = np.abs(color - comp) / scale
            assert rel.max() <= COMPOSITE_RTOL * 10, rel.max()
            assert np.percentile(rel, 99.9) <= COMPOSITE_RTOL, np.percentile(rel, 99.9)


def test_restir_converges_to_mis_path_tracer(cuda):
    """ReSTIR DI's primary direct light is unbiased: over independent
    initial-only frames, the image sum's mean matches the MIS path
    tracer's (a two-sample z-test on per-frame image sums)."""
    scene = scenes.restir_room(seed=1, size=32, emitters=100, sigma=0.5)
    view, w2c = scenes.orbit_camera(0)
    n = 400
    mis_sums, restir_sums = [], []
    with cuda.CudaOffscreenRenderer(0) as r:
        cuda.check(r.update_scene(scene), "update_scene")
        for k in range(n):
            mis = abi.default_settings(integrator=abi.INTEGRATOR_WAVEFRONT,
                                       light_sampling=abi.LIGHT_SAMPLING_MIS, max_bounces=2,
                                       sample_index=k)
            res, img = r.render_scene(abi.make_frame(w2c, 32, 32, mis, 1))
            cuda.check(res, "MIS frame")
            mis_sums.append(img[..., :3].sum())
            st = abi.default_settings(integrator=abi.INTEGRATOR_WAVEFRONT,
                                      light_sampling=abi.LIGHT_SAMPLING_RESTIR_INITIAL, max_bounces=2,
                                      sample_index=50000 + k, restir_candidates=8)
            res, img = r.render_temporal(abi.temporal_desc(abi.make_frame(w2c, 32, 32, st, 1), view))
            cuda.check(res, "ReSTIR frame")
            restir_sums.append(img[..., :3].sum())
    a, b = np.array(mis_sums), np.array(restir_sums)
    z = (a.mean() - b.mean()) / np.sqrt(a.var() / n + b.var() / n)
    print("MIS", a.mean(), "ReSTIR", b.mean(), "z", z, "variance ratio", b.var() / a.var())
    assert abs(z) < 4.0, z


def test_fp16_moments(cuda):
    """The FP16 moment mode (LOTUS_MOMENTS_FP16): the stored first moment is
    half-valued (on the fresh frame, the FP32 mode's rounded to half
    precision, saturating at 65504); the central second moment is kept at
    half precision, so the second moment the passes use stays within a few
    half rounding steps of the FP32 mode's (relative 4e-3, away from the
    saturation); the variance the GPU derives from the stored moments
    matches the reference's CPU EstimateTemporalVariance on the same moments
    at its published tolerances, and the composite stays within 5e-2 relMSE
    of the FP32 mode's (the a-trous edge-stopping weighs the variance, which
    keeps about 11 bits)."""
    scene, descs32 = temporal_frames(abi.INTEGRATOR_WAVEFRONT)
    _, descs16 = temporal_frames(abi.INTEGRATOR_WAVEFRONT)
    for d in descs16:
        d.moment_precision = abi.MOMENTS_FP16
    from hydra_lotus_b200 import metrics
    with cuda.CudaOffscreenRenderer(0) as r32, cuda.CudaOffscreenRenderer(0) as r16:
        cuda.check(r32.update_scene(scene), "update_scene")
        cuda.check(r16.update_scene(scene), "update_scene")
        for k, (d32, d16) in enumerate(zip(descs32, descs16)):
            res32, c32 = r32.render_temporal(d32)
            cuda.check(res32, "FP32 frame")
            res16, c16 = r16.render_temporal(d16)
            cuda.check(res16, "FP16 frame")
            p32 = products(r32, SIZE, SIZE, ["surface", "radiance"])
            p16 = products(r16, SIZE, SIZE, ["surface", "radiance"])
            a1, b1 = p32["radiance"]["moments"][..., 0], p16["radiance"]["moments"][..., 0]
            a2, b2 = p32["radiance"]["moments"][..., 1], p16["radiance"]["moments"][..., 1]
            assert np.array_equal(b1, b1.astype(np.float16).astype(np.float32), equal_nan=True)
            half1 = np.where(a1 > 65504.0, np.float32(65504.0), a1).astype(np.float16).astype(np.float32)
            if k == 0:
                assert np.array_equal(b1, half1, equal_nan=True)
            calm = (a2 < 1.0e4) & (a1 < 1.0e2)
            bad = calm & (np.abs(a2 - b2) > 4e-3 * np.abs(a2) + 1e-6)
            assert not bad.any(), (k, bad.sum(), a2[bad][:5], b2[bad][:5])
            var = ref.estimate_variance(p16["surface"], p16["radiance"], 1, d16.max_history_samples)
            np.testing.assert_allclose(p16["radiance"]["variance"], var, rtol=VARIANCE_RTOL, atol=VARIANCE_ATOL)
            err = metrics.relmse(c16, c32)
            print(k, "composite relMSE FP16 vs FP32", err)
            assert err <= 5e-2, err
