"""What the trained network gains: on held-out scenes (seeds never rendered
for training), a few-spp frame denoised by the committed U-Net weights is
compared with the same frame raw and filtered by the a-trous filter (the
reference's denoiser), against FP64 ground truth."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SIZE, SPP, GT_SPP = 256, 4, 4096


@pytest.fixture(scope="module")
def pt(built):
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return built


@pytest.mark.parametrize("kind,seed", [("spheres", 4001), ("room", 4002)])
def test_trained_unet_beats_raw_and_atrous(pt, kind, seed):
    from photon_tracer_b200 import denoiser, metrics
    net = denoiser.trained()
    g, scene, cam = denoiser.scene_and_camera(kind, seed, 1.0, jitter=True)
    gt = metrics.GroundTruth(scene, cam, SIZE, SIZE, seed=seed, pass_spp=256)
    gt.add(GT_SPP // 256)
    truth = gt.image()
    noisy, unet, _ = metrics.render_and_unet(net, scene, cam, SIZE, SIZE, SPP, seed)
    noisy2, atrous, _ = metrics.render_and_denoise(scene, cam, SIZE, SIZE, SPP, seed)
    np.testing.assert_array_equal(noisy, noisy2)  # the same frame goes to both denoisers
    e_raw, e_atrous, e_unet = (metrics.relmse(x, truth) for x in (noisy, atrous, unet))
    s_raw, s_atrous, s_unet = (metrics.ssim(x, truth) for x in (noisy, atrous, unet))
    print(f"{kind}: relMSE raw {e_raw:.4f} atrous {e_atrous:.4f} unet {e_unet:.4f}; "
          f"SSIM raw {s_raw:.3f} atrous {s_atrous:.3f} unet {s_unet:.3f}")
    assert e_unet < 0.25 * e_raw
    assert e_unet < e_atrous
    assert s_unet > max(s_raw, s_atrous)
