"""Ground truth built over two runs equals one built in a single run: FP64
sums of 2 passes saved, resumed into a new GroundTruth and extended by 2 more
passes are bit-identical to 4 passes in one go (the resumed passes continue
the per-pixel sample numbers)."""
import pytest


@pytest.mark.gpu
def test_resumed_ground_truth_equals_an_uninterrupted_one(built, tmp_path):
    import torch
    import photon_tracer_b200 as pt
    from photon_tracer_b200 import abi, metrics
    torch.cuda.set_device(0)
    g = pt.Generated(abi.PT_GEN_RANDOM_SPHERES, seed=1001)
    scene = pt.Scene(g)
    w, h = 400, 225
    whole = metrics.GroundTruth(scene, g.camera, w, h, seed=1001, pass_spp=64)
    whole.add(4)
    first = metrics.GroundTruth(scene, g.camera, w, h, seed=1001, pass_spp=64)
    first.add(2)
    path = str(tmp_path / "gt.npz")
    first.save(path, "spheres:1001")
    resumed = metrics.GroundTruth(scene, g.camera, w, h, seed=1001, pass_spp=64)
    resumed.resume(path, "spheres:1001")
    resumed.add(2)
    scene.close()
    assert resumed.spp == whole.spp == 256
    assert resumed.sum.cpu().numpy().tobytes() == whole.sum.cpu().numpy().tobytes()
