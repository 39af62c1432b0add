"""Ground-truth checkpoints (metrics.GroundTruth.save / resume) on the CPU:
the FP64 sums and their sample count come back bit for bit, and a checkpoint
of another frame, scene or sampling is refused. The sums live on the device
in use; here they are host tensors, which the checkpoint code treats alike."""
import numpy as np
import pytest
import torch


def make_gt(w=5, h=3, seed=1001, spp=512, fill=None):
    from photon_tracer_b200.metrics import GroundTruth
    gt = GroundTruth.__new__(GroundTruth)
    gt.w, gt.h, gt.seed, gt.depth, gt.pass_spp, gt.first, gt.spp = w, h, seed, 10, 256, 1 << 20, spp
    gt.sum = torch.zeros((h, w, 3), dtype=torch.float64) if fill is None else fill.clone()
    return gt


def test_resume_restores_sums_and_samples(tmp_path):
    rng = np.random.default_rng(3)
    sums = torch.from_numpy(rng.random((3, 5, 3)) * 1e3)
    a = make_gt(fill=sums)
    path = str(tmp_path / "gt.npz")
    a.save(path, "room:1001")
    b = make_gt(spp=0)
    b.resume(path, "room:1001")
    assert b.spp == 512
    assert b.sum.numpy().tobytes() == sums.numpy().tobytes()
    assert np.array_equal(b.image(), a.image())


@pytest.mark.parametrize("field,value", [("w", 6), ("seed", 1002), ("pass_spp", 128), ("first", 0), ("depth", 5)])
def test_resume_refuses_another_frame(tmp_path, field, value):
    path = str(tmp_path / "gt.npz")
    make_gt().save(path, "room:1001")
    b = make_gt(spp=0)
    setattr(b, field, value)
    if field == "w":
        b.sum = torch.zeros((3, 6, 3), dtype=torch.float64)
    with pytest.raises(ValueError):
        b.resume(path, "room:1001")
    assert b.spp == 0


def test_resume_refuses_another_scene(tmp_path):
    path = str(tmp_path / "gt.npz")
    make_gt().save(path, "room:1001")
    with pytest.raises(ValueError):
        make_gt(spp=0).resume(path, "spheres:1001")


def test_save_replaces_the_checkpoint_whole(tmp_path):
    path = str(tmp_path / "gt.npz")
    make_gt(spp=256).save(path, "room:1001")
    make_gt(spp=768, fill=torch.ones((3, 5, 3), dtype=torch.float64)).save(path, "room:1001")
    b = make_gt(spp=0)
    b.resume(path, "room:1001")
    assert b.spp == 768 and float(b.sum.sum()) == 45.0
    assert not (tmp_path / "gt.npz.tmp").exists()


class FakeGT:
    """Stands in for GroundTruth in bench.extend_ground_truth: add() counts
    passes, save() / resume() record their calls."""

    def __init__(self):
        self.w, self.h, self.pass_spp, self.spp = 1920, 1080, 256, 0
        self.saved, self.resumed = [], []

    def add(self, passes):
        self.spp += passes * self.pass_spp

    def save(self, path, tag):
        self.saved.append((path, tag, self.spp))
        open(path, "wb").close()

    def resume(self, path, tag):
        self.resumed.append((path, tag))
        self.spp = 4096


def args_for(tmp_path, gt_spp, budget=None):
    import argparse
    return argparse.Namespace(gt_cache=str(tmp_path / "gt"), gt_spp=gt_spp, gt_budget_s=budget, gt_only=True)


def test_extend_saves_every_16_passes_and_at_the_end(tmp_path):
    import time
    import bench
    gt = FakeGT()
    assert bench.extend_ground_truth(gt, args_for(tmp_path, 40 * 256), "room", 1001, time.perf_counter())
    assert gt.spp == 40 * 256
    assert [s[2] for s in gt.saved] == [16 * 256, 32 * 256, 40 * 256]
    assert gt.saved[0][0].endswith("gt_room_1001_1920x1080.npz") and gt.saved[0][1] == "room:1001"
    assert gt.resumed == []


def test_extend_resumes_an_existing_checkpoint(tmp_path):
    import time
    import bench
    (tmp_path / "gt").mkdir()
    (tmp_path / "gt" / "gt_room_1001_1920x1080.npz").write_bytes(b"")
    gt = FakeGT()
    assert bench.extend_ground_truth(gt, args_for(tmp_path, 4096 + 512), "room", 1001, time.perf_counter())
    assert gt.resumed and gt.spp == 4096 + 512 and gt.saved[-1][2] == 4096 + 512


def test_extend_stops_at_its_time_budget(tmp_path):
    import time
    import bench
    gt = FakeGT()
    assert not bench.extend_ground_truth(gt, args_for(tmp_path, 65536, budget=0.0), "room", 1001,
                                         time.perf_counter() - 1.0)
    assert gt.spp == 0 and gt.saved == []
