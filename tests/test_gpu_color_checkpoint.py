"""Checkpoint and resume of the learned colour stage on the GPU: a run of 2 x 150 Adam steps with
a save and a load between them gives the model of one 300-step run bit for bit (parameters,
latents, the loss of every step, the gate's statistics), a loaded model renders exactly what the
saved one rendered, and a checkpoint is refused for a scene of another size."""
import numpy as np
import pytest

from helpers import tile_raster_camera

pytestmark = pytest.mark.gpu


def test_resume_from_a_checkpoint_equals_one_run(gpu, tmp_path):
    from gsr_b200 import scenes

    scene = scenes.make_scene(30_000, seed=21, ball_radius=3.0)
    gs = gpu.GpuScene(scene)
    kw = dict(batch=8192, directions=32, seed=3, gate=0.05)
    whole = gpu.ColorModel(gs, steps=300, **kw)
    first = gpu.ColorModel(gs, steps=150, **kw)
    path = tmp_path / "half.gsrc"
    first.save(path)
    ck = gpu.read_color_checkpoint(path)
    assert ck["step"] == 150 and ck["count"] == scene.count and ck["loss"].size == 150
    loaded = gpu.ColorModel.load(gs, path)
    # the loaded model renders what the saved one rendered
    cam = tile_raster_camera()
    images = []
    for m in (first, loaded):
        r = gpu.Renderer(gs, gpu.Settings(adaptive_list=False))
        r.set_color_model(m)
        r.render(cam)
        images.append(r.read_back_image())
        r.close()
    assert np.array_equal(images[0], images[1])
    loaded.resume(150)
    a, b = whole.read(), loaded.read()
    for x, y, name in zip(a, b, ("latents", "params", "loss")):
        assert x.tobytes() == y.tobytes(), name
    sa, sb = whole.stats(), loaded.stats()
    for k in ("steps", "fallback", "first_loss", "final_loss", "max_error_kept"):
        assert sa[k] == sb[k], k
    # a checkpoint for another scene
    other = gpu.GpuScene(scenes.make_scene(1000, seed=1, ball_radius=3.0))
    with pytest.raises(gpu.GsrError):
        gpu.ColorModel.load(other, path)
    for m in (whole, first, loaded):
        m.close()
    other.close()
    gs.close()
