"""Failure detection without a GPU fault: a bounded device wait that runs out
reports RB_ERR_DEVICE_TIMEOUT and leaves the context usable; an injected
host-side allocation failure surfaces as RB_ERR_OUT_OF_MEMORY and the next
call succeeds; a truncated checkpoint is refused. Nothing here traps, faults
or hangs the device."""
import numpy as np
import pytest

import rainbow_b200 as rb

pytestmark = pytest.mark.gpu

RB_ERR_OUT_OF_MEMORY, RB_ERR_CHECKPOINT, RB_ERR_DEVICE_TIMEOUT = 3, 9, 10


def test_bounded_wait_runs_out_and_context_stays_usable():
    scene = rb.generate_scene(rb.RB_SCENE_BOX, width=16, height=16)
    with rb.Context(0) as ctx:
        assert ctx.check_bounded_wait(2000) == RB_ERR_DEVICE_TIMEOUT
        ctx.upload(scene)
        img = ctx.render(scene.camera, 4, max_depth=5)
        assert ctx.stats().device_error == 0 and np.isfinite(img).all() and img.mean() > 0


@pytest.mark.parametrize("after", [0, 3, 9])
def test_allocation_failure_is_reported_and_recoverable(after):
    scene = rb.generate_scene(rb.RB_SCENE_SPHERES, seed=2, width=32, height=32, num_spheres=8, subdivision=2)
    with rb.Context(0) as ctx:
        try:
            rb.inject_allocation_failure(after)
            with pytest.raises(rb.RbError) as e:
                ctx.upload(scene)
                ctx.render(scene.camera, 2, max_depth=5)
            assert e.value.status == RB_ERR_OUT_OF_MEMORY
        finally:
            rb.inject_allocation_failure(-1)
        ctx.upload(scene)
        ref = ctx.render(scene.camera, 2, max_depth=5, seed=1)
    with rb.Context(0) as fresh:
        fresh.upload(scene)
        assert np.array_equal(ref, fresh.render(scene.camera, 2, max_depth=5, seed=1))


def test_truncated_checkpoint_is_refused(tmp_path):
    scene = rb.generate_scene(rb.RB_SCENE_BOX, width=16, height=16)
    with rb.Context(0) as ctx:
        ctx.upload(scene)
        ctx.render(scene.camera, 4, max_depth=5, want_image=False)
        path = tmp_path / "ck.bin"
        ctx.checkpoint_save(str(path))
        data = path.read_bytes()
        path.write_bytes(data[:-100])
        with pytest.raises(rb.RbError) as e:
            ctx.checkpoint_load(str(path))
        assert e.value.status == RB_ERR_CHECKPOINT
        ctx.render(scene.camera, 4, max_depth=5, want_image=False)
        assert ctx.stats().device_error == 0


def test_cpp_program_on_the_c_abi():
    """A C++ program using only include/rbgpu.h: single render, batched render of
    two scenes, and the batch's box film equal to the single render's."""
    import os
    import subprocess
    exe = os.path.join(os.path.dirname(os.path.abspath(__file__)), "native", "c_abi_example")
    out = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0 and out.stdout.startswith("ok "), out.stdout + out.stderr
