"""Multi-rank path: each rank renders its own range of sample indices of the
same image (weak scaling, no collective on the data path) and one all-reduce
sums the film (rainbow_b200.distributed, the code bench.py --gpus N runs over
NCCL). Run here as two gloo ranks on the CPU, each rank rendering with the C
restatement; the reduced film must equal a single-process render of the
union of the sample ranges."""
import os
import socket

import numpy as np
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import rainbow_b200 as rb
from oracle import port
from rainbow_b200.distributed import reduce_film_tensors, sample_range

SPP_PER_RANK = 4


def _worker(rank, world, port_no, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port_no)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    scene = rb.generate_scene(rb.RB_SCENE_BOX, width=16, height=16)
    sb = scene.with_bvh(rb.build_bvh(scene))
    first, n = sample_range(rank, SPP_PER_RANK)
    s, q, _ = port.render(sb, scene.camera, n, first, 5, 1.0, seed=0, threads=1)
    ts, tq = torch.from_numpy(s.ravel().copy()), torch.from_numpy(q.ravel().copy())
    tc = torch.full((16 * 16,), n, dtype=torch.int32)
    reduce_film_tensors(ts, tq, tc)
    if rank == 0:
        out.put((np.concatenate([ts.numpy(), tq.numpy()]), tc.numpy()))
    dist.barrier()
    dist.destroy_process_group()


def _free_port():
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        return sk.getsockname()[1]


def test_two_rank_sample_ranges_reduce_to_single_render():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port_no = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port_no, q)) for r in range(2)]
    for p in procs:
        p.start()
    reduced, counts = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    scene = rb.generate_scene(rb.RB_SCENE_BOX, width=16, height=16)
    sb = scene.with_bvh(rb.build_bvh(scene))
    s, sq, _ = port.render(sb, scene.camera, 2 * SPP_PER_RANK, 0, 5, 1.0, seed=0, threads=2)
    want = np.concatenate([s.ravel(), sq.ravel()])
    np.testing.assert_allclose(reduced, want, rtol=1e-12, atol=1e-12)
    assert (counts == 2 * SPP_PER_RANK).all()


def test_sample_ranges_are_disjoint_and_cover():
    ranges = [sample_range(r, 8) for r in range(4)]
    covered = sorted(i for f, n in ranges for i in range(f, f + n))
    assert covered == list(range(32))
