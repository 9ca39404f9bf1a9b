"""Renders over several GPUs: sample ranges per rank and one film reduction.

Pixels and samples are independent, so every rank renders the whole image
with its own range of sample indices (weak scaling: no collective while
rendering), then the ranks sum their FP64 film accumulators once. The
reduction is a torch.distributed all-reduce (NCCL over NVLink / NVSwitch on
GPUs; gloo on CPU tensors in the tests) of the accumulators that
rb_film_to_device copies out of each context; rb_film_from_device puts the
sums back, so every rank's context then holds the film of all the samples.
"""
from __future__ import annotations

import ctypes as C

from ._native import check, lib


def sample_range(rank: int, spp: int, stride: int | None = None) -> tuple:
    """First sample index and count of `rank` when every rank renders `spp`
    samples per pixel; ranks start `stride` (default spp) indices apart."""
    return rank * (spp if stride is None else stride), spp


def reduce_film_tensors(sum_rgb, sum_sq_rgb, count, group=None) -> None:
    """Sums the three accumulator tensors over the ranks of `group`, in place,
    in a fixed order (sums, squared sums, counts). Counts are int32 (the
    per-pixel uint32 counts stay below 2^31)."""
    import torch.distributed as dist
    for t in (sum_rgb, sum_sq_rgb, count):
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)


def reduce_context_film(ctx, samples_per_pixel: int, group=None) -> None:
    """All-reduces the film of `ctx` (a rainbow_b200.Context on this rank's GPU)
    over `group`; afterwards the context's film holds every rank's samples,
    `samples_per_pixel` of them per pixel in total."""
    import torch
    w, h = ctx._last_camera_shape()
    dev = torch.device("cuda", torch.cuda.current_device())
    s = torch.empty(3 * w * h, dtype=torch.float64, device=dev)
    q = torch.empty_like(s)
    c = torch.empty(w * h, dtype=torch.int32, device=dev)
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    L = lib()
    check(L.rb_film_to_device(ctx._h, s.data_ptr(), q.data_ptr(), c.data_ptr(), stream), "rb_film_to_device")
    reduce_film_tensors(s, q, c, group)
    check(L.rb_film_from_device(ctx._h, s.data_ptr(), q.data_ptr(), c.data_ptr(), samples_per_pixel, stream),
          "rb_film_from_device")
