"""Multi-GPU rendering and inverse rendering: one process per GPU, the image
split into row bands.

The reference renders one image per process on the CPU (renderer/src/
renderer.rs: rayon over the pixels); here a job can span several GPUs, each
rank rendering the rows of its band through `tpt_render_pixels_device` and the
bands gathered into one image (NCCL all-gather over NVLink; gloo on CPU in the
tests).  Pixel streams depend only on (pixel, sample), so the gathered image
is bit-identical to a one-GPU render of the whole job.

The adjoint shards the same way: each rank replays the paths of its band
(`tpt_adjoint_desc.first_pixel/num_pixels`, dLoss/dimage of its band only) and
the FP64 gradients are summed with one all-reduce, which equals the one-GPU
gradient up to the order of the FP64 sums.

torch.distributed is the plumbing only; every pixel is rendered by the
library's kernels.
"""
from __future__ import annotations

import torch
import torch.distributed as dist

import tpt


def pixel_band(rank: int, world: int, width: int, height: int) -> tuple[int, int]:
    """(first_pixel, num_pixels) of `rank`'s band: rows
    [rank*height//world, (rank+1)*height//world), so bands differ by one row at most."""
    if not 0 <= rank < world:
        raise ValueError("rank outside [0, world)")
    r0, r1 = rank * height // world, (rank + 1) * height // world
    return r0 * width, (r1 - r0) * width


def _world(group):
    if dist.is_available() and dist.is_initialized():
        return dist.get_rank(group), dist.get_world_size(group)
    return 0, 1


def gather_bands(band: torch.Tensor, width: int, height: int, group=None) -> torch.Tensor:
    """All-gathers every rank's band (float32 [num_pixels*3], from `pixel_band`)
    into the image float32 [height, width, 3] on every rank.  The bands are
    padded to the tallest band's size for the collective."""
    rank, world = _world(group)
    first, n = pixel_band(rank, world, width, height)
    if band.numel() != n * 3:
        raise ValueError("band size does not match pixel_band")
    if world == 1:
        return band.view(height, width, 3)
    rows_max = -(-height // world)
    padded = torch.zeros(rows_max * width * 3, dtype=torch.float32, device=band.device)
    padded[: n * 3] = band
    out = torch.empty(world * padded.numel(), dtype=torch.float32, device=band.device)
    dist.all_gather_into_tensor(out, padded, group=group)
    out = out.view(world, -1)
    image = torch.empty(height * width * 3, dtype=torch.float32, device=band.device)
    for r in range(world):
        f, k = pixel_band(r, world, width, height)
        image[f * 3:(f + k) * 3] = out[r, : k * 3]
    return image.view(height, width, 3)


def sum_gradients(grad: torch.Tensor, group=None) -> torch.Tensor:
    """Sums each rank's float64 material gradients in place (one all-reduce)."""
    if grad.dtype != torch.float64:
        raise TypeError("gradients are float64")
    _, world = _world(group)
    if world > 1:
        dist.all_reduce(grad, op=dist.ReduceOp.SUM, group=group)
    return grad


def render_sharded(scene: "tpt.Scene", job, group=None, stream=None) -> torch.Tensor:
    """The job's image float32 [height, width, 3] on this rank's GPU: this rank
    renders its band, then the bands are all-gathered."""
    rank, world = _world(group)
    first, n = pixel_band(rank, world, job.width, job.height)
    band = torch.empty(n * 3, dtype=torch.float32, device="cuda")
    s = stream if stream is not None else torch.cuda.current_stream().cuda_stream
    if n:
        scene.render_pixels_device(job, first, n, band.data_ptr(), s)
    return gather_bands(band, job.width, job.height, group)


def adjoint_sharded(scene: "tpt.Scene", job, d_image: torch.Tensor, mask: int = 0, fd_step: float = 0.0,
                    group=None, stream=None) -> torch.Tensor:
    """dLoss/d(material parameters), float64 [n_materials, 7], summed over the
    ranks.  d_image: dLoss/dimage float32 [height, width, 3] (whole image; each
    rank reads its band) on this rank's GPU."""
    rank, world = _world(group)
    first, n = pixel_band(rank, world, job.width, job.height)
    d = d_image.contiguous().view(-1)
    if d.numel() != job.width * job.height * 3:
        raise ValueError("d_image must cover the whole image")
    band = d[first * 3:(first + n) * 3].contiguous()
    grad = torch.zeros(scene.n_materials * tpt.GRAD_PARAMS, dtype=torch.float64, device="cuda")
    s = stream if stream is not None else torch.cuda.current_stream().cuda_stream
    if n:
        scene.adjoint_device(job, band.data_ptr(), grad.data_ptr(), mask, fd_step, s, first_pixel=first,
                             num_pixels=n)
    return sum_gradients(grad, group).view(scene.n_materials, tpt.GRAD_PARAMS)
