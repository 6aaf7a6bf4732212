"""Multi-GPU rendering and inverse rendering: one process per GPU, the image
split into row bands.

The reference renders one image per process on the CPU (renderer/src/
renderer.rs: rayon over the pixels); here a job can span several GPUs, each
rank rendering the rows of its band through `tpt_render_pixels_device` (equal
rows, or a cost-weighted static partition from a 1-sample pilot:
estimate_row_cost + balanced_bands) and the bands gathered into one image
(NCCL all-gather over NVLink; gloo on CPU in the tests).  Pixel streams depend only on (pixel, sample), so the gathered image
is bit-identical to a one-GPU render of the whole job.

The adjoint shards the same way: each rank replays the paths of its band
(`tpt_adjoint_desc.first_pixel/num_pixels`, dLoss/dimage of its band only) and
the FP64 gradients are summed with one all-reduce, which equals the one-GPU
gradient up to the order of the FP64 sums.

A batch of jobs splits by job instead (render_batch_sharded): a
longest-processing-time-first partition on the jobs' costs, each rank
rendering its jobs in one batched launch sequence.

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


def balanced_bands(row_cost, world: int) -> list[tuple[int, int]]:
    """Cost-weighted static partition: (first_row, rows) per rank, contiguous
    and in order, so that every band's summed row cost is close to
    total / world: the boundary after band r is the row boundary whose cost
    prefix is nearest to (r+1)/world of the total.  Bands may be empty when a
    few rows carry most of the cost."""
    import numpy as np

    c = np.asarray(row_cost, np.float64)
    if c.ndim != 1 or c.size == 0 or not np.all(np.isfinite(c)) or np.any(c < 0):
        raise ValueError("row costs: a non-empty vector of finite, non-negative numbers")
    if world < 1:
        raise ValueError("world >= 1")
    height = c.size
    prefix = np.concatenate([[0.0], np.cumsum(c)])
    total = prefix[-1]
    if total <= 0:
        return [(r * height // world, (r + 1) * height // world - r * height // world) for r in range(world)]
    ends = []
    for r in range(1, world):
        target = total * r / world
        k = int(np.searchsorted(prefix, target, side="left"))
        # the boundary row nearer the target: the band either ends before or after row k-1
        if k > 0 and abs(prefix[k - 1] - target) <= abs(prefix[k] - target):
            k -= 1
        ends.append(min(max(k, ends[-1] if ends else 0), height))
    bounds = [0] + ends + [height]
    return [(bounds[r], bounds[r + 1] - bounds[r]) for r in range(world)]


def estimate_row_cost(scene: "tpt.Scene", job, slabs: int = 0, group=None) -> "np.ndarray":
    """Per-row cost of `job` for balanced_bands, from a 1-sample pilot: the
    rows are cut into `slabs` equal slabs (default 4 per rank), rank s % world
    renders and times slab s on the device (CUDA events around
    tpt_render_pixels_device), the times are summed over the ranks, and each
    row gets its slab's time per row.  Every rank returns the same vector."""
    import numpy as np

    rank, world = _world(group)
    slabs = slabs or 4 * world
    slabs = max(1, min(slabs, job.height))
    pilot = tpt.RenderJob.from_buffer_copy(job)
    pilot.spp = 1
    width, height = job.width, job.height
    times = torch.zeros(slabs, dtype=torch.float64)
    out = torch.empty(-(-height // slabs) * width * 3, dtype=torch.float32, device="cuda")
    s = torch.cuda.current_stream()
    for k in range(rank, slabs, world):
        r0, r1 = k * height // slabs, (k + 1) * height // slabs
        if r1 == r0:
            continue
        scene.render_pixels_device(pilot, r0 * width, (r1 - r0) * width, out.data_ptr(), s.cuda_stream)  # warm
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        scene.render_pixels_device(pilot, r0 * width, (r1 - r0) * width, out.data_ptr(), s.cuda_stream)
        e1.record(s)
        e1.synchronize()
        times[k] = e0.elapsed_time(e1)
    if world > 1:
        t = times.to("cuda" if dist.get_backend(group) == "nccl" else "cpu")
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
        times = t.cpu()
    cost = np.empty(height, np.float64)
    for k in range(slabs):
        r0, r1 = k * height // slabs, (k + 1) * height // slabs
        if r1 > r0:
            cost[r0:r1] = float(times[k]) / (r1 - r0)
    return cost


def _stream_for(stream):
    """The raw stream the library launches on and a function that makes torch's
    current stream (where the collectives run) wait for it.  A caller's own
    stream first waits for the current one, whose tensors it reads."""
    cur = torch.cuda.current_stream()
    if stream is None:
        return cur.cuda_stream, lambda: None
    ext = torch.cuda.ExternalStream(stream)
    ext.wait_stream(cur)
    return stream, lambda: cur.wait_stream(ext)


def _world(group):
    if dist.is_available() and dist.is_initialized():
        return dist.get_rank(group), dist.get_world_size(group)
    return 0, 1


def _band_pixels(rank, world, width, height, bands):
    """(first_pixel, num_pixels) of `rank`: the equal-row band, or bands[rank]
    = (first_row, rows) of a balanced_bands partition."""
    if bands is None:
        return pixel_band(rank, world, width, height)
    if len(bands) != world:
        raise ValueError("one band per rank")
    pos = 0
    for r0, rows in bands:
        if r0 != pos or rows < 0:
            raise ValueError("bands must tile the rows in order")
        pos += rows
    if pos != height:
        raise ValueError("bands must cover every row")
    r0, rows = bands[rank]
    return r0 * width, rows * width


def gather_bands(band: torch.Tensor, width: int, height: int, group=None, bands=None) -> torch.Tensor:
    """All-gathers every rank's band (float32 [num_pixels*3]; the equal-row
    `pixel_band`, or `bands` from balanced_bands) into the image float32
    [height, width, 3] on every rank.  The bands are padded to the tallest
    band's size for the collective."""
    rank, world = _world(group)
    first, n = _band_pixels(rank, world, width, height, bands)
    if band.numel() != n * 3:
        raise ValueError("band size does not match the partition")
    if world == 1:
        return band.view(height, width, 3)
    sizes = [_band_pixels(r, world, width, height, bands) for r in range(world)]
    n_max = max(k for _, k in sizes)
    padded = torch.zeros(max(1, n_max) * 3, dtype=torch.float32, device=band.device)
    padded[: n * 3] = band
    out = torch.empty(world * padded.numel(), dtype=torch.float32, device=band.device)
    dist.all_gather_into_tensor(out, padded, group=group)
    out = out.view(world, -1)
    image = torch.empty(height * width * 3, dtype=torch.float32, device=band.device)
    for r, (f, k) in enumerate(sizes):
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


def render_sharded(scene: "tpt.Scene", job, group=None, stream=None, bands=None) -> torch.Tensor:
    """The job's image float32 [height, width, 3] on this rank's GPU: this rank
    renders its band (equal rows, or `bands` from balanced_bands, the same
    list on every rank), then the bands are all-gathered."""
    rank, world = _world(group)
    first, n = _band_pixels(rank, world, job.width, job.height, bands)
    band = torch.empty(n * 3, dtype=torch.float32, device="cuda")
    s, join = _stream_for(stream)
    if n:
        scene.render_pixels_device(job, first, n, band.data_ptr(), s)
    join()
    return gather_bands(band, job.width, job.height, group, bands)


def adjoint_sharded(scene: "tpt.Scene", job, d_image: torch.Tensor, mask: int = 0, fd_step: float = 0.0,
                    group=None, stream=None, bands=None) -> torch.Tensor:
    """dLoss/d(material parameters), float64 [n_materials, 7], summed over the
    ranks.  d_image: dLoss/dimage float32 [height, width, 3] (whole image; each
    rank reads its band) on this rank's GPU."""
    rank, world = _world(group)
    first, n = _band_pixels(rank, world, job.width, job.height, bands)
    d = d_image.contiguous().view(-1)
    if d.numel() != job.width * job.height * 3:
        raise ValueError("d_image must cover the whole image")
    band = d[first * 3:(first + n) * 3].contiguous()
    grad = torch.zeros(scene.n_materials * tpt.GRAD_PARAMS, dtype=torch.float64, device="cuda")
    s, join = _stream_for(stream)
    if n:
        scene.adjoint_device(job, band.data_ptr(), grad.data_ptr(), mask, fd_step, s, first_pixel=first,
                             num_pixels=n)
    join()
    return sum_gradients(grad, group).view(scene.n_materials, tpt.GRAD_PARAMS)


def partition_jobs(job_costs, world: int) -> list[list[int]]:
    """Cost-weighted static partition of a batch of jobs over the ranks:
    longest-processing-time-first (jobs by decreasing cost, ties by index, each
    to the rank with the least cost so far, ties to the lower rank), so the
    slowest rank's cost is at most 4/3 of the best possible.  Returns each
    rank's job indices in increasing order; the same list on every rank."""
    costs = [float(c) for c in job_costs]
    if any(not (c >= 0.0) or c == float("inf") for c in costs):
        raise ValueError("job costs: finite, non-negative numbers")
    if world < 1:
        raise ValueError("world >= 1")
    load = [0.0] * world
    owned = [[] for _ in range(world)]
    for j in sorted(range(len(costs)), key=lambda j: (-costs[j], j)):
        r = min(range(world), key=lambda r: (load[r], r))
        load[r] += costs[j]
        owned[r].append(j)
    return [sorted(o) for o in owned]


def job_cost(job) -> float:
    """Default job cost for partition_jobs: its samples (width x height x spp)."""
    return float(job.width) * float(job.height) * float(job.spp)


def render_batch_sharded(ctx: "tpt.Context", jobs, group=None, stream=None, costs=None):
    """Splits a batch of jobs over the ranks (partition_jobs on `costs`, default
    job_cost) and renders this rank's jobs in one `tpt_render_batch_device`
    call.  Returns {job index: float32 [height, width, 3] device image} for the
    jobs this rank owns; no image crosses ranks (a serving caller answers each
    job from the rank that rendered it)."""
    rank, world = _world(group)
    owned = partition_jobs(costs if costs is not None else [job_cost(j) for j in jobs], world)[rank]
    images = {j: torch.empty(jobs[j].height, jobs[j].width, 3, dtype=torch.float32, device="cuda") for j in owned}
    s, join = _stream_for(stream)
    if owned:
        ctx.render_batch_device([jobs[j] for j in owned], [images[j].data_ptr() for j in owned], s)
    join()
    return images
