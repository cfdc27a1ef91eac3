"""Benchmark: one full iteration (forward + volume VJP + per-view pose VJP) of the FP32
projector on the full-scan workload, printed as one JSON line.

Workload (one step): 256^3 FP32 chest-like phantom at 0.8 mm (seeded, synthetic), 360
cone-beam views over 360 deg (SID 1000 mm, SDD 1500 mm), 512x512 detector at 0.8 mm,
1024 clipped midpoint samples per ray; L2 loss against a seeded target image, its
gradient with respect to the field and to a per-view 6-DoF pose tangent.

Metric: realised ray-samples per second of the full iteration (a realised ray-sample
is one midpoint sample on a ray whose clipped span is non-empty; S per such ray).
``value`` is timed on the device with the inputs resident; ``e2e`` includes the
host->device upload of field, target and pose tangent from pinned memory and the
device->host read of loss, image and gradients every step.  Between timed steps the
L2 cache is flushed by writing a 256 MiB buffer.

Besides the timings, the 1-GPU line carries (all computed outside the timed region):
``parity`` (the adjoint identity on the step itself, the FP32 image against strict FP64 on
8 views, one view against the CPU oracle bit for bit), ``forms`` (the same step with a
BF16-stored field in the compensated form and in strict FP64, and the FP32 / BF16 errors
against FP64), ``config1`` (the small plain workload on the GPU and on the CPU oracle) and
``cpu_baseline`` (the CPU oracle on a fixed sample: 8 evenly spaced views x the centre 128
detector rows).

``--impl reference`` times the CPU restatement of the reference projector (the oracle,
all host threads) on the same fixed sample and prints the same line with
``"impl": "reference"``.

Multi-GPU (torchrun, one rank per GPU): every rank projects its own 360 views (the views
of an N x 360-view acquisition, sharded by view) and the volume gradient is summed over
ranks with an NCCL all-reduce; ``value`` is the realised samples of all ranks divided
by the slowest rank's time (weak scaling).
"""

from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

METRIC = "ray-samples/s fwd+vol+pose VJP vs plain FP32; served p50/p99 at FP64 err≤1e-4"
UNIT = "ray-samples/s"
WORKLOAD = "fullscan 256^3 chest 0.8mm, 360 cone views SID1000/SDD1500, 512x512 @0.8mm, S=1024, L2 loss"


def parse() -> argparse.Namespace:
    parser = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    parser.add_argument("--gpus", type=int, default=1)
    parser.add_argument("--steps", type=int, default=5)
    parser.add_argument("--warmup", type=int, default=3)
    parser.add_argument("--impl", choices=("dpt_b200", "reference"), default="dpt_b200")
    parser.add_argument("--views", type=int, default=360, help="views per rank")
    parser.add_argument("--size", type=int, default=256, help="grid samples per axis")
    parser.add_argument("--spacing", type=float, default=None,
                        help="voxel size in mm (default 0.8 * 256 / size: the full scan's 204.8 mm cube)")
    parser.add_argument("--detector", type=int, default=512)
    parser.add_argument("--samples", type=int, default=1024)
    parser.add_argument("--storage", choices=("float32", "bfloat16", "float16"), default="float32")
    parser.add_argument("--no-cpu-baseline", action="store_true")
    parser.add_argument("--seed", type=int, default=20261203)
    parser.add_argument("--mode", choices=("iteration", "serving", "precision", "pointwise", "gather", "panels",
                                           "table", "packed"),
                        default="iteration",
                        help="iteration: full-scan fwd+VJP step (the headline); serving: mixed request stream")
    parser.add_argument("--requests", type=int, default=48, help="serving mode: requests in the stream")
    parser.add_argument("--slots", type=int, default=4, help="serving mode: concurrent request streams")
    parser.add_argument("--no-autotune", action="store_true", help="serving mode: default detector tiles")
    parser.add_argument("--no-graphs", action="store_true", help="serving mode: no CUDA graph replay")
    parser.add_argument("--no-packing", action="store_true",
                        help="serving mode: no packed launches of small forward requests")
    parser.add_argument("--priority", action="store_true",
                        help="serving mode: requests that do not fill the GPU on high-priority streams")
    parser.add_argument("--pack-min", type=int, default=8,
                        help="serving mode: small forward requests of one class that must wait to form a pack")
    parser.add_argument("--pack-samples", type=int, default=1 << 26,
                        help="serving mode: forward requests below this many nominal ray-samples may be packed")
    return parser.parse_args()


def rank_info() -> tuple[int, int, int]:
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


class ClockSampler:
    """nvidia-smi clock / throttle-reason samples every 200 ms during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int) -> None:
        self.index = index
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.process = None

    def start(self) -> None:
        try:
            self.process = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=self.file, stderr=subprocess.DEVNULL)
        except OSError:
            self.process = None

    def stop(self) -> dict | None:
        if self.process is None:
            return None
        self.process.terminate()
        try:
            self.process.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.process.kill()
        self.file.flush()
        rows = [line.split(", ") for line in Path(self.file.name).read_text().splitlines() if line.strip()]
        os.unlink(self.file.name)
        samples = []
        reasons: set[str] = set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for row in rows:
            try:
                sm, sm_max = float(row[1]), float(row[2])
            except (ValueError, IndexError):
                continue
            samples.append((sm, sm_max, float(row[3]) if row[3] not in ("[N/A]", "") else 0.0))
            for name, flag in zip(names, row[5:9], strict=False):
                if flag.strip().lower() == "active":
                    reasons.add(name)
        if not samples:
            return None
        loaded = [s for s in samples if s[2] > 300.0] or samples
        return {"sm_mhz": statistics.median(s[0] for s in loaded), "sm_max_mhz": max(s[1] for s in samples),
                "power_w_max": max(s[2] for s in samples), "samples": len(samples),
                "reasons": sorted(reasons)}


def build_workload(args, device):
    """Grid, geometry, phantom, target pose tangent and seeded target image (untimed)."""
    import numpy as np
    import torch

    from dpt_b200.geometry import ConeBeamIntrinsics
    from dpt_b200.phantoms import centred_grid, chest_phantom

    spacing = args.spacing if args.spacing else 0.8 * 256.0 / args.size
    grid = centred_grid((args.size,) * 3, (spacing,) * 3)
    intrinsics = ConeBeamIntrinsics(1000.0, 1500.0, (args.detector, args.detector),
                                    (0.8 * 512.0 / args.detector,) * 2)
    rank, world, _ = rank_info()
    total_views = args.views * world
    angles = tuple(2.0 * math.pi * (rank * args.views + k) / total_views for k in range(args.views))
    geometry = intrinsics.batch(angles)
    values = chest_phantom(grid, seed=args.seed)
    rng = np.random.default_rng(args.seed + 1)
    truth = rng.normal(size=(args.views, 6)) * np.array([0.5, 0.5, 0.5, 0.004, 0.004, 0.004])
    return grid, geometry, values, torch.tensor(truth, dtype=torch.float64, device=device)


# ------------------------------------------------------------------ helpers

def measured_peak() -> tuple[float, str]:
    path = ROOT / "MEASURED_PEAKS.json"
    try:
        return float(json.loads(path.read_text())["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def measured_l2_gbs(device) -> float:
    """Read bandwidth of a 64 MiB buffer that stays resident in the 126 MB L2, measured with
    the library's read probe (float4 .cg loads, eight 256-thread blocks per SM, 20 passes
    per launch, best of 10 launches after 10 warm-up launches): the L2 roofline of the gather kernels, whose corner
    reads are served by L1 and L2 rather than by HBM."""
    import torch

    from dpt_b200 import _native as N

    lib = N.library()
    nbytes, passes = 64 << 20, 20
    source = torch.ones(nbytes // 4, dtype=torch.float32, device=device)
    sink = torch.zeros(1, dtype=torch.float32, device=device)
    stream = torch.cuda.current_stream(device).cuda_stream

    def launch() -> None:
        code = lib.dpt_b200_read_probe(source.data_ptr(), nbytes, passes, sink.data_ptr(), stream)
        if code != 0:
            raise RuntimeError(f"read probe failed: {code}")

    for _ in range(10):
        launch()
    best = 0.0
    for _ in range(10):
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record()
        launch()
        end.record()
        end.synchronize()
        best = max(best, nbytes * passes / (start.elapsed_time(end) * 1e-3) / 1e9)
    return best


def profile_traffic() -> dict | None:
    """DRAM bytes per realised sample per kernel and storage, from the committed ncu summaries."""
    path = ROOT / "profiles" / "traffic.json"
    try:
        return json.loads(path.read_text())
    except (OSError, ValueError):
        return None


def algorithmic_bytes(kernel: str, storage_bytes: int) -> int:
    """Bytes per realised ray-sample of a sampling launch: forward 8 b_s (the forward that
    also stores the pose moments reads the same eight corners); joint volume + pose VJP
    8 b_s + 32; volume-only VJP 32 (FP32 increments, the field is not read); pose-only VJP
    8 b_s."""
    return {"forward": 8 * storage_bytes, "forward_moments": 8 * storage_bytes,
            "vjp": 8 * storage_bytes + 32, "vjp_volume": 32, "vjp_pose": 8 * storage_bytes}.get(kernel, 0)


def host_cpu() -> dict:
    """Model name and logical core count of this host."""
    model = "unknown"
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("model name"):
                model = line.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    return {"model": model, "nproc": os.cpu_count() or 1}


# The fixed CPU sample of the full-scan workload: these views (evenly spaced over the
# scan) and the centre rows of each, forward + joint volume/pose VJP.
CPU_SAMPLE_VIEWS = 8
CPU_SAMPLE_ROWS = 128


def cpu_sample_rate(grid, geometry, values, samples: int, threads: int):
    """Time the CPU oracle (forward + joint volume/pose VJP) on the fixed sample: 8 evenly
    spaced views x the centre 128 detector rows of each.  Returns (realised samples/s,
    description, seconds)."""
    import numpy as np

    from dpt_b200.geometry import DetectorGeometry
    from dpt_b200.plan import plan_rays
    from oracle import oracle as O

    views = len(geometry.views)
    chosen = sorted({k * views // CPU_SAMPLE_VIEWS for k in range(CPU_SAMPLE_VIEWS)})
    pose = np.asarray((1.0, 0, 0, 0, 1.0, 0, 0, 0, 1.0, 0, 0, 0))
    realised_total, seconds = 0, 0.0
    for view in chosen:
        panel = geometry.views[view]
        rows, cols = panel.shape
        count = min(rows, CPU_SAMPLE_ROWS)
        first = (rows - count) // 2
        origin = tuple(panel.origin_mm[k] + first * panel.spacing_mm[1] * panel.v[k] for k in range(3))
        sub = DetectorGeometry(panel.source_mm, origin, panel.u, panel.v, panel.spacing_mm, (count, cols))
        plan = plan_rays(grid, sub)
        lower, upper, _ = O.counts(plan, pose, samples=samples, threads=threads)
        realised_total += int((upper > lower).sum()) * samples
        seed = np.linspace(0.1, 1.0, plan.rays, dtype=np.float32)
        start = time.perf_counter()
        O.forward(plan, values, pose, samples=samples, threads=threads)
        O.vjp(plan, values, pose, seed, samples=samples, flags=O.VJP_VOLUME | O.VJP_POSE12, threads=threads)
        seconds += time.perf_counter() - start
    sample = (f"views {chosen} of {views}, centre {min(CPU_SAMPLE_ROWS, geometry.views[0].shape[0])} detector "
              f"rows of each ({realised_total} realised ray-samples), forward + joint volume/pose VJP")
    return realised_total / seconds, sample, seconds


def config1_workload():
    """The small plain workload: 64^3 at 1 mm, seeded 6-ellipsoid phantom, 8 cone views over
    360 deg (SOD 500, SDD 1000), 64^2 detector at 1.5 mm, S = 128; loss = mean over the
    central 32 x 32 pixels of every view."""
    from dpt_b200.geometry import ConeBeamIntrinsics
    from dpt_b200.phantoms import centred_grid, ellipsoid_phantom

    grid = centred_grid((64, 64, 64), (1.0, 1.0, 1.0))
    values, _ = ellipsoid_phantom(grid, seed=0)
    geometry = ConeBeamIntrinsics(500.0, 1000.0, (64, 64), (1.5, 1.5)).batch(
        tuple(2 * math.pi * k / 8 for k in range(8)))
    return grid, geometry, values


def config1_cpu(threads: int) -> dict:
    """The small plain workload in full on the CPU oracle: forward and the volume VJP of the
    central mean (best of 3)."""
    import numpy as np

    from dpt_b200.plan import plan_rays
    from oracle import oracle as O

    grid, geometry, values = config1_workload()
    plan = plan_rays(grid, geometry)
    poses = np.tile(np.asarray((1.0, 0, 0, 0, 1.0, 0, 0, 0, 1.0, 0, 0, 0)), (8, 1))
    cot = np.zeros((8, 64, 64), dtype=np.float32)
    cot[:, 16:48, 16:48] = 1.0 / (8 * 32 * 32)
    lower, upper, _ = O.counts(plan, poses, samples=128, threads=threads)
    realised = int((upper > lower).sum()) * 128
    best_f = best_v = math.inf
    for _ in range(3):
        start = time.perf_counter()
        O.forward(plan, values, poses, samples=128, threads=threads)
        middle = time.perf_counter()
        O.vjp(plan, values, poses, cot, samples=128, flags=O.VJP_VOLUME, threads=threads)
        end = time.perf_counter()
        best_f, best_v = min(best_f, middle - start), min(best_v, end - middle)
    return {"forward_ms": round(1e3 * best_f, 3), "volume_vjp_ms": round(1e3 * best_v, 3),
            "realised_ray_samples": realised, "threads": threads,
            "fwd_plus_vjp_samples_per_s": realised / (best_f + best_v)}


def config1_gpu(device) -> dict:
    """The small plain workload on the GPU through the public Projector: forward + volume VJP
    of the central mean (median device time of 20 iterations after 5 warm-up)."""
    import torch

    from dpt_b200.torch import Projector

    grid, geometry, values = config1_workload()
    projector = Projector(grid=grid, geometry=geometry, precision="fp32", samples_per_ray=128)
    field = torch.tensor(values, device=device)

    def iteration():
        f = field.detach().requires_grad_(True)
        image = projector(f)
        (gradient,) = torch.autograd.grad(image[:, 16:48, 16:48].mean(), (f,))
        return gradient

    for _ in range(5):
        iteration()
    torch.cuda.synchronize()
    times = []
    for _ in range(20):
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record()
        iteration()
        end.record()
        end.synchronize()
        times.append(start.elapsed_time(end))
    return {"fwd_plus_vjp_ms": round(statistics.median(times), 4)}


def reference_cotangent(view_indices, rows: int, cols: int, total_views: int):
    """The reference full-scan cotangent formula (benchmarks/config/fullscan.json:45-57):
    raw = 1 + 0.20 sin(theta) + 0.10 cos(2 theta) + 0.15 r + 0.10 c + 0.05 sin(theta) c with
    theta = 2 pi k / views, r, c the pixel centre in [-1, 1]; here divided by the L1 sum over
    the listed views (FP64), then rounded once to FP32."""
    import numpy as np

    theta = 2.0 * np.pi * np.asarray(view_indices, dtype=np.float64) / total_views
    r = 2.0 * (np.arange(rows) + 0.5) / rows - 1.0
    c = 2.0 * (np.arange(cols) + 0.5) / cols - 1.0
    t = theta[:, None, None]
    raw = (1.0 + 0.20 * np.sin(t) + 0.10 * np.cos(2 * t) + 0.15 * r[None, :, None] + 0.10 * c[None, None, :]
           + 0.05 * np.sin(t) * c[None, None, :])
    return (raw / np.abs(raw).sum()).astype(np.float32)


class FormTimer:
    """Device time of a training step: W warm-up steps, then K steps each after a 256 MiB L2
    flush, bracketed by CUDA events on the current stream; per-kernel event times of the
    projector's C-ABI launches from the workspace launch log."""

    def __init__(self, flush) -> None:
        self.flush = flush

    def run(self, step, workspace_of, steps: int, warmup: int, dist=None, clocks=None):
        import torch

        for _ in range(warmup):
            step()
        torch.cuda.synchronize()
        ws = workspace_of()
        ws.launch_log = []
        launches_before = ws.launches
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()
        if clocks:
            clocks.start()
        stream = torch.cuda.current_stream()
        spans = []
        for _ in range(steps):
            self.flush.zero_()
            start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            start.record(stream)
            step()
            end.record(stream)
            spans.append((start, end))
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        clock_record = clocks.stop() if clocks else None
        step_ms = sum(s.elapsed_time(e) for s, e in spans) / steps
        log, ws.launch_log = ws.launch_log, None
        return step_ms, ws.launches - launches_before, log, clock_record


def kernel_times(log, realised_per_view):
    """Per kernel name: summed event times (ms) and realised samples of each launch."""
    per_kernel: dict[str, list[float]] = {}
    per_kernel_samples: dict[str, list[int]] = {}
    for name, first, count, start, end in log:
        per_kernel.setdefault(name, []).append(start.elapsed_time(end))
        per_kernel_samples.setdefault(name, []).append(int(realised_per_view[first:first + count].sum()))
    return per_kernel, per_kernel_samples


def as_built_bytes(per_kernel_samples, storage_bytes: int, steps: int) -> float:
    """Algorithmic bytes per step of the sampling launches the step actually made."""
    return sum(algorithmic_bytes(name, storage_bytes) * sum(samples)
               for name, samples in per_kernel_samples.items()) / steps


def run_gpu(args) -> None:
    import numpy as np
    import torch

    rank, world, local = rank_info()
    device = torch.device(f"cuda:{local}")
    torch.cuda.set_device(device)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=900), device_id=device)

    from dpt_b200.distributed import reduce_volume_gradient
    from dpt_b200.torch import Projector
    from dpt_b200.torch import _projection_ops as ops

    grid, geometry, values, truth = build_workload(args, device)
    dtype = {"float32": torch.float32, "bfloat16": torch.bfloat16, "float16": torch.float16}[args.storage]
    storage_bytes = 4 if args.storage == "float32" else 2
    projector = Projector(grid=grid, geometry=geometry, precision="fp32", samples_per_ray=args.samples)
    field = torch.tensor(values, device=device).to(dtype).contiguous()
    views = len(geometry.views)
    with torch.no_grad():
        target = projector(field, truth)
        noise = torch.Generator(device=device).manual_seed(args.seed + 2)
        target += 0.01 * torch.randn(target.shape, generator=noise, device=device)
    tangent = torch.zeros((views, 6), dtype=torch.float64, device=device)

    def step_with(module):
        def step(f, t, xi):
            f = f.detach().requires_grad_(True)
            xi = xi.detach().requires_grad_(True)
            image = module(f, xi)
            residual = image - t
            loss = 0.5 * (residual.double() * residual.double()).sum()
            grad_field, grad_pose = torch.autograd.grad(loss, (f, xi))
            reduce_volume_gradient(grad_field)
            return loss.detach(), image.detach(), grad_field, grad_pose
        return step

    step = step_with(projector)
    step(field, target, tangent)
    ws = ops.workspace(field, projector.configuration, True, True)
    identity = torch.tensor((1.0, 0, 0, 0, 1.0, 0, 0, 0, 1.0, 0, 0, 0), dtype=torch.float64,
                            device=device).expand(views, 12).contiguous()

    def realised_of(workspace):
        lower, upper, _ = workspace.counts(identity)
        nonempty = (upper > lower).reshape(views, -1).sum(dim=1).cpu().numpy().astype(np.int64)
        return nonempty * args.samples

    realised_per_view = realised_of(ws)
    realised = int(realised_per_view.sum())
    nominal = views * args.detector * args.detector * args.samples
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=device)
    timer = FormTimer(flush)

    # ---- device-resident timing of the headline form
    sampler = ClockSampler(torch.cuda.current_device()) if rank == 0 else None
    step_ms, gpu_launches, log, clocks = timer.run(lambda: step(field, target, tangent), lambda: ws,
                                                   args.steps, max(args.warmup, 3), dist, sampler)
    per_kernel, per_kernel_samples = kernel_times(log, realised_per_view)
    totals = {name: sum(times) for name, times in per_kernel.items()}
    dominant = max((k for k in totals if algorithmic_bytes(k, storage_bytes)), key=lambda k: totals[k])
    hbm_peak, hbm_kind = measured_peak()
    launches = len(per_kernel[dominant])
    mean_ms = totals[dominant] / launches
    bytes_per_launch = algorithmic_bytes(dominant, storage_bytes) * sum(per_kernel_samples[dominant]) / launches
    achieved = bytes_per_launch / (mean_ms * 1e-3) / 1e9
    # DRAM bytes per launch of the dominant kernel: the per-realised-sample figure of its ncu
    # capture on the 4-view slice of this workload, scaled to the samples one launch realises
    traffic_record = profile_traffic()
    traffic = None
    per_sample = (traffic_record or {}).get("dram_bytes_per_realised_sample", {}).get(f"{dominant}:{args.storage}")
    if per_sample is not None and args.size == 256 and args.detector == 512 and args.samples == 1024:
        traffic = round(per_sample * sum(per_kernel_samples[dominant]) / launches)
    l2 = measured_l2_gbs(device)
    built = as_built_bytes(per_kernel_samples, storage_bytes, args.steps)
    contract = (16 * storage_bytes + 32) * realised
    roofline = {
        "bound": "l2", "kernel": dominant, "achieved": round(achieved, 1), "peak": round(l2, 1), "unit": "GB/s",
        "frac": round(achieved / l2, 4), "traffic": traffic,
        "peak_source": "measured in this run: dpt_b200_read_probe, float4 .cg loads of a 64 MiB L2-resident "
                       "buffer, best of 10 launches of 20 passes",
        "bytes_per_sample": algorithmic_bytes(dominant, storage_bytes),
        "limiter": "FP32 pipe (ncu on the forward with pose moments: FMA pipe 65.6% of active cycles, "
                   "math-pipe throttle the top stall; L1 hit 92.7%, L2 hit 86.8%, DRAM 0.21 B per realised sample)",
        "hbm": {"peak": hbm_peak, "peak_source": f"{hbm_kind} MEASURED_PEAKS hbm_gbs",
                "dram_gbs": None if traffic is None else round(traffic / (mean_ms * 1e-3) / 1e9, 1),
                "frac": None if traffic is None else round(traffic / (mean_ms * 1e-3) / 1e9 / hbm_peak, 4)},
        "iteration": {
            "as_built_bytes_per_sample": round(built / realised, 2),
            "as_built_achieved": round(built / (step_ms * 1e-3) / 1e9, 1),
            "as_built_frac_l2": round(built / (step_ms * 1e-3) / 1e9 / l2, 4),
            "contract_bytes_per_sample": 16 * storage_bytes + 32,
            "contract_achieved": round(contract / (step_ms * 1e-3) / 1e9, 1),
            "contract_frac_l2": round(contract / (step_ms * 1e-3) / 1e9 / l2, 4)},
        "kernel_ms": {k: round(v / args.steps, 3) for k, v in sorted(totals.items())},
        "launches_per_step": {k: len(v) // args.steps for k, v in sorted(per_kernel.items())},
    }

    # ---- end to end through the public API with host buffers
    host_field = field.cpu().pin_memory()
    host_target = target.cpu().pin_memory()
    host_tangent = tangent.cpu().pin_memory()
    out_image = torch.empty(target.shape, dtype=target.dtype).pin_memory()
    out_grad = torch.empty(field.shape, dtype=field.dtype).pin_memory()
    out_pose = torch.empty(tangent.shape, dtype=torch.float64).pin_memory()
    out_loss = torch.empty((), dtype=torch.float64).pin_memory()
    h2d = host_field.numel() * host_field.element_size() + host_target.numel() * 4 + host_tangent.numel() * 8
    d2h = out_image.numel() * 4 + out_grad.numel() * out_grad.element_size() + out_pose.numel() * 8 + 8

    # The same step through the public Projector with host buffers.  The target upload runs on a
    # copy stream beside the forward and the image download beside the VJP; the main stream
    # waits for both, so every copy is inside the step's events.
    copies = torch.cuda.Stream(device)

    def e2e_step():
        main = torch.cuda.current_stream(device)
        f = host_field.to(device, non_blocking=True).detach().requires_grad_(True)
        xi = host_tangent.to(device, non_blocking=True).detach().requires_grad_(True)
        copies.wait_stream(main)
        with torch.cuda.stream(copies):
            t = host_target.to(device, non_blocking=True)
        image = projector(f, xi)
        forward_done = torch.cuda.Event()
        forward_done.record(main)
        main.wait_stream(copies)
        t.record_stream(main)
        residual = image - t
        loss = 0.5 * (residual.double() * residual.double()).sum()
        with torch.cuda.stream(copies):
            copies.wait_event(forward_done)
            image.record_stream(copies)
            out_image.copy_(image.detach(), non_blocking=True)
        gf, gp = torch.autograd.grad(loss, (f, xi))
        reduce_volume_gradient(gf)
        out_loss.copy_(loss.detach(), non_blocking=True)
        out_grad.copy_(gf, non_blocking=True)
        out_pose.copy_(gp, non_blocking=True)
        main.wait_stream(copies)

    e2e_ms, _, _, _ = timer.run(e2e_step, lambda: ws, args.steps, 1, dist)

    # max over ranks
    if dist is not None:
        timing = torch.tensor([step_ms, e2e_ms], dtype=torch.float64, device=device)
        dist.all_reduce(timing, op=dist.ReduceOp.MAX)
        step_ms, e2e_ms = timing.tolist()
        total = torch.tensor([realised], dtype=torch.float64, device=device)
        dist.all_reduce(total)
        realised_all = int(total.item())
    else:
        realised_all = realised

    parity = forms = cpu_baseline = config1 = None
    if rank == 0 and world == 1:
        parity = parity_record(args, grid, geometry, values, field, target, tangent, step, identity)
        forms = forms_record(args, grid, geometry, values, target, truth, tangent, timer, step_ms,
                             realised_per_view, storage_bytes, step_with, identity)
        config1 = {"gpu": config1_gpu(device)}
        if not args.no_cpu_baseline:
            threads = os.cpu_count() or 1
            rate, sample, seconds = cpu_sample_rate(grid, geometry, values, args.samples, threads)
            cpu_baseline = {"value": rate, "unit": UNIT, "cores": threads, "kind": "port",
                            "sample": sample + f"; {seconds:.1f} s on {threads} threads (C oracle -O3 -fopenmp)",
                            "host": host_cpu()}
            config1["cpu"] = config1_cpu(threads)

    if rank == 0:
        line = {
            "metric": METRIC,
            "value": realised_all / (step_ms * 1e-3),
            "unit": UNIT,
            "n_gpus": world,
            "steps": args.steps,
            "warmup": max(args.warmup, 3),
            "ms_per_step": step_ms,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32" if args.storage == "float32" else f"f32 ({args.storage} storage)",
            "data": "synthetic (seeded chest-like HU phantom, 60 keV water model; no scanned volume)",
            "config": {"workload": WORKLOAD if (args.size, args.views, args.detector, args.samples, args.spacing)
                       == (256, 360, 512, 1024, None)
                       else f"{args.size}^3 at {grid.spacing_mm[0]:g} mm, {args.views} views, {args.detector}^2, "
                            f"S={args.samples}",
                       "grid": [args.size] * 3, "views_per_gpu": len(geometry.views),
                       "detector": [args.detector, args.detector], "samples_per_ray": args.samples,
                       "storage": args.storage, "precision": "fp32",
                       "realised_ray_samples_per_step": realised_all,
                       "nominal_ray_samples_per_step": nominal * world,
                       "l2": "flushed between timed steps (256 MiB write)",
                       "parallelism": f"views sharded over {world} GPU(s), NCCL all-reduce of the volume gradient"
                       if world > 1 else "1 GPU"},
            "e2e": {"value": realised_all / (e2e_ms * 1e-3), "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "ms_per_step": e2e_ms},
            "gpu_launches": gpu_launches,
            "roofline": roofline,
            "cpu_baseline": cpu_baseline,
            "clocks": clocks,
            "parity": parity,
            "forms": forms,
            "config1": config1,
        }
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


PARITY_VIEW = 90


def parity_record(args, grid, geometry, values, field, target, tangent, step, identity) -> dict:
    """Correctness of the timed step, checked outside the timed region with the reference's
    full-scan quality bounds (benchmarks/config/fullscan.json:85-103):

    * adjoint: |<A x, y> - <x, A^T y>| / max(|.|) <= 2e-5 on the step itself (x = field,
      y = the loss cotangent = residual, A x = the image, A^T y = the volume gradient);
    * image_fp32_vs_fp64: relative L2 of the step's FP32 image against the strict FP64
      projection on 8 evenly spaced views, <= 1e-5;
    * oracle_view: view 90 of the step against the CPU oracle on the same inputs: image bit
      for bit, that view's pose gradient (rtol 1e-9) and volume gradient (relative L2 2e-6)
      for the step's cotangent."""
    import numpy as np
    import torch

    from dpt_b200.geometry import BatchedGeometry
    from dpt_b200.plan import plan_rays
    from dpt_b200.projection import ProjectionSpec, ProjectionWorkspace
    from oracle import oracle as O

    device = field.device
    loss, image, grad_field, _ = step(field, target, tangent)
    residual = (image - target).float()
    lhs = float((image.double() * residual.double()).sum())
    rhs = float((field.double() * grad_field.double()).sum())
    adjoint = abs(lhs - rhs) / max(abs(lhs), abs(rhs), 1e-300)

    views = len(geometry.views)
    subset = sorted({k * views // 8 for k in range(8)})  # 8 evenly spaced views (fewer when fewer exist)
    sub_geometry = BatchedGeometry(tuple(geometry.views[k] for k in subset))
    exact = ProjectionWorkspace(plan_rays(grid, sub_geometry),
                                ProjectionSpec(args.samples, precision="float64", sampling_precision="float64"),
                                device)
    image64 = exact.forward(field.float(), identity[: len(subset)].contiguous())
    image32 = image[subset].double()
    image_rel = float((image32 - image64).norm() / image64.norm())
    del exact

    view = min(PARITY_VIEW, views - 1)
    single = BatchedGeometry((geometry.views[view],))
    plan = plan_rays(grid, single)
    ws = ProjectionWorkspace(plan, ProjectionSpec(args.samples, sampling_precision="float32"), device)
    pose1 = identity[:1].contiguous()
    image1 = ws.forward(field.float(), pose1)
    cot1 = residual[view:view + 1].contiguous()
    volume1, pose_grad1 = ws.vjp(field.float(), pose1, cot1, volume=True, pose="matrix")
    threads = os.cpu_count() or 1
    host_values = field.float().cpu().numpy()
    poses_host = identity[:1].cpu().numpy()
    e_image, status = O.forward(plan, host_values, poses_host, samples=args.samples, threads=threads)
    e_volume, e_pose, status_v = O.vjp(plan, host_values, poses_host, cot1.cpu().numpy(), samples=args.samples,
                                       flags=O.VJP_VOLUME | O.VJP_POSE12, threads=threads)
    got_image = image1.cpu().numpy().reshape(-1)
    step_view = image[view].cpu().numpy().reshape(-1)
    pose_err = float(np.max(np.abs(pose_grad1.cpu().numpy() - e_pose) / np.maximum(np.abs(e_pose), 1e-300)))
    volume_rel = float(np.linalg.norm(volume1.cpu().numpy().reshape(-1) - e_volume) / np.linalg.norm(e_volume))
    del ws
    torch.cuda.empty_cache()
    return {
        "adjoint": {"value": adjoint, "bound": 2e-5, "ok": adjoint <= 2e-5,
                    "lhs": lhs, "rhs": rhs, "what": "<image, residual> vs <field, volume gradient> of the step"},
        "image_fp32_vs_fp64": {"value": image_rel, "bound": 1e-5, "ok": image_rel <= 1e-5, "views": subset},
        "oracle_view": {"view": view, "rays": int(plan.rays),
                        "image_bit_exact": bool(np.array_equal(got_image, e_image)),
                        "step_image_bit_exact": bool(np.array_equal(step_view, e_image)),
                        "pose12_max_rel_err": pose_err, "pose_bound": 1e-9, "pose_ok": pose_err <= 1e-9,
                        "volume_rel_l2": volume_rel, "volume_bound": 2e-6, "volume_ok": volume_rel <= 2e-6,
                        "status_clear": bool(not status.any() and not status_v.any())},
        "loss": float(loss),
    }


def forms_record(args, grid, geometry, values, target, truth, tangent, timer, fp32_ms, realised_per_view,
                 storage_bytes, step_with, identity) -> dict:
    """The same training step in the BF16-storage form (FP32 interpolation, compensated ray
    sums) and in strict FP64, timed like the headline (fewer steps), plus the relative L2
    of image, volume gradient and per-view pose gradient of the FP32 and BF16 forms against
    the strict FP64 path on the same stored values: 8 evenly spaced views, the reference
    full-scan cotangent formula."""
    import torch

    from dpt_b200.geometry import BatchedGeometry
    from dpt_b200.plan import plan_rays
    from dpt_b200.projection import ProjectionSpec, ProjectionWorkspace
    from dpt_b200.torch import Projector
    from dpt_b200.torch import _projection_ops as ops

    device = target.device
    views = len(geometry.views)
    realised = int(realised_per_view.sum())
    out = {}
    for name, dtype, precision, steps, warmup in (("bf16", torch.bfloat16, "fp32", 3, 3),
                                                  ("fp64", torch.float32, "fp64", 2, 3)):
        module = Projector(grid=grid, geometry=geometry, precision=precision, samples_per_ray=args.samples)
        field = torch.tensor(values, device=device).to(dtype).contiguous()
        step = step_with(module)
        step(field, target, tangent)
        ws = ops.workspace(field, module.configuration, True, True)
        lower, upper, _ = ws.counts(identity)
        form_realised = int((upper > lower).sum()) * args.samples
        ms, launches, log, _ = timer.run(lambda s=step, f=field: s(f, target, tangent), lambda w=ws: w,
                                         steps, warmup)
        per_kernel, per_kernel_samples = kernel_times(log, realised_per_view)
        form_storage = 2 if dtype == torch.bfloat16 else 4
        built = as_built_bytes(per_kernel_samples, form_storage, steps)
        out[name] = {"ms_per_step": ms, "value": form_realised / (ms * 1e-3), "unit": UNIT,
                     "speedup_vs_fp32": fp32_ms / ms, "steps": steps, "warmup": warmup,
                     "realised_ray_samples_per_step": form_realised, "gpu_launches": launches,
                     "kernel_ms": {k: round(sum(v) / steps, 3) for k, v in sorted(per_kernel.items())},
                     "as_built_bytes_per_sample": round(built / form_realised, 2),
                     "storage": "bfloat16" if dtype == torch.bfloat16 else "float32",
                     "arithmetic": "compensated FP32 (FP64 clip and pose chain)" if name == "bf16"
                     else "strict FP64"}
        del ws, module, step
        ops.clear_cache()
        torch.cuda.empty_cache()

    # errors against strict FP64 on the same stored values (8 views, fixed cotangent)
    subset = sorted({k * views // 8 for k in range(8)})  # 8 evenly spaced views (fewer when fewer exist)
    sub_geometry = BatchedGeometry(tuple(geometry.views[k] for k in subset))
    plan = plan_rays(grid, sub_geometry)
    rows, cols = sub_geometry.shape_rows_columns
    cot = torch.tensor(reference_cotangent(subset, rows, cols, views), device=device)
    poses = identity[: len(subset)].contiguous()

    def rel(a, b):
        return float((a.double() - b.double()).norm() / b.double().norm())

    field32 = torch.tensor(values, device=device)
    for name, storage, sampling in (("fp32", "float32", "float32"), ("bf16", "bfloat16", "compensated")):
        stored = field32.to(torch.bfloat16) if storage == "bfloat16" else field32
        decoded = stored.float()
        exact = ProjectionWorkspace(plan, ProjectionSpec(args.samples, precision="float64",
                                                         sampling_precision="float64"), device)
        image64 = exact.forward(decoded, poses)
        vol64, pose64 = exact.vjp(decoded, poses, cot.double(), volume=True, pose="tangent",
                                  volume_dtype=torch.float64)
        ws = ProjectionWorkspace(plan, ProjectionSpec(args.samples, sampling_precision=sampling,
                                                      storage_precision=storage), device)
        image = ws.forward(stored, poses)
        vol, pose = ws.vjp(stored, poses, cot, volume=True, pose="tangent")
        errors = {"image_rel_l2": rel(image, image64), "volume_grad_rel_l2": rel(vol, vol64),
                  "pose_grad_rel_l2": rel(pose, pose64)}
        if name == "bf16":
            errors["storage_rounding_rel_l2"] = rel(decoded, field32)
            errors["image_ok"] = errors["image_rel_l2"] <= 1e-4
        out.setdefault(name, {})["vs_fp64"] = errors
        del exact, ws
    out["vs_fp64_case"] = {"views": subset, "cotangent": "reference full-scan formula, L1-normalised over "
                                                         "these views, FP32",
                           "reference": "strict FP64 projection of the same stored (decoded) values"}
    torch.cuda.empty_cache()
    return out


def run_reference(args) -> None:
    """CPU restatement of the reference projector (the oracle), timed on this host's cores on
    the fixed sample of the workload (8 evenly spaced views x the centre 128 detector rows,
    forward + joint volume/pose VJP), and the small plain workload in full."""
    rank, world, _ = rank_info()
    if rank != 0:
        return
    import torch

    grid, geometry, values, _ = build_workload(args, torch.device("cpu"))
    threads = os.cpu_count() or 1
    for _ in range(args.warmup):
        cpu_sample_rate(grid, geometry, values, args.samples, threads)
    rates, seconds, sample = [], 0.0, ""
    for _ in range(args.steps):
        rate, sample, took = cpu_sample_rate(grid, geometry, values, args.samples, threads)
        rates.append(rate)
        seconds += took
    value = statistics.median(rates)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * seconds / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "impl": "reference",
        "data": "synthetic (seeded chest-like HU phantom, 60 keV water model; no scanned volume)",
        "config": {"workload": WORKLOAD, "grid": [args.size] * 3, "views": args.views,
                   "detector": [args.detector, args.detector], "samples_per_ray": args.samples,
                   "parallelism": f"{threads} host threads"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": "per step: " + sample + " (median over steps)", "host": host_cpu(),
                         "rates": rates},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "config1": {"cpu": config1_cpu(threads)},
        "reference_projector": "the reference's own CPU path needs warp-lang 1.17.0, which is not installed on "
                               "this host (import warp fails); the oracle restatement stands in",
    }
    print(json.dumps(line), flush=True)


def serving_requests(args, device):
    """Seeded mixed request stream: resident volumes of 64^3, 128^3, 256^3 and 512x512x128 in
    FP32 or BF16, 1-64 views (log-uniform), square detectors 128^2-1024^2, 128-1024 samples;
    60% forward, 30% forward + volume VJP, 10% forward + pose VJP; Poisson arrivals."""
    import numpy as np

    from dpt_b200.geometry import ConeBeamIntrinsics
    from dpt_b200.phantoms import centred_grid, chest_phantom
    from dpt_b200.serving import ProjectionRequest

    rng = np.random.default_rng(args.seed)
    volumes = {}
    for name, shape, spacing in (("v64", (64, 64, 64), 3.2), ("v128", (128, 128, 128), 1.6),
                                 ("v256", (256, 256, 256), 0.8), ("v512", (128, 512, 512), 0.4)):
        grid = centred_grid(shape, (spacing, spacing, spacing * (4.0 if name == "v512" else 1.0)))
        volumes[name] = (grid, chest_phantom(grid, seed=args.seed))
    requests = []
    for _ in range(args.requests):
        name = ("v64", "v128", "v256", "v512")[int(rng.integers(4))]
        storage = "bfloat16" if rng.random() < 0.5 else "float32"
        views = int(round(math.exp(rng.uniform(0.0, math.log(64.0)))))
        detector = int(rng.choice((128, 256, 512, 1024)))
        samples = int(rng.choice((128, 256, 512, 1024)))
        kind = ("forward", "volume", "pose")[int(rng.choice(3, p=(0.6, 0.3, 0.1)))]
        pitch = 409.6 / detector
        geometry = ConeBeamIntrinsics(1000.0, 1500.0, (detector, detector), (pitch, pitch)).batch(
            tuple(2.0 * math.pi * k / views + float(rng.uniform(0, 0.1)) for k in range(views)))
        requests.append((ProjectionRequest(f"{name}:{storage}", geometry, samples, kind), storage, name))
    return volumes, requests


def small_burst(args, server, volumes) -> dict:
    """128 small forward requests submitted at once (64^3 / 128^3 volumes in FP32 or BF16, 1-4
    views, 128^2 or 256^2 detectors, S 128 or 256: DRR-sized previews), served with packed
    launches, served without them, and run one after another through the server's launch
    sequence; requests/s of each (best of 3 after a warm round)."""
    import numpy as np
    import torch

    from dpt_b200.geometry import ConeBeamIntrinsics
    from dpt_b200.serving import ProjectionRequest

    rng = np.random.default_rng(args.seed + 11)
    requests = []
    for _ in range(128):
        name = ("v64", "v128")[int(rng.integers(2))]
        storage = "bfloat16" if rng.random() < 0.5 else "float32"
        views = int(rng.integers(1, 5))
        detector = int(rng.choice((128, 256)))
        samples = int(rng.choice((128, 256)))
        pitch = 409.6 / detector
        geometry = ConeBeamIntrinsics(1000.0, 1500.0, (detector, detector), (pitch, pitch)).batch(
            tuple(2.0 * math.pi * k / views + float(rng.uniform(0, 0.1)) for k in range(views)))
        requests.append(ProjectionRequest(f"{name}:{storage}", geometry, samples, "forward"))

    def served() -> float:
        start = time.perf_counter()
        results = [future.result() for future in [server.submit(r) for r in requests]]
        return max(r.finished for r in results) - start

    def alone() -> float:
        start = time.perf_counter()
        for request in requests:
            server.run_alone(request)
        torch.cuda.synchronize()
        return time.perf_counter() - start

    out = {}
    packs = server.packs
    for name, packing, run in (("served_packed", True, served), ("served_unpacked", False, served),
                               ("sequential_same_arithmetic", True, alone)):
        server.packing = packing
        run()
        out[name + "_requests_per_s"] = len(requests) / min(run() for _ in range(3))
    server.packing = True
    out["packed_launches"] = server.packs - packs
    out["speedup_packed_vs_sequential_same_arithmetic"] = (out["served_packed_requests_per_s"]
                                                           / out["sequential_same_arithmetic_requests_per_s"])
    out["speedup_packed_vs_unpacked"] = out["served_packed_requests_per_s"] / out["served_unpacked_requests_per_s"]
    out["requests"] = len(requests)
    return out


def run_serving(args) -> None:
    """Served mixed stream against the same requests run one after another through the plain
    FP32 projector (and, for reference, through the server's own launch sequence alone).

    Capacity: every request submitted at once, time until the last completes (the server
    overlaps requests on its slots' streams).
    Latency: Poisson arrivals at 70% of the measured served capacity, p50/p99 from submit
    to result."""
    import numpy as np
    import torch

    from dpt_b200.serving import ProjectionServer, percentile

    device = torch.device("cuda:0")
    volumes, stream = serving_requests(args, device)
    requests = [request for request, _, _ in stream]

    def saturated(server) -> float:
        start = time.perf_counter()
        futures = [server.submit(request) for request in requests]
        results = [future.result() for future in futures]
        return max(r.finished for r in results) - start

    # sequential plain calls: each request through the public FP32 Projector (autograd for
    # the gradients), one after another, each result read before the next call
    from dpt_b200.torch import Projector
    from dpt_b200.torch import _projection_ops as ops

    ops.set_cache_limit(4 * len(stream))  # every request's plan and field copy stays warm
    fields32 = {name: torch.tensor(values, device=device) for name, (_, values) in volumes.items()}
    modules = [Projector(grid=volumes[name][0], geometry=request.geometry, precision="fp32",
                         samples_per_ray=request.samples_per_ray) for request, _, name in stream]

    def plain(k: int) -> float:
        request, _, name = stream[k]
        field = fields32[name]
        if request.kind == "forward":
            with torch.no_grad():
                return float(modules[k](field).sum())
        if request.kind == "volume":
            f = field.detach().requires_grad_(True)
            image = modules[k](f)
            loss = 0.5 * (image.double() * image.double()).sum()
            loss.backward()
            return float(loss.detach()) + float(f.grad.reshape(-1)[0])
        tangent = torch.zeros(6, dtype=torch.float64, device=device, requires_grad=True)
        image = modules[k](field, tangent)
        loss = 0.5 * (image.double() * image.double()).sum()
        loss.backward()
        return float(loss.detach()) + float(tangent.grad[0])

    for k in range(len(stream)):  # warm-up: workspaces, field copies
        plain(k)
    torch.cuda.synchronize()
    sequential_s = math.inf
    for _ in range(2):  # best of two passes, as the served stream is best of three
        start = time.perf_counter()
        for k in range(len(stream)):
            plain(k)
        torch.cuda.synchronize()
        sequential_s = min(sequential_s, time.perf_counter() - start)
    del modules

    with ProjectionServer(str(device), slots=args.slots, autotune=not args.no_autotune,
                          graphs=not args.no_graphs, packing=not args.no_packing,
                          pack_samples=args.pack_samples, priorities=args.priority, pack_min=args.pack_min) as server:
        for name, (grid, values) in volumes.items():
            for storage in ("float32", "bfloat16"):
                server.add_volume(f"{name}:{storage}", grid, values, storage=storage)
        for request in requests:
            server.run_alone(request)  # warm-up: workspaces, packed copies
        torch.cuda.synchronize()
        alone_s = math.inf
        for _ in range(2):
            start = time.perf_counter()
            for request in requests:
                server.run_alone(request)
            torch.cuda.synchronize()
            alone_s = min(alone_s, time.perf_counter() - start)
        # the same launch sequences back to back on one stream, one synchronisation at the end:
        # the time the GPU needs for this work with no gap between requests, so
        # alone_s / chained_s bounds what any overlap of requests can gain
        chained_s = math.inf
        for _ in range(2):
            start = time.perf_counter()
            server.run_chained(requests)
            torch.cuda.synchronize()
            chained_s = min(chained_s, time.perf_counter() - start)
        for _ in range(2):  # warm the served path: workspaces, tiles and graphs on the slots
            saturated(server)
        packs, packed = server.packs, server.packed_requests
        served_s = min(saturated(server) for _ in range(3))
        packs, packed = (server.packs - packs) / 3, (server.packed_requests - packed) / 3
        rng = np.random.default_rng(args.seed + 7)
        rate = 0.7 * len(requests) / served_s
        latencies = []
        for _ in range(4):
            arrivals = np.cumsum(rng.exponential(1.0 / rate, len(requests)))
            start = time.perf_counter()
            futures = []
            for request, arrival in zip(requests, arrivals, strict=True):
                delay = start + arrival - time.perf_counter()
                if delay > 0:
                    time.sleep(delay)
                futures.append(server.submit(request))
            latencies += [future.result().latency * 1e3 for future in futures]
        burst = small_burst(args, server, volumes) if not args.no_packing else None
    samples_total = sum(sum(v.pixels for v in r.geometry.views) * r.samples_per_ray for r in requests)
    line = {
        "metric": "served mixed projection stream",
        "value": len(requests) / served_s,
        "unit": "requests/s",
        "sequential_requests_per_s": len(requests) / sequential_s,
        "speedup_vs_sequential": sequential_s / served_s,
        "sequential_same_arithmetic_requests_per_s": len(requests) / alone_s,
        "speedup_vs_sequential_same_arithmetic": alone_s / served_s,
        "chained_same_arithmetic_requests_per_s": len(requests) / chained_s,
        "overlap_bound": alone_s / chained_s,
        "p50_ms": percentile(latencies, 50),
        "p99_ms": percentile(latencies, 99),
        "latency_load_requests_per_s": rate,
        "latency_samples": len(latencies),
        "requests": len(requests),
        "packed_launches_per_round": packs,
        "packed_requests_per_round": packed,
        "small_burst": burst,
        "nominal_ray_samples": samples_total,
        "higher_is_better": True,
        "config": {"workload": "Poisson mix: 64^3/128^3/256^3/512x512x128 volumes FP32|BF16, 1-64 views, "
                               "128^2-1024^2 detectors, S 128-1024, 60/30/10 forward/volume/pose",
                   "sequential": "plain FP32 Projector calls (FP32 copies of the BF16 volumes), one "
                                 "after another, each result read before the next call",
                   "sequential_same_arithmetic": "the server's own launch sequence per request, one "
                                                 "after another on one stream (BF16 volumes in the "
                                                 "compensated form)",
                   "chained_same_arithmetic": "the same launch sequences back to back on one stream with "
                                              "one synchronisation at the end (no gap between requests)",
                   "capacity": "all requests submitted at once, best of 3 after 2 warm rounds (the sequential "
                               "runs: best of 2 after a warm one)",
                   "latency": "Poisson arrivals at 70% of served capacity, 4 rounds",
                   "slots": args.slots, "memory_budget_gib": 120, "autotune": not args.no_autotune,
                   "graphs": not args.no_graphs, "packing": not args.no_packing,
                   "pack_samples": args.pack_samples, "pack_min": args.pack_min,
                   "priorities": args.priority},
    }
    print(json.dumps(line), flush=True)


def run_precision(args) -> None:
    """Relative L2 of image, volume gradient and pose gradient of every precision form
    against the FP64 path on the same stored values (S = 1024): the 64^3 ellipsoid scan
    (8 views, 64^2 at 1.5 mm, loss = mean over the central 32x32 detector region) and a
    512^3 0.5 mm variant (8 views, 512^2)."""
    import numpy as np
    import torch

    from dpt_b200.geometry import ConeBeamIntrinsics, RigidTransform
    from dpt_b200.phantoms import centred_grid, chest_phantom, ellipsoid_phantom
    from dpt_b200.plan import plan_rays
    from dpt_b200.projection import ProjectionSpec, ProjectionWorkspace

    device = torch.device("cuda:0")
    cases = []
    grid = centred_grid((64, 64, 64), (1.0, 1.0, 1.0))
    values, _ = ellipsoid_phantom(grid, seed=args.seed)
    geometry = ConeBeamIntrinsics(500.0, 1000.0, (64, 64), (1.5, 1.5)).batch(
        tuple(2 * math.pi * k / 8 for k in range(8)))
    cases.append(("64^3 1mm ellipsoids, 8 views 64^2", grid, geometry, values, 32))
    if args.size >= 512:
        big = centred_grid((512, 512, 512), (0.5, 0.5, 0.5))
        cases.append(("512^3 0.5mm chest, 8 views 512^2", big,
                      ConeBeamIntrinsics(1000.0, 1500.0, (512, 512), (0.8, 0.8)).batch(
                          tuple(2 * math.pi * k / 8 for k in range(8))), chest_phantom(big, seed=args.seed), 256))
    report = []
    for name, grid, geometry, values, central in cases:
        plan = plan_rays(grid, geometry)
        views = len(geometry.views)
        rows, cols = geometry.shape_rows_columns
        cot = torch.zeros(geometry.shape, dtype=torch.float64, device=device)
        r0, c0 = (rows - central) // 2, (cols - central) // 2
        cot[:, r0:r0 + central, c0:c0 + central] = 1.0 / (views * central * central)
        poses = torch.tensor(RigidTransform().packed(), dtype=torch.float64, device=device).expand(views, 12).contiguous()
        field32 = torch.tensor(values, device=device)
        for storage, dtype in (("float32", torch.float32), ("bfloat16", torch.bfloat16), ("float16", torch.float16)):
            stored = field32.to(dtype)
            decoded = stored.float()
            exact = ProjectionWorkspace(plan, ProjectionSpec(1024, precision="float64", sampling_precision="float64"), device)
            image64 = exact.forward(decoded, poses)
            vol64, pose64 = exact.vjp(decoded, poses, cot, volume=True, pose="tangent", volume_dtype=torch.float64)
            forms = [("compensated", stored)] if storage != "float32" else [("float32", decoded), ("compensated", decoded)]
            for sampling, tensor in forms:
                ws = ProjectionWorkspace(plan, ProjectionSpec(1024, sampling_precision=sampling, storage_precision=storage), device)
                image = ws.forward(tensor, poses)
                vol, pose = ws.vjp(tensor, poses, cot.float(), volume=True, pose="tangent")

                def rel(a, b):
                    return float((a.double() - b.double()).norm() / b.double().norm())

                report.append({"case": name, "storage": storage, "sampling": sampling,
                               "image_rel_l2": rel(image, image64), "volume_grad_rel_l2": rel(vol, vol64),
                               "pose_grad_rel_l2": rel(pose, pose64),
                               "storage_rounding_rel_l2": rel(decoded, field32)})
    print(json.dumps({"metric": "relative L2 vs FP64 on the stored values, S=1024", "results": report}), flush=True)


def run_pointwise(args) -> None:
    """HBM roofline of the image-space kernels on the full scan's image (views x detector^2
    FP32 pixels, larger than L2): transmission forward (T; counts from a per-pixel beam), its
    VJP, the inverse of the removed fraction, the input check and the fused Poisson
    objective + seed.  Each op is launched unchecked back to back on one stream and timed
    with CUDA events; achieved = algorithmic bytes (inputs read once, outputs written once)
    / time.  The oracle's time on 2^22 pixels (one host thread) is printed beside it."""
    import numpy as np
    import torch

    from dpt_b200 import _native as N
    from dpt_b200.objectives import ObjectiveSpec, evaluate_objective, prepare_objective
    from dpt_b200.transmission import (TransmissionSpec, optical_depth_from_removed, prepare_transmission,
                                       transmission_vjp, transmit)

    device = torch.device("cuda:0")
    n = args.views * args.detector * args.detector
    generator = torch.Generator(device=device).manual_seed(args.seed)
    depth = torch.rand(n, device=device, generator=generator) * 6
    beam = torch.rand(n, device=device, generator=generator) * 1000 + 10
    seed = torch.rand(n, device=device, generator=generator) - 0.5
    out = torch.empty(n, device=device)
    grad = torch.empty(n, device=device)
    removed = torch.rand(n, device=device, generator=generator) * 0.9
    observation = torch.poisson(beam * torch.exp(-depth), generator=generator)
    prediction = beam * torch.exp(-depth) + 0.5
    loss = torch.empty(1, dtype=torch.float64, device=device)
    plain = prepare_transmission(max_pixels=n, device=device)
    counted = prepare_transmission(TransmissionSpec(beam="per-pixel"), max_pixels=n, device=device)
    poisson = prepare_objective(ObjectiveSpec(kind="poisson", domain="counts"), max_pixels=n, device=device)
    lib = N.library()
    stream = torch.cuda.current_stream(device)
    ops = [
        ("transmit T", 8, lambda: transmit(depth, out_T=out, workspace=plain, validate=False)),
        ("transmit counts (per-pixel beam)", 12,
         lambda: transmit(depth, beam, out_counts=out, workspace=counted, validate=False)),
        ("transmission VJP (T cotangent)", 12,
         lambda: transmission_vjp(depth, cotangent_T=seed, out_grad_L=grad, workspace=plain, validate=False)),
        ("optical depth from removed", 8,
         lambda: optical_depth_from_removed(removed, out_L=out, workspace=plain, validate=False)),
        ("input check (finite, nonnegative)", 4,
         lambda: lib.dpt_b200_check_values(depth.data_ptr(), n, N.CHECK_FINITE_NONNEGATIVE, plain.status.ptr,
                                           stream.cuda_stream)),
        ("Poisson objective + seed", 12,
         lambda: evaluate_objective(prediction, observation, out_loss=loss, out_cotangent=grad, workspace=poisson,
                                    validate=False)),
    ]
    peak, peak_kind = measured_peak()
    results = []
    for name, bytes_per_pixel, op in ops:
        for _ in range(max(3, args.warmup)):
            op()
        torch.cuda.synchronize()
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record(stream)
        for _ in range(args.steps):
            op()
        end.record(stream)
        end.synchronize()
        seconds = start.elapsed_time(end) * 1e-3 / args.steps
        achieved = bytes_per_pixel * n / seconds / 1e9
        results.append({"op": name, "pixels": n, "bytes_per_pixel": bytes_per_pixel,
                        "us_per_launch": round(seconds * 1e6, 1), "achieved_gbs": round(achieved, 1),
                        "frac_hbm": round(achieved / peak, 3)})
    for ws in (plain, counted):
        ws.consume_status()
    poisson.consume_status()
    cpu = None
    if not args.no_cpu_baseline:
        from oracle import pointwise as P

        sample = 1 << 22
        d = depth[:sample].cpu().numpy()
        started = time.perf_counter()
        P.transmit(d)
        P.objective(prediction[:sample].cpu().numpy(), observation[:sample].cpu().numpy(), poisson=True)
        elapsed = time.perf_counter() - started
        cpu = {"value": round(2 * sample / elapsed / 1e6, 1), "unit": "Mpixel-ops/s", "cores": 1, "kind": "port",
               "sample": f"transmit (all four outputs) + Poisson objective on {sample} pixels"}
    print(json.dumps({"metric": "image-space kernels, HBM roofline", "unit": "GB/s",
                      "config": {"workload": f"{args.views} x {args.detector}^2 FP32 image ({n} pixels)",
                                 "l2": "inputs larger than L2"},
                      "peak": {"hbm_gbs": peak, "source": f"{peak_kind} MEASURED_PEAKS hbm_gbs"},
                      "results": results, "cpu_baseline": cpu}), flush=True)


def run_gather(args) -> None:
    """Deterministic adjoint gather of the strict FP64 midpoint projector on a scan of
    ``--views`` cone views of ``--detector``^2 pixels over a ``--size``^3 chest phantom grid
    (S = ``--samples``): plan preparation once, then the culled per-voxel gather timed with
    CUDA events over ``--steps`` launches, beside the strict FP64 scatter VJP of the same
    cotangent.  Reports voxel-views, visited (voxel, sample) nodes and per-voxel node rate."""
    import numpy as np
    import torch

    from dpt_b200.geometry import ConeBeamIntrinsics
    from dpt_b200.phantoms import centred_grid
    from dpt_b200.projection import (ProjectionSpec, prepare_projection, prepare_projection_adjoint,
                                     projection_adjoint_gather, projection_vjp)

    device = torch.device("cuda:0")
    spacing = 0.8 * 256.0 / args.size
    grid = centred_grid((args.size,) * 3, (spacing,) * 3)
    geometry = ConeBeamIntrinsics(1000.0, 1500.0, (args.detector, args.detector),
                                  (0.8 * 512.0 / args.detector,) * 2).batch(
        tuple(2.0 * math.pi * k / args.views for k in range(args.views)))
    spec = ProjectionSpec(args.samples, active_pose=False, active_volume=True, precision="float64",
                          field_domain="signed_linear", validate="never")
    ws = prepare_projection(grid, geometry, spec, device=device)
    poses = torch.tensor(np.tile([1.0, 0, 0, 0, 1.0, 0, 0, 0, 1.0, 0, 0, 0], (args.views, 1)), device=device)
    plan = prepare_projection_adjoint(poses, workspace=ws, max_work=2**62, max_prepare_voxels=2**31,
                                      max_rays_per_voxel=1 << 20, max_bytes=1 << 40)
    generator = torch.Generator(device=device).manual_seed(args.seed)
    cot = torch.randn(ws.plan.image_shape, dtype=torch.float64, device=device, generator=generator)
    out = torch.empty(grid.shape, dtype=torch.float64, device=device)
    field = torch.zeros(grid.shape, dtype=torch.float32, device=device)

    def timed(fn, steps):
        for _ in range(max(1, args.warmup)):
            fn()
        torch.cuda.synchronize()
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record()
        for _ in range(steps):
            fn()
        end.record()
        end.synchronize()
        return start.elapsed_time(end) / 1e3 / steps

    gather_s = timed(lambda: projection_adjoint_gather(plan, cotangent=cot, workspace=ws, out_mu=out,
                                                       max_work=2**62, validate="never"), args.steps)
    first = out.clone()
    projection_adjoint_gather(plan, cotangent=cot, workspace=ws, out_mu=out, max_work=2**62, validate="never")
    repeatable = bool(torch.equal(first, out))
    scatter_s = timed(lambda: projection_vjp(field, poses, cotangent=cot, workspace=ws, pose_gradient=None,
                                             volume_gradient_precision="float64"), args.steps)
    voxel_views = grid.voxels * args.views
    print(json.dumps({
        "metric": "deterministic adjoint gather, strict FP64 midpoint", "unit": "voxel-views/s",
        "value": round(voxel_views / gather_s, 1),
        "config": {"workload": f"{args.size}^3 grid, {args.views} cone views {args.detector}^2, S={args.samples}",
                   "plan": {"candidate_rays": plan.candidate_rays, "quadrature_nodes": plan.quadrature_nodes,
                            "fallback_voxels": plan.fallback_voxels, "device_bytes": plan.device_bytes}},
        "gather_ms": round(gather_s * 1e3, 3), "nodes_per_s": round(plan.quadrature_nodes / gather_s, 1),
        "repeatable_bitwise": repeatable,
        "scatter_vjp_fp64_ms": round(scatter_s * 1e3, 3)}), flush=True)


def run_packed(args) -> None:
    """K forward requests of one shape (FP32 arithmetic, seeded chest phantom, cone views over
    360 deg with per-request angle offsets): one launch sequence each (``forward``) against one
    packed launch (``forward_packed``), 20 repetitions after 3 warm ones, CUDA events around
    the whole batch (host launch cost included: both are enqueued back to back).  Every packed
    image is first checked equal to its own forward."""
    import numpy as np
    import torch

    from dpt_b200.geometry import ConeBeamIntrinsics, RigidTransform
    from dpt_b200.phantoms import centred_grid, chest_phantom
    from dpt_b200.plan import plan_rays
    from dpt_b200.projection import ProjectionSpec, ProjectionWorkspace, forward_packed

    device = "cuda:0"
    rows = []
    for shape, detector, views, samples, count in ((64, 128, 1, 128, 32), (128, 128, 2, 256, 32),
                                                   (128, 256, 4, 256, 16), (256, 512, 8, 512, 8)):
        grid = centred_grid((shape,) * 3, (1.0, 1.0, 1.0))
        field = torch.tensor(chest_phantom(grid, seed=args.seed), device=device)
        pitch = 409.6 / detector
        pose = torch.tensor(np.tile(RigidTransform().packed(), (views, 1)), dtype=torch.float64, device=device)
        spaces = []
        for k in range(count):
            geometry = ConeBeamIntrinsics(1000.0, 1500.0, (detector, detector), (pitch, pitch)).batch(
                tuple(2 * math.pi * j / views + 0.01 * k for j in range(views)))
            spaces.append(ProjectionWorkspace(plan_rays(grid, geometry),
                                              ProjectionSpec(samples, sampling_precision="float32"), device))

        def each():
            return [ws.forward(field, pose, checked=False) for ws in spaces]

        def packed():
            return forward_packed([(ws, field, pose) for ws in spaces], checked=False)

        if not all(torch.equal(a, b) for a, b in zip(each(), packed(), strict=True)):
            raise SystemExit("packed images differ from the single-request forwards")
        times = {}
        for name, run in (("each", each), ("packed", packed)):
            for _ in range(3):
                run()
            torch.cuda.synchronize()
            start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            start.record()
            for _ in range(20):
                run()
            end.record()
            torch.cuda.synchronize()
            times[name] = start.elapsed_time(end) / 20
        rows.append({"requests": count, "grid": shape, "views": views, "detector": detector, "samples": samples,
                     "one_launch_each_ms": times["each"], "packed_ms": times["packed"],
                     "speedup": times["each"] / times["packed"]})
    print(json.dumps({"metric": "packed forward against one launch per request", "unit": "ms per batch",
                      "arithmetic": "FP32", "rows": rows}), flush=True)


def run_panels(args) -> None:
    """Panel kinds and the per-ray pose Jacobian on the full-scan volume: the FP32 forward
    over ``--views`` views of ``--detector``^2 as cone panels, as parallel panels (each
    view's rays along its central ray, SDD long) and as cylindrical panels (around each
    view's source), each in one launch; and, on the cone panels, the per-ray 6-row pose
    Jacobian (48 FP64 bytes written per ray) beside the per-view pose VJP of the same
    cotangent.  Rates are realised ray-samples per second (CUDA events, 3 launches after a
    warm-up)."""
    import numpy as np
    import torch

    from dpt_b200.geometry import (BatchedGeometry, ConeBeamIntrinsics, CurvedDetectorGeometry,
                                   ParallelGeometry)
    from dpt_b200.phantoms import centred_grid, chest_phantom
    from dpt_b200.projection import ProjectionSpec, ProjectionWorkspace
    from dpt_b200.plan import plan_rays

    device = torch.device("cuda:0")
    spacing = args.spacing if args.spacing else 0.8 * 256.0 / args.size
    grid = centred_grid((args.size,) * 3, (spacing,) * 3)
    intrinsics = ConeBeamIntrinsics(1000.0, 1500.0, (args.detector, args.detector),
                                    (0.8 * 512.0 / args.detector,) * 2)
    cones = [intrinsics.view(2.0 * math.pi * k / args.views) for k in range(args.views)]

    def parallel(c):
        centre = [c.origin_mm[k] + 0.5 * (c.shape[1] - 1) * c.spacing_mm[0] * c.u[k]
                  + 0.5 * (c.shape[0] - 1) * c.spacing_mm[1] * c.v[k] for k in range(3)]
        axis = [centre[k] - c.source_mm[k] for k in range(3)]
        norm = math.sqrt(sum(x * x for x in axis))
        return ParallelGeometry(c.origin_mm, tuple(x / norm for x in axis), 1500.0, c.u, c.v, c.spacing_mm, c.shape)

    def curved(c):
        # cylinder of radius SDD about the axis through the source along v, centred on the
        # central ray; pixel (0, 0) sits at arc angle a0 with u tangent there
        centre = [c.origin_mm[k] + 0.5 * (c.shape[1] - 1) * c.spacing_mm[0] * c.u[k]
                  + 0.5 * (c.shape[0] - 1) * c.spacing_mm[1] * c.v[k] for k in range(3)]
        n = [centre[k] - c.source_mm[k] for k in range(3)]
        norm = math.sqrt(sum(x * x for x in n))
        n = [x / norm for x in n]
        radius = 1500.0
        a0 = -0.5 * (c.shape[1] - 1) * c.spacing_mm[0] / radius
        row0 = -0.5 * (c.shape[0] - 1) * c.spacing_mm[1]
        origin = tuple(c.source_mm[k] + radius * (math.cos(a0) * n[k] + math.sin(a0) * c.u[k]) + row0 * c.v[k]
                       for k in range(3))
        u = tuple(-math.sin(a0) * n[k] + math.cos(a0) * c.u[k] for k in range(3))
        return CurvedDetectorGeometry(c.source_mm, origin, u, c.v, c.spacing_mm, c.shape)

    kinds = {
        "cone": BatchedGeometry(tuple(cones)),
        "parallel": BatchedGeometry(tuple(parallel(c) for c in cones)),
        "curved": BatchedGeometry(tuple(curved(c) for c in cones)),
    }
    field = torch.tensor(chest_phantom(grid, seed=args.seed), device=device)
    poses = torch.tensor(np.tile([1.0, 0, 0, 0, 1.0, 0, 0, 0, 1.0, 0, 0, 0], (args.views, 1)), device=device)

    def timed(fn, repeats=3):
        fn()
        torch.cuda.synchronize()
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record()
        for _ in range(repeats):
            fn()
        end.record()
        end.synchronize()
        return start.elapsed_time(end) / 1e3 / repeats

    results = {}
    cone_ws = None
    for name, geometry in kinds.items():
        ws = ProjectionWorkspace(plan_rays(grid, geometry),
                                 ProjectionSpec(args.samples, precision="float32", sampling_precision="float32",
                                                validate="never"), device)
        lower, upper, _ = ws.counts(poses)
        realised = int((upper > lower).sum()) * args.samples
        seconds = timed(lambda: ws.forward(field, poses))
        results[name] = {"forward_ms": round(seconds * 1e3, 3), "realised_samples": realised,
                         "samples_per_s": round(realised / seconds, 1)}
        if name == "cone":
            cone_ws = ws
    cot = torch.randn(cone_ws.plan.image_shape, device=device,
                      generator=torch.Generator(device=device).manual_seed(args.seed))
    rays = cone_ws.plan.rays
    jacobian_s = timed(lambda: cone_ws.pose_sensitivities(field, poses, cot, checked=False))
    pose_s = timed(lambda: cone_ws.vjp(field, poses, cot, volume=False, pose="tangent"))
    peak, peak_kind = measured_peak()
    print(json.dumps({
        "metric": "panel kinds and per-ray pose Jacobian, FP32 arithmetic", "unit": "ray-samples/s",
        "config": {"workload": f"{args.size}^3 chest, {args.views} views {args.detector}^2, S={args.samples}"},
        "forward": results,
        "per_ray_jacobian": {"ms": round(jacobian_s * 1e3, 3), "rays_per_s": round(rays / jacobian_s, 1),
                             "output_gbs": round(48 * rays / jacobian_s / 1e9, 1),
                             "per_view_pose_vjp_ms": round(pose_s * 1e3, 3),
                             "hbm_peak_gbs": peak, "peak_source": f"{peak_kind} MEASURED_PEAKS hbm_gbs"}}),
          flush=True)


def run_table(args) -> None:
    """Per-operation device times of the reference's published tables, on B200.

    Full scan (the headline workload: 256^3 chest at 0.8 mm, ``--views`` views of 512^2,
    S = 1024): forward, volume VJP, per-view pose VJP and the full iteration (forward +
    joint volume and pose VJP) in the FP32 and strict FP64 forms (the reference's
    ``fp32`` / ``fp64`` Projector precisions, python/dpt/torch/modules.py:69-228), and the
    FP64 cell-Gauss form.  Native chest (a synthetic chest on the 512 x 512 x 139 grid at
    0.7617 x 0.7617 x 2.5 mm standing in for the CT file; three 512^2 views at pi, pi/2 and
    3 pi/4 with the reference benchmark's geometry rule, SOD = max(1000, 2 diag), SDD =
    max(1500, 3 diag), detector width 1.05 diag SDD / (SOD - diag/2)): the strict FP64,
    mixed FP32 and fast FP32 forwards with FP64 output.  Each operation: one warm-up, then
    ``--steps`` launches, each bracketed by CUDA events with a 256 MiB L2 flush between."""
    import numpy as np
    import torch

    from dpt_b200.geometry import ConeBeamIntrinsics
    from dpt_b200.phantoms import centred_grid, chest_phantom
    from dpt_b200.plan import plan_rays
    from dpt_b200.projection import ProjectionSpec, ProjectionWorkspace

    device = torch.device("cuda:0")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=device)

    def timed(fn):
        fn()
        torch.cuda.synchronize()
        spans = []
        for _ in range(args.steps):
            flush.zero_()
            start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            start.record()
            fn()
            end.record()
            spans.append((start, end))
        torch.cuda.synchronize()
        times = sorted(s.elapsed_time(e) for s, e in spans)
        return round(times[len(times) // 2], 3)

    def identity(views):
        return torch.tensor(np.tile([1.0, 0, 0, 0, 1.0, 0, 0, 0, 1.0, 0, 0, 0], (views, 1)), device=device)

    # ---- full scan
    spacing = 0.8 * 256.0 / args.size
    grid = centred_grid((args.size,) * 3, (spacing,) * 3)
    geometry = ConeBeamIntrinsics(1000.0, 1500.0, (args.detector, args.detector),
                                  (0.8 * 512.0 / args.detector,) * 2).batch(
        tuple(2.0 * math.pi * k / args.views for k in range(args.views)))
    plan = plan_rays(grid, geometry)
    values = torch.tensor(chest_phantom(grid, seed=args.seed), device=device)
    poses = identity(args.views)
    cot = torch.randn(plan.image_shape, dtype=torch.float64, device=device,
                      generator=torch.Generator(device=device).manual_seed(args.seed))
    forms = {
        "fp32": (ProjectionSpec(args.samples, active_volume=True, precision="float32",
                                sampling_precision="float32"), torch.float32),
        "fp64": (ProjectionSpec(args.samples, active_volume=True, precision="float64",
                                sampling_precision="float64"), torch.float64),
        "cell_gauss_fp64": (ProjectionSpec(args.samples, active_volume=True, precision="float64",
                                           sampling_precision="float64", integration="cell_gauss"), torch.float64),
    }
    fullscan = {}
    realised = None
    for name, (spec, out_dtype) in forms.items():
        ws = ProjectionWorkspace(plan, spec, device)
        if realised is None:
            lower, upper, _ = ws.counts(poses)
            realised = int((upper > lower).sum()) * args.samples
        seed = cot.to(spec.image_dtype)
        volume_dtype = torch.float32 if name == "fp32" else torch.float64
        moments = ws.moments_preferred()

        def iteration():
            ws.forward(values, poses, moments=moments)
            ws.vjp(values, poses, seed, volume=True, pose="tangent", volume_dtype=volume_dtype)

        row = {"forward_ms": timed(lambda: ws.forward(values, poses)),
               "volume_vjp_ms": timed(lambda: ws.vjp(values, poses, seed, volume=True, pose=None,
                                                     volume_dtype=volume_dtype)),
               "pose_vjp_ms": timed(lambda: ws.vjp(values, poses, seed, volume=False, pose="tangent")),
               "iteration_ms": timed(iteration)}
        if spec.integration == "midpoint":
            row["iteration_realised_samples_per_s"] = round(realised / (row["iteration_ms"] * 1e-3), 1)
        fullscan[name] = row
        del ws
        torch.cuda.empty_cache()

    # ---- native chest stand-in
    shape = (139, 512, 512)
    chest_spacing = (0.7617, 0.7617, 2.5)
    chest_grid = centred_grid(shape, chest_spacing)
    diagonal = math.sqrt(sum((n * h) ** 2 for n, h in zip(shape[::-1], chest_spacing, strict=True)))
    sod, sdd = max(1000.0, 2.0 * diagonal), max(1500.0, 3.0 * diagonal)
    width = 1.05 * diagonal * sdd / (sod - diagonal / 2.0)
    chest_geometry = ConeBeamIntrinsics(sod, sdd, (512, 512), (width / 512, width / 512)).batch(
        (math.pi, math.pi / 2.0, 3.0 * math.pi / 4.0))
    chest_plan = plan_rays(chest_grid, chest_geometry)
    chest_values = torch.tensor(chest_phantom(chest_grid, seed=args.seed), device=device)
    chest_poses = identity(3)
    native = {}
    for mode in ("float64", "mixed_float32", "fast_float32"):
        ws = ProjectionWorkspace(chest_plan, ProjectionSpec(args.samples, active_pose=False, precision="float64",
                                                            sampling_precision=mode), device)
        native[mode] = {"forward_ms": timed(lambda: ws.forward(chest_values, chest_poses))}
        del ws
    print(json.dumps({
        "metric": "per-operation device time (median of --steps launches)", "unit": "ms",
        "fullscan": {"config": {"workload": f"{args.size}^3 chest at {spacing} mm, {args.views} views "
                                            f"{args.detector}^2, S={args.samples}",
                                "realised_ray_samples": realised,
                                "nominal_ray_samples": args.views * args.detector ** 2 * args.samples},
                     "results": fullscan},
        "native_chest": {"config": {"workload": "synthetic chest on 512x512x139 at 0.7617x0.7617x2.5 mm, "
                                                f"3 views 512^2, S={args.samples}, FP64 output",
                                    "sod_mm": round(sod, 3), "sdd_mm": round(sdd, 3),
                                    "detector_pitch_mm": round(width / 512, 5)},
                         "results": native},
        "data": "synthetic", "steps": args.steps}), flush=True)


def main() -> None:
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    elif args.mode == "serving":
        run_serving(args)
    elif args.mode == "precision":
        run_precision(args)
    elif args.mode == "pointwise":
        run_pointwise(args)
    elif args.mode == "gather":
        run_gather(args)
    elif args.mode == "panels":
        run_panels(args)
    elif args.mode == "table":
        run_table(args)
    elif args.mode == "packed":
        run_packed(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
