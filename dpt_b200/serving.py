"""Device-resident projection serving with continuous batching.

The reference has no serving layer; this module is the request loop the package
adds on top of the projector:

* volumes are registered once and stay resident (with their corner-replicated copy);
* requests (forward, forward + volume VJP, forward + pose VJP) of any grid, view count,
  detector and sample count arrive on a queue;
* an admission loop starts a request as soon as a stream slot is free and its device
  memory fits the budget (first fit over a bounded look-ahead, so a large request
  waiting for memory does not block small ones behind it);
* every admitted request runs on its own CUDA stream, so requests that arrive while
  others are on the GPU overlap on the device; requests that fill the GPU on their own
  (``exclusive_samples`` nominal ray-samples and more) run one at a time, with only small
  ones (under ``beside_samples``) beside them, because requests that run at once interleave
  their blocks and evict each other's field copy and accumulator records from L2 (with
  ``priorities=True`` the smaller ones run
  on high-priority streams, so their blocks start as soon as blocks of the large request
  retire: p50 latency 4.0 against 8.4 ms on a 48-request mix, at 0.66-0.99x the throughput);
* repeated request shapes below ``graph_samples`` nominal ray-samples replay a captured
  CUDA graph of their launch sequence (larger requests are launch-count bound no more, and
  a replay must copy its outputs out of the graph's static buffers);
* forward requests below ``pack_samples`` nominal ray-samples may run on a pack lane of
  their own beside the general slots: when ``pack_min`` or more of them wait on volumes of
  one storage dtype at one precision, the lane takes them as one packed launch (up to
  ``MAX_PACK``: one block per (request, view, tile) item of them all), so a burst of small
  requests costs one launch instead of one launch sequence each.  A few small requests go
  to the general slots instead: on a mixed stream a fifth concurrent stream interleaves
  their blocks with a large request's and costs more than their launches (96-request mix:
  157-170 requests/s packing every small forward, 185-187 without);
* the detector tile of each request class comes from a small autotuner that times each
  candidate tile three times the first time a class is seen and keeps the default unless
  another is 3 % faster;
* which waiting requests start is decided by ``LaunchPolicy`` (no GPU needed, so its rules
  are tested on the CPU).

Results are exactly those of the same request run alone: the kernels are the same and
requests share no scratch (each slot owns its workspaces).  Packed launches take their
workspaces from one server-wide set (one per request class, kept across packs) and run one
at a time; requests of one class packed together share that class's workspace and its
status words, so a status bit one of them raises is reported to each of them.
"""

from __future__ import annotations

import itertools
import queue
import threading
import time
from collections import OrderedDict, deque
from collections.abc import Callable
from concurrent.futures import Future
from dataclasses import dataclass, field
from typing import Any, Literal

from .contracts import ContractError, integer
from .projection import FieldCopies, ScratchPool

RequestKind = Literal["forward", "volume", "pose"]


@dataclass(frozen=True)
class ProjectionRequest:
    """One projection job against a registered volume.

    ``kind``: ``"forward"`` returns the image; ``"volume"`` also returns the gradient of
    ``0.5 * |image - target|^2`` with respect to the volume; ``"pose"`` the gradient with
    respect to the per-view pose tangent.  ``target`` (host or device, image shape)
    defaults to zeros.  ``tangent`` is an optional ``(views, 6)`` pose increment.
    """

    volume: str
    geometry: Any
    samples_per_ray: int
    kind: RequestKind = "forward"
    target: Any = None
    tangent: Any = None
    precision: Literal["fp32", "fp64"] = "fp32"

    def __post_init__(self) -> None:
        integer(self.samples_per_ray, "samples_per_ray", minimum=1)
        if self.kind not in ("forward", "volume", "pose"):
            raise ContractError("request kind must be forward, volume or pose")
        if self.precision not in ("fp32", "fp64"):
            raise ContractError("precision must be fp32 or fp64")


@dataclass
class ProjectionResult:
    image: Any
    loss: float | None = None
    volume_gradient: Any = None
    pose_gradient: Any = None
    submitted: float = 0.0
    started: float = 0.0
    finished: float = 0.0

    @property
    def latency(self) -> float:
        return self.finished - self.submitted


class Admission:
    """Memory-budget admission with a bounded first-fit look-ahead (no GPU needed).

    ``offer(item, bytes)`` queues a request; ``take(free_slots)`` returns the requests that
    can start now in arrival order, skipping (up to ``lookahead`` entries) those that do
    not fit the remaining budget; ``release(bytes)`` returns memory when one finishes.
    A request larger than the whole budget is rejected at ``offer``.
    """

    def __init__(self, budget_bytes: int, lookahead: int = 16) -> None:
        if budget_bytes <= 0:
            raise ContractError("memory budget must be positive")
        self.budget = int(budget_bytes)
        self.lookahead = lookahead
        self.in_use = 0
        self.peak = 0
        self.waiting: deque[tuple[Any, int]] = deque()

    def offer(self, item: Any, nbytes: int) -> None:
        if nbytes > self.budget:
            raise ContractError(f"request needs {nbytes} bytes, more than the {self.budget}-byte budget")
        self.waiting.append((item, int(nbytes)))

    def take(self, free_slots: int, eligible: Callable[[Any], bool] | None = None) -> list[tuple[Any, int]]:
        """Start what fits, in arrival order; ``eligible(item)`` (called in that order, once
        per candidate that fits the budget) may hold an item back for now."""
        started: list[tuple[Any, int]] = []
        index = 0
        while free_slots > 0 and index < min(len(self.waiting), self.lookahead):
            item, nbytes = self.waiting[index]
            if self.in_use + nbytes <= self.budget and (eligible is None or eligible(item)):
                del self.waiting[index]
                self.in_use += nbytes
                self.peak = max(self.peak, self.in_use)
                started.append((item, nbytes))
                free_slots -= 1
            else:
                index += 1
        return started

    def take_matching(self, match: Callable[[Any], bool], limit: int) -> list[tuple[Any, int]]:
        """Start up to ``limit`` more waiting items for which ``match(item)`` holds and that fit
        the budget, in arrival order over the whole queue (companions of a packed launch)."""
        started: list[tuple[Any, int]] = []
        index = 0
        while len(started) < limit and index < len(self.waiting):
            item, nbytes = self.waiting[index]
            if self.in_use + nbytes <= self.budget and match(item):
                del self.waiting[index]
                self.in_use += nbytes
                self.peak = max(self.peak, self.in_use)
                started.append((item, nbytes))
            else:
                index += 1
        return started

    def release(self, nbytes: int) -> None:
        self.in_use -= int(nbytes)
        if self.in_use < 0:
            raise ContractError("released more memory than was admitted")


class LaunchPolicy:
    """Which waiting requests start now (no GPU needed).

    Items carry ``pack_class`` (None, or the class of a forward request small enough to pack),
    ``large`` (fills the GPU on its own) and ``medium`` (too large to run beside a large one).
    With a pack lane, a pack class is due when ``pack_min`` or more of its items wait; the lane
    takes the oldest due item's class whole (up to ``max_pack``), and the general slots leave
    the items of a due class for it.  Large items run one at a time; while one runs, medium
    items wait too.
    """

    def __init__(self, pack_min: int, max_pack: int, lane: bool) -> None:
        self.pack_min = pack_min
        self.max_pack = max_pack
        self.lane = lane

    @staticmethod
    def pack_counts(admission: Admission) -> dict[Any, int]:
        counts: dict[Any, int] = {}
        for item, _ in admission.waiting:
            if item.pack_class is not None:
                counts[item.pack_class] = counts.get(item.pack_class, 0) + 1
        return counts

    def held(self, item: Any, counts: dict[Any, int]) -> bool:
        """Whether a waiting item is kept for the pack lane's next launch."""
        return self.lane and counts.get(item.pack_class, 0) >= self.pack_min

    def take_pack(self, admission: Admission) -> list[Any]:
        """The due pack, taken from the queue (empty when none is due or none fits)."""
        if not self.lane:
            return []
        counts = self.pack_counts(admission)
        first = next((item for item, _ in admission.waiting
                      if counts.get(item.pack_class, 0) >= self.pack_min), None)
        if first is None:
            return []
        return [item for item, _ in admission.take_matching(
            lambda other, c=first.pack_class: other.pack_class == c, self.max_pack)]

    def take_singles(self, admission: Admission, free_slots: int, large_running: int) -> tuple[list[Any], int]:
        """Items for the free general slots, in arrival order, and the new large count."""
        counts = self.pack_counts(admission)
        large_now = large_running

        def eligible(item: Any) -> bool:
            nonlocal large_now
            if self.held(item, counts) or (item.medium and large_now):
                return False
            if not item.large:
                return True
            if large_now:
                return False
            large_now += 1
            return True

        taken = [item for item, _ in admission.take(free_slots, eligible)]
        return taken, large_now

    def startable(self, admission: Admission, lane_free: bool, any_slot_free: bool, large_running: int) -> bool:
        """Whether a scheduling pass would start something (the scheduler sleeps otherwise)."""
        if not admission.waiting:
            return False
        counts = self.pack_counts(admission)
        if self.lane and lane_free and counts and max(counts.values()) >= self.pack_min:
            return True
        if not any_slot_free:
            return False
        window = itertools.islice(admission.waiting, admission.lookahead)
        return any(not self.held(item, counts) and not ((item.large or item.medium) and large_running)
                   for item, _ in window)


class TileTuner:
    """Chooses the detector block tile (8, 16, 32 or 64 columns) per request class.

    ``choose(key, run)`` calls ``run(block_cols)`` -> seconds ``repeats`` times per candidate
    the first time a class is seen and keeps the fastest by its best time; a candidate must
    beat the default tile (16 columns, the first candidate) by ``margin`` to replace it, so
    timing noise cannot swap the default for a tile that is no faster.  Later calls return the
    choice directly.
    """

    CANDIDATES = (16, 32, 8, 64)

    def __init__(self, repeats: int = 3, margin: float = 0.03) -> None:
        self.repeats = repeats
        self.margin = margin
        self.choices: dict[Any, int] = {}
        self.timings: dict[Any, dict[int, float]] = {}
        self.lock = threading.Lock()

    def choose(self, key: Any, run: Callable[[int], float]) -> int:
        with self.lock:
            if key in self.choices:
                return self.choices[key]
        timings = {cols: min(run(cols) for _ in range(self.repeats)) for cols in self.CANDIDATES}
        default = self.CANDIDATES[0]
        best = min(timings, key=timings.get)
        if timings[best] * (1.0 + self.margin) > timings[default]:
            best = default
        with self.lock:
            self.timings[key] = timings
            self.choices[key] = best
        return best


def percentile(values: list[float], q: float) -> float:
    """Nearest-rank percentile (q in [0, 100])."""
    if not values:
        raise ContractError("no values")
    ordered = sorted(values)
    rank = max(1, min(len(ordered), int(-(-q * len(ordered) // 100))))
    return ordered[rank - 1]


# ----------------------------------------------------------------- the server


@dataclass
class _Volume:
    grid: Any
    field: Any  # device tensor, contiguous, storage dtype


@dataclass
class _Job:
    request: ProjectionRequest
    future: Future
    submitted: float
    nbytes: int = 0
    slot: Any = None
    started: float = 0.0
    event: Any = None
    outputs: dict = field(default_factory=dict)
    workspace: Any = None
    key: Any = None  # request class: volume, geometry, samples, precision, kind
    large: bool = False  # fills the GPU on its own: runs while no other large request does
    medium: bool = False  # not large, but too large to run beside a large request
    private_host: bool = False  # own pinned readback buffers instead of the slot's
    pack_class: Any = None  # (storage dtype, precision) of a forward request that may be packed
    group: list | None = None  # [members still running] of the packed launch this job is in


class _Slot:
    """CUDA streams with their own workspaces (scratch is never shared across slots) and
    reusable pinned staging buffers (a slot runs one request at a time).  With priorities, a
    request that fills the GPU runs on the slot's normal-priority stream and every other one on
    its high-priority stream: the block scheduler then starts a small request's blocks as the
    large request's blocks retire instead of after the large request's whole kernel."""

    def __init__(self, torch, device, index: int, stream=None, priorities: bool = False) -> None:
        self.torch = torch
        self.index = index
        if stream is None:
            self.normal = torch.cuda.Stream(device=device)
            self.urgent = torch.cuda.Stream(device=device, priority=-1) if priorities else self.normal
        else:
            self.normal = self.urgent = stream
        self.stream = self.normal  # the stream of the request the slot runs
        self.workspaces: OrderedDict[Any, Any] = OrderedDict()
        self.graphs: dict[Any, Any] = {}
        self.pool = ScratchPool(device)  # gradient scratch shared by this slot's workspaces
        self.classes: set[Any] = set()  # request classes whose workspace (and graph) this slot holds
        self.busy = False
        self._pinned: dict[str, Any] = {}

    def pinned(self, name: str, count: int, dtype):
        """A pinned host buffer of at least ``count`` elements, reused across requests."""
        buffer = self._pinned.get(name)
        if buffer is None or buffer.numel() < count or buffer.dtype != dtype:
            buffer = self.torch.empty(max(count, 64), dtype=dtype, pin_memory=True)
            self._pinned[name] = buffer
        return buffer[:count]


class ProjectionServer:
    """Continuous-batching request loop over resident volumes on one GPU.

    ``submit`` returns a ``concurrent.futures.Future`` resolving to a
    ``ProjectionResult`` whose tensors stay on the device.  ``slots`` requests run
    concurrently, each on its own stream; admission also respects
    ``memory_budget_bytes`` (120 GiB by default).  ``graphs=True`` captures the
    launch sequence of each (slot, request class) after its first run and replays it;
    ``autotune=True`` picks the detector tile per request class; ``packing=True`` runs forward
    requests below ``pack_samples`` nominal ray-samples as one launch when ``pack_min`` or more
    of one class wait together; while a request of ``exclusive_samples`` or more runs, only
    requests under ``beside_samples`` start beside it; ``priorities=True`` runs requests that
    do not fill the GPU on high-priority streams (lower
    latency for them; on the mixed stream, less throughput: their blocks then interleave with
    the large request's and evict its data from L2).
    """

    def __init__(self, device: str = "cuda:0", *, memory_budget_bytes: int = 120 << 30, slots: int = 4,
                 graphs: bool = True, autotune: bool = True, workspaces_per_slot: int = 64,
                 graph_samples: int = 1 << 30, exclusive_samples: int = 1 << 30, packing: bool = True,
                 pack_samples: int = 1 << 26, pack_min: int = 8, priorities: bool = False,
                 beside_samples: int = 1 << 28) -> None:
        import torch

        self.torch = torch
        self.device = torch.device(device)
        if self.device.type != "cuda":
            raise ContractError("the projection server runs on a CUDA device")
        integer(slots, "slots", minimum=1, maximum=64)
        self.slots = [_Slot(torch, self.device, k, priorities=priorities) for k in range(slots)]
        self.admission = Admission(memory_budget_bytes)
        self.tuner = TileTuner()
        self.graphs = graphs
        self.graph_samples = graph_samples
        self.exclusive_samples = exclusive_samples
        self.beside_samples = beside_samples
        self.large_running = 0
        self.packing = packing
        self.pack_samples = pack_samples
        self.pack_min = pack_min
        self.packs = 0  # packed launches made
        self.packed_requests = 0  # requests that ran inside them
        # packed launches run on a lane of their own (one pack at a time: packs share the
        # server-wide pack workspaces), beside the general slots
        self.pack_lane = _Slot(torch, self.device, slots, priorities=priorities) if packing else None
        if self.pack_lane is not None:
            self.pack_lane.stream = self.pack_lane.urgent
        from ._native import MAX_PACK

        self.policy = LaunchPolicy(pack_min, MAX_PACK, self.pack_lane is not None)
        self.pack_workspaces: OrderedDict[Any, Any] = OrderedDict()
        self.pack_workspace_limit = 256
        self.autotune = autotune
        self.workspaces_per_slot = workspaces_per_slot
        self.volumes: dict[str, _Volume] = {}
        # one sampling copy per resident volume and layout, shared by all slots and classes
        self.copies = FieldCopies()
        self._alone: _Slot | None = None
        self._identity: dict[int, Any] = {}
        self.lock = threading.Condition()
        self.inbox: queue.Queue = queue.Queue()
        self.running: deque[_Job] = deque()
        self.closed = False
        self.errors: list[BaseException] = []
        self._scheduler = threading.Thread(target=self._schedule, name="dpt-schedule", daemon=True)
        self._completer = threading.Thread(target=self._complete, name="dpt-complete", daemon=True)
        self._scheduler.start()
        self._completer.start()

    # ----------------------------------------------------------- volumes
    def add_volume(self, name: str, grid, values, storage: str = "float32") -> None:
        """Upload (or adopt) a volume; it stays resident until ``remove_volume``."""
        torch = self.torch
        dtype = {"float32": torch.float32, "float16": torch.float16, "bfloat16": torch.bfloat16}[storage]
        tensor = values if isinstance(values, torch.Tensor) else torch.as_tensor(values)
        tensor = tensor.to(device=self.device, dtype=dtype).contiguous()
        if tuple(tensor.shape) != tuple(grid.shape):
            raise ContractError("volume values must have grid shape (nz, ny, nx)")
        with self.lock:
            self.volumes[name] = _Volume(grid, tensor)

    def remove_volume(self, name: str) -> None:
        with self.lock:
            self.volumes.pop(name)
            for key in [k for k in self.pack_workspaces if k[0] == name]:
                del self.pack_workspaces[key]
            for slot in self._lanes():
                for key in [k for k in slot.workspaces if k[0] == name]:
                    del slot.workspaces[key]
                for key in [k for k in slot.graphs if k[0] == name]:
                    del slot.graphs[key]

    # -------------------------------------------------------------- API
    def submit(self, request: ProjectionRequest) -> Future:
        if request.volume not in self.volumes:
            raise ContractError(f"unknown volume {request.volume!r}")
        from .plan import batched

        future: Future = Future()
        job = _Job(request, future, time.perf_counter())
        job.nbytes = self.request_bytes(request)
        job.large = self._large(request)
        job.medium = not job.large and self._large(request, self.beside_samples)
        job.key = (request.volume, batched(request.geometry), request.samples_per_ray, request.precision,
                   request.kind)
        if self.packing and request.kind == "forward" and not job.large and \
                batched(request.geometry).pixels * request.samples_per_ray < self.pack_samples:
            job.pack_class = (str(self.volumes[request.volume].field.dtype), request.precision)
        with self.lock:
            if self.closed:
                raise ContractError("server is closed")
            self.admission.offer(job, job.nbytes)
            self.lock.notify_all()
        return future

    def run_alone(self, request: ProjectionRequest) -> ProjectionResult:
        """Run one request synchronously on the caller's stream (the sequential baseline:
        plain calls with their workspaces kept warm, no graphs, no tuning)."""
        if self._alone is None:
            self._alone = _Slot(self.torch, self.device, -1, self.torch.cuda.current_stream(self.device))
        job = _Job(request, Future(), time.perf_counter())
        job.slot = self._alone
        job.started = time.perf_counter()
        self._launch(job, use_graph=False)
        job.event.synchronize()
        return self._finish(job)

    def run_chained(self, requests: list[ProjectionRequest]) -> list[ProjectionResult]:
        """Enqueue the launch sequences of ``requests`` back to back on the caller's stream with
        no synchronisation between them (the same arithmetic as ``run_alone``); return their
        results once the stream has finished them all."""
        if self._alone is None:
            self._alone = _Slot(self.torch, self.device, -1, self.torch.cuda.current_stream(self.device))
        jobs = []
        for request in requests:
            job = _Job(request, Future(), time.perf_counter())
            job.slot = self._alone
            job.private_host = True
            job.started = time.perf_counter()
            self._launch(job, use_graph=False)
            jobs.append(job)
        if jobs:
            jobs[-1].event.synchronize()
        return [self._finish(job) for job in jobs]

    def close(self) -> None:
        with self.lock:
            self.closed = True
            self.lock.notify_all()
        self._scheduler.join()
        self._completer.join()

    def __enter__(self):
        return self

    def __exit__(self, *exc) -> None:
        self.close()

    def _lanes(self) -> list[_Slot]:
        return self.slots + ([self.pack_lane] if self.pack_lane is not None else [])

    # ---------------------------------------------------------- sizing
    def _large(self, request: ProjectionRequest, threshold: int | None = None) -> bool:
        """Whether a request fills the GPU on its own (nominal ray-samples of its passes at least
        ``exclusive_samples``, or ``threshold``): such requests run one at a time, because two
        of them interleave their blocks and evict each other's field copy and accumulator
        records from L2."""
        from .plan import batched

        passes = 1 if request.kind == "forward" else 2
        limit = self.exclusive_samples if threshold is None else threshold
        return batched(request.geometry).pixels * request.samples_per_ray * passes >= limit

    def _small(self, request: ProjectionRequest) -> bool:
        """Whether a request is small enough for graph replay to pay (nominal ray-samples)."""
        from .plan import batched

        return batched(request.geometry).pixels * request.samples_per_ray < self.graph_samples

    def request_bytes(self, request: ProjectionRequest) -> int:
        from .plan import batched

        volume = self.volumes[request.volume]
        geometry = batched(request.geometry)
        rays = geometry.pixels
        image = 8 if request.precision == "fp64" else 4
        total = 3 * rays * image + 4096
        voxels = volume.grid.voxels
        # the field copy and the slot's gradient scratch are shared and counted once, when
        # the volume is added; a request needs its images, gradient and pose partials
        if request.kind == "volume":
            total += voxels * 4
        if request.kind == "pose":
            total += len(geometry.views) * ((rays // len(geometry.views)) // 256 + 1) * 96 + 96 * rays // 256
        return total

    # ------------------------------------------------------- scheduling
    def _schedule(self) -> None:
        while True:
            with self.lock:
                while not self.closed and not self._startable():
                    self.lock.wait(0.05)
                if self.closed and not self.admission.waiting:
                    return
                launches = []
                lane = self.pack_lane
                if lane is not None and not lane.busy:
                    group = self.policy.take_pack(self.admission)
                    if group:
                        lane.busy = True
                        running = [len(group)]
                        for member in group:
                            member.slot = lane
                            member.group = running
                        launches.append(group)
                free = [slot for slot in self.slots if not slot.busy]
                taken, self.large_running = self.policy.take_singles(self.admission, len(free), self.large_running)
                for job in taken:
                    # prefer a free slot that already holds this class's workspace and graph
                    slot = next((s for s in free if job.key in s.classes), free[0])
                    free.remove(slot)
                    slot.busy = True
                    slot.classes.add(job.key)
                    slot.stream = slot.normal if job.large else slot.urgent
                    job.slot = slot
                    launches.append([job])
                if not launches:
                    # nothing fits the memory budget now: wait for a completion to release some
                    self.lock.wait(0.05)
                    continue
            for group in launches:
                started = time.perf_counter()
                try:
                    for job in group:
                        job.started = started
                    if group[0].group is not None:
                        self._launch_pack(group)
                    else:
                        self._launch(group[0], use_graph=self.graphs and self._small(group[0].request))
                except BaseException as error:  # surfaced through the futures
                    for job in group:
                        job.outputs["error"] = error
                        job.event = None
                with self.lock:
                    self.running.extend(group)
                    self.lock.notify_all()

    def _startable(self) -> bool:
        lane = self.pack_lane
        return self.policy.startable(self.admission, lane is not None and not lane.busy,
                                     any(not slot.busy for slot in self.slots), self.large_running)

    def _complete(self) -> None:
        while True:
            with self.lock:
                while not self.running and not (self.closed and not self.admission.waiting
                                                and not any(s.busy for s in self._lanes())):
                    self.lock.wait(0.05)
                if not self.running:
                    return
                # complete whichever request finished first: no head-of-line blocking
                job = next((j for j in self.running if j.event is None or j.event.query()), None)
                if job is None:
                    self.lock.wait(0.0002)
                    continue
                self.running.remove(job)
            try:
                if "error" in job.outputs:
                    raise job.outputs["error"]
                result = self._finish(job)
                job.future.set_result(result)
            except BaseException as error:
                job.future.set_exception(error)
            with self.lock:
                if job.group is not None:
                    job.group[0] -= 1  # the lane is free once every member of its pack is done
                if job.group is None or job.group[0] == 0:
                    job.slot.busy = False
                if job.large:
                    self.large_running -= 1
                self.admission.release(job.nbytes)
                self.lock.notify_all()

    # -------------------------------------------------------- execution
    def _workspace_key(self, request: ProjectionRequest, block_cols: int):
        from .plan import batched

        volume = self.volumes[request.volume]
        return (request.volume, batched(request.geometry), request.samples_per_ray, request.precision,
                request.kind, volume.field.dtype, block_cols)

    def _new_workspace(self, request: ProjectionRequest, block_cols: int, pool):
        from .plan import batched, plan_rays
        from .projection import ProjectionSpec, ProjectionWorkspace

        volume = self.volumes[request.volume]
        half = volume.field.dtype != self.torch.float32
        sampling = "compensated" if half else ("float64" if request.precision == "fp64" else "float32")
        storage = {self.torch.float16: "float16", self.torch.bfloat16: "bfloat16"}.get(volume.field.dtype, "float32")
        spec = ProjectionSpec(request.samples_per_ray, active_pose=request.kind == "pose",
                              active_volume=request.kind == "volume",
                              precision="float64" if request.precision == "fp64" else "float32",
                              sampling_precision=sampling, storage_precision=storage, block_cols=block_cols)
        return ProjectionWorkspace(plan_rays(volume.grid, batched(request.geometry)), spec, self.device,
                                   copies=self.copies, pool=pool)

    def _pack_workspace(self, request: ProjectionRequest, block_cols: int):
        """The server-wide workspace of a packable request class (forward only: no scratch)."""
        key = self._workspace_key(request, block_cols)
        found = self.pack_workspaces.get(key)
        if found is None:
            found = self._new_workspace(request, block_cols, None)
            self.pack_workspaces[key] = found
            while len(self.pack_workspaces) > self.pack_workspace_limit:
                self.pack_workspaces.popitem(last=False)
        else:
            self.pack_workspaces.move_to_end(key)
        return found

    def _workspace(self, slot: _Slot, request: ProjectionRequest, block_cols: int):
        key = self._workspace_key(request, block_cols)
        found = slot.workspaces.get(key)
        if found is None:
            found = self._new_workspace(request, block_cols, slot.pool)
            slot.workspaces[key] = found
            while len(slot.workspaces) > self.workspaces_per_slot:
                evicted, _ = slot.workspaces.popitem(last=False)
                # a captured graph points into its workspace's scratch: drop them together
                slot.graphs.pop(evicted, None)
                slot.classes.discard(evicted[:5])
        else:
            slot.workspaces.move_to_end(key)
        return key, found

    def _poses(self, request: ProjectionRequest, views: int, slot: _Slot | None = None):
        """Device poses ``(views, 12)``: a cached identity, or the composed tangent staged
        through the slot's pinned buffer."""
        import numpy as np

        from .geometry import RigidTransform, compose_pose

        torch = self.torch
        if request.tangent is None:
            found = self._identity.get(views)
            if found is None:
                identity = torch.tensor(RigidTransform().packed(), dtype=torch.float64, device=self.device)
                found = identity.expand(views, 12).contiguous()
                self._identity[views] = found
            return found
        tangent = np.asarray(request.tangent, dtype=np.float64).reshape(-1, 6)
        tangent = np.broadcast_to(tangent, (views, 6))
        packed = np.asarray([compose_pose(RigidTransform(), tuple(map(float, t))).packed() for t in tangent])
        if slot is None:
            return torch.tensor(packed, dtype=torch.float64, device=self.device)
        host = slot.pinned("poses", views * 12, torch.float64)
        host.copy_(torch.from_numpy(packed.reshape(-1)))
        return host.view(views, 12).to(self.device, non_blocking=True)

    def _block_cols(self, request: ProjectionRequest, slot: _Slot) -> int:
        from .plan import batched

        if not self.autotune:
            return 0
        volume = self.volumes[request.volume]
        geometry = batched(request.geometry)
        key = (volume.grid.shape, geometry.shape, request.samples_per_ray, request.kind, request.precision,
               str(volume.field.dtype))
        torch = self.torch

        def run(cols: int) -> float:
            _, ws = self._workspace(slot, request, cols)
            poses = self._poses(request, len(geometry.views))
            with torch.cuda.stream(slot.stream):
                ws.forward(volume.field, poses, checked=False)  # warm
                start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                start.record(slot.stream)
                ws.forward(volume.field, poses, checked=False)
                end.record(slot.stream)
            end.synchronize()
            ws.status.zero_()
            return start.elapsed_time(end)

        return self.tuner.choose(key, run)

    def _launch(self, job: _Job, use_graph: bool) -> None:
        torch = self.torch
        request, slot = job.request, job.slot
        block_cols = self._block_cols(request, slot) if slot.index >= 0 else 0
        key, ws = self._workspace(slot, request, block_cols)
        volume = self.volumes[request.volume]
        views = ws.plan.views
        with torch.cuda.stream(slot.stream):
            state = slot.graphs.get(key) if use_graph else None
            if state is None:
                # chained requests stage no host data through the slot's shared pinned buffer
                staging = None if job.private_host else slot
                inputs = {"poses": self._poses(request, views, staging), "target": self._target(request, ws)}
                outputs = self._body(ws, volume.field, inputs, request)
                if use_graph:
                    self._capture(slot, key, ws, volume.field, request, inputs)
            else:
                graph, inputs, outputs = state
                inputs["poses"].copy_(self._poses(request, views, slot), non_blocking=True)
                if inputs["target"] is not None:
                    inputs["target"].copy_(self._target(request, ws), non_blocking=True)
                graph.replay()
                outputs = {name: value.clone() for name, value in outputs.items()}
            # a slot runs one request at a time and reuses its pinned buffers; requests chained
            # without synchronisation each need their own
            def host(name: str, count: int, dtype):
                if job.private_host:
                    return torch.empty(count, dtype=dtype, pin_memory=True)
                return slot.pinned(name, count, dtype)

            status_host = host("status", views, torch.int32)
            status_host.copy_(ws.status, non_blocking=True)
            ws.status.zero_()
            job.outputs = dict(outputs, status=status_host)
            if "loss" in outputs:  # read back with the status, no host synchronisation later
                loss_host = host("loss", 1, torch.float64)
                loss_host.copy_(outputs["loss"].reshape(1), non_blocking=True)
                job.outputs["loss_host"] = loss_host
            job.workspace = ws
            job.event = torch.cuda.Event()
            job.event.record(slot.stream)

    def _launch_pack(self, jobs: list[_Job]) -> None:
        """One packed forward launch for ``jobs`` (small forward requests of one class) on
        their common slot; each job gets its image, status words and the launch's event."""
        from .projection import forward_packed

        torch = self.torch
        slot = jobs[0].slot
        calls, spaces = [], []
        for job in jobs:
            request = job.request
            block_cols = self._block_cols(request, slot)
            ws = self._pack_workspace(request, block_cols)
            # poses through a pageable copy: the slot's pinned staging holds one request's only
            poses = self._poses(request, ws.plan.views)
            calls.append((ws, self.volumes[request.volume].field, poses))
            spaces.append(ws)
        with torch.cuda.stream(slot.stream):
            images = forward_packed(calls, checked=False)
            readback = {}
            for k, ws in enumerate(dict.fromkeys(spaces)):
                host = slot.pinned(f"status{k}", ws.plan.views, torch.int32)
                host.copy_(ws.status, non_blocking=True)
                readback[id(ws)] = host
            for ws in dict.fromkeys(spaces):
                ws.status.zero_()
            event = torch.cuda.Event()
            event.record(slot.stream)
        for job, ws, image in zip(jobs, spaces, images, strict=True):
            job.workspace = ws
            job.outputs = {"image": image, "status": readback[id(ws)]}
            job.event = event
        self.packs += 1
        self.packed_requests += len(jobs)

    def _as_device(self, value):
        torch = self.torch
        tensor = value if isinstance(value, torch.Tensor) else torch.as_tensor(value)
        return tensor.to(self.device, non_blocking=True)

    def _target(self, request: ProjectionRequest, ws):
        """Device target image, or None for a zero target (the residual is then the image)."""
        if request.kind == "forward" or request.target is None:
            return None
        return self._as_device(request.target).to(ws.spec.image_dtype).reshape(ws.plan.image_shape).clone()

    def _body(self, ws, field_tensor, inputs, request: ProjectionRequest) -> dict:
        """Launch sequence of one request on the current stream (no host synchronisation).
        A pose request in FP32 arithmetic stores its rays' pose moments in the forward, so its
        pose VJP applies the residual without a second sampling pass."""
        moments = request.kind == "pose" and ws.moments_preferred()
        image = ws.forward(field_tensor, inputs["poses"], checked=False, moments=moments)
        out = {"image": image}
        if request.kind != "forward":
            residual = image if inputs["target"] is None else image - inputs["target"]
            out["loss"] = 0.5 * (residual.double() * residual.double()).sum()
            if request.kind == "volume":
                out["volume_gradient"], _ = ws.vjp(field_tensor, inputs["poses"], residual, volume=True,
                                                   pose=None, checked=False)
            else:
                _, out["pose_gradient"] = ws.vjp(field_tensor, inputs["poses"], residual, volume=False,
                                                 pose="tangent", checked=False)
        return out

    def _capture(self, slot: _Slot, key, ws, field_tensor, request, inputs) -> None:
        torch = self.torch
        static = {"poses": inputs["poses"].clone(),
                  "target": None if inputs["target"] is None else inputs["target"].clone()}
        graph = torch.cuda.CUDAGraph()
        slot.stream.synchronize()
        # capture on the slot's stream alone: the torch.cuda.graph context would synchronise the
        # whole device and empty the allocator's cache first, holding every queued request
        # behind the long requests on the other slots.  Thread-local capture: the completion
        # thread may read finished results meanwhile.
        with torch.cuda.stream(slot.stream):
            graph.capture_begin(capture_error_mode="thread_local")
            try:
                outputs = self._body(ws, field_tensor, static, request)
            finally:
                graph.capture_end()
        ws.status.zero_()
        slot.graphs[key] = (graph, static, outputs)

    def _finish(self, job: _Job) -> ProjectionResult:
        from .contracts import NumericalError, raise_device_status

        outputs = job.outputs
        codes = outputs["status"].tolist()
        for view, code in enumerate(codes):
            if code:
                try:
                    raise_device_status(code, "projection")
                except (ContractError, NumericalError) as error:
                    error.args = (f"projection view {view}: {error}", *error.args[1:])
                    raise
        loss = outputs.get("loss_host")
        return ProjectionResult(
            image=outputs["image"],
            loss=None if loss is None else float(loss[0]),
            volume_gradient=outputs.get("volume_gradient"),
            pose_gradient=outputs.get("pose_gradient"),
            submitted=job.submitted,
            started=job.started,
            finished=time.perf_counter(),
        )


_ids = itertools.count()
