"""Projection workspaces: device tables, scratch and checked calls over the C ABI.

``ProjectionSpec`` and ``prepare_projection`` mirror the reference's lower-level
operator layer (hcltech-robotics/dpt ``python/dpt/projection.py:67-140`` and
``:526-622``); ``project_optical_depth``, ``projection_vjp`` and
``projection_pose_sensitivities`` mirror ``:747-809``, ``:871-1018`` and
``:1021-1084``.  Arrays are torch CUDA tensors and work is enqueued on the
caller's current torch stream.

A workspace owns, per device:

* the panel table or ray bundle of its plan (uploaded once),
* the corner-replicated copy of the last prepared field (reused while the same
  tensor is passed again unchanged, tracked through torch's version counter),
* the per-cell FP32 volume accumulator (kept zero between calls), an FP64 running
  total for the widening of the volume gradient, FP64 pose partials,
* one int32 status word per view and a pinned host copy for the checkpoint.

Checked calls end with one status readback and a wait on the stream (the
reference's ``StatusCheckpoint``, ``python/dpt/_runtime.py:318-446``); a nonzero
word raises ``ContractError`` (bit 1), ``TrialDomainError`` (bit 8) or
``NumericalError`` (bit 2), names the view and clears the words, so the next
call starts clean.
"""

from __future__ import annotations

import contextlib
import ctypes
import threading
import weakref
from dataclasses import dataclass
from typing import Literal

import torch

from . import _native as N
from .contracts import ContractError, NumericalError, integer, raise_device_status
from .plan import RayPlan, plan_rays
from .volumes import GridSpec

SamplingPrecision = Literal["float32", "float64", "mixed_float32", "fast_float32", "compensated"]
StoragePrecision = Literal["float32", "float16", "bfloat16"]

_STORAGE = {"float32": (N.F32, torch.float32), "float16": (N.F16, torch.float16),
            "bfloat16": (N.BF16, torch.bfloat16)}
_ARITH = {"float32": N.ARITH_F32, "float64": N.ARITH_F64, "mixed_float32": N.ARITH_MIXED,
          "fast_float32": N.ARITH_FAST, "compensated": N.ARITH_F32C}


@dataclass(frozen=True, slots=True)
class ProjectionSpec:
    """Quadrature and arithmetic of one projector (reference ``ProjectionSpec``,
    python/dpt/projection.py:67-140, with this package's launch options).

    ``integration``: ``"midpoint"`` uses ``samples_per_ray`` clipped midpoints;
    ``"cell_gauss"`` splits the ray at every interpolation plane and integrates each
    cubic segment exactly with two Gauss nodes (FP64 sampling; the sample count is then
    ignored).  ``sampling_precision``: ``"float64"`` the reference strict projector;
    ``"float32"`` the reference FP32 projector (FP64 ray setup, FP32 clip, interpolation
    and serial ray sum; FP32 storage); ``"mixed_float32"`` FP32 marching and corner
    weights with FP64 products and sums, ``"fast_float32"`` the same with an FP32 cell
    sum (both fixed-pose); ``"compensated"`` this package's precision form for FP16/BF16
    storage (closed-form sums over the cell runs, compensated FP32 ray sum).
    ``storage_precision`` FP32, FP16 or BF16 field storage (decoded exactly on the
    device); ``field_domain`` ``"physical"`` (finite, non-negative attenuation) or
    ``"signed_linear"`` (any finite value); ``validate`` ``"once"``/``"always"`` check
    field and poses on every call (the check is fused into the pass that writes the
    field copy), ``"never"`` skips reading the status words back.  ``precision`` is the
    image / cotangent dtype.  ``widen_views`` is how many views accumulate in FP32
    before the volume gradient is widened into its FP64 total (the reference uses 8 for
    FP32 and 2 for FP64 sampling; the compensated form defaults to 32).  ``layout`` selects the field copy or direct gathers;
    ``block_cols`` the detector tile of one block (8, 16, 32 or 64 columns; 0 = 16), a
    launch-shape choice that does not change results.
    """

    samples_per_ray: int
    active_pose: bool = True
    active_volume: bool = False
    precision: Literal["float32", "float64"] = "float32"
    sampling_precision: SamplingPrecision = "float64"
    storage_precision: StoragePrecision = "float32"
    widen_views: int | None = None
    layout: Literal["replicated", "direct"] = "replicated"
    block_cols: int = 0
    integration: Literal["midpoint", "cell_gauss"] = "midpoint"
    field_domain: Literal["physical", "signed_linear"] = "physical"
    validate: Literal["once", "always", "never"] = "once"

    def __post_init__(self) -> None:
        integer(self.samples_per_ray, "samples_per_ray", minimum=1)
        if self.integration not in ("midpoint", "cell_gauss"):
            raise ContractError("projection integration must be midpoint or cell_gauss")
        if self.precision not in ("float32", "float64"):
            raise ContractError("projection precision must be float32 or float64")
        if self.field_domain not in ("physical", "signed_linear"):
            raise ContractError("projection field_domain must be physical or signed_linear")
        if self.sampling_precision not in _ARITH:
            raise ContractError("sampling_precision must be float32, float64, mixed_float32, fast_float32 "
                                "or compensated")
        if self.storage_precision not in _STORAGE:
            raise ContractError("storage_precision must be float32, float16 or bfloat16")
        if self.sampling_precision in ("mixed_float32", "fast_float32") and (
            self.integration != "midpoint" or self.active_pose
        ):
            raise ContractError("FP32 sampling requires midpoint integration and fixed pose")
        if self.sampling_precision == "float32" and (
            self.integration != "midpoint" or self.storage_precision != "float32"
        ):
            raise ContractError("FP32 arithmetic requires midpoint integration and FP32 field storage")
        if self.sampling_precision == "compensated" and self.integration != "midpoint":
            raise ContractError("compensated sampling requires midpoint integration")
        if type(self.active_pose) is not bool or type(self.active_volume) is not bool:
            raise ContractError("active input flags must be booleans")
        if self.validate not in ("once", "always", "never"):
            raise ContractError("projection validate must be once, always or never")
        if self.widen_views is not None:
            integer(self.widen_views, "widen_views", minimum=1)
        if self.layout not in ("replicated", "direct"):
            raise ContractError("layout must be replicated or direct")
        if self.layout == "direct" and self.storage_precision != "float32":
            raise ContractError("the direct layout reads FP32 storage only")
        if self.block_cols not in (0, 8, 16, 32, 64):
            raise ContractError("block_cols must be 0 (default), 8, 16, 32 or 64")

    @property
    def arith(self) -> int:
        if self.integration == "cell_gauss":
            return N.ARITH_CELLS
        return _ARITH[self.sampling_precision]

    @property
    def domain_code(self) -> int:
        return N.DOMAIN_SIGNED if self.field_domain == "signed_linear" else N.DOMAIN_PHYSICAL

    @property
    def field_code(self) -> int:
        return _STORAGE[self.storage_precision][0]

    @property
    def field_dtype(self) -> torch.dtype:
        return _STORAGE[self.storage_precision][1]

    @property
    def image_code(self) -> int:
        return N.F64 if self.precision == "float64" else N.F32

    @property
    def image_dtype(self) -> torch.dtype:
        return torch.float64 if self.precision == "float64" else torch.float32

    @property
    def batch_views(self) -> int:
        if self.widen_views is not None:
            return self.widen_views
        if self.sampling_precision in ("float64", "mixed_float32", "fast_float32"):
            return 2
        # the compensated form's cell-run sums reach the accumulator already aggregated per
        # cell crossing: 32 views in FP32 keep the widened gradient within 1e-6 of FP64 while
        # folding a quarter as often as the reference's 8
        return 32 if self.sampling_precision == "compensated" else 8


def _ptr(tensor: torch.Tensor | None) -> int | None:
    return None if tensor is None else tensor.data_ptr()


def _stream(device: torch.device) -> int:
    return torch.cuda.current_stream(device).cuda_stream


class FieldCopies:
    """Field copies (the replicated or polynomial sampling layout) shared by every workspace
    on one device that samples the same field with the same layout, so that many request
    classes over one resident volume hold one copy instead of one each.

    An entry is keyed by the field's storage pointer, its version counter and the layout; it
    lives while the field does.  A workspace that finds the copy written on another stream
    waits for the event recorded after the write before it samples the copy.
    """

    def __init__(self) -> None:
        self._entries: dict[tuple, tuple] = {}
        self._lock = threading.Lock()

    def lookup(self, key: tuple, field: torch.Tensor):
        with self._lock:
            entry = self._entries.get(key)
            if entry is None:
                return None
            ref, tensor, event = entry
            if ref() is not field:
                del self._entries[key]
                return None
            return tensor, event

    def store(self, key: tuple, field: torch.Tensor, tensor: torch.Tensor, event) -> None:
        with self._lock:
            # drop copies of dead fields and older versions of this one (same pointer, layout)
            for stale in [k for k, (ref, _, _) in self._entries.items()
                          if ref() is None or (k[0] == key[0] and k[2:] == key[2:])]:
                del self._entries[stale]
            self._entries[key] = (weakref.ref(field), tensor, event)

    def bytes(self) -> int:
        with self._lock:
            return sum(t.numel() * t.element_size() for _, t, _ in self._entries.values())


class ScratchPool:
    """Volume-gradient scratch (the 32-byte corner-sum records and the FP64 running total)
    shared by workspaces that never run at the same time, e.g. the request classes of one
    serving stream: one buffer per voxel count instead of one per workspace.  The records
    are left zeroed by every fold, so a workspace can take over the buffer another left."""

    def __init__(self, device: torch.device | str) -> None:
        self.device = torch.device(device)
        self._accumulators: dict[int, torch.Tensor] = {}
        self._totals: dict[int, torch.Tensor] = {}

    def accumulator(self, floats: int) -> torch.Tensor:
        found = self._accumulators.get(floats)
        if found is None:
            found = torch.zeros(floats, dtype=torch.float32, device=self.device)
            self._accumulators[floats] = found
        return found

    def total(self, voxels: int) -> torch.Tensor:
        found = self._totals.get(voxels)
        if found is None:
            found = torch.empty(voxels, dtype=torch.float64, device=self.device)
            self._totals[voxels] = found
        return found


class ProjectionWorkspace:
    """Device state of one (grid, geometry, spec) on one CUDA device.

    ``copies`` (a FieldCopies) shares the field's sampling copy with other workspaces;
    ``pool`` (a ScratchPool) shares the volume-gradient scratch with workspaces that never
    run concurrently with this one."""

    def __init__(self, plan: RayPlan, spec: ProjectionSpec, device: torch.device | str, *,
                 copies: FieldCopies | None = None, pool: ScratchPool | None = None) -> None:
        device = torch.device(device)
        if device.type != "cuda":
            raise ContractError("the B200 projector runs on CUDA devices only")
        if spec.sampling_precision != "float64" and max(plan.grid.shape) > 2**24:
            raise ContractError("FP32 sampling requires grid axis counts at most 2**24")
        N.library()
        self.plan = plan
        self.spec = spec
        self.device = device
        self.lock = threading.RLock()
        self.copies = copies
        self.pool = pool
        self.problem = plan.problem(
            spec.samples_per_ray,
            spec.arith,
            field_dtype=spec.field_code,
            image_dtype=spec.image_code,
            layout=N.LAYOUT_DIRECT if spec.layout == "direct" else N.LAYOUT_REPLICATED,
            block_cols=spec.block_cols,
            field_domain=spec.domain_code,
        )
        with torch.cuda.device(device):
            self.view_table = (
                torch.from_numpy(plan.view_table).to(device) if plan.view_table is not None else None
            )
            self.sources = torch.from_numpy(plan.sources).to(device) if plan.sources is not None else None
            self.endpoints = (
                torch.from_numpy(plan.endpoints).to(device) if plan.endpoints is not None else None
            )
            self.status = torch.zeros(plan.views, dtype=torch.int32, device=device)
            self.status_host = torch.zeros(plan.views, dtype=torch.int32, pin_memory=True)
        self._packed: torch.Tensor | None = None
        self._packed_for: tuple | None = None
        self._accumulator: torch.Tensor | None = None
        self._total: torch.Tensor | None = None
        self._partials: torch.Tensor | None = None
        self._moments: torch.Tensor | None = None
        self._moments_for: tuple | None = None
        # Optional instrumentation: a list receiving (name, view_begin, view_count,
        # start_event, end_event) per C-ABI call, and a count of C-ABI calls.
        self.launch_log: list | None = None
        self.launches = 0

    # ------------------------------------------------------------ scratch
    @property
    def views(self) -> int:
        return self.plan.views

    def scratch_bytes(self) -> int:
        total = 0
        for tensor in (self._packed, self._accumulator, self._total, self._partials, self._moments):
            if tensor is not None:
                total += tensor.numel() * tensor.element_size()
        return total

    def release_scratch(self) -> None:
        """Drop the cached field copy and gradient scratch (allocated again on demand)."""
        self._packed = self._packed_for = None
        self._accumulator = self._total = self._partials = None
        self._moments = self._moments_for = None

    def _bytes(self, size: int) -> torch.Tensor:
        # 256-byte aligned storage from the caching allocator
        return torch.empty(max(size, 1), dtype=torch.uint8, device=self.device)

    def accumulator(self) -> torch.Tensor:
        if self._accumulator is None:
            size = N.library().dpt_b200_accumulator_bytes(self.problem)
            if self.pool is not None:
                self._accumulator = self.pool.accumulator(size // 4)
            else:
                self._accumulator = torch.zeros(size // 4, dtype=torch.float32, device=self.device)
        return self._accumulator

    def total(self) -> torch.Tensor:
        if self._total is None:
            if self.pool is not None:
                self._total = self.pool.total(self.plan.grid.voxels)
            else:
                self._total = torch.empty(self.plan.grid.voxels, dtype=torch.float64, device=self.device)
        return self._total

    def partials(self) -> torch.Tensor:
        size = N.library().dpt_b200_pose_partials_bytes(self.problem, self.views)
        if self._partials is None or self._partials.numel() * 8 < size:
            self._partials = torch.empty(max(size // 8, 1), dtype=torch.float64, device=self.device)
        return self._partials

    # ------------------------------------------------------------- inputs
    def check_field(self, field: torch.Tensor) -> torch.Tensor:
        if not isinstance(field, torch.Tensor):
            raise ContractError("field must be a Torch tensor")
        if field.device != self.device:
            raise ContractError("field must be on the workspace device")
        if field.dtype != self.spec.field_dtype:
            raise ContractError(f"field must use {self.spec.storage_precision} storage")
        if field.numel() != self.plan.grid.voxels or not field.is_contiguous():
            raise ContractError("field must be contiguous with grid shape (nz,ny,nx)")
        return field

    def check_poses(self, poses: torch.Tensor) -> torch.Tensor:
        if not isinstance(poses, torch.Tensor) or poses.dtype != torch.float64:
            raise ContractError("poses must be a float64 Torch tensor")
        if poses.device != self.device:
            raise ContractError("poses must be on the workspace device")
        if poses.numel() == 12 and self.views > 1:
            poses = poses.reshape(1, 12).expand(self.views, 12)
        if tuple(poses.shape) not in ((self.views, 12), (12,)) or poses.numel() != 12 * self.views:
            raise ContractError(f"poses must have shape ({self.views}, 12)")
        return poses.reshape(self.views, 12).contiguous()

    def rays(self, poses: torch.Tensor, view_begin: int = 0, view_count: int | None = None) -> N.Rays:
        r = N.Rays()
        r.poses = poses.data_ptr()
        r.view_table = _ptr(self.view_table)
        r.ray_sources = _ptr(self.sources)
        r.ray_endpoints = _ptr(self.endpoints)
        r.view_begin = view_begin
        r.view_count = self.views - view_begin if view_count is None else view_count
        return r

    def prepare_field(self, field: torch.Tensor, poses: torch.Tensor) -> torch.Tensor:
        """Validate field and poses (status bits 8 and 1) and return the sampling layout."""
        lib = N.library()
        if self.spec.layout == "direct":
            self._run("prepare_field", lambda: lib.dpt_b200_prepare_field(self.problem, field.data_ptr(), None, poses.data_ptr(),
                                           self.status.data_ptr(), _stream(self.device)))
            return field
        if self._packed is not None and self._packed_for is not None:
            ref, version, pointer = self._packed_for
            if ref() is field and version == field._version and pointer == field.data_ptr():
                # unchanged field: validate again (field and poses) without rewriting the copy
                self._run("prepare_field", lambda: lib.dpt_b200_prepare_field(self.problem, field.data_ptr(), None,
                                               poses.data_ptr(), self.status.data_ptr(),
                                               _stream(self.device)))
                return self._packed
        size = lib.dpt_b200_packed_bytes(self.problem)
        key = (field.data_ptr(), field._version, self.problem.arith == N.ARITH_F32C, size)
        if self.copies is not None:
            found = self.copies.lookup(key, field)
            if found is not None:
                copy, event = found
                torch.cuda.current_stream(self.device).wait_event(event)
                self._run("prepare_field", lambda: lib.dpt_b200_prepare_field(
                    self.problem, field.data_ptr(), None, poses.data_ptr(), self.status.data_ptr(),
                    _stream(self.device)))
                self._packed = copy
                self._packed_for = (weakref.ref(field), field._version, field.data_ptr())
                return copy
            self._packed = None  # never write into a copy other workspaces share
        if self._packed is None or self._packed.numel() < size:
            self._packed = self._bytes(size)
        self._run("prepare_field", lambda: lib.dpt_b200_prepare_field(self.problem, field.data_ptr(), self._packed.data_ptr(),
                                       poses.data_ptr(), self.status.data_ptr(), _stream(self.device)))
        self._packed_for = (weakref.ref(field), field._version, field.data_ptr())
        if self.copies is not None:
            event = torch.cuda.Event()
            event.record(torch.cuda.current_stream(self.device))
            self.copies.store(key, field, self._packed, event)
        return self._packed

    # ----------------------------------------------------------- launches
    def _run(self, name: str, call, view_begin: int = 0, view_count: int | None = None) -> None:
        """Make one C-ABI call; with ``launch_log`` set, bracket it with CUDA events."""
        self.launches += 1
        log = self.launch_log
        if log is None:
            N.check(call(), name)
            return
        stream = torch.cuda.current_stream(self.device)
        start = torch.cuda.Event(enable_timing=True)
        end = torch.cuda.Event(enable_timing=True)
        start.record(stream)
        code = call()
        end.record(stream)
        N.check(code, name)
        count = self.views - view_begin if view_count is None else view_count
        log.append((name, view_begin, count, start, end))

    # --------------------------------------------------------- checkpoint
    def consume_status(self, operator: str = "projection") -> None:
        """Read every status word once, raise the first typed error, clear the words."""
        self.status_host.copy_(self.status, non_blocking=True)
        torch.cuda.current_stream(self.device).synchronize()
        codes = self.status_host.tolist()
        if any(codes):
            self.status.zero_()
            failures = []
            for view, code in enumerate(codes):
                if code:
                    try:
                        raise_device_status(code, operator)
                    except (ContractError, NumericalError) as error:
                        error.args = (f"{operator} view {view}: {error}", *error.args[1:])
                        failures.append(error)
            first = failures[0]
            for view, code in enumerate(codes):
                if code:
                    first.add_note(f"view {view} status {code}")
            raise first

    # ------------------------------------------------------------ compute
    # Largest stored pose moments (FP32 words) a workspace keeps between a forward and its VJP.
    MOMENT_BYTES_LIMIT = 16 << 30

    def moments_supported(self) -> bool:
        """Whether a forward can store the pose moments for a later pose VJP (FP32 or
        compensated arithmetic, FP32 images, within MOMENT_BYTES_LIMIT)."""
        return (self.spec.arith in (N.ARITH_F32, N.ARITH_F32C) and self.spec.image_code == N.F32 and
                N.library().dpt_b200_moments_bytes(self.problem, self.views) <= self.MOMENT_BYTES_LIMIT)

    def moments_preferred(self) -> bool:
        """Whether a training step should store the pose moments in its forward (and run the
        volume-only scatter in its VJP) rather than run a plain forward and a joint volume +
        pose VJP.  Measured on 64 views of the 256^3 / 512^2 / S = 1024 full scan: FP32
        arithmetic 101.1 ms split against 114.5 ms joint; the compensated form 65.4 ms split
        against 64.2 ms joint (its moment-storing forward costs more than the pose terms add
        to a pass bound by its scatter)."""
        return self.spec.arith == N.ARITH_F32 and self.moments_supported()

    def _moments_match(self, field: torch.Tensor, poses: torch.Tensor) -> bool:
        """Whether the stored moments belong to these inputs.  The workspace holds the
        inputs of the forward that stored them, so equal storage pointers cannot come from
        another tensor reusing the memory; equal version counters mean unchanged contents."""
        kept = self._moments_for
        if kept is None:
            return False
        f0, p0, fv, pv = kept
        return (field.data_ptr() == f0.data_ptr() and poses.data_ptr() == p0.data_ptr()
                and field._version == fv and poses._version == pv)

    def forward(self, field: torch.Tensor, poses: torch.Tensor, out: torch.Tensor | None = None,
                *, checked: bool = True, moments: bool = False) -> torch.Tensor:
        """Optical depth ``(views, rows, cols)`` (bundles: ``(rays,)``).

        ``moments=True`` (FP32 or compensated arithmetic) also stores each ray's pose moments, so that a
        following ``vjp`` with the same field and poses forms the pose gradient without
        sampling again; the image is identical either way."""
        with self.lock, torch.cuda.device(self.device):
            field = self.check_field(field)
            poses = self.check_poses(poses)
            if out is None:
                out = torch.empty(self.plan.image_shape, dtype=self.spec.image_dtype, device=self.device)
            elif (tuple(out.shape) != self.plan.image_shape or out.dtype != self.spec.image_dtype
                  or out.device != self.device or not out.is_contiguous()):
                raise ContractError("out must match the projector's shape, dtype and input device")
            packed = self.prepare_field(field, poses)
            self._moments_for = None
            if moments and self.moments_supported():
                lib = N.library()
                size = lib.dpt_b200_moments_bytes(self.problem, self.views)
                if self._moments is None or self._moments.numel() * 4 < size:
                    self._moments = torch.empty(size // 4, dtype=torch.float32, device=self.device)
                self._run("forward_moments", lambda: lib.dpt_b200_forward_moments(
                    self.problem, self.rays(poses), packed.data_ptr(), out.data_ptr(),
                    self._moments.data_ptr(), self.status.data_ptr(), _stream(self.device)))
                self._moments_for = (field, poses, field._version, poses._version)
            else:
                self._run("forward", lambda: N.library().dpt_b200_forward(self.problem, self.rays(poses), packed.data_ptr(),
                                                 out.data_ptr(), self.status.data_ptr(),
                                                 _stream(self.device)))
            if checked and self.spec.validate != "never":
                self.consume_status()
            return out

    def vjp(self, field: torch.Tensor, poses: torch.Tensor, cotangent: torch.Tensor, *,
            volume: bool, pose: Literal["matrix", "tangent", None] = "matrix",
            volume_dtype: torch.dtype = torch.float32, checked: bool = True,
            ) -> tuple[torch.Tensor | None, torch.Tensor | None]:
        """Volume gradient (voxels, ``volume_dtype``) and per-view pose gradient
        (``(views, 12)`` packed or ``(views, 6)`` local-right tangent)."""
        if not volume and pose is None:
            raise ContractError("request at least one projection gradient")
        with self.lock, torch.cuda.device(self.device):
            lib = N.library()
            field = self.check_field(field)
            poses = self.check_poses(poses)
            cot = self._cotangent(cotangent)
            packed = self.prepare_field(field, poses)
            flags = N.VJP_VOLUME if volume else 0
            components = 0
            if pose == "matrix":
                flags |= N.VJP_POSE12
                components = 12
            elif pose == "tangent":
                flags |= N.VJP_POSE6
                components = 6
            # pose moments stored by the forward of these same inputs: the pose VJP needs no
            # sampling and the sampling pass scatters the volume cotangent alone
            split = bool(components) and self._moments_match(field, poses)
            if split:
                flags &= N.VJP_VOLUME
                self._moments_for = None  # consumed: release the forward's inputs
            accumulator = self.accumulator().data_ptr() if volume else None
            partials = self.partials() if components else None
            gradient = (torch.empty(self.plan.grid.shape, dtype=volume_dtype, device=self.device)
                        if volume else None)
            grad_code = N.F64 if volume_dtype == torch.float64 else N.F32
            stream = _stream(self.device)
            batch = self.spec.batch_views if volume else self.views
            rays_per_view = self.plan.rays_per_view
            element = cot.element_size()
            # launch-log label: what each sampling launch computes
            label = "vjp" if (volume and components and not split) else "vjp_volume" if volume else "vjp_pose"
            if split:
                self._run("pose_from_moments", lambda: lib.dpt_b200_pose_from_moments(
                    self.problem, self.rays(poses), self._moments.data_ptr(), cot.data_ptr(),
                    N.VJP_POSE12 if components == 12 else N.VJP_POSE6, partials.data_ptr(),
                    self.status.data_ptr(), stream))
            for first in range(0, self.views if volume else 0 if split else self.views, batch):
                count = min(batch, self.views - first)
                seed_ptr = cot.data_ptr() + first * rays_per_view * element
                part_ptr = None
                if partials is not None and not split:
                    tiles = lib.dpt_b200_pose_partials_bytes(self.problem, 1) // (12 * 8)
                    part_ptr = partials.data_ptr() + first * tiles * components * 8
                self._run(label, lambda: lib.dpt_b200_vjp(self.problem, self.rays(poses, first, count), packed.data_ptr(),
                                     seed_ptr, flags, accumulator, part_ptr, self.status.data_ptr(),
                                     stream), first, count)
                if volume:
                    last = first + count >= self.views
                    single = count >= self.views
                    self._run("fold", lambda: lib.dpt_b200_fold_volume(
                            self.problem, accumulator,
                            None if single else self.total().data_ptr(),
                            1 if first > 0 else 0,
                            gradient.data_ptr() if last else None, grad_code, 1,
                            self.status.data_ptr(), stream))
            pose_gradient = None
            if components:
                pose_gradient = torch.empty((self.views, components), dtype=torch.float64,
                                            device=self.device)
                self._run("finish_pose", lambda: lib.dpt_b200_finish_pose(self.problem, 0, self.views, components,
                                             partials.data_ptr(), pose_gradient.data_ptr(), 0,
                                             self.status.data_ptr(), stream))
            if checked and self.spec.validate != "never":
                self.consume_status()
            return gradient, pose_gradient

    def pose_sensitivities(self, field: torch.Tensor, poses: torch.Tensor, cotangent: torch.Tensor,
                           *, checked: bool = True) -> torch.Tensor:
        """Per-ray rows ``cotangent[p] * dL[p]/d xi`` in local-right order, shape (rays, 6)."""
        with self.lock, torch.cuda.device(self.device):
            field = self.check_field(field)
            poses = self.check_poses(poses)
            cot = self._cotangent(cotangent)
            packed = self.prepare_field(field, poses)
            out = torch.empty((self.plan.rays, 6), dtype=torch.float64, device=self.device)
            self._run("pose_sensitivities", lambda: N.library().dpt_b200_vjp(self.problem, self.rays(poses), packed.data_ptr(),
                                         cot.data_ptr(), N.VJP_PER_RAY6, None, out.data_ptr(),
                                         self.status.data_ptr(), _stream(self.device)))
            if checked and self.spec.validate != "never":
                self.consume_status()
            return out

    def counts(self, poses: torch.Tensor) -> tuple[torch.Tensor, torch.Tensor, torch.Tensor]:
        """Per-ray clip interval (lower, upper) and realised midpoint count."""
        with self.lock, torch.cuda.device(self.device):
            poses = self.check_poses(poses)
            n = self.plan.rays
            lower = torch.empty(n, dtype=torch.float64, device=self.device)
            upper = torch.empty(n, dtype=torch.float64, device=self.device)
            realised = torch.empty(n, dtype=torch.int32, device=self.device)
            self._run("counts", lambda: N.library().dpt_b200_counts(self.problem, self.rays(poses), lower.data_ptr(),
                                            upper.data_ptr(), realised.data_ptr(),
                                            self.status.data_ptr(), _stream(self.device)))
            return lower, upper, realised

    # ------------------------------------------------------------ helpers
    def _cotangent(self, cotangent: torch.Tensor) -> torch.Tensor:
        if not isinstance(cotangent, torch.Tensor) or cotangent.device != self.device:
            raise ContractError("cotangent must be a Torch tensor on the workspace device")
        if cotangent.dtype != self.spec.image_dtype or cotangent.numel() != self.plan.rays:
            raise ContractError("cotangent must match the projected image shape and dtype")
        flat = cotangent.contiguous().reshape(-1)
        if flat.stride() != (1,):
            flat = flat.clone()
        return flat


def forward_packed(calls, *, checked: bool = True) -> list[torch.Tensor]:
    """Optical depth of several workspaces in one launch.

    ``calls`` is a sequence of ``(workspace, field, poses)`` or ``(workspace, field, poses,
    out)``: at most ``N.MAX_PACK`` of them, on one device, with one sampling arithmetic, field
    layout and image dtype; a workspace may appear more than once, with one field (its
    sampling copy is shared by those calls) and any poses.  Each field is validated (and its
    sampling copy written) as by ``ProjectionWorkspace.forward``; one launch then walks the (view, tile) blocks of every call,
    so many small projections fill the GPU without a launch (and a tail) each.  Every image
    equals that workspace's own forward bit for bit.  Returns the images in call order."""
    calls = list(calls)
    if not 1 <= len(calls) <= N.MAX_PACK:
        raise ContractError(f"a packed forward takes 1 to {N.MAX_PACK} calls")
    spaces = [call[0] for call in calls]
    first = spaces[0]
    for ws in spaces:
        if not isinstance(ws, ProjectionWorkspace) or ws.device != first.device:
            raise ContractError("packed calls need projection workspaces on one device")
        if (ws.spec.arith, ws.problem.layout, ws.spec.image_code) != (first.spec.arith, first.problem.layout,
                                                                    first.spec.image_code):
            raise ContractError("packed calls need one sampling arithmetic, field layout and image dtype")
    with contextlib.ExitStack() as stack, torch.cuda.device(first.device):
        # each workspace once, in one global order (by identity), so that two packed calls
        # naming the same workspaces in different orders cannot each hold what the other waits for
        for ws in sorted(dict.fromkeys(spaces), key=id):
            stack.enter_context(ws.lock)
        count = len(calls)
        problems = (N.Problem * count)()
        rays = (N.Rays * count)()
        copies = (ctypes.c_void_p * count)()
        images = (ctypes.c_void_p * count)()
        status = (ctypes.c_void_p * count)()
        outs, keep, fields_of = [], [], {}
        for k, call in enumerate(calls):
            ws, field, poses = call[0], call[1], call[2]
            out = call[3] if len(call) > 3 else None
            # a workspace holds one sampling copy: it repeats in a pack only with one field
            if ws.problem.layout != N.LAYOUT_DIRECT and fields_of.setdefault(id(ws), field) is not field:
                raise ContractError("a workspace repeats in a packed forward only with the same field")
            field = ws.check_field(field)
            poses = ws.check_poses(poses)
            if out is None:
                out = torch.empty(ws.plan.image_shape, dtype=ws.spec.image_dtype, device=ws.device)
            elif (tuple(out.shape) != ws.plan.image_shape or out.dtype != ws.spec.image_dtype
                  or out.device != ws.device or not out.is_contiguous()):
                raise ContractError("out must match the projector's shape, dtype and input device")
            copy = ws.prepare_field(field, poses)
            ws._moments_for = None
            problems[k] = ws.problem
            rays[k] = ws.rays(poses)
            copies[k] = copy.data_ptr()
            images[k] = out.data_ptr()
            status[k] = ws.status.data_ptr()
            outs.append(out)
            keep.append((field, poses, copy))
        N.check(N.library().dpt_b200_forward_packed(count, problems, rays, copies, images, status,
                                                    _stream(first.device)), "forward_packed")
        for ws in dict.fromkeys(spaces):
            ws.launches += 1
            if checked and ws.spec.validate != "never":
                ws.consume_status()
        return outs


def prepare_projection(grid: GridSpec, geometry, spec: ProjectionSpec, *,
                       device: str | torch.device = "cuda:0") -> ProjectionWorkspace:
    """Build the plan of ``grid`` and ``geometry`` and its device workspace."""
    if not isinstance(spec, ProjectionSpec):
        raise ContractError("spec must be a ProjectionSpec")
    return ProjectionWorkspace(plan_rays(grid, geometry), spec, device)


def project_optical_depth(field: torch.Tensor, pose: torch.Tensor, *, workspace: ProjectionWorkspace,
                          out_L: torch.Tensor | None = None) -> torch.Tensor:
    """``L[p] = integral mu(r_p(s)) ds`` for every ray of the workspace."""
    return workspace.forward(field, pose, out_L)


def projection_vjp(field: torch.Tensor, pose: torch.Tensor, *, cotangent: torch.Tensor,
                   workspace: ProjectionWorkspace, pose_gradient: Literal["matrix", "tangent", None] = "tangent",
                   volume_gradient: bool = True,
                   volume_gradient_precision: Literal["float32", "float64"] = "float32"):
    """``(grad_mu, grad_pose) = J^T cotangent`` of the projection."""
    dtype = torch.float64 if volume_gradient_precision == "float64" else torch.float32
    return workspace.vjp(field, pose, cotangent, volume=volume_gradient, pose=pose_gradient,
                         volume_dtype=dtype)


def projection_pose_sensitivities(field: torch.Tensor, pose: torch.Tensor, *, cotangent: torch.Tensor,
                                  workspace: ProjectionWorkspace) -> torch.Tensor:
    """Per-ray weighted local-right pose Jacobian rows, shape (rays, 6)."""
    return workspace.pose_sensitivities(field, pose, cotangent)


# ------------------------------------------------------------ deterministic adjoint gather

def _gather_metadata(workspace: ProjectionWorkspace) -> tuple:
    spec = workspace.spec
    return (id(workspace.plan), spec.samples_per_ray, spec.sampling_precision, spec.integration, spec.precision)


def _gather_problem(workspace: ProjectionWorkspace) -> N.Problem:
    arith = N.ARITH_CELLS if workspace.spec.integration == "cell_gauss" else N.ARITH_F64
    return workspace.plan.problem(workspace.spec.samples_per_ray, arith, image_dtype=workspace.spec.image_code)


@dataclass(frozen=True, eq=False)
class PreparedProjectionAdjoint:
    """Captured rays and culling metrics of the strict FP64 midpoint operator A(pose) of one
    workspace (reference ``PreparedProjectionAdjoint``, python/dpt/projection.py:1087-1247).

    The plan owns its FP64 ray records (independent of later changes to the pose buffer);
    ``candidate_rays`` and ``quadrature_nodes`` count the (voxel, ray) and (voxel, sample)
    pairs the culled gather visits, ``fallback_voxels`` the voxels whose detector bounds fell
    back to the whole panel, ``device_bytes`` the plan's device memory."""

    workspace: ProjectionWorkspace
    records: torch.Tensor
    poses: torch.Tensor
    candidate_rays: int
    quadrature_nodes: int
    fallback_voxels: int
    device_bytes: int
    preparation_work_bound: int
    metadata: tuple

    @property
    def work_bound(self) -> int:
        return self.workspace.plan.grid.voxels + self.candidate_rays + self.quadrature_nodes


def _write_gather_plan(workspace: ProjectionWorkspace, poses: torch.Tensor, nbytes: int) -> torch.Tensor:
    lib = N.library()
    problem = _gather_problem(workspace)
    records = torch.empty(nbytes // 8, dtype=torch.float64, device=workspace.device)
    rays = workspace.rays(poses)
    workspace._run("gather_prepare", lambda: lib.dpt_b200_gather_prepare(
        problem, rays, records.data_ptr(), workspace.status.data_ptr(), _stream(workspace.device)))
    workspace.consume_status("prepared gather")
    return records


def prepare_projection_adjoint(pose: torch.Tensor, *, workspace: ProjectionWorkspace, max_work: int = 10_000_000,
                               max_prepare_voxels: int = 16_777_216, max_rays_per_voxel: int = 256,
                               max_bytes: int = 256 * 1024 * 1024) -> PreparedProjectionAdjoint:
    """Capture the ray setup of A(pose) and its conservative strict-midpoint gather bounds.

    Validates the poses (rigid) and every ray and sample node, then counts the candidate rays
    and nodes of every voxel.  ``max_prepare_voxels`` and ``max_rays_per_voxel`` bound the
    preparation and each voxel's candidate rectangle, ``max_work`` the all-node validation
    and the plan's gather queries, ``max_bytes`` the plan's device memory."""
    spec = workspace.spec
    if spec.sampling_precision != "float64" or spec.integration != "midpoint":
        raise ContractError("prepared gather requires strict float64 midpoint sampling")
    for value, name in ((max_work, "max_work"), (max_prepare_voxels, "max_prepare_voxels"),
                        (max_rays_per_voxel, "max_rays_per_voxel"), (max_bytes, "max_bytes")):
        integer(value, name, minimum=1, maximum=2**63 - 1)
    integer(max_rays_per_voxel, "max_rays_per_voxel", minimum=1, maximum=2**31 - 1)
    voxels, pixels = workspace.plan.grid.voxels, workspace.plan.rays
    setup_nodes = pixels * spec.samples_per_ray
    if voxels > max_prepare_voxels or voxels > max_work:
        raise ContractError("prepared gather exceeds max_prepare_voxels or max_work")
    if setup_nodes > max_work:
        raise ContractError("all-node ray validation exceeds max_work")
    if voxels * pixels * (spec.samples_per_ray + 1) + voxels > 2**63 - 1:
        raise ContractError("prepared gather work counters exceed signed 64-bit range")
    lib = N.library()
    problem = _gather_problem(workspace)
    device_bytes = lib.dpt_b200_gather_plan_bytes(problem, workspace.views) + 12 * 8 * workspace.views + 32
    if device_bytes > max_bytes:
        raise ContractError(f"prepared gather requires {device_bytes} device bytes; max_bytes is {max_bytes}")
    poses = workspace.check_poses(pose).clone()
    records = _write_gather_plan(workspace, poses, device_bytes - 12 * 8 * workspace.views - 32)
    totals = torch.zeros(4, dtype=torch.int64, device=workspace.device)
    rays = workspace.rays(poses)
    workspace._run("gather_count", lambda: lib.dpt_b200_gather_count(
        problem, rays, records.data_ptr(), max_rays_per_voxel, totals.data_ptr(), _stream(workspace.device)))
    candidate_rays, nodes, limited, fallbacks = (int(v) for v in totals.cpu().tolist())
    if limited:
        raise ContractError(f"{limited} voxel bounds exceed max_rays_per_voxel")
    work = voxels + candidate_rays + nodes
    if work > max_work:
        raise ContractError(f"prepared gather needs {work} bounded queries; max_work is {max_work}")
    return PreparedProjectionAdjoint(
        workspace, records, poses, candidate_rays, nodes, fallbacks, device_bytes,
        setup_nodes + pixels + voxels * min(pixels, max_rays_per_voxel), _gather_metadata(workspace))


def projection_adjoint_gather(pose, *, cotangent: torch.Tensor, workspace: ProjectionWorkspace,
                              out_mu: torch.Tensor | None = None,
                              volume_gradient_precision: Literal["float32", "float64"] = "float64",
                              accumulate: bool = False, validate: Literal["once", "always", "never"] | None = None,
                              max_work: int = 10_000_000) -> torch.Tensor:
    """``out_mu[v] = sum_p A(pose)[p, v] cotangent[p]``: the fixed-pose transpose of the strict
    FP64 projection (midpoint, or cell-Gauss with a raw pose), gathered per voxel in a fixed
    order (views ascending, each
    view's FP64 sum added to the running value; then rows, columns, samples ascending), so it
    is bitwise reproducible (reference python/dpt/projection.py:1250-1405).

    ``pose`` is a (views, 12) FP64 pose tensor or a ``PreparedProjectionAdjoint`` of this
    workspace; ``cotangent`` has the image's shape and dtype; ``out_mu`` (voxels, FP64 by
    default or FP32) is written, or added to with ``accumulate``, and returned.  A raw pose
    bounds its all-ray work voxels x rays x samples by ``max_work`` before writing; a
    prepared plan checks its retained bound."""
    spec = workspace.spec
    if spec.sampling_precision != "float64":
        raise ContractError("deterministic gather requires strict float64 sampling")
    if volume_gradient_precision not in ("float32", "float64"):
        raise ContractError("volume_gradient_precision must be float32 or float64")
    if type(accumulate) is not bool:
        raise ContractError("accumulate must be a boolean")
    integer(max_work, "max_work", minimum=1, maximum=2**63 - 1)
    plan = pose if isinstance(pose, PreparedProjectionAdjoint) else None
    if plan is not None and (plan.workspace is not workspace or plan.metadata != _gather_metadata(workspace)):
        raise ContractError("prepared adjoint belongs to its original workspace configuration")
    voxels, pixels = workspace.plan.grid.voxels, workspace.plan.rays
    nodes = 2 * (sum(workspace.plan.grid.shape) + 1) if spec.integration == "cell_gauss" else spec.samples_per_ray
    work = plan.work_bound if plan is not None else voxels * pixels * nodes
    if work > max_work:
        raise ContractError(f"deterministic gather needs at most {work} voxel/ray quadrature evaluations; "
                            f"max_work is {max_work}")
    flat = workspace._cotangent(cotangent)
    dtype = torch.float64 if volume_gradient_precision == "float64" else torch.float32
    if out_mu is None:
        if accumulate:
            raise ContractError("accumulate needs an out_mu to add to")
        out_mu = torch.empty(workspace.plan.grid.shape, dtype=dtype, device=workspace.device)
    if (not isinstance(out_mu, torch.Tensor) or out_mu.dtype != dtype or out_mu.device != workspace.device
            or out_mu.numel() != voxels or not out_mu.is_contiguous()):
        raise ContractError(f"out_mu must be a contiguous {dtype} tensor of {voxels} voxels on the workspace device")
    reads = [("cotangent", flat)]
    if plan is not None:
        reads.append(("prepared metrics", plan.records))
    for name, tensor in reads:
        a0, a1 = out_mu.data_ptr(), out_mu.data_ptr() + out_mu.numel() * out_mu.element_size()
        b0, b1 = tensor.data_ptr(), tensor.data_ptr() + tensor.numel() * tensor.element_size()
        if a0 < b1 and b0 < a1:
            raise ContractError(f"out_mu overlaps {name}")
    policy = spec.validate if validate is None else validate
    if policy not in ("once", "always", "never"):
        raise ContractError("validate must be once, always or never")
    if policy != "never" and not bool(torch.isfinite(flat).all()):
        raise NumericalError("projection: the cotangent must be finite")
    if plan is not None:
        records, poses = plan.records, plan.poses
    else:
        poses = workspace.check_poses(pose)
        nbytes = N.library().dpt_b200_gather_plan_bytes(_gather_problem(workspace), workspace.views)
        records = _write_gather_plan(workspace, poses, nbytes)
    lib = N.library()
    problem = _gather_problem(workspace)
    rays = workspace.rays(poses)
    code = N.F64 if dtype == torch.float64 else N.F32
    workspace._run("gather", lambda: lib.dpt_b200_gather(
        problem, rays, records.data_ptr(), flat.data_ptr(), out_mu.data_ptr(), code, int(accumulate),
        workspace.status.data_ptr(), _stream(workspace.device)))
    if policy != "never":
        workspace.consume_status("deterministic gather")
    return out_mu
