"""dpt_b200 - B200-native differentiable CT projector.

Optical depth of an attenuation volume along finite cone-beam (or parallel /
curved-panel) rays, its volume VJP and its per-view rigid-pose VJP, computed by
hand-written CUDA kernels for sm_100a behind a C ABI (``include/dpt_b200.h``).
The Python surface mirrors the reference projector (hcltech-robotics/dpt):
``project``, ``dpt_b200.torch.Projector``, the ``dpt::project*`` Torch
operators and the geometry objects.
"""

from .api import project
from .contracts import ContractError, NumericalError, TrialDomainError
from .geometry import (
    BatchedGeometry,
    ConeBeamIntrinsics,
    CurvedDetectorGeometry,
    DetectorGeometry,
    ParallelGeometry,
    RayBundleGeometry,
    RigidTransform,
    chart_gradient,
    compose_pose,
    right_jacobian_se3,
)
from .imaging import ImagingMetadata, ImagingVolume, ct_to_attenuation, standard_views
from .volumes import GridSpec

__all__ = [
    "BatchedGeometry",
    "ConeBeamIntrinsics",
    "ContractError",
    "CurvedDetectorGeometry",
    "DetectorGeometry",
    "GridSpec",
    "ImagingMetadata",
    "ImagingVolume",
    "NumericalError",
    "ParallelGeometry",
    "RayBundleGeometry",
    "RigidTransform",
    "TrialDomainError",
    "chart_gradient",
    "compose_pose",
    "ct_to_attenuation",
    "project",
    "right_jacobian_se3",
    "standard_views",
]
