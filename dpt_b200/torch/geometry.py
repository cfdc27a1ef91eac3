"""``compose_pose(anchor, tangent) = anchor @ exp(tangent^)`` on packed Torch poses.

Same contract as the reference chart (hcltech-robotics/dpt
``python/dpt/torch/geometry.py:19-63``): ``anchor`` has trailing shape (12,) -
row-major rotation then translation in mm - and ``tangent`` trailing shape (6,) -
``(tx, ty, tz, rx, ry, rz)`` in mm and radians, acting on the right in object
axes.  Leading dimensions broadcast; both tensors are FP64 on one device.  The
SE(3) exponential is evaluated as the matrix exponential of the 4x4 twist, so
Torch differentiates it (including the translation/rotation coupling) and
carries packed-pose gradients back to the tangent and the anchor.
"""

from __future__ import annotations

import torch

from ..contracts import ContractError


def compose_pose(anchor: torch.Tensor, tangent: torch.Tensor) -> torch.Tensor:
    """Packed ``anchor @ exp(tangent^)``, shape ``broadcast(leading) + (12,)``."""
    if not isinstance(anchor, torch.Tensor) or not isinstance(tangent, torch.Tensor):
        raise ContractError("anchor and tangent must be Torch tensors")
    if anchor.dtype != torch.float64 or tangent.dtype != torch.float64:
        raise ContractError("rigid pose charts require float64 tensors")
    if anchor.device != tangent.device or anchor.device.type not in ("cpu", "cuda"):
        raise ContractError("anchor and tangent must share a CPU or CUDA device")
    if anchor.ndim < 1 or anchor.shape[-1] != 12 or tangent.ndim < 1 or tangent.shape[-1] != 6:
        raise ContractError("anchor and tangent require trailing shapes (12,) and (6,)")
    if anchor.numel() == 0 or tangent.numel() == 0:
        raise ContractError("pose charts require nonempty tensor dimensions")
    try:
        leading = torch.broadcast_shapes(anchor.shape[:-1], tangent.shape[:-1])
    except RuntimeError as error:
        raise ContractError("anchor and tangent leading dimensions do not broadcast") from error
    rho, omega = tangent[..., :3], tangent[..., 3:]
    wx, wy, wz = omega.unbind(-1)
    zero = torch.zeros_like(wx)
    # 4x4 twist [[w^, rho], [0, 0]]
    twist = torch.stack(
        (
            zero, -wz, wy, rho[..., 0],
            wz, zero, -wx, rho[..., 1],
            -wy, wx, zero, rho[..., 2],
            zero, zero, zero, zero,
        ),
        dim=-1,
    ).reshape(*tangent.shape[:-1], 4, 4)
    motion = torch.linalg.matrix_exp(twist)
    rotation = anchor[..., :9].reshape(*anchor.shape[:-1], 3, 3)
    composed = rotation @ motion[..., :3, :3]
    translation = (rotation @ motion[..., :3, 3:4]).squeeze(-1) + anchor[..., 9:]
    composed = composed.expand(*leading, 3, 3)
    translation = translation.expand(*leading, 3)
    return torch.cat((composed.reshape(*leading, 9), translation), dim=-1).contiguous()
