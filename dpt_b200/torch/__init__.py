"""PyTorch adapter: the ``Projector`` module, the ``dpt::*`` operators and ``compose_pose``."""

from .geometry import compose_pose
from .modules import Projector

__all__ = ["Projector", "compose_pose"]
