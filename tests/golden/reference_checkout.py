"""Locate the reference project (hcltech-robotics/dpt) for the fixture generators.

The generators import the reference's host code (which runs without Warp) to compute
golden values.  The checkout is given by ``--reference PATH`` on the command line or by
the ``DPT_REFERENCE`` environment variable; nothing else is assumed about where it lives.
"""

from __future__ import annotations

import os
import sys
from pathlib import Path


def reference_root(argv: list[str] | None = None) -> Path:
    """Return the reference checkout and put its ``python/`` and root on ``sys.path``."""
    argv = sys.argv[1:] if argv is None else argv
    path = None
    for k, arg in enumerate(argv):
        if arg == "--reference" and k + 1 < len(argv):
            path = argv[k + 1]
        elif arg.startswith("--reference="):
            path = arg.split("=", 1)[1]
    if path is None:
        path = os.environ.get("DPT_REFERENCE")
    if not path:
        raise SystemExit("give the reference checkout: --reference PATH or DPT_REFERENCE=PATH")
    root = Path(path).resolve()
    if not (root / "python" / "dpt").is_dir():
        raise SystemExit(f"{root} does not look like a dpt checkout (no python/dpt)")
    for entry in (str(root / "python"), str(root)):
        if entry not in sys.path:
            sys.path.insert(0, entry)
    return root
