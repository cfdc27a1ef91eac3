"""Generate ``config1.npz``: the reference's independent FP64 midpoint values on the small
plain workload (64^3 at 1 mm, seeded ellipsoid phantom, 8 cone views over 360 deg,
SOD 500 / SDD 1000, 64x64 detector at 1.5 mm, 128 midpoint samples per ray).

    python tests/golden/make_config1_golden.py --reference PATH

Values computed with the reference's scalar integrator
``python/dpt/validation/projection.py`` ``integrate_sampled_field`` (FP64 clip and
midpoints, ``math.fsum`` over the samples), on the reference's own ``GridSpec`` and
``DetectorGeometry`` objects built from this package's scene description:

* ``image``: the optical depth of all 8 x 64 x 64 rays;
* ``vjp_voxels`` / ``vjp_values``: the volume cotangent of the mean over the central
  32 x 32 detector pixels of every view, at seeded voxels inside the region the central
  rays cross: column ``v`` of the operator is the integral of the basis field ``e_v``, so
  ``(A^T m)[v] = sum_p m_p integral_p(e_v)``.

The field itself is this package's seeded phantom; its SHA-256 is stored so a test can tell
when the phantom generator no longer produces the values the fixture was made from.
"""

from __future__ import annotations

import hashlib
import multiprocessing
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))
sys.path.insert(0, str(HERE.parent))
sys.path.insert(0, str(HERE.parent.parent))

from reference_checkout import reference_root  # noqa: E402

REFERENCE = reference_root()

from dpt import geometry as rg  # noqa: E402
from dpt.validation import projection as rv  # noqa: E402
from dpt.volumes import GridSpec as ReferenceGrid  # noqa: E402
from scenes import config1_scene  # noqa: E402

SAMPLES = 128
CENTRAL = 32
VJP_VOXELS = 8


def _reference_objects():
    grid, geometry, values = config1_scene()
    ref_grid = ReferenceGrid(grid.shape, grid.spacing_mm, grid.origin_mm, grid.orientation)
    panels = [rg.DetectorGeometry(p.source_mm, p.origin_mm, p.u, p.v, p.spacing_mm, p.shape)
              for p in geometry.views]
    return ref_grid, panels, values


def _image_rows(task):
    view, row = task
    grid, panels, values = _reference_objects()
    flat = values.reshape(-1).astype(np.float64).tolist()
    return [rv.integrate_sampled_field(flat, grid, panels[view], rg.RigidTransform(), row, column,
                                       midpoint_samples=SAMPLES, validate=False)
            for column in range(panels[view].shape[1])]


def _column(voxel):
    grid, panels, _ = _reference_objects()
    basis = [0.0] * grid.voxels
    basis[voxel] = 1.0
    rows, cols = panels[0].shape
    r0, c0 = (rows - CENTRAL) // 2, (cols - CENTRAL) // 2
    weight = 1.0 / (len(panels) * CENTRAL * CENTRAL)
    terms = []
    for panel in panels:
        for row in range(r0, r0 + CENTRAL):
            for column in range(c0, c0 + CENTRAL):
                terms.append(weight * rv.integrate_sampled_field(
                    basis, grid, panel, rg.RigidTransform(), row, column,
                    midpoint_samples=SAMPLES, validate=False))
    import math
    return math.fsum(terms)


def main() -> None:
    grid, panels, values = _reference_objects()
    views = len(panels)
    rows, cols = panels[0].shape
    context = multiprocessing.get_context("spawn")
    with context.Pool() as pool:
        image = np.asarray(pool.map(_image_rows, [(v, r) for v in range(views) for r in range(rows)]),
                           dtype=np.float64).reshape(views, rows, cols)
        # voxels near the centre, where every view's central rays pass
        rng = np.random.default_rng(11)
        nz, ny, nx = grid.shape
        picks = []
        while len(picks) < VJP_VOXELS:
            x, y, z = (int(rng.integers(n // 2 - 8, n // 2 + 8)) for n in (nx, ny, nz))
            voxel = (z * ny + y) * nx + x
            if voxel not in picks:
                picks.append(voxel)
        columns = np.asarray(pool.map(_column, picks), dtype=np.float64)
    digest = hashlib.sha256(np.ascontiguousarray(values, dtype=np.float32).tobytes()).hexdigest()
    np.savez_compressed(HERE / "config1.npz", image=image, vjp_voxels=np.asarray(picks, dtype=np.int64),
                        vjp_values=columns, samples=np.int64(SAMPLES), central=np.int64(CENTRAL),
                        field_sha256=np.bytes_(digest))
    print(f"config1.npz: image {image.shape}, {len(picks)} VJP voxels, field sha256 {digest[:16]}")


if __name__ == "__main__":
    main()
