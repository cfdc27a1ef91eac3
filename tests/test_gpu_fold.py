"""The fold of the corner-replicated FP32 accumulator into the FP64 volume gradient
(dpt_b200_fold_volume: the widening the reference applies every few views,
python/dpt/torch/_projection_ops.py:304-352) is bit-exact against a Python restatement
that sums each voxel's corner slots in FP64 in the fixed order (z source, then y, then x;
the cell's own corner before the one below), on shapes with one-cell axes, ragged tiles and
the edges of every axis, with and without a running FP64 total."""

from __future__ import annotations

import numpy as np
import pytest
import torch

from dpt_b200 import _native as N

pytestmark = pytest.mark.gpu

SHAPES = [(1, 1, 1), (1, 5, 7), (4, 1, 9), (1, 3, 40), (16, 8, 31), (17, 9, 32), (33, 17, 65), (5, 24, 62)]


def sources(v: int, n: int) -> list[tuple[int, int]]:
    """(cell, corner bit) pairs along one axis whose corner lands on coordinate v."""
    if n == 1:
        return [(0, 0), (0, 1)]
    out = []
    if v <= n - 2:
        out.append((v, 0))
    if v >= 1:
        out.append((v - 1, 1))
    return out


def fold_reference(acc: np.ndarray) -> np.ndarray:
    nz, ny, nx, _ = acc.shape
    out = np.zeros((nz, ny, nx), dtype=np.float64)
    for z in range(nz):
        for y in range(ny):
            for x in range(nx):
                total = 0.0
                for cz, bz in sources(z, nz):
                    for cy, by in sources(y, ny):
                        for cx, bx in sources(x, nx):
                            total += float(acc[cz, cy, cx, bx | (by << 1) | (bz << 2)])
                out[z, y, x] = total
    return out


def accumulator(shape, seed: int) -> np.ndarray:
    """Random slots with the invariant of the scatter kernels: a cell at index n - 1 of an
    axis with n >= 2 is never a lower cell, so its record stays zero."""
    nz, ny, nx = shape
    rng = np.random.default_rng(seed)
    acc = rng.standard_normal((nz, ny, nx, 8)).astype(np.float32) * np.float32(1e-3)
    acc *= np.float32(10.0) ** rng.integers(-6, 6, size=acc.shape).astype(np.float32)
    if nx >= 2:
        acc[:, :, nx - 1, :] = 0
    if ny >= 2:
        acc[:, ny - 1, :, :] = 0
    if nz >= 2:
        acc[nz - 1, :, :, :] = 0
    return acc


def problem(shape) -> N.Problem:
    p = N.Problem()
    p.nz, p.ny, p.nx = shape
    p.views, p.rows, p.cols, p.samples = 1, 1, 1, 1
    return p


@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("gradient_dtype", [torch.float32, torch.float64])
def test_fold_matches_fixed_order_sum(shape, gradient_dtype):
    lib = N.library()
    device = torch.device("cuda:0")
    acc_host = accumulator(shape, seed=sum(shape))
    expected = fold_reference(acc_host)
    acc = torch.tensor(acc_host, device=device).contiguous()
    prior = torch.tensor(np.random.default_rng(7).standard_normal(shape), device=device)
    total = prior.clone()
    gradient = torch.empty(shape, dtype=gradient_dtype, device=device)
    status = torch.zeros(1, dtype=torch.int32, device=device)
    stream = torch.cuda.current_stream().cuda_stream
    code = N.F64 if gradient_dtype == torch.float64 else N.F32
    assert lib.dpt_b200_fold_volume(problem(shape), acc.data_ptr(), total.data_ptr(), 1, gradient.data_ptr(),
                                    code, 1, status.data_ptr(), stream) == 0
    want_total = expected + prior.cpu().numpy()
    assert np.array_equal(total.cpu().numpy(), want_total)
    assert np.array_equal(gradient.cpu().numpy(), want_total.astype(gradient.cpu().numpy().dtype))
    assert int(status.item()) == 0
    assert not bool(acc.any())  # cleared for the next batch

    # first batch of a total, no gradient yet: total = fold
    acc.copy_(torch.tensor(acc_host, device=device))
    assert lib.dpt_b200_fold_volume(problem(shape), acc.data_ptr(), total.data_ptr(), 0, None, N.F32, 0,
                                    status.data_ptr(), stream) == 0
    assert np.array_equal(total.cpu().numpy(), expected)
    assert np.array_equal(acc.cpu().numpy(), acc_host)  # clear = 0 keeps the accumulator


def test_fold_reports_non_finite_gradient():
    lib = N.library()
    device = torch.device("cuda:0")
    shape = (3, 4, 5)
    acc = torch.zeros(shape + (8,), dtype=torch.float32, device=device)
    acc[1, 2, 3, 0] = float("inf")
    gradient = torch.empty(shape, dtype=torch.float32, device=device)
    status = torch.zeros(1, dtype=torch.int32, device=device)
    stream = torch.cuda.current_stream().cuda_stream
    assert lib.dpt_b200_fold_volume(problem(shape), acc.data_ptr(), None, 0, gradient.data_ptr(), N.F32, 1,
                                    status.data_ptr(), stream) == 0
    assert int(status.item()) & 2
