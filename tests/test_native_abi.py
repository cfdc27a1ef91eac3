"""The C ABI: exported symbols, constants and struct layout match include/dpt_b200.h,
and host-side argument checks reject bad calls before anything is launched.
No test here launches a kernel, so the suite runs without a GPU."""

from __future__ import annotations

import ctypes
import re
import subprocess
from pathlib import Path

import pytest

from dpt_b200 import _native as N
from oracle import oracle as O

ROOT = Path(__file__).resolve().parents[1]
HEADER = (ROOT / "include" / "dpt_b200.h").read_text()


def declared_functions() -> set[str]:
    return set(re.findall(r"^\s*(?:int|size_t|const char\*)\s+(dpt_b200_\w+)\(", HEADER, re.M))


def header_constants() -> dict[str, int]:
    values = {name: int(value) for name, value in re.findall(r"\b(DPT_\w+)\s*=\s*(-?\d+)", HEADER)}
    values.update({name: int(value) for name, value in re.findall(r"#define\s+(DPT_\w+)\s+(\d+)", HEADER)})
    return values


def test_library_exports_every_declared_entry_point():
    lib = N.library()
    declared = declared_functions()
    assert declared == set(N.EXPORTS)
    for name in declared:
        assert hasattr(lib, name), name
    assert lib.dpt_b200_abi_version() == N.ABI_VERSION == header_constants()["DPT_B200_ABI_VERSION"]


def test_constants_match_header():
    c = header_constants()
    pairs = {
        "DPT_F32": N.F32, "DPT_F64": N.F64, "DPT_F16": N.F16, "DPT_BF16": N.BF16,
        "DPT_ARITH_F32": N.ARITH_F32, "DPT_ARITH_F64": N.ARITH_F64, "DPT_ARITH_F32C": N.ARITH_F32C,
        "DPT_RAYS_PANELS": N.RAYS_PANELS, "DPT_RAYS_BUNDLE": N.RAYS_BUNDLE,
        "DPT_PANEL_CONE": N.PANEL_CONE, "DPT_PANEL_PARALLEL": N.PANEL_PARALLEL,
        "DPT_PANEL_CURVED": N.PANEL_CURVED, "DPT_VIEW_WORDS": N.VIEW_WORDS,
        "DPT_VIEW_MODE_WORD": N.VIEW_MODE_WORD, "DPT_LAYOUT_REPLICATED": N.LAYOUT_REPLICATED,
        "DPT_LAYOUT_DIRECT": N.LAYOUT_DIRECT, "DPT_VJP_VOLUME": N.VJP_VOLUME,
        "DPT_VJP_POSE12": N.VJP_POSE12, "DPT_VJP_POSE6": N.VJP_POSE6, "DPT_VJP_PER_RAY6": N.VJP_PER_RAY6,
    }
    for name, value in pairs.items():
        assert c[name] == value, name
    assert (O.F32, O.F64, O.F16, O.BF16) == (N.F32, N.F64, N.F16, N.BF16)
    assert (O.VJP_VOLUME, O.VJP_POSE12, O.VJP_POSE6, O.VJP_PER_RAY6) == (1, 2, 4, 8)


def test_struct_layout_matches_c_compiler(tmp_path):
    program = tmp_path / "layout.c"
    program.write_text(
        '#include <stdio.h>\n#include <stddef.h>\n#include "dpt_b200.h"\n'
        "int main(void) {\n"
        ' printf("%zu %zu %zu %zu\\n", sizeof(dpt_problem), offsetof(dpt_problem, layout),'
        " offsetof(dpt_problem, object_to_grid), offsetof(dpt_problem, grid_origin));\n"
        ' printf("%zu %zu %zu\\n", sizeof(dpt_rays), offsetof(dpt_rays, view_begin),'
        " offsetof(dpt_rays, view_count));\n"
        " return 0; }\n"
    )
    binary = tmp_path / "layout"
    subprocess.run(["gcc", "-I", str(ROOT / "include"), str(program), "-o", str(binary)], check=True)
    lines = subprocess.run([str(binary)], check=True, capture_output=True, text=True).stdout.split("\n")
    problem = [int(x) for x in lines[0].split()]
    rays = [int(x) for x in lines[1].split()]
    assert problem == [ctypes.sizeof(N.Problem), N.Problem.layout.offset, N.Problem.object_to_grid.offset,
                       N.Problem.grid_origin.offset]
    assert rays == [ctypes.sizeof(N.Rays), N.Rays.view_begin.offset, N.Rays.view_count.offset]
    assert ctypes.sizeof(O._Problem) == ctypes.sizeof(N.Problem)


def problem(**overrides) -> N.Problem:
    p = N.Problem()
    p.nx, p.ny, p.nz = 8, 9, 10
    p.views, p.rows, p.cols, p.samples = 3, 4, 5, 16
    for key, value in overrides.items():
        setattr(p, key, value)
    return p


def test_scratch_sizes():
    lib = N.library()
    p = problem()
    assert lib.dpt_b200_packed_bytes(p) == 8 * 9 * 10 * 16
    assert lib.dpt_b200_accumulator_bytes(p) == 8 * 9 * 10 * 32
    tiles = 1  # 4x5 detector fits one 16x16 tile
    assert lib.dpt_b200_pose_partials_bytes(p, 3) == 3 * tiles * 12 * 8
    assert lib.dpt_b200_packed_bytes(problem(layout=N.LAYOUT_DIRECT)) == 0
    assert lib.dpt_b200_packed_bytes(problem(nx=0)) == 0


@pytest.mark.parametrize(
    "overrides, code",
    [
        ({"nx": 0}, -2),
        ({"samples": 0}, -2),
        ({"field_dtype": N.BF16}, -3),  # half storage needs compensated arithmetic
        ({"arith": 7}, -3),
        ({"image_dtype": N.F16}, -3),
        ({"ray_kind": 5}, -4),
        ({"layout": N.LAYOUT_DIRECT, "field_dtype": N.F16, "arith": N.ARITH_F32C}, -3),
        ({"nx": 1 << 25, "ny": 1, "nz": 1}, -2),  # FP32 grid coordinates exact to 2^24 only
    ],
)
def test_argument_checks_return_codes_without_launching(overrides, code):
    lib = N.library()
    p = problem(**overrides)
    rays = N.Rays()
    rays.poses = 8
    rays.view_table = 8
    rays.view_count = 1
    assert lib.dpt_b200_forward(p, rays, 16, 16, 16, None) == code


def test_null_pointers_and_view_ranges_are_rejected():
    lib = N.library()
    p = problem()
    rays = N.Rays()
    rays.view_count = 1
    assert lib.dpt_b200_forward(p, rays, 16, 16, 16, None) == -1  # null poses
    rays.poses = 16
    assert lib.dpt_b200_forward(p, rays, 16, 16, 16, None) == -1  # null panel table
    rays.view_table = 16
    rays.view_begin, rays.view_count = 2, 2
    assert lib.dpt_b200_forward(p, rays, 16, 16, 16, None) == -5
    rays.view_begin, rays.view_count = 0, 3
    assert lib.dpt_b200_forward(p, rays, 24, 16, 16, None) == -6  # packed not 16-byte aligned
    assert lib.dpt_b200_vjp(p, rays, 16, 16, 0, None, None, 16, None) == -4  # no gradient requested
    assert lib.dpt_b200_vjp(p, rays, 16, 16, N.VJP_POSE12 | N.VJP_POSE6, None, 16, 16, None) == -4
    assert lib.dpt_b200_vjp(p, rays, 16, 16, N.VJP_VOLUME | N.VJP_PER_RAY6, 32, 16, 16, None) == -4
    assert lib.dpt_b200_vjp(p, rays, 16, 16, N.VJP_VOLUME, None, None, 16, None) == -1
    assert lib.dpt_b200_vjp(p, rays, 16, 16, N.VJP_VOLUME, 16, None, 16, None) == -6  # accumulator alignment
    assert lib.dpt_b200_finish_pose(p, 0, 3, 7, 16, 16, 0, 16, None) == -4
    assert lib.dpt_b200_finish_pose(p, 2, 3, 12, 16, 16, 0, 16, None) == -5
    assert lib.dpt_b200_fold_volume(p, 32, None, 0, None, N.F32, 1, 16, None) == -1
    assert lib.dpt_b200_error_string(-5) == b"view range outside the problem"


def test_read_probe_rejects_bad_buffers_without_launching():
    lib = N.library()
    assert lib.dpt_b200_read_probe(None, 16, 1, 16, None) == -1
    assert lib.dpt_b200_read_probe(16, 16, 1, None, None) == -1
    assert lib.dpt_b200_read_probe(16, 24, 1, 16, None) == -2  # not a multiple of 16 bytes
    assert lib.dpt_b200_read_probe(16, 0, 1, 16, None) == -2
    assert lib.dpt_b200_read_probe(16, 16, 0, 16, None) == -2
    assert lib.dpt_b200_read_probe(24, 16, 1, 16, None) == -6  # buffer not 16-byte aligned


def test_packed_forward_checks_every_descriptor_without_launching():
    lib = N.library()
    count = 2
    problems = (N.Problem * count)(problem(), problem())
    rays = (N.Rays * count)()
    for r in rays:
        r.poses, r.view_table, r.view_count = 16, 16, 1
    ptrs = lambda *v: (ctypes.c_void_p * count)(*v)  # noqa: E731
    good = ptrs(16, 16)
    assert lib.dpt_b200_forward_packed(0, problems, rays, good, good, good, None) == -2
    assert lib.dpt_b200_forward_packed(N.MAX_PACK + 1, problems, rays, good, good, good, None) == -7
    assert lib.dpt_b200_forward_packed(count, None, rays, good, good, good, None) == -1
    assert lib.dpt_b200_forward_packed(count, problems, rays, ptrs(16, None), good, good, None) == -1
    assert lib.dpt_b200_forward_packed(count, problems, rays, ptrs(16, 24), good, good, None) == -6
    rays[1].view_begin = 3  # view 3 of a three-view problem
    assert lib.dpt_b200_forward_packed(count, problems, rays, good, good, good, None) == -5
    rays[1].view_begin = 0
    problems[1] = problem(arith=N.ARITH_F64, image_dtype=N.F64)  # a second kernel instantiation
    assert lib.dpt_b200_forward_packed(count, problems, rays, good, good, good, None) == -4
    problems[1] = problem(samples=0)
    assert lib.dpt_b200_forward_packed(count, problems, rays, good, good, good, None) == -2
