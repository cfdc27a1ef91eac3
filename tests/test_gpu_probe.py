"""The read-bandwidth probe behind the benchmark's L2 roofline reads every byte it is given:
a NaN anywhere in the buffer (first or last 16 bytes, or the middle) reaches the sink, and
a finite buffer leaves the sink untouched."""

from __future__ import annotations

import math

import pytest
import torch

from dpt_b200 import _native as N

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("position", ["first", "middle", "last", "none"])
def test_probe_reads_the_whole_buffer(position):
    lib = N.library()
    quads = (1 << 20) + 3  # not a multiple of the grid's stride
    buffer = torch.ones(4 * quads, dtype=torch.float32, device="cuda:0")
    index = {"first": 0, "middle": 2 * quads + 1, "last": 4 * quads - 1, "none": None}[position]
    if index is not None:
        buffer[index] = math.nan
    sink = torch.zeros(1, dtype=torch.float32, device="cuda:0")
    stream = torch.cuda.current_stream().cuda_stream
    assert lib.dpt_b200_read_probe(buffer.data_ptr(), 16 * quads, 2, sink.data_ptr(), stream) == 0
    value = float(sink.item())
    assert math.isnan(value) == (index is not None)
    if index is None:
        assert value == 0.0
