"""Host contracts of the transmission and objective operators that need no GPU: spec
validation (reference python/dpt/transmission.py:68-81, python/dpt/objectives.py:36-62),
CPU devices rejected, and the C ABI's argument checks, which return before any launch."""

from __future__ import annotations

import pytest

from dpt_b200 import _native as N
from dpt_b200.contracts import ContractError
from dpt_b200.objectives import ObjectiveSpec, prepare_objective
from dpt_b200.transmission import TransmissionError, TransmissionOutputs, TransmissionSpec, prepare_transmission


def test_transmission_spec_contracts():
    TransmissionSpec(beam="per-pixel", active_beam=True)
    with pytest.raises(TransmissionError, match="unsupported beam"):
        TransmissionSpec(beam="sometimes")
    with pytest.raises(TransmissionError, match="CUDA array"):
        TransmissionSpec(beam="scalar", active_beam=True)
    with pytest.raises(TransmissionError, match="at least one"):
        TransmissionOutputs()
    with pytest.raises(TransmissionError, match="CUDA devices"):
        prepare_transmission(max_pixels=4, device="cpu")
    with pytest.raises(TransmissionError):
        prepare_transmission(max_pixels=-1)
    with pytest.raises(TransmissionError, match="TransmissionSpec"):
        prepare_transmission("scalar", max_pixels=1)


def test_objective_spec_contracts():
    ObjectiveSpec(kind="poisson", domain="counts", weighted=True, masked=True, precision="float64")
    for kwargs, message in (
        ({"kind": "huber"}, "unsupported"),
        ({"precision": "float16"}, "precision"),
        ({"domain": "photons"}, "domain"),
        ({"kind": "poisson", "domain": "signal"}, "count-domain"),
        ({"integer_counts": 1}, "boolean"),
        ({"reduction": "max"}, "reduction"),
    ):
        with pytest.raises(ContractError, match=message):
            ObjectiveSpec(**kwargs)
    with pytest.raises(ContractError, match="CUDA devices"):
        prepare_objective(ObjectiveSpec(), max_pixels=4, device="cpu")


def test_c_abi_rejects_bad_arguments_before_launching():
    lib = N.library()
    assert lib.dpt_b200_reduction_bytes(0) == 8
    assert lib.dpt_b200_reduction_bytes(256) == 16
    assert lib.dpt_b200_reduction_bytes(257) == (2 + 1 + 1) * 8
    assert lib.dpt_b200_reduction_bytes(-1) == 0
    fake = 16  # never dereferenced: every call below fails its argument checks
    assert lib.dpt_b200_transmit(fake, 4, 0, 0, None, 0.0, fake, None, None, None, None) == N_E("FLAGS")
    assert lib.dpt_b200_transmit(fake, 4, 2, 0, None, 0.0, None, fake, None, None, None) == N_E("FLAGS")
    assert lib.dpt_b200_transmit(fake, 4, 1, 0, None, 0.0, None, None, None, None, None) == N_E("NULL")
    assert lib.dpt_b200_transmit(fake, -1, 1, 0, None, 0.0, fake, None, None, None, None) == N_E("SHAPE")
    assert lib.dpt_b200_transmit(fake, 0, 1, 0, None, 0.0, fake, None, None, None, None) == 0
    assert lib.dpt_b200_transmit_vjp(fake, 4, 1, None, 0.0, fake, None, None, None, None, fake, None, 0, fake,
                                     None) == N_E("FLAGS")  # a pointwise beam gradient needs a beam array
    assert lib.dpt_b200_transmit_vjp(fake, 4, 2, fake, 0.0, None, fake, None, None, None, fake, None, 0, fake,
                                     None) == N_E("NULL")  # a shared beam gradient needs scratch
    assert lib.dpt_b200_check_values(fake, 4, 7, fake, None) == N_E("FLAGS")
    assert lib.dpt_b200_objective(fake, N.F32, 0, fake, None, None, 4, 2, 1.0, 1.0, fake, fake, fake, fake,
                                  None) == N_E("FLAGS")
    assert lib.dpt_b200_objective(fake, N.F64, 0, fake, None, None, 4, 0, 1.0, 1.0, fake, fake, fake, fake,
                                  None) == N_E("DTYPE")
    assert lib.dpt_b200_objective(fake, N.F32, 0, fake, None, None, 4, 0, 1.0, 1.0, None, None, None, fake,
                                  None) == N_E("FLAGS")
    assert lib.dpt_b200_objective_check(fake, 2, fake, None, None, 4, 0, 1, fake, None) == N_E("DTYPE")
    assert lib.dpt_b200_reduce_sum(fake, 4, None, fake, fake, None) == N_E("NULL")


def N_E(name: str) -> int:
    return {"NULL": -1, "SHAPE": -2, "DTYPE": -3, "FLAGS": -4}[name]
