"""The benchmark's synthetic operands equal the reference's appendFill
construction (checked with the oracle's restatement of appendFill)."""
import numpy as np
import pytest

import oracle
from oracle import wahgen as G
from libfastlib_b200 import workloads as W


def test_runs_identical_to_fixture_generator():
    for seed, d in ((1, 1e-3), (2, 0.5)):
        assert np.array_equal(W.geometric_runs(seed, 1 << 18, d), G.geometric_runs(seed, 1 << 18, d))


@pytest.mark.parametrize("density", [1e-4, 1e-3, 1e-2, 0.1, 0.5])
def test_operand_equals_appendfill(density):
    for seed in (3, 4):
        for nbits in (1 << 18, (1 << 18) + 17):
            runs = W.geometric_runs(seed, nbits, density)
            assert np.array_equal(W.raw_wah_operand(seed, nbits, density), oracle.build_runs(runs))
