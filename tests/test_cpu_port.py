"""The threaded C restatement (timed CPU baseline) agrees with the NumPy oracle."""
import os

import numpy as np
import pytest

from oracle import model
from oracle.cpu_baseline import CpuOperator
from tests.conftest import GOLDEN, golden_dirs


@pytest.mark.parametrize('name', golden_dirs('atomistic'))
def test_c_port_matvec_matches_oracle(name):
    s = model.System.from_keywords(os.path.join(GOLDEN, name, 'input.kw'))
    op = model.Operator(s)
    cpu = CpuOperator(s, n_threads=3)
    rng = np.random.default_rng(3)
    x = rng.standard_normal(s.n_var) + 1j * rng.standard_normal(s.n_var)
    for i in sorted({0, len(s.freqs) - 1}):
        y = cpu.matvec(i, x)
        ref = op.matvec(i, x)
        assert np.linalg.norm(y - ref) <= 1e-12 * np.linalg.norm(ref)
