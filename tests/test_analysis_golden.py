"""The analysis step against the reference's own analysis tests: the oracle's
induced field |E|/E0 and density reproduce the cube files the reference wrote
(sampled every 5th grid point, at their E14.6 print), from the solutions and
geometry the reference stored.  The GPU kernel is held to the same files in
test_gpu_analysis.py."""
import json
import os

import numpy as np
import pytest

from oracle.analysis import field_and_density
from tests.conftest import GOLDEN

TO_BOHR = 1.8897261254578281
NAMES = ['analysis_field_3d_x_wfq_sodium', 'analysis_field_3d_x_y_z_wfqfmu_ag', 'analysis_density_3d_x_wfq_sodium']


def load_case(name):
    with open(os.path.join(GOLDEN, name, 'analysis.json')) as f:
        a = json.load(f)
    coords = np.array(a['coords_ang'])
    lo = coords.min(axis=0) - a['offset_ang']
    hi = coords.max(axis=0) + a['offset_ang']
    n = np.array(a['n'])
    step = (hi - lo) / (n - 1)
    idx = np.array(a['sample_index'])
    ijk = np.stack([idx // (n[1] * n[2]), (idx // n[2]) % n[1], idx % n[2]], axis=1)
    pts_bohr = (lo[None, :] + ijk * step[None, :]) * TO_BOHR
    x = np.array(a['x'])[:, 0] + 1j * np.array(a['x'])[:, 1]
    return a, coords * TO_BOHR, pts_bohr, x, lo, step


def quantity(a, E, rho):
    if a['quantity'] == 'field':
        return np.sqrt((np.abs(E) ** 2).sum(axis=1)) / a['e0']
    return rho.real


@pytest.mark.parametrize('name', NAMES)
def test_oracle_reproduces_reference_cube(name):
    a, coords, pts, x, lo, step = load_case(name)
    assert np.allclose(lo * TO_BOHR, a['cube_origin_bohr'], atol=5e-7)
    assert np.allclose(step * TO_BOHR, a['cube_step_bohr'], atol=5e-7)
    N = coords.shape[0]
    E, rho = field_and_density(coords, np.full(N, a['rq']), np.full(N, a['rmu']), x, a['e0'], a['pol'], pts,
                               a['model'] == 'wfqfmu')
    v = quantity(a, E, rho)
    ref = np.array(a['sample_value'])
    # E14.6: half a unit in the 6th digit, or the 1e-99 floor the writer prints as zero
    tol = 5.01e-6 * np.abs(ref) + 1e-30
    bad = np.abs(v - ref) > tol
    assert not bad.any(), (np.nonzero(bad)[0][:5], v[bad][:5], ref[bad][:5])
