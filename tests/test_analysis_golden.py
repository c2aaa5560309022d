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


# ---- the product's grid, cube and maximum formatting (plasmonx_b200/analysis.py) ----

def _grid(a):
    from plasmonx_b200 import analysis as A
    return A.cubic_grid(np.array(a['coords_ang']), tuple(a['n']), a['offset_ang'])


ALL = NAMES + ['analysis_field_3d_y_bem']


@pytest.mark.parametrize('name', ALL)
def test_grid_block_matches_reference_log(name):
    with open(os.path.join(GOLDEN, name, 'analysis.json')) as f:
        a = json.load(f)
    mine = _grid(a).info_text().splitlines()
    assert [l.rstrip() for l in mine] == [l.rstrip() for l in a['log_grid']]


@pytest.mark.parametrize('name', ALL)
def test_cube_header_matches_reference(name):
    """Origin, steps and atoms of the cube header: the same numbers as printed (the
    reference's archived cubes come from a release that wrote the counts as i5; the
    current writer, plot_module.f90:512, uses i8)."""
    from plasmonx_b200 import analysis as A
    with open(os.path.join(GOLDEN, name, 'analysis.json')) as f:
        a = json.load(f)
    g = _grid(a)
    text = A.cube_text(g, np.zeros(tuple(a['n'])), a['z'], np.array(a['coords_ang']))
    head = text.splitlines()[2:6 + len(a['z'])]
    assert [l.split() for l in head] == [l.split() for l in a['cube_head']]
    atom_lines = head[4:]
    assert all(m == r for m, r in zip(atom_lines, a['cube_head'][4:]))     # (i5,1x,f10.6,3f12.6) unchanged


@pytest.mark.parametrize('name', NAMES)
def test_maximum_lines_match_reference_log(name):
    """The oracle's full grid, through the product's grid order and maximum search,
    gives the maximum the reference's analysis log printed (value at E13.6; the
    location is the reference's or a symmetric point whose value ties within 1e-12)."""
    from plasmonx_b200 import analysis as A
    a, coords, _, x, _, _ = load_case(name)
    g = _grid(a)
    pts = g.points_ang() * TO_BOHR
    N = coords.shape[0]
    E, rho = field_and_density(coords, np.full(N, a['rq']), np.full(N, a['rmu']), x, a['e0'], a['pol'], pts,
                               a['model'] == 'wfqfmu')
    nx, ny, nz = a['n']
    shape = lambda v: v.reshape(nz, ny, nx).transpose(2, 1, 0)  # noqa: E731
    pol = 'E' + 'xyz'[a['pol']]
    if a['quantity'] == 'field':
        blocks = [('Field', shape(np.sqrt((np.abs(E) ** 2).sum(axis=1)) / a['e0']))]
    else:
        blocks = [('RhoRe', shape(rho.real)), ('RhoIm', shape(rho.imag))]
    ref = a['log_max']
    for b, (kind, vals) in enumerate(blocks):
        lines = A.maximum_lines(kind, pol, g, vals).splitlines()
        assert lines[0] == ref[2 * b]
        mine, theirs = lines[1].split(), ref[2 * b + 1].split()
        assert mine[0] == theirs[0] and mine[4] == theirs[4]
        if mine[1:4] != theirs[1:4]:
            at = np.array([float(v) for v in theirs[1:4]])
            ijk = np.rint((at - g.lo) / g.step).astype(int)
            m, _ = A.maximum(g, vals)
            assert abs(vals[tuple(ijk)] - m) <= 1e-12 * abs(m)


def _bem_case():
    with open(os.path.join(GOLDEN, 'analysis_field_3d_y_bem', 'analysis.json')) as f:
        a = json.load(f)
    centres = np.array(a['coords_ang']) * TO_BOHR
    q = np.array(a['x'])[:, 0] + 1j * np.array(a['x'])[:, 1]
    return a, centres, q


def test_oracle_reproduces_reference_bem_cube_and_maximum():
    """BEM field |E|/E0 (point charges at the tessera centres, zero inside the
    surface) against the reference's BEM analysis test: the sampled cube values at
    E14.6 and the maximum line of its log."""
    from oracle.analysis import bem_field
    from plasmonx_b200 import analysis as A
    a, centres, q = _bem_case()
    g = _grid(a)
    pts = g.points_ang() * TO_BOHR
    E = bem_field(centres, q, a['e0'], a['pol'], pts)
    v = np.sqrt((np.abs(E) ** 2).sum(axis=1)) / a['e0']
    nx, ny, nz = a['n']
    vals = v.reshape(nz, ny, nx).transpose(2, 1, 0)
    flat = vals.ravel()                 # cube order: x outer, z fastest
    idx = np.array(a['sample_index'])
    ref = np.array(a['sample_value'])
    assert np.all(np.abs(flat[idx] - ref) <= 5.01e-6 * np.abs(ref) + 1e-30)
    assert np.mean(ref == 0.0) > 0.01           # the inside of the surface is zero
    lines = A.maximum_lines('Field', 'Ey', g, vals).splitlines()
    assert lines == a['log_max']
