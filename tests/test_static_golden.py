"""Static FQ / FQFMu against the reference's five static regression tests.

The oracle (oracle/static.py) reproduces every number the reference logs print
for fq_energy, fq_polarizability, fq_principal_axis_energy, fqfmu_energy and
fqfmu_rq_rmu_energy, at their printed precision: the static matrix and J^-1
(E11.4: half a unit of the 4th digit), the right-hand sides, charges and
dipoles (E14.6), the energy (F14.8), the polarizability tensor (E11.4) and its
isotropic value (F19.10), and the rotated geometry (F20.6, Angstrom).  The
host side of the library is checked here too: its keyword-file reader builds
the same problem, and its principal-axis rotation (plx_principal_axes, host
code of the C ABI) gives the log's rotated geometry.  The device solve is held
to the same numbers in test_gpu_static.py.
"""
import json
import os

import numpy as np
import pytest

from oracle import static as ost
from tests.conftest import GOLDEN, golden_dirs

CASES = golden_dirs('static')


def _load(name):
    with open(os.path.join(GOLDEN, name, 'expected.json')) as f:
        return json.load(f)


def e_tol(v, digits):
    """Half a unit of the last printed digit of an E-format value with `digits` digits."""
    v = abs(v)
    if v == 0.0:
        return 0.0
    return 0.5 * 10.0 ** (np.floor(np.log10(v)) + 1 - digits)


def check_printed_matrix(entries, M, digits, floor=1e-13):
    for key, v in entries.items():
        r, c = (int(t) - 1 for t in key.split(','))
        assert abs(M[r, c] - v) <= e_tol(v, digits) * 1.0001 + floor, (key, M[r, c], v)


def test_five_static_cases_present():
    assert CASES == ['fq_energy', 'fq_polarizability', 'fq_principal_axis_energy', 'fqfmu_energy',
                     'fqfmu_rq_rmu_energy']


@pytest.mark.parametrize('name', CASES)
def test_oracle_reproduces_reference_log(name):
    exp = _load(name)
    st, what, rotated = ost.static_from_keyword_file(os.path.join(GOLDEN, name, 'input.kw'))
    assert what == exp['what']
    out = st.solve(what)
    if 'matrix' in exp:
        check_printed_matrix(exp['matrix'], st.matrix(), 4)
    if 'rhs' in exp:
        rhs = np.array(exp['rhs'])
        assert rhs.shape == out['rhs'].shape
        for a, b in zip(out['rhs'].ravel(), rhs.ravel()):
            assert abs(a - b) <= e_tol(b, 6) * 1.0001 + 1e-300
    q = np.array(exp['charges'])
    assert q.shape == out['charges'].shape
    for a, b in zip(out['charges'].ravel(), q.ravel()):
        assert abs(a - b) <= e_tol(b, 6) * 1.0001 + 1e-300, (a, b)
    assert np.all(np.abs(np.array(exp['charge_err'])) < 1e-14)
    assert np.all(np.abs(out['charge_sum']) < 1e-13)
    if 'dipoles' in exp:
        mu = np.array(exp['dipoles'])
        for a, b in zip(out['dipoles'].ravel(), mu.ravel()):
            # components printed at ~1e-17 are rounding noise of an exact zero
            assert abs(a - b) <= e_tol(b, 6) * 1.0001 + 1e-15, (a, b)
    if 'energy' in exp:
        assert abs(out['energy'] - exp['energy']) <= 0.5e-8 * 1.0001
    if 'polar' in exp:
        check_printed_matrix(exp['polar'], out['polar'], 4, floor=1e-13)
        assert abs(out['polar_iso'] - exp['polar_iso']) <= 0.5e-10 * 1.0001
        check_printed_matrix(exp['j_inverse'], out['j_inverse'], 4)
        check_printed_matrix(exp['j_1_1'], out['j_1_1'], 4)
    if 'rotated' in exp:
        assert rotated is not None
        assert np.max(np.abs(rotated - np.array(exp['rotated']))) <= 0.5e-6 * 1.0001


@pytest.mark.parametrize('name', CASES)
def test_library_reader_builds_the_oracle_problem(name):
    """The product's keyword reader (and, for the principal-axis case, its host
    rotation through the C ABI) gives the oracle's problem."""
    from plasmonx_b200.static import StaticProblem
    path = os.path.join(GOLDEN, name, 'input.kw')
    p = StaticProblem.from_keyword_file(path)
    st, what, rotated = ost.static_from_keyword_file(path)
    assert (p.what, p.forcefield, p.kernel, p.n_var) == (what, st.ff, st.kernel, st.n_var)
    assert list(p.apm) == st.apm
    assert np.max(np.abs(p.coord - st.coord)) < 1e-12
    for a, b in ((p.chi, st.chi), (p.eta, st.eta), (p.alpha, st.alpha), (p.r_q, st.r_q), (p.r_mu, st.r_mu)):
        assert np.array_equal(a, b)
    if p.rotated:
        exp = _load(name)
        assert np.max(np.abs(p.coord / ost.TO_BOHR - np.array(exp['rotated']))) <= 0.5e-6 * 1.0001
        w = p.inertia['eigenvalues']
        assert np.all(np.diff(w) >= 0)


def test_host_rotation_matches_the_oracle_on_random_geometries():
    from plasmonx_b200.static import rotate_principal_axes
    rng = np.random.default_rng(5)
    for n in (2, 3, 17, 200):
        c = rng.standard_normal((n, 3)) * 4.0 + rng.standard_normal(3) * 10.0
        z = rng.choice([1, 6, 8, 47, 79], size=n)
        mine, w, V = rotate_principal_axes(c, z)
        ref, wr, Vr = ost.principal_axes(c, z)
        assert np.allclose(w, wr, rtol=1e-12, atol=1e-9)
        if np.min(np.diff(wr)) > 1e-6 * wr[-1]:
            # distinct eigenvalues: the axes are unique up to sign, fixed by the rule
            assert np.allclose(V, Vr, atol=1e-9)
            assert np.allclose(mine, ref, atol=1e-9)
        else:
            assert n == 2     # a linear molecule: a degenerate pair of axes
        # a rotation: distances are kept
        d0 = np.linalg.norm(c[:, None] - c[None], axis=-1)
        d1 = np.linalg.norm(mine[:, None] - mine[None], axis=-1)
        assert np.allclose(d0, d1, atol=1e-10)


def test_host_rotation_refuses_unknown_elements():
    from plasmonx_b200.static import rotate_principal_axes
    with pytest.raises(Exception, match='mass'):
        rotate_principal_axes(np.zeros((2, 3)) + [[0, 0, 0], [1, 0, 0]], [8, 0])


@pytest.mark.parametrize('imol,apm', [([1, 1, 1], [3]), ([1, 1, 2, 2, 2], [2, 3]), ([4, 4, 1, 1, 1, 7], [2, 3, 1]),
                                      ([1, 2, 3], [1, 1, 1])])
def test_molecule_sizes(imol, apm):
    from plasmonx_b200.static import atoms_per_molecule
    assert atoms_per_molecule(imol) == apm == ost.atoms_per_molecule(imol)


def test_constraint_rows_follow_the_reference_indexing():
    """add_lagrangian_blocks places molecule k at rows apm(k-1)(k-1)+1.. (1-based):
    right for molecules of equal size, shifted otherwise, refused past the atoms."""
    L = ost.lagrangian_rows(6, [3, 3])
    assert L[:, 0].tolist() == [1, 1, 1, 0, 0, 0] and L[:, 1].tolist() == [0, 0, 0, 1, 1, 1]
    L = ost.lagrangian_rows(7, [2, 5])
    assert L[:, 1].tolist() == [0, 0, 1, 1, 1, 1, 1]
    with pytest.raises(ValueError):
        ost.lagrangian_rows(7, [1, 3, 3])


def test_log_lines_in_reference_format():
    from plasmonx_b200.static import energy_line, polar_iso_line
    assert energy_line(-0.06107854876354285) == ' Energy =    -0.06107855 a.u.'
    assert polar_iso_line(12.252887542004643) == ' Polar Iso  =       12.2528875420 a.u.'
