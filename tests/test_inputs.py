"""Host-side input handling agrees with the oracle's independent reading of the same keyword files."""
import os

import numpy as np
import pytest

from oracle import model
from plasmonx_b200.inputs import Problem
from tests.conftest import GOLDEN, golden_dirs


@pytest.mark.parametrize('name', golden_dirs('atomistic'))
def test_problem_matches_oracle_system(name):
    path = os.path.join(GOLDEN, name, 'input.kw')
    p = Problem.from_keyword_file(path)
    s = model.System.from_keywords(path)
    assert p.model == s.model and p.n_var == s.n_var
    np.testing.assert_array_equal(p.coord, s.coord)
    np.testing.assert_array_equal(p.atom_types, s.types)
    np.testing.assert_array_equal(p.freqs, s.freqs)
    np.testing.assert_array_equal(p.density, s.density)
    np.testing.assert_array_equal(p.tau, s.tau)
    np.testing.assert_array_equal(p.neighbours, s.neighbours)
    np.testing.assert_array_equal(p.n_neighbours, s.n_neighbours)
    np.testing.assert_array_equal(p.fermi_d, s.fermi_d)
    np.testing.assert_array_equal(p.fermi_s, s.fermi_s)
    assert p.tol == s.tol and p.e0 == s.e0
    if s.alpha_w is not None:
        np.testing.assert_allclose(p.alpha_w, s.alpha_w, rtol=1e-15, atol=0)


@pytest.mark.parametrize('name', golden_dirs('bem'))
def test_bem_problem_matches_oracle(name):
    """Mesh reading (nodes in Angstrom scaled to bohr, triangles from element lines with
    at least 8 integers), eps(w) and the solver keywords agree with the oracle's reading."""
    from oracle import bem as obem
    from plasmonx_b200.bem import BemProblem
    path = os.path.join(GOLDEN, name, 'input.kw')
    p = BemProblem.from_keyword_file(path)
    o = obem.Bem(path)
    assert p.n_tess == o.n_var and p.variant == o.variant and p.green == o.green
    np.testing.assert_array_equal(p.triangles, o.t['tri'])
    np.testing.assert_allclose(p.eps, o.eps, rtol=1e-15, atol=0)
    np.testing.assert_array_equal(p.freqs, o.freqs)
    assert p.sphere_radius == o.sphere_r and p.eps_solvent == o.eps_s and p.tol == o.tol and p.e0 == o.e0


def test_bem_keyword_files_round_trip(tmp_path):
    """A synthetic surface written as the reference's input (keyword file, GMSH mesh,
    permittivity table) reads back to the same triangles, eps(w) and settings."""
    from plasmonx_b200.bem import BemProblem, bem_surface
    p = bem_surface(180, variant='iefpcm', shape='rod', n_freq=5, green='accurate', method='iterative',
                    tolerance=1e-9)
    q = BemProblem.from_keyword_file(p.write_keyword_files(str(tmp_path), 'rod'))
    np.testing.assert_allclose(q.triangles, p.triangles, rtol=1e-15, atol=1e-13)
    np.testing.assert_array_equal(q.freqs, p.freqs)
    np.testing.assert_array_equal(q.eps, p.eps)
    assert (q.variant, q.green, q.method, q.sphere_radius, q.tol) == (p.variant, p.green, p.method,
                                                                       p.sphere_radius, p.tol)


def test_synthetic_surface_sizes_and_orientation():
    """20 nu^2 tesserae; normals (a x b, factor +1) point outwards; total area within
    2% of 4 pi R^2 (an inscribed polyhedron at nu = 5)."""
    from plasmonx_b200.bem import synthetic_surface
    for n, expect in ((2000, 2000), (8000, 8000), (20000, 20480)):
        assert len(synthetic_surface('sphere', n, jitter=0.0)) == expect
    t = synthetic_surface('sphere', 500, jitter=0.0)
    c = t.mean(axis=1)
    nrm = np.cross(t[:, 1] - t[:, 0], t[:, 2] - t[:, 0])
    assert np.all(np.einsum('ij,ij->i', nrm, c) > 0)
    r = 100.0 * 1.8897261254578281
    area = 0.5 * np.linalg.norm(nrm, axis=1).sum()
    assert abs(area / (4 * np.pi * r * r) - 1) < 0.02


def test_bem_sphere_oracle_near_quasistatic_mie():
    """The oracle's DPCM and IEFPCM polarizability of a 500-tessera, 2%-jittered sphere
    is within 5% of the quasi-static Mie value R^3 (eps - 1) / (eps + 2)."""
    import tempfile
    from oracle import bem as obem
    from plasmonx_b200.bem import bem_surface
    for variant in ('dpcm', 'iefpcm'):
        p = bem_surface(500, variant=variant, n_freq=3)
        with tempfile.TemporaryDirectory() as d:
            o = obem.Bem(p.write_keyword_files(d, 's'))
        out = o.solve('inversion')
        R = 100.0 * 1.8897261254578281
        for i in range(3):
            mie = R ** 3 * (o.eps[i] - 1) / (o.eps[i] + 2)
            al = o.polar(out['x'][i])
            for k in range(3):
                assert abs(al[k, k] - mie) / abs(mie) < 0.05


def test_neighbour_counts_edge_of_nearest_distance():
    """fcc a = 4.08 A puts nearest neighbours at 2.88499... A, within r0 = 2.885 A; the
    comparison is made on Angstrom differences times ToBohr, as the reference does."""
    from plasmonx_b200 import geometry as G
    from plasmonx_b200.inputs import neighbour_counts
    pts = G.sphere('fcc', 4.08, 6.0)
    types = np.zeros(len(pts), dtype=np.int32)
    z = np.full(len(pts), 47)
    nb, nn = neighbour_counts(pts, types, z, 1)
    nb_o, nn_o = model.get_neighbours(pts, types, z, 1)
    np.testing.assert_array_equal(nn, nn_o)
    np.testing.assert_array_equal(nb, nb_o)
    assert nn.max() == 13     # 12 neighbours + itself in the bulk
