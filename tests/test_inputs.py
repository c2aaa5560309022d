"""Host-side input handling agrees with the oracle's independent reading of the same keyword files."""
import os

import numpy as np
import pytest

from oracle import model
from plasmonx_b200.inputs import Problem
from tests.conftest import GOLDEN, golden_dirs


@pytest.mark.parametrize('name', golden_dirs())
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
