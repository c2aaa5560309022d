"""Induced field and plasmon density at points (plx_field_at_points) against the
oracle's restatement of the reference's analysis step; relative 1e-12 norm-wise,
on random points around the particle and on points sitting on atoms (inside the
0.1 bohr cut-off of the field terms)."""
import numpy as np
import pytest

from oracle.analysis import field_and_density
from plasmonx_b200 import configs
from plasmonx_b200.solver import Context, Solver

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize('metal', ['Na', 'Ag'])
def test_field_and_density_match_oracle(metal):
    p = configs.particle(metal, 'sphere', 9.0, n_freq=2, method='iterative', tolerance=1e-9)
    rng = np.random.default_rng(5)
    x = rng.standard_normal(p.n_var) + 1j * rng.standard_normal(p.n_var)
    ext = np.abs(p.coord).max()
    pts = rng.uniform(-1.5 * ext, 1.5 * ext, size=(300, 3))
    pts[:5] = p.coord[:5]                                  # on atoms
    rq, rmu = p.r_q[p.atom_types], p.r_mu[p.atom_types]
    with _ctx() as ctx:
        with Solver(p, ctx=ctx) as sv:
            for pol in (0, 2):
                f, d = sv.field_at_points(pol, x, pts)
                fr, dr = field_and_density(p.coord, rq, rmu, x, p.e0, pol, pts, p.model == 'wfqfmu')
                assert np.linalg.norm(f - fr) <= 1e-12 * np.linalg.norm(fr)
                assert np.linalg.norm(d - dr) <= 1e-12 * np.linalg.norm(dr)


class _ctx:
    def __enter__(self):
        self.c = Context(0)
        return self.c

    def __exit__(self, *a):
        self.c.close()


@pytest.mark.parametrize('name', ['analysis_field_3d_x_wfq_sodium', 'analysis_field_3d_x_y_z_wfqfmu_ag',
                                  'analysis_density_3d_x_wfq_sodium'])
def test_field_and_density_reproduce_reference_cubes(name):
    """The kernel against the cube files of the reference's analysis tests (E14.6)."""
    from tests.test_analysis_golden import load_case, quantity
    a, coords, pts, x, _, _ = load_case(name)
    metal = {11: 'Na', 47: 'Ag', 79: 'Au'}[a['z'][0]]
    p = configs.build(a['model'], np.array(a['coords_ang']), [metal], np.zeros(len(coords), np.int32),
                      np.array([0.1]), e0=a['e0'])
    assert np.isclose(p.r_q[0], a['rq']) and (a['model'] == 'wfq' or np.isclose(p.r_mu[0], a['rmu']))
    with _ctx() as ctx:
        with Solver(p, ctx=ctx) as sv:
            E, rho = sv.field_at_points(a['pol'], x, pts)
    v = quantity(a, E, rho)
    ref = np.array(a['sample_value'])
    assert np.all(np.abs(v - ref) <= 5.01e-6 * np.abs(ref) + 1e-30)
