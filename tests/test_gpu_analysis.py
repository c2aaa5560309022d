"""Induced field and plasmon density at points (plx_field_at_points) against the
oracle's restatement of the reference's analysis step; relative 1e-12 norm-wise,
on random points around the particle and on points sitting on atoms (inside the
0.1 bohr cut-off of the field terms)."""
import os

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


@pytest.mark.parametrize('name', ['analysis_field_3d_x_wfq_sodium', 'analysis_field_3d_x_y_z_wfqfmu_ag',
                                  'analysis_density_3d_x_wfq_sodium'])
def test_full_grid_on_device_reproduces_reference_analysis(name, tmp_path):
    """The whole 30^3 grid through the product's analysis module: the cube's sampled
    values at E14.6 and the maximum line of the reference's analysis log."""
    from plasmonx_b200 import analysis as A
    from tests.test_analysis_golden import load_case
    a, coords, _, x, _, _ = load_case(name)
    metal = {11: 'Na', 47: 'Ag', 79: 'Au'}[a['z'][0]]
    p = configs.build(a['model'], np.array(a['coords_ang']), [metal], np.zeros(len(coords), np.int32),
                      np.array([0.1]), e0=a['e0'])
    g = A.cubic_grid(np.array(a['coords_ang']), tuple(a['n']), a['offset_ang'])
    pol = 'E' + 'xyz'[a['pol']]
    with _ctx() as ctx:
        with Solver(p, ctx=ctx, store_t=False) as sv:
            if a['quantity'] == 'field':
                blocks = [('Field', A.field_on_grid(sv, x, a['pol'], g, a['e0']))]
            else:
                rho = A.density_on_grid(sv, x, g)
                blocks = [('RhoRe', rho.real), ('RhoIm', rho.imag)]
    # the cube of the quantity the reference test wrote
    cube = A.cube_text(g, blocks[0][1], a['z'], np.array(a['coords_ang'])).splitlines()[6 + len(a['z']):]
    vals = np.array([float(v) for l in cube for v in l.split()])
    ref = np.array(a['sample_value'])
    mine = vals[np.array(a['sample_index'])]
    assert np.all(np.abs(mine - ref) <= 1.0001e-6 * np.abs(ref) + 1e-30)    # one unit of the 6th digit
    assert np.mean(mine == ref) > 0.99                                         # and mostly the same digits
    for b, (kind, v) in enumerate(blocks):
        lines = A.maximum_lines(kind, pol, g, v).splitlines()
        theirs = a['log_max'][2 * b + 1].split()
        assert lines[0] == a['log_max'][2 * b] and lines[1].split()[4] == theirs[4]
        at = np.array([float(t) for t in theirs[1:4]])
        ijk = tuple(np.rint((at - g.lo) / g.step).astype(int))
        m, _ = A.maximum(g, v)
        assert abs(v[ijk] - m) <= 1e-12 * abs(m)


def test_analysis_from_a_run_archive(tmp_path):
    """A spectrum packed with save_info / save_freq, read back as the reference's
    analysis program reads it, gives the same field on the grid as the run's solver."""
    from plasmonx_b200 import analysis as A
    from plasmonx_b200 import outputs as O
    p = configs.particle('Na', 'sphere', 8.0, n_freq=2, method='inversion')
    stem = str(tmp_path / 'na')
    with _ctx() as ctx:
        with Solver(p, ctx=ctx) as sv:
            out = O.solve_spectrum(sv, stem, save_freq=True, save_info=True)
            info, sols = A.read_archive(out['paths']['tar'])
            assert info['n_atoms'] == p.n_atoms and len(sols) == 2
            label = sorted(sols)[0]
            g = A.cubic_grid(info['coord_ang'], (12, 10, 8), 5.0)
            direct = A.field_on_grid(sv, sols[label][2]['x'], 0, g, p.e0)
        q = A.problem_from_info(info)
        with Solver(q, ctx=ctx, store_t=False) as sv2:
            grid, files = A.write_cubes(stem + '.tar.gz', sv2, info, sols[label], pols=('x',), n=(12, 10, 8),
                                        offset=5.0)
            again = A.field_on_grid(sv2, sols[label][2]['x'], 0, grid, info['e0'])
    assert np.allclose(again, direct, rtol=1e-12, atol=0)
    assert [os.path.basename(f) for f in files] == ['na-Ex-%s.cube' % label]
    with open(files[0]) as f:
        text = f.read().splitlines()
    assert text[0] == 'Generated by plasmonX analysis' and int(text[2].split()[0]) == p.n_atoms


def test_bem_field_on_device_reproduces_reference_analysis(tmp_path):
    """The BEM field kernel over the whole 30^3 grid against the oracle (1e-12) and the
    reference's BEM analysis test (cube samples at E14.6, maximum line)."""
    from oracle.analysis import bem_field
    from plasmonx_b200 import analysis as A
    from tests.test_analysis_golden import TO_BOHR, _bem_case, _grid
    a, centres, q = _bem_case()
    g = _grid(a)
    with _ctx() as ctx:
        vals = A.bem_field_on_grid(ctx, np.array(a['coords_ang']), q, a['e0'], a['pol'], g)
        pts = g.points_ang()[::37] * TO_BOHR
        from plasmonx_b200 import _lib
        c = np.ascontiguousarray(np.array(a['coords_ang']) * TO_BOHR)
        E = np.zeros((len(pts), 3), dtype=np.complex128)
        pts = np.ascontiguousarray(pts)
        ctx.check(ctx.lib.plx_bem_field_at_points(ctx.h, len(c), _lib.ptr(c), _lib.ptr(q.view(np.float64)),
                                                  a['e0'], a['pol'], len(pts), _lib.ptr(pts),
                                                  _lib.ptr(E.view(np.float64))))
    Er = bem_field(centres, q, a['e0'], a['pol'], pts)
    assert np.linalg.norm(E - Er) <= 1e-12 * np.linalg.norm(Er)
    flat = vals.ravel()
    ref = np.array(a['sample_value'])
    assert np.all(np.abs(flat[np.array(a['sample_index'])] - ref) <= 5.01e-6 * np.abs(ref) + 1e-30)
    assert A.maximum_lines('Field', 'Ey', g, vals).splitlines() == a['log_max']


def _grid_cases():
    from tests import analysis_grid_cases as G
    return G.GRIDS


@pytest.mark.parametrize('name', _grid_cases())
def test_grid_analyses_on_device_reproduce_reference(name):
    """The device kernels through the product's grids and writers against every grid
    analysis test of the reference (as test_analysis_extra.py does with the oracle)."""
    from plasmonx_b200 import analysis as A
    from tests import analysis_grid_cases as G
    a = G.load(name)
    g = G.grid_for(a)
    with _ctx() as ctx:
        if a['model'] == 'bem':
            files = G.outputs(a, g, lambda x, ip, gg, t: A.bem_field_on_grid(ctx, a['centres_ang'], x, a['e0'], ip,
                                                                             gg, t), None)
        else:
            metal = {11: 'Na', 47: 'Ag', 79: 'Au'}[a['z'][0]]
            coords = np.array(a['coords_ang'])
            p = configs.build(a['model'], coords, [metal], np.zeros(len(coords), np.int32), np.array([0.1]),
                              e0=a['e0'])
            assert np.isclose(p.r_q[0], a['rq']) and (a['model'] == 'wfq' or np.isclose(p.r_mu[0], a['rmu']))
            with Solver(p, ctx=ctx, store_t=False) as sv:
                files = G.outputs(a, g, lambda x, ip, gg, t: A.field_on_grid(sv, x, ip, gg, a['e0'], t),
                                  lambda x, gg, t: A.density_on_grid(sv, x, gg, t))
    G.check(a, g, files)
