"""Shared checks for the reference's grid analysis tests (fixtures in
``tests/golden/analysis_grids``, made by ``make_golden.py --analysis-grids``).

For one test: rebuild its grid (cube, slab or planes) from the test's own
options, evaluate |E|/E0 or the density with a given backend (the oracle on
the CPU, the device kernels on a B200), write the files through the product's
writers (plasmonx_b200/analysis.py) and compare them with the reference's
sampled output files and log lines:
  * .csv planes: coordinates to every printed digit, values within 1e-10;
  * .cube: header numbers as printed, values within half a unit of the 6th digit;
  * .plt: header integers and floats, values within one float32 ulp;
  * the maximum's log lines (value as printed; the location the reference's or a
    point whose value ties within 1e-12) and the effective-volume lines.
"""
import json
import os
import struct

import numpy as np

from tests.conftest import GOLDEN

TO_BOHR = 1.8897261254578281
GRIDS_DIR = os.path.join(GOLDEN, 'analysis_grids')
GRIDS = sorted(f[:-5] for f in os.listdir(GRIDS_DIR) if f.endswith('.json'))


def load(name):
    with open(os.path.join(GRIDS_DIR, name + '.json')) as f:
        return json.load(f)


def _vec(s):
    return np.array([float(v) for v in str(s).split(',')])


def positions(a):
    return np.array(a['centres_ang'] if a['model'] == 'bem' else a['coords_ang'])


def grid_for(a):
    from plasmonx_b200 import analysis as A
    o = a['options']
    n = [int(a['log_grid'][k].split()[-1]) for k in (4, 6, 8)]
    lo = _vec(o['min_grid']) if 'min_grid' in o else None
    hi = _vec(o['max_grid']) if 'max_grid' in o else None
    if 'plane' in o:
        axes = {'xy': (0, 1), 'xz': (0, 2), 'yz': (1, 2)}[o['plane']]
        return A.plane_grid(positions(a), o['plane'], tuple(n[k] for k in axes), 10.0, lo=lo, hi=hi)
    return A.cubic_grid(positions(a), n, 10.0, lo=lo, hi=hi)


def planes(a):
    """Third coordinates of the planes: start + i * step_plane."""
    o = a['options']
    if 'plane' not in o:
        return [0.0]
    step = float(o.get('step_plane', 0.0))
    return [float(o['start']) + i * step for i in range(int(o.get('n_plane', 1)))]


def solution(a, p):
    x = np.array(a['x'][p])
    return x[:, 0] + 1j * x[:, 1]


def outputs(a, g, field_fn, density_fn):
    """{file name: (kind, values)} the test wrote; field_fn(x, i_pol, grid, third) and
    density_fn(x, grid, third) return (nx, ny, nz) arrays."""
    from plasmonx_b200 import analysis as A
    from plasmonx_b200 import outputs as O
    o = a['options']
    out = {}
    ext = '.plt' if o.get('format_grid') == 'plt' else '.cube'
    for p in a['pols']:
        x = solution(a, p)
        for third in planes(a):
            if a['what'] == 'field':
                vals = [('', field_fn(x, 'xyz'.index(p), g, third))]
            else:
                rho = density_fn(x, g, third)
                vals = [('-densityRe', rho.real), ('-densityIm', rho.imag)]
            for suffix, v in vals:
                if 'plane' in o:
                    tag = '-p-' + O.fortran_f(third, 20, 2).strip()
                    out['%s-E%s-%s%s%s.csv' % (a['name'], p, a['label'], tag, suffix)] = ('csv', A.on_plane(g, v))
                else:
                    out['%s-E%s-%s%s%s' % (a['name'], p, a['label'], suffix, ext)] = (ext[1:], v)
    return out


def check(a, g, files):
    """Compare the writers' output for `files` (from outputs()) with the reference."""
    from plasmonx_b200 import analysis as A
    assert [l.rstrip() for l in g.info_text().splitlines()] == [l.rstrip() for l in a['log_grid']]
    assert sorted(files) == sorted(a['files'])
    pos = positions(a)
    bem = a['model'] == 'bem'
    for fn, (kind, v) in files.items():
        ref = a['files'][fn]
        if kind == 'csv':
            mine = A.plane_csv_text(g, v).splitlines()
            assert len(mine) == ref['n_lines'], fn
            for i, line in zip(ref['index'], ref['lines']):
                m, r = mine[i].split(), line.split()
                assert m[:2] == r[:2] and len(mine[i]) == len(line), (fn, i, mine[i], line)
                if r:
                    assert abs(float(m[2]) - float(r[2])) <= 1e-10 * abs(float(r[2])) + 1e-300, (fn, i, mine[i], line)
        elif kind == 'cube':
            text = (A.cube_text(g, v, centres_ang=pos) if bem else A.cube_text(g, v, a['z'], pos)).splitlines()
            assert len(text) == ref['n_lines'], fn
            head = 6 + len(pos)
            for i, line in zip(ref['index'], ref['lines']):
                if i == 0:
                    continue                      # the title names the releasing program
                if i < head:
                    assert text[i].split() == line.split(), (fn, i)
                    continue
                for m, r in zip(text[i].split(), line.split()):
                    assert abs(float(m) - float(r)) <= 5.01e-6 * abs(float(r)) + 1e-30, (fn, i, text[i], line)
        else:
            data = A.plt_bytes(g, v)
            assert len(data) == ref['bytes']
            assert list(struct.unpack('<5i', data[:20])) == ref['head_i']
            assert list(struct.unpack('<6f', data[20:44])) == ref['head_f']
            mine = np.frombuffer(data[44:], dtype='<f4')[np.array(ref['index'])]
            theirs = np.array(ref['values'], dtype=np.float32)
            assert np.all(np.abs(mine - theirs) <= np.spacing(np.abs(theirs))), fn
    # the maximum's lines (3D runs, log order: per polarisation the field, or the
    # density's real then imaginary part) and the effective volume (slabs)
    blocks = []
    for p in a['pols']:
        mine = sorted((fn, val) for fn, (kind, val) in files.items() if '-E%s-' % p in fn)
        if a['what'] == 'field':
            blocks += [('Field', 'E' + p, val) for fn, val in mine]
        else:
            blocks += [('RhoRe' if 'densityRe' in fn else 'RhoIm', 'E' + p, val)
                       for fn, val in sorted(mine, key=lambda t: 'densityIm' in t[0])]
    if a['log_max']:
        assert len(blocks) == len(a['log_max'])
        for (kind, pol, v), (rh, rl) in zip(blocks, a['log_max']):
            mh, ml = A.maximum_lines(kind, pol, g, v).splitlines()
            assert mh == rh
            m, r = ml.split(), rl.split()
            assert m[0] == r[0] and m[4] == r[4], (ml, rl)
            if m[1:4] != r[1:4]:
                at = np.array([float(t) for t in r[1:4]])
                ijk = tuple(np.rint((at - g.lo) / np.where(g.step > 0, g.step, 1.0)).astype(int))
                peak, _ = A.maximum(g, v)
                assert abs(v[ijk] - peak) <= 1e-12 * abs(peak), (ml, rl)
    for lines in a['volume_lines']:
        v = [val for fn, (kind, val) in files.items()][0]
        assert A.effective_volume_lines(lines[0].split()[-1], g, v).splitlines() == lines
