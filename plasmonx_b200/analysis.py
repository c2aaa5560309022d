"""Field and density on grids: the analysis step of the reference on the device.

The reference's analysis program (src/plasmonX_analysis) reads a run's
``.tar.gz`` (the ``.info`` description and the ``.freq`` solutions), builds a
grid around the particle and writes |E|/E0 or the plasmon density on it:
  * grids: create_cubic_grid / create_plane_grid (grid_module.f90:64-154) --
    the atoms' bounding box (Angstrom) widened by ``offset`` on every side,
    or bounds given by the user, with n points per axis and
    step = (max - min) / (n - 1); a plane keeps its third coordinate fixed;
  * values: calculate_field_3d / calculate_density_3d (grid_module.f90:200-301)
    and their plane versions (:310-453), evaluated here for all points at once
    by plx_field_at_points (csrc/analysis.cu); |E| is the norm of the complex
    field over its six real components, divided by E0;
  * files: the cube file (write_cube_file, plot_module.f90:496-562: origin and
    steps in bohr, atoms as atomic number, 0.0 and bohr coordinates, values
    E14.6 six per line with z fastest), the binary .plt (write_plt_file,
    :452-490), the plane .csv (write_csv_file, :568-611), the maximum's log
    lines (print_quantity_analysis_3d, :620-669: the first maximum in Fortran
    order, x fastest) and the effective volume and area of a slab
    (print_effective_volume_area, :680-735).
Grid arrays here are indexed [i, j, k] = [x, y, z].
"""
import os
import tarfile
from fractions import Fraction

import numpy as np

from . import materials as M
from . import outputs as O


class Grid:
    """A regular grid: bounds (Angstrom), points per axis (0 for the fixed axis of a plane)."""

    def __init__(self, lo, hi, n):
        self.lo = np.asarray(lo, dtype=np.float64)
        self.hi = np.asarray(hi, dtype=np.float64)
        self.n = [int(v) for v in n]
        self.step = np.array([(self.hi[k] - self.lo[k]) / (self.n[k] - 1) if self.n[k] > 1 else 0.0
                              for k in range(3)])

    def axes(self):
        """Coordinates along each axis, lo + i * step rounded once (as a fused
        multiply-add): the reference's build contracts min_coord + (i-1)*step this
        way, which its plane .csv files show in their last printed digit."""
        out = []
        for k in range(3):
            lo, st = Fraction(float(self.lo[k])), Fraction(float(self.step[k]))
            out.append(np.array([float(lo + i * st) for i in range(max(self.n[k], 1))]))
        return out

    def points_ang(self):
        """(nx * ny * nz, 3) points, x fastest (the reference's loop order)."""
        ax, ay, az = self.axes()
        Z, Y, X = np.meshgrid(az, ay, ax, indexing='ij')
        return np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1)

    def shape(self):
        return tuple(max(v, 1) for v in self.n)

    def info_text(self):
        """Grid Information block of the analysis log (print_grid_3d_info, grid_module.f90:159-192)."""
        s = O.STICKS
        L = [' ' * 27 + 'Grid Information (Angstrom)', s,
             (' ' * 10 + ''.join('%s%s  ' % (lab, O.fortran_f(v, 12, 4)) for lab, v in
                                 zip(('StepX: ', 'StepY: ', 'StepZ: '), self.step))).rstrip(), s]
        for k, ax in enumerate('XYZ'):
            L += [' ' * 10 + '%sminGrid:%s  %smaxGrid:%s  %s NPoints:%7d' % (
                ax, O.fortran_f(self.lo[k], 10, 4), ax, O.fortran_f(self.hi[k], 10, 4), ax, self.n[k]), s]
        return '\n'.join(L) + '\n'


def cubic_grid(coord_ang, n=(30, 30, 30), offset=10.0, lo=None, hi=None):
    """create_cubic_grid: the bounding box of the atoms +- offset (Angstrom), or lo / hi."""
    c = np.asarray(coord_ang, dtype=np.float64).reshape(-1, 3)
    lo = c.min(axis=0) - offset if lo is None else lo
    hi = c.max(axis=0) + offset if hi is None else hi
    return Grid(lo, hi, n)


def plane_grid(coord_ang, plane, n=(30, 30), offset=10.0, lo=None, hi=None):
    """create_plane_grid: plane 'xy', 'xz' or 'yz'; the fixed axis has bounds 0 and
    no points (its coordinate is given when the plane is evaluated)."""
    axes = {'xy': (0, 1), 'xz': (0, 2), 'yz': (1, 2)}[plane]
    c = np.asarray(coord_ang, dtype=np.float64).reshape(-1, 3)
    glo, ghi, gn = np.zeros(3), np.zeros(3), [0, 0, 0]
    for a, m in zip(axes, n):
        glo[a] = c[:, a].min() - offset if lo is None else lo[a]
        ghi[a] = c[:, a].max() + offset if hi is None else hi[a]
        gn[a] = m
    g = Grid(glo, ghi, gn)
    g.plane = plane
    return g


def _points_bohr(grid, third=0.0):
    """Grid points in bohr; a plane's fixed coordinate is `third` (Angstrom)."""
    pts = grid.points_ang()
    plane = getattr(grid, 'plane', None)
    if plane is not None:
        fixed = {'xy': 2, 'xz': 1, 'yz': 0}[plane]
        pts[:, fixed] = third
    return pts * M.TO_BOHR


def field_on_grid(solver, x, i_pol, grid, e0, third=0.0):
    """|E| / E0 on the grid (nx, ny, nz) for solution x of polarisation i_pol."""
    E, _ = solver.field_at_points(i_pol, x, _points_bohr(grid, third))
    v = np.sqrt((E.real ** 2 + E.imag ** 2).sum(axis=1)) / e0
    nx, ny, nz = grid.shape()
    return v.reshape(nz, ny, nx).transpose(2, 1, 0)


def bem_field_on_grid(ctx, centres_ang, q, e0, i_pol, grid, third=0.0):
    """|E| / E0 of a BEM solution on the grid: the tessera charges q (area-weighted,
    as a .freq file holds them) at their centres, zero inside the surface
    (plx_bem_field_at_points)."""
    from . import _lib
    c = np.ascontiguousarray(np.asarray(centres_ang, dtype=np.float64) * M.TO_BOHR)
    qq = np.ascontiguousarray(q, dtype=np.complex128)
    pts = np.ascontiguousarray(_points_bohr(grid, third))
    E = np.zeros((pts.shape[0], 3), dtype=np.complex128)
    ctx.check(ctx.lib.plx_bem_field_at_points(ctx.h, len(c), _lib.ptr(c), _lib.ptr(qq.view(np.float64)), float(e0),
                                              int(i_pol), pts.shape[0], _lib.ptr(pts), _lib.ptr(E.view(np.float64))))
    v = np.sqrt((E.real ** 2 + E.imag ** 2).sum(axis=1)) / e0
    nx, ny, nz = grid.shape()
    return v.reshape(nz, ny, nx).transpose(2, 1, 0)


def density_on_grid(solver, x, grid, third=0.0):
    """The plasmon density (complex) on the grid (nx, ny, nz)."""
    _, rho = solver.field_at_points(0, x, _points_bohr(grid, third))
    nx, ny, nz = grid.shape()
    return rho.reshape(nz, ny, nx).transpose(2, 1, 0)


def on_plane(grid, values):
    """A plane grid's (n1, n2) array from a (nx, ny, nz) array with one fixed axis."""
    fixed = {'xy': 2, 'xz': 1, 'yz': 0}[grid.plane]
    return np.take(values, 0, axis=fixed)


def plane_csv_text(grid, values):
    """write_csv_file (plot_module.f90:568-611): one line per point, x and y the two
    in-plane coordinates (Angstrom) and the value, E25.16 each, three blanks apart;
    a blank line after each row of the first in-plane axis."""
    i1, i2 = {'xy': (0, 1), 'xz': (0, 2), 'yz': (1, 2)}[grid.plane]
    v = np.asarray(values, dtype=np.float64)
    n1, n2 = v.shape
    ax = grid.axes()
    L = []
    for i in range(n1):
        x = ax[i1][i]
        for j in range(n2):
            y = ax[i2][j]
            q = v[i, j] if abs(v[i, j]) > 1.0e-99 else 0.0
            L.append('   '.join(O.fortran_e(t, 25, 16) for t in (x, y, q)))   # trailing 3x writes nothing
        L.append('')
    return '\n'.join(L) + '\n'


def plt_bytes(grid, values):
    """write_plt_file (plot_module.f90:452-490): one unformatted record of int32 3,
    200, nz, ny, nx, float32 z, y and x bounds, then the values as float32 with x
    fastest."""
    import struct
    v = np.asarray(values, dtype=np.float64)
    nx, ny, nz = v.shape
    head = struct.pack('<5i', 3, 200, nz, ny, nx)
    head += np.array([grid.lo[2], grid.hi[2], grid.lo[1], grid.hi[1], grid.lo[0], grid.hi[0]],
                     dtype='<f4').tobytes()
    return head + v.transpose(2, 1, 0).astype('<f4').tobytes()


def effective_volume_lines(pol_name, grid, values):
    """print_effective_volume_area (plot_module.f90:680-735) for |E|/E0 on a slab:
    V = sum(|E|^2) dx dy dz / max(|E|)^2 and A = V / (the slab's smallest extent)."""
    v = np.asarray(values, dtype=np.float64)
    integral = float((v ** 2).sum()) * grid.step[0] * grid.step[1] * grid.step[2]
    peak = float(v.max()) ** 2
    ext = grid.hi - grid.lo
    k = int(np.argmin(ext))
    if not all(ext[k] < ext[o] for o in range(3) if o != k):
        raise ValueError('The provided grid cannot be used for effective volume or area calculations')
    if ext[k] < 1.0e-14:
        raise ValueError('The minimum distance in the grid is zero')
    vol = integral / peak
    area = vol / ext[k]
    return (' Calculation of effective volume and area for polarization: %s\n' % pol_name +
            ' The slice has minimum distance in %s direction: %s Angstrom.\n' % ('XYZ'[k], O.fortran_f(ext[k], 6, 3)) +
            '\n Effective Volume : %s nm^3\n' % O.fortran_f(vol / 10 ** 3, 15, 5) +
            ' Effective Area   : %s nm^2\n' % O.fortran_f(area / 10 ** 2, 15, 5))


def cube_text(grid, values, z=None, coord_ang=None, centres_ang=None, title='Generated by plasmonX analysis'):
    """write_cube_file: atoms (z, coord_ang) or, for BEM, tessera centres."""
    vals = np.asarray(values, dtype=np.float64)
    nx, ny, nz = vals.shape
    bem = centres_ang is not None
    pos = np.asarray(centres_ang if bem else coord_ang, dtype=np.float64).reshape(-1, 3)
    f12 = lambda v: O.fortran_f(v, 12, 6)  # noqa: E731
    L = [title, '',
         '%8d' % len(pos) + ''.join(f12(v * M.TO_BOHR) for v in grid.lo),
         '%8d' % nx + f12(grid.step[0] * M.TO_BOHR) + f12(0.0) + f12(0.0),
         '%8d' % ny + f12(0.0) + f12(grid.step[1] * M.TO_BOHR) + f12(0.0),
         '%8d' % nz + f12(0.0) + f12(0.0) + f12(grid.step[2] * M.TO_BOHR)]
    for a in range(len(pos)):
        L.append('%5d ' % (0 if bem else int(z[a])) + O.fortran_f(0.0, 10, 6) +
                 ''.join(f12(v * M.TO_BOHR) for v in pos[a]))
    for i in range(nx):
        for j in range(ny):
            row = vals[i, j]
            row = np.where(np.abs(row) > 1.0e-99, row, 0.0)
            for k0 in range(0, nz, 6):
                L.append(''.join(' ' + O.fortran_e(v, 14, 6) for v in row[k0:k0 + 6]))
    return '\n'.join(L) + '\n'


def maximum(grid, values):
    """Value and grid coordinates (Angstrom) of the first maximum in Fortran order."""
    v = np.asarray(values)
    flat = v.transpose(2, 1, 0).ravel()            # x fastest
    idx = int(np.argmax(flat))
    nx, ny, _ = v.shape
    i, j, k = idx % nx, (idx // nx) % ny, idx // (nx * ny)
    ax = grid.axes()
    return float(flat[idx]), np.array([ax[0][i], ax[1][j], ax[2][k]])


def maximum_lines(kind, pol_name, grid, values):
    """print_quantity_analysis_3d lines: kind 'Field', 'RhoRe' or 'RhoIm'."""
    m, at = maximum(grid, values)
    return ('  %s%sX%sY%sZ%sMax.\n' % (kind, ' ' * 11, ' ' * 16, ' ' * 16, ' ' * 13) +
            '   %s  %s   %s\n' % (pol_name, ''.join(O.fortran_f(c, 15, 5) + '  ' for c in at),
                                 O.fortran_e(m, 13, 6)))


# van der Waals radii (Angstrom) the .pqr files carry (assign_atomic_radius,
# src/target/target_module.f90:581-632); 0 for elements without one
VDW_RADIUS = {'H': 1.20, 'He': 1.40, 'Li': 1.82, 'Be': 1.53, 'B': 1.92, 'C': 1.70, 'N': 1.55, 'O': 1.52,
              'F': 1.47, 'Ne': 1.54, 'Na': 2.27, 'Mg': 1.73, 'Al': 1.84, 'Si': 2.10, 'P': 1.80, 'S': 1.80,
              'Cl': 1.75, 'Ar': 1.88, 'Ag': 1.72, 'Au': 1.66}


def element_symbol(z):
    """assign_atom_name (src/target/target_module.f90:524-575): the element symbol
    of an atomic number the reference knows, '' otherwise."""
    for name, num in M.ELEMENTS.items():
        if num == int(z):
            return name.capitalize()
    return ''


def pqr_line(k, name, xyz_ang, value, radius, bem=False):
    """One line of write_pqr_file (plot_module.f90:401-446)."""
    f8 = ''.join(O.fortran_f(v, 8, 3) for v in xyz_ang)
    if bem:
        return 'ATOM   %4d   X  DUM     1    %s%s %s' % (k, f8, O.fortran_e(value, 11, 3), O.fortran_f(1.0, 5, 3))
    return 'ATOM   %4d  %s    X     1    %s%s %s' % (k, _a(name, 2) if len(name) < 2 else name[:2], f8,
                                                 O.fortran_e(value, 11, 3), O.fortran_f(radius, 5, 3))


def _a(v, w):
    return str(v).rjust(w)[:w]


def pqr_text(info, values):
    """A .pqr file of one polarisation's real or imaginary charges (values, n_var)."""
    bem = info['model'] == 'bem'
    if not bem and info['forcefield'] == 'fqfmu':
        raise ValueError('PQR not implemented for FQFMu')
    pos = info['centres_ang'] if bem else info['coord_ang']
    L = []
    for k in range(len(pos)):
        name = '' if bem else element_symbol(info['z'][k])
        L.append(pqr_line(k + 1, name, pos[k], values[k], VDW_RADIUS.get(name, 0.0), bem))
    return '\n'.join(L) + '\n'


def xyz_text(info):
    """plot_xyz (plot_module.f90:20-67): the count, a blank line, then element (or X
    for tesserae) and the Angstrom coordinates, f25.16."""
    bem = info['model'] == 'bem'
    pos = info['centres_ang'] if bem else info['coord_ang']
    L = [str(len(pos)).ljust(10), '']       # adjustl of an i10 field
    for k in range(len(pos)):
        name = 'X ' if bem else element_symbol(info['z'][k]).ljust(2)
        # (a2,2x,3(f25.16,1x)): the trailing 1x writes nothing
        L.append(name + '  ' + ' '.join(O.fortran_f(v, 25, 16) for v in pos[k]))
    return '\n'.join(L) + '\n'


def read_archive(path):
    """The .info description and the .freq solutions of a run's .tar.gz:
    (info dict, {freq label: (variable, freq eV, {'x'|'y'|'z': complex array})})."""
    sols = {}
    info = None
    with tarfile.open(path) as tf:
        for m in tf.getmembers():
            text = tf.extractfile(m).read().decode()
            if m.name.endswith('.info'):
                info = O.read_info(text)
            elif m.name.endswith('.freq'):
                label = m.name[:-5].rsplit('-', 1)[1]
                sols[label] = O.read_freq(text)
    if info is None:
        raise ValueError('%s holds no .info file' % path)
    return info, sols


def problem_from_info(info):
    """A dynamic atomistic problem with the geometry, widths and dynamic parameters of a
    .info file (what the analysis step needs: positions, r_q, r_mu, E0)."""
    from .inputs import Problem
    if info['model'] not in ('wfq', 'wfqfmu'):
        raise ValueError('analysis on the device: atomistic runs only (the .info model is %r)' % info['model'])
    names = [t[0] for t in info['types']]
    nt = len(names)
    par = [t[1] for t in info['types']]
    if info['model'] == 'wfq':
        chi, eta, rq = ([p[k] for p in par] for k in range(3))
        alpha, rmu = [0.0] * nt, [0.0] * nt
    else:
        chi, eta, alpha, rq, rmu = ([p[k] for p in par] for k in range(5))
    dyn = np.array(info['dynamic'])
    # each atom takes the type of its element (the .info names the types by element)
    type_of_z = {M.atomic_number(nm): t for t, nm in enumerate(names)}
    if len(type_of_z) != nt:
        raise ValueError('two atom types of the .info share an element: atoms cannot be mapped to them')
    try:
        types = [type_of_z[int(v)] for v in info['z']]
    except KeyError:
        raise ValueError('an atom whose element names no atom type of the .info')
    freqs = np.asarray(info.get('freqs_ev', []), dtype=np.float64) / M.AU_TO_EV
    return Problem(info['model'], info['coord_ang'], names, types, eta, rq, rmu, dyn[:, 0], dyn[:, 1], [1.0] * nt,
                   dyn[:, 2], np.diag(dyn[:, 3]), np.diag(dyn[:, 4]), freqs, e0=info['e0'],
                   alpha_w=None if info['model'] == 'wfq' else np.zeros((nt, len(freqs)), complex),
                   fermi_energy=dyn[:, 5], kernel=info['kernel'], chi=chi, alpha=alpha,
                   mol_index=info['mol_index'], atom_names=[names[t] for t in types])


def cube_path(root, pol_name, freq_label, suffix=''):
    """<root>-<Ex|Ey|Ez>-<freq f12.10><suffix>.cube, as plot_field_or_density names them."""
    return '%s-%s-%s%s.cube' % (root, pol_name, freq_label, suffix)


def _quantities(solver, info, x, i_pol, what, grid, third=0.0):
    """[(suffix, values)] of one polarisation: |E|/E0, or the density's two parts."""
    if info['model'] == 'bem':
        if what != 'field':
            raise ValueError('Density plot not allowed for BEM')
        return [('', bem_field_on_grid(solver, info['centres_ang'], x, info['e0'], i_pol, grid, third))]
    if what == 'field':
        return [('', field_on_grid(solver, x, i_pol, grid, info['e0'], third))]
    rho = density_on_grid(solver, x, grid, third)
    return [('-densityRe', rho.real), ('-densityIm', rho.imag)]


def _root(path, root):
    if root is not None:
        return root
    return path[:-len('.tar.gz')] if path.endswith('.tar.gz') else os.path.splitext(path)[0]


def write_cubes(path, solver, info, solution, pols=('x', 'y', 'z'), what='field', n=(30, 30, 30), offset=10.0,
                root=None, lo=None, hi=None, fmt='cube'):
    """The 3D files of one frequency's solutions (a read_freq triple) for the given
    polarisations, named as plot_field_or_density names them (plot_module.f90:124-292):
    |E|/E0 (what='field') or the density's real and imaginary parts, as cube files
    (fmt='cube') or binary .plt files (fmt='plt'), on the atoms' box widened by
    `offset` or on the bounds lo / hi.  `solver` is a Solver of the run's geometry for
    atomistic runs, a Context for BEM runs (field only, as in the reference).
    Returns the grid and the paths written."""
    variable, ev, blocks = solution
    label = O.fortran_f(ev, 12, 10).strip()
    root = _root(path, root)
    bem = info['model'] == 'bem'
    pos = info['centres_ang'] if bem else info['coord_ang']
    grid = cubic_grid(pos, n, offset, lo=lo, hi=hi)
    written = []
    for p in pols:
        if p not in blocks:
            continue
        for suffix, v in _quantities(solver, info, blocks[p], 'xyz'.index(p), what, grid):
            fn = cube_path(root, 'E' + p, label, suffix)
            if fmt == 'plt':
                fn = fn[:-len('.cube')] + '.plt'
                with open(fn, 'wb') as f:
                    f.write(plt_bytes(grid, v))
            else:
                with open(fn, 'w') as f:
                    f.write(cube_text(grid, v, centres_ang=pos) if bem else cube_text(grid, v, info['z'], pos))
            written.append(fn)
    return grid, written


def write_planes(path, solver, info, solution, plane, start, n_plane=1, step=0.0, pols=('x', 'y', 'z'),
                 what='field', n=(100, 100), offset=10.0, root=None, lo=None, hi=None):
    """The plane .csv files of one frequency's solutions (plot_field_on_planes /
    plot_density_on_planes, plot_module.f90:299-394): planes at start + i * step
    (i < n_plane) of the fixed axis, named <root>-E<p>-<freq>-p-<coordinate, f20.2>.csv
    (with -densityRe / -densityIm for the density).  Returns the grid and the paths."""
    variable, ev, blocks = solution
    label = O.fortran_f(ev, 12, 10).strip()
    root = _root(path, root)
    pos = info['centres_ang'] if info['model'] == 'bem' else info['coord_ang']
    grid = plane_grid(pos, plane, n, offset, lo=lo, hi=hi)
    written = []
    for p in pols:
        if p not in blocks:
            continue
        for k in range(n_plane):
            third = start + k * step
            tag = '-p-' + O.fortran_f(third, 20, 2).strip()
            for suffix, v in _quantities(solver, info, blocks[p], 'xyz'.index(p), what, grid, third):
                fn = '%s-E%s-%s%s%s.csv' % (root, p, label, tag, suffix)
                with open(fn, 'w') as f:
                    f.write(plane_csv_text(grid, on_plane(grid, v)))
                written.append(fn)
    return grid, written
