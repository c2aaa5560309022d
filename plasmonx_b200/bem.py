"""Boundary-element (DPCM / IEFPCM) problems: surface meshes and eps(w).

``read_msh`` reads the GMSH 2.2 ASCII files the reference reads
(read_gmsh_file / read_nodes_index_coord / read_faces,
src/bem/bem_module.f90:224-415): the node block between ``$Nodes`` and
``$EndNodes`` (index, x, y, z in Angstrom, tabs allowed), and from the element
block every line with at least 8 integers as a triangle whose node indices are
fields 6-8.  ``BemProblem`` holds what ``plx_bem_create`` needs: the triangles
in bohr (vertices scaled by ToBohr as read_nodes_index_coord does), the normal
factor, the sphere radius of the approximate Green function, the solvent
permittivity, eps(w) of the metal (Etchegoin fits or a CSV table,
input_module.f90:241-245) and the solver keywords (tolerance times
sqrt(n_tess), input_module.f90:250-251).

The synthetic surfaces of the benchmark (a sphere and a prolate rod meshed
into 20 nu^2 triangles by geodesic subdivision of an icosahedron, with a seeded
radial vertex jitter) and the Drude-Lorentz permittivity come from the shape
definitions alone; the reference meshes its surfaces with GMSH outside the
solve.
"""
import math
import os

import numpy as np

from . import materials as M
from .inputs import read_keywords

VARIANTS = {'dpcm': 'bem_dpcm', 'iefpcm': 'bem_ief'}


def _f(text):
    return float(text.replace('d', 'e').replace('D', 'e'))


def read_msh(path):
    """(node index array, xyz Angstrom (n, 3), faces (m, 3) of node indices)."""
    with open(path) as f:
        lines = f.read().replace('\t', ' ').splitlines()
    low = [l.strip().lower() for l in lines]
    try:
        i0, i1 = low.index('$nodes'), low.index('$endnodes')
    except ValueError:
        raise ValueError('Unrecognised .msh file - $Nodes/$EndNodes not found - ASCII2 format is required')
    idx, xyz = [], []
    for line in lines[i0 + 2:i1]:
        p = line.split()
        idx.append(int(p[0]))
        xyz.append([_f(p[1]), _f(p[2]), _f(p[3])])
    e0 = low.index('$elements')
    ne = int(lines[e0 + 1].split()[0])
    faces = []
    for line in lines[e0 + 2:e0 + 2 + ne]:
        p = line.split()
        if len(p) >= 8:
            faces.append([int(p[5]), int(p[6]), int(p[7])])
    return np.array(idx, dtype=np.int64), np.array(xyz, dtype=np.float64), np.array(faces, dtype=np.int64)


def triangles_from_mesh(idx, xyz_ang, faces):
    """(m, 3 vertices, 3) triangle corners in bohr."""
    where = {int(k): i for i, k in enumerate(idx)}
    xyz = np.asarray(xyz_ang, dtype=np.float64) * M.TO_BOHR
    return np.ascontiguousarray(np.array([[xyz[where[int(f)]] for f in face] for face in faces]))


# ---- synthetic surfaces ------------------------------------------------------

def _icosahedron():
    t = (1.0 + math.sqrt(5.0)) / 2.0
    v = np.array([[-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0], [0, -1, t], [0, 1, t], [0, -1, -t], [0, 1, -t],
                  [t, 0, -1], [t, 0, 1], [-t, 0, -1], [-t, 0, 1]], dtype=np.float64)
    f = [[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11], [1, 5, 9], [5, 11, 4], [11, 10, 2],
         [10, 7, 6], [7, 1, 8], [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8], [3, 8, 9], [4, 9, 5], [2, 4, 11],
         [6, 2, 10], [8, 6, 7], [9, 8, 1]]
    return v / np.linalg.norm(v, axis=1)[:, None], np.array(f)


def geodesic_sphere(nu):
    """Unit-sphere mesh of 20 nu^2 triangles, counter-clockwise seen from outside;
    shared vertices merged."""
    v0, f0 = _icosahedron()
    verts, key, faces = [], {}, []

    def vid(p):
        q = p / np.linalg.norm(p)
        k = tuple(np.round(q, 12))
        if k not in key:
            key[k] = len(verts)
            verts.append(q)
        return key[k]

    for a, b, c in f0:
        A, B, C = v0[a], v0[b], v0[c]
        grid = {}
        for i in range(nu + 1):
            for j in range(nu + 1 - i):
                grid[i, j] = vid(A + (B - A) * (i / nu) + (C - A) * (j / nu))
        for i in range(nu):
            for j in range(nu - i):
                faces.append([grid[i, j], grid[i + 1, j], grid[i, j + 1]])
                if i + j < nu - 1:
                    faces.append([grid[i + 1, j], grid[i + 1, j + 1], grid[i, j + 1]])
    return np.array(verts), np.array(faces)


def _nu_for(n_tess):
    return max(1, int(round(math.sqrt(n_tess / 20.0))))


def synthetic_surface(shape, n_tess, jitter=0.02, seed=1, radius_nm=10.0, length_nm=40.0, rod_radius_nm=5.0):
    """Triangles (bohr) of a sphere or a prolate rod (spheroid of the given length and radius).

    The mesh has 20 nu^2 tesserae with nu = round(sqrt(n_tess / 20)) (2000, 8000 and
    20480 for 2k, 8k, 20k); each vertex is moved radially by a factor 1 + U(-jitter, jitter)."""
    v, f = geodesic_sphere(_nu_for(n_tess))
    rng = np.random.default_rng(seed)
    v = v * (1.0 + rng.uniform(-jitter, jitter, size=(len(v), 1)))
    if shape == 'sphere':
        scale = np.array([radius_nm] * 3)
    elif shape == 'rod':
        scale = np.array([rod_radius_nm, rod_radius_nm, length_nm / 2.0])
    else:
        raise ValueError('shape must be sphere or rod, got %r' % shape)
    ang = v * scale * 10.0
    return np.ascontiguousarray(ang[f] * M.TO_BOHR)


def drude_lorentz(freqs_au, wp=9.0, gamma=0.07, w0=4.0, strength=1.0, width=0.5, eps_inf=1.0):
    """eps(w) = eps_inf - wp^2 / (w (w + i gamma)) + f w0^2 / (w0^2 - w^2 - i width w), energies in eV."""
    w = np.asarray(freqs_au, dtype=np.float64) * M.AU_TO_EV
    return eps_inf - wp ** 2 / (w * (w + 1j * gamma)) + strength * w0 ** 2 / (w0 ** 2 - w ** 2 - 1j * width * w)


class BemProblem:
    """A BEM surface with its permittivity and solver settings."""

    def __init__(self, triangles, eps, freqs, variant='dpcm', green='approximate', sphere_radius=0.0,
                 eps_solvent=1.0, normal_factor=1.0, e0=1e-4, polarization='all', method='inversion',
                 tolerance=1e-9, gmres_dim=1000):
        if variant not in VARIANTS:
            raise ValueError('bem variant must be dpcm or iefpcm, got %r' % variant)
        if green not in ('approximate', 'accurate'):
            raise ValueError('bem green function must be approximate or accurate, got %r' % green)
        self.triangles = np.ascontiguousarray(triangles, dtype=np.float64).reshape(-1, 3, 3)
        self.n_tess = self.n_var = len(self.triangles)
        self.variant = variant
        self.model = VARIANTS[variant]
        self.green = green
        self.accurate = green == 'accurate'
        self.sphere_radius = float(sphere_radius)
        self.eps_solvent = float(eps_solvent)
        self.normal_factor = float(normal_factor)
        self.freqs = np.asarray(freqs, dtype=np.float64)
        self.eps = np.ascontiguousarray(eps, dtype=np.complex128).reshape(len(self.freqs))
        self.e0 = float(e0)
        self.polarization = polarization
        self.method = method
        self.tolerance_input = float(tolerance)
        self.tol = self.tolerance_input * math.sqrt(self.n_var)
        self.gmres_dim = int(gmres_dim)

    @property
    def pol_mask(self):
        return {'all': 7, 'x': 1, 'y': 2, 'z': 4}[self.polarization]

    @property
    def alpha_w(self):
        """eps(w) in the per-frequency slot plx_set_frequencies reads for BEM."""
        return self.eps.reshape(1, -1)

    def write_keyword_files(self, directory, stem='surface'):
        """The problem as the reference's input: ``<stem>.kw`` keyword file, ``<stem>.msh``
        (GMSH 2.2 ASCII, three nodes per triangle, Angstrom) and ``<stem>_eps.csv``
        ('eV Re Im' rows, the bem permittivity file format).  Returns the keyword-file path."""
        os.makedirs(directory, exist_ok=True)
        msh = os.path.join(directory, stem + '.msh')
        ang = self.triangles.reshape(-1, 3) / M.TO_BOHR
        with open(msh, 'w') as f:
            f.write('$MeshFormat\n2.2 0 8\n$EndMeshFormat\n$Nodes\n%d\n' % len(ang))
            for k, (x, y, z) in enumerate(ang):
                f.write('%d %.17g %.17g %.17g\n' % (k + 1, x, y, z))
            f.write('$EndNodes\n$Elements\n%d\n' % self.n_tess)
            for t in range(self.n_tess):
                f.write('%d 2 2 0 1 %d %d %d\n' % (t + 1, 3 * t + 1, 3 * t + 2, 3 * t + 3))
            f.write('$EndElements\n')
        csv = os.path.join(directory, stem + '_eps.csv')
        with open(csv, 'w') as f:
            f.write('# freq(eV) Re(eps) Im(eps)\n')
            for w, e in zip(self.freqs, self.eps):
                f.write('%r %r %r\n' % (float(w * M.AU_TO_EV), float(e.real), float(e.imag)))
        L = ['what: dynamic response', 'algorithm method: %s' % self.method,
             'algorithm tolerance: %r' % self.tolerance_input, 'algorithm gmres dimension: %d' % self.gmres_dim,
             'forcefield dynamic: none', 'field rhs type: field', 'field field intensity: %r' % self.e0,
             'field nfreq: %d' % len(self.freqs), 'field min freq: 0.0', 'field max freq: 0.0',
             'field step freq: 0.0', 'field external freq: ' + ' '.join(repr(float(w)) for w in self.freqs),
             'field polarization: %s' % self.polarization, 'bem mesh file: %s' % os.path.basename(msh),
             'bem normal scalar factor: %r' % self.normal_factor,
             'bem permittivity file: %s' % os.path.basename(csv), 'bem permittivity: none',
             'bem green function: %s' % self.green, 'bem sphere radius: %r' % self.sphere_radius,
             'bem epsilon solvent: %r' % self.eps_solvent, 'bem variant: %s' % self.variant,
             'atom_types number: 0', 'number of atoms: 0']
        kwp = os.path.join(directory, stem + '.kw')
        with open(kwp, 'w') as f:
            f.write('\n'.join(L) + '\n')
        return kwp

    @classmethod
    def from_keyword_text(cls, text, base_dir='.'):
        kw = read_keywords(text)[0]

        def num(k, d):
            return _f(str(kw.get(k, d)))

        msh = kw['bem mesh file'].strip()
        idx, xyz, faces = read_msh(msh if os.path.isabs(msh) else os.path.join(base_dir, msh))
        nf = int(float(kw['field nfreq']))
        fmin, fmax = float(kw['field min freq']), float(kw['field max freq'])
        if fmin == 0.0 and fmax == 0.0:
            freqs = [float(x) for x in kw['field external freq'].replace(',', ' ').split()][:nf]
        else:
            st = float(kw['field step freq'])
            freqs = [fmin + st * i for i in range(nf)]
        perm = kw.get('bem permittivity', 'none').strip()
        pfile = kw.get('bem permittivity file', 'none').strip()
        if perm != 'none':
            eps = M.fitted(perm, freqs, 'epsilon')
        else:
            eps = M.read_table(pfile if os.path.isabs(pfile) else os.path.join(base_dir, pfile), freqs)
        return cls(triangles_from_mesh(idx, xyz, faces), eps, freqs,
                   variant=kw.get('bem variant', 'dpcm').strip(),
                   green=kw.get('bem green function', 'approximate').strip(),
                   sphere_radius=num('bem sphere radius', 0.0), eps_solvent=num('bem epsilon solvent', 1.0),
                   normal_factor=num('bem normal scalar factor', 1.0), e0=num('field field intensity', 1e-4),
                   polarization=kw.get('field polarization', 'all').strip(),
                   method=kw.get('algorithm method', 'inversion').strip(),
                   tolerance=num('algorithm tolerance', 0.0),
                   gmres_dim=int(num('algorithm gmres dimension', 1000)))

    @classmethod
    def from_keyword_file(cls, path):
        with open(path) as f:
            return cls.from_keyword_text(f.read(), base_dir=os.path.dirname(os.path.abspath(path)))


def bem_surface(n_tess=2000, variant='dpcm', shape='sphere', n_freq=301, seed=1, green='approximate', **kw):
    """Synthetic BEM workload: a 10 nm sphere or a 40 x 10 nm prolate rod in vacuum, eps from
    the Drude-Lorentz model, 1.5-4.5 eV.  The approximate Green function uses the sphere
    radius (10 nm; for the rod its semi-minor axis, 5 nm)."""
    from .configs import ev_grid
    tri = synthetic_surface(shape, n_tess, seed=seed)
    freqs = ev_grid(1.5, 4.5, n_freq)
    r_nm = 10.0 if shape == 'sphere' else 5.0
    return BemProblem(tri, drude_lorentz(freqs), freqs, variant=variant, green=green,
                      sphere_radius=r_nm * 10.0 * M.TO_BOHR, **kw)
