"""Output and restart files of a spectrum, in the reference's formats.

* ``<stem>-<eV, f7.5>.plasmonX.bk`` — the per-frequency backup written after a
  frequency is solved (save_intermediate_results, src/target/target_module.f90:
  1765-1848) and read back on restart (check_if_restart /
  recover_from_backup_file, src/solvers/algorithm_module.f90:716-805: the
  results are re-read from their E14.6 print, so a recovered frequency carries
  the printed digits);
* ``<stem>.csv`` — the 20 results per frequency after a 21-line header
  (save_csv_file, target_module.f90:1853-1911), written when there is more
  than one frequency (algorithm_module.f90:176);
* ``<stem>-<eV, f12.10>.freq`` — the complex charges (and dipoles) of the x, y
  and z solutions (save_dynamic_variables, algorithm_module.f90:811-904; DPCM
  charges weighted by the tessera area);
* the maxima analysis of the log (print_maxima, algorithm_module.f90:907-978):
  interior local maxima of |sigma| (absorption, scattering or extinction);
* ``<stem>.info`` — the run's description that the reference's analysis tool
  reads (initialize_save_info, src/input_output/input_module.f90:1077-1230:
  sizes, field, kernel, model, the input geometry, the parameters, molecules,
  the dynamic parameters and the frequencies; the rotated geometry appended by
  rotate_principal_axis, src/target/target_module.f90:810-832), and
  ``<stem>.tar.gz`` packing it with the CSV and the ``.freq`` files
  (make_targz, src/input_output/output_module.f90:192-264).

``solve_spectrum`` runs a spectrum the way the reference's per-frequency loops
do with backups: frequencies whose backup exists are recovered instead of
solved, the others are solved in blocks with their backups written after each
block, then the CSV and the maxima are written and the backups of the run are
removed (output_module.f90:174-186 removes every ``*.plasmonX.bk`` of the
working directory; here only this stem's).

Numbers are formatted as Fortran's E and F edit descriptors print them
(``fortran_e``: ``0.ddddddE+xx``, the leading zero dropped when the width is
exhausted by a sign, as gfortran does).
"""
import math
import os

import numpy as np

from . import materials as M

RESULT_LABELS = ['Isotr. Real Polar.       = ', 'Isotr. Imag Polar.       = ', 'Long. Real Polar. X      = ',
                 'Long. Real Polar. Y      = ', 'Long. Real Polar. Z      = ', 'Long. Imag Polar. X      = ',
                 'Long. Imag Polar. Y      = ', 'Long. Imag Polar. Z      = ', 'Iso. Abs. Cross. Sect.   = ',
                 'Long Abs. Cross. Sect. X = ', 'Long Abs. Cross. Sect. Y = ', 'Long Abs. Cross. Sect. Z = ',
                 'Iso. Sca. Cross. Sect.   = ', 'Long Sca. Cross. Sect. X = ', 'Long Sca. Cross. Sect. Y = ',
                 'Long Sca. Cross. Sect. Z = ', 'Iso. Ext. Cross. Sect.   = ', 'Long Ext. Cross. Sect. X = ',
                 'Long Ext. Cross. Sect. Y = ', 'Long Ext. Cross. Sect. Z = ']
CSV_COLUMNS = ['Frequency (eV)', 'Isotr. Real Polar.', 'Isotr. Imag Polar.', 'Long. Real Polar. X',
               'Long. Real Polar. Y', 'Long. Real Polar. Z', 'Long. Imag Polar. X', 'Long. Imag Polar. Y',
               'Long. Imag Polar. Z', 'Iso. Abs. Cross. Sect.', 'Long Abs. Cross. Sect. X',
               'Long Abs. Cross. Sect. Y', 'Long Abs. Cross. Sect. Z', 'Iso. Sca. Cross. Sect.',
               'Long Sca. Cross. Sect. X', 'Long Sca. Cross. Sect. Y', 'Long Sca. Cross. Sect. Z',
               'Iso. Ext. Cross. Sect.', 'Long Ext. Cross. Sect. X', 'Long Ext. Cross. Sect. Y',
               'Long Ext. Cross. Sect. Z']
STICKS = ' ' + '-' * 80
MAXIMA = {'absorption': (8, 'Isotr. Abs. Cross. Sec. '), 'scattering': (12, 'Isotr. Sca. Cross. Sec. '),
          'exctinction': (16, 'Isotr. Ext. Cross. Sec. ')}


def fortran_e(x, w, d):
    """Fortran Ew.d: 0.<d digits>E<sign><2 digits>, right-justified in w columns."""
    x = float(x)
    if x == 0.0:
        # gfortran keeps the sign of a negative zero
        body = ('-' if math.copysign(1.0, x) < 0 else '') + '0.' + '0' * d + 'E+00'
    else:
        mant, ex = ('%.*e' % (d - 1, abs(x))).split('e')
        e = int(ex) + 1
        body = '0.' + mant.replace('.', '') + ('E%+03d' % e if abs(e) <= 99 else '%+04d' % e)
        if x < 0:
            body = '-' + body
    if len(body) > w and body.startswith('-0.'):
        body = '-' + body[2:]
    elif len(body) > w and body.startswith('0.'):
        body = body[1:]
    return body.rjust(w) if len(body) <= w else '*' * w


def fortran_f(x, w, d):
    s = '%*.*f' % (w, d, float(x))
    return s if len(s) <= w else '*' * w


def freq_ev(w_au):
    return float(w_au) * M.AU_TO_EV


def freq_nm(w_au):
    return M.au_to_nm(float(w_au))


def backup_path(stem, w_au):
    return '%s-%s.plasmonX.bk' % (stem, fortran_f(freq_ev(w_au), 7, 5))


def backup_text(w_au, row):
    lines = [STICKS,
             ' Results for w = %s a.u.   %s nm   %s eV' % (fortran_e(w_au, 9, 3), fortran_e(freq_nm(w_au), 9, 3),
                                                           fortran_e(freq_ev(w_au), 9, 3)),
             '']
    lines += [' %s      %s a.u.' % (lab, fortran_e(v, 14, 6)) for lab, v in zip(RESULT_LABELS, row)]
    lines.append(STICKS)
    return '\n'.join(lines) + '\n'


def write_backup(stem, w_au, row):
    path = backup_path(stem, w_au)
    with open(path, 'w') as f:
        f.write(backup_text(w_au, row))
    return path


def read_backup(path):
    """The 20 results of a backup file, read as the reference reads them (columns 35-48)."""
    with open(path) as f:
        lines = f.read().splitlines()
    vals = [float(l[34:48].replace('D', 'E')) for l in lines[3:23]]
    if len(vals) != 20:
        raise ValueError('truncated backup file %s' % path)
    return np.array(vals)


def csv_text(freqs_au, results):
    lines = ['#------------------------------------------', '#    Column          Quantity',
             '#------------------------------------------']
    for k, name in enumerate(CSV_COLUMNS):
        lines.append(('#      %-9d%-27s' % (k + 1, name)))
    lines.append('#------------------------------------------')
    for w, row in zip(freqs_au, results):
        lines.append(' ' + fortran_e(freq_ev(w), 12, 5) + ''.join('   ' + fortran_e(v, 14, 6) for v in row))
    return '\n'.join(lines) + '\n'


def write_csv(stem, freqs_au, results):
    path = stem + '.csv'
    with open(path, 'w') as f:
        f.write(csv_text(freqs_au, results))
    return path


def freq_text(w_au, x, variable='Charges', weights=None):
    """x: (n_var, 3) complex solutions (x, y, z polarisation)."""
    ev = freq_ev(w_au)
    x = np.asarray(x)
    wts = np.ones(x.shape[0]) if weights is None else np.asarray(weights)
    lines = []
    for c, lab in enumerate('xyz'):
        lines.append('complex %s: %s. freq = %s' % (variable, lab, fortran_f(ev, 25, 16)))
        for i in range(x.shape[0]):
            # (i8,5x,2(f25.16,3x)): a trailing 3x writes nothing at the end of a record
            lines.append('%8d     %s   %s' % (i + 1, fortran_f(x[i, c].real * wts[i], 25, 16),
                                             fortran_f(x[i, c].imag * wts[i], 25, 16)))
    return '\n'.join(lines) + '\n'


def read_freq(text):
    """The blocks of a .freq file: (variable name, frequency in eV, {'x'|'y'|'z': complex
    array}) -- the solutions the analysis step starts from."""
    blocks, name, ev, cur = {}, None, None, None
    for line in text.splitlines():
        if line.startswith('complex '):
            head, _, f = line.partition('. freq =')
            name, lab = head[len('complex '):].rsplit(':', 1)
            ev = float(f)
            cur = blocks.setdefault(lab.strip(), [])
        elif line.strip() and cur is not None:
            p = line.split()
            cur.append(complex(float(p[1]), float(p[2])))
    return name, ev, {k: np.array(v) for k, v in blocks.items()}


def freq_path(stem, w_au):
    return '%s-%s.freq' % (stem, fortran_f(freq_ev(w_au), 12, 10).strip())


def maxima(freqs_au, results, kind='absorption'):
    """Interior local maxima of |results[:, col]|: [(state, freq_eV, value)]."""
    col = MAXIMA[kind][0]
    out = []
    for i in range(1, len(freqs_au) - 1):
        a, b, c = abs(results[i - 1, col]), abs(results[i, col]), abs(results[i + 1, col])
        if a < b and c < b:
            out.append((len(out) + 1, freq_ev(freqs_au[i]), float(results[i, col])))
    return out


def maxima_text(n_freq, peaks, kind='absorption'):
    if not peaks:
        return ''
    lines = [' Maxima Analysis: NumExFreq = %6d' % n_freq, '',
             '          NState      Freq(eV)     %s (a.u.)' % MAXIMA[kind][1]]
    for s, ev, v in peaks:
        lines.append('          %3d     %s             %s' % (s, fortran_f(ev, 10, 3), fortran_e(v, 12, 5)))
    lines.append(STICKS)
    return '\n'.join(lines) + '\n'


def _a(v, w):
    """Fortran Aw output: right-justified in w columns, truncated to w."""
    v = str(v)
    return v.rjust(w) if len(v) <= w else v[:w]


def _info_kind(problem):
    if getattr(problem, 'triangles', None) is not None:
        return 'bem'
    return problem.forcefield if getattr(problem, 'what', None) is not None else problem.model


def info_text(problem):
    """The .info file of a run (initialize_save_info, input_module.f90:1077-1230), for a
    dynamic atomistic Problem, a BemProblem or a StaticProblem.  The rotated geometry
    of a principal-axis run is appended as rotate_principal_axis does."""
    kind = _info_kind(problem)
    bem = kind == 'bem'
    static = getattr(problem, 'what', None) is not None
    freqs = [] if static else list(np.asarray(problem.freqs, dtype=np.float64))
    if static:
        field = 'static' if problem.what == 'static' else 'absent'
    else:
        field = 'dynamic'
    kernel = 'none' if bem else problem.kernel
    forcefield = 'none' if bem else problem.forcefield
    pa = bool(getattr(problem, 'principal_axes', False) or getattr(problem, 'rotated', False))
    L = ['NAtoms     : %10d' % (0 if bem else problem.n_atoms),
         'NMolec     : %10d' % (0 if bem else problem.n_mol),
         'NVar       : %10d' % problem.n_var,
         'Field      : ' + _a(field, 10),
         'Kernel     : ' + _a(kernel, 10),
         'Model      : ' + _a(kind, 10),
         'NumExFreq  : %10d' % len(freqs),
         'Input |E|  : ' + fortran_e(problem.e0, 13, 6),
         'PrincAxes  : ' + _a('T' if pa else 'F', 10),
         'ForceField : ' + _a(forcefield, 10),
         'Input Geometry (angstrom)']
    if bem:
        t = problem.triangles
        centres = (t[:, 0] + t[:, 1] + t[:, 2]) / 3.0
        for i, c in enumerate(centres):
            L.append('%8d' % (i + 1) + ''.join(' ' + fortran_f(v / M.TO_BOHR, 25, 16) for v in c))
    else:
        coord_in = problem.coord_ang * M.TO_BOHR     # the input geometry, before any rotation
        z = problem.znum
        for i in range(problem.n_atoms):
            L.append(fortran_f(float(z[i]), 4, 1) + '  ' + '%8d' % int(problem.mol_index[i]) +
                     ''.join(' ' + fortran_f(v / M.TO_BOHR, 25, 16) for v in coord_in[i]))
        L.append('Parameters:  ' + _a(problem.forcefield, 10))
        L.append('Num. AtomTypes : %3d' % len(problem.type_names))
        for t, name in enumerate(problem.type_names):
            if problem.forcefield == 'fq' and problem.kernel != 'gaussian':
                vals = (problem.chi[t], problem.eta[t])
            elif problem.forcefield == 'fq':
                vals = (problem.chi[t], problem.eta[t], problem.r_q[t])
            else:
                vals = (problem.chi[t], problem.eta[t], problem.alpha[t], problem.r_q[t], problem.r_mu[t])
            L.append(name[:2].ljust(2) + ''.join(' ' + fortran_f(v, 25, 16) for v in vals))
        L.append('Number of atoms per IMol')
        for k, a in enumerate(problem.apm):
            L.append('%8d  %8d' % (k + 1, a))
    if kind in ('wfq', 'wfqfmu'):
        L.append('Dynamic parameters: 6')
        fe = problem.raw['fermi_energy'] or [0.0] * len(problem.type_names)
        for t in range(len(problem.type_names)):
            lab = str(t + 1) if t < 9 else '*'
            for v in (problem.tau[t], problem.sigma0[t], problem.a_ij[t], problem.fermi_d[t, t],
                      problem.fermi_s[t, t], fe[t]):
                L.append(lab + '   ' + fortran_f(v, 30, 16))
    if freqs:
        L.append('Frequencies (eV)')
        L += [fortran_f(freq_ev(w), 25, 16) for w in freqs]
    if pa and not bem:
        L.append('Rotated Geometry (Angstrom)')
        for i in range(problem.n_atoms):
            L.append(fortran_f(float(problem.znum[i]), 4, 1) + '  ' +
                     ''.join(' ' + fortran_f(v / M.TO_BOHR, 25, 16) for v in problem.coord[i]))
    return '\n'.join(L) + '\n'


def write_info(stem, problem):
    path = stem + '.info'
    with open(path, 'w') as f:
        f.write(info_text(problem))
    return path


def read_info(text):
    """The fields of a .info file (the reference's or this package's)."""
    lines = text.splitlines()
    head = {}
    for l in lines[:10]:
        k, _, v = l.partition(':')
        head[k.strip()] = v.strip()
    out = {'n_atoms': int(head['NAtoms']), 'n_mol': int(head['NMolec']), 'n_var': int(head['NVar']),
           'field': head['Field'], 'kernel': head['Kernel'], 'model': head['Model'],
           'n_freq': int(head['NumExFreq']), 'e0': float(head['Input |E|']),
           'principal_axes': head['PrincAxes'] == 'T', 'forcefield': head['ForceField']}
    i = lines.index('Input Geometry (angstrom)') + 1
    if out['model'] == 'bem':
        rows = [l.split() for l in lines[i:i + out['n_var']]]
        out['centres_ang'] = np.array([[float(v) for v in r[1:4]] for r in rows])
        i += out['n_var']
    else:
        rows = [l.split() for l in lines[i:i + out['n_atoms']]]
        out['z'] = np.array([int(float(r[0])) for r in rows])
        out['mol_index'] = np.array([int(r[1]) for r in rows])
        out['coord_ang'] = np.array([[float(v) for v in r[2:5]] for r in rows])
        i += out['n_atoms'] + 1
        nt = int(lines[i].split(':')[1])
        out['types'] = [(l[:2].strip(), [float(v) for v in l[2:].split()]) for l in lines[i + 1:i + 1 + nt]]
        i += 1 + nt + 1
        out['atoms_per_molecule'] = [int(l.split()[1]) for l in lines[i:i + out['n_mol']]]
        i += out['n_mol']
        if i < len(lines) and lines[i].startswith('Dynamic parameters'):
            vals = [float(l.split()[1]) for l in lines[i + 1:i + 1 + 6 * nt]]
            out['dynamic'] = [vals[6 * t:6 * t + 6] for t in range(nt)]
            i += 1 + 6 * nt
    if i < len(lines) and lines[i].startswith('Frequencies'):
        out['freqs_ev'] = np.array([float(l) for l in lines[i + 1:i + 1 + out['n_freq']]])
        i += 1 + out['n_freq']
    if i < len(lines) and lines[i].startswith('Rotated Geometry'):
        rows = [l.split() for l in lines[i + 1:i + 1 + out['n_atoms']]]
        out['rotated_ang'] = np.array([[float(v) for v in r[1:4]] for r in rows])
    out['terminated'] = any('Normal termination' in l for l in lines)
    return out


def make_targz(stem, freq_files=()):
    """make_targz (output_module.f90:192-264): close the .info with the termination
    lines and pack it with the CSV (when there is one) and the given .freq files into
    <stem>.tar.gz; the .info and the packed .freq files are removed (the reference
    removes every .freq of the directory; here only those of the run)."""
    import tarfile
    info = stem + '.info'
    with open(info, 'a') as f:
        f.write(STICKS + '\n' + ' ' * 24 + 'Normal termination of plasmonX\n' + STICKS + '\n')
    members = [info] + ([stem + '.csv'] if os.path.exists(stem + '.csv') else []) + list(freq_files)
    path = stem + '.tar.gz'
    with tarfile.open(path, 'w:gz') as tf:
        for m in members:
            tf.add(m, arcname=os.path.basename(m))
    for m in [info] + list(freq_files):
        os.remove(m)
    return path


def _weights(problem):
    if getattr(problem, 'triangles', None) is not None and problem.variant == 'dpcm':
        t = problem.triangles
        return 0.5 * np.linalg.norm(np.cross(t[:, 1] - t[:, 0], t[:, 2] - t[:, 0]), axis=1)
    return None


def solve_spectrum(solver, stem, restart=True, save_freq=False, block=0, maxima_kind='absorption',
                   cleanup=True, save_info=False, **solve_kw):
    """Solve the spectrum of `solver` with backups: recovered frequencies are not
    solved; the others are solved in blocks of `block` frequencies (0: all at once),
    each block's backups written when it is done.  With save_info the run's .info is
    written first and, at the end, packed with the CSV and the .freq files into
    <stem>.tar.gz.  Returns the results (F x 20), the indices recovered from backups,
    the maxima and the paths written."""
    prob = solver.prob
    if save_info:
        write_info(stem, prob)
    freqs = np.asarray(solver.freqs, dtype=np.float64)
    aw = None if prob.alpha_w is None else np.asarray(prob.alpha_w)
    F = len(freqs)
    results = np.zeros((F, 20))
    recovered, todo = [], []
    for i, w in enumerate(freqs):
        if restart and os.path.exists(backup_path(stem, w)):
            results[i] = read_backup(backup_path(stem, w))
            recovered.append(i)
        else:
            todo.append(i)
    written, freq_files = [], []
    step = block if block > 0 else max(1, len(todo))
    variable = 'Charges/Dipoles' if getattr(prob, 'model', '') == 'wfqfmu' else 'Charges'
    try:
        for b0 in range(0, len(todo), step):
            idx = todo[b0:b0 + step]
            solver.set_frequencies(freqs[idx], None if aw is None else aw[:, idx])
            out = solver.solve(want_x=save_freq, **solve_kw)
            if 'error' in out:
                raise out['error']
            for k, i in enumerate(idx):
                results[i] = out['results'][k]
                written.append(write_backup(stem, freqs[i], results[i]))
                if save_freq:
                    with open(freq_path(stem, freqs[i]), 'w') as f:
                        f.write(freq_text(freqs[i], out['x'][k], variable, _weights(prob)))
                    freq_files.append(freq_path(stem, freqs[i]))
    finally:
        solver.set_frequencies(freqs, aw)
    paths = {}
    if F > 1:
        paths['csv'] = write_csv(stem, freqs, results)
    peaks = maxima(freqs, results, maxima_kind)
    if cleanup:
        for i in range(F):
            p = backup_path(stem, freqs[i])
            if os.path.exists(p):
                os.remove(p)
    if save_info:
        paths['tar'] = make_targz(stem, freq_files)
    return {'results': results, 'recovered': recovered, 'maxima': peaks,
            'maxima_text': maxima_text(F, peaks, maxima_kind), 'paths': paths}
