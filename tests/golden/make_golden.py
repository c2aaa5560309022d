"""Generate the golden fixtures under tests/golden/ from the plasmonX reference tree.

Run in a container that has the reference checked out (read-only is fine):

    python tests/golden/make_golden.py /path/to/plasmonX

For each hot-path regression test of the reference (``tests/<name>/``) this
script
  1. runs the reference's own Python front end (``python/input_``) on the
     test's YAML, with a stub for the optional ``ase`` package, and stores the
     keyword file it writes (what the reference Fortran reads) as
     ``<name>/input.kw``;
  2. copies the rows of any permittivity / interband-polarizability CSV that
     the test's frequencies use;
  3. parses the reference log ``tests/<name>/reference/<name>.log`` and stores
     the printed numbers in ``<name>/expected.json``: the final per-frequency
     results block (20 values), the charge / dipole tables, the GMRES residual
     traces, when printed the full dynamic matrix, the maxima analysis and the
     frequencies recovered from backup files;
  4. copies the test's backup files (``bk/*.plasmonX.bk``, restart tests).
With ``--geom`` it does the same for the tests whose geometry the reference's
``geom`` generator built (a submodule that is not in the reference tree): the
test's YAML is given an external .xyz of the geometry its log printed in place
of the generator section.
With ``--analysis`` it instead stores, for three analysis tests of the
reference, the inputs of the field / density step and a sample of the cube
file the reference wrote (``<name>/analysis.json``).  With ``--analysis-grids`` it stores, for fourteen more analysis tests
(planes, user-bounded planes and slabs with their effective volume, the
binary .plt format, wFQFMu densities, a BEM plane), their inputs and sampled
outputs in ``analysis_grids/``; with ``--pqr-xyz`` sampled lines of its .pqr
and .xyz outputs in ``analysis_extra/``.  With
``--info`` it copies three
``.info`` files and one ``.freq`` file out of the reference's analysis-test
tarballs into ``info/`` (the files its analysis tool reads).  With ``--static`` it
stores, for the five static FQ / FQFMu tests, the keyword file and the numbers
their logs print (static matrix, right-hand side, charges, dipoles, energy,
J^-1, the polarizability tensor, the rotated geometry) in ``expected.json``.
Nothing at run time of the tests reads the reference tree; only these files.
"""
import json
import os
import re
import shutil
import sys
import tempfile
import time

HERE = os.path.dirname(os.path.abspath(__file__))

TESTS = [
    'wfq_sodium_inversion',
    'wfq_sodium_iterative_on_memory',
    'wfq_sodium_iterative_on_the_fly',
    'wfq_sodium_minimal_input',
    'wfqfmu_ag_inversion',
    'wfqfmu_ag_iterative_on_memory',
    'wfqfmu_ag_iterative_on_the_fly',
    'wfqfmu_ag_internal_permittivity',
    'wfqfmu_ag_minimal_input',
    'wfqfmu_au_minimal_input',
    'wfqfmu_hetero_agau_inversion',
    'wfqfmu_hetero_agau_iterative_on_memory',
    'wfqfmu_hetero_agau_iterative_on_the_fly',
    'wfqfmu_hetero_agau_default_int_param_inversion',
    'wfqfmu_hetero_agau_read_1param_inversion',
    'wfqfmu_hetero_agau_minimal_input',
    'bem_ief_approximate_inversion',
    'bem_ief_accurate_inversion',
    'bem_dpcm_accurate_inversion',
    'bem_dpcm_accurate_iterative_on_memory',
    'wfq_sodium_restart',
    'wfqfmu_ag_restart',
    'wfq_graphene_disk_inversion',
    'wfq_graphene_ribbon_inversion',
    'wfq_graphene_triangle_inversion',
    'wfq_graphene_minimal_input',
    'wfqfmu_ag_diff_units',
    'wfqfmu_ag_read_xyz',
    'wfqfmu_au_read_xyz',
    'wfqfmu_hetero_agau_read_xyz',
    'bem_dpcm_external_brendel_bormann_ag',
]

# tests whose geometry the reference's geom generator (a submodule absent from
# the tree) built; their logs print it, and that printed geometry stands in
GEOM_TESTS = [
    'wfq_sodium_geom_rod',
    'wfq_sodium_geom_sphere',
    'wfq_graphene_geom_disk',
    'wfq_graphene_geom_ribbon_main_armchair',
    'wfq_graphene_geom_ribbon_main_zigzag',
    'wfq_graphene_geom_ring',
    'wfq_graphene_geom_triangle_armchair',
    'wfq_graphene_geom_triangle_zigzag',
    'wfqfmu_ag_geom_decahedron',
    'wfqfmu_ag_geom_dimer_bowtie',
    'wfqfmu_ag_geom_rod_x',
    'wfqfmu_ag_geom_sphere',
    'wfqfmu_ag_geom_sphere_units',
    'wfqfmu_au_geom_cuboctahedron',
    'wfqfmu_au_geom_dimer_z',
    'wfqfmu_au_geom_icosahedron',
    'wfqfmu_au_geom_paraboloid',
    'wfqfmu_hetero_agau_geom_rod_core_shell',
    'wfqfmu_hetero_agau_geom_sphere_core_shell',
]

NUM = r'[-+]?\d*\.\d+(?:[EeDd][-+]?\d+)?'

XYZ_STUB = '''class _Atom:
    def __init__(self, symbol, position):
        self.symbol = symbol
        self.position = position


def read(path, *a, **k):
    with open(path) as f:
        lines = f.read().splitlines()
    n = int(lines[0].split()[0])
    atoms = []
    for line in lines[2:2 + n]:
        p = line.split()
        atoms.append(_Atom(p[0], [float(p[1]), float(p[2]), float(p[3])]))
    return atoms
'''


def run_front_end(ref, test_dir, yaml_name, work):
    stub = os.path.join(work, 'stub', 'ase')
    os.makedirs(stub, exist_ok=True)
    with open(os.path.join(stub, '__init__.py'), 'w') as f:
        f.write('')
    with open(os.path.join(stub, 'io.py'), 'w') as f:
        # a plain-XYZ reader standing in for ase.io.read (count line, comment line,
        # then 'symbol x y z' per atom): what the front end needs for an external
        # xyz geometry
        f.write(XYZ_STUB)
    for fn in os.listdir(test_dir):
        p = os.path.join(test_dir, fn)
        if os.path.isfile(p):
            shutil.copy(p, work)
    sys.path[:0] = [os.path.join(work, 'stub'), os.path.join(ref, 'python')]
    from input_ import yaml_to_fortran_input  # noqa: E402  (reference front end)
    cwd = os.getcwd()
    os.chdir(work)
    try:
        t0, w0 = time.process_time(), time.time()
        yaml_to_fortran_input(t0, w0, yaml_name, 'input.kw', yaml_name[:-5] + '.log', 8, 31.07, ref,
                              {'front end': 'reference'}, [])
        with open('input.kw') as f:
            return f.read()
    finally:
        os.chdir(cwd)


def parse_log(text):
    out = {}
    # final results block, after the backup clean-up message
    tail = text.split('I am cleaning up the backup')[-1]
    res = []
    for blk in re.split(r'Results for w =', tail)[1:]:
        head = blk.split('\n', 1)[0]
        vals = re.findall(r'=\s+(' + NUM + r') a\.u\.', blk)
        if len(vals) >= 20:
            w_au = float(re.findall(NUM, head)[0])
            res.append({'w_au_printed': w_au, 'values': [float(v) for v in vals[:20]]})
    out['results'] = res
    # charge / dipole tables (verbose >= 2)
    tables = []
    for m in re.finditer(r'(wFQ Charges|wFMu Dipoles|BEM Charges)\n(.*?)(?:\n -{20,}|\nChErr)', text, re.S):
        rows = []
        for line in m.group(2).splitlines():
            nums = re.findall(NUM, line)
            if re.match(r'^\s+\d+\s', line) and len(nums) == 6:
                rows.append([float(v) for v in nums])
        tables.append({'kind': m.group(1), 'rows': rows})
    out['tables'] = tables
    # GMRES residual traces
    traces = []
    for m in re.finditer(r'Freq:\s+(' + NUM + r') eV.*?\n(.*?)(?=GMRES Iterative|wFQ Charges|Results for w|\Z)', text, re.S):
        freq_ev = float(m.group(1))
        for pm in re.finditer(r'- Polarization: ([XYZ])\s+Iteration\s+Residual\n((?:\s+\d+\s+' + NUM + r'\n)+)',
                              m.group(2)):
            vals = [float(v) for v in re.findall(r'\s+\d+\s+(' + NUM + r')\n', pm.group(2))]
            traces.append({'freq_ev': freq_ev, 'pol': pm.group(1), 'residuals': vals})
    out['gmres'] = traces
    # maxima analysis (print_maxima) and frequencies recovered from backups
    m = re.search(r'Maxima Analysis: NumExFreq =\s+(\d+)\n\n.*?\n((?:\s+\d+\s+' + NUM + r'\s+' + NUM + r'\n)+)',
                  text)
    if m:
        out['maxima'] = {'n_freq': int(m.group(1)),
                         'rows': [[float(v) for v in re.findall(NUM, l)] for l in m.group(2).splitlines()]}
    out['recovered_ev'] = [float(v) for v in re.findall(r'Recovering from backup frequency:\s+(' + NUM + r') eV',
                                                        text)]
    # full dynamic matrix print (verbose 3, inversion)
    for part in ('Real', 'IMag'):
        key = 'matrix_' + part.lower()
        m = re.search(r'(?:wfqfmu|wFQ) Matrix: ' + part + r' Part\n -+\n(.*?)\n -{20,}', text, re.S)
        if not m:
            continue
        entries = {}
        cols = None
        for line in m.group(1).splitlines():
            if not line.strip():
                continue
            toks = line.split()
            if all(re.fullmatch(r'\d+', t) for t in toks):
                cols = [int(t) for t in toks]
                continue
            if cols and re.fullmatch(r'\d+', toks[0]):
                r = int(toks[0])
                for c, v in zip(cols, toks[1:]):
                    entries['%d,%d' % (r, c)] = float(v.replace('D', 'E'))
        out[key] = entries
    return out


def filters(text):
    """Argument strings of every get_filter(...) call (balanced parentheses)."""
    out = []
    for m in re.finditer(r'get_filter\(', text):
        depth, i = 1, m.end()
        while depth and i < len(text):
            depth += {'(': 1, ')': -1}.get(text[i], 0)
            i += 1
        out.append(text[m.end():i - 1])
    return out


def csv_subset(path, freqs_ev):
    keep = []
    with open(path) as f:
        for line in f:
            if '#' in line:
                keep.append(line)
                continue
            p = line.replace(',', ' ').split()
            if len(p) >= 3 and any(abs(float(p[0]) - e) <= 1e-6 for e in freqs_ev):
                keep.append(line)
    return ''.join(keep)


def main(ref):
    import subprocess
    for name in TESTS:
        # one process per test: the front end keeps module-level state
        subprocess.run([sys.executable, os.path.abspath(__file__), '--one', name, ref], check=True,
                       stderr=subprocess.DEVNULL)


def log_geometry(text):
    """(symbol, x, y, z) strings of the log's 'Input Geometry (Ang)' block
    (print_geometry, src/target/target_module.f90:1501-1508: F20.6 in Angstrom)."""
    rows = []
    for line in text.split('Input Geometry (Ang)', 1)[1].splitlines():
        p = line.split()
        if len(p) != 5 or not p[0].isdigit():
            if rows:
                break
            continue
        assert int(p[0]) == len(rows) + 1
        rows.append(tuple(p[1:]))
    return rows


def geom_front_end(ref, tdir, yaml_name, work):
    """The keyword file of a test whose geometry the geom generator built (the
    generator is not in the reference tree): the test's YAML with its
    input_geometry section replaced by an external .xyz of the geometry its log
    printed, run through the same front end (geometry from the generator and from
    an .xyz reach the keyword writer in the same form, geom_interface.py:427-438
    and io_operations.py:107-118)."""
    import yaml
    name = os.path.basename(tdir)
    with open(os.path.join(tdir, 'reference', name + '.log')) as f:
        rows = log_geometry(f.read())
    src = os.path.join(work, 'src')
    os.makedirs(src)
    with open(os.path.join(tdir, yaml_name)) as f:
        data = yaml.safe_load(f)
    data['input_geometry'] = {'external xyz file': 'printed_geometry.xyz'}
    with open(os.path.join(src, yaml_name), 'w') as f:
        yaml.safe_dump(data, f, sort_keys=False)
    with open(os.path.join(src, 'printed_geometry.xyz'), 'w') as f:
        f.write('%d\n\n' % len(rows) + ''.join('%s %s %s %s\n' % r for r in rows))
    kw = run_front_end(ref, src, yaml_name, os.path.join(work, 'run'))
    # the keyword file carries the printed coordinates, in order
    lines = kw.split('input_geometry', 1)[1].splitlines()[1:1 + len(rows)]
    for line, r in zip(lines, rows):
        p = line.split()
        assert p[0] == r[0] and all(abs(float(a) - float(b)) <= 5e-7 for a, b in zip(p[2:5], r[1:])), (line, r)
    return kw


def one(name, ref):
    if True:
        tdir = os.path.join(ref, 'tests', name)
        yamls = [f for f in os.listdir(tdir) if f.endswith('.yaml')]
        with tempfile.TemporaryDirectory() as work:
            if name in GEOM_TESTS:
                kw = geom_front_end(ref, tdir, yamls[0], work)
            else:
                kw = run_front_end(ref, tdir, yamls[0], work)
        odir = os.path.join(HERE, name)
        os.makedirs(odir, exist_ok=True)
        with open(os.path.join(odir, 'input.kw'), 'w') as f:
            f.write(kw)
        # frequencies (a.u. -> eV) for CSV row selection
        vals = dict(l.split(':', 1) for l in kw.splitlines() if ':' in l and not l.startswith('#'))
        nf = int(float(vals['field nfreq']))
        fmin, fmax, fstep = (float(vals['field min freq']), float(vals['field max freq']),
                             float(vals['field step freq']))
        if fmin == 0.0 and fmax == 0.0:
            fr = [float(x) for x in vals['field external freq'].replace(',', ' ').split()][:nf]
        else:
            fr = [fmin + fstep * i for i in range(nf)]
        fev = [w * 27.211386245981 for w in fr]
        for line in kw.splitlines():
            if line.startswith('bem mesh file:'):
                fn = line.split(':', 1)[1].strip()
                if fn != 'none':
                    shutil.copy(os.path.join(tdir, fn), os.path.join(odir, os.path.basename(fn)))
            if line.startswith('bem permittivity file:'):
                fn = line.split(':', 1)[1].strip()
                if fn != 'none':
                    with open(os.path.join(odir, os.path.basename(fn)), 'w') as f:
                        f.write(csv_subset(os.path.join(tdir, fn), fev))
            if 'wfqfmu file:' in line:
                fn = line.split(':', 1)[1].strip()
                if fn != 'none':
                    src = os.path.join(tdir, fn)
                    with open(os.path.join(odir, os.path.basename(fn)), 'w') as f:
                        f.write(csv_subset(src, fev))
        bkdir = os.path.join(tdir, 'bk')
        if os.path.isdir(bkdir):
            os.makedirs(os.path.join(odir, 'bk'), exist_ok=True)
            for fn in os.listdir(bkdir):
                shutil.copy(os.path.join(bkdir, fn), os.path.join(odir, 'bk', fn))
        with open(os.path.join(tdir, 'reference', name + '.log')) as f:
            parsed = parse_log(f.read())
        with open(os.path.join(tdir, 'test')) as f:
            parsed['runtest_filter'] = filters(f.read())
        with open(os.path.join(odir, 'expected.json'), 'w') as f:
            json.dump(parsed, f, indent=0)
        print(name, len(parsed['results']), 'results,', len(parsed['tables']), 'tables,',
              len(parsed['gmres']), 'traces', 'matrix' if 'matrix_real' in parsed else '')


# analysis step (post-processing) of the reference: test name -> (cube file
# suffix, quantity, polarisation index of the .freq block, frequency label)
ANALYSIS = {
    'analysis_field_3d_x_wfq_sodium': ('-Ex-1.5800000000.cube', 'field', 0, '1.5800000000'),
    'analysis_field_3d_x_y_z_wfqfmu_ag': ('-Ez-3.0000000000.cube', 'field', 2, '3.0000000000'),
    'analysis_density_3d_x_wfq_sodium': ('-Ex-1.5800000000-densityRe.cube', 'density_re', 0, '1.5800000000'),
    'analysis_field_3d_y_bem': ('-Ey-1.9100000000.cube', 'field', 1, '1.9100000000'),
}


def one_analysis(name, ref, stride=5):
    """Inputs (geometry, widths, the solution of one polarisation) and a strided
    sample of the reference's output cube for one analysis test."""
    import tarfile
    suffix, what, pol, flabel = ANALYSIS[name]
    tdir = os.path.join(ref, 'tests', name)
    with tempfile.TemporaryDirectory() as work:
        with tarfile.open(os.path.join(tdir, name + '.tar.gz')) as tf:
            tf.extractall(work)
        with open(os.path.join(work, name + '.info')) as f:
            info = f.read().splitlines()
        with open(os.path.join(work, '%s-%s.freq' % (name, flabel))) as f:
            freq = f.read().splitlines()
    model = info[5].split(':')[1].strip()
    e0 = float(info[7].split(':')[1])
    g0 = info.index('Input Geometry (angstrom)') + 1
    if model == 'bem':
        # tessera centres (i8, 3 f25.16); the cube lists them as atoms 0
        n_atoms = int(info[2].split(':')[1])
        coords = [[float(v) for v in l.split()[1:4]] for l in info[g0:g0 + n_atoms]]
        zs = [0] * n_atoms
        rq = rmu = 0.0
    else:
        n_atoms = int(info[0].split(':')[1])
        coords = [[float(v) for v in l.split()[2:5]] for l in info[g0:g0 + n_atoms]]
        zs = [int(float(l.split()[0])) for l in info[g0:g0 + n_atoms]]
        p0 = next(i for i, l in enumerate(info) if l.startswith('Parameters:'))
        par = [float(v) for v in info[p0 + 2].split()[1:]]
        rq = par[2] if model == 'wfq' else par[3]
        rmu = par[4] if model == 'wfqfmu' else 0.0
    heads = [i for i, l in enumerate(freq) if l.startswith('complex')]
    rows = freq[heads[pol] + 1:(heads[pol + 1] if pol + 1 < len(heads) else len(freq))]
    x = [[float(l.split()[1]), float(l.split()[2])] for l in rows if l.strip()]
    with open(os.path.join(tdir, 'reference', 'post_process_' + name, name + suffix)) as f:
        cube = f.read().splitlines()
    dims = [int(cube[3 + k].split()[0]) for k in range(3)]
    vals = [float(v) for l in cube[6 + n_atoms:] for v in l.split()]
    assert len(vals) == dims[0] * dims[1] * dims[2]
    idx = list(range(0, len(vals), stride))
    # the cube header after its title line, and the analysis log's grid block and
    # the maximum lines of this polarisation
    cube_head = cube[2:6 + n_atoms]
    logs = [f for f in os.listdir(os.path.join(tdir, 'reference', 'post_process_' + name)) if f.endswith('.log')]
    with open(os.path.join(tdir, 'reference', 'post_process_' + name, logs[0])) as f:
        log = f.read().splitlines()
    g = log.index(next(l for l in log if 'Grid Information (Angstrom)' in l))
    log_grid = log[g:g + 10]
    log_max = []
    for k, l in enumerate(log):
        if l.startswith('   E' + 'xyz'[pol] + ' ') and k > 0 and 'Max.' in log[k - 1]:
            log_max += [log[k - 1], l]
    out_extra = {'cube_head': cube_head, 'log_grid': log_grid, 'log_max': log_max}
    out = {'name': name, 'model': model, 'e0': e0, 'coords_ang': coords, 'z': zs, 'rq': rq, 'rmu': rmu,
           'pol': pol, 'quantity': what, 'x': x, 'n': dims, 'offset_ang': 10.0,
           'cube_origin_bohr': [float(v) for v in cube[2].split()[1:4]],
           'cube_step_bohr': [float(cube[3 + k].split()[1 + k]) for k in range(3)],
           'sample_index': idx, 'sample_value': [vals[i] for i in idx]}
    out.update(out_extra)
    odir = os.path.join(HERE, name)
    os.makedirs(odir, exist_ok=True)
    with open(os.path.join(odir, 'analysis.json'), 'w') as f:
        json.dump(out, f)
    print(name, n_atoms, 'atoms', len(x), 'unknowns', len(idx), 'cube samples')


STATIC = ['fq_energy', 'fq_polarizability', 'fq_principal_axis_energy', 'fqfmu_energy', 'fqfmu_rq_rmu_energy']


def parse_matrix(text, title):
    """Entries {"r,c": value} of a matrix printed by print_matrix under `title`."""
    i = text.find(title)
    if i < 0:
        return None
    lines = text[i:].splitlines()[2:]
    entries, cols, seen = {}, None, False
    for line in lines:
        if line.startswith(' ---'):
            if seen:
                break
            continue
        toks = line.split()
        if not toks:
            continue
        if all(re.fullmatch(r'\d+', t) for t in toks):
            cols = [int(t) for t in toks]
            continue
        if cols and re.fullmatch(r'\d+', toks[0]):
            seen = True
            for c, v in zip(cols, toks[1:]):
                entries['%s,%d' % (toks[0], c)] = float(v.replace('D', 'E'))
    return entries


def parse_table(text, title, width):
    """Rows [index, values...] of a charges / dipoles / RHS table."""
    i = text.find(title)
    if i < 0:
        return None
    rows = []
    for line in text[i:].splitlines()[1:]:
        if line.startswith(' ---') or line.startswith(' ChErr'):
            break
        toks = line.split()
        if len(toks) == width + 1 and re.fullmatch(r'\d+', toks[0]):
            rows.append([float(v.replace('D', 'E')) for v in toks[1:]])
    return rows


def one_static(name, ref):
    tdir = os.path.join(ref, 'tests', name)
    yamls = [f for f in os.listdir(tdir) if f.endswith('.yaml')]
    with tempfile.TemporaryDirectory() as work:
        kw = run_front_end(ref, tdir, yamls[0], work)
    odir = os.path.join(HERE, name)
    os.makedirs(odir, exist_ok=True)
    with open(os.path.join(odir, 'input.kw'), 'w') as f:
        f.write(kw)
    with open(os.path.join(tdir, 'reference', name + '.log')) as f:
        text = f.read()
    static = 'static response' in kw
    width = 3 if static else 1
    out = {'what': 'static' if static else 'energy'}
    for key, title in (('matrix', ' FQ Matrix\n'), ('matrix', ' FQFMu Matrix\n'), ('j_inverse', ' JMatrix-1\n'),
                       ('j_1_1', ' J_1_1 in calculate_static_polar\n'), ('polar', ' polarizability tensor (a.u.)\n')):
        m = parse_matrix(text, title)
        if m is not None:
            out[key] = m
    for key, title in (('rhs', ' RHS \n'), ('charges', ' Charges \n'), ('dipoles', ' Dipoles \n')):
        t = parse_table(text, title, width)
        if t is not None:
            out[key] = t
    m = re.search(r'ChErr\s+((?:' + NUM + r'\s+)+)', text)
    if m:
        out['charge_err'] = [float(v.replace('D', 'E')) for v in m.group(1).split()]
    m = re.search(r'Energy =\s+(' + NUM + ')', text)
    if m:
        out['energy'] = float(m.group(1))
    m = re.search(r'Polar Iso  =\s+(' + NUM + ')', text)
    if m:
        out['polar_iso'] = float(m.group(1))
    i = text.find('Rotated Geometry (Ang)')
    if i >= 0:
        out['rotated'] = [[float(v) for v in l.split()[2:5]] for l in text[i:].splitlines()[5:]
                          if re.match(r'^\s+\d+\s+\S+\s+' + NUM, l)]
    with open(os.path.join(tdir, 'test')) as f:
        out['runtest_filter'] = filters(f.read())
    with open(os.path.join(odir, 'expected.json'), 'w') as f:
        json.dump(out, f, indent=0)
    print(name, sorted(out))


INFO = {'analysis_field_3d_x_wfq_sodium': ['analysis_field_3d_x_wfq_sodium.info'],
        'analysis_field_3d_x_y_z_wfqfmu_ag': ['analysis_field_3d_x_y_z_wfqfmu_ag.info',
                                              'analysis_field_3d_x_y_z_wfqfmu_ag-3.0000000000.freq'],
        'analysis_pqr_bem': ['analysis_pqr_bem.info']}


def copy_info(ref):
    import tarfile
    odir = os.path.join(HERE, 'info')
    os.makedirs(odir, exist_ok=True)
    for name, members in INFO.items():
        with tarfile.open(os.path.join(ref, 'tests', name, name + '.tar.gz')) as tf:
            for m in members:
                with open(os.path.join(odir, m), 'wb') as f:
                    f.write(tf.extractfile(m).read())
                print('info/' + m)


# every grid-producing analysis test the reference has beyond the three cube
# tests above: planes (one or several), user-bounded planes and slabs, the
# binary .plt format, wFQFMu densities, BEM planes
ANALYSIS_GRIDS = [
    'analysis_field_2d_x_yz_wfq_sodium', 'analysis_density_2d_x_wfq_sodium',
    'analysis_density_2d_x_wfq_sodium_n_planes', 'analysis_density_2d_y_xy_wfqfmu_ag',
    'analysis_field_2d_y_xy_bem', 'analysis_field_2d_z_xz_wfqfmu_ag', 'analysis_field_2d_z_xz_wfqfmu_ag_reduced',
    'analysis_field_volume_x_wfq_sodium', 'analysis_field_volume_z_wfqfmu_au',
    'analysis_field_3d_x_wfq_sodium_plt', 'analysis_density_3d_x_wfq_sodium_plt',
    'analysis_field_3d_x_y_z_wfqfmu_ag_plt', 'analysis_density_3d_y_wfqfmu_au', 'analysis_density_3d_y_wfqfmu_au_plt',
]


def _analysis_options(test_text):
    """The analysis command line of a reference test: its options as a dict."""
    line = re.search(r"input_files=\['[^ ]+ (.*?)'\]", test_text).group(1)
    toks = line.replace('=', ' ').split()
    opts, k = {}, 0
    while k < len(toks):
        key = toks[k].lstrip('-')
        if k + 1 < len(toks) and not re.fullmatch(r'-[a-z_]+', toks[k + 1]):
            opts[key] = toks[k + 1]
            k += 2
        else:
            opts[key] = True
            k += 1
    return opts


def one_analysis_grid(name, ref, max_lines=150):
    """Inputs and sampled outputs of one grid analysis test (``analysis_grids/<name>.json``)."""
    import struct
    import tarfile
    sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
    from plasmonx_b200 import outputs as O
    tdir = os.path.join(ref, 'tests', name)
    opts = _analysis_options(open(os.path.join(tdir, 'test')).read())
    label = O.fortran_f(float(opts['freq']), 12, 10).strip()
    with tarfile.open(os.path.join(tdir, name + '.tar.gz')) as tf:
        info = O.read_info(tf.extractfile(name + '.info').read().decode())
        _, _, blocks = O.read_freq(tf.extractfile('%s-%s.freq' % (name, label)).read().decode())
    pols = list(opts['field_dir']) if 'field_dir' in opts else ['x', 'y', 'z']
    bem = info['model'] == 'bem'
    out = {'name': name, 'model': info['model'], 'e0': info['e0'], 'what': opts['w'], 'label': label,
           'pols': pols, 'options': {k: v for k, v in opts.items() if k not in ('w', 'n', 'freq')},
           'x': {p: [[float(v.real), float(v.imag)] for v in blocks[p]] for p in pols}}
    if bem:
        out['centres_ang'] = info['centres_ang'].tolist()
    else:
        par = info['types'][0][1]
        out.update(coords_ang=info['coord_ang'].tolist(), z=[int(v) for v in info['z']],
                   rq=par[2] if info['model'] == 'wfq' else par[3], rmu=par[4] if info['model'] == 'wfqfmu' else 0.0)
    post = os.path.join(tdir, 'reference', 'post_process_' + name)
    log = open(os.path.join(post, name + '_analysis.log')).read().splitlines()
    g = next(i for i, l in enumerate(log) if 'Grid Information (Angstrom)' in l)
    out['log_grid'] = log[g:g + 10]
    out['log_max'] = [log[i:i + 2] for i, l in enumerate(log) if 'Max.' in l and not l.startswith(' Max. Freq')]
    v = [i for i, l in enumerate(log) if 'Calculation of effective volume' in l]
    out['volume_lines'] = [log[i:i + 5] for i in v]
    files = {}
    for fn in sorted(os.listdir(post)) + sorted(os.path.join('planes', d, f) for d in
                                                (os.listdir(os.path.join(post, 'planes'))
                                                 if os.path.isdir(os.path.join(post, 'planes')) else [])
                                                for f in os.listdir(os.path.join(post, 'planes', d))):
        path = os.path.join(post, fn)
        if fn.endswith('.csv') or fn.endswith('.cube'):
            lines = open(path).read().splitlines()
            idx = list(range(0, len(lines), max(1, len(lines) // max_lines)))
            files[os.path.basename(fn)] = {'n_lines': len(lines), 'index': idx, 'lines': [lines[i] for i in idx]}
        elif fn.endswith('.plt'):
            data = open(path, 'rb').read()
            vals = struct.unpack('<%df' % ((len(data) - 44) // 4), data[44:])
            idx = list(range(0, len(vals), max(1, len(vals) // max_lines)))
            files[os.path.basename(fn)] = {'bytes': len(data), 'head_i': list(struct.unpack('<5i', data[:20])),
                                           'head_f': list(struct.unpack('<6f', data[20:44])), 'index': idx,
                                           'values': [vals[i] for i in idx]}
    out['files'] = files
    odir = os.path.join(HERE, 'analysis_grids')
    os.makedirs(odir, exist_ok=True)
    with open(os.path.join(odir, name + '.json'), 'w') as f:
        json.dump(out, f)
    print('analysis_grids/' + name, sorted(files))


def pqr_xyz(ref, stride=4):
    """Sampled lines of the reference's .pqr and .xyz outputs with the .info / .freq
    values each line is written from (``analysis_extra/pqr_xyz.json``)."""
    import glob
    import tarfile
    sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
    from plasmonx_b200 import outputs as O
    cases = []
    for name, label in (('analysis_pqr_wfq_sodium', '1.5800000000'), ('analysis_pqr_bem', '1.9100000000')):
        with tarfile.open(os.path.join(ref, 'tests', name, name + '.tar.gz')) as tf:
            info = O.read_info(tf.extractfile(name + '.info').read().decode())
            _, _, blocks = O.read_freq(tf.extractfile('%s-%s.freq' % (name, label)).read().decode())
        bem = info['model'] == 'bem'
        pos = info['centres_ang'] if bem else info['coord_ang']
        for pol, part in (('x', 'Re'), ('z', 'Im')):
            f = glob.glob(os.path.join(ref, 'tests', name, 'reference', '*', '%s-E%s-%s-%s.pqr' % (name, pol, label,
                                                                                                  part)))[0]
            lines = open(f).read().splitlines()
            vals = blocks[pol].real if part == 'Re' else blocks[pol].imag
            idx = list(range(0, len(lines), stride))
            cases.append({'kind': 'pqr', 'name': name, 'bem': bem, 'index': idx, 'lines': [lines[i] for i in idx],
                          'pos': [list(pos[i]) for i in idx], 'value': [float(vals[i]) for i in idx],
                          'z': [0 if bem else int(info['z'][i]) for i in idx]})
    for name in ('analysis_xyz', 'analysis_xyz_bem'):
        with tarfile.open(os.path.join(ref, 'tests', name, name + '.tar.gz')) as tf:
            mem = [m for m in tf.getnames() if m.endswith('.info')][0]
            info = O.read_info(tf.extractfile(mem).read().decode())
        bem = info['model'] == 'bem'
        pos = info['centres_ang'] if bem else info['coord_ang']
        lines = open(glob.glob(os.path.join(ref, 'tests', name, 'reference', '*', '*.xyz'))[0]).read().splitlines()
        idx = list(range(0, len(pos), stride))
        cases.append({'kind': 'xyz', 'name': name, 'bem': bem, 'head': lines[:2], 'n': len(pos), 'index': idx,
                      'lines': [lines[2 + i] for i in idx], 'pos': [list(pos[i]) for i in idx],
                      'z': [0 if bem else int(info['z'][i]) for i in idx]})
    odir = os.path.join(HERE, 'analysis_extra')
    os.makedirs(odir, exist_ok=True)
    with open(os.path.join(odir, 'pqr_xyz.json'), 'w') as f:
        json.dump(cases, f)
    print('analysis_extra/pqr_xyz.json', len(cases), 'cases')


if __name__ == '__main__':
    if len(sys.argv) > 2 and sys.argv[1] == '--analysis-grids':
        for nm in ANALYSIS_GRIDS:
            one_analysis_grid(nm, sys.argv[2])
        sys.exit(0)
    if len(sys.argv) > 2 and sys.argv[1] == '--pqr-xyz':
        pqr_xyz(sys.argv[2])
        sys.exit(0)
    if len(sys.argv) > 2 and sys.argv[1] == '--info':
        copy_info(sys.argv[2])
        sys.exit(0)
    if len(sys.argv) > 2 and sys.argv[1] == '--static':
        import subprocess
        for nm in STATIC:
            subprocess.run([sys.executable, os.path.abspath(__file__), '--one-static', nm, sys.argv[2]],
                           check=True, stderr=subprocess.DEVNULL)
        sys.exit(0)
    if len(sys.argv) > 3 and sys.argv[1] == '--one-static':
        one_static(sys.argv[2], sys.argv[3])
        sys.exit(0)
    if len(sys.argv) > 2 and sys.argv[1] == '--analysis':
        for nm in ANALYSIS:
            one_analysis(nm, sys.argv[2])
        sys.exit(0)
    if len(sys.argv) > 2 and sys.argv[1] == '--geom':
        import subprocess
        for nm in GEOM_TESTS:
            subprocess.run([sys.executable, os.path.abspath(__file__), '--one', nm, sys.argv[2]], check=True,
                           stderr=subprocess.DEVNULL)
        sys.exit(0)
    if len(sys.argv) > 2 and sys.argv[1] == '--one':
        one(sys.argv[2], sys.argv[3])
    else:
        tree = sys.argv[1] if len(sys.argv) > 1 else os.environ.get('PLASMONX_REFERENCE')
        if not tree:
            sys.exit('usage: make_golden.py /path/to/plasmonX  (or set PLASMONX_REFERENCE)')
        main(tree)
