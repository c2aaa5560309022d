"""Minimal, independent reader of the reference keyword file (test oracle).

The reference's Python front end (``python/input_/io_operations.py:264-513``)
turns a YAML input into ``key: value`` lines that the Fortran executable reads
(``src/input_output/input_module.f90:156-258``, ``:680-1000``).  This reader
follows that Fortran parser: repeated ``atom_types name`` / ``parameters
atomtype name`` lines open a new block, ``parameters interaction name: A->B``
addresses the (A, B) entry of the Fermi d/s matrices, and the geometry follows
the ``input_geometry`` line as ``name imol x y z`` (Angstrom).
"""
TO_BOHR = 1.8897261254578281
AU_TO_EV = 27.211386245981


def _val(v):
    v = v.strip()
    try:
        return float(v.replace('d', 'e').replace('D', 'e'))
    except ValueError:
        return v


def read_keyword_text(text):
    lines = text.splitlines()
    kw = {}
    atomtypes, params, inter = [], [], []
    geom = []
    i_geom = None
    for idx, line in enumerate(lines):
        if line.startswith('input_geometry'):
            i_geom = idx
            break
        if not line.strip() or line.lstrip().startswith('#'):
            continue
        key, _, value = line.partition(':')
        key = key.strip()
        value = value.strip()
        if key == 'atom_types name':
            atomtypes.append({'name': value})
        elif key.startswith('atom_types ') and key != 'atom_types number':
            atomtypes[-1][key[len('atom_types '):]] = _val(value)
        elif key == 'parameters atomtype name':
            params.append({'name': value})
        elif key.startswith('parameters atomtype '):
            params[-1][key[len('parameters atomtype '):]] = _val(value)
        elif key == 'parameters interaction name':
            a, b = value.split('->')
            inter.append({'pair': (a.strip(), b.strip())})
        elif key.startswith('parameters interaction '):
            inter[-1][key[len('parameters interaction '):]] = _val(value)
        else:
            kw[key] = value
    if i_geom is not None:
        n = int(float(kw.get('number of atoms', 0)))
        for line in lines[i_geom + 1:i_geom + 1 + n]:
            p = line.split()
            geom.append((p[0], float(p[2]), float(p[3]), float(p[4])))
    return kw, atomtypes, params, inter, geom


def read_keyword_file(path):
    with open(path) as f:
        return read_keyword_text(f.read())
