"""The C ABI library builds, loads and exports every entry point of include/plasmonx_b200.h."""
import os
import re
import subprocess

import pytest

from tests.conftest import ROOT

HEADER = os.path.join(ROOT, 'include', 'plasmonx_b200.h')


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r'/\*.*?\*/', '', text, flags=re.S)
    return sorted(set(re.findall(r'\b(plx_[a-z0-9_]+)\s*\(', text)))


def test_library_builds_and_exports_header_symbols():
    from plasmonx_b200 import build, _lib
    path = build.build()
    out = subprocess.run(['nm', '-D', '--defined-only', path], capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r'\bT (plx_[a-z0-9_]+)', out))
    missing = [f for f in declared_functions() if f not in exported]
    assert not missing, missing
    lib = _lib.load()
    for f in declared_functions():
        assert hasattr(lib, f)
    assert set(_lib.EXPORTS) <= set(declared_functions())


def test_product_has_no_cpu_fallback():
    """The package never imports the oracle and refuses to run without its CUDA library."""
    pkg = os.path.join(ROOT, 'plasmonx_b200')
    for dirpath, _, files in os.walk(pkg):
        for fn in files:
            if fn.endswith('.py'):
                src = open(os.path.join(dirpath, fn)).read()
                assert 'oracle' not in re.sub(r'#.*', '', src).replace('"""', ''), fn


def test_missing_library_raises(monkeypatch, tmp_path):
    from plasmonx_b200 import _lib
    monkeypatch.setattr(_lib, 'LIB_PATH', str(tmp_path / 'nope.so'))
    monkeypatch.setattr(_lib, '_lib', None)
    with pytest.raises(OSError):
        _lib.load()


def test_ctypes_structs_match_the_header_layout(tmp_path):
    """Every descriptor struct of the header has the same size and field offsets in
    C (compiled here with gcc against include/plasmonx_b200.h) as in the ctypes
    binding the Python host side passes."""
    import ctypes as C
    from plasmonx_b200 import _lib
    structs = {'plx_geometry_desc': _lib.GeometryDesc, 'plx_bem_desc': _lib.BemDesc,
               'plx_solve_desc': _lib.SolveDesc, 'plx_static_desc': _lib.StaticDesc}
    src = ['#include <stdio.h>', '#include <stddef.h>', '#include "plasmonx_b200.h"', 'int main(void) {']
    for cname, cls in structs.items():
        src.append('printf("%s sizeof %%zu\\n", sizeof(%s));' % (cname, cname))
        for fname, _ in cls._fields_:
            src.append('printf("%s %s %%zu\\n", offsetof(%s, %s));' % (cname, fname, cname, fname))
    src.append('return 0; }')
    c = tmp_path / 'layout.c'
    c.write_text('\n'.join(src))
    exe = tmp_path / 'layout'
    subprocess.run(['gcc', '-I', os.path.join(ROOT, 'include'), str(c), '-o', str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split('\n')
    got = {tuple(l.split()[:2]): int(l.split()[2]) for l in out if l.strip()}
    for cname, cls in structs.items():
        assert got[(cname, 'sizeof')] == C.sizeof(cls), cname
        for fname, _ in cls._fields_:
            assert got[(cname, fname)] == getattr(cls, fname).offset, (cname, fname)
