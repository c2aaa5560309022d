import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, 'tests', 'golden')


def pytest_configure(config):
    config.addinivalue_line('markers', 'gpu: needs a CUDA device (B200, sm_100a)')
    config.addinivalue_line('markers', 'slow: takes more than a few seconds on CPU')


def golden_dirs(kind=None):
    """Fixture directories of one kind: 'atomistic' (wFQ / wFQFMu spectra), 'bem'
    or 'static' (static FQ / FQFMu); None lists them all."""
    out = []
    for d in sorted(os.listdir(GOLDEN)):
        if not os.path.isfile(os.path.join(GOLDEN, d, 'expected.json')):
            continue
        k = 'bem' if d.startswith('bem_') else ('static' if d.startswith('fq') else 'atomistic')
        if kind is None or kind == k:
            out.append(d)
    return out
