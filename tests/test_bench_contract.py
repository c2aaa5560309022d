"""The reference arm of bench.py runs on the host (the reference's algorithm on the
CPU cores) and prints the one JSON line the harness reads; checked here on CPU with a
minimal sample (one step, one on-the-fly product)."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_prints_the_contract_line():
    out = subprocess.run([sys.executable, os.path.join(ROOT, 'bench.py'), '--impl', 'reference', '--steps', '1',
                          '--warmup', '1', '--cpu-matvecs', '1'], capture_output=True, text=True, timeout=600,
                         cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.strip().startswith('{')]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in ('metric', 'value', 'unit', 'n_gpus', 'steps', 'warmup', 'ms_per_step', 'higher_is_better', 'scaling',
              'vs_baseline', 'dtype', 'data', 'config', 'cpu_baseline', 'e2e'):
        assert k in d, k
    sys.path.insert(0, ROOT)
    import bench
    assert d['impl'] == 'reference' and d['metric'] == bench.METRIC
    assert d['n_gpus'] == 1 and d['steps'] == 1 and d['warmup'] == 1 and d['higher_is_better'] is True
    assert d['value'] > 0 and d['cpu_baseline']['value'] == d['value']
    assert d['cpu_baseline']['kind'] == 'port' and d['cpu_baseline']['cores'] >= 1
    assert d['e2e'] == {'value': d['value'], 'unit': d['unit'], 'h2d_bytes_per_step': 0, 'd2h_bytes_per_step': 0}
    assert d['config']['n_var'] == 41892


def test_static_reference_arm_prints_the_contract_line():
    """The static workload's reference arm: the oracle's solve of a small water cluster."""
    out = subprocess.run([sys.executable, os.path.join(ROOT, 'bench.py'), '--impl', 'reference', '--config',
                          'fq_water', '--waters', '40', '--steps', '1', '--warmup', '0'], capture_output=True,
                         text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.strip().startswith('{')]
    assert len(lines) == 1
    d = json.loads(lines[0])
    sys.path.insert(0, ROOT)
    import bench
    assert d['impl'] == 'reference' and d['metric'] == bench.STATIC_METRIC and d['unit'] == 'solves/s'
    assert d['config']['n_var'] == 160 and d['value'] > 0
    assert d['e2e']['h2d_bytes_per_step'] == 0 and d['cpu_baseline']['kind'] == 'port'


def test_field_grid_reference_arm_prints_the_contract_line():
    """The analysis workload's reference arm: the oracle's field and density on a
    bounded sample of a small grid."""
    out = subprocess.run([sys.executable, os.path.join(ROOT, 'bench.py'), '--impl', 'reference', '--config',
                          'field_grid', '--radius', '8', '--grid', '12', '--steps', '1', '--warmup', '0'],
                         capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.strip().startswith('{')]
    assert len(lines) == 1
    d = json.loads(lines[0])
    sys.path.insert(0, ROOT)
    import bench
    assert d['impl'] == 'reference' and d['metric'] == bench.POINTS_METRIC and d['unit'] == 'points/s'
    assert d['config']['n_points'] == 12 ** 3 and d['value'] > 0
    assert d['e2e']['h2d_bytes_per_step'] == 0 and d['cpu_baseline']['kind'] == 'port'


def test_inversion_reference_arm_times_the_lu():
    """Config 1 in inversion mode: the reference arm times a complex LU and its
    three solves per frequency (zgetrf / zgetrs), not GMRES products."""
    out = subprocess.run([sys.executable, os.path.join(ROOT, 'bench.py'), '--impl', 'reference', '--config',
                          'na_sphere', '--mode', 'inversion', '--steps', '1', '--warmup', '0'], capture_output=True,
                         text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.strip().startswith('{')]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d['impl'] == 'reference' and d['config']['mode'] == 'inversion' and d['value'] > 0
    assert 'LU' in d['cpu_baseline']['sample'] and d['cpu_baseline']['steps_per_solve'] is None
    assert d['e2e']['h2d_bytes_per_step'] == 0


def test_serving_reference_arm_reports_unavailable():
    out = subprocess.run([sys.executable, os.path.join(ROOT, 'bench.py'), '--impl', 'reference', '--config',
                          'serving'], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    d = json.loads([l for l in out.stdout.splitlines() if l.strip().startswith('{')][-1])
    assert d['impl'] == 'reference' and 'unavailable' in d


def test_contraction_roofline_names_the_binding_resource():
    sys.path.insert(0, ROOT)
    import bench
    # one product, few columns: 3.5 GB streamed in 0.95 ms, 0.19 PFLOP issued
    roof = {'bound': 'tensor', 'achieved': 200.0, 'peak': 1400.0, 'unit': 'TFLOP/s', 'avg_launch_ms': 0.95,
            'bytes_per_launch': 3.5e9, 'issued_tensor_tflops': 200.0, 'achieved_hbm_gbs': 3.5e9 / 0.95e-3 / 1e9}
    r = bench.contraction_bound(dict(roof), 6650.0)
    assert r['binding'] == 'hbm' and r['bound'] == 'hbm' and r['unit'] == 'GB/s' and r['peak'] == 6650.0
    assert abs(r['frac'] - r['achieved'] / 6650.0) < 1e-12 and r['achieved_algorithmic_tflops'] == 200.0
    assert abs(r['bound_frac'] - (3.5e9 / 6650e9 * 1e3) / 0.95) < 1e-12
    # three products, many columns: the tensor issue binds and the line stays in TFLOP/s
    roof.update(issued_tensor_tflops=1000.0, avg_launch_ms=1.9, bytes_per_launch=7.0e9,
                achieved_hbm_gbs=7.0e9 / 1.9e-3 / 1e9, achieved=333.0)
    r = bench.contraction_bound(dict(roof), 6650.0)
    assert r['binding'] == 'tensor issue' and r['bound'] == 'tensor' and r['unit'] == 'TFLOP/s'
    assert r['achieved'] == 333.0 and r['peak'] == 1400.0
