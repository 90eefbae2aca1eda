"""The bench's host-side helpers (no GPU): the algorithmic-bytes model of the topology+solve launch,
the measured HBM peak, the clock sampler's summary of nvidia-smi lines (throttle reasons, median
SM clock), the workload description and the CPU baselines on a tiny sample."""

import json
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


def test_alg_bytes_model():
    s = {'dynamic_bodies': 100, 'manifolds': 250, 'contacts': 470, 'adjacency': 500, 'incidences': 940}
    N, M, P, A, P2 = 100, 250, 470, 500, 940
    topo, warm, vel = 24 * M + 16 * A + 32 * N, 144 * N, 88 * N
    primal, dual = 140 * N + 92 * A + 64 * P2, 144 * M + 92 * P
    assert bench.alg_bytes(s) == topo + warm + 10 * (primal + dual) + vel


def test_measured_peak_reads_the_driver_file():
    peak, kind = bench.measured_peak()
    path = os.path.join(ROOT, 'MEASURED_PEAKS.json')
    if os.path.exists(path):
        assert kind == 'measured' and peak == float(json.load(open(path))['hbm_gbs'])
    else:
        assert (peak, kind) == (6650.0, 'fallback')


def test_clock_summary():
    c = bench.ClockSampler(0)
    c.lines = [
        '0, 1965, 1965, 812.50, 0x0000000000000000, Not Active, Not Active, Not Active, Not Active',
        '0, 1950, 1965, 990.10, 0x0000000000000004, Not Active, Not Active, Not Active, Active',
        '0, 1965, 1965, 995.00, 0x0000000000000004, Not Active, Not Active, Not Active, Active',
        'garbage line',
    ]
    s = c.summary()
    assert s == {'sm_mhz': 1965.0, 'sm_max_mhz': 1965.0, 'reasons': ['sw_power_cap'], 'samples': 3}
    c.lines = ['0, 1200, 1965, 500.0, 0x0000000000000008, Active, Not Active, Not Active, Not Active']
    assert c.summary()['reasons'] == ['hw_slowdown']
    c.lines = []
    assert c.summary() == {'sm_mhz': None, 'sm_max_mhz': None, 'reasons': [], 'samples': 0}


def test_workload_config_names_the_pile():
    cfg = bench.workload_config(100_000, 20)
    assert cfg['bodies'] == 100_000 and cfg['iterations'] == 10 and cfg['seed'] == 1 and cfg['window'] == [201, 220]
    assert 'drop pile' in cfg['workload'] and 'rolled 200 steps untimed, timed steps 201..220' in cfg['workload']


def test_cpu_baselines_on_a_tiny_sample():
    r = bench.cpu_reference(60, 5, 3, 2)
    assert r['value'] > 0 and r['unit'] == bench.UNIT and r['cores'] >= 1 and '60 bodies' in r['sample'] and 'steps 6..8' in r['sample']
    u = bench.cpu_upstream_pyramid(2)
    assert u['value'] > 0 and u['cores'] == 1 and 'pyramid' in u['sample'] and 'double' in u['sample']
    f = bench.cpu_upstream_pyramid(2, fp32=True)
    assert f['value'] > 0 and f['cores'] == 1 and 'float' in f['sample']


def test_reference_arm_line():
    """`bench.py --impl reference` prints the contract's line on rank 0, nothing on other ranks."""
    import subprocess
    env = dict(os.environ, RANK='0', WORLD_SIZE='1')
    out = subprocess.run([sys.executable, os.path.join(ROOT, 'bench.py'), '--impl', 'reference', '--steps', '3', '--warmup', '3', '--bodies', '300',
                          '--roll', '20'], capture_output=True, text=True, env=env, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr
    line = json.loads(out.stdout.strip().splitlines()[-1])
    for key in ('metric', 'value', 'unit', 'n_gpus', 'steps', 'warmup', 'ms_per_step', 'higher_is_better', 'scaling', 'vs_baseline', 'dtype',
                'data', 'config', 'impl', 'cpu_baseline', 'e2e'):
        assert key in line, key
    assert line['impl'] == 'reference' and line['metric'] == bench.METRIC and line['steps'] == 3 and line['warmup'] == 3
    assert line['e2e']['h2d_bytes_per_step'] == 0 and line['cpu_baseline']['value'] == line['value']
    assert line['config']['window'] == [21, 23] and line['config']['bodies'] == 300
    env = dict(os.environ, RANK='1', WORLD_SIZE='2')
    out = subprocess.run([sys.executable, os.path.join(ROOT, 'bench.py'), '--impl', 'reference', '--steps', '3', '--warmup', '3'],
                         capture_output=True, text=True, env=env, timeout=600, cwd=ROOT)
    assert out.returncode == 0 and out.stdout.strip() == ''
