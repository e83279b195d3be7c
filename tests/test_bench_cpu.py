"""
The bench.py JSON contract on the CPU: the reference arm (the reference package's own Solution on its torch-CPU
backend, or the numpy oracle where the package is absent) prints one line with the contract's keys, and under
torchrun with two ranks only rank 0 prints it while the other exits 0.
"""
import json
import os
import socket
import subprocess
import sys

from conftest import ROOT

KEYS = {'impl', 'metric', 'value', 'unit', 'n_gpus', 'steps', 'warmup', 'ms_per_step', 'higher_is_better', 'scaling',
        'vs_baseline', 'dtype', 'data', 'config', 'cpu_baseline', 'e2e'}
ARGS = ['--impl', 'reference', '--workload', 'spheres3d', '--size', '32', '--steps', '2', '--warmup', '3']


def _json_lines(out: str):
    return [json.loads(l) for l in out.splitlines() if l.startswith('{')]


def _reference_arm(env=None):
    r = subprocess.run([sys.executable, 'bench.py', *ARGS], cwd=ROOT, capture_output=True, text=True, timeout=240,
                       env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = _json_lines(r.stdout)
    assert len(lines) == 1
    d = lines[0]
    assert KEYS <= set(d)
    assert d['impl'] == 'reference' and d['n_gpus'] == 1 and d['steps'] == 2 and d['warmup'] == 3
    assert d['unit'] == 'voxel-it/s' and d['higher_is_better'] is True and d['value'] > 0
    assert d['config']['grid'] == [32, 32, 32] and d['config']['components'] == 3
    assert d['config']['parallelism'] == 'replicas x1'  # the same config dict as the device arm's line
    assert d['cpu_baseline']['value'] == d['value']
    assert d['e2e'] == {'value': d['value'], 'unit': d['unit'], 'h2d_bytes_per_step': 0, 'd2h_bytes_per_step': 0}
    return d


def test_reference_arm_prints_the_contract_line():
    from oracle.refimport import reference_available
    d = _reference_arm()
    # the reference package's own Solution where it is present, else the numpy restatement
    assert d['cpu_baseline']['kind'] == ('reference' if reference_available() else 'port')


def test_reference_arm_falls_back_to_the_oracle_without_the_package():
    d = _reference_arm(dict(os.environ, MACROMAX_REFERENCE=os.path.join(ROOT, 'no-such-directory')))
    assert d['cpu_baseline']['kind'] == 'port'


def test_reference_arm_under_torchrun_prints_once():
    with socket.socket() as s:
        s.bind(('127.0.0.1', 0))
        port = s.getsockname()[1]
    cmd = [sys.executable, '-m', 'torch.distributed.run', '--nnodes=1', '--nproc-per-node', '2', '--master-addr',
           '127.0.0.1', '--master-port', str(port), 'bench.py', '--gpus', '2', *ARGS]
    env = dict(os.environ, OMP_NUM_THREADS='2')
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=300, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = _json_lines(r.stdout)
    assert len(lines) == 1 and lines[0]['impl'] == 'reference' and lines[0]['n_gpus'] == 2
    assert lines[0]['config']['parallelism'] == 'replicas x2'
