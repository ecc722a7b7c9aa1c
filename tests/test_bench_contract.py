"""bench.py on the host: the reference arm prints one JSON line per workload,
an explicit `unavailable` line where nAPMO has no counterpart, and the
numerical-orbital reference sample restates nAPMO's operators."""
import json
import os
import subprocess
import sys

import pytest

from conftest import ROOT


def _run(*args):
    out = subprocess.run([sys.executable, os.path.join(ROOT, 'bench.py')] + list(args),
                         capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith('{')]
    assert len(lines) == 1, out.stdout
    return json.loads(lines[0])


@pytest.mark.parametrize('workload', ['c3', 'c5'])
def test_reference_arm_unavailable_lines(workload):
    d = _run('--impl', 'reference', '--workload', workload, '--steps', '1', '--warmup', '0')
    assert d['impl'] == 'reference' and d['workload'] == workload and d['unavailable']


def test_reference_arm_c7_line():
    d = _run('--impl', 'reference', '--workload', 'c7', '--steps', '1', '--warmup', '0')
    assert d['impl'] == 'reference' and d['unit'] == 's per S,T,V'
    assert d['higher_is_better'] is False and d['value'] > 0
    assert d['cpu_baseline']['kind'] == 'port' and d['e2e']['value'] == d['value']


def test_reference_arm_c1_times_the_oracle_scf():
    """The C1 host arm runs the oracle's grid SCF (one iteration per step) and
    reports seconds per SCF at the oracle's iteration count."""
    d = _run('--impl', 'reference', '--workload', 'c1', '--steps', '1', '--warmup', '0')
    assert d['impl'] == 'reference' and d['unit'] == 's per SCF'
    assert d['higher_is_better'] is False and d['value'] > 0
    assert d['value'] == pytest.approx(d['ms_per_step'] / 1e3 * d['sample_scale_to_scf'])
    assert d['cpu_baseline']['kind'] == 'port' and d['e2e']['value'] == d['value']
