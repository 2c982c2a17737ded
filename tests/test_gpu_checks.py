"""The self-checking build on the GPU: the uneven-walker Dimer (the call sequence of both
earlier out-of-bounds incidents: three-image batch, list reuse, work queues), and the ionic
force path through both its kernels, run on libakmc_b200_checks.so in a child process; no
index check may fire.  The checks record and skip; nothing traps."""
import json
import os
import subprocess
import sys

import pytest

from akmc_b200 import build

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_no_index_check_fires(gpu):
    path = build.build(checks=True)
    env = dict(os.environ, AKMC_LIB=path)
    r = subprocess.run([sys.executable, os.path.join(ROOT, "tests", "checks_scenario.py")], env=env,
                       capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stderr[-3000:]
    out = json.loads(r.stdout.strip().splitlines()[-1])
    assert out["dimer_converged"] > 80
    assert out["ionic_5_status"] == 0 and out["ionic_8_status"] == 0
    fired = {(f, c): (out["hits"][32 * f + c], out["first"][32 * f + c])
             for f in range(3) for c in range(32) if out["hits"][32 * f + c]}
    assert not fired, fired
