"""GPU parity of the dataflow exchange kernel (one persistent launch for the
three FFT passes, selected with CPPHF_EXCHANGE_FLOW=1).

The library reads the switch once per process, so the exchange parity tests
of test_gpu_parity.py (full / elementwise / scalar / HCP / complex64 / shift,
meshes 1x1 .. 192x192) and the Fock-build tests run again in a child process
with the switch set; shapes the dataflow kernel does not take (non-square,
HCP, lines without a codelet) run the three-launch passes there too.
"""

from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]


def test_exchange_parity_under_dataflow_kernel():
    env = dict(os.environ, CPPHF_EXCHANGE_FLOW="1")
    r = subprocess.run([sys.executable, "-m", "pytest", "-q", "-x", "tests/test_gpu_parity.py", "-k",
                        "exchange or build_fock", "-p", "no:cacheprovider"],
                       cwd=ROOT, env=env, capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout[-4000:] + r.stderr[-2000:]
