"""Record the reference's own test suite's calls into its native module.

Run where a checkout of the reference is present, its root directory given by
the ``CPPHF_REFERENCE`` environment variable (required, no default):

    CPPHF_REFERENCE=<reference checkout> python tests/golden/make_reference_calls.py

The reference's pytest suite runs with the oracle (``oracle/native_np.py``)
installed as ``cpp_hf._native`` through the recording plugin
``oracle/_record_native.py``; every call the suite's Python layer and tests
make (function, arguments, the oracle's result) is written to
``tests/golden/reference_calls.pkl.gz``.  ``tests/test_gpu_reference_calls.py``
replays them through the B200 module, so the reference's tests exercise the
GPU path without the reference being present where the GPU is.
"""

from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]


def main() -> int:
    root = os.environ.get("CPPHF_REFERENCE")
    if not root:
        raise SystemExit("set CPPHF_REFERENCE to the root of a cpp_hf checkout")
    ref = Path(root)
    env = dict(os.environ)
    env["PYTHONPATH"] = os.pathsep.join([str(REPO), str(ref / "src"), env.get("PYTHONPATH", "")])
    env["PYTHONDONTWRITEBYTECODE"] = "1"
    env["CPPHF_RECORD_OUT"] = str(HERE / "reference_calls.pkl.gz")
    cmd = [sys.executable, "-m", "pytest", str(ref / "tests"), "-q", "-p", "no:cacheprovider",
           "-p", "oracle._record_native", "--rootdir", str(ref / "tests")]
    return subprocess.call(cmd, env=env, cwd=str(REPO))


if __name__ == "__main__":
    sys.exit(main())
