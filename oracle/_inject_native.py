"""pytest plugin: install the oracle as ``cpp_hf._native`` before cpp_hf is imported.

Test infrastructure for ``oracle/pin_reference_suite.py`` only.  The reference's
Python layer imports its native module with ``from . import _native``
(``src/cpp_hf/_compat.py:14-20``); pre-seeding ``sys.modules`` makes that import
resolve to the NumPy restatement in ``oracle/native_np.py``.
"""

import sys

from oracle import native_np

sys.modules["cpp_hf._native"] = native_np
