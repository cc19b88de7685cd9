"""pytest plugin: run the reference's suite on the oracle and record every call it
makes into ``cpp_hf._native``.

Test infrastructure for ``tests/golden/make_reference_calls.py`` only.  A proxy
module is installed as ``cpp_hf._native`` (the import of
``src/cpp_hf/_compat.py:14-20``); each function forwards to ``oracle.native_np``
and appends (test id, function name, arguments, result) to a list that is
written, pickled and gzip-compressed, to the path in ``CPPHF_RECORD_OUT`` when
the session ends.  Calls that pass a Python callable (a projector callback)
cannot be replayed elsewhere and are counted but not stored.
"""

from __future__ import annotations

import copy
import gzip
import os
import pickle
import sys
import types

import numpy as np

from oracle import native_np

_records: list = []
_skipped = {"callable": 0}
_current = {"test": None}


def _has_callable(x):
    if callable(x) and not isinstance(x, (np.ndarray, type)):
        return True
    if isinstance(x, dict):
        return any(_has_callable(v) for v in x.values())
    if isinstance(x, (list, tuple)):
        return any(_has_callable(v) for v in x)
    return False


def _wrap(name, fn):
    def call(*args, **kwargs):
        record = not (_has_callable(args) or _has_callable(kwargs))
        saved = (copy.deepcopy(args), copy.deepcopy(kwargs)) if record else None
        out = fn(*args, **kwargs)
        if record:
            _records.append({"test": _current["test"], "name": name, "args": saved[0], "kwargs": saved[1],
                             "result": copy.deepcopy(out)})
        else:
            _skipped["callable"] += 1
        return out

    call.__name__ = name
    return call


proxy = types.ModuleType("cpp_hf._native")
for _name in native_np.__all__:
    setattr(proxy, _name, _wrap(_name, getattr(native_np, _name)))
proxy.__all__ = list(native_np.__all__)
sys.modules["cpp_hf._native"] = proxy


def pytest_runtest_setup(item):
    _current["test"] = item.nodeid


def pytest_sessionfinish(session, exitstatus):
    out = os.environ.get("CPPHF_RECORD_OUT")
    if out:
        with gzip.open(out, "wb") as f:
            pickle.dump({"calls": _records, "skipped_callable": _skipped["callable"]}, f, protocol=4)
