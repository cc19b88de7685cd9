"""CPU: the recorded solves flagged as rounding-sensitive really are.

``tests/golden/reference_calls_sensitive.json`` lists the recorded solver calls
whose oracle result changes when the in-loop chemical-potential sums are taken
exactly instead of in NumPy's pairwise order (utils.hpp:79-116 branches on the
sign of a rounding-level residual).  Both results are re-derived here from the
recorded arguments, so the GPU replay's wider acceptance for those calls rests
on the reference's own arithmetic, not on a list.
"""

from __future__ import annotations

import gzip
import importlib.util
import json
import pickle

import pytest

from conftest import GOLDEN

_CALLS = GOLDEN / "reference_calls.pkl.gz"
_SENS = GOLDEN / "reference_calls_sensitive.json"


def _maker():
    spec = importlib.util.spec_from_file_location("make_reference_sensitivity",
                                                  GOLDEN / "make_reference_sensitivity.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


@pytest.mark.skipif(not (_CALLS.exists() and _SENS.exists()), reason="fixtures absent")
def test_sensitive_calls_change_with_exact_mu_sums():
    calls = pickle.load(gzip.open(_CALLS))["calls"]
    sens = json.loads(_SENS.read_text())["calls"]
    assert sens, "no sensitive calls recorded"
    mk = _maker()
    for key, rec in sens.items():
        c = calls[int(key)]
        assert c["name"] == rec["name"]
        it0, e0 = mk.recorded(c)
        it1, e1 = mk.rerun_exact(c)
        assert [it0, it1] == rec["iterations"]
        assert [e0, e1] == pytest.approx(rec["energy"], rel=1e-12, abs=1e-14)
        assert it0 != it1 or abs(e0 - e1) > 1e-12 * max(1.0, abs(e0))


@pytest.mark.skipif(not _CALLS.exists(), reason="fixture absent")
def test_insensitive_call_is_unchanged_with_exact_mu_sums():
    """A recorded solve not in the list (4 x 4 mesh, cold start) keeps its result."""
    calls = pickle.load(gzip.open(_CALLS))["calls"]
    sens = json.loads(_SENS.read_text())["calls"] if _SENS.exists() else {}
    assert "19" not in sens
    mk = _maker()
    c = calls[19]
    assert mk.rerun_exact(c) == mk.recorded(c)
