"""The drop-in boundary as the reference's own adapters use it (baselines/*/render.py).

tests/golden/adapter_calls.json records, read from the adapters' source, every name they
import from the five renderer packages and every call they make on those names (number of
positional arguments, keyword names). Here each import must resolve to this repository's
package and each call must bind to the signature of the object it reaches (constructor,
``forward`` of an nn.Module called as ``renderer(...)``, ``__call__``, or the method).
When a reference checkout is given in $US3D_REFERENCE, the fixture must also equal what the
adapters say today.
"""

from __future__ import annotations

import importlib
import inspect
import json
import os
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
PKG_ROOT = ROOT / "ultrasound-3d-reconstruction_b200"
FIXTURE = ROOT / "tests" / "golden" / "adapter_calls.json"


def _calls():
    return json.loads(FIXTURE.read_text())


def _target(call):
    mod = importlib.import_module(call["module"])
    obj = getattr(mod, call["name"])
    if call["kind"] == "call":
        return obj
    if call["kind"] == "method":
        return getattr(obj, call["method"])
    import torch.nn as nn

    if inspect.isclass(obj) and issubclass(obj, nn.Module):
        return obj.forward  # renderer(...) runs Module.__call__ -> forward
    return obj.__call__


@pytest.mark.parametrize("adapter", sorted(_calls()))
def test_adapter_imports_resolve_here(adapter):
    for imp in _calls()[adapter]["imports"]:
        mod = importlib.import_module(imp["module"])
        assert Path(mod.__file__).resolve().is_relative_to(PKG_ROOT), (imp, mod.__file__)
        assert hasattr(mod, imp["name"]), imp


@pytest.mark.parametrize("adapter", sorted(_calls()))
def test_adapter_calls_bind(adapter):
    calls = _calls()[adapter]["calls"]
    assert calls, adapter
    for call in calls:
        fn = _target(call)
        sig = inspect.signature(fn)
        positional = [object()] * call["n_positional"]
        if call["kind"] in ("method", "instance_call") and "self" in sig.parameters:
            positional = [object()] + positional
        try:
            sig.bind(*positional, **{k: object() for k in call["keywords"]})
        except TypeError as ex:
            pytest.fail(f"{adapter} line {call['line']}: {call['name']} {call['kind']} does not bind: {ex}")


def test_fixture_matches_reference_adapters():
    ref = os.environ.get("US3D_REFERENCE")
    if not ref or not (Path(ref) / "baselines").is_dir():
        pytest.skip("set US3D_REFERENCE to a reference checkout to re-read its adapters")
    import sys

    sys.path.insert(0, str(ROOT / "tests" / "golden"))
    import make_adapter_calls

    assert make_adapter_calls.collect(Path(ref)) == _calls()
