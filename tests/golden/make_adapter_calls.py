"""Generates tests/golden/adapter_calls.json: what the reference's five adapters
(baselines/*/render.py) import from the renderer packages and how they call them, read from
their source with ``ast`` (nothing of theirs is imported or run).

For every adapter it records each ``from X import Y`` of a renderer package, and each call
of an imported name or of an object built from one (``renderer = UltraGaussRenderer(cfg)``
then ``renderer(...)``): the callee, whether it constructs or calls an instance, the number
of positional arguments and the keyword names. tests/test_cpu_adapter_boundary.py binds
those calls against this repository's packages.

Usage: python tests/golden/make_adapter_calls.py --reference /path/to/reference
       (default: $US3D_REFERENCE)
"""

from __future__ import annotations

import argparse
import ast
import json
import os
from pathlib import Path

HERE = Path(__file__).resolve().parent
ADAPTERS = ("gaussianpile", "slice_adapted_3dgs", "ultrags_baseline", "ultragauss", "ultragray")
PACKAGES = ("gaussianplie_renderer", "slice_adapted_3dgs_renderer", "ultrags_baseline_renderer",
            "ultragauss_renderer", "ultragray_renderer")


def scan(source: str) -> dict:
    tree = ast.parse(source)
    imports, calls = [], []
    imported = {}  # local name -> (module, name)
    for node in ast.walk(tree):
        if isinstance(node, ast.ImportFrom) and node.module and node.module.split(".")[0] in PACKAGES:
            for a in node.names:
                imports.append({"module": node.module, "name": a.name})
                imported[a.asname or a.name] = (node.module, a.name)
    instances = {}  # variable -> imported class it was built from
    dicts = {}  # variable -> keys of the dict literal assigned to it
    for node in ast.walk(tree):
        if isinstance(node, ast.Assign) and isinstance(node.value, ast.Call):
            f = node.value.func
            if isinstance(f, ast.Name) and f.id in imported:
                for t in node.targets:
                    if isinstance(t, ast.Name):
                        instances[t.id] = f.id
        if isinstance(node, ast.Assign) and isinstance(node.value, ast.Dict):
            if all(isinstance(k, ast.Constant) and isinstance(k.value, str) for k in node.value.keys):
                for t in node.targets:
                    if isinstance(t, ast.Name):
                        dicts[t.id] = [k.value for k in node.value.keys]
    for node in ast.walk(tree):
        if not isinstance(node, ast.Call):
            continue
        method = None
        if isinstance(node.func, ast.Name):
            name = node.func.id
        elif isinstance(node.func, ast.Attribute) and isinstance(node.func.value, ast.Name):
            name, method = node.func.value.id, node.func.attr
            if name not in instances:
                continue
        else:
            continue
        if method is not None:
            kind, target = "method", imported[instances[name]]
        elif name in imported:
            kind, target = "call", imported[name]
        elif name in instances:
            kind, target = "instance_call", imported[instances[name]]
        else:
            continue
        if any(isinstance(a, ast.Starred) for a in node.args):
            raise ValueError(f"line {node.lineno}: *args calls are not recorded")
        keywords = []
        for k in node.keywords:
            if k.arg is not None:
                keywords.append(k.arg)
            elif isinstance(k.value, ast.Name) and k.value.id in dicts:
                keywords += dicts[k.value.id]  # **kwargs of a dict literal: its keys
            else:
                raise ValueError(f"line {node.lineno}: **kwargs of unknown keys")
        calls.append({"module": target[0], "name": target[1], "kind": kind, "method": method, "line": node.lineno,
                      "n_positional": len(node.args), "keywords": keywords})
    return {"imports": imports, "calls": sorted(calls, key=lambda c: c["line"])}


def collect(reference: Path) -> dict:
    return {a: scan((reference / "baselines" / a / "render.py").read_text()) for a in ADAPTERS}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", type=Path, default=os.environ.get("US3D_REFERENCE"),
                    required=not os.environ.get("US3D_REFERENCE"),
                    help="reference checkout (default: $US3D_REFERENCE)")
    ap.add_argument("--out", type=Path, default=HERE / "adapter_calls.json")
    a = ap.parse_args()
    data = collect(Path(a.reference))
    a.out.write_text(json.dumps(data, indent=1, sort_keys=True) + "\n")
    for k, v in data.items():
        print(k, len(v["imports"]), "imports,", len(v["calls"]), "calls")


if __name__ == "__main__":
    main()
