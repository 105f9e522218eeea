"""A dict whose selected entries are computed on first access.

The reference's renderers return per-pixel candidate lists in an ``intermediates`` dict
on every call. Materialising them costs more memory traffic than rendering, so the drop-in
renderers return this mapping instead: same keys, same tensors, computed only if read.
"""

from __future__ import annotations

from typing import Callable, Dict


class LazyDict(dict):
    def __init__(self, lazy: Dict[str, Callable[[], object]] | None = None, **eager):
        super().__init__(**eager)
        self._lazy: Dict[str, Callable[[], object]] = dict(lazy or {})

    def _resolve(self, key) -> None:
        fn = self._lazy.pop(key, None)
        if fn is not None:
            dict.__setitem__(self, key, fn())

    def _resolve_all(self) -> None:
        for k in list(self._lazy):
            self._resolve(k)

    def is_materialized(self, key) -> bool:
        return key not in self._lazy

    def __getitem__(self, key):
        self._resolve(key)
        return dict.__getitem__(self, key)

    def get(self, key, default=None):
        self._resolve(key)
        return dict.get(self, key, default)

    def __setitem__(self, key, value):
        self._lazy.pop(key, None)
        dict.__setitem__(self, key, value)

    def __delitem__(self, key):
        if key in self._lazy:
            del self._lazy[key]
            if not dict.__contains__(self, key):
                return
        dict.__delitem__(self, key)

    def pop(self, key, *default):
        self._resolve(key)
        return dict.pop(self, key, *default)

    def __contains__(self, key):
        return key in self._lazy or dict.__contains__(self, key)

    def __iter__(self):
        yield from list(dict.keys(self)) + [k for k in self._lazy if not dict.__contains__(self, k)]

    def __len__(self):
        return len(set(dict.keys(self)) | set(self._lazy))

    def keys(self):
        return list(iter(self))

    def items(self):
        self._resolve_all()
        return dict.items(self)

    def values(self):
        self._resolve_all()
        return dict.values(self)

    def copy(self):
        self._resolve_all()
        return dict(dict.items(self))

    def __repr__(self):
        shown = {k: (dict.__getitem__(self, k) if dict.__contains__(self, k) else "<lazy>") for k in self}
        return f"LazyDict({shown!r})"
