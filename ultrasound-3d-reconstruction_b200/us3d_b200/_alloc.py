"""Output tensors of one library call carved from a single device allocation.

A renderer's backward returns several gradient tensors; allocating them one by one costs a
caching-allocator round trip each on the host, while the device waits for the launch (the
forward synchronised to return its instance count). Here they are views of one float32 buffer,
each starting on a 16-byte boundary.
"""

from __future__ import annotations

import math
from typing import Iterable, List, Sequence, Tuple

import torch


def float_outputs(device: torch.device, shapes: Sequence[Tuple[int, ...]],
                  zero: Iterable[int] = ()) -> List[torch.Tensor]:
    """Float32 tensors of ``shapes`` sharing one allocation; those whose index is in ``zero`` are
    zero-filled, the others are left for the library to write in full."""
    sizes = [math.prod(s) for s in shapes]
    offsets, n = [], 0
    for k in sizes:
        offsets.append(n)
        n += (k + 3) // 4 * 4
    buf = torch.empty(max(n, 4), dtype=torch.float32, device=device)
    out = [buf[o:o + k].view(s) for o, k, s in zip(offsets, sizes, shapes)]
    for i in zero:
        out[i].zero_()
    return out
