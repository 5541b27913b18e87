"""Morton keys (the reference's ``FlashKNN/functions/z_order.py:xyz2key``).

Same bit layout: the low 16 bits of x, y, z interleaved with x at bit 3b+2,
y at 3b+1, z at 3b, and the batch id in bits 48 and up.  Computed by the
CUDA kernel behind ``fknn_morton_encode``; inputs must be CUDA tensors.
"""
from __future__ import annotations

from typing import Optional, Union

import torch

from . import ops


def xyz2key(x: torch.Tensor, y: torch.Tensor, z: torch.Tensor,
            b: Optional[Union[torch.Tensor, int]] = None, depth: int = 16) -> torch.Tensor:
    if depth != 16:
        raise ValueError("only the 16-bit-per-axis key of the reference query path is provided")
    grid = torch.stack([x.long(), y.long(), z.long()], dim=1)
    batch = None
    if b is not None:
        batch = b.long() if isinstance(b, torch.Tensor) else torch.full_like(grid[:, 0], int(b))
    return ops.morton_encode(grid, batch)
