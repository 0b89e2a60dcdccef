"""Learned initialiser of the contraction search: host side.

The network (a 3-layer MLP over the 256-bin rotational profile plus a
4-convolution CNN over the 256 x 256 polar half spectrum) runs in the
library's own BF16 kernels; this module finds, loads and saves its weights.
"""
from __future__ import annotations

import os

HERE = os.path.dirname(os.path.abspath(__file__))
WEIGHTS_PATH = os.path.join(HERE, "weights", "ctf_init.bin")


def learned_available(path: str = WEIGHTS_PATH) -> bool:
    """True when trained weights are present."""
    return os.path.exists(path)


def load_learned(ctx, path: str = WEIGHTS_PATH) -> None:
    """Load trained weights into a Context (raises when absent)."""
    if not learned_available(path):
        raise FileNotFoundError(path)
    ctx.load_weights(path)
