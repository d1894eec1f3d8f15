"""Array files between the prep and decode stages.

The reference writes ``Dsw``/``dirich``/``Ds`` as PyTables real/imag EArrays
(``vtem/utils/simpleio.py:10-66, :129-149``).  PyTables is not part of this
stack, so the same hand-off uses NumPy ``.npy`` files holding the full
(possibly complex) array.
"""
from __future__ import annotations

import numpy as np


def write_memory_to_file(A, filename, mode="w", title="test"):
    """Write an array (numpy or torch, any device) to ``filename``."""
    try:
        import torch
        if isinstance(A, torch.Tensor):
            A = A.detach().cpu().numpy()
    except ImportError:
        pass
    with open(filename, "wb") as f:
        np.save(f, np.asarray(A))


def read_file(filename):
    """Read an array written by :func:`write_memory_to_file`."""
    with open(filename, "rb") as f:
        return np.load(f)
