"""Host SoA planes of a Pauli sum: the wire format of the C ABI.

A sum of n terms over AS = ceil(N/64) words crosses the boundary as
``x``/``z`` of shape (AS, n) uint64 (word k of term i at ``x[k, i]``, the
layout ``x[k*stride + i]`` of ``include/gpu/GpuPauliSum.h:8-12``),
``flags`` (n,) uint8 (bit0 = i, bit1 = -) and ``val`` (n,) float64.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass
class Planes:
    """Host SoA planes of a Pauli sum (the wire format of the C ABIs)."""

    x: np.ndarray  # (AS, n) uint64
    z: np.ndarray  # (AS, n) uint64
    flags: np.ndarray  # (n,) uint8
    val: np.ndarray  # (n,) float64

    @property
    def n(self) -> int:
        return int(self.val.shape[0])

    @property
    def array_size(self) -> int:
        return int(self.x.shape[0])

    def copy(self) -> "Planes":
        return Planes(self.x.copy(), self.z.copy(), self.flags.copy(), self.val.copy())

    @staticmethod
    def empty(array_size: int, n: int) -> "Planes":
        return Planes(
            np.zeros((array_size, n), np.uint64),
            np.zeros((array_size, n), np.uint64),
            np.zeros(n, np.uint8),
            np.zeros(n, np.float64),
        )
