"""Pauli string text format, as PauliStringUtils.h (:41-98) defines it.

``[+|-][i]<ops>`` with ops from ``IXYZ``; qubit q is character q.  The
prefix maps to the flags byte (bit0 imaginary, bit1 sign); printing uses the
prefixes ``"", "i", "-", "-i"`` for flags 0..3.  Encoding per qubit:
I=(x0,z0) X=(x1,z0) Z=(x0,z1) Y=(x1,z1).
"""
from __future__ import annotations

import numpy as np

_PREFIX = ("", "i", "-", "-i")


def parse(s: str, capacity_words: int | None = None):
    """Return (x_words, z_words, flags, num_qubits) for one Pauli string."""
    if not s:
        raise ValueError("Pauli string is empty")
    sign = imag = False
    pos = 0
    if s.startswith("-i"):
        sign = imag = True
        pos = 2
    elif s.startswith("+i"):
        imag = True
        pos = 2
    elif s[0] == "-":
        sign = True
        pos = 1
    elif s[0] in "+i":
        imag = s[0] == "i"
        pos = 1
    ops = s[pos:]
    nq = len(ops)
    aw = capacity_words if capacity_words is not None else max(1, (nq + 63) // 64)
    if nq > 64 * aw:
        raise ValueError(f"Pauli string has {nq} operator characters, exceeding the capacity "
                         f"of {64 * aw} qubits")
    x = [0] * aw
    z = [0] * aw
    for q, ch in enumerate(ops):
        w, b = divmod(q, 64)
        if ch == "X":
            x[w] |= 1 << b
        elif ch == "Z":
            z[w] |= 1 << b
        elif ch == "Y":
            x[w] |= 1 << b
            z[w] |= 1 << b
        elif ch != "I":
            raise ValueError("Invalid Pauli character")
    flags = (2 if sign else 0) | (1 if imag else 0)
    return x, z, flags, nq


def fmt(x_words, z_words, flags: int, num_qubits: int) -> str:
    out = []
    for q in range(num_qubits):
        w, b = divmod(q, 64)
        xb = (int(x_words[w]) >> b) & 1
        zb = (int(z_words[w]) >> b) & 1
        out.append("Y" if xb and zb else "X" if xb else "Z" if zb else "I")
    return _PREFIX[int(flags) & 3] + "".join(out)


def planes_from_terms(terms, capacity_words: int | None = None):
    """[(string, coeff)] or [string] -> (x (AS,n), z (AS,n), flags, val, num_qubits)."""
    items = [(t, 1.0) if isinstance(t, str) else (t[0], float(t[1])) for t in terms]
    nq = 0
    parsed = []
    for s, c in items:
        px, pz, pf, q = parse(s, capacity_words)
        parsed.append((px, pz, pf, c))
        nq = max(nq, q)
    aw = capacity_words if capacity_words is not None else max(1, (nq + 63) // 64)
    n = len(parsed)
    x = np.zeros((aw, n), np.uint64)
    z = np.zeros((aw, n), np.uint64)
    f = np.zeros(n, np.uint8)
    v = np.zeros(n, np.float64)
    for i, (px, pz, pf, c) in enumerate(parsed):
        for k in range(aw):
            x[k, i] = px[k] if k < len(px) else 0
            z[k, i] = pz[k] if k < len(pz) else 0
        f[i] = pf
        v[i] = c
    return x, z, f, v, nq


def get_str(x, z, flags, val, num_qubits: int) -> str:
    """PauliSum::get_str (PauliSumUtils.h:19-33): '<%f coeff> * <string>' lines."""
    lines = []
    for i in range(len(val)):
        lines.append(f"{float(val[i]):f} * " + fmt(x[:, i], z[:, i], flags[i], num_qubits) + "\n")
    return "".join(lines)


def multiply_words(ax, az, fa: int, bx, bz, fb: int):
    """(x, z, flags) of the product of two strings given as word lists:
    x = ax ^ bx, z = az ^ bz, flags = (fa + fb + popc(c1) + 2 parity(c2))
    mod 4 with the per-word phase accumulators of PauliStringCore.h:150-174.
    The single-string value algebra of PauliString; sums multiply on the
    device."""
    c1 = c2 = 0
    x, z = [], []
    for a_x, a_z, b_x, b_z in zip(ax, az, bx, bz):
        a_x, a_z, b_x, b_z = int(a_x), int(a_z), int(b_x), int(b_z)
        xbz = a_x & b_z
        anti = (b_x & a_z) ^ xbz
        c2 ^= (c1 ^ a_x ^ a_z ^ b_x ^ b_z ^ xbz) & anti
        c1 ^= anti
        x.append(a_x ^ b_x)
        z.append(a_z ^ b_z)
    f = (int(fa) + int(fb) + bin(c1).count("1") + 2 * (bin(c2).count("1") & 1)) & 3
    return x, z, f


def anticommute_words(ax, az, bx, bz) -> int:
    """Symplectic inner product (0: commute, 1: anticommute),
    PauliStringCore.h:126-146."""
    p = 0
    for a_x, a_z, b_x, b_z in zip(ax, az, bx, bz):
        p ^= (int(a_x) & int(b_z)) ^ (int(a_z) & int(b_x))
    return bin(p).count("1") & 1


class MT19937_64:
    """std::mt19937_64 (the 64-bit Mersenne Twister of Matsumoto and
    Nishimura, as the C++ standard specifies it), whose raw outputs are what
    std::uniform_int_distribution<uint64_t> over the full range returns:
    the generator behind random_pauli_sum (PauliSumUtils.h:114-154)."""

    N, M = 312, 156
    MATRIX_A = 0xB5026F5AA96619E9
    UPPER, LOWER = 0xFFFFFFFF80000000, 0x7FFFFFFF
    MASK = (1 << 64) - 1

    def __init__(self, seed: int = 5489):
        mt = [int(seed) & self.MASK]
        for i in range(1, self.N):
            prev = mt[-1]
            mt.append((6364136223846793005 * (prev ^ (prev >> 62)) + i) & self.MASK)
        self.mt = mt
        self.i = self.N

    def _twist(self):
        mt, n, m = self.mt, self.N, self.M
        for k in range(n):
            y = (mt[k] & self.UPPER) | (mt[(k + 1) % n] & self.LOWER)
            mt[k] = mt[(k + m) % n] ^ (y >> 1) ^ (self.MATRIX_A if y & 1 else 0)
        self.i = 0

    def __call__(self) -> int:
        if self.i >= self.N:
            self._twist()
        y = self.mt[self.i]
        self.i += 1
        y ^= (y >> 29) & 0x5555555555555555
        y ^= (y << 17) & 0x71D67FFFEDA60000
        y ^= (y << 37) & 0xFFF7EEE000000000
        y ^= y >> 43
        return y & self.MASK


def random_planes(num_terms: int, seed: int, num_qubits: int, words: int):
    """The terms random_pauli_sum(num_terms, seed, num_qubits) draws
    (PauliSumUtils.h:114-154): per term the sign bit, the phase bit, then the
    x and z word of every word covering num_qubits (the last one masked to
    the remaining qubits), all coefficients 1."""
    rng = MT19937_64(seed)
    full, rem = divmod(int(num_qubits), 64)
    n = int(num_terms)
    x = np.zeros((words, n), np.uint64)
    z = np.zeros((words, n), np.uint64)
    f = np.zeros(n, np.uint8)
    for t in range(n):
        sign = rng() & 1
        phase = rng() & 1
        f[t] = (sign << 1) | phase
        for w in range(full):
            x[w, t] = rng()
            z[w, t] = rng()
        if rem:
            pad = (1 << rem) - 1
            x[full, t] = rng() & pad
            z[full, t] = rng() & pad
    return x, z, f, np.ones(n, np.float64)
