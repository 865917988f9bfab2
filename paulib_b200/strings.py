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
