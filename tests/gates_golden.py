"""Known answers of the reference's gate tests, shared by the CPU and GPU
gate tests: single-qubit truth tables (CliffordExtendedTests.cpp:24-118,
PauliSumTests.cpp:285-330), two-qubit truth tables of the controlled-Pauli
family and SWAP (CliffordExtendedTests.cpp:123-258) and the rotation-gate
results (PauliSumTests.cpp:202-280).  Gate numbers are PL_GATE_* values."""

GATE = {"H": 1, "S": 2, "H_YZ": 3, "H_XY": 4, "SQRT_X": 5, "SQRT_Y": 6, "X": 7, "Y": 8,
        "Z": 9, "I": 10, "CNOT": 11, "CZ": 12, "CY": 13, "XC_X": 14, "XC_Y": 15, "XC_Z": 16,
        "YC_X": 17, "YC_Y": 18, "YC_Z": 19, "SWAP": 20, "ISWAP": 21}

ONE_QUBIT = {
    "H": {"I": "I", "X": "Z", "Y": "-Y", "Z": "X"},
    "H_YZ": {"I": "I", "X": "-X", "Y": "Z", "Z": "Y"},
    "H_XY": {"I": "I", "X": "Y", "Y": "X", "Z": "-Z"},
    "SQRT_X": {"I": "I", "X": "X", "Y": "Z", "Z": "-Y"},
    "SQRT_Y": {"I": "I", "X": "-Z", "Y": "Y", "Z": "X"},
    "X": {"I": "I", "X": "X", "Y": "-Y", "Z": "-Z"},
    "Y": {"I": "I", "X": "-X", "Y": "Y", "Z": "-Z"},
    "Z": {"I": "I", "X": "-X", "Y": "-Y", "Z": "Z"},
    "I": {"I": "I", "X": "X", "Y": "Y", "Z": "Z"},
}


def _table(s):
    keys = ["II", "IX", "IY", "IZ", "XI", "XX", "XY", "XZ", "YI", "YX", "YY", "YZ",
            "ZI", "ZX", "ZY", "ZZ"]
    return dict(zip(keys, s.split()))


TWO_QUBIT = {
    "CY": _table("II ZX IY ZZ XY -YZ XI YX YY XZ YI -XX ZI IX ZY IZ"),
    "XC_X": _table("II IX XY XZ XI XX IY IZ YX YI ZZ -ZY ZX ZI -YZ YY"),
    "XC_Z": _table("II XX XY IZ XI IX IY XZ YZ ZY -ZX YI ZZ -YY YX ZI"),
    "XC_Y": _table("II XX IY XZ XI IX XY IZ YY -ZZ YI ZX ZY YZ ZI -YX"),
    "YC_X": _table("II IX YY YZ XX XI -ZZ ZY YI YX IY IZ ZX ZI XZ -XY"),
    "YC_Z": _table("II YX YY IZ XZ -ZY ZX XI YI IX IY YZ ZZ XY -XX ZI"),
    "YC_Y": _table("II YX IY YZ XY ZZ XI -ZX YI IX YY IZ ZY -XZ ZI XX"),
    "SWAP": _table("II XI YI ZI IX XX YX ZX IY XY YY ZY IZ XZ YZ ZZ"),
}

# (axis, input, expected get_str) for angle pi/3; axis 1 X, 2 Y, 3 Z
ROTATIONS = [
    (3, [("X", 1.0)], "0.866025 * X\n0.500000 * -Y\n"),
    (3, [("Z", 2.0), ("X", 1.0)], "2.000000 * Z\n0.866025 * X\n0.500000 * -Y\n"),
    (1, [("Z", 1.0)], "0.866025 * Z\n0.500000 * Y\n"),
    (2, [("Z", 1.0)], "0.866025 * Z\n0.500000 * -X\n"),
    (2, [("X", 1.0)], "0.500000 * Z\n0.866025 * X\n"),
]
