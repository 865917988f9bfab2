"""The compiled-extension names of the reference's Python package
(python/bindings.cpp:300-379), over this library's device-resident sums.

One class per 64-bit word count -- ``PauliString_<N>`` and ``PauliSum_<N>``
for N = 64, 128, ..., 1024 qubits of capacity -- plus ``random_pauli_sum_<N>``,
``trace_product_<N>``, ``commutator_<N>``, ``i_commutator_<N>`` and
``propagate_expectation_<N>``, ``TruncationOptions`` and
``SUPPORTED_CAPACITIES``.  The sums' methods run on the GPU through the C
ABI (libpaulib_b200.so); there is no CPU path for them.
"""
from __future__ import annotations

import numpy as np

from paulib_b200 import paulib as _core
from paulib_b200 import strings as _strings

SIZE_MAX = (1 << 64) - 1
SUPPORTED_CAPACITIES = [64 * k for k in range(1, 17)]


class TruncationOptions:
    """TruncationOptions<double> (PauliPropagation.h:27-31): strings acting
    on more than max_weight qubits, with |coefficient| below
    coefficient_cutoff, or beyond the max_terms largest are dropped."""

    def __init__(self):
        self.max_weight = SIZE_MAX
        self.coefficient_cutoff = 0.0
        self.max_terms = SIZE_MAX


def _opts(o: TruncationOptions) -> _core.TruncationOptions:
    mw = None if o.max_weight >= SIZE_MAX else int(o.max_weight)
    mt = None if o.max_terms >= SIZE_MAX else int(o.max_terms)
    return _core.TruncationOptions(mw, float(o.coefficient_cutoff), mt)


def _make(cap: int):
    words = cap // 64

    class PauliStringN(_core.PauliString):
        CAPACITY = cap

    class PauliSumN(_core._PauliSum):
        CAPACITY = cap

        def __init__(self, arg=None):
            """PauliSum_<N>(num_qubits=N) (an empty sum), PauliSum_<N>(list of
            strings) or PauliSum_<N>(list of (string, coefficient))."""
            if arg is None or isinstance(arg, int):
                nq = cap if arg is None else int(arg)
                if nq > cap:
                    raise ValueError(f"qubit count exceeds capacity {cap}")
                _core._PauliSum.__init__(self, nq, words=words)
                return
            terms = list(arg)
            if not terms:
                _core._PauliSum.__init__(self, cap, words=words)
                return
            x, z, f, v, nq = _strings.planes_from_terms(terms, words)
            _core._PauliSum.__init__(self, nq, x, z, f, v, words=words)

        def _string_cls(self):
            return PauliStringN

    PauliStringN.__name__ = PauliStringN.__qualname__ = f"PauliString_{cap}"
    PauliSumN.__name__ = PauliSumN.__qualname__ = f"PauliSum_{cap}"

    def random_pauli_sum(num_terms: int, seed: int = 42, num_qubits: int = cap):
        """random_pauli_sum<N, double> (PauliSumUtils.h:114-154): the same
        std::mt19937_64 draws, so the same terms as the reference's."""
        if num_qubits > cap:
            raise ValueError("qubit count exceeds capacity")
        x, z, f, v = _strings.random_planes(num_terms, seed, num_qubits, words)
        s = PauliSumN(int(num_qubits))
        if num_terms:
            s._st.upload(x, z, f, v)
        return s

    def commutator(a, b):
        """[A, B], canonicalized."""
        return _core.commutator(a, b)

    def i_commutator(a, b):
        """i[A, B], canonicalized (Hermitian for Hermitian inputs)."""
        return _core.i_commutator(a, b)

    def trace_product(a, b) -> float:
        """Re tr(A*B), computed without forming the product."""
        return _core.trace_product(a, b)

    def propagate_expectation(observable, rotations, options=None) -> float:
        """Pauli propagation: <0|U^dagger O U|0> for the rotation circuit U
        (term = generator, coefficient = angle; PauliPropagation.h:65-71)."""
        o = options if options is not None else TruncationOptions()
        return _core.propagate_expectation(observable, rotations, _opts(o))

    return {f"PauliString_{cap}": PauliStringN, f"PauliSum_{cap}": PauliSumN,
            f"random_pauli_sum_{cap}": random_pauli_sum, f"commutator_{cap}": commutator,
            f"i_commutator_{cap}": i_commutator, f"trace_product_{cap}": trace_product,
            f"propagate_expectation_{cap}": propagate_expectation}


for _cap in SUPPORTED_CAPACITIES:
    globals().update(_make(_cap))
del _cap
