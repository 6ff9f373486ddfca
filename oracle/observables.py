"""State-vector checks of MPS observables (small chains).

TEST INFRASTRUCTURE ONLY -- the parity oracle; see ``oracle/qtensor.py``.

An MPS (U(1) block tensors or dense arrays, indices (left link, site, right
link)) is contracted into its full 2^L amplitude vector, index
sum_i s_i 2^i with s_i = 1 for Up -- the basis of ``oracle/ed.py`` -- and
overlaps, expectation values of a term list and <Sz_i Sz_j> are evaluated
exactly on it.  This pins ``psiphi``/``psiHphi`` (mps/observables.cpp:25-103,
382-450) and the correlator kernels without restating their contraction order.
"""
from __future__ import annotations

from typing import Sequence

import numpy as np

from .qtensor import to_dense


def state_vector(tensors: Sequence[np.ndarray]) -> np.ndarray:
    """Amplitudes of an MPS given as dense (left, site, right) arrays."""
    M = tensors[0][0]  # (2, d1)
    for A in tensors[1:]:
        # M: (2^i, d) ; A: (d, 2, d') -> index s_i * 2^i + old
        M = np.einsum("od,dse->soe", M, A).reshape(-1, A.shape[2])
    return M[:, 0]


def qmps_state_vector(qtensors) -> np.ndarray:
    return state_vector([to_dense(T) for T in qtensors])


def sz_correlators(v: np.ndarray, L: int):
    """(<Sz_i>, <Sz_i Sz_j>) of the normalised state v."""
    p = np.abs(v) ** 2
    p = p / p.sum()
    idx = np.arange(len(v))
    sz = np.array([((idx >> i) & 1) - 0.5 for i in range(L)])  # (L, 2^L)
    one = sz @ p
    two = (sz * p) @ sz.T
    return one, two
