"""Exact known answers of free-fermion spin chains, for pinning the DMRG
oracle and the GPU path at chain lengths beyond exact diagonalisation.

Test infrastructure, like the rest of ``oracle/``: only ``tests/`` use it.
The reference has no counterpart; these are textbook results (Jordan-Wigner
transformation; Lieb, Schultz and Mattis, Ann. Phys. 16, 407 (1961);
Pfeuty, Ann. Phys. 57, 79 (1970)), checked here against exact
diagonalisation at small L (``tests/test_oracle_observables.py``,
``tests/test_oracle_ed.py``).

* Open XX chain, H = sum_i (S+_i S-_{i+1} + S-_i S+_{i+1}) / 2: fermions
  hopping with amplitude 1/2, single-particle orbitals
  phi_k(i) = sqrt(2 / (L + 1)) sin(pi k i / (L + 1)) with energies
  cos(pi k / (L + 1)), k, i = 1..L.  The Sz = 0 ground state fills the L/2
  lowest; with G_ij = <c+_i c_j> = sum_occupied phi_k(i) phi_k(j) (G_ii = 1/2
  at half filling), Wick's theorem gives <Sz_i Sz_j> = -G_ij^2 for i != j.
* Open transverse-field Ising chain, H = -sum Z_i Z_{i+1} - g sum X_i:
  free Majorana fermions, E0 = -(sum of the singular values of the L x L
  bidiagonal matrix with g on the diagonal and 1 above it).
"""
import numpy as np


def xx_orbitals(L: int):
    """(orbitals phi[k, i], energies eps[k]) of the open XX chain."""
    k = np.arange(1, L + 1)
    i = np.arange(1, L + 1)
    phi = np.sqrt(2.0 / (L + 1)) * np.sin(np.pi * np.outer(k, i) / (L + 1))
    return phi, np.cos(np.pi * k / (L + 1))


def xx_chain_energy(L: int) -> float:
    """Sz = 0 ground energy of the open XX chain (L even)."""
    _, eps = xx_orbitals(L)
    return float(np.sort(eps)[: L // 2].sum())


def xx_chain_szsz(L: int) -> np.ndarray:
    """<Sz_i Sz_j> (L x L) in the Sz = 0 ground state of the open XX chain."""
    phi, eps = xx_orbitals(L)
    occ = np.argsort(eps)[: L // 2]
    G = phi[occ].T @ phi[occ]
    out = -G * G
    np.fill_diagonal(out, 0.25)
    return out


def tfi_chain_energy(L: int, g: float) -> float:
    """Ground energy of H = -sum Z_i Z_{i+1} - g sum X_i on the open chain."""
    B = np.diag(np.full(L, float(g))) + np.diag(np.ones(L - 1), 1)
    return float(-np.linalg.svd(B, compute_uv=False).sum())
