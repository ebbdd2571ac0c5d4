"""Host-side 2x2 / 4x4 linear algebra of the BASS driver.

These run once per gate or once per qubit per optimisation pass and stay in
numpy / Python floats so that the device receives exactly the gate matrices
the reference computes:

  * frame conjugation G~ = U^dagger G U        bass_simulator.py:864, 870-871
  * kron(U_q1, U_q2) by 2x2 block assembly     bass_simulator.py:357-383
  * the diagonal test (tolerance 1e-12)        bass_simulator.py:473-475
  * the analytic 2x2 Hermitian eigensolver     bass_simulator.py:386-437
"""
from __future__ import annotations

from math import sqrt

import numpy as np


def kron_2x2(A, B) -> np.ndarray:
    """A (x) B for 2x2 A, B: C[2i:2i+2, 2j:2j+2] = A[i, j] * B."""
    C = np.empty((4, 4), dtype=np.complex128)
    for i in range(2):
        for j in range(2):
            C[2 * i:2 * i + 2, 2 * j:2 * j + 2] = A[i, j] * B
    return C


def is_gate_diagonal(G, tol=1e-12) -> bool:
    return bool(np.max(np.abs(G - np.diag(np.diag(G)))) < tol)


def eigh_2x2(rho):
    """Eigen-decomposition of a Hermitian 2x2: eigenvalues descending and the
    eigenvectors as columns of V.  If |rho01|^2 < 1e-28 the matrix is treated
    as diagonal (V = identity, or the swap if rho00 < rho11).  Python float
    arithmetic is IEEE double, math.sqrt is correctly rounded."""
    a = float(rho[0, 0].real)
    d = float(rho[1, 1].real)
    b = complex(rho[0, 1])
    b_sq = b.real ** 2 + b.imag ** 2
    tau = (d - a) * 0.5
    disc = sqrt(tau * tau + b_sq)
    V = np.zeros((2, 2), dtype=np.complex128)
    if b_sq < 1e-28:
        if a >= d:
            V[0, 0] = 1.0
            V[1, 1] = 1.0
        else:
            V[0, 1] = 1.0
            V[1, 0] = 1.0
    else:
        tdp = tau + disc
        tdm = tau - disc
        n0 = sqrt(b_sq + tdp * tdp)
        n1 = sqrt(b_sq + tdm * tdm)
        V[0, 0] = complex(b.real / n0, b.imag / n0)
        V[1, 0] = tdp / n0
        V[0, 1] = complex(b.real / n1, b.imag / n1)
        V[1, 1] = tdm / n1
    return np.array([(a + d) * 0.5 + disc, (a + d) * 0.5 - disc]), V


def eigh_numpy(rho):
    """The use_fast_eigh=False path (bass_simulator.py:759-763)."""
    evals, V = np.linalg.eigh(rho)
    V = V[:, np.argsort(-evals)]
    if np.linalg.det(V).real < 0:
        V[:, 1] *= -1
    return evals, V


def eigh_2x2_many(r):
    """eigh_2x2 of many 2x2 RDMs at once: r holds rows (rho00, rho11, Re rho01,
    Im rho01); returns V as an (M, 2, 2) array.  The same IEEE operations as
    eigh_2x2, element by element (numpy's sqrt is correctly rounded too)."""
    r = np.asarray(r, dtype=np.float64).reshape(-1, 4)
    a, d, br, bi = r[:, 0], r[:, 1], r[:, 2], r[:, 3]
    b_sq = br * br + bi * bi
    tau = (d - a) * 0.5
    disc = np.sqrt(tau * tau + b_sq)
    tdp = tau + disc
    tdm = tau - disc
    with np.errstate(divide="ignore", invalid="ignore"):
        n0 = np.sqrt(b_sq + tdp * tdp)
        n1 = np.sqrt(b_sq + tdm * tdm)
        V = np.zeros((len(a), 2, 2), dtype=np.complex128)
        V[:, 0, 0] = br / n0 + 1j * (bi / n0)
        V[:, 1, 0] = tdp / n0
        V[:, 0, 1] = br / n1 + 1j * (bi / n1)
        V[:, 1, 1] = tdm / n1
    diag = b_sq < 1e-28
    keep = diag & (a >= d)
    swap = diag & ~(a >= d)
    V[keep] = np.eye(2)
    V[swap] = np.array([[0.0, 1.0], [1.0, 0.0]])
    return V
