"""The cosine basis that diagonalises the solver's pseudo-Laplacian.

The reference assembles M = -L with 2 on the diagonal and -1/2 at the four
diagonal neighbours, indices clamped at the border (otlib/otsolver_2dgrid.cpp:284-311).
That is M = 2 I - 1/2 (S (x) S) with S the 1-D "sum of clamped neighbours"
operator, which the orthonormal DCT-II diagonalises with eigenvalues
2 cos(pi k / n); hence M = C2^T diag(lambda) C2 with C2 = C (x) C and
lambda_kl = 2 - 2 cos(pi k/n) cos(pi l/n). Only lambda_00 vanishes (constants).
The CUDA library builds the same tables on the device; these host copies are
for documentation and tests.
"""

import numpy as np


def basis(n: int) -> np.ndarray:
    """Orthonormal DCT-II matrix, C[k, i] = s_k cos(pi (i + 1/2) k / n)."""
    k = np.arange(n, dtype=np.float64)[:, None]
    i = np.arange(n, dtype=np.float64)[None, :]
    C = np.cos(np.pi * (i + 0.5) * k / n) * np.sqrt(2.0 / n)
    C[0, :] = np.sqrt(1.0 / n)
    return C


def eigenvalues(n: int) -> np.ndarray:
    """lambda[k, l] = 2 - 2 cos(pi k / n) cos(pi l / n)."""
    c = np.cos(np.pi * np.arange(n, dtype=np.float64) / n)
    return 2.0 - 2.0 * np.outer(c, c)
