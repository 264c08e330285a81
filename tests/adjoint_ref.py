"""FP64 reference gradient of a loss of the forward mesh with respect to the density,
built on the CPU with explicit sparse matrices (test infrastructure).

G   : vertex-gradient operator (otsolver_2dgrid.cpp:362-423), 2V x N
dAdg: derivative of the quad areas (otsolver_2dgrid.cpp:425-447) w.r.t. the vertex
      displacements at a given forward mesh, N x 2V
J = dAdg G; lambda from the bordered system [[J^T, 1], [1^T, 0]] [lambda; mu] = [G^T q; 0];
dL/drho = (lambda - (lambda . rho) / S) / S for the normalisation of otsolver_2dgrid.cpp:53-55.
"""

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla


def grad_operator(n):
    V = (n + 1) ** 2
    rows, cols, vals = [], [], []
    hw = 0.5 * n
    cl = lambda v: min(max(v, 0), n - 1)
    for vi in range(n + 1):
        for vj in range(n + 1):
            v = vj + vi * (n + 1)
            for a in (0, 1):
                for b in (0, 1):
                    f = cl(vj - 1 + b) + cl(vi - 1 + a) * n
                    rows += [2 * v, 2 * v + 1]
                    cols += [f, f]
                    vals += [(2 * a - 1) * hw, (2 * b - 1) * hw]
    return sp.csr_matrix((vals, (rows, cols)), shape=(2 * V, n * n))


def area_jacobian(fwd, n):
    e = 1.0 / n
    t = np.arange(n + 1) * (1.0 / n)
    grid = np.stack([np.repeat(t, n + 1), np.tile(t, n + 1)], axis=1)
    g = fwd - grid
    rows, cols, vals = [], [], []
    for ci in range(n):
        for cj in range(n):
            c = cj + ci * n
            v00 = cj + ci * (n + 1)
            v10 = cj + (ci + 1) * (n + 1)
            v01 = cj + 1 + ci * (n + 1)
            v11 = cj + 1 + (ci + 1) * (n + 1)
            D1 = g[v11] - g[v00] + np.array([e, e])
            D2 = g[v01] - g[v10] + np.array([-e, e])
            dD1 = 0.5 * np.array([D2[1], -D2[0]])
            dD2 = 0.5 * np.array([-D1[1], D1[0]])
            for v, w in ((v11, dD1), (v00, -dD1), (v01, dD2), (v10, -dD2)):
                rows += [c, c]
                cols += [2 * v, 2 * v + 1]
                vals += [w[0], w[1]]
    return sp.csr_matrix((vals, (rows, cols)), shape=(n * n, 2 * (n + 1) ** 2))


def reference_gradient(fwd, density_raw, grad_fwd, n):
    G = grad_operator(n)
    J = (area_jacobian(fwd, n) @ G).tocsr()
    b = G.T @ grad_fwd.reshape(-1)
    N = n * n
    ones = sp.csr_matrix(np.ones((N, 1)))
    K = sp.bmat([[J.T, ones], [ones.T, None]], format="csc")
    sol = spla.spsolve(K, np.concatenate([b, [0.0]]))
    lam = sol[:N]
    S = density_raw.sum()
    return (lam - lam @ density_raw / S) / S, J
