"""Float64 reference for the resistivity-tomography misfit and its gradient (TEST ONLY).

The forward operator is the SIGMA7 operator of ``oracle.mg.Sigma7`` (face means of per-cell
conductivities, wall faces use the cell's own conductivity, ghost potential zero:
``Anisotropic Resistivity Tomography/README:14-26``), assembled as a sparse matrix and
solved directly (``scipy.sparse.linalg.splu``), so the reference has no iteration error.
J = 1/2 sum_s |P u_s - d_s|^2; the gradient with respect to log sigma comes from the adjoint
fields (A lam_s = P^T (P u_s - d_s)) and is also checked against central finite differences
of J itself in the CPU tests.
"""
import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spl


def assemble(sig, c=(1.0, 1.0, 1.0)):
    """Sparse float64 matrix of the SIGMA7 operator; sig = (sx, sy, sz) arrays (Z, Y, X)."""
    sx, sy, sz = (np.asarray(a, np.float64) for a in sig)
    cz, cy, cx = c
    Z, Y, X = sx.shape
    n = Z * Y * X
    idx = np.arange(n).reshape(Z, Y, X)
    rows, cols, vals = [], [], []
    diag = np.zeros((Z, Y, X))
    for arr, axis, cc in ((sx, 2, cx), (sy, 1, cy), (sz, 0, cz)):
        m = arr.shape[axis]
        lo = [slice(None)] * 3
        hi = [slice(None)] * 3
        lo[axis] = slice(0, m - 1)
        hi[axis] = slice(1, m)
        a = cc * 0.5 * (arr[tuple(lo)] + arr[tuple(hi)])  # interior faces
        i, j = idx[tuple(lo)].ravel(), idx[tuple(hi)].ravel()
        rows += [i, j]
        cols += [j, i]
        vals += [-a.ravel(), -a.ravel()]
        diag[tuple(lo)] += a
        diag[tuple(hi)] += a
        first = [slice(None)] * 3
        last = [slice(None)] * 3
        first[axis] = slice(0, 1)
        last[axis] = slice(m - 1, m)
        diag[tuple(first)] += cc * arr[tuple(first)]  # wall faces
        diag[tuple(last)] += cc * arr[tuple(last)]
    rows.append(idx.ravel())
    cols.append(idx.ravel())
    vals.append(diag.ravel())
    return sp.csc_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                         shape=(n, n))


def grad_logsigma(sig, u, lam, c=(1.0, 1.0, 1.0)):
    """-sigma_d(c) sum_s dA/dsigma_d(c)[lam_s, u_s]; u, lam arrays (S, Z, Y, X)."""
    sx, sy, sz = (np.asarray(a, np.float64) for a in sig)
    cz, cy, cx = c
    out = []
    for arr, axis, cc in ((sx, 3, cx), (sy, 2, cy), (sz, 1, cz)):
        g = np.zeros(arr.shape)
        m = u.shape[axis]
        lo = [slice(None)] * 4
        hi = [slice(None)] * 4
        lo[axis] = slice(0, m - 1)
        hi[axis] = slice(1, m)
        term = 0.5 * ((lam[tuple(lo)] - lam[tuple(hi)]) * (u[tuple(lo)] - u[tuple(hi)])).sum(0)
        g[tuple(s for s in lo[1:])] += term
        g[tuple(s for s in hi[1:])] += term
        first = [slice(None)] * 4
        last = [slice(None)] * 4
        first[axis] = slice(0, 1)
        last[axis] = slice(m - 1, m)
        g[tuple(first[1:])] += (lam[tuple(first)] * u[tuple(first)]).sum(0)
        g[tuple(last[1:])] += (lam[tuple(last)] * u[tuple(last)]).sum(0)
        out.append(-arr * cc * g)
    return np.stack(out)


def misfit(sig, q, rec, d_obs, c=(1.0, 1.0, 1.0), want_grad=True):
    """J and (optionally) dJ/dlog sigma.  q: (S, Z, Y, X) sources; rec: flat receiver indices;
    d_obs: (S, len(rec)) observed data."""
    A = assemble(sig, c)
    lu = spl.splu(A)
    S = q.shape[0]
    shape = q.shape[1:]
    u = np.stack([lu.solve(q[s].ravel().astype(np.float64)) for s in range(S)])
    res = u[:, rec] - d_obs
    J = 0.5 * float((res ** 2).sum())
    if not want_grad:
        return J, None, u.reshape((S,) + shape)
    rhs = np.zeros_like(u)
    rhs[:, rec] = res
    lam = np.stack([lu.solve(rhs[s]) for s in range(S)])
    g = grad_logsigma(sig, u.reshape((S,) + shape), lam.reshape((S,) + shape), c)
    return J, g, u.reshape((S,) + shape)
