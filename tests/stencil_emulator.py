"""numpy emulation of the step kernels' arithmetic (test helper).

Evaluates, on the CPU, the update formula the CUDA kernels implement
(wakis_b200/csrc/fit_common.cuh): per-row factors from the material table
and the separable metric tables, column factors from the 1-D lengths with
the PEC/PMC face masks, flat-offset neighbours, products rounded one by one
and the four terms summed in the kernels' order.  Comparing it with the
oracle's sparse mat-vec on the CPU checks the compact coefficients and the
formula before any GPU run.
"""

import numpy as np


def _cells(shape):
    Nx, Ny, Nz = shape
    n = np.arange(Nx * Ny * Nz)
    return n, n % Nx, (n // Nx) % Ny, n // (Nx * Ny)


def face_val(f, d, i, j, k, shape):
    Nx, Ny, Nz = shape
    v = np.ones_like(i)
    if d != 0:
        v = np.where(i == 0, f[0], v)
        v = np.where(i == Nx - 1, f[1], v)
    if d != 1:
        v = np.where(j == 0, f[2], v)
        v = np.where(j == Ny - 1, f[3], v)
    if d != 2:
        v = np.where(k == 0, f[4], v)
        v = np.where(k == Nz - 1, f[5], v)
    return v


def _cell_of(m, shape):
    Nx, Ny, _ = shape
    return m % Nx, (m // Nx) % Ny, m // (Nx * Ny)


def _len(coef, d, i, j, k, dual):
    a = ((coef.tLx, coef.tLy, coef.tLz) if dual else (coef.Lx, coef.Ly, coef.Lz))[d]
    idx = (i, j, k)[d]
    return a[np.clip(idx, 0, len(a) - 1)]


def _col_factor(coef, d, m, valid, dual):
    shape = coef.shape
    i, j, k = _cell_of(np.where(valid, m, 0), shape)
    L = _len(coef, d, i, j, k, dual)
    if dual:
        if coef.has_pmc:
            L = np.where(face_val(coef.pmc_face, d, i, j, k, shape) == 0, 0, L)
    elif coef.has_pec:
        L = np.where(face_val(coef.pec_face, d, i, j, k, shape) == 0, 0, L)
    return np.where(valid, L, 0).astype(coef.dtype)


def _sum4(t, desc):
    z = np.zeros_like(t[0])
    order = t[::-1] if desc else t
    acc = z
    for x in order:
        acc = acc + x
    return acc


H_TERMS = {  # (comp, offset key, sign)
    0: [(1, 0, 1), (1, "z", -1), (2, 0, -1), (2, "y", 1)],
    1: [(0, 0, -1), (0, "z", 1), (2, 0, 1), (2, "x", -1)],
    2: [(0, 0, 1), (0, "y", -1), (1, 0, -1), (1, "x", 1)],
}
E_TERMS = {
    0: [(1, "z", 1), (1, 0, -1), (2, "y", -1), (2, 0, 1)],
    1: [(0, "z", -1), (0, 0, 1), (2, "x", 1), (2, 0, -1)],
    2: [(0, "y", 1), (0, 0, -1), (1, "x", -1), (1, 0, 1)],
}


def _offset(key, shape):
    Nx, Ny, _ = shape
    return {0: 0, "x": 1, "y": Nx, "z": Nx * Ny}[key]


def h_update(coef, E, H, dt):
    shape = coef.shape
    N = int(np.prod(shape))
    n, i, j, k = _cells(shape)
    ids = coef.ids.astype(np.int64)
    out = H.copy()
    iA = (coef.iAx[j, k], coef.iAy[i, k], coef.iAz[i, j])
    for d in range(3):
        R = iA[d] * coef.table[ids, 3 + d]
        if coef.has_pmc:
            R = np.where(face_val(coef.pmc_face, d, i, j, k, shape) == 0, coef.dtype(0), R)
        terms = []
        for e, key, sgn in H_TERMS[d]:
            m = n + _offset(key, shape)
            valid = m < N
            L = _col_factor(coef, e, m, valid, dual=False)
            ev = E[e * N + np.where(valid, m, 0)]
            v = (dt * (R * L)) * ev
            terms.append(v if sgn > 0 else -v)
        out[d * N:(d + 1) * N] = H[d * N:(d + 1) * N] - _sum4(terms, coef.h_sum_desc)
    return out


def e_update(coef, E, Hn, J, dt):
    shape = coef.shape
    N = int(np.prod(shape))
    n, i, j, k = _cells(shape)
    ids = coef.ids.astype(np.int64)
    out = E.copy()
    itA = (coef.itAx[j, k], coef.itAy[i, k], coef.itAz[i, j])
    for d in range(3):
        ieps = coef.table[ids, d]
        R = ieps * itA[d]
        if coef.has_pec:
            R = np.where(face_val(coef.pec_face, d, i, j, k, shape) == 0, coef.dtype(0), R)
        terms = []
        for e, key, sgn in E_TERMS[d]:
            m = n - _offset(key, shape)
            valid = m >= 0
            L = _col_factor(coef, e, m, valid, dual=True)
            hv = Hn[e * N + np.where(valid, m, 0)]
            v = (R * L) * hv
            terms.append(v if sgn > 0 else -v)
        curl = _sum4(terms, False)
        out[d * N:(d + 1) * N] = E[d * N:(d + 1) * N] + dt * (curl - ieps * J[d * N:(d + 1) * N])
    return out


def lean_cells(shape, kind):
    """Flat indices of the cells the kernels update with the lean formulas."""
    n, i, j, k = _cells(shape)
    Nx, Ny, Nz = shape
    if kind == "h":
        m = (i >= 1) & (i <= Nx - 3) & (j >= 1) & (j <= Ny - 3) & (k >= 1) & (k <= Nz - 3)
    else:
        m = (i >= 2) & (i <= Nx - 2) & (j >= 2) & (j <= Ny - 2) & (k >= 2) & (k <= Nz - 2)
    return n[m]


def h_lean(coef, E, H, dt, cells):
    """The kernels' interior H update (h_lean in fit_common.cuh) on `cells`."""
    Nx, Ny, Nz = coef.shape
    N = Nx * Ny * Nz
    n = cells
    i, j, k = n % Nx, (n // Nx) % Ny, n // (Nx * Ny)
    t = coef.table[coef.ids.astype(np.int64)[n]]
    ex, ey, ez = (E[d * N:(d + 1) * N] for d in range(3))
    R0, R1, R2 = coef.iAx[j, k] * t[:, 3], coef.iAy[i, k] * t[:, 4], coef.iAz[i, j] * t[:, 5]
    Lx, Ly, Lz = coef.Lx[i], coef.Ly[j], coef.Lz[k]
    desc = coef.h_sum_desc
    out = []
    a, b = dt * (R0 * Ly), dt * (R0 * Lz)
    t0, t1, t2, t3 = a * ey[n], a * ey[n + Nx * Ny], b * ez[n], b * ez[n + Nx]
    out.append(H[n] - ((((t3 - t2) - t1) + t0) if desc else (((t0 - t1) - t2) + t3)))
    a, b = dt * (R1 * Lx), dt * (R1 * Lz)
    t0, t1, t2, t3 = a * ex[n], a * ex[n + Nx * Ny], b * ez[n], b * ez[n + 1]
    out.append(H[N + n] - ((((t2 - t3) + t1) - t0) if desc else (((t1 - t0) + t2) - t3)))
    a, b = dt * (R2 * Lx), dt * (R2 * Ly)
    t0, t1, t2, t3 = a * ex[n], a * ex[n + Nx], b * ey[n], b * ey[n + 1]
    out.append(H[2 * N + n] - ((((t3 - t2) - t1) + t0) if desc else (((t0 - t1) - t2) + t3)))
    return out


def e_lean_curl(coef, Hn, cells):
    Nx, Ny, Nz = coef.shape
    N = Nx * Ny * Nz
    n = cells
    i, j, k = n % Nx, (n // Nx) % Ny, n // (Nx * Ny)
    t = coef.table[coef.ids.astype(np.int64)[n]]
    hx, hy, hz = (Hn[d * N:(d + 1) * N] for d in range(3))
    R0, R1, R2 = t[:, 0] * coef.itAx[j, k], t[:, 1] * coef.itAy[i, k], t[:, 2] * coef.itAz[i, j]
    tLx, tLy, tLz = coef.tLx[i], coef.tLy[j], coef.tLz[k]
    c1, c2 = R0 * tLy, R0 * tLz
    cx = (((c1 * hy[n - Nx * Ny]) - (c1 * hy[n])) - (c2 * hz[n - Nx])) + (c2 * hz[n])
    c1, c2 = R1 * tLx, R1 * tLz
    cy = (((c1 * hx[n]) - (c1 * hx[n - Nx * Ny])) + (c2 * hz[n - 1])) - (c2 * hz[n])
    c1, c2 = R2 * tLx, R2 * tLy
    cz = (((c1 * hx[n - Nx])) - (c1 * hx[n]) - (c2 * hy[n - 1])) + (c2 * hy[n])
    return cx, cy, cz
