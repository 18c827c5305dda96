"""CPU restatement of the reference's extra order parameters (src/parameter_order.cpp:129-245): Polarization,
Splay_magnitude, Splay_divergence, Radial_order, with the reference's float site terms and double sums.

TEST INFRASTRUCTURE ONLY: the checker of mcl_measure_extras (mclics_b200/csrc/extras.cu) in tests/.
"""
import numpy as np

DIRS = [(1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1)]


def _nb(i, n, periodic):
    if 0 <= i < n:
        return i
    return i % n if periodic else None


def extras(ni, pt, shape, periodic, director):
    """ni: (N, 3) float32 in the reference order, pt: (N,) point types (0 empty), shape (Nx, Ny, Nz), periodic
    (3 bools), director (3,). Returns dict P, dtheta, divn, Sr_sph, Pr_sph, Sr_cyl, Pr_cyl."""
    Nx, Ny, Nz = shape
    ni = np.asarray(ni, np.float32).reshape(-1, 3)
    f = np.float32
    d = np.asarray(director, np.float32)
    idx = lambda i, j, k: i + Nx * (j + Ny * k)  # noqa: E731
    sP, vP = 0.0, 0
    sv = np.zeros(3)
    nB = 0
    sdiv, vdiv = 0.0, 0
    rad = {False: [0.0, 0.0, 0], True: [0.0, 0.0, 0]}
    cx, cy, cz = f(Nx // 2), f(Ny // 2), f(Nz // 2)
    for k in range(Nz):
        for j in range(Ny):
            for i in range(Nx):
                q = idx(i, j, k)
                if not pt[q]:
                    continue
                a = ni[q]
                sP += float(f(d[0] * a[0]) + f(d[1] * a[1]) + f(d[2] * a[2]))  # parameter_order.cpp:137
                vP += 1
                for dx, dy, dz in DIRS:  # parameter_order.cpp:158-170
                    ii, jj, kk = _nb(i + dx, Nx, periodic[0]), _nb(j + dy, Ny, periodic[1]), _nb(k + dz, Nz, periodic[2])
                    if ii is None or jj is None or kk is None or not pt[idx(ii, jj, kk)]:
                        continue
                    b = ni[idx(ii, jj, kk)]
                    r = np.array([dx, dy, dz], np.float32)
                    ra, rb, ab = f(np.dot(a, r)), f(np.dot(b, r)), f(np.dot(a, b))
                    sv += 0.5 * (b.astype(np.float64) * rb - a * ra + a * ab * rb - b * ab * ra).astype(np.float32)
                    nB += 1
                div = 0.0  # parameter_order.cpp:192-210
                for ax in range(3):
                    dd, cnt = 0.0, 0
                    for s in (-1, 1):
                        c = [i, j, k]
                        c[ax] += s
                        ii, jj, kk = _nb(c[0], Nx, periodic[0]), _nb(c[1], Ny, periodic[1]), _nb(c[2], Nz, periodic[2])
                        if ii is None or jj is None or kk is None or not pt[idx(ii, jj, kk)]:
                            continue
                        dd += float(f(s) * f(ni[idx(ii, jj, kk)][ax] - a[ax]))
                        cnt += 1
                    if cnt:
                        div += dd / cnt
                sdiv += div
                vdiv += 1
                for cyl in (False, True):  # parameter_order.cpp:225-240
                    rx, ry, rz = f(i) - cx, f(j) - cy, (f(0) if cyl else f(k) - cz)
                    r = f(np.sqrt(f(rx * rx + ry * ry + rz * rz)))
                    if r < 0.5:
                        continue
                    c = float(f(f(a[0] * rx + a[1] * ry + a[2] * rz) / r))
                    rad[cyl][0] += 1.5 * c * c - 0.5
                    rad[cyl][1] += c
                    rad[cyl][2] += 1
    out = {"P": abs(sP) / vP if vP else 0.0,
           "dtheta": 1.5 * float(np.sqrt(np.dot(sv, sv))) / nB if nB else 0.0,
           "divn": sdiv / vdiv if vdiv else 0.0}
    for cyl, name in ((False, "sph"), (True, "cyl")):
        s_, p_, n_ = rad[cyl]
        out["Sr_" + name] = s_ / n_ if n_ else 0.0
        out["Pr_" + name] = p_ / n_ if n_ else 0.0
    return out


def local_S(ni, pt, shape, periodic, i, j, k):
    """lattice_order_parameter (src/parameter_order.cpp:75-127): Q over the site and its present neighbours in the
    reference's visiting order, float accumulation, largest eigenvalue in double."""
    Nx, Ny, Nz = shape
    ni = np.asarray(ni, np.float32).reshape(-1, 3)
    f = np.float32
    Q = np.zeros(9, np.float32)
    points = 0
    for di in (-1, 0, 1):
        for dj in (-1, 0, 1):
            for dk in (-1, 0, 1):
                if abs(di) + abs(dj) + abs(dk) > 1:
                    continue
                ii, jj, kk = _nb(i + di, Nx, periodic[0]), _nb(j + dj, Ny, periodic[1]), _nb(k + dk, Nz, periodic[2])
                if ii is None or jj is None or kk is None:
                    continue
                q = ii + Nx * (jj + Ny * kk)
                if not pt[q]:
                    continue
                for l in range(3):
                    for m in range(l + 1):
                        Q[3 * m + l] = f(float(Q[3 * m + l]) + 3.0 * float(f(ni[q][l] * ni[q][m])))
                    Q[4 * l] = f(Q[4 * l] - f(1))
                points += 1
    den = 2.0 * points
    q = [float(f(float(Q[c]) / den)) for c in (0, 1, 2, 4, 5, 8)]
    m = np.array([[q[0], q[1], q[2]], [q[1], q[3], q[4]], [q[2], q[4], q[5]]])
    return float(np.linalg.eigvalsh(m)[-1])
