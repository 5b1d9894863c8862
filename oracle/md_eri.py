"""Independent McMurchie-Davidson ERI (numpy/scipy) -- test infrastructure.

A second, algorithmically unrelated check of the oracle: Hermite expansion
coefficients E_t^{ij} and Hermite Coulomb integrals R_{tuv}, with the Boys
function from scipy's regularised incomplete gamma function.  Pure-Python
loops: small cases only.  Nothing from the reference is restated here; it
pins the mathematics the reference's recurrences implement.
"""
from math import pi, sqrt

import numpy as np
from scipy.special import gammainc, gamma


def boys(n, T):
    if T < 1e-12:
        return 1.0 / (2 * n + 1) - T / (2 * n + 3)
    return gamma(n + 0.5) * gammainc(n + 0.5, T) / (2.0 * T ** (n + 0.5))


def hermite_E(i, j, Xab, a, b):
    """E_t^{ij} for t = 0..i+j (1D, with the Gaussian product factor)."""
    p = a + b
    mu = a * b / p
    Xpa = -b / p * Xab
    Xpb = a / p * Xab
    E = np.zeros((i + 1, j + 1, i + j + 2))
    E[0, 0, 0] = np.exp(-mu * Xab * Xab)
    for ii in range(i + 1):
        for jj in range(j + 1):
            if ii == 0 and jj == 0:
                continue
            for t in range(ii + jj + 1):
                if ii > 0:
                    v = Xpa * E[ii - 1, jj, t]
                    if t > 0:
                        v += E[ii - 1, jj, t - 1] / (2 * p)
                    v += (t + 1) * E[ii - 1, jj, t + 1]
                else:
                    v = Xpb * E[ii, jj - 1, t]
                    if t > 0:
                        v += E[ii, jj - 1, t - 1] / (2 * p)
                    v += (t + 1) * E[ii, jj - 1, t + 1]
                E[ii, jj, t] = v
    return E[i, j, :i + j + 1]


def hermite_R(tmax, alpha, PQ):
    """R_{tuv} (n = 0) for t+u+v <= tmax."""
    T = alpha * float(PQ @ PQ)
    R = np.zeros((tmax + 1, tmax + 1, tmax + 1, tmax + 1))  # [n][t][u][v]
    for n in range(tmax + 1):
        R[n, 0, 0, 0] = (-2 * alpha) ** n * boys(n, T)
    for s in range(1, tmax + 1):
        for n in range(tmax - s + 1):
            for t in range(s + 1):
                for u in range(s - t + 1):
                    v = s - t - u
                    if t > 0:
                        val = PQ[0] * R[n + 1, t - 1, u, v] + ((t - 1) * R[n + 1, t - 2, u, v] if t > 1 else 0.0)
                    elif u > 0:
                        val = PQ[1] * R[n + 1, t, u - 1, v] + ((u - 1) * R[n + 1, t, u - 2, v] if u > 1 else 0.0)
                    else:
                        val = PQ[2] * R[n + 1, t, u, v - 1] + ((v - 1) * R[n + 1, t, u, v - 2] if v > 1 else 0.0)
                    R[n, t, u, v] = val
    return R[0]


def cart_comps(l):
    return [(mx, my, l - mx - my) for mx in range(l, -1, -1) for my in range(l - mx, -1, -1)]


def prim_eri(la, lb, lc, ld, a, b, c, d, A, B, C, D):
    """Primitive Cartesian (ab|cd) block [ia][ib][ic][id] (unnormalised)."""
    p, q = a + b, c + d
    P = (a * A + b * B) / p
    Q = (c * C + d * D) / q
    alpha = p * q / (p + q)
    R = hermite_R(la + lb + lc + ld, alpha, P - Q)
    Eab = [[[hermite_E(i, j, A[k] - B[k], a, b) for j in range(lb + 1)] for i in range(la + 1)] for k in range(3)]
    Ecd = [[[hermite_E(i, j, C[k] - D[k], c, d) for j in range(ld + 1)] for i in range(lc + 1)] for k in range(3)]
    pref = 2 * pi ** 2.5 / (p * q * sqrt(p + q))
    ca, cb, cc, cd = cart_comps(la), cart_comps(lb), cart_comps(lc), cart_comps(ld)
    out = np.zeros((len(ca), len(cb), len(cc), len(cd)))
    for ia, ea in enumerate(ca):
        for ib, eb in enumerate(cb):
            ex, ey, ez = (Eab[k][ea[k]][eb[k]] for k in range(3))
            for ic, ec in enumerate(cc):
                for id_, ed in enumerate(cd):
                    fx, fy, fz = (Ecd[k][ec[k]][ed[k]] for k in range(3))
                    s = 0.0
                    for t in range(len(ex)):
                        for u in range(len(ey)):
                            for v in range(len(ez)):
                                e1 = ex[t] * ey[u] * ez[v]
                                if e1 == 0.0:
                                    continue
                                for tau in range(len(fx)):
                                    for nu in range(len(fy)):
                                        for phi in range(len(fz)):
                                            sgn = -1.0 if (tau + nu + phi) % 2 else 1.0
                                            s += e1 * sgn * fx[tau] * fy[nu] * fz[phi] * R[t + tau, u + nu, v + phi]
                    out[ia, ib, ic, id_] = pref * s
    return out


def contracted_eri(shells):
    """shells: four (l, exps, coefs, centre) tuples; returns the Cartesian block
    flattened with a fastest (ia + na*(ib + nb*(ic + nc*id)))."""
    (la, xa, ca, A), (lb, xb, cb, B), (lc, xc, cc, C), (ld, xd, cd, D) = shells
    acc = None
    for i, a in enumerate(xa):
        for j, b in enumerate(xb):
            for k, c in enumerate(xc):
                for m, d in enumerate(xd):
                    blk = ca[i] * cb[j] * cc[k] * cd[m] * prim_eri(la, lb, lc, ld, a, b, c, d,
                                                                   np.asarray(A), np.asarray(B),
                                                                   np.asarray(C), np.asarray(D))
                    acc = blk if acc is None else acc + blk
    return acc.transpose(3, 2, 1, 0).ravel()
