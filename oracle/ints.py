"""CPU restatement of the one-electron integrals nAPMO takes from libint
(test infrastructure only): overlap, kinetic energy and nuclear attraction
over unit-normalised contracted Cartesian Gaussians
(src/ints/libint_iface.cpp:55-190 renormalises every function; nAPMO's own
primitive overlap is src/ints/overlap.cpp:12-64).

McMurchie-Davidson by direct recursion (Helgaker, Jorgensen, Olsen, Molecular
Electronic-Structure Theory, eqs. 9.5.6-9.5.7, 9.9.18-9.9.20), the Boys
function from the confluent hypergeometric identity
F_m(T) = 1F1(m + 1/2; m + 3/2; -T) / (2m + 1) (scipy).  Pinned by nAPMO's
compiled ContractedGaussian_overlap (tests/golden/reference_vectors.npz,
'ints_*_S') and by the H2/STO-3G values of Szabo and Ostlund, Modern Quantum
Chemistry, section 3.5.2.
"""
import math

import numpy as np
from scipy.special import hyp1f1

import oracle as O


def boys(m, T):
    return hyp1f1(m + 0.5, m + 1.5, -T) / (2 * m + 1)


def _E(i, j, t, PA, PB, p):
    if t < 0 or t > i + j or i < 0 or j < 0:
        return 0.0
    if i == 0 and j == 0:
        return 1.0
    if j == 0:
        return (_E(i - 1, 0, t - 1, PA, PB, p) / (2 * p) + PA * _E(i - 1, 0, t, PA, PB, p)
                + (t + 1) * _E(i - 1, 0, t + 1, PA, PB, p))
    return (_E(i, j - 1, t - 1, PA, PB, p) / (2 * p) + PB * _E(i, j - 1, t, PA, PB, p)
            + (t + 1) * _E(i, j - 1, t + 1, PA, PB, p))


def _R(t, u, v, n, p, PC, cache):
    key = (t, u, v, n)
    if key in cache:
        return cache[key]
    if t < 0 or u < 0 or v < 0:
        return 0.0
    if t == 0 and u == 0 and v == 0:
        r = (-2 * p) ** n * boys(n, p * float(PC @ PC))
    elif t > 0:
        r = (t - 1) * _R(t - 2, u, v, n + 1, p, PC, cache) + PC[0] * _R(t - 1, u, v, n + 1, p, PC, cache)
    elif u > 0:
        r = (u - 1) * _R(t, u - 2, v, n + 1, p, PC, cache) + PC[1] * _R(t, u - 1, v, n + 1, p, PC, cache)
    else:
        r = (v - 1) * _R(t, u, v - 2, n + 1, p, PC, cache) + PC[2] * _R(t, u, v - 1, n + 1, p, PC, cache)
    cache[key] = r
    return r


def primitive(la, A, a, lb, B, b, charges):
    """(S, T, V) of x_A^la e^{-a r_A^2} and x_B^lb e^{-b r_B^2} (unnormalised)."""
    A, B = np.asarray(A, float), np.asarray(B, float)
    p = a + b
    P = (a * A + b * B) / p
    K = math.exp(-a * b / p * float((A - B) @ (A - B)))
    PA, PB = P - A, P - B
    s = [_E(la[d], lb[d], 0, PA[d], PB[d], p) * math.sqrt(math.pi / p) for d in range(3)]
    t = []
    for d in range(3):
        j = lb[d]
        sp = _E(la[d], j + 2, 0, PA[d], PB[d], p) * math.sqrt(math.pi / p)
        sm = _E(la[d], j - 2, 0, PA[d], PB[d], p) * math.sqrt(math.pi / p) if j >= 2 else 0.0
        t.append(-2 * b * b * sp + b * (2 * j + 1) * s[d] - 0.5 * j * (j - 1) * sm)
    S = K * s[0] * s[1] * s[2]
    T = K * (t[0] * s[1] * s[2] + s[0] * t[1] * s[2] + s[0] * s[1] * t[2])
    V = 0.0
    for (Z, C) in charges:
        PC = P - np.asarray(C, float)
        cache = {}
        acc = 0.0
        for tt in range(la[0] + lb[0] + 1):
            for uu in range(la[1] + lb[1] + 1):
                for vv in range(la[2] + lb[2] + 1):
                    acc += (_E(la[0], lb[0], tt, PA[0], PB[0], p) *
                            _E(la[1], lb[1], uu, PA[1], PB[1], p) *
                            _E(la[2], lb[2], vv, PA[2], PB[2], p) *
                            _R(tt, uu, vv, 0, p, PC, cache))
        V -= Z * K * 2 * math.pi / p * acc
    return S, T, V


def one_body(fb, charges):
    """(S, T, V) [n][n] of an oracle flat basis (oracle.flat_basis) with every
    function normalised to one; charges = [(Z, (x, y, z))] in bohr."""
    n = fb['nf']
    funcs = []
    for f in range(n):
        l = [int(x) for x in fb['l'][3 * f:3 * f + 3]]
        o = fb['origin'][3 * f:3 * f + 3]
        k0, nk = fb['off'][f], fb['nprim'][f]
        zs = fb['zeta'][k0:k0 + nk]
        cs = [c * O.lib.orc_prim_norm(np.array(l, np.int32), z)
              for c, z in zip(fb['coeff'][k0:k0 + nk], zs)]
        funcs.append((l, o, zs, cs))
    S, T, V = (np.zeros((n, n)) for _ in range(3))
    for i in range(n):
        for j in range(i + 1):
            li, oi, zi, ci = funcs[i]
            lj, oj, zj, cj = funcs[j]
            s = t = v = 0.0
            for a, ca in zip(zi, ci):
                for b, cb in zip(zj, cj):
                    ps, pt, pv = primitive(li, oi, a, lj, oj, b, charges)
                    s += ca * cb * ps
                    t += ca * cb * pt
                    v += ca * cb * pv
            S[i, j] = S[j, i] = s
            T[i, j] = T[j, i] = t
            V[i, j] = V[j, i] = v
    nrm = 1.0 / np.sqrt(np.diag(S).copy())
    return tuple(M * nrm[:, None] * nrm[None, :] for M in (S, T, V))
