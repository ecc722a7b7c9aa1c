"""CPU restatement of the int8-slice contractions of napmo_b200/csrc/tc.cu.

Test infrastructure only: the GPU tests check that the tensor-core kernels
compute exactly this scheme (integer parts exact, FP64 sums reordered) and,
separately, how far the scheme is from the FP64 path.  nAPMO has no mixed
precision, so this file restates the library's own scheme, not nAPMO code.

Point screening (screen()): the int8 mode keeps only the points whose
weight can matter and runs both contractions on those points, compacted in
grid order; rho is 0 at the others.

Scheme: the values x of a group (one basis function over 1024 points for the
quadrature; all basis functions at one point, and one row of D, for the
density) share e = frexp exponent of max |x| (clamped at -960); each value is
rounded to Y = rint(x 2^(30-e)) and written in balanced base 256 as
Y = d0 2^24 + d1 2^16 + d2 2^8 + d3.  Products keep d_i d'_j for
i + j <= 4.  The quadrature splits the weight
by c(p) = floor(log2 |wb w| / 2): A = phi 2^c, B = A wv 2^-2c (from A's
integers, see quadrature()).
"""
import numpy as np

EMIN = -960
BLOCK = 1024


def group_exponent(m):
    m = np.asarray(m, dtype=np.float64)
    e = np.frexp(m)[1].astype(np.int64)
    e = np.where(m > 0, e, 0)
    return np.maximum(e, EMIN)


def digits(x, e, ns=4):
    """ns balanced base-256 digits (most significant first) of
    rint(x 2^(8 ns - 2 - e)); e broadcasts against x."""
    Y = np.rint(np.ldexp(np.asarray(x, np.float64),
                         (8 * ns - 2 - e).astype(np.int64))).astype(np.int64)
    out = []
    for _ in range(ns - 1):
        d = ((Y + 128) & 255) - 128
        out.append(d)
        Y = (Y - d) >> 8
    out.append(Y)
    return out[::-1]


def balance(wb, w):
    """sc = 2^c, isc = 2^-c with c = floor(log2 |wb w| / 2) (0 for t = 0;
    Lebedev rules with negative weights keep the sign in wv)."""
    t = np.abs(np.asarray(wb, np.float64) * np.asarray(w, np.float64))
    ex = np.frexp(t)[1].astype(np.int64)
    c = np.where((t > 0) & (t < 1e300), (ex - 1) >> 1, 0)
    c = np.clip(c, -400, 400)
    return np.ldexp(1.0, c), np.ldexp(1.0, -c)


def _combine(acc, ndiag):
    comb = np.zeros_like(acc[0], dtype=np.float64)
    # int64 combination as the kernels do: ((acc0 * 256 + acc1) * 256 + ...)
    c = acc[0].astype(np.int64)
    for d in range(1, ndiag):
        c = c * 256 + acc[d].astype(np.int64)
    comb[...] = c.astype(np.float64)
    return comb


def quadrature(phi, wv, wb, w, block=BLOCK):
    """F[mu][nu] = sum_p phi[mu][p] wv[p] phi[nu][p], int8 slices, i + j <= 4.
    phi [n][N]; wv, wb, w [N].  A = phi 2^c is sliced per (row, block); B is
    derived from A's integers: g = wv 2^-2c, eg = block exponent of g,
    gs = g 2^-eg, x = Y_A gs, Y_B = rint(x 2^s) with s = 30 - (block exponent
    of max |x| of the row), and B's exponent e_A + eg - s."""
    phi = np.asarray(phi, np.float64)
    n, N = phi.shape
    sc, isc = balance(wb, w)
    A = phi * sc
    g = np.asarray(wv, np.float64) * isc * isc
    F = np.zeros((n, n))
    for b0 in range(0, N, block):
        a = A[:, b0:b0 + block]
        gb = g[b0:b0 + block]
        ea = group_exponent(np.abs(a).max(axis=1))
        eg = int(group_exponent(np.abs(gb).max()))
        gs = gb * np.ldexp(1.0, -eg)
        da = digits(a, ea[:, None])
        Ya = ((da[0] * 256 + da[1]) * 256 + da[2]) * 256 + da[3]
        x = Ya.astype(np.float64) * gs
        sh = 30 - group_exponent(np.abs(x).max(axis=1))
        Yb = np.rint(x * np.ldexp(1.0, sh)[:, None]).astype(np.int64)
        db = []
        for _ in range(3):
            d = ((Yb + 128) & 255) - 128
            db.append(d)
            Yb = (Yb - d) >> 8
        db.append(Yb)
        db = db[::-1]
        eb = ea + eg - sh
        acc = [np.zeros((n, n)) for _ in range(5)]
        for i in range(4):
            for j in range(4):
                if i + j <= 4:
                    acc[i + j] += da[i].astype(np.float64) @ db[j].T.astype(np.float64)
        comb = _combine([np.rint(x).astype(np.int64) for x in acc], 5)
        F += comb * np.ldexp(1.0, (ea[:, None] + eb[None, :] - 44))
    return np.triu(F) + np.triu(F, 1).T


DENS_BLOCK, DENS_STAGE = 96, 64
SCREEN_TOL = 1e-24


def screen(phi, wb, w, tol=SCREEN_TOL):
    """Points kept by the int8 mode's screening: (|wb w| max_mu |phi_mu|)
    max_mu |phi_mu| >= tol, in that order of products (boolean [N])."""
    mx = np.abs(np.asarray(phi, np.float64)).max(axis=0)
    t = np.abs(np.asarray(wb, np.float64) * np.asarray(w, np.float64))
    return (t * mx) * mx >= tol


def fold_density_matrix(D):
    """D' with sum D' phi phi = sum D phi phi and zeros below each block's
    first stage: function block m = mu // 96 accumulates nu >= c(mu) =
    64 ((96 m) // 64); D'[mu][nu] = D[mu][nu] + D[nu][mu] where the mirror
    entry lies below its own block's cut (mu < c(nu)), D[mu][nu] otherwise."""
    D = np.asarray(D, np.float64)
    n = D.shape[0]
    idx = np.arange(n)
    c = (idx // DENS_BLOCK) * DENS_BLOCK // DENS_STAGE * DENS_STAGE
    keep = idx[None, :] >= c[:, None]                  # nu >= c(mu)
    mirror = keep & (idx[:, None] < c[None, :])        # mu < c(nu)
    return np.where(keep, D + np.where(mirror, D.T, 0.0), 0.0)


def density(phi, D):
    """rho[p] = sum_{mu,nu} D[mu][nu] phi[mu][p] phi[nu][p], int8 slices
    (phi 4 digits per point, D' = fold_density_matrix(D) 5 digits per row),
    i + j <= 4.  phi [n][N], D [n][n]."""
    phi = np.asarray(phi, np.float64)
    D = fold_density_matrix(D)
    ep = group_exponent(np.abs(phi).max(axis=0))      # per point
    eD = group_exponent(np.abs(D).max(axis=1))        # per row of D
    dp = digits(phi, ep[None, :])
    dD = digits(D, eD[:, None], ns=5)                 # D: 5 digits, 2^(38-e)
    acc = [np.zeros(phi.shape) for _ in range(5)]     # T[mu][p] diagonals
    for i in range(4):
        for j in range(5):
            if i + j <= 4:
                acc[i + j] += dD[j].astype(np.float64) @ dp[i].astype(np.float64)
    comb = _combine([np.rint(x).astype(np.int64) for x in acc], 5)
    yphi = ((dp[0] * 256 + dp[1]) * 256 + dp[2]) * 256 + dp[3]
    s = (yphi.astype(np.float64) * np.ldexp(1.0, eD)[:, None] * comb).sum(axis=0)
    return s * np.ldexp(1.0, ep - 37) * np.ldexp(1.0, ep - 37)
