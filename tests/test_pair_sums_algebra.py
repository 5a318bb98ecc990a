"""The element-pair kernel's per-trial-point sums (sym_pairs_kernel, assembly.cu)
reproduce the direct per-point-pair Burton-Miller combination, in FP64 on the
CPU (no GPU).

The direct form is the combination the reference forms per point pair
(src/BeatEngineCpuBurtonMiller.jl:53-167): for test point x on face tau and
trial point y on face sigma, G = exp(ikr) / (4 pi r), order 1's kernel value
-dG/dn_y - i eta k^2 (n_tau . n_sigma) G against phi_a(x) phi_b(y), order 2's
(tau and sigma swapped) likewise, and the right-hand-side values
-G - i eta dG/dn_x of each order against the test basis.  The kernel instead
accumulates, per test point, three basis-weighted sums over the trial points
(w G, w G'/r and w (r . n_tau) G'/r) and forms both orders' blocks, both
right-hand-side blocks and the curl term's Green sum from them.  Both are
evaluated here for random well-separated triangles and compared entry by
entry.
"""
import numpy as np
import pytest

A4, B4 = 0.445948490915965, 0.091576213509771
PTS = np.array([[A4, A4], [1 - 2 * A4, A4], [A4, 1 - 2 * A4], [B4, B4], [1 - 2 * B4, B4], [B4, 1 - 2 * B4]])
W = np.array([0.223381589678011] * 3 + [0.109951743655322] * 3)
PHI = np.stack([1 - PTS[:, 0] - PTS[:, 1], PTS[:, 0], PTS[:, 1]], 1)  # Q x 3 basis values
INV4PI = 1.0 / (4.0 * np.pi)


def triangle(rng, shift):
    v = rng.standard_normal((3, 3)) + shift
    e1, e2 = v[1] - v[0], v[2] - v[0]
    n = np.cross(e1, e2)
    n /= np.linalg.norm(n)
    return v, n, v[0] + PTS[:, :1] * e1 + PTS[:, 1:] * e2


def direct(X, Y, nt, ns, k, eta):
    """Per point pair: both orders' 3 x 3 blocks, both right-hand-side
    3-vectors (order 1: rows tau, order 2: rows sigma), the Green sum."""
    k2n = eta * k * k * (nt @ ns)
    L1 = np.zeros((3, 3), complex)
    L2 = np.zeros((3, 3), complex)
    R1 = np.zeros(3, complex)
    R2 = np.zeros(3, complex)
    gsum = 0j
    for qt in range(6):
        for qs in range(6):
            r = Y[qs] - X[qt]
            rr = np.linalg.norm(r)
            w = W[qt] * W[qs] * INV4PI
            g = w * np.exp(1j * k * rr) / rr
            dg = g * (1j * k - 1.0 / rr)  # dG/dr
            dn_y = dg * (r @ ns) / rr       # dG/dn_sigma at y
            dn_x = -dg * (r @ nt) / rr      # dG/dn_tau at x
            # order 1 (test tau, trial sigma) and order 2 (test sigma, trial tau)
            L1 += np.outer(PHI[qt], PHI[qs]) * (-dn_y - 1j * k2n * g)
            L2 += np.outer(PHI[qs], PHI[qt]) * (-dn_x - 1j * k2n * g)
            R1 += PHI[qt] * (-g - 1j * eta * dn_x)
            R2 += PHI[qs] * (-g - 1j * eta * dn_y)
            gsum += g
    return L1, L2, R1, R2, gsum


def kernel_sums(X, Y, nt, ns, k, eta):
    """The kernel's formulation (three packed sums per trial point)."""
    k2n = eta * k * k * (nt @ ns)
    dtau, dsig = X[0] @ nt, Y[0] @ ns
    ync = Y @ nt - dtau  # r . n_tau per trial point, the same for every x on tau
    L1 = np.zeros((3, 3), complex)
    L2 = np.zeros((3, 3), complex)
    R1 = np.zeros(3, complex)
    TC = np.zeros(3, complex)
    for qt in range(6):
        x = X[qt]
        wt = W[qt] * INV4PI
        xns = dsig - x @ ns  # r . n_sigma, the same for every y on sigma
        C = np.zeros(3, complex)
        H = np.zeros(3, complex)
        P = np.zeros(3, complex)
        for qs in range(6):
            r = Y[qs] - x
            ir = 1.0 / np.linalg.norm(r)
            g = W[qs] * np.exp(1j * k / ir) * ir
            h = g * (1j * k - ir) * ir
            C += PHI[qs] * g
            H += PHI[qs] * h
            P += PHI[qs] * ync[qs] * h
        U = -C.sum() + 1j * eta * P.sum()
        S = -xns * H - 1j * k2n * C
        P = P - 1j * k2n * C
        TC += wt * C
        ba = PHI[qt] * wt
        L1 += np.outer(ba, S)
        L2 += np.outer(P, ba)
        R1 += ba * U
    R2 = -(1 + eta * k2n) * TC + 1j * eta * L1.sum(axis=0)
    return L1, L2, R1, R2, TC.sum()


@pytest.mark.parametrize("seed,k,eta_sign", [(1, 7.3, 1.0), (2, 36.6, 1.0), (3, 110.0, -1.0), (4, 0.5, 1.0)])
def test_kernel_sums_equal_direct_combination(seed, k, eta_sign):
    rng = np.random.default_rng(seed)
    _, nt, X = triangle(rng, 0.0)
    _, ns, Y = triangle(rng, 3.0)
    eta = eta_sign / k
    for a, b, name in zip(direct(X, Y, nt, ns, k, eta), kernel_sums(X, Y, nt, ns, k, eta),
                          ("L1", "L2", "R1", "R2", "Green sum")):
        scale = np.max(np.abs(a))
        assert np.max(np.abs(a - b)) <= 1e-13 * scale, name
