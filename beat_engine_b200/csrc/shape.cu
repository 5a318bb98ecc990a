// shape.cu -- gradient of a far-field functional with respect to the vertex
// positions (shape derivative), by reverse-mode differentiation of the
// discrete assembly, far field and identity terms.
//
// No counterpart in the reference (it computes no gradients).  With the
// forward model of the admittance/adjoint code,
//     A' p = B q0,  q = q0 - diag(a) P p,  p_inf = Fp p + Fq q,
// and g = dJ/d conj(p_inf), z = A'^-H E^H g (E = Fp - Fq diag(a) P, the
// adjoint solve), a real functional J changes with the vertices X as
//     dJ = 2 Re[ g^H (dFp p + dFq q) + z^H (dB q - dA p) ],
// A, B, Fp, Fq being the only operators that depend on X.  Every term is a sum
// over element pairs (or faces) of quadrature-point contributions, so the
// gradient is accumulated in one reverse pass per term:
//   * point pair (x on the test face, y on the trial face, rule weight w):
//     the pair's contribution to z^H (dB q - dA p) is
//         w [G alpha + G' beta],   G = exp(ik|r|) / (4 pi |r|), G' = dG/d|r|,
//         alpha = eta (S2 - k^2 (n_t . n_s) S1) - S3,
//         beta  = -(S1 (r . n_s) / |r| + eta S3 (-(r . n_t) / |r|)),
//     with S1 = sum_ij W_ij phi_i(x) phi_j(y), S2 = sum_ij W_ij curl_i . curl_j,
//     S3 = sum_i U_i phi_i(x), W_ij = -sum_r conj(z_ri) p_rj, U_i = sum_r
//     conj(z_ri) q_r(s); its derivatives with respect to x, y, the normals,
//     the curls and the pair Jacobian 4 A_t A_s are formed per point;
//   * far field: each source's contribution w E(d) [(-ik)(d . n) p - q];
//   * identity: 1/2 M and -1/2 eta M_p1dp0 scale with the face area.
// All chain-rule factors past a point are real (geometry), so each face
// collects the real parts of its adjoints in a 22-double record
// (three vertex positions, normal, three curls, area), and a last per-face
// pass maps the normal, curls and area to the vertices by forward-mode
// derivatives of the face geometry (normal = e1 x e2 / |e1 x e2|, area, and
// curl_i = n x grad phi_i through the Gram inverse, as the assembly's set-up
// computes them).  FP64 throughout.
//
// Symmetry images.  Each image pass of the assembly integrates every
// (test, reflected trial) element pair by the regular rule, touching or not;
// the reflected trial element has its points and normal times the image's
// signs s and its curls times det s.  The touching image pairs then add the
// Duffy integral minus that regular one.  The reverse passes repeat both on the
// same reflected geometry, and map the trial face's adjoints back through the
// reflection (positions and normal times s, curls times det s: s is its own
// inverse).  The far field's image sources (reflected positions and normals,
// the same densities) are mapped back the same way.  The rows of vertices on a
// symmetry plane are weighted after assembly, so every test-vertex row of the
// adjoint z is taken times that weight.  In the x and xy modes a vertex on a
// symmetry plane must stay on it, so its gradient's component normal to that
// plane is returned as zero (the ground mode's plane has no weights and no
// such constraint).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "internal.cuh"
#include "phase.cuh"

namespace bb {

constexpr int SG_REC = 22;                               // per-face adjoint record
constexpr int SG_V = 0, SG_N = 9, SG_C = 12, SG_A = 21;  // vertices [a][k], normal, curls [i][k], area
constexpr int SG_TT = 64, SG_VT = 80, SG_TS = 16, SG_VS = 32;  // the FP64 test / trial tilings
constexpr int SG_THREADS = 256;
constexpr int SG_RC = 16;  // right-hand sides per pass

struct ShapeRule {
    int n;
    double w[8];
    double b[8][3];
};

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 cscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
__device__ __forceinline__ double2 times_i_eta(double2 a, double eta) { return make_double2(-eta * a.y, eta * a.x); }

// adjoints of one element pair, real parts (jac not yet applied)
struct PairAdj {
    double xbar[3][3], ybar[3][3];  // test / trial vertex positions
    double ntbar[3], nsbar[3];
    double2 phi;                    // sum of the contributions (complex)
    double2 gsum;                   // sum of w G (complex)
};

__device__ __forceinline__ void pair_adj_zero(PairAdj &a) {
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int k = 0; k < 3; ++k) a.xbar[i][k] = a.ybar[i][k] = 0.0;
#pragma unroll
    for (int k = 0; k < 3; ++k) a.ntbar[k] = a.nsbar[k] = 0.0;
    a.phi = a.gsum = make_double2(0.0, 0.0);
}

// one point pair: x = sum bt_a X_a on the test face, y = sum bs_b Y_b on the trial face
__device__ __forceinline__ void reverse_point(const double (&x)[3], const double (&y)[3], const double (&bt)[3],
                                              const double (&bs)[3], double w, const double (&nt)[3],
                                              const double (&ns)[3], double nn, double k, double eta,
                                              const double2 (&W)[3][3], const double2 (&U)[3], double2 S2,
                                              PairAdj &acc) {
    const double r[3] = {y[0] - x[0], y[1] - x[1], y[2] - x[2]};
    const double r2 = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
    if (r2 == 0.0) return;
    const double iR = rsqrt(r2), R = r2 * iR;
    const double rh[3] = {r[0] * iR, r[1] * iR, r[2] * iR};
    double sn_, cs_;
    sincos_cw(k * R, &sn_, &cs_);
    const double gsc = w * 0.07957747154594767 * iR;
    const double2 G = make_double2(cs_ * gsc, sn_ * gsc);
    const double2 f = make_double2(-iR, k);                          // ik - 1/R
    const double2 gs = cmul(G, f);                                   // dG/dR
    const double2 dgs = cmul(G, make_double2(2.0 * iR * iR - k * k, -2.0 * k * iR));  // G ((ik - 1/R)^2 + 1/R^2)
    const double a = rh[0] * ns[0] + rh[1] * ns[1] + rh[2] * ns[2];
    const double c = -(rh[0] * nt[0] + rh[1] * nt[1] + rh[2] * nt[2]);
    double2 S1 = make_double2(0.0, 0.0), S3 = make_double2(0.0, 0.0);
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const double2 wi = cadd(cadd(cscale(W[i][0], bs[0]), cscale(W[i][1], bs[1])), cscale(W[i][2], bs[2]));
        S1 = cadd(S1, cscale(wi, bt[i]));
        S3 = cadd(S3, cscale(U[i], bt[i]));
    }
    const double2 etaS3 = times_i_eta(S3, eta);
    // alpha = eta (S2 - k^2 nn S1) - S3, beta = -(S1 a + eta S3 c)
    const double2 inner = make_double2(S2.x - k * k * nn * S1.x, S2.y - k * k * nn * S1.y);
    const double2 alpha = make_double2(-eta * inner.y - S3.x, eta * inner.x - S3.y);
    const double2 beta = make_double2(-(S1.x * a + etaS3.x * c), -(S1.y * a + etaS3.y * c));
    acc.phi = cadd(acc.phi, cadd(cmul(G, alpha), cmul(gs, beta)));
    acc.gsum = cadd(acc.gsum, G);
    const double phR = cmul(alpha, gs).x + cmul(beta, dgs).x;  // real parts
    const double pha = -cmul(gs, S1).x;
    const double phc = -cmul(gs, etaS3).x;
    const double phnn = -k * k * cmul(G, times_i_eta(S1, eta)).x;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const double dr = phR * rh[d] + pha * (ns[d] - a * rh[d]) * iR - phc * (nt[d] + c * rh[d]) * iR;
#pragma unroll
        for (int v = 0; v < 3; ++v) {
            acc.ybar[v][d] += bs[v] * dr;
            acc.xbar[v][d] -= bt[v] * dr;
        }
        acc.nsbar[d] += pha * rh[d] + phnn * nt[d];
        acc.ntbar[d] += -phc * rh[d] + phnn * ns[d];
    }
}

// W, U of a pair from conj(z) rows of the test vertices, p rows of the trial
// vertices and the trial face's q, for rc columns
__device__ __forceinline__ void pair_weights(const double2 *zt0, const double2 *zt1, const double2 *zt2,
                                             const double2 *ps0, const double2 *ps1, const double2 *ps2,
                                             const double2 *qs, int rc, double2 (&W)[3][3], double2 (&U)[3]) {
    const double2 *zt[3] = {zt0, zt1, zt2}, *pp[3] = {ps0, ps1, ps2};
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        U[i] = make_double2(0.0, 0.0);
#pragma unroll
        for (int j = 0; j < 3; ++j) W[i][j] = make_double2(0.0, 0.0);
    }
    for (int r = 0; r < rc; ++r) {
        const double2 q = qs[r];
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            const double2 zc = make_double2(zt[i][r].x, -zt[i][r].y);
            U[i] = cadd(U[i], cmul(zc, q));
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                const double2 m = cmul(zc, pp[j][r]);
                W[i][j] = make_double2(W[i][j].x - m.x, W[i][j].y - m.y);
            }
        }
    }
}

// the pair's curl term and its record updates (jac applied): curls of the
// test face ct[i][k], of the trial face cs[j][k]
__device__ __forceinline__ double2 curl_term(const double2 (&W)[3][3], const double *ct, const double *cs) {
    double2 S2 = make_double2(0.0, 0.0);
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            const double d = ct[3 * i] * cs[3 * j] + ct[3 * i + 1] * cs[3 * j + 1] + ct[3 * i + 2] * cs[3 * j + 2];
            S2 = cadd(S2, cscale(W[i][j], d));
        }
    return S2;
}

// The trial element of an image pass is reflected: positions and normal
// times s, curls times det s (on = 0: the mesh itself, s = 1, det = 1).
struct ShapeImage {
    int on;
    double s[3];
    double det;
};
__host__ __device__ inline ShapeImage no_image() { return ShapeImage{0, {1.0, 1.0, 1.0}, 1.0}; }

// adds a pair's adjoints (times jac) to the two face records; the trial
// face's adjoints, taken with respect to its reflected copy im, are mapped
// back to the face itself
__device__ __forceinline__ void pair_records(const PairAdj &acc, const double2 (&W)[3][3], const double *ct,
                                             const double *cs, double jac, double at, double as, double eta,
                                             double *rt, double *rs, const ShapeImage &im) {
#pragma unroll
    for (int v = 0; v < 3; ++v)
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            atomicAdd(&rt[SG_V + 3 * v + d], jac * acc.xbar[v][d]);
            atomicAdd(&rs[SG_V + 3 * v + d], jac * acc.ybar[v][d] * im.s[d]);
        }
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        atomicAdd(&rt[SG_N + d], jac * acc.ntbar[d]);
        atomicAdd(&rs[SG_N + d], jac * acc.nsbar[d] * im.s[d]);
    }
    // curls: d phi / d curl_t[i] = jac Gamma sum_j W_ij curl_s[j], Gamma = eta sum w G
    const double2 gam = times_i_eta(acc.gsum, eta);
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            double2 st = make_double2(0.0, 0.0), ss = make_double2(0.0, 0.0);
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                st = cadd(st, cscale(W[i][j], cs[3 * j + d]));
                ss = cadd(ss, cscale(W[j][i], ct[3 * j + d]));
            }
            atomicAdd(&rt[SG_C + 3 * i + d], jac * cmul(gam, st).x);
            atomicAdd(&rs[SG_C + 3 * i + d], jac * cmul(gam, ss).x * im.det * im.s[d]);
        }
    // jac = 4 A_t A_s
    atomicAdd(&rt[SG_A], jac * acc.phi.x / at);
    atomicAdd(&rs[SG_A], jac * acc.phi.x / as);
}

struct ShapeTileArgs {
    const double *qpts, *normal, *curl, *area;  // by position (FP64 copies)
    const int *gvert, *face_id;
    const int *t_fstart, *t_vstart, *t_verts, *t_local;
    const int *s_fstart, *s_vstart, *s_verts, *s_local;
    const double2 *z, *p, *q;                   // N x R, N x R, F x R column-major
    int N, F, R, r0;
    double k, eta;
    ShapeRule rule;
    ShapeImage img;                             // the pass's reflection of the trial elements
    double *rec;                                // F x SG_REC
};

// regular (non-touching) pairs: grid = (trial tiles, test tiles)
template <int Q>
__global__ void __launch_bounds__(SG_THREADS, 1) shape_pairs_kernel(ShapeTileArgs g) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2 *zt = reinterpret_cast<double2 *>(smem_raw);  // [SG_VT][SG_RC]
    double2 *ps = zt + SG_VT * SG_RC;                     // [SG_VS][SG_RC]
    double2 *qs = ps + SG_VS * SG_RC;                     // [SG_TS][SG_RC]
    double *tq = reinterpret_cast<double *>(qs + SG_TS * SG_RC);  // [SG_TT][Q][3]
    double *tn = tq + SG_TT * Q * 3, *tc = tn + SG_TT * 3, *ta = tc + SG_TT * 9;
    double *sq = ta + SG_TT, *sn = sq + SG_TS * Q * 3, *sc = sn + SG_TS * 3, *sa = sc + SG_TS * 9;
    double *rt = sa + SG_TS;        // [SG_TT][SG_REC]
    double *rs = rt + SG_TT * SG_REC;  // [SG_TS][SG_REC]
    int *tgv = reinterpret_cast<int *>(rs + SG_TS * SG_REC);  // [SG_TT][3]
    int *tlv = tgv + SG_TT * 3, *sgv = tlv + SG_TT * 3, *slv = sgv + SG_TS * 3;

    const int tid = threadIdx.x;
    const int t0 = g.t_fstart[blockIdx.y], nt = g.t_fstart[blockIdx.y + 1] - t0;
    const int s0 = g.s_fstart[blockIdx.x], ns = g.s_fstart[blockIdx.x + 1] - s0;
    const int tv0 = g.t_vstart[blockIdx.y], nvt = g.t_vstart[blockIdx.y + 1] - tv0;
    const int sv0 = g.s_vstart[blockIdx.x], nvs = g.s_vstart[blockIdx.x + 1] - sv0;
    const int rc = min(SG_RC, g.R - g.r0);
    for (int i = tid; i < SG_VT * SG_RC; i += SG_THREADS) {
        const int v = i / SG_RC, r = i % SG_RC;
        zt[i] = (v < nvt && r < rc) ? g.z[(size_t)(g.r0 + r) * g.N + g.t_verts[tv0 + v]] : make_double2(0, 0);
    }
    for (int i = tid; i < SG_VS * SG_RC; i += SG_THREADS) {
        const int v = i / SG_RC, r = i % SG_RC;
        ps[i] = (v < nvs && r < rc) ? g.p[(size_t)(g.r0 + r) * g.N + g.s_verts[sv0 + v]] : make_double2(0, 0);
    }
    for (int i = tid; i < SG_TS * SG_RC; i += SG_THREADS) {
        const int f = i / SG_RC, r = i % SG_RC;
        qs[i] = (f < ns && r < rc) ? g.q[(size_t)(g.r0 + r) * g.F + g.face_id[s0 + f]] : make_double2(0, 0);
    }
    for (int i = tid; i < nt * Q * 3; i += SG_THREADS) tq[i] = g.qpts[(size_t)t0 * Q * 3 + i];
    for (int i = tid; i < nt * 3; i += SG_THREADS) {
        tn[i] = g.normal[(size_t)t0 * 3 + i];
        tgv[i] = g.gvert[(size_t)t0 * 3 + i];
        tlv[i] = g.t_local[(size_t)t0 * 3 + i];
    }
    for (int i = tid; i < nt * 9; i += SG_THREADS) tc[i] = g.curl[(size_t)t0 * 9 + i];
    for (int i = tid; i < nt; i += SG_THREADS) ta[i] = g.area[t0 + i];
    for (int i = tid; i < ns * Q * 3; i += SG_THREADS) sq[i] = g.qpts[(size_t)s0 * Q * 3 + i];
    for (int i = tid; i < ns * 3; i += SG_THREADS) {
        sn[i] = g.normal[(size_t)s0 * 3 + i];
        sgv[i] = g.gvert[(size_t)s0 * 3 + i];
        slv[i] = g.s_local[(size_t)s0 * 3 + i];
    }
    for (int i = tid; i < ns * 9; i += SG_THREADS) sc[i] = g.curl[(size_t)s0 * 9 + i];
    for (int i = tid; i < ns; i += SG_THREADS) sa[i] = g.area[s0 + i];
    for (int i = tid; i < (SG_TT + SG_TS) * SG_REC; i += SG_THREADS) rt[i] = 0.0;
    __syncthreads();
    if (g.img.on) {  // an image pass: the trial tile reflected
        for (int i = tid; i < ns * Q * 3; i += SG_THREADS) sq[i] *= g.img.s[i % 3];
        for (int i = tid; i < ns * 3; i += SG_THREADS) sn[i] *= g.img.s[i % 3];
        for (int i = tid; i < ns * 9; i += SG_THREADS) sc[i] *= g.img.det * g.img.s[i % 3];
        __syncthreads();
    }

    for (int pr = tid; pr < SG_TT * SG_TS; pr += SG_THREADS) {
        const int tl = pr / SG_TS, sl = pr % SG_TS;
        if (tl >= nt || sl >= ns) continue;
        const int *tv = tgv + 3 * tl, *sv = sgv + 3 * sl;
        if (!g.img.on && (tv[0] == sv[0] || tv[0] == sv[1] || tv[0] == sv[2] || tv[1] == sv[0] || tv[1] == sv[1] ||
                          tv[1] == sv[2] || tv[2] == sv[0] || tv[2] == sv[1] || tv[2] == sv[2]))
            continue;  // touching: the Duffy pass (an image pass keeps every pair, as the assembly does)
        double2 W[3][3], U[3];
        pair_weights(zt + tlv[3 * tl] * SG_RC, zt + tlv[3 * tl + 1] * SG_RC, zt + tlv[3 * tl + 2] * SG_RC,
                     ps + slv[3 * sl] * SG_RC, ps + slv[3 * sl + 1] * SG_RC, ps + slv[3 * sl + 2] * SG_RC,
                     qs + sl * SG_RC, rc, W, U);
        const double *ct = tc + 9 * tl, *cs = sc + 9 * sl;
        const double2 S2 = curl_term(W, ct, cs);
        const double nT[3] = {tn[3 * tl], tn[3 * tl + 1], tn[3 * tl + 2]};
        const double nS[3] = {sn[3 * sl], sn[3 * sl + 1], sn[3 * sl + 2]};
        const double nn = nT[0] * nS[0] + nT[1] * nS[1] + nT[2] * nS[2];
        PairAdj acc;
        pair_adj_zero(acc);
#pragma unroll 1
        for (int qt = 0; qt < Q; ++qt) {
            const double x[3] = {tq[(tl * Q + qt) * 3], tq[(tl * Q + qt) * 3 + 1], tq[(tl * Q + qt) * 3 + 2]};
            const double bt[3] = {g.rule.b[qt][0], g.rule.b[qt][1], g.rule.b[qt][2]};
#pragma unroll 1
            for (int qq = 0; qq < Q; ++qq) {
                const double y[3] = {sq[(sl * Q + qq) * 3], sq[(sl * Q + qq) * 3 + 1], sq[(sl * Q + qq) * 3 + 2]};
                const double bs[3] = {g.rule.b[qq][0], g.rule.b[qq][1], g.rule.b[qq][2]};
                reverse_point(x, y, bt, bs, g.rule.w[qt] * g.rule.w[qq], nT, nS, nn, g.k, g.eta, W, U, S2, acc);
            }
        }
        const double jac = 4.0 * ta[tl] * sa[sl];
        pair_records(acc, W, ct, cs, jac, ta[tl], sa[sl], g.eta, rt + tl * SG_REC, rs + sl * SG_REC, g.img);
    }
    __syncthreads();
    for (int i = tid; i < nt * SG_REC; i += SG_THREADS) {
        const double v = rt[i];
        if (v != 0.0) atomicAdd(&g.rec[(size_t)g.face_id[t0 + i / SG_REC] * SG_REC + i % SG_REC], v);
    }
    for (int i = tid; i < ns * SG_REC; i += SG_THREADS) {
        const double v = rs[i];
        if (v != 0.0) atomicAdd(&g.rec[(size_t)g.face_id[s0 + i / SG_REC] * SG_REC + i % SG_REC], v);
    }
}

template <int Q> static size_t shape_pairs_smem() {
    return sizeof(double2) * (SG_VT + SG_VS + SG_TS) * SG_RC +
           sizeof(double) * ((SG_TT + SG_TS) * (Q * 3 + 3 + 9 + 1) + (SG_TT + SG_TS) * SG_REC) +
           sizeof(int) * (SG_TT + SG_TS) * 6;
}

struct ShapeSingArgs {
    const int *test, *trial, *rule;
    const int *img;           // touching image pairs: the image of each pair (NULL: the mesh's own pairs)
    ShapeImage xf[3];         // the images' reflections
    ShapeRule reg;            // the regular rule an image pass applied to the pair
    const int *rule_start;
    const double *rule_data;  // per point: test xi, eta, trial xi, eta, weight
    const double *verts, *normals, *curls, *areas;
    const int *faces;
    const double2 *z, *p, *q;
    int N, F, R;
    int64_t npairs;
    double k, eta;
    double *rec;
};

// touching pairs: one warp per pair, Duffy points over the lanes, then the
// lanes' adjoints summed and added to the two face records.  A touching image
// pair (test t, trial s reflected) takes the Duffy points on the reflected
// trial element minus the regular rule's points there (the part the image
// pass integrated), and maps the trial face's adjoints back through the
// reflection.
__global__ void __launch_bounds__(256) shape_singular_kernel(ShapeSingArgs g) {
    const int lane = threadIdx.x & 31;
    const int64_t pair = (int64_t)blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
    if (pair >= g.npairs) return;
    const int t = g.test[pair], s = g.trial[pair], ru = g.rule[pair];
    const ShapeImage im = g.img ? g.xf[g.img[pair]] : no_image();
    const int *ft = g.faces + 3 * t, *fs = g.faces + 3 * s;
    double tv[3][3], sv[3][3];
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            tv[a][c] = g.verts[3 * ft[a] + c];
            sv[a][c] = im.s[c] * g.verts[3 * fs[a] + c];
        }
    const double nT[3] = {g.normals[3 * t], g.normals[3 * t + 1], g.normals[3 * t + 2]};
    const double nS[3] = {im.s[0] * g.normals[3 * s], im.s[1] * g.normals[3 * s + 1], im.s[2] * g.normals[3 * s + 2]};
    const double nn = nT[0] * nS[0] + nT[1] * nS[1] + nT[2] * nS[2];
    double2 W[3][3], U[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        U[i] = make_double2(0.0, 0.0);
#pragma unroll
        for (int j = 0; j < 3; ++j) W[i][j] = make_double2(0.0, 0.0);
    }
    for (int r = 0; r < g.R; ++r) {
        const double2 q = g.q[(size_t)r * g.F + s];
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            const double2 zi = g.z[(size_t)r * g.N + ft[i]];
            const double2 zc = make_double2(zi.x, -zi.y);
            U[i] = cadd(U[i], cmul(zc, q));
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                const double2 m = cmul(zc, g.p[(size_t)r * g.N + fs[j]]);
                W[i][j] = make_double2(W[i][j].x - m.x, W[i][j].y - m.y);
            }
        }
    }
    const double *ct = g.curls + 9 * t;
    double cs[9];  // the trial curls, reflected with the element
#pragma unroll
    for (int i = 0; i < 9; ++i) cs[i] = im.det * im.s[i % 3] * g.curls[9 * s + i];
    const double2 S2 = curl_term(W, ct, cs);
    PairAdj acc;
    pair_adj_zero(acc);
    const int q1 = g.rule_start[ru + 1];
    for (int qi = g.rule_start[ru] + lane; qi < q1; qi += 32) {
        const double *d = g.rule_data + 5 * (size_t)qi;
        const double bt[3] = {1.0 - d[0] - d[1], d[0], d[1]}, bs[3] = {1.0 - d[2] - d[3], d[2], d[3]};
        double x[3], y[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            x[c] = bt[0] * tv[0][c] + bt[1] * tv[1][c] + bt[2] * tv[2][c];
            y[c] = bs[0] * sv[0][c] + bs[1] * sv[1][c] + bs[2] * sv[2][c];
        }
        reverse_point(x, y, bt, bs, d[4], nT, nS, nn, g.k, g.eta, W, U, S2, acc);
    }
    if (g.img) {  // minus the regular rule's points, which the image pass added
        for (int pq = lane; pq < g.reg.n * g.reg.n; pq += 32) {
            const int qt = pq / g.reg.n, qs = pq % g.reg.n;
            const double bt[3] = {g.reg.b[qt][0], g.reg.b[qt][1], g.reg.b[qt][2]};
            const double bs[3] = {g.reg.b[qs][0], g.reg.b[qs][1], g.reg.b[qs][2]};
            double x[3], y[3];
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                x[c] = bt[0] * tv[0][c] + bt[1] * tv[1][c] + bt[2] * tv[2][c];
                y[c] = bs[0] * sv[0][c] + bs[1] * sv[1][c] + bs[2] * sv[2][c];
            }
            reverse_point(x, y, bt, bs, -g.reg.w[qt] * g.reg.w[qs], nT, nS, nn, g.k, g.eta, W, U, S2, acc);
        }
    }
    // sum over the lanes
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
        for (int v = 0; v < 3; ++v)
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                acc.xbar[v][d] += __shfl_xor_sync(0xffffffffu, acc.xbar[v][d], o);
                acc.ybar[v][d] += __shfl_xor_sync(0xffffffffu, acc.ybar[v][d], o);
            }
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            acc.ntbar[d] += __shfl_xor_sync(0xffffffffu, acc.ntbar[d], o);
            acc.nsbar[d] += __shfl_xor_sync(0xffffffffu, acc.nsbar[d], o);
        }
        acc.phi.x += __shfl_xor_sync(0xffffffffu, acc.phi.x, o);
        acc.phi.y += __shfl_xor_sync(0xffffffffu, acc.phi.y, o);
        acc.gsum.x += __shfl_xor_sync(0xffffffffu, acc.gsum.x, o);
        acc.gsum.y += __shfl_xor_sync(0xffffffffu, acc.gsum.y, o);
    }
    if (lane == 0) {
        const double at = g.areas[t], as = g.areas[s];
        pair_records(acc, W, ct, cs, 4.0 * at * as, at, as, g.eta, g.rec + (size_t)t * SG_REC,
                     g.rec + (size_t)s * SG_REC, im);
    }
}

// identity terms: 1/2 M_p1p1 in A and -1/2 eta M_p1dp0 in B scale with the area
__global__ void shape_identity_kernel(const int *faces, const double *areas, int F, int N, int R, ShapeRule rule,
                                      double eta, const double2 *z, const double2 *p, const double2 *q,
                                      double *rec) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= F) return;
    const int *fc = faces + 3 * f;
    double blk[3][3] = {}, col[3] = {};
    for (int j = 0; j < rule.n; ++j)
        for (int a = 0; a < 3; ++a) {
            col[a] += rule.w[j] * rule.b[j][a];
            for (int b = 0; b < 3; ++b) blk[a][b] += rule.w[j] * rule.b[j][a] * rule.b[j][b];
        }
    // phi / A: the area factor 2A of M and M_p1dp0 divided out
    double2 phi = make_double2(0.0, 0.0);
    for (int r = 0; r < R; ++r) {
        const double2 qq = q[(size_t)r * F + f];
        for (int a = 0; a < 3; ++a) {
            const double2 zi = z[(size_t)r * N + fc[a]];
            const double2 zc = make_double2(zi.x, -zi.y);
            for (int b = 0; b < 3; ++b)  // W_ab 1/2 M_ab, W = -conj(z) p
                phi = cadd(phi, cscale(cmul(zc, p[(size_t)r * N + fc[b]]), -0.5 * 2.0 * blk[a][b]));
            // U_a (-1/2 eta col_a)
            phi = cadd(phi, times_i_eta(cscale(cmul(zc, qq), -0.5 * 2.0 * col[a]), eta));
        }
    }
    atomicAdd(&rec[(size_t)f * SG_REC + SG_A], phi.x);
}

// the mesh itself and its symmetry images (signs of x, y, z per copy)
struct ShapeCopies {
    int n;
    double s[4][3];
};

// far field: p_inf(d) = sum_src w e(d) [(-ik)(d . n) p_src - q], e = exp(-ik d.y) / (4 pi),
// the sources being the mesh's and, with symmetry images, their reflections
// (position and normal times the signs, the same densities)
__global__ void shape_farfield_kernel(const double *qpts, const double *normals, const double *areas,
                                      const int *faces, int F, int Q, ShapeRule rule, int N, const double *dirs,
                                      int M, const double2 *g, int R, double k, const double2 *p, const double2 *q,
                                      ShapeCopies copies, double *rec) {
    const int sidx = blockIdx.x * blockDim.x + threadIdx.x;
    if (sidx >= F * Q) return;
    const int f = sidx / Q, qi = sidx % Q;
    const double w = rule.w[qi] * 2.0 * areas[f];
    const double y0[3] = {qpts[3 * (size_t)sidx], qpts[3 * (size_t)sidx + 1], qpts[3 * (size_t)sidx + 2]};
    const double n0[3] = {normals[3 * f], normals[3 * f + 1], normals[3 * f + 2]};
    const int *fc = faces + 3 * f;
    double ybar[3] = {0, 0, 0}, nbar[3] = {0, 0, 0};
    double2 phi = make_double2(0.0, 0.0);
    for (int mc = 0; mc < M * copies.n; ++mc) {
        const int m = mc / copies.n, ix = mc % copies.n;
        double sg[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {  // copies.s[ix] by selects (no local-memory copy of the parameter)
            sg[c] = copies.s[0][c];
#pragma unroll
            for (int j = 1; j < 4; ++j)
                if (ix == j) sg[c] = copies.s[j][c];
        }
        const double y[3] = {sg[0] * y0[0], sg[1] * y0[1], sg[2] * y0[2]};
        const double n[3] = {sg[0] * n0[0], sg[1] * n0[1], sg[2] * n0[2]};
        double d[3] = {dirs[3 * m], dirs[3 * m + 1], dirs[3 * m + 2]};
        const double dl = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
        d[0] /= dl;
        d[1] /= dl;
        d[2] /= dl;
        const double dn = d[0] * n[0] + d[1] * n[1] + d[2] * n[2];
        double sn_, cs_;
        sincos_cw(-k * (d[0] * y[0] + d[1] * y[1] + d[2] * y[2]), &sn_, &cs_);
        const double2 e = make_double2(cs_ * 0.07957747154594767 * w, sn_ * 0.07957747154594767 * w);
        double2 h = make_double2(0.0, 0.0), hp = make_double2(0.0, 0.0);  // sum conj(g) [..], sum conj(g) p
        for (int r = 0; r < R; ++r) {
            const double2 gc = make_double2(g[(size_t)r * M + m].x, -g[(size_t)r * M + m].y);
            const double2 a = p[(size_t)r * N + fc[0]], b = p[(size_t)r * N + fc[1]], c = p[(size_t)r * N + fc[2]];
            const double2 ps = make_double2(rule.b[qi][0] * a.x + rule.b[qi][1] * b.x + rule.b[qi][2] * c.x,
                                            rule.b[qi][0] * a.y + rule.b[qi][1] * b.y + rule.b[qi][2] * c.y);
            const double2 qq = q[(size_t)r * F + f];
            // (-ik)(dn) ps - q
            const double2 term = make_double2(k * dn * ps.y - qq.x, -k * dn * ps.x - qq.y);
            h = cadd(h, cmul(gc, term));
            hp = cadd(hp, cmul(gc, ps));
        }
        const double2 eh = cmul(e, h);
        phi = cadd(phi, eh);
        // d/dy: e (-ik d) h;  d/dn: e (-ik) hp d
        const double dy = cmul(make_double2(0.0, -k), eh).x;
        const double dnr = cmul(make_double2(0.0, -k), cmul(e, hp)).x;
        for (int c = 0; c < 3; ++c) {  // back through the reflection
            ybar[c] += dy * d[c] * sg[c];
            nbar[c] += dnr * d[c] * sg[c];
        }
    }
    double *rf = rec + (size_t)f * SG_REC;
    for (int a = 0; a < 3; ++a)
        for (int c = 0; c < 3; ++c) atomicAdd(&rf[SG_V + 3 * a + c], rule.b[qi][a] * ybar[c]);
    for (int c = 0; c < 3; ++c) atomicAdd(&rf[SG_N + c], nbar[c]);
    atomicAdd(&rf[SG_A], phi.x / areas[f]);
}

// forward-mode number: value and one directional derivative
struct Dual {
    double v, d;
};
__device__ __forceinline__ Dual operator+(Dual a, Dual b) { return {a.v + b.v, a.d + b.d}; }
__device__ __forceinline__ Dual operator-(Dual a, Dual b) { return {a.v - b.v, a.d - b.d}; }
__device__ __forceinline__ Dual operator*(Dual a, Dual b) { return {a.v * b.v, a.d * b.v + a.v * b.d}; }
__device__ __forceinline__ Dual operator/(Dual a, Dual b) {
    return {a.v / b.v, (a.d * b.v - a.v * b.d) / (b.v * b.v)};
}
__device__ __forceinline__ Dual dsqrt(Dual a) {
    const double s = sqrt(a.v);
    return {s, a.d / (2.0 * s)};
}

// records -> vertex gradient: gX[v] += 2 (position adjoint + normal, curl and
// area adjoints through the face geometry's derivatives)
__global__ void shape_vertices_kernel(const double *verts, const int *faces, int F, const double *rec, double *gX) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= F) return;
    const int *fc = faces + 3 * f;
    const double *rf = rec + (size_t)f * SG_REC;
    for (int a = 0; a < 3; ++a)
        for (int kk = 0; kk < 3; ++kk) {
            Dual V[3][3];
            for (int b = 0; b < 3; ++b)
                for (int c = 0; c < 3; ++c) V[b][c] = {verts[3 * fc[b] + c], (b == a && c == kk) ? 1.0 : 0.0};
            Dual e1[3], e2[3];
            for (int c = 0; c < 3; ++c) {
                e1[c] = V[1][c] - V[0][c];
                e2[c] = V[2][c] - V[0][c];
            }
            const Dual cr[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2],
                                e1[0] * e2[1] - e1[1] * e2[0]};
            const Dual nrm = dsqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]);
            const Dual n[3] = {cr[0] / nrm, cr[1] / nrm, cr[2] / nrm};
            const Dual area = nrm * Dual{0.5, 0.0};
            const Dual g11 = e1[0] * e1[0] + e1[1] * e1[1] + e1[2] * e1[2];
            const Dual g12 = e1[0] * e2[0] + e1[1] * e2[1] + e1[2] * e2[2];
            const Dual g22 = e2[0] * e2[0] + e2[1] * e2[1] + e2[2] * e2[2];
            const Dual det = g11 * g22 - g12 * g12;
            const Dual i11 = g22 / det, i12 = Dual{0.0, 0.0} - g12 / det, i22 = g11 / det;
            Dual l1[3], l2[3], gr[3][3];
            for (int c = 0; c < 3; ++c) {
                l1[c] = e1[c] * i11 + e2[c] * i12;
                l2[c] = e1[c] * i12 + e2[c] * i22;
                gr[0][c] = Dual{0.0, 0.0} - l1[c] - l2[c];
                gr[1][c] = l1[c];
                gr[2][c] = l2[c];
            }
            double s = rf[SG_V + 3 * a + kk] + rf[SG_A] * area.d;
            for (int c = 0; c < 3; ++c) s += rf[SG_N + c] * n[c].d;
            for (int i = 0; i < 3; ++i) {
                const Dual cu[3] = {n[1] * gr[i][2] - n[2] * gr[i][1], n[2] * gr[i][0] - n[0] * gr[i][2],
                                    n[0] * gr[i][1] - n[1] * gr[i][0]};
                for (int c = 0; c < 3; ++c) s += rf[SG_C + 3 * i + c] * cu[c].d;
            }
            atomicAdd(&gX[3 * fc[a] + kk], 2.0 * s);
        }
}

// z with the rows of the vertices on a symmetry plane times their orbit
// weights (the weights the assembly gives those rows of A and B); zw holds a
// copy of z, and the weighted rows are rewritten from z
__global__ void shape_scale_rows_kernel(const double2 *z, double2 *zw, int N, int R, const int *wv,
                                        const double *ww, int nw) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (int64_t)nw * R) return;
    const int v = (int)(i % nw), r = (int)(i / nw);
    const size_t e = (size_t)r * N + wv[v];
    zw[e] = make_double2(z[e].x * ww[v], z[e].y * ww[v]);
}

// a vertex on a symmetry plane stays on it: its gradient's component normal
// to that plane (coordinate exactly 0 after the set-up's snapping) is zero
__global__ void shape_plane_project_kernel(const double *verts, const int *wv, int nw, int axes, double *gX) {
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= nw) return;
    const int u = wv[v];
    for (int a = 0; a < 3; ++a)
        if ((axes >> a & 1) && verts[3 * (size_t)u + a] == 0.0) gX[3 * (size_t)u + a] = 0.0;
}

static ShapeRule shape_rule(const std::vector<double> &pts, const std::vector<double> &w) {
    ShapeRule r{};
    r.n = (int)w.size();
    for (int j = 0; j < r.n; ++j) {
        r.w[j] = w[j];
        r.b[j][0] = 1.0 - pts[2 * j] - pts[2 * j + 1];
        r.b[j][1] = pts[2 * j];
        r.b[j][2] = pts[2 * j + 1];
    }
    return r;
}

template <int Q> static void launch_shape_pairs(beat_b200_ctx *c, ShapeTileArgs &a) {
    const size_t smem = shape_pairs_smem<Q>();
    BB_CUDA(cudaFuncSetAttribute(shape_pairs_kernel<Q>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    for (a.r0 = 0; a.r0 < a.R; a.r0 += SG_RC) {
        shape_pairs_kernel<Q><<<dim3(c->trial_tiles.ntiles, c->test_tiles.ntiles), SG_THREADS, smem, c->stream>>>(a);
        BB_CUDA(cudaGetLastError());
    }
}

void shape_gradient(beat_b200_ctx *c, double k, double eta, int M, const double *dirs_dev, int R,
                    const double *p_dev, const double *q_dev, const double *g_dev, const double *z_dev,
                    double *gX_dev) {
    BB_REQUIRE(c->test_tiles.tile_faces <= SG_TT && c->test_tiles.tile_verts <= SG_VT &&
                   c->trial_tiles.tile_faces <= SG_TS && c->trial_tiles.tile_verts <= SG_VS,
               BEAT_B200_STATE, "shape gradient: unexpected tiling");
    const int N = c->V, F = c->F, Q = c->Q;
    // the face records, then (with weighted rows) the row-weighted copy of z
    const size_t rec_bytes = sizeof(double) * (size_t)F * SG_REC;
    const size_t zw_off = (rec_bytes + 255) / 256 * 256;
    const bool weighted = c->nweighted > 0;
    DevBuf &buf = c->ws.grad;
    buf.alloc(zw_off + (weighted ? sizeof(double2) * (size_t)N * R : 0));
    double *rec = buf.as<double>();
    BB_CUDA(cudaMemsetAsync(rec, 0, rec_bytes, c->stream));
    BB_CUDA(cudaMemsetAsync(gX_dev, 0, sizeof(double) * 3 * (size_t)N, c->stream));
    const ShapeRule rule = shape_rule(c->rule_pts, c->rule_w);
    const double2 *p = reinterpret_cast<const double2 *>(p_dev), *q = reinterpret_cast<const double2 *>(q_dev);
    const double2 *z = reinterpret_cast<const double2 *>(z_dev);
    if (weighted) {
        double2 *zw = reinterpret_cast<double2 *>(static_cast<char *>(buf.p) + zw_off);
        BB_CUDA(cudaMemcpyAsync(zw, z, sizeof(double2) * (size_t)N * R, cudaMemcpyDeviceToDevice, c->stream));
        const int64_t n = (int64_t)c->nweighted * R;
        shape_scale_rows_kernel<<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(
            z, zw, N, R, c->rw_vert.as<int>(), c->rw_weight.as<double>(), c->nweighted);
        BB_CUDA(cudaGetLastError());
        z = zw;
    }
    ShapeImage xf[3] = {no_image(), no_image(), no_image()};
    for (int ix = 0; ix < c->nimg; ++ix) {
        xf[ix].on = 1;
        for (int i = 0; i < 3; ++i) xf[ix].s[i] = c->img_sign[ix][i];
        xf[ix].det = c->img_det[ix];
    }
    ShapeTileArgs a;
    a.qpts = c->pos_qpts64.as<double>();
    a.normal = c->pos_normal64.as<double>();
    a.curl = c->pos_curl64.as<double>();
    a.area = c->pos_area64.as<double>();
    a.gvert = c->pos_gvert.as<int>();
    a.face_id = c->pos_face.as<int>();
    a.t_fstart = c->test_tiles.face_start.as<int>();
    a.t_vstart = c->test_tiles.vert_start.as<int>();
    a.t_verts = c->test_tiles.verts.as<int>();
    a.t_local = c->test_tiles.local_vert.as<int>();
    a.s_fstart = c->trial_tiles.face_start.as<int>();
    a.s_vstart = c->trial_tiles.vert_start.as<int>();
    a.s_verts = c->trial_tiles.verts.as<int>();
    a.s_local = c->trial_tiles.local_vert.as<int>();
    a.z = z;
    a.p = p;
    a.q = q;
    a.N = N;
    a.F = F;
    a.R = R;
    a.r0 = 0;
    a.k = k;
    a.eta = eta;
    a.rule = rule;
    a.rec = rec;
    for (int img = -1; img < c->nimg; ++img) {  // the mesh itself, then one pass per symmetry image
        a.img = img < 0 ? no_image() : xf[img];
        switch (Q) {
            case 1: launch_shape_pairs<1>(c, a); break;
            case 3: launch_shape_pairs<3>(c, a); break;
            default: launch_shape_pairs<6>(c, a); break;
        }
    }
    ShapeSingArgs s;
    s.rule_start = c->rule_start.as<int>();
    s.rule_data = c->rule_data.as<double>();
    s.verts = c->d_verts.as<double>();
    s.normals = c->d_normals.as<double>();
    s.curls = c->d_curls.as<double>();
    s.areas = c->d_areas.as<double>();
    s.faces = c->d_faces.as<int>();
    s.z = z;
    s.p = p;
    s.q = q;
    s.N = N;
    s.F = F;
    s.R = R;
    s.k = k;
    s.eta = eta;
    s.rec = rec;
    s.reg = rule;
    for (int ix = 0; ix < 3; ++ix) s.xf[ix] = xf[ix];
    if (c->npairs > 0) {
        s.test = c->sp_test.as<int>();
        s.trial = c->sp_trial.as<int>();
        s.rule = c->sp_rule.as<int>();
        s.img = nullptr;
        s.npairs = c->npairs;
        shape_singular_kernel<<<(unsigned)((c->npairs + 7) / 8), 256, 0, c->stream>>>(s);
        BB_CUDA(cudaGetLastError());
    }
    if (c->nimg_pairs > 0) {  // touching image pairs: Duffy minus the image pass's regular rule
        s.test = c->ip_test.as<int>();
        s.trial = c->ip_trial.as<int>();
        s.rule = c->ip_rule.as<int>();
        s.img = c->ip_img.as<int>();
        s.npairs = c->nimg_pairs;
        shape_singular_kernel<<<(unsigned)((c->nimg_pairs + 7) / 8), 256, 0, c->stream>>>(s);
        BB_CUDA(cudaGetLastError());
    }
    shape_identity_kernel<<<(F + 255) / 256, 256, 0, c->stream>>>(c->d_faces.as<int>(), c->d_areas.as<double>(), F,
                                                                   N, R, rule, eta, z, p, q, rec);
    BB_CUDA(cudaGetLastError());
    ShapeCopies copies;
    copies.n = 1 + c->nimg;
    for (int i = 0; i < 3; ++i) copies.s[0][i] = 1.0;
    for (int ix = 0; ix < c->nimg; ++ix)
        for (int i = 0; i < 3; ++i) copies.s[1 + ix][i] = c->img_sign[ix][i];
    shape_farfield_kernel<<<(F * Q + 127) / 128, 128, 0, c->stream>>>(
        c->d_qpts.as<double>(), c->d_normals.as<double>(), c->d_areas.as<double>(), c->d_faces.as<int>(), F, Q,
        rule, N, dirs_dev, M, reinterpret_cast<const double2 *>(g_dev), R, k, p, q, copies, rec);
    BB_CUDA(cudaGetLastError());
    shape_vertices_kernel<<<(F + 127) / 128, 128, 0, c->stream>>>(c->d_verts.as<double>(), c->d_faces.as<int>(), F,
                                                                  rec, gX_dev);
    BB_CUDA(cudaGetLastError());
    if (weighted) {  // the planes are those the images reflect across (a sign of -1)
        int axes = 0;
        for (int ix = 0; ix < c->nimg; ++ix)
            for (int i = 0; i < 3; ++i)
                if (c->img_sign[ix][i] < 0) axes |= 1 << i;
        shape_plane_project_kernel<<<(c->nweighted + 127) / 128, 128, 0, c->stream>>>(
            c->d_verts.as<double>(), c->rw_vert.as<int>(), c->nweighted, axes, gX_dev);
        BB_CUDA(cudaGetLastError());
    }
}

}  // namespace bb
