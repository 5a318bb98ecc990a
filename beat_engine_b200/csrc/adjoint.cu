// adjoint.cu -- admittance boundary condition and adjoint gradients of a
// far-field functional.  Neither exists in the reference's exterior path (its
// admittance is a coupled-FEM wall model, BeatEngineCoupled.jl:594-623); the
// definitions are this library's:
//
//   boundary condition   q = q0 - diag(a) P p,  P = face average of the P1
//                        pressure (its L2 projection onto face constants)
//   system               (A + B diag(a) P) p = B q0,  A' := A + B diag(a) P
//   far field            p_inf = Fp p + Fq q    (the r -> inf field sum)
//   functional           J real, g = dJ/d conj(p_inf)  (M x R, given)
//   adjoint              y = E^H g with E = Fp - Fq diag(a) P,
//                        z = A'^-H y,  w = B^H z + Fq^H g,
//                        dJ/d conj(q0) = w,
//                        dJ/d conj(a_f) = - sum_r w_{f,r} conj((P p_r)_f).
// With a = 0 the solve is the reference's.  A normal-velocity admittance Y
// (v = v0 - Y p, exp(-i omega t)) gives a = neumann_scale * Y.
#include <cuda_runtime.h>

#include <cmath>
#include <vector>

#include "internal.cuh"
#include "phase.cuh"

namespace bb {

// ---------------------------------------------------------------------------
// admittance terms
// ---------------------------------------------------------------------------

// A[i][j] += sum_{f incident to j} (a_f / 3) B[i][f]   (row i = blockIdx.y)
template <typename T>
__global__ void admittance_lhs_kernel(Cx<T> *A, int64_t ld, const Cx<T> *B, int n, int F, const int *vf_start,
                                      const int *vf_face, const double2 *a) {
    const int i = blockIdx.y, j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const Cx<T> *brow = B + (int64_t)i * F;
    double sr = 0, si = 0;
    for (int t = vf_start[j]; t < vf_start[j + 1]; ++t) {
        const int f = vf_face[t];
        const Cx<T> bv = brow[f];
        const double2 af = a[f];
        sr += af.x * (double)bv.re - af.y * (double)bv.im;
        si += af.x * (double)bv.im + af.y * (double)bv.re;
    }
    Cx<T> &d = A[(int64_t)i * ld + j];
    d.re += (T)(sr / 3.0);
    d.im += (T)(si / 3.0);
}

void apply_admittance_lhs(beat_b200_ctx *c, int precision) {
    if (!c->adm_set) return;
    Workspace &w = c->ws;
    const int n = c->V, F = c->F;
    const dim3 grid((n + 255) / 256, n);
    if (precision == BEAT_B200_FP64)
        admittance_lhs_kernel<double><<<grid, 256, 0, c->stream>>>(w.A.as<Cx<double>>(), w.ld, w.B.as<Cx<double>>(),
                                                                   n, F, c->vf_start.as<int>(), c->vf_face.as<int>(),
                                                                   c->adm.as<double2>());
    else
        admittance_lhs_kernel<float><<<grid, 256, 0, c->stream>>>(w.A.as<Cx<float>>(), w.ld, w.B.as<Cx<float>>(), n,
                                                                  F, c->vf_start.as<int>(), c->vf_face.as<int>(),
                                                                  c->adm.as<double2>());
    BB_CUDA(cudaGetLastError());
}

// out[f, r] = q[f, r] - a_f (P p_r)_f  (a may be null: a plain copy)
__global__ void effective_neumann_kernel(const int *faces, int F, int N, int R, const double2 *a, const double2 *p,
                                         const double2 *q, double2 *out) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (int64_t)F * R) return;
    const int f = (int)(idx % F), r = (int)(idx / F);
    double2 v = q[idx];
    if (a) {
        const double2 p0 = p[(size_t)r * N + faces[3 * f]], p1 = p[(size_t)r * N + faces[3 * f + 1]],
                      p2 = p[(size_t)r * N + faces[3 * f + 2]];
        const double pr = (p0.x + p1.x + p2.x) / 3.0, pi = (p0.y + p1.y + p2.y) / 3.0;
        const double2 af = a[f];
        v.x -= af.x * pr - af.y * pi;
        v.y -= af.x * pi + af.y * pr;
    }
    out[idx] = v;
}

void effective_neumann(beat_b200_ctx *c, int R, const double *p_dev, const double *q_dev, double *q_eff) {
    const int64_t total = (int64_t)c->F * R;
    effective_neumann_kernel<<<(unsigned)((total + 255) / 256), 256, 0, c->stream>>>(
        c->d_faces.as<int>(), c->F, c->V, R, c->adm_set ? c->adm.as<double2>() : nullptr,
        reinterpret_cast<const double2 *>(p_dev), reinterpret_cast<const double2 *>(q_dev),
        reinterpret_cast<double2 *>(q_eff));
    BB_CUDA(cudaGetLastError());
}

// y[i, r] -= sum_{f incident to i} conj(a_f) wq[f, r] / 3     (P^T diag(conj a))
__global__ void admittance_transpose_kernel(int N, int F, int R, const int *vf_start, const int *vf_face,
                                            const double2 *a, const double2 *wq, double2 *y) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (int64_t)N * R) return;
    const int i = (int)(idx % N), r = (int)(idx / N);
    double sr = 0, si = 0;
    for (int t = vf_start[i]; t < vf_start[i + 1]; ++t) {
        const int f = vf_face[t];
        const double2 af = a[f], wv = wq[(size_t)r * F + f];
        sr += af.x * wv.x + af.y * wv.y;  // conj(a) w
        si += af.x * wv.y - af.y * wv.x;
    }
    y[idx].x -= sr / 3.0;
    y[idx].y -= si / 3.0;
}

// ga[f] = - sum_r w[f, r] conj((P p_r)_f)
__global__ void admittance_gradient_kernel(const int *faces, int F, int N, int R, const double2 *p, const double2 *w,
                                           double2 *ga) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= F) return;
    double sr = 0, si = 0;
    for (int r = 0; r < R; ++r) {
        const double2 p0 = p[(size_t)r * N + faces[3 * f]], p1 = p[(size_t)r * N + faces[3 * f + 1]],
                      p2 = p[(size_t)r * N + faces[3 * f + 2]];
        const double pr = (p0.x + p1.x + p2.x) / 3.0, pi = (p0.y + p1.y + p2.y) / 3.0;
        const double2 wv = w[(size_t)r * F + f];
        sr -= wv.x * pr + wv.y * pi;  // w conj(Pp)
        si -= wv.y * pr - wv.x * pi;
    }
    ga[f] = make_double2(sr, si);
}

// ---------------------------------------------------------------------------
// transposed far field: per source s (rule point of face f, weight w_s, basis
// values b_a), with E = e^{-ik d.y}/(4 pi) and D = E (-ik d.n) as in the far
// field, Gp_s = sum_m conj(D) g_m and Gq_s = sum_m conj(E) g_m; then
//   (Fp^H g)_v += w_s b_a Gp_s for the vertices v = v_a(f),
//   (Fq^H g)_f -= w_s Gq_s.
// ---------------------------------------------------------------------------
constexpr int FA_RC = 16, FA_CHUNK = 64, FA_THREADS = 128;

struct AdjImages {
    int n;           // the mesh itself, then its symmetry images
    double s[4][3];  // signs per copy
};

__global__ void __launch_bounds__(FA_THREADS) farfield_adjoint_kernel(
    const double *qpts, const double *normals, const double *areas, const int *faces, int F, int Q,
    const double *rule_w3, int N, const double *dirs, int M, const double2 *g, int R, int r0, double k, double2 *yp,
    double2 *wq, AdjImages images) {
    __shared__ double sd[FA_CHUNK][3];
    __shared__ double2 sg[FA_RC][FA_CHUNK];
    const int S = F * Q;
    const int s = blockIdx.x * FA_THREADS + threadIdx.x;
    const int rc = min(FA_RC, R - r0);
    double y0 = 0, y1 = 0, y2 = 0, n0 = 0, n1 = 0, n2 = 0;
    int f = 0, qi = 0;
    if (s < S) {
        f = s / Q;
        qi = s % Q;
        y0 = qpts[3 * (size_t)s];
        y1 = qpts[3 * (size_t)s + 1];
        y2 = qpts[3 * (size_t)s + 2];
        n0 = normals[3 * f];
        n1 = normals[3 * f + 1];
        n2 = normals[3 * f + 2];
    }
    double pr[FA_RC], pi[FA_RC], qr[FA_RC], qim[FA_RC];
#pragma unroll
    for (int r = 0; r < FA_RC; ++r) pr[r] = pi[r] = qr[r] = qim[r] = 0.0;
    const double inv4pi = 0.07957747154594767;
    for (int m0 = 0; m0 < M; m0 += FA_CHUNK) {
        const int mn = min(FA_CHUNK, M - m0);
        __syncthreads();
        for (int i = threadIdx.x; i < mn; i += FA_THREADS) {
            const double d0 = dirs[3 * (m0 + i)], d1 = dirs[3 * (m0 + i) + 1], d2 = dirs[3 * (m0 + i) + 2];
            const double nn = sqrt(d0 * d0 + d1 * d1 + d2 * d2);
            sd[i][0] = d0 / nn;
            sd[i][1] = d1 / nn;
            sd[i][2] = d2 / nn;
        }
        for (int i = threadIdx.x; i < FA_RC * FA_CHUNK; i += FA_THREADS) {
            const int r = i / FA_CHUNK, j = i % FA_CHUNK;
            sg[r][j] = (r < rc && j < mn) ? g[(size_t)(r0 + r) * M + m0 + j] : make_double2(0, 0);
        }
        __syncthreads();
        if (s >= S) continue;
        for (int j = 0; j < mn * images.n; ++j) {
            // direction j % mn against copy j / mn of the source (reflected y and n)
            const int jm = j % mn, ix = j / mn;
            const double d0 = sd[jm][0] * images.s[ix][0], d1 = sd[jm][1] * images.s[ix][1],
                         d2 = sd[jm][2] * images.s[ix][2];  // d.(S y) = (S d).y
            double sn_, cs_;
            sincos_cw(-k * (d0 * y0 + d1 * y1 + d2 * y2), &sn_, &cs_);
            const double er = cs_ * inv4pi, ei = sn_ * inv4pi;  // E
            const double dn = d0 * n0 + d1 * n1 + d2 * n2;
            const double dr = ei * k * dn, di = -er * k * dn;  // D = E (-ik dn)
#pragma unroll
            for (int r = 0; r < FA_RC; ++r) {
                const double2 gv = sg[r][jm];
                pr[r] += dr * gv.x + di * gv.y;  // conj(D) g
                pi[r] += dr * gv.y - di * gv.x;
                qr[r] += er * gv.x + ei * gv.y;  // conj(E) g
                qim[r] += er * gv.y - ei * gv.x;
            }
        }
    }
    if (s >= S) return;
    const double w = rule_w3[4 * qi] * 2.0 * areas[f];
    const double b[3] = {rule_w3[4 * qi + 1], rule_w3[4 * qi + 2], rule_w3[4 * qi + 3]};
    const int v[3] = {faces[3 * f], faces[3 * f + 1], faces[3 * f + 2]};
#pragma unroll
    for (int r = 0; r < FA_RC; ++r) {
        if (r >= rc) break;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            double2 *d = &yp[(size_t)(r0 + r) * N + v[a]];
            atomicAdd(&d->x, w * b[a] * pr[r]);
            atomicAdd(&d->y, w * b[a] * pi[r]);
        }
        double2 *e = &wq[(size_t)(r0 + r) * F + f];
        atomicAdd(&e->x, -w * qr[r]);
        atomicAdd(&e->y, -w * qim[r]);
    }
}

// ---------------------------------------------------------------------------
// A^-H with the stored factors (P A = L U, unit L, row-major in A):
//   A^H = U^H L^H P  =>  z = P^T L^-H U^-H y.
// Blocked over 64-row blocks in FP64 arithmetic: the off-block sums
// (sum_j conj(F[j][col]) z_j over rows j outside the block) are a
// column-block product over row slices; the 64 x 64 diagonal blocks are
// substituted by one CTA, one thread per right-hand side.
// ---------------------------------------------------------------------------
constexpr int AB = 64;

// Z[col0 + il, r] -= sum_{j in [j0, j1)} conj(A[j][col0 + il]) Z[j, r]
template <typename T>
__global__ void __launch_bounds__(256) colblock_update_kernel(const Cx<T> *A, int64_t ld, int n, int col0, int ncol,
                                                              int j0, int j1, int jslice, double2 *Z, int R) {
    const int il = threadIdx.x % AB, rg = threadIdx.x / AB;  // 4 groups of 4 columns
    const int jb = j0 + blockIdx.x * jslice, je = min(j1, jb + jslice);
    for (int r0 = 0; r0 < R; r0 += 16) {
        double ar[4] = {0, 0, 0, 0}, ai[4] = {0, 0, 0, 0};
        if (il < ncol) {
            for (int j = jb; j < je; ++j) {
                const Cx<T> m = A[(int64_t)j * ld + col0 + il];
                const double mr = (double)m.re, mi = -(double)m.im;
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    const int r = r0 + rg * 4 + e;
                    if (r < R) {
                        const double2 z = Z[(size_t)r * n + j];
                        ar[e] += mr * z.x - mi * z.y;
                        ai[e] += mr * z.y + mi * z.x;
                    }
                }
            }
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const int r = r0 + rg * 4 + e;
                if (r < R) {
                    atomicAdd(&Z[(size_t)r * n + col0 + il].x, -ar[e]);
                    atomicAdd(&Z[(size_t)r * n + col0 + il].y, -ai[e]);
                }
            }
        }
    }
}

// UPPER: solve U_bb^H z = rhs (forward, diagonal conj(U_ii)); else
// L_bb^H z = rhs (backward, unit diagonal); block rows [b0, b0 + nb)
template <typename T, bool UPPER>
__global__ void __launch_bounds__(64) diag_adjoint_kernel(const Cx<T> *A, int64_t ld, int n, int b0, int nb, double2 *Z,
                                                          int R, int *status) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    auto blk = reinterpret_cast<Cx<double>(*)[AB + 1]>(smem_raw);                               // [AB][AB + 1]
    auto zb = reinterpret_cast<Cx<double>(*)[AB + 1]>(smem_raw + sizeof(Cx<double>) * AB * (AB + 1));  // [row][r]
    for (int i = threadIdx.x; i < nb * nb; i += blockDim.x) {
        const Cx<T> v = A[(int64_t)(b0 + i / nb) * ld + b0 + i % nb];
        blk[i / nb][i % nb] = Cx<double>{(double)v.re, (double)v.im};
    }
    for (int rb = 0; rb < R; rb += AB) {
        const int rn = min(AB, R - rb);
        __syncthreads();
        for (int i = threadIdx.x; i < nb * rn; i += blockDim.x) {
            const double2 z = Z[(size_t)(rb + i / nb) * n + b0 + i % nb];
            zb[i % nb][i / nb] = Cx<double>{z.x, z.y};
        }
        __syncthreads();
        const int r = threadIdx.x;
        if (r < rn) {
            if (UPPER) {
                for (int i = 0; i < nb; ++i) {
                    double sr = zb[i][r].re, si = zb[i][r].im;
                    for (int j = 0; j < i; ++j) {  // conj(U[j][i]) z_j
                        const Cx<double> u = blk[j][i], z = zb[j][r];
                        sr -= u.re * z.re + u.im * z.im;
                        si -= u.re * z.im - u.im * z.re;
                    }
                    const Cx<double> d = blk[i][i];  // divide by conj(d)
                    const double den = d.re * d.re + d.im * d.im;
                    if (!(den > 0.0)) {
                        atomicOr(status, (int)DEV_ZERO_PIVOT);
                        zb[i][r] = Cx<double>{0, 0};
                    } else {
                        zb[i][r] = Cx<double>{(sr * d.re - si * d.im) / den, (si * d.re + sr * d.im) / den};
                    }
                }
            } else {
                for (int i = nb - 1; i >= 0; --i) {
                    double sr = zb[i][r].re, si = zb[i][r].im;
                    for (int j = i + 1; j < nb; ++j) {  // conj(L[j][i]) z_j
                        const Cx<double> l = blk[j][i], z = zb[j][r];
                        sr -= l.re * z.re + l.im * z.im;
                        si -= l.re * z.im - l.im * z.re;
                    }
                    zb[i][r] = Cx<double>{sr, si};
                }
            }
        }
        __syncthreads();
        for (int i = threadIdx.x; i < nb * rn; i += blockDim.x) {
            const Cx<double> v = zb[i % nb][i / nb];
            Z[(size_t)(rb + i / nb) * n + b0 + i % nb] = make_double2(v.re, v.im);
        }
    }
}

// out[perm[i]] = in[i]
__global__ void unpermute_rows_kernel(const double2 *in, double2 *out, const int *perm, int n, int R) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int dst = perm[i];
    for (int r = 0; r < R; ++r) out[(size_t)r * n + dst] = in[(size_t)r * n + i];
}

template <typename T> static void lu_solve_adjoint_t(beat_b200_ctx *c, int R, const double *in, double *out) {
    Workspace &w = c->ws;
    const int n = c->V;
    const Cx<T> *A = w.A.as<Cx<T>>();
    w.x.alloc(sizeof(double2) * (size_t)n * R);
    double2 *Z = w.x.as<double2>();
    BB_CUDA(cudaMemcpyAsync(Z, in, sizeof(double2) * (size_t)n * R, cudaMemcpyDeviceToDevice, c->stream));
    const int nblk = (n + AB - 1) / AB;
    constexpr int JS = 256;  // rows per CTA of the off-block sums
    const size_t dsmem = 2 * sizeof(Cx<double>) * AB * (AB + 1);
    BB_CUDA(cudaFuncSetAttribute(diag_adjoint_kernel<T, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dsmem));
    BB_CUDA(cudaFuncSetAttribute(diag_adjoint_kernel<T, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dsmem));
    for (int b = 0; b < nblk; ++b) {  // U^H: forward
        const int b0 = b * AB, nb = std::min(AB, n - b0);
        if (b0 > 0)
            colblock_update_kernel<T><<<(b0 + JS - 1) / JS, 256, 0, c->stream>>>(A, w.ld, n, b0, nb, 0, b0, JS, Z, R);
        diag_adjoint_kernel<T, true><<<1, 64, dsmem, c->stream>>>(A, w.ld, n, b0, nb, Z, R, c->status.as<int>());
    }
    for (int b = nblk - 1; b >= 0; --b) {  // L^H: backward
        const int b0 = b * AB, nb = std::min(AB, n - b0), b1 = b0 + nb;
        if (b1 < n)
            colblock_update_kernel<T><<<(n - b1 + JS - 1) / JS, 256, 0, c->stream>>>(A, w.ld, n, b0, nb, b1, n, JS, Z,
                                                                                    R);
        diag_adjoint_kernel<T, false><<<1, 64, dsmem, c->stream>>>(A, w.ld, n, b0, nb, Z, R, c->status.as<int>());
    }
    unpermute_rows_kernel<<<(n + 255) / 256, 256, 0, c->stream>>>(Z, reinterpret_cast<double2 *>(out),
                                                                  w.perm.as<int>(), n, R);
    BB_CUDA(cudaGetLastError());
}

void lu_solve_adjoint(beat_b200_ctx *c, int R, const double *in, double *out) {
    if (c->ws.precision == BEAT_B200_FP64)
        lu_solve_adjoint_t<double>(c, R, in, out);
    else
        lu_solve_adjoint_t<float>(c, R, in, out);
}

// ---------------------------------------------------------------------------
// the adjoint driver
// ---------------------------------------------------------------------------
void adjoint(beat_b200_ctx *c, double k, int M, const double *dirs_host, int R, const double *p_dev,
             const double *g_dev, double *w_dev, double *ga_dev, const beat_b200_opts &o, IrResult *ir,
             const double **z_out) {
    Workspace &w = c->ws;
    BB_REQUIRE(w.lu_valid, BEAT_B200_STATE, "adjoint: no factorisation on this context (solve first)");
    BB_REQUIRE(w.rhs_cached, BEAT_B200_STATE,
               "adjoint: the last solve formed its right-hand sides matrix-free, so the mapping B is not "
               "resident; solve with the cached right-hand-side mapping (BEAT_B200_FLAG_RHS_CACHED)");
    BB_REQUIRE(k == c->last_k, BEAT_B200_STATE, "adjoint: the wavenumber differs from the last solve's");
    BB_REQUIRE(M >= 1 && R >= 1, BEAT_B200_INVALID_ARG, "adjoint: M and R must be >= 1");
    const int n = c->V, F = c->F, Q = c->Q;
    // scratch: rule table, directions, y (N x R), z (N x R)
    const size_t nd = (4 * (size_t)Q + 3 * (size_t)M + 1) & ~(size_t)1;
    w.field.alloc(sizeof(double) * nd + sizeof(double2) * 2 * (size_t)n * R);
    double *d_rw = w.field.as<double>(), *d_dirs = d_rw + 4 * Q;
    double2 *y = reinterpret_cast<double2 *>(d_rw + nd), *z = y + (size_t)n * R;
    std::vector<double> rw3(4 * (size_t)Q);
    for (int q = 0; q < Q; ++q) {
        rw3[4 * q] = c->rule_w[q];
        rw3[4 * q + 1] = 1.0 - c->rule_pts[2 * q] - c->rule_pts[2 * q + 1];
        rw3[4 * q + 2] = c->rule_pts[2 * q];
        rw3[4 * q + 3] = c->rule_pts[2 * q + 1];
    }
    BB_CUDA(cudaMemcpyAsync(d_rw, rw3.data(), sizeof(double) * 4 * Q, cudaMemcpyHostToDevice, c->stream));
    BB_CUDA(cudaMemcpyAsync(d_dirs, dirs_host, sizeof(double) * 3 * M, cudaMemcpyHostToDevice, c->stream));
    // 1. y = Fp^H g, w = Fq^H g
    BB_CUDA(cudaMemsetAsync(y, 0, sizeof(double2) * (size_t)n * R, c->stream));
    BB_CUDA(cudaMemsetAsync(w_dev, 0, sizeof(double2) * (size_t)F * R, c->stream));
    const int S = F * Q;
    AdjImages images;
    images.n = 1 + c->nimg;
    for (int i = 0; i < 3; ++i) images.s[0][i] = 1.0;
    for (int ix = 0; ix < c->nimg; ++ix)
        for (int i = 0; i < 3; ++i) images.s[1 + ix][i] = c->img_sign[ix][i];
    for (int r0 = 0; r0 < R; r0 += FA_RC)
        farfield_adjoint_kernel<<<(S + FA_THREADS - 1) / FA_THREADS, FA_THREADS, 0, c->stream>>>(
            c->d_qpts.as<double>(), c->d_normals.as<double>(), c->d_areas.as<double>(), c->d_faces.as<int>(), F, Q,
            d_rw, n, d_dirs, M, reinterpret_cast<const double2 *>(g_dev), R, r0, k, y,
            reinterpret_cast<double2 *>(w_dev), images);
    BB_CUDA(cudaGetLastError());
    // 2. y -= P^T diag(conj a) Fq^H g
    if (c->adm_set) {
        const int64_t tot = (int64_t)n * R;
        admittance_transpose_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, c->stream>>>(
            n, F, R, c->vf_start.as<int>(), c->vf_face.as<int>(), c->adm.as<double2>(),
            reinterpret_cast<const double2 *>(w_dev), y);
        BB_CUDA(cudaGetLastError());
    }
    // 3. z = A'^-H y (mixed form: FP32 factors + FP64 refinement on the stored operator)
    BB_CUDA(cudaMemsetAsync(c->status.p, 0, sizeof(int), c->stream));
    lu_solve_adjoint(c, R, reinterpret_cast<const double *>(y), reinterpret_cast<double *>(z));
    *ir = IrResult{0, 1, 0.0};
    if (w.precision != BEAT_B200_FP64)
        *ir = gmres_refine_adjoint(c, R, reinterpret_cast<double *>(z), reinterpret_cast<const double *>(y),
                                   o.ir_restart, o.ir_max_iters, o.ir_rtol);
    // 4. w += B^H z
    if (w.precision == BEAT_B200_FP64)
        tall_gemm_h<double>(c->stream, c->sm_count, w.B.as<Cx<double>>(), F, n, F, reinterpret_cast<const double *>(z),
                            w_dev, R, 1.0);
    else
        tall_gemm_h<float>(c->stream, c->sm_count, w.B.as<Cx<float>>(), F, n, F, reinterpret_cast<const double *>(z),
                           w_dev, R, 1.0);
    // 5. admittance gradient
    if (ga_dev) {
        admittance_gradient_kernel<<<(F + 255) / 256, 256, 0, c->stream>>>(
            c->d_faces.as<int>(), F, n, R, reinterpret_cast<const double2 *>(p_dev),
            reinterpret_cast<const double2 *>(w_dev), reinterpret_cast<double2 *>(ga_dev));
        BB_CUDA(cudaGetLastError());
    }
    BB_CUDA(cudaStreamSynchronize(c->stream));
    const int st = read_status(c);
    BB_REQUIRE(!(st & DEV_ZERO_PIVOT), BEAT_B200_SINGULAR, "adjoint: zero pivot in the factors");
    if (z_out) *z_out = reinterpret_cast<const double *>(z);  // stays valid until the next use of ws.field
}

}  // namespace bb
