// field.cu -- observation-point pressure and far-field pattern for all right
// hand sides in one pass over the boundary sources.
//
// Reference: build_field_evaluation_cache (src/BeatEngineCore.jl:1770-1810),
// _cuda_weighted_field_sources_kernel! (src/BeatEngineCudaField.jl:161-197),
// _cuda_field_eval_kernel! (:240-327), evaluate_galerkin_field_cpu
// (src/BeatEngineCpuField.jl:1-49):
//     p(x) = sum_src w [ G (ik - 1/r)(r.n / r) p_src - G q_src ],  r = y - x
// The far-field pattern has no reference counterpart; it is the r -> inf limit
// of the same sum with the same signed k:
//     p_inf(d) = sum_src exp(-ik d.y)/(4 pi) [ (-ik)(d.n) p_src - q_src ].
//
// The reference launches one field kernel per excitation and output; here one
// kernel evaluates G once per (point, source) for every column.  Points run
// over threads, sources are staged through shared memory in chunks and the
// source range is split over CTAs, which add their partial sums with
// red.global.add.  FP64 in both precision forms.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <utility>
#include <vector>

#include "internal.cuh"
#include "phase.cuh"

namespace bb {

constexpr int FLD_RC = 16;      // right-hand sides per pass
constexpr int FLD_CHUNK = 32;   // sources per shared-memory chunk
constexpr int FLD_THREADS = 128;

struct FieldImages {
    int n;            // copies: the mesh itself, then its symmetry images
    double s[4][3];   // per copy: signs of x, y, z
};

// per source: position, normal, p-density and q-density for R columns, for
// the mesh and each symmetry image (reflected position and normal, the same
// densities); copy ix of source s is entry ix * F Q + s of arrays of stride
// ST = images.n F Q
__global__ void field_sources_kernel(const double *qpts, const double *normals, const double *areas,
                                     const int *faces, int F, int Q, const double *rule_w3, int N,
                                     const double2 *p, const double2 *q, int R, double *ys, double *ns,
                                     double2 *ps, double2 *qs, FieldImages images) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    const int S = F * Q, ST = S * images.n;
    if (s >= S) return;
    const int f = s / Q, qi = s % Q;
    const double w = rule_w3[4 * qi] * 2.0 * areas[f];
    const double b0 = rule_w3[4 * qi + 1], b1 = rule_w3[4 * qi + 2], b2 = rule_w3[4 * qi + 3];
    for (int ix = 0; ix < images.n; ++ix)
        for (int c = 0; c < 3; ++c) {
            ys[3 * ((size_t)ix * S + s) + c] = images.s[ix][c] * qpts[3 * (size_t)s + c];
            ns[3 * ((size_t)ix * S + s) + c] = images.s[ix][c] * normals[3 * f + c];
        }
    const int v0 = faces[3 * f], v1 = faces[3 * f + 1], v2 = faces[3 * f + 2];
    for (int r = 0; r < R; ++r) {
        const double2 a = p[(size_t)r * N + v0], b = p[(size_t)r * N + v1], c = p[(size_t)r * N + v2];
        const double2 pv = make_double2((b0 * a.x + b1 * b.x + b2 * c.x) * w, (b0 * a.y + b1 * b.y + b2 * c.y) * w);
        const double2 qq = q[(size_t)r * F + f];
        const double2 qv = make_double2(qq.x * w, qq.y * w);
        for (int ix = 0; ix < images.n; ++ix) {
            ps[(size_t)r * ST + (size_t)ix * S + s] = pv;
            qs[(size_t)r * ST + (size_t)ix * S + s] = qv;
        }
    }
}

template <bool FAR>
__global__ void __launch_bounds__(FLD_THREADS) field_eval_kernel(const double *pts, int M, const double *ys,
                                                                 const double *ns, const double2 *ps,
                                                                 const double2 *qs, int S, int R, int r0,
                                                                 int per_cta, double k, double2 *out) {
    __shared__ double sy[FLD_CHUNK][3], sn[FLD_CHUNK][3];
    __shared__ double2 sp[FLD_RC][FLD_CHUNK], sq[FLD_RC][FLD_CHUNK];
    const int m = blockIdx.x * FLD_THREADS + threadIdx.x;
    const int s_begin = blockIdx.y * per_cta, s_end = min(S, s_begin + per_cta);
    const int rc = min(FLD_RC, R - r0);
    double x0 = 0, x1 = 0, x2 = 0;
    if (m < M) {
        x0 = pts[3 * m];
        x1 = pts[3 * m + 1];
        x2 = pts[3 * m + 2];
        if (FAR) {
            const double nn = sqrt(x0 * x0 + x1 * x1 + x2 * x2);
            x0 /= nn;
            x1 /= nn;
            x2 /= nn;
        }
    }
    double ar[FLD_RC], ai[FLD_RC];
#pragma unroll
    for (int r = 0; r < FLD_RC; ++r) ar[r] = ai[r] = 0.0;
    const double inv4pi = 0.07957747154594767;
    for (int c0 = s_begin; c0 < s_end; c0 += FLD_CHUNK) {
        const int cn = min(FLD_CHUNK, s_end - c0);
        __syncthreads();
        for (int i = threadIdx.x; i < cn * 3; i += FLD_THREADS) {
            sy[i / 3][i % 3] = ys[3 * (size_t)c0 + i];
            sn[i / 3][i % 3] = ns[3 * (size_t)c0 + i];
        }
        for (int i = threadIdx.x; i < FLD_RC * FLD_CHUNK; i += FLD_THREADS) {
            const int r = i / FLD_CHUNK, j = i % FLD_CHUNK;
            const bool ok = r < rc && j < cn;
            sp[r][j] = ok ? ps[(size_t)(r0 + r) * S + c0 + j] : make_double2(0, 0);
            sq[r][j] = ok ? qs[(size_t)(r0 + r) * S + c0 + j] : make_double2(0, 0);
        }
        __syncthreads();
        if (m >= M) continue;
        for (int j = 0; j < cn; ++j) {
            double gr, gi, dr, di;  // green and double-layer factors
            if (!FAR) {
                const double rx = sy[j][0] - x0, ry = sy[j][1] - x1, rz = sy[j][2] - x2;
                const double r2 = rx * rx + ry * ry + rz * rz;
                if (r2 == 0.0) continue;
                const double ir = rsqrt(r2), rad = r2 * ir;
                double sn_, cs_;
                sincos_cw(k * rad, &sn_, &cs_);
                gr = cs_ * inv4pi * ir;
                gi = sn_ * inv4pi * ir;
                const double proj = (rx * sn[j][0] + ry * sn[j][1] + rz * sn[j][2]) * ir;
                // G (ik - 1/r) proj
                dr = (gr * -ir - gi * k) * proj;
                di = (gr * k + gi * -ir) * proj;
            } else {
                const double ph = -k * (x0 * sy[j][0] + x1 * sy[j][1] + x2 * sy[j][2]);
                double sn_, cs_;
                sincos_cw(ph, &sn_, &cs_);
                gr = cs_ * inv4pi;
                gi = sn_ * inv4pi;
                const double dn = x0 * sn[j][0] + x1 * sn[j][1] + x2 * sn[j][2];
                // e (-ik dn)
                dr = gi * k * dn;
                di = -gr * k * dn;
            }
#pragma unroll
            for (int r = 0; r < FLD_RC; ++r) {
                const double2 pv = sp[r][j], qv = sq[r][j];
                ar[r] += dr * pv.x - di * pv.y - (gr * qv.x - gi * qv.y);
                ai[r] += dr * pv.y + di * pv.x - (gr * qv.y + gi * qv.x);
            }
        }
    }
    if (m < M) {
#pragma unroll
        for (int r = 0; r < FLD_RC; ++r)
            if (r < rc) {
                atomicAdd(&out[(size_t)(r0 + r) * M + m].x, ar[r]);
                atomicAdd(&out[(size_t)(r0 + r) * M + m].y, ai[r]);
            }
    }
}

// boundary sources of the mesh and its images, staged in c->ws.field
struct StagedSources {
    const double *ys = nullptr, *ns = nullptr, *pts = nullptr;
    const double2 *ps = nullptr, *qs = nullptr;
    const double2 *q = nullptr;  // the Neumann data used (admittance term included)
    int S = 0;                   // sources per column
};

static StagedSources stage_sources(beat_b200_ctx *c, int M, const double *pts_host, int R, const double *p_dev,
                                   const double *q_dev) {
    const int F = c->F, Q = c->Q, N = c->V;
    FieldImages images;
    images.n = 1 + c->nimg;
    for (int i = 0; i < 3; ++i) images.s[0][i] = 1.0;
    for (int ix = 0; ix < c->nimg; ++ix)
        for (int i = 0; i < 3; ++i) images.s[1 + ix][i] = c->img_sign[ix][i];
    const int S = F * Q * images.n;  // sources of the mesh and its images
    if (c->adm_set) {  // the boundary's Neumann data include the admittance term
        c->ws.qeff.alloc(sizeof(double2) * (size_t)F * R);
        effective_neumann(c, R, p_dev, q_dev, c->ws.qeff.as<double>());
        q_dev = c->ws.qeff.as<double>();
    }
    // rule weight + basis per point
    std::vector<double> rw3(4 * (size_t)Q);
    for (int q = 0; q < Q; ++q) {
        rw3[4 * q] = c->rule_w[q];
        rw3[4 * q + 1] = 1.0 - c->rule_pts[2 * q] - c->rule_pts[2 * q + 1];
        rw3[4 * q + 2] = c->rule_pts[2 * q];
        rw3[4 * q + 3] = c->rule_pts[2 * q + 1];
    }
    DevBuf &scratch = c->ws.field;  // kept across calls: no allocation on the steady path
    // doubles before the double2 arrays, rounded up to an even count so the
    // double2 arrays start on a 16-byte boundary
    const size_t nd = (4 * (size_t)Q + 6 * (size_t)S + 3 * (size_t)M + 1) & ~(size_t)1;
    const size_t bytes = sizeof(double) * nd + sizeof(double2) * 2 * (size_t)S * R;
    scratch.alloc(bytes);
    double *d_rw = scratch.as<double>();
    double *ys = d_rw + 4 * Q, *ns = ys + 3 * (size_t)S, *d_pts = ns + 3 * (size_t)S;
    double2 *ps = reinterpret_cast<double2 *>(d_rw + nd), *qs = ps + (size_t)S * R;
    BB_CUDA(cudaMemcpyAsync(d_rw, rw3.data(), sizeof(double) * 4 * Q, cudaMemcpyHostToDevice, c->stream));
    BB_CUDA(cudaMemcpyAsync(d_pts, pts_host, sizeof(double) * 3 * M, cudaMemcpyHostToDevice, c->stream));
    field_sources_kernel<<<(F * Q + 255) / 256, 256, 0, c->stream>>>(
        c->d_qpts.as<double>(), c->d_normals.as<double>(), c->d_areas.as<double>(), c->d_faces.as<int>(), F, Q, d_rw,
        N, reinterpret_cast<const double2 *>(p_dev), reinterpret_cast<const double2 *>(q_dev), R, ys, ns, ps, qs,
        images);
    BB_CUDA(cudaGetLastError());
    StagedSources st;
    st.ys = ys;
    st.ns = ns;
    st.pts = d_pts;
    st.ps = ps;
    st.qs = qs;
    st.q = reinterpret_cast<const double2 *>(q_dev);
    st.S = S;
    return st;
}

// CTAs over the source range so that the grid fills the GPU: (grid, sources per CTA)
static std::pair<dim3, int> source_split(const beat_b200_ctx *c, int M, int S, int threads, int chunk) {
    const int mt = (M + threads - 1) / threads;
    const int want = std::max(1, (4 * c->sm_count) / mt);
    int per = std::max(chunk, (S + want - 1) / want);
    per = (per + chunk - 1) / chunk * chunk;
    return {dim3(mt, (S + per - 1) / per), per};
}

void farfield(beat_b200_ctx *c, double k, int M, const double *pts_host, int R, const double *p_dev,
              const double *q_dev, double *out_dev, bool far) {
    BB_REQUIRE(c->F > 0, BEAT_B200_STATE, "no mesh: call beat_b200_set_mesh first");
    BB_REQUIRE(M >= 0 && R >= 1, BEAT_B200_INVALID_ARG, "field: M must be >= 0 and R >= 1");
    if (M == 0) return;
    const StagedSources st = stage_sources(c, M, pts_host, R, p_dev, q_dev);
    BB_CUDA(cudaMemsetAsync(out_dev, 0, sizeof(double2) * (size_t)M * R, c->stream));
    const auto [grid, per] = source_split(c, M, st.S, FLD_THREADS, FLD_CHUNK);
    for (int r0 = 0; r0 < R; r0 += FLD_RC) {
        if (far)
            field_eval_kernel<true><<<grid, FLD_THREADS, 0, c->stream>>>(st.pts, M, st.ys, st.ns, st.ps, st.qs, st.S,
                                                                         R, r0, per, k,
                                                                         reinterpret_cast<double2 *>(out_dev));
        else
            field_eval_kernel<false><<<grid, FLD_THREADS, 0, c->stream>>>(st.pts, M, st.ys, st.ns, st.ps, st.qs, st.S,
                                                                          R, r0, per, k,
                                                                          reinterpret_cast<double2 *>(out_dev));
        BB_CUDA(cudaGetLastError());
    }
    BB_CUDA(cudaStreamSynchronize(c->stream));
}

// ---------------------------------------------------------------------------
// pressure and its gradient (pressure_gradient_v1)
//
// Reference: field_value_gradient, _gradient_triangle,
// _adaptive_gradient_triangle, correct_field_gradient!,
// evaluate_galerkin_field_gradient_cpu (src/BeatEngineFieldGradient.jl:1-88),
// evaluate_galerkin_field_gradient_cuda (src/BeatEngineCudaFieldGradient.jl:
// 1-38).  With r = y - x, u = r / |r|, G = exp(ik|r|) / (4 pi |r|),
// a = ik - 1/|r|, b = 3/|r|^2 - k^2 - 3ik/|r|:
//     value    = G (a (u.n) p - q)
//     gradient = G (a q u - p (b (u.n) u + (a / |r|) n))
// summed over the regular sources, then for every face (and symmetry image)
// whose centroid lies within 3 diameters of the point, the face's regular
// contribution is replaced by adaptive quadrature: the face is split into
// four by its edge midpoints until a piece's diameter is at most 0.4 x the
// distance from the point to its centroid and |k| x diameter <= 0.7, each
// leaf taking the fourth-order rule; a piece still too large at depth 12
// means the point is too close to the boundary (an error, as in the
// reference).  The reference runs that correction on host threads after the
// device sum; here both run on the device, the correction one thread per
// (point, near face) with an explicit subdivision stack.
//
// Output layout: M x 4 x R complex, column-major, component d (0 value,
// 1..3 d/dx, d/dy, d/dz) of column r at out[m + M (d + 4 r)].
// ---------------------------------------------------------------------------
constexpr int FG_RC = 4;          // right-hand sides per pass
constexpr int FG_CHUNK = 32;
constexpr int FG_THREADS = 128;
constexpr int FG_MAX_DEPTH = 12;
constexpr int FG_STACK = 3 * FG_MAX_DEPTH + 1;   // pending pieces of a depth-first split, at most
constexpr int FG_SCALE = 1 << FG_MAX_DEPTH;      // piece vertices are multiples of 1/4096 in face coordinates
constexpr long long FG_PIECE_BUDGET = 1 << 22;   // pieces per (point, face): a bound on runaway refinement
constexpr int FG_ERR_TOO_CLOSE = 1, FG_ERR_BUDGET = 2;

struct GradRule {
    int n;
    double w[8];      // weights (summing to 1/2)
    double b[8][3];   // barycentric coordinates of the points
};

// contribution of one source (weight w) to value + gradient of rc columns;
// P[c], Qn[c]: p and q of column c at the source
template <int RC>
__device__ __forceinline__ void grad_source(double x0, double x1, double x2, double y0, double y1, double y2, double n0,
                                            double n1, double n2, double w, double k, const double2 *P,
                                            const double2 *Qn, double (&acc)[RC][8]) {
    const double rx = y0 - x0, ry = y1 - x1, rz = y2 - x2;
    const double r2 = rx * rx + ry * ry + rz * rz;
    if (r2 == 0.0) return;
    const double ir = rsqrt(r2), rad = r2 * ir;
    const double u[3] = {rx * ir, ry * ir, rz * ir}, nn[3] = {n0, n1, n2};
    double sn_, cs_;
    sincos_cw(k * rad, &sn_, &cs_);
    const double gs = w * 0.07957747154594767 * ir;
    const double gr = cs_ * gs, gi = sn_ * gs;
    // Ga = G a, a = (-1/r, k); Gb = G b, b = (3/r^2 - k^2, -3k/r)
    const double gar = -gr * ir - gi * k, gai = gr * k - gi * ir;
    const double br = 3.0 * ir * ir - k * k, bi = -3.0 * k * ir;
    const double gbr = gr * br - gi * bi, gbi = gr * bi + gi * br;
    const double proj = u[0] * n0 + u[1] * n1 + u[2] * n2;
    double cdr[3], cdi[3];  // G b proj u_d + G a n_d / r
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        cdr[d] = gbr * proj * u[d] + gar * ir * nn[d];
        cdi[d] = gbi * proj * u[d] + gai * ir * nn[d];
    }
#pragma unroll
    for (int cc = 0; cc < RC; ++cc) {
        const double2 p = P[cc], q = Qn[cc];
        acc[cc][0] += (gar * p.x - gai * p.y) * proj - (gr * q.x - gi * q.y);
        acc[cc][1] += (gar * p.y + gai * p.x) * proj - (gr * q.y + gi * q.x);
        const double aqr = gar * q.x - gai * q.y, aqi = gar * q.y + gai * q.x;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            acc[cc][2 + 2 * d] += u[d] * aqr - (cdr[d] * p.x - cdi[d] * p.y);
            acc[cc][3 + 2 * d] += u[d] * aqi - (cdr[d] * p.y + cdi[d] * p.x);
        }
    }
}

// regular sum over the staged sources (weights and densities premultiplied)
template <int RC>
__global__ void __launch_bounds__(FG_THREADS) field_grad_kernel(const double *pts, int M, const double *ys,
                                                                const double *ns, const double2 *ps,
                                                                const double2 *qs, int S, int R, int r0, int per_cta,
                                                                double k, double2 *out) {
    __shared__ double sy[FG_CHUNK][3], sn[FG_CHUNK][3];
    __shared__ double2 sp[FG_CHUNK][RC], sq[FG_CHUNK][RC];
    const int m = blockIdx.x * FG_THREADS + threadIdx.x;
    const int s_begin = blockIdx.y * per_cta, s_end = min(S, s_begin + per_cta);
    const int rc = min(RC, R - r0);
    double x0 = 0, x1 = 0, x2 = 0;
    if (m < M) {
        x0 = pts[3 * m];
        x1 = pts[3 * m + 1];
        x2 = pts[3 * m + 2];
    }
    double acc[RC][8];
#pragma unroll
    for (int r = 0; r < RC; ++r)
#pragma unroll
        for (int e = 0; e < 8; ++e) acc[r][e] = 0.0;
    for (int c0 = s_begin; c0 < s_end; c0 += FG_CHUNK) {
        const int cn = min(FG_CHUNK, s_end - c0);
        __syncthreads();
        for (int i = threadIdx.x; i < cn * 3; i += FG_THREADS) {
            sy[i / 3][i % 3] = ys[3 * (size_t)c0 + i];
            sn[i / 3][i % 3] = ns[3 * (size_t)c0 + i];
        }
        for (int i = threadIdx.x; i < RC * FG_CHUNK; i += FG_THREADS) {
            const int r = i / FG_CHUNK, j = i % FG_CHUNK;
            const bool ok = r < rc && j < cn;
            sp[j][r] = ok ? ps[(size_t)(r0 + r) * S + c0 + j] : make_double2(0, 0);
            sq[j][r] = ok ? qs[(size_t)(r0 + r) * S + c0 + j] : make_double2(0, 0);
        }
        __syncthreads();
        if (m >= M) continue;
        for (int j = 0; j < cn; ++j)
            grad_source<RC>(x0, x1, x2, sy[j][0], sy[j][1], sy[j][2], sn[j][0], sn[j][1], sn[j][2], 1.0, k, sp[j],
                               sq[j], acc);
    }
    if (m < M) {
        for (int r = 0; r < rc; ++r)
#pragma unroll
            for (int d = 0; d < 4; ++d) {
                double2 *o = &out[(size_t)m + (size_t)M * (d + 4 * (size_t)(r0 + r))];
                atomicAdd(&o->x, acc[r][2 * d]);
                atomicAdd(&o->y, acc[r][2 * d + 1]);
            }
    }
}

__device__ __forceinline__ void face_corners(const double *verts, const int *faces, int f, const double *sg,
                                             double (&v)[3][3]) {
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const int vi = faces[3 * f + a];
#pragma unroll
        for (int d = 0; d < 3; ++d) v[a][d] = sg[d] * verts[3 * (size_t)vi + d];
    }
}

__device__ __forceinline__ double tri_diameter(const double (&v)[3][3]) {
    double e[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const int b = (a + 1) % 3;
        const double dx = v[a][0] - v[b][0], dy = v[a][1] - v[b][1], dz = v[a][2] - v[b][2];
        e[a] = sqrt(dx * dx + dy * dy + dz * dz);
    }
    return fmax(fmax(e[0], e[1]), e[2]);
}

__device__ __forceinline__ double dist_to_centroid(const double (&v)[3][3], double x0, double x1, double x2) {
    const double cx = (v[0][0] + v[1][0] + v[2][0]) / 3.0, cy = (v[0][1] + v[1][1] + v[2][1]) / 3.0,
                 cz = (v[0][2] + v[1][2] + v[2][2]) / 3.0;
    const double dx = x0 - cx, dy = x1 - cy, dz = x2 - cz;
    return sqrt(dx * dx + dy * dy + dz * dz);
}

// (point, face copy) pairs with the face's centroid within 3 diameters of the
// point; item = m * (F * copies) + copy * F + f, written while slots last
__global__ void near_pairs_kernel(const double *pts, int M, const double *verts, const int *faces, int F,
                                  FieldImages images, long long *items, long long cap, unsigned long long *count) {
    const long long total = (long long)M * F * images.n;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        const int f = (int)(t % F);
        const long long rest = t / F;
        const int ix = (int)(rest % images.n), m = (int)(rest / images.n);
        double v[3][3];
        face_corners(verts, faces, f, images.s[ix], v);
        const double diam = tri_diameter(v);
        if (dist_to_centroid(v, pts[3 * m], pts[3 * m + 1], pts[3 * m + 2]) <= 3.0 * diam) {
            const unsigned long long slot = atomicAdd(count, 1ull);
            if ((long long)slot < cap) items[slot] = t;
        }
    }
}

// one thread per (near pair, column group): adds adaptive - regular
template <int RC>
__global__ void __launch_bounds__(FG_THREADS) near_correction_kernel(
    const double *pts, int M, const double *verts, const int *faces, const double *normals, int F, int N,
    FieldImages images, const long long *items, long long nitems, const double2 *p, const double2 *q, int R,
    GradRule coarse, GradRule fine, double k, double2 *out, int *err) {
    const long long it = blockIdx.x * (long long)FG_THREADS + threadIdx.x;
    if (it >= nitems) return;
    const int r0 = blockIdx.y * RC, rc = min(RC, R - r0);
    const long long t = items[it];
    const int f = (int)(t % F);
    const long long rest = t / F;
    const int ix = (int)(rest % images.n), m = (int)(rest / images.n);
    const double *sg = images.s[ix];
    const double x0 = pts[3 * m], x1 = pts[3 * m + 1], x2 = pts[3 * m + 2];
    double v[3][3];
    face_corners(verts, faces, f, sg, v);
    const double n0 = sg[0] * normals[3 * f], n1 = sg[1] * normals[3 * f + 1], n2 = sg[2] * normals[3 * f + 2];
    double2 pv[3][RC], qv[RC];
#pragma unroll
    for (int cc = 0; cc < RC; ++cc) {
        const bool ok = cc < rc;
#pragma unroll
        for (int a = 0; a < 3; ++a)
            pv[a][cc] = ok ? p[(size_t)(r0 + cc) * N + faces[3 * f + a]] : make_double2(0, 0);
        qv[cc] = ok ? q[(size_t)(r0 + cc) * F + f] : make_double2(0, 0);
    }
    const double e1[3] = {v[1][0] - v[0][0], v[1][1] - v[0][1], v[1][2] - v[0][2]};
    const double e2[3] = {v[2][0] - v[0][0], v[2][1] - v[0][1], v[2][2] - v[0][2]};
    double acc[RC][8];  // adaptive minus regular
#pragma unroll
    for (int cc = 0; cc < RC; ++cc)
#pragma unroll
        for (int e = 0; e < 8; ++e) acc[cc][e] = 0.0;

    // rule applied (scaled by sign) to the piece with corners pc, which are
    // s[0..2] in face coordinates
    auto integrate = [&](const double (&pc)[3][3], const double (&s)[3][2], const GradRule &rule, double sign) {
        const double a1[3] = {pc[1][0] - pc[0][0], pc[1][1] - pc[0][1], pc[1][2] - pc[0][2]};
        const double a2[3] = {pc[2][0] - pc[0][0], pc[2][1] - pc[0][1], pc[2][2] - pc[0][2]};
        const double cx = a1[1] * a2[2] - a1[2] * a2[1], cy = a1[2] * a2[0] - a1[0] * a2[2],
                     cz = a1[0] * a2[1] - a1[1] * a2[0];
        const double jac = sqrt(cx * cx + cy * cy + cz * cz);
        for (int j = 0; j < rule.n; ++j) {
            const double b0 = rule.b[j][0], b1 = rule.b[j][1], b2 = rule.b[j][2];
            const double y0 = b0 * pc[0][0] + b1 * pc[1][0] + b2 * pc[2][0];
            const double y1 = b0 * pc[0][1] + b1 * pc[1][1] + b2 * pc[2][1];
            const double y2 = b0 * pc[0][2] + b1 * pc[1][2] + b2 * pc[2][2];
            // P1 basis of the face at the point
            const double xi = b0 * s[0][0] + b1 * s[1][0] + b2 * s[2][0];
            const double et = b0 * s[0][1] + b1 * s[1][1] + b2 * s[2][1];
            const double l0 = 1.0 - xi - et;
            double2 P[RC];
#pragma unroll
            for (int cc = 0; cc < RC; ++cc)
                P[cc] = make_double2(l0 * pv[0][cc].x + xi * pv[1][cc].x + et * pv[2][cc].x,
                                     l0 * pv[0][cc].y + xi * pv[1][cc].y + et * pv[2][cc].y);
            grad_source<RC>(x0, x1, x2, y0, y1, y2, n0, n1, n2, sign * jac * rule.w[j], k, P, qv, acc);
        }
    };

    {  // the regular rule on the whole face: what the regular sum added
        const double s[3][2] = {{0, 0}, {1, 0}, {0, 1}};
        integrate(v, s, coarse, -1.0);
    }
    // depth-first split; a piece is three corners in face coordinates
    // (multiples of 1/4096 while depth <= 12, so exact in 16-bit integers)
    struct Piece {
        unsigned short c[3][2];
        unsigned char depth;
    };
    Piece stack[FG_STACK];
    int top = 0;
    stack[top++] = Piece{{{0, 0}, {FG_SCALE, 0}, {0, FG_SCALE}}, 0};
    long long pieces = 0;
    const double inv = 1.0 / FG_SCALE;
    while (top > 0) {
        const Piece pc = stack[--top];
        double s[3][2], g[3][3];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            s[a][0] = pc.c[a][0] * inv;
            s[a][1] = pc.c[a][1] * inv;
#pragma unroll
            for (int d = 0; d < 3; ++d) g[a][d] = v[0][d] + s[a][0] * e1[d] + s[a][1] * e2[d];
        }
        const double diam = tri_diameter(g);
        if (diam <= 0.4 * dist_to_centroid(g, x0, x1, x2) && fabs(k) * diam <= 0.7) {
            integrate(g, s, fine, 1.0);
            continue;
        }
        if (pc.depth >= FG_MAX_DEPTH) {
            atomicOr(err, FG_ERR_TOO_CLOSE);
            return;
        }
        if (++pieces > FG_PIECE_BUDGET) {
            atomicOr(err, FG_ERR_BUDGET);
            return;
        }
        unsigned short mid[3][2];  // ab, bc, ca
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int d = 0; d < 2; ++d)
                mid[a][d] = (unsigned short)((pc.c[a][d] + pc.c[(a + 1) % 3][d]) / 2);
        const unsigned char dd = pc.depth + 1;
        // children (a, ab, ca), (ab, b, bc), (ca, bc, c), (ab, bc, ca)
        stack[top++] = Piece{{{mid[0][0], mid[0][1]}, {mid[1][0], mid[1][1]}, {mid[2][0], mid[2][1]}}, dd};
        stack[top++] = Piece{{{mid[2][0], mid[2][1]}, {mid[1][0], mid[1][1]}, {pc.c[2][0], pc.c[2][1]}}, dd};
        stack[top++] = Piece{{{mid[0][0], mid[0][1]}, {pc.c[1][0], pc.c[1][1]}, {mid[1][0], mid[1][1]}}, dd};
        stack[top++] = Piece{{{pc.c[0][0], pc.c[0][1]}, {mid[0][0], mid[0][1]}, {mid[2][0], mid[2][1]}}, dd};
    }
    for (int cc = 0; cc < rc; ++cc)
#pragma unroll
        for (int d = 0; d < 4; ++d) {
            double2 *o = &out[(size_t)m + (size_t)M * (d + 4 * (size_t)(r0 + cc))];
            atomicAdd(&o->x, acc[cc][2 * d]);
            atomicAdd(&o->y, acc[cc][2 * d + 1]);
        }
}

static GradRule grad_rule(const std::vector<double> &pts, const std::vector<double> &w) {
    GradRule r{};
    r.n = (int)w.size();
    for (int j = 0; j < r.n; ++j) {
        r.w[j] = w[j];
        r.b[j][0] = 1.0 - pts[2 * j] - pts[2 * j + 1];
        r.b[j][1] = pts[2 * j];
        r.b[j][2] = pts[2 * j + 1];
    }
    return r;
}

void field_gradient(beat_b200_ctx *c, double k, int M, const double *pts_host, int R, const double *p_dev,
                    const double *q_dev, double *out_dev) {
    BB_REQUIRE(c->F > 0, BEAT_B200_STATE, "no mesh: call beat_b200_set_mesh first");
    BB_REQUIRE(M >= 0 && R >= 1, BEAT_B200_INVALID_ARG, "field gradient: M must be >= 0 and R >= 1");
    if (M == 0) return;
    const int F = c->F, N = c->V;
    const StagedSources st = stage_sources(c, M, pts_host, R, p_dev, q_dev);
    double2 *out = reinterpret_cast<double2 *>(out_dev);
    BB_CUDA(cudaMemsetAsync(out, 0, sizeof(double2) * 4 * (size_t)M * R, c->stream));
    {
        const auto [grid, per] = source_split(c, M, st.S, FG_THREADS, FG_CHUNK);
        for (int r0 = 0; r0 < R; r0 += FG_RC) {
            if (R == 1)
                field_grad_kernel<1><<<grid, FG_THREADS, 0, c->stream>>>(st.pts, M, st.ys, st.ns, st.ps, st.qs, st.S,
                                                                         R, r0, per, k, out);
            else
                field_grad_kernel<FG_RC><<<grid, FG_THREADS, 0, c->stream>>>(st.pts, M, st.ys, st.ns, st.ps, st.qs,
                                                                             st.S, R, r0, per, k, out);
            BB_CUDA(cudaGetLastError());
        }
    }
    FieldImages images;
    images.n = 1 + c->nimg;
    for (int i = 0; i < 3; ++i) images.s[0][i] = 1.0;
    for (int ix = 0; ix < c->nimg; ++ix)
        for (int i = 0; i < 3; ++i) images.s[1 + ix][i] = c->img_sign[ix][i];
    // near pairs: count and list in one pass; a second pass if the list overflowed
    DevBuf &nb = c->ws.grad;  // [count u64][error int, pad][items i64 ...], grow-only
    const size_t head = 16;
    long long cap = nb.bytes > head ? (long long)((nb.bytes - head) / sizeof(long long)) : 0;
    if (cap < 1024) {
        nb.alloc(head + 1024 * sizeof(long long));
        cap = 1024;
    }
    const long long total = (long long)M * F * images.n;
    const int blocks = (int)std::min<long long>((total + 255) / 256, 16LL * c->sm_count);
    unsigned long long count = 0;
    for (int pass = 0; pass < 2; ++pass) {
        BB_CUDA(cudaMemsetAsync(nb.p, 0, head, c->stream));
        near_pairs_kernel<<<blocks, 256, 0, c->stream>>>(
            st.pts, M, c->d_verts.as<double>(), c->d_faces.as<int>(), F, images,
            reinterpret_cast<long long *>(static_cast<char *>(nb.p) + head), cap,
            static_cast<unsigned long long *>(nb.p));
        BB_CUDA(cudaGetLastError());
        BB_CUDA(cudaMemcpyAsync(&count, nb.p, sizeof(count), cudaMemcpyDeviceToHost, c->stream));
        BB_CUDA(cudaStreamSynchronize(c->stream));
        if ((long long)count <= cap) break;
        BB_REQUIRE(pass == 0, BEAT_B200_CUDA_ERROR, "field gradient: near-pair list overflowed twice");
        cap = (long long)count;
        nb.alloc(head + (size_t)cap * sizeof(long long));
    }
    int err = 0;
    if (count > 0) {
        std::vector<double> p4, w4;
        triangle_rule(4, p4, w4);
        const GradRule coarse = grad_rule(c->rule_pts, c->rule_w), fine = grad_rule(p4, w4);
        int *d_err = reinterpret_cast<int *>(static_cast<char *>(nb.p) + 8);
        const long long *items = reinterpret_cast<const long long *>(static_cast<char *>(nb.p) + head);
        const unsigned nblk = (unsigned)((count + FG_THREADS - 1) / FG_THREADS);
        if (R == 1)
            near_correction_kernel<1><<<dim3(nblk, 1), FG_THREADS, 0, c->stream>>>(
                st.pts, M, c->d_verts.as<double>(), c->d_faces.as<int>(), c->d_normals.as<double>(), F, N, images,
                items, (long long)count, reinterpret_cast<const double2 *>(p_dev), st.q, R, coarse, fine, k, out,
                d_err);
        else
            near_correction_kernel<FG_RC><<<dim3(nblk, (R + FG_RC - 1) / FG_RC), FG_THREADS, 0, c->stream>>>(
                st.pts, M, c->d_verts.as<double>(), c->d_faces.as<int>(), c->d_normals.as<double>(), F, N, images,
                items, (long long)count, reinterpret_cast<const double2 *>(p_dev), st.q, R, coarse, fine, k, out,
                d_err);
        BB_CUDA(cudaGetLastError());
        BB_CUDA(cudaMemcpyAsync(&err, d_err, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    }
    BB_CUDA(cudaStreamSynchronize(c->stream));
    BB_REQUIRE(!(err & FG_ERR_TOO_CLOSE), BEAT_B200_INVALID_ARG,
               "field gradient: a point is too close to the boundary for reliable evaluation");
    BB_REQUIRE(!(err & FG_ERR_BUDGET), BEAT_B200_INVALID_ARG,
               "field gradient: adaptive refinement exceeded its piece budget (mesh too coarse for k)");
}

}  // namespace bb
