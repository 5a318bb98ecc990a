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

#include <cmath>

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
                const double rad = sqrt(rx * rx + ry * ry + rz * rz);
                if (rad == 0.0) continue;
                const double ir = 1.0 / rad;
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

void farfield(beat_b200_ctx *c, double k, int M, const double *pts_host, int R, const double *p_dev,
              const double *q_dev, double *out_dev, bool far) {
    BB_REQUIRE(c->F > 0, BEAT_B200_STATE, "no mesh: call beat_b200_set_mesh first");
    BB_REQUIRE(M >= 0 && R >= 1, BEAT_B200_INVALID_ARG, "field: M must be >= 0 and R >= 1");
    if (M == 0) return;
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
    {
        double *d_rw = scratch.as<double>();
        double *ys = d_rw + 4 * Q, *ns = ys + 3 * (size_t)S, *d_pts = ns + 3 * (size_t)S;
        double2 *ps = reinterpret_cast<double2 *>(d_rw + nd), *qs = ps + (size_t)S * R;
        BB_CUDA(cudaMemcpyAsync(d_rw, rw3.data(), sizeof(double) * 4 * Q, cudaMemcpyHostToDevice, c->stream));
        BB_CUDA(cudaMemcpyAsync(d_pts, pts_host, sizeof(double) * 3 * M, cudaMemcpyHostToDevice, c->stream));
        BB_CUDA(cudaMemsetAsync(out_dev, 0, sizeof(double2) * (size_t)M * R, c->stream));
        field_sources_kernel<<<(F * Q + 255) / 256, 256, 0, c->stream>>>(
            c->d_qpts.as<double>(), c->d_normals.as<double>(), c->d_areas.as<double>(), c->d_faces.as<int>(), F, Q,
            d_rw, N, reinterpret_cast<const double2 *>(p_dev), reinterpret_cast<const double2 *>(q_dev), R, ys, ns, ps,
            qs, images);
        BB_CUDA(cudaGetLastError());
        const int mt = (M + FLD_THREADS - 1) / FLD_THREADS;
        const int want = std::max(1, (4 * c->sm_count) / mt);
        int per = std::max(FLD_CHUNK, (S + want - 1) / want);
        per = (per + FLD_CHUNK - 1) / FLD_CHUNK * FLD_CHUNK;
        dim3 grid(mt, (S + per - 1) / per);
        for (int r0 = 0; r0 < R; r0 += FLD_RC) {
            if (far)
                field_eval_kernel<true><<<grid, FLD_THREADS, 0, c->stream>>>(d_pts, M, ys, ns, ps, qs, S, R, r0, per, k,
                                                                             reinterpret_cast<double2 *>(out_dev));
            else
                field_eval_kernel<false><<<grid, FLD_THREADS, 0, c->stream>>>(d_pts, M, ys, ns, ps, qs, S, R, r0, per,
                                                                              k, reinterpret_cast<double2 *>(out_dev));
            BB_CUDA(cudaGetLastError());
        }
        BB_CUDA(cudaStreamSynchronize(c->stream));
    }
}

}  // namespace bb
