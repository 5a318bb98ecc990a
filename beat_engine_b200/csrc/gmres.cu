// gmres.cu -- FP64 GMRES iterative refinement of the mixed-precision solve.
//
// Right-preconditioned restarted GMRES (flexible form: the preconditioned
// directions Z are kept) on the assembled operator A, one independent Krylov
// space per right-hand side, all columns advanced in lock-step:
//   operator      y = A x with A stored in FP32, arithmetic and vectors FP64
//   preconditioner z = (L U)^-1 P v with the FP32 factors (lu.cu)
//   orthogonalisation classical Gram-Schmidt with one re-orthogonalisation
//   convergence  ||b - A x|| / ||b|| <= rtol for every column
// The reference's nearest counterparts are beat_gmres! (FP64 Krylov space,
// src/BeatEngineDenseSolve.jl:521-665) and beat_refine_cpu_lu (FP64 residual
// of a ComplexF32 LU, src/BeatEngineCpuRefinement.jl:5-78).  Like the latter
// this refines the operator as assembled: FP32 regular-pair arithmetic stays
// in the answer (about 1e-7 relative on these systems).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <complex>
#include <vector>

#include "internal.cuh"

namespace bb {

// ---------------------------------------------------------------------------
// Tall-skinny complex product Y += alpha M X (M rows x K complex in the
// workspace precision, row-major; X, Y FP64 column-major with R columns).
// One thread per row of M, all TG_RC right-hand sides of a chunk in FP64
// registers: an M entry read from shared memory feeds 4 TG_RC DFMA, the X
// entries are warp-broadcast loads.  The K range is cut into slices so that
// about two CTAs per SM are resident; slices add into Y with FP64 atomics.
// Bound: FP64 FMA issue (4 DFMA per complex multiply-add).
// ---------------------------------------------------------------------------
constexpr int TG_THREADS = 256, TG_RC = 16;

// one 8- or 16-byte element global -> shared through the asynchronous copy
// unit, or zeros (nothing is read) when `in` is false
template <typename E> __device__ __forceinline__ void cp_async_zfill(E *smem, const E *gmem, bool in) {
    static_assert(sizeof(E) == 8 || sizeof(E) == 16, "8- or 16-byte elements");
    const unsigned dst = (unsigned)__cvta_generic_to_shared(smem);
    const int n = in ? (int)sizeof(E) : 0;
    if constexpr (sizeof(E) == 8)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(dst), "l"(gmem), "r"(n) : "memory");
    else
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(gmem), "r"(n) : "memory");
}
template <typename T> struct TgChunk {
    static constexpr int KC = 32;  // K entries per shared-memory chunk (c64 M)
    static constexpr int STAGE_UNROLL = 1;  // unrolling of the chunk's copy loop (no spills at 128 registers)
};
template <> struct TgChunk<double> {
    static constexpr int KC = 16;
    static constexpr int STAGE_UNROLL = 4;
};

template <typename T>
__global__ void __launch_bounds__(TG_THREADS, 2) tall_gemm_kernel(const Cx<T> *M, int64_t ld, int rows, int K,
                                                                  const double2 *X, double2 *Y, int R, int r0,
                                                                  double alpha, int kslice) {
    constexpr int KC = TgChunk<T>::KC;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Cx<T> *sM = reinterpret_cast<Cx<T> *>(smem_raw);                                          // TG_THREADS x (KC + 1)
    double2 *sX = reinterpret_cast<double2 *>(smem_raw + sizeof(Cx<T>) * TG_THREADS * (KC + 1));  // KC x TG_RC
    const int row0 = blockIdx.x * TG_THREADS, row = row0 + (int)threadIdx.x;
    const int kb = blockIdx.y * kslice, ke = min(K, kb + kslice);
    const int rc = min(TG_RC, R - r0);
    double ar[TG_RC], ai[TG_RC];
#pragma unroll
    for (int e = 0; e < TG_RC; ++e) ar[e] = ai[e] = 0.0;
    for (int k0 = kb; k0 < ke; k0 += KC) {
        const int kn = min(KC, ke - k0);
        // the chunk of M and of X by asynchronous copies, all in flight at
        // once; entries past the matrix are zero-filled
#pragma unroll TgChunk<T>::STAGE_UNROLL
        for (int i = threadIdx.x; i < TG_THREADS * KC; i += TG_THREADS) {
            const int r = i / KC, k = i % KC;  // consecutive threads: consecutive k of one row
            const bool in = row0 + r < rows && k < kn;
            cp_async_zfill(&sM[r * (KC + 1) + k], in ? &M[(int64_t)(row0 + r) * ld + k0 + k] : M, in);
        }
        for (int i = threadIdx.x; i < KC * TG_RC; i += TG_THREADS) {
            const int c = i / KC, k = i % KC;
            const bool in = c < rc && k < kn;
            cp_async_zfill(&sX[k * TG_RC + c], in ? &X[(size_t)(r0 + c) * K + k0 + k] : X, in);
        }
        asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
        __syncthreads();
#pragma unroll 2
        for (int k = 0; k < KC; ++k) {
            const Cx<T> m = sM[threadIdx.x * (KC + 1) + k];
            const double mr = (double)m.re, mi = (double)m.im;
#pragma unroll
            for (int e = 0; e < TG_RC; ++e) {
                const double2 x = sX[k * TG_RC + e];
                ar[e] = fma(mr, x.x, fma(-mi, x.y, ar[e]));
                ai[e] = fma(mr, x.y, fma(mi, x.x, ai[e]));
            }
        }
        __syncthreads();
    }
    if (row < rows) {
#pragma unroll
        for (int e = 0; e < TG_RC; ++e)
            if (e < rc) {
                double2 *y = &Y[(size_t)(r0 + e) * rows + row];
                atomicAdd(&y->x, alpha * ar[e]);
                atomicAdd(&y->y, alpha * ai[e]);
            }
    }
}

// Y += alpha * M X for all R columns (Y must hold its starting value)
template <typename T>
void tall_gemm(cudaStream_t st, int sm_count, const Cx<T> *M, int64_t ld, int rows, int K, const double *X, double *Y,
               int R, double alpha) {
    constexpr int KC = TgChunk<T>::KC;
    const size_t smem = sizeof(Cx<T>) * TG_THREADS * (KC + 1) + sizeof(double2) * KC * TG_RC;
    BB_CUDA(cudaFuncSetAttribute(tall_gemm_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const int row_tiles = (rows + TG_THREADS - 1) / TG_THREADS;
    // K slices so that about two CTAs per SM run
    int slices = std::max(1, (2 * sm_count + row_tiles / 2) / row_tiles);
    int kslice = (K + slices - 1) / slices;
    kslice = (kslice + KC - 1) / KC * KC;
    slices = (K + kslice - 1) / kslice;
    for (int r0 = 0; r0 < R; r0 += TG_RC)
        tall_gemm_kernel<T><<<dim3(row_tiles, slices), TG_THREADS, smem, st>>>(
            M, ld, rows, K, reinterpret_cast<const double2 *>(X), reinterpret_cast<double2 *>(Y), R, r0, alpha, kslice);
    BB_CUDA(cudaGetLastError());
}
template void tall_gemm<float>(cudaStream_t, int, const Cx<float> *, int64_t, int, int, const double *, double *, int,
                               double);
template void tall_gemm<double>(cudaStream_t, int, const Cx<double> *, int64_t, int, int, const double *, double *,
                                int, double);

// ---------------------------------------------------------------------------
// Conjugate-transposed tall product Y += alpha M^H X: M complex row-major
// rows x cols, X FP64 column-major rows x R, Y FP64 column-major cols x R.
// One thread per column of M (consecutive threads read consecutive entries of
// a row), all TG_RC right-hand sides in FP64 registers, rows of X staged
// through shared memory; row slices add into Y with FP64 atomics.  Used by
// the adjoint (B^H, and A^H inside the adjoint refinement).
// ---------------------------------------------------------------------------
constexpr int TGH_KC = 32;

template <typename T>
__global__ void __launch_bounds__(TG_THREADS, 2) tall_gemm_h_kernel(const Cx<T> *M, int64_t ld, int rows, int cols,
                                                                    const double2 *X, double2 *Y, int R, int r0,
                                                                    double alpha, int islice) {
    __shared__ double2 sX[TGH_KC][TG_RC];
    const int j = blockIdx.x * TG_THREADS + (int)threadIdx.x;
    const int ib = blockIdx.y * islice, ie = min(rows, ib + islice);
    const int rc = min(TG_RC, R - r0);
    double ar[TG_RC], ai[TG_RC];
#pragma unroll
    for (int e = 0; e < TG_RC; ++e) ar[e] = ai[e] = 0.0;
    for (int i0 = ib; i0 < ie; i0 += TGH_KC) {
        const int kn = min(TGH_KC, ie - i0);
        __syncthreads();
        for (int t = threadIdx.x; t < TGH_KC * TG_RC; t += TG_THREADS) {
            const int cidx = t / TGH_KC, k = t % TGH_KC;
            sX[k][cidx] = (cidx < rc && k < kn) ? X[(size_t)(r0 + cidx) * rows + i0 + k] : make_double2(0, 0);
        }
        __syncthreads();
        if (j < cols) {
#pragma unroll 4
            for (int k = 0; k < kn; ++k) {
                const Cx<T> m = M[(int64_t)(i0 + k) * ld + j];
                const double mr = (double)m.re, mi = -(double)m.im;  // conj(M[i][j])
#pragma unroll
                for (int e = 0; e < TG_RC; ++e) {
                    const double2 x = sX[k][e];
                    ar[e] = fma(mr, x.x, fma(-mi, x.y, ar[e]));
                    ai[e] = fma(mr, x.y, fma(mi, x.x, ai[e]));
                }
            }
        }
    }
    if (j < cols) {
#pragma unroll
        for (int e = 0; e < TG_RC; ++e)
            if (e < rc) {
                double2 *y = &Y[(size_t)(r0 + e) * cols + j];
                atomicAdd(&y->x, alpha * ar[e]);
                atomicAdd(&y->y, alpha * ai[e]);
            }
    }
}

template <typename T>
void tall_gemm_h(cudaStream_t st, int sm_count, const Cx<T> *M, int64_t ld, int rows, int cols, const double *X,
                 double *Y, int R, double alpha) {
    const int col_tiles = (cols + TG_THREADS - 1) / TG_THREADS;
    int slices = std::max(1, (2 * sm_count + col_tiles / 2) / col_tiles);
    int islice = (rows + slices - 1) / slices;
    islice = (islice + TGH_KC - 1) / TGH_KC * TGH_KC;
    slices = (rows + islice - 1) / islice;
    for (int r0 = 0; r0 < R; r0 += TG_RC)
        tall_gemm_h_kernel<T><<<dim3(col_tiles, slices), TG_THREADS, 0, st>>>(
            M, ld, rows, cols, reinterpret_cast<const double2 *>(X), reinterpret_cast<double2 *>(Y), R, r0, alpha,
            islice);
    BB_CUDA(cudaGetLastError());
}
template void tall_gemm_h<float>(cudaStream_t, int, const Cx<float> *, int64_t, int, int, const double *, double *,
                                 int, double);
template void tall_gemm_h<double>(cudaStream_t, int, const Cx<double> *, int64_t, int, int, const double *,
                                  double *, int, double);

// Y = alpha * A X + beta * Y with beta in {0, 1}
// (with ADJ: Y = alpha * A^H X + beta * Y)
template <typename T, bool ADJ = false>
static void matvec(beat_b200_ctx *c, const Cx<T> *A, const double *X, double *Y, int R, double alpha, double beta) {
    const int n = c->V;
    if (beta == 0.0) BB_CUDA(cudaMemsetAsync(Y, 0, sizeof(double2) * (size_t)n * R, c->stream));
    if (ADJ)
        tall_gemm_h<T>(c->stream, c->sm_count, A, c->ws.ld, n, n, X, Y, R, alpha);
    else
        tall_gemm<T>(c->stream, c->sm_count, A, c->ws.ld, n, n, X, Y, R, alpha);
}

// H[i*R + r] = sum_n conj(V_i[n, r]) W[n, r] for i < nv   (one CTA per (i, r))
__global__ void block_dot_kernel(const double2 *V, size_t vstride, int nv, const double2 *W, int n, int R,
                                 double2 *H) {
    const int i = blockIdx.x / R, r = blockIdx.x % R;
    if (i >= nv) return;
    const double2 *v = V + i * vstride + (size_t)r * n, *w = W + (size_t)r * n;
    double sr = 0, si = 0;
    for (int t = threadIdx.x; t < n; t += blockDim.x) {
        const double2 a = v[t], b = w[t];
        sr += a.x * b.x + a.y * b.y;
        si += a.x * b.y - a.y * b.x;
    }
    __shared__ double rr[32], ri[32];
    for (int o = 16; o > 0; o >>= 1) {
        sr += __shfl_xor_sync(0xffffffffu, sr, o);
        si += __shfl_xor_sync(0xffffffffu, si, o);
    }
    if ((threadIdx.x & 31) == 0) {
        rr[threadIdx.x >> 5] = sr;
        ri[threadIdx.x >> 5] = si;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0, b = 0;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) {
            a += rr[k];
            b += ri[k];
        }
        H[(size_t)i * R + r] = make_double2(a, b);
    }
}

// W[:, r] -= sum_i V_i[:, r] H[i, r]; optionally accumulates H into Hacc
__global__ void block_axpy_kernel(const double2 *V, size_t vstride, int nv, double2 *W, int n, int R,
                                  const double2 *H, double2 *Hacc) {
    const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx < (size_t)nv * R && Hacc) {
        Hacc[idx].x += H[idx].x;
        Hacc[idx].y += H[idx].y;
    }
    if (idx >= (size_t)n * R) return;
    const int r = (int)(idx / n);
    double sr = 0, si = 0;
    for (int i = 0; i < nv; ++i) {
        const double2 v = V[i * vstride + idx], h = H[(size_t)i * R + r];
        sr += v.x * h.x - v.y * h.y;
        si += v.x * h.y + v.y * h.x;
    }
    W[idx].x -= sr;
    W[idx].y -= si;
}

// column norms: out[r] = ||W[:, r]||^2 (real, stored in .x)
__global__ void col_norm2_kernel(const double2 *W, int n, int R, double2 *out) {
    const int r = blockIdx.x;
    double s = 0;
    for (int t = threadIdx.x; t < n; t += blockDim.x) {
        const double2 a = W[(size_t)r * n + t];
        s += a.x * a.x + a.y * a.y;
    }
    __shared__ double red[32];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) a += red[k];
        out[r] = make_double2(a, 0.0);
    }
}

// dst[:, r] = src[:, r] * scale[r] (real scale)
__global__ void col_scale_kernel(const double2 *src, double2 *dst, int n, int R, const double *scale) {
    const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (size_t)n * R) return;
    const double s = scale[idx / n];
    dst[idx] = make_double2(src[idx].x * s, src[idx].y * s);
}

// x[:, r] += sum_i Z_i[:, r] y[i, r]
__global__ void update_x_kernel(const double2 *Z, size_t zstride, int nz, double2 *X, int n, int R,
                                const double2 *y) {
    const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (size_t)n * R) return;
    const int r = (int)(idx / n);
    double sr = 0, si = 0;
    for (int i = 0; i < nz; ++i) {
        const double2 z = Z[i * zstride + idx], h = y[(size_t)i * R + r];
        sr += z.x * h.x - z.y * h.y;
        si += z.x * h.y + z.y * h.x;
    }
    X[idx].x += sr;
    X[idx].y += si;
}

using cd = std::complex<double>;

// FGMRES on A (ADJ: on A^H) with the FP32 LU (ADJ: its conjugate transpose)
// as right preconditioner
template <typename T, bool ADJ>
static IrResult gmres_t(beat_b200_ctx *c, int R, double *x_dev, const double *b_dev, int m, int max_iters,
                        double rtol) {
    Workspace &w = c->ws;
    const int n = c->V;
    const size_t vs = (size_t)n * R;  // stride between basis vectors (complex entries)
    const Cx<T> *A = (sizeof(T) == 8) ? w.A.as<Cx<T>>() : w.Aop.as<Cx<T>>();
    w.krylov.alloc(sizeof(double2) * vs * (2 * (size_t)m + 3));
    double2 *V = w.krylov.as<double2>();          // m + 1 vectors
    double2 *Z = V + vs * (m + 1);                // m vectors
    double2 *W = Z + vs * m;                      // work vector
    w.small.alloc(sizeof(double2) * ((size_t)(m + 2) * R * 3 + 4 * R));
    double2 *dH = w.small.as<double2>();          // (m+1) x R
    double2 *dH2 = dH + (size_t)(m + 2) * R;
    double2 *dY = dH2 + (size_t)(m + 2) * R;
    double *dscale = reinterpret_cast<double *>(dY + (size_t)(m + 2) * R);
    const int th = 256;
    const unsigned blocks_nr = (unsigned)((vs + th - 1) / th);

    std::vector<double> bnorm(R), res(R, 1.0);
    std::vector<double2> hbuf((size_t)(m + 2) * R);
    col_norm2_kernel<<<R, 256, 0, c->stream>>>(reinterpret_cast<const double2 *>(b_dev), n, R, dH);
    BB_CUDA(cudaMemcpyAsync(hbuf.data(), dH, sizeof(double2) * R, cudaMemcpyDeviceToHost, c->stream));
    BB_CUDA(cudaStreamSynchronize(c->stream));
    for (int r = 0; r < R; ++r) bnorm[r] = std::sqrt(hbuf[r].x);

    int iters = 0;
    bool converged = false;
    std::vector<std::vector<cd>> H(R, std::vector<cd>((size_t)(m + 1) * m));
    std::vector<std::vector<cd>> g(R, std::vector<cd>(m + 1)), cs(R, std::vector<cd>(m)), sn(R, std::vector<cd>(m));
    std::vector<double> cs_r;
    while (iters < max_iters) {
        // r = b - A x
        BB_CUDA(cudaMemcpyAsync(W, b_dev, sizeof(double2) * vs, cudaMemcpyDeviceToDevice, c->stream));
        matvec<T, ADJ>(c, A, x_dev, reinterpret_cast<double *>(W), R, -1.0, 1.0);
        col_norm2_kernel<<<R, 256, 0, c->stream>>>(W, n, R, dH);
        BB_CUDA(cudaMemcpyAsync(hbuf.data(), dH, sizeof(double2) * R, cudaMemcpyDeviceToHost, c->stream));
        BB_CUDA(cudaStreamSynchronize(c->stream));
        std::vector<double> beta(R), sc(R);
        converged = true;
        for (int r = 0; r < R; ++r) {
            beta[r] = std::sqrt(hbuf[r].x);
            res[r] = bnorm[r] > 0 ? beta[r] / bnorm[r] : (beta[r] == 0 ? 0.0 : INFINITY);
            if (!(res[r] <= rtol)) converged = false;
            sc[r] = beta[r] > 0 ? 1.0 / beta[r] : 0.0;
            std::fill(g[r].begin(), g[r].end(), cd(0));
            g[r][0] = beta[r];
        }
        if (converged) break;
        BB_CUDA(cudaMemcpyAsync(dscale, sc.data(), sizeof(double) * R, cudaMemcpyHostToDevice, c->stream));
        col_scale_kernel<<<blocks_nr, th, 0, c->stream>>>(W, V, n, R, dscale);
        int j = 0;
        for (; j < m && iters < max_iters; ++j, ++iters) {
            if (ADJ)
                lu_solve_adjoint(c, R, reinterpret_cast<const double *>(V + vs * j),
                                 reinterpret_cast<double *>(Z + vs * j));
            else
                lu_precond_fp32(c, R, reinterpret_cast<const double *>(V + vs * j),
                                reinterpret_cast<double *>(Z + vs * j));
            matvec<T, ADJ>(c, A, reinterpret_cast<const double *>(Z + vs * j), reinterpret_cast<double *>(W), R, 1.0,
                           0.0);
            // CGS2
            BB_CUDA(cudaMemsetAsync(dH2, 0, sizeof(double2) * (size_t)(j + 1) * R, c->stream));
            for (int pass = 0; pass < 2; ++pass) {
                block_dot_kernel<<<(j + 1) * R, 256, 0, c->stream>>>(V, vs, j + 1, W, n, R, dH);
                block_axpy_kernel<<<blocks_nr, th, 0, c->stream>>>(V, vs, j + 1, W, n, R, dH, dH2);
            }
            col_norm2_kernel<<<R, 256, 0, c->stream>>>(W, n, R, dH2 + (size_t)(j + 1) * R);
            BB_CUDA(cudaMemcpyAsync(hbuf.data(), dH2, sizeof(double2) * (size_t)(j + 2) * R, cudaMemcpyDeviceToHost,
                                    c->stream));
            BB_CUDA(cudaStreamSynchronize(c->stream));
            bool all_ok = true;
            for (int r = 0; r < R; ++r) {
                std::vector<cd> &h = H[r];
                for (int i = 0; i <= j; ++i) h[(size_t)i * m + j] = cd(hbuf[(size_t)i * R + r].x, hbuf[(size_t)i * R + r].y);
                const double hn = std::sqrt(hbuf[(size_t)(j + 1) * R + r].x);
                sc[r] = hn > 0 ? 1.0 / hn : 0.0;
                // apply previous rotations
                for (int i = 0; i < j; ++i) {
                    const cd a = h[(size_t)i * m + j], b = h[(size_t)(i + 1) * m + j];
                    h[(size_t)i * m + j] = std::conj(cs[r][i]) * a + std::conj(sn[r][i]) * b;
                    h[(size_t)(i + 1) * m + j] = -sn[r][i] * a + cs[r][i] * b;
                }
                const cd a = h[(size_t)j * m + j];
                const double den = std::sqrt(std::norm(a) + hn * hn);
                if (den > 0) {
                    cs[r][j] = a / den;
                    sn[r][j] = cd(hn / den, 0.0);
                } else {
                    cs[r][j] = 1.0;
                    sn[r][j] = 0.0;
                }
                h[(size_t)j * m + j] = std::conj(cs[r][j]) * a + std::conj(sn[r][j]) * hn;
                const cd gj = g[r][j];
                g[r][j] = std::conj(cs[r][j]) * gj;
                g[r][j + 1] = -sn[r][j] * gj;
                const double est = bnorm[r] > 0 ? std::abs(g[r][j + 1]) / bnorm[r] : 0.0;
                if (!(est <= rtol)) all_ok = false;
            }
            BB_CUDA(cudaMemcpyAsync(dscale, sc.data(), sizeof(double) * R, cudaMemcpyHostToDevice, c->stream));
            col_scale_kernel<<<blocks_nr, th, 0, c->stream>>>(W, V + vs * (j + 1), n, R, dscale);
            if (all_ok) {
                ++j;
                ++iters;
                break;
            }
        }
        // back substitution per column, x += Z y
        std::vector<double2> yv((size_t)j * R);
        for (int r = 0; r < R; ++r) {
            std::vector<cd> y(j);
            for (int i = j - 1; i >= 0; --i) {
                cd s = g[r][i];
                for (int l = i + 1; l < j; ++l) s -= H[r][(size_t)i * m + l] * y[l];
                const cd d = H[r][(size_t)i * m + i];
                y[i] = std::abs(d) > 0 ? s / d : cd(0);
            }
            for (int i = 0; i < j; ++i) yv[(size_t)i * R + r] = make_double2(y[i].real(), y[i].imag());
        }
        BB_CUDA(cudaMemcpyAsync(dY, yv.data(), sizeof(double2) * yv.size(), cudaMemcpyHostToDevice, c->stream));
        update_x_kernel<<<blocks_nr, th, 0, c->stream>>>(Z, vs, j, reinterpret_cast<double2 *>(x_dev), n, R, dY);
        BB_CUDA(cudaGetLastError());
    }
    if (!converged) {
        // final true residual
        BB_CUDA(cudaMemcpyAsync(W, b_dev, sizeof(double2) * vs, cudaMemcpyDeviceToDevice, c->stream));
        matvec<T, ADJ>(c, A, x_dev, reinterpret_cast<double *>(W), R, -1.0, 1.0);
        col_norm2_kernel<<<R, 256, 0, c->stream>>>(W, n, R, dH);
        BB_CUDA(cudaMemcpyAsync(hbuf.data(), dH, sizeof(double2) * R, cudaMemcpyDeviceToHost, c->stream));
        BB_CUDA(cudaStreamSynchronize(c->stream));
        converged = true;
        for (int r = 0; r < R; ++r) {
            res[r] = bnorm[r] > 0 ? std::sqrt(hbuf[r].x) / bnorm[r] : 0.0;
            if (!(res[r] <= rtol)) converged = false;
        }
    }
    double worst = 0;
    for (int r = 0; r < R; ++r) worst = std::max(worst, res[r]);
    return IrResult{iters, converged ? 1 : 0, worst};
}

IrResult gmres_refine(beat_b200_ctx *c, int R, double *x_dev, const double *b_dev, int restart, int max_iters,
                      double rtol) {
    BB_REQUIRE(restart >= 1 && restart <= 200, BEAT_B200_INVALID_ARG, "GMRES restart must be in 1..200");
    BB_REQUIRE(rtol > 0 && std::isfinite(rtol), BEAT_B200_INVALID_ARG, "GMRES tolerance must be positive");
    return gmres_t<float, false>(c, R, x_dev, b_dev, restart, max_iters, rtol);
}

IrResult gmres_refine_adjoint(beat_b200_ctx *c, int R, double *x_dev, const double *b_dev, int restart, int max_iters,
                              double rtol) {
    BB_REQUIRE(restart >= 1 && restart <= 200, BEAT_B200_INVALID_ARG, "GMRES restart must be in 1..200");
    BB_REQUIRE(rtol > 0 && std::isfinite(rtol), BEAT_B200_INVALID_ARG, "GMRES tolerance must be positive");
    return gmres_t<float, true>(c, R, x_dev, b_dev, restart, max_iters, rtol);
}

}  // namespace bb
