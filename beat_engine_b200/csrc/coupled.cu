// coupled.cu -- the coupled FEM-BEM path's combined BEM operators and the
// products that turn them into the coupled system's BEM blocks.
//
// Reference: assemble_coupled_burton_miller_cuda and
// build_cuda_combined_bem_blocks (src/BeatEngineCudaCoupledBurtonMiller.jl:
// 496-640), tested by tests/coupled_bem_cuda_tests.jl:4-53:
//     A = 1/2 M_p1p1 - D + alpha H,   C = S + alpha (K' + 1/2 M_p1dp0),
//     alpha = burton_miller_coupling(k) = i / k_signed,
// both with the symmetry images and the orbit row weights (the reference's
// identity matrices already carry the weights, assemble_l2_identity_matrix,
// BeatEngineCore.jl:1208-1211).  These are the direct system's operators at
// eta = i / k: A is the direct A and C = -B, so the same element-pair kernels
// assemble them (cached right-hand-side mode, B kept); this file adds the
// exports in the reference's column-major layouts and the block products
//     interface  = C Q       (Q: F x ncols sparse, CSC)
//     motion     = C D_m     (F x nm dense)
//     prescribed = -C D_p    (F x np dense).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>

#include "internal.cuh"

namespace bb {

// row-major (rows x cols, row stride lds) -> column-major (rows x cols) times
// scale, through a 32 x 32 shared tile
template <typename T>
__global__ void to_colmajor_kernel(const Cx<T> *src, int64_t lds, int rows, int cols, T scale, Cx<T> *dst) {
    __shared__ Cx<T> tile[32][33];
    const int c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
    for (int i = threadIdx.y; i < 32; i += blockDim.y) {
        const int r = r0 + i, cc = c0 + threadIdx.x;
        if (r < rows && cc < cols) {
            const Cx<T> v = src[(int64_t)r * lds + cc];
            tile[i][threadIdx.x] = Cx<T>{scale * v.re, scale * v.im};
        }
    }
    __syncthreads();
    for (int i = threadIdx.y; i < 32; i += blockDim.y) {
        const int cc = c0 + i, r = r0 + threadIdx.x;
        if (r < rows && cc < cols) dst[(int64_t)cc * rows + r] = tile[threadIdx.x][i];
    }
}

// out (n x ncols, column-major) = C Q: thread per (row, column), the column's
// nonzeros read by every row (one owner per entry, no atomics, as the
// reference's _cuda_combined_projection_kernel!).  colptr / rowval are
// 1-based (Julia CSC); an index outside [1, nnz] or a row outside [1, F] sets
// err and is skipped.
template <typename T>
__global__ void csc_projection_kernel(const Cx<T> *C, int n, int F, const int *colptr, const int *rowval,
                                      const Cx<T> *nz, int64_t nnz, int ncols, Cx<T> *out, int *err) {
    const int64_t total = (int64_t)n * ncols;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int row = (int)(i % n), col = (int)(i / n);
        const int64_t p0 = colptr[col], p1 = colptr[col + 1];
        T sr = T(0), si = T(0);
        if (p0 < 1 || p1 < p0 || p1 > nnz + 1) {
            atomicOr(err, 1);
        } else {
            for (int64_t pos = p0; pos < p1; ++pos) {
                const int f = rowval[pos - 1];
                if (f < 1 || f > F) {
                    atomicOr(err, 1);
                    continue;
                }
                const Cx<T> a = C[(int64_t)(f - 1) * n + row], b = nz[pos - 1];
                sr += a.re * b.re - a.im * b.im;
                si += a.re * b.im + a.im * b.re;
            }
        }
        out[i] = Cx<T>{sr, si};
    }
}

// out (n x m, column-major) = scale C D, C n x F and D F x m column-major:
// one thread per row, CP_COLS columns of D per pass staged through shared
// memory, C read once per pass (coalesced down the rows)
constexpr int CP_COLS = 8, CP_KCHUNK = 64, CP_THREADS = 256;

template <typename T>
__global__ void __launch_bounds__(CP_THREADS) dense_product_kernel(const Cx<T> *C, int n, int F, const Cx<T> *D,
                                                                    int m, int j0, T scale, Cx<T> *out) {
    __shared__ Cx<T> sd[CP_KCHUNK][CP_COLS];
    const int row = blockIdx.x * CP_THREADS + threadIdx.x;
    const int jc = min(CP_COLS, m - j0);
    T ar[CP_COLS], ai[CP_COLS];
#pragma unroll
    for (int j = 0; j < CP_COLS; ++j) ar[j] = ai[j] = T(0);
    for (int f0 = 0; f0 < F; f0 += CP_KCHUNK) {
        const int fc = min(CP_KCHUNK, F - f0);
        __syncthreads();
        for (int i = threadIdx.x; i < CP_KCHUNK * CP_COLS; i += CP_THREADS) {
            const int f = i / CP_COLS, j = i % CP_COLS;
            sd[f][j] = (f < fc && j < jc) ? D[(int64_t)(j0 + j) * F + f0 + f] : Cx<T>{T(0), T(0)};
        }
        __syncthreads();
        if (row >= n) continue;
        for (int f = 0; f < fc; ++f) {
            const Cx<T> a = C[(int64_t)(f0 + f) * n + row];
#pragma unroll
            for (int j = 0; j < CP_COLS; ++j) {
                const Cx<T> b = sd[f][j];
                ar[j] += a.re * b.re - a.im * b.im;
                ai[j] += a.re * b.im + a.im * b.re;
            }
        }
    }
    if (row < n)
        for (int j = 0; j < jc; ++j) out[(int64_t)(j0 + j) * n + row] = Cx<T>{scale * ar[j], scale * ai[j]};
}

template <typename T>
static void export_coupled(beat_b200_ctx *c, void *d_A, void *d_C) {
    Workspace &w = c->ws;
    const int n = c->V, F = c->F;
    dim3 block(32, 8);
    if (d_A) {
        to_colmajor_kernel<T><<<dim3((n + 31) / 32, (n + 31) / 32), block, 0, c->stream>>>(
            w.A.as<Cx<T>>(), w.ld, n, n, T(1), static_cast<Cx<T> *>(d_A));
        BB_CUDA(cudaGetLastError());
    }
    if (d_C) {  // C = -B
        to_colmajor_kernel<T><<<dim3((F + 31) / 32, (n + 31) / 32), block, 0, c->stream>>>(
            w.B.as<Cx<T>>(), F, n, F, T(-1), static_cast<Cx<T> *>(d_C));
        BB_CUDA(cudaGetLastError());
    }
}

void assemble_coupled(beat_b200_ctx *c, double k, int precision, void *d_A, void *d_C) {
    BB_REQUIRE(c->F > 0, BEAT_B200_STATE, "no mesh: call beat_b200_set_mesh first");
    BB_REQUIRE(std::isfinite(k) && k != 0.0, BEAT_B200_INVALID_ARG, "coupled assembly: wavenumber must be finite "
                                                                     "and nonzero");
    BB_REQUIRE(precision == BEAT_B200_FP64 || precision == BEAT_B200_MIXED_FP32_IR, BEAT_B200_INVALID_ARG,
               "unknown precision form");
    ensure_workspace(c, precision, 1, BEAT_B200_RHS_CACHED);
    BB_REQUIRE(c->ws.rhs_cached, BEAT_B200_OOM, "coupled assembly: the N x F operator C does not fit in memory");
    Workspace &w = c->ws;
    BB_CUDA(cudaMemsetAsync(w.q.p, 0, (size_t)c->F * 16, c->stream));
    assemble(c, k, 1.0 / k, precision, 1, w.q.p, nullptr, nullptr);  // alpha = i / k
    w.lu_valid = 0;
    if (precision == BEAT_B200_FP64)
        export_coupled<double>(c, d_A, d_C);
    else
        export_coupled<float>(c, d_A, d_C);
    BB_CUDA(cudaStreamSynchronize(c->stream));
}

template <typename T>
static void blocks_t(beat_b200_ctx *c, const void *d_C, int ncols, const int *colptr, const int *rowval,
                     const void *nzval, int64_t nnz, void *d_interface, int nm, const void *d_motion,
                     void *d_motion_out, int np, const void *d_prescribed, void *d_prescribed_out) {
    const int n = c->V, F = c->F;
    const Cx<T> *C = static_cast<const Cx<T> *>(d_C);
    int err = 0;
    if (ncols > 0) {
        c->ws.grad.alloc(std::max<size_t>(c->ws.grad.bytes, 16));  // error word (grow-only scratch)
        int *d_err = c->ws.grad.as<int>();
        BB_CUDA(cudaMemsetAsync(d_err, 0, sizeof(int), c->stream));
        const int64_t total = (int64_t)n * ncols;
        const int blocks = (int)std::min<int64_t>((total + 255) / 256, 16LL * c->sm_count);
        csc_projection_kernel<T><<<blocks, 256, 0, c->stream>>>(C, n, F, colptr, rowval,
                                                                 static_cast<const Cx<T> *>(nzval), nnz, ncols,
                                                                 static_cast<Cx<T> *>(d_interface), d_err);
        BB_CUDA(cudaGetLastError());
        BB_CUDA(cudaMemcpyAsync(&err, d_err, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    }
    const int rb = (n + CP_THREADS - 1) / CP_THREADS;
    for (int j0 = 0; j0 < nm; j0 += CP_COLS) {
        dense_product_kernel<T><<<rb, CP_THREADS, 0, c->stream>>>(C, n, F, static_cast<const Cx<T> *>(d_motion), nm,
                                                                 j0, T(1), static_cast<Cx<T> *>(d_motion_out));
        BB_CUDA(cudaGetLastError());
    }
    for (int j0 = 0; j0 < np; j0 += CP_COLS) {
        dense_product_kernel<T><<<rb, CP_THREADS, 0, c->stream>>>(C, n, F, static_cast<const Cx<T> *>(d_prescribed),
                                                                 np, j0, T(-1),
                                                                 static_cast<Cx<T> *>(d_prescribed_out));
        BB_CUDA(cudaGetLastError());
    }
    BB_CUDA(cudaStreamSynchronize(c->stream));
    BB_REQUIRE(!err, BEAT_B200_INVALID_ARG,
               "coupled blocks: a CSC column pointer or row index is outside the matrix (1-based, rows 1..F)");
}

void coupled_blocks(beat_b200_ctx *c, int precision, const void *d_C, int ncols, const int *colptr,
                    const int *rowval, const void *nzval, int64_t nnz, void *d_interface, int nm,
                    const void *d_motion, void *d_motion_out, int np, const void *d_prescribed,
                    void *d_prescribed_out) {
    BB_REQUIRE(c->F > 0, BEAT_B200_STATE, "no mesh: call beat_b200_set_mesh first");
    BB_REQUIRE(precision == BEAT_B200_FP64 || precision == BEAT_B200_MIXED_FP32_IR, BEAT_B200_INVALID_ARG,
               "unknown precision form");
    BB_REQUIRE(d_C && ncols >= 0 && nm >= 0 && np >= 0 && nnz >= 0, BEAT_B200_INVALID_ARG,
               "coupled blocks: bad arguments");
    BB_REQUIRE(ncols == 0 || (colptr && rowval && (nzval || nnz == 0) && d_interface), BEAT_B200_INVALID_ARG,
               "coupled blocks: null sparse-map pointer");
    BB_REQUIRE(nm == 0 || (d_motion && d_motion_out), BEAT_B200_INVALID_ARG, "coupled blocks: null motion pointer");
    BB_REQUIRE(np == 0 || (d_prescribed && d_prescribed_out), BEAT_B200_INVALID_ARG,
               "coupled blocks: null prescribed pointer");
    if (precision == BEAT_B200_FP64)
        blocks_t<double>(c, d_C, ncols, colptr, rowval, nzval, nnz, d_interface, nm, d_motion, d_motion_out, np,
                         d_prescribed, d_prescribed_out);
    else
        blocks_t<float>(c, d_C, ncols, colptr, rowval, nzval, nnz, d_interface, nm, d_motion, d_motion_out, np,
                        d_prescribed, d_prescribed_out);
}

}  // namespace bb
