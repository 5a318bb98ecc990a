// lu.cu -- blocked right-looking complex LU with partial pivoting, and the
// multi-right-hand-side triangular solves, on one B200.
//
// Replaces the reference's lu!(system.matrix) / factorization \ rhs
// (BeatEngineCompiledDriver.jl:902-903 -> cuSOLVER getrf/getrs through
// CUDA.jl, and OpenBLAS zgetrf on the CPU path, BeatEngineDenseSolve.jl:1104-1110).
// Pivoting is the partial pivoting LAPACK uses (first maximum of |re| + |im|
// in the column), so the factorisation is P A = L U with unit-lower L.
//
// Layout: A is row-major complex, row stride ld (complex entries).  Row
// interchanges are then contiguous copies.
//
// Per panel of nb columns:
//   1. panel_kernel: a cooperative kernel; the panel rows are split over the
//      CTAs and held in shared memory.  Per column every CTA publishes its
//      best candidate row and record, passes one grid-wide barrier (an
//      arrival counter), reads all records at once, picks the same winner,
//      swaps and eliminates locally.  Slots are double-buffered by column
//      parity so one barrier per column suffices.
//   2. laswp_kernel: the panel's interchanges on all other columns (and on
//      the running row permutation).
//   3. trsm_kernel: U12 = L11^-1 A12.
//   4. trailing update A22 -= L21 U12: SIMT complex GEMM here (FP64 form),
//      tcgen05 FP16-split tensor-core GEMM for the FP32 form (tc_gemm.cu).
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>

#include "internal.cuh"

namespace bb {

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned *p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

template <typename T> __device__ __forceinline__ T cabs1(Cx<T> v) { return fabs(v.re) + fabs(v.im); }
// correctly rounded reciprocal (the same value as 1 / x)
__device__ __forceinline__ float rcp_rn(float x) { return __frcp_rn(x); }
__device__ __forceinline__ double rcp_rn(double x) { return __drcp_rn(x); }
template <typename T> __device__ __forceinline__ Cx<T> cms(Cx<T> x, Cx<T> l, Cx<T> u) {  // x - l u
    return Cx<T>{x.re - (l.re * u.re - l.im * u.im), x.im - (l.re * u.im + l.im * u.re)};
}

// L2-coherent loads of values other CTAs published before a grid barrier
__device__ __forceinline__ Cx<double> ldcg(const Cx<double> *p) {
    const double2 v = __ldcg(reinterpret_cast<const double2 *>(p));
    return Cx<double>{v.x, v.y};
}
__device__ __forceinline__ Cx<float> ldcg(const Cx<float> *p) {
    const float2 v = __ldcg(reinterpret_cast<const float2 *>(p));
    return Cx<float>{v.x, v.y};
}
__device__ __forceinline__ double ldcg(const double *p) { return __ldcg(p); }
__device__ __forceinline__ float ldcg(const float *p) { return __ldcg(p); }
__device__ __forceinline__ int ldcg(const int *p) { return __ldcg(p); }

// Pivot candidate of one CTA for one column (value |re| + |im| and global row).
struct PivotRec {
    double val;
    int idx;
    int pad;
};

template <typename T> struct PanelArgs {
    Cx<T> *A;
    int64_t ld;
    int n, k, nb;
    int rpc;            // rows per CTA
    int *ipiv;
    Cx<T> *pub_rows;    // [2][G][nb]
    Cx<T> *pub_diag;    // [2][nb]
    PivotRec *recs;     // [2][G]
    unsigned *counter;  // grid-barrier arrivals of this panel launch (zeroed before it)
    int *status;
    unsigned spin_limit;
};

constexpr int PANEL_THREADS = 256;

template <typename T> __global__ void __launch_bounds__(PANEL_THREADS) panel_kernel(PanelArgs<T> a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int nb = a.nb, G = gridDim.x, cta = blockIdx.x, tid = threadIdx.x;
    Cx<T> *P = reinterpret_cast<Cx<T> *>(smem_raw);  // rpc x nb
    Cx<T> *prow = P + (size_t)a.rpc * nb;             // nb
    Cx<T> *drow = prow + nb;                          // nb
    Cx<T> *lcol = drow + nb;                          // rpc
    __shared__ T red_v[PANEL_THREADS / 32];
    __shared__ int red_i[PANEL_THREADS / 32];
    __shared__ int red_c[PANEL_THREADS / 32];
    __shared__ int s_piv;
    __shared__ T s_pv;

    const int gr0 = a.k + cta * a.rpc;
    const int nrows = max(0, min(a.rpc, a.n - gr0));
    batched_copy<PANEL_THREADS, 8, Cx<T>>(
        nrows * nb, [&](int i) { return a.A[(int64_t)(gr0 + i / nb) * a.ld + a.k + i % nb]; },
        [&](int i, Cx<T> v) { P[i] = v; });
    __syncthreads();

    for (int j = 0; j < nb && a.k + j < a.n; ++j) {
        const int jr = a.k + j, par = j & 1;
        // local candidate: first maximum of |re|+|im| among own rows >= jr
        T bv = T(-1);
        int bi = -1;
        for (int i = tid; i < nrows; i += PANEL_THREADS) {
            if (gr0 + i < jr) continue;
            const T v = cabs1(P[i * nb + j]);
            if (v > bv) {
                bv = v;
                bi = gr0 + i;
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const T ov = __shfl_xor_sync(0xffffffffu, bv, o);
            const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
            if (ov > bv || (ov == bv && oi >= 0 && (bi < 0 || oi < bi))) {
                bv = ov;
                bi = oi;
            }
        }
        if ((tid & 31) == 0) {
            red_v[tid >> 5] = bv;
            red_i[tid >> 5] = bi;
        }
        __syncthreads();
        if (tid == 0) {
            for (int w = 1; w < PANEL_THREADS / 32; ++w)
                if (red_v[w] > bv || (red_v[w] == bv && red_i[w] >= 0 && (bi < 0 || red_i[w] < bi))) {
                    bv = red_v[w];
                    bi = red_i[w];
                }
            s_piv = bi;
            s_pv = bv;
        }
        __syncthreads();
        const int mine = s_piv;
        if (mine >= 0)
            for (int c = tid; c < nb; c += PANEL_THREADS)
                a.pub_rows[((size_t)par * G + cta) * nb + c] = P[(mine - gr0) * nb + c];
        if (jr >= gr0 && jr < gr0 + nrows)
            for (int c = tid; c < nb; c += PANEL_THREADS) a.pub_diag[(size_t)par * nb + c] = P[(jr - gr0) * nb + c];
        __syncthreads();
        // candidate record, then one grid-wide barrier: each CTA adds one
        // arrival (release) and waits until all G arrivals of this column are in
        if (tid == 0) {
            PivotRec *rec = &a.recs[par * G + cta];
            rec->val = (double)s_pv;
            rec->idx = mine;
            __threadfence();
            asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(a.counter), "r"(1u) : "memory");
            const unsigned target = (unsigned)(j + 1) * (unsigned)G;
            unsigned it = 0;
            while (true) {
                unsigned v;
                asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(a.counter) : "memory");
                if (v >= target) break;
                if ((*(volatile int *)a.status & DEV_BARRIER_TIMEOUT) || ++it > a.spin_limit) {
                    atomicOr(a.status, (int)DEV_BARRIER_TIMEOUT);
                    break;
                }
            }
        }
        __syncthreads();
        // every CTA reads all G records at once and picks the same winner
        {
            T wv = T(-1);
            int wi = -1, wc = -1;
            if (tid < G) {
                const PivotRec *rec = &a.recs[par * G + tid];
                wi = __ldcg(&rec->idx);
                wv = wi >= 0 ? (T)__ldcg(&rec->val) : T(-1);
                wc = tid;
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                const T ov = __shfl_xor_sync(0xffffffffu, wv, o);
                const int oi = __shfl_xor_sync(0xffffffffu, wi, o);
                const int oc = __shfl_xor_sync(0xffffffffu, wc, o);
                if (oi >= 0 && (ov > wv || (ov == wv && (wi < 0 || oi < wi)))) {
                    wv = ov;
                    wi = oi;
                    wc = oc;
                }
            }
            if ((tid & 31) == 0) {
                red_v[tid >> 5] = wv;
                red_i[tid >> 5] = wi;
                red_c[tid >> 5] = wc;
            }
            __syncthreads();
            if (tid == 0) {
                for (int w = 1; w < PANEL_THREADS / 32; ++w)
                    if (red_i[w] >= 0 && (red_v[w] > wv || (red_v[w] == wv && (wi < 0 || red_i[w] < wi)))) {
                        wv = red_v[w];
                        wi = red_i[w];
                        wc = red_c[w];
                    }
                s_piv = wi < 0 ? jr : wi;
                s_pv = wv;
                red_i[0] = wc;
                if (wv <= T(0)) atomicOr(a.status, (int)DEV_ZERO_PIVOT);
                if (cta == 0) a.ipiv[jr] = s_piv;
            }
        }
        __syncthreads();
        const int p = s_piv, wc = red_i[0];
        for (int c = tid; c < nb; c += PANEL_THREADS) {
            prow[c] = wc >= 0 ? ldcg(&a.pub_rows[((size_t)par * G + wc) * nb + c]) : Cx<T>{T(0), T(0)};
            drow[c] = ldcg(&a.pub_diag[(size_t)par * nb + c]);
        }
        __syncthreads();
        if (p != jr) {
            if (jr >= gr0 && jr < gr0 + nrows)
                for (int c = tid; c < nb; c += PANEL_THREADS) P[(jr - gr0) * nb + c] = prow[c];
            if (p >= gr0 && p < gr0 + nrows)
                for (int c = tid; c < nb; c += PANEL_THREADS) P[(p - gr0) * nb + c] = drow[c];
        }
        __syncthreads();
        // eliminate below the pivot
        const Cx<T> pv = prow[j];
        const T den = pv.re * pv.re + pv.im * pv.im;
        const Cx<T> inv = den > T(0) ? Cx<T>{pv.re / den, -pv.im / den} : Cx<T>{T(0), T(0)};
        const int first = max(0, jr + 1 - gr0);
        for (int i = first + tid; i < nrows; i += PANEL_THREADS) lcol[i] = cmul(P[i * nb + j], inv);
        __syncthreads();
        const int w = nb - j - 1;
        if (w > 0) {
            for (int idx = tid; idx < (nrows - first) * w; idx += PANEL_THREADS) {
                const int i = first + idx / w, c = j + 1 + idx % w;
                const Cx<T> l = lcol[i], u = prow[c];
                Cx<T> &d = P[i * nb + c];
                d.re -= l.re * u.re - l.im * u.im;
                d.im -= l.re * u.im + l.im * u.re;
            }
        }
        for (int i = first + tid; i < nrows; i += PANEL_THREADS) P[i * nb + j] = lcol[i];
        __syncthreads();
    }
    for (int i = tid; i < nrows * nb; i += PANEL_THREADS) {
        const int r = i / nb, c = i % nb;
        a.A[(int64_t)(gr0 + r) * a.ld + a.k + c] = P[i];
    }
}

// row interchanges of one panel on all columns outside it; the extra
// "column" -1 applies them to the running permutation perm[]
template <typename T>
__global__ void laswp_kernel(Cx<T> *A, int64_t ld, int n, int k, int nb, const int *ipiv, int *perm) {
    __shared__ int sp[256];
    for (int j = threadIdx.x; j < nb; j += blockDim.x) sp[j] = ipiv[k + j];
    __syncthreads();
    const int c = (int)(blockIdx.x * blockDim.x + threadIdx.x) - 1;
    const int jmax = min(nb, n - k);
    if (c == -1) {
        for (int j = 0; j < jmax; ++j) {
            const int p = sp[j];
            if (p > k + j && p < n) {
                const int t = perm[k + j];
                perm[k + j] = perm[p];
                perm[p] = t;
            }
        }
        return;
    }
    if (c >= n || (c >= k && c < k + nb)) return;
    for (int j = 0; j < jmax; ++j) {
        const int p = sp[j];
        if (p > k + j && p < n) {  // an interchange always names a later row
            const Cx<T> t = A[(int64_t)(k + j) * ld + c];
            A[(int64_t)(k + j) * ld + c] = A[(int64_t)p * ld + c];
            A[(int64_t)p * ld + c] = t;
        }
    }
}

// Row interchanges ipiv[k .. k+nsw) on the columns [c_lo, c_hi) outside
// [x_lo, x_hi); with perm non-null, one extra thread applies them to the
// running permutation.  (The look-ahead LU swaps a sub-panel's rows inside its
// panel first and on the other columns once per panel.)
template <typename T>
__global__ void laswp_range_kernel(Cx<T> *A, int64_t ld, int n, int k, int nsw, const int *ipiv, int c_lo, int c_hi,
                                   int x_lo, int x_hi, int *perm) {
    __shared__ int sp[256];
    for (int j = threadIdx.x; j < nsw; j += blockDim.x) sp[j] = ipiv[k + j];
    __syncthreads();
    const int jmax = min(nsw, n - k);
    const int c = c_lo - 1 + (int)(blockIdx.x * blockDim.x + threadIdx.x);
    if (c == c_lo - 1) {
        if (!perm) return;
        for (int j = 0; j < jmax; ++j) {
            const int p = sp[j];
            if (p > k + j && p < n) {
                const int t = perm[k + j];
                perm[k + j] = perm[p];
                perm[p] = t;
            }
        }
        return;
    }
    if (c >= c_hi || (c >= x_lo && c < x_hi)) return;
    for (int j = 0; j < jmax; ++j) {
        const int p = sp[j];
        if (p > k + j && p < n) {  // an interchange always names a later row
            const Cx<T> t = A[(int64_t)(k + j) * ld + c];
            A[(int64_t)(k + j) * ld + c] = A[(int64_t)p * ld + c];
            A[(int64_t)p * ld + c] = t;
        }
    }
}

// The same interchanges as laswp_range_kernel (nsw <= LS_MAX), as one
// permutation of at most 2 nsw rows: every CTA derives the moves from ipiv,
// then loads every moved entry of its LS_COLS columns before it stores any, so
// no column walks a chain of dependent global loads.  With swap j exchanging
// positions k + j and p_j >= k + j, position k + j is final after swap j; its
// content then is what stood at p_j just before, and
//   X_j (the content of k + j just before swap j) = X_prevX[j], or the row k + j
//       itself when no earlier swap's far end was k + j;
//   V_j (the content of p_j just before swap j) = X_j when p_j = k + j, else
//       X_lastP[j] for the last earlier swap with the same far end, else p_j.
// Final contents: k + j <- V_j; a far end q >= k + nsw <- X_j of the last swap
// that names it.  X is a root search over prevX (pointer jumping).
constexpr int LS_MAX = 256;
template <typename T> __host__ __device__ constexpr int ls_cols() { return sizeof(T) == 4 ? 32 : 16; }
template <typename T> static size_t laswp_panel_smem(int nsw) {
    return sizeof(Cx<T>) * 2 * (size_t)nsw * ls_cols<T>();
}
template <typename T>
__global__ void __launch_bounds__(256) laswp_panel_kernel(Cx<T> *A, int64_t ld, int n, int k, int nsw, const int *ipiv,
                                                          int c_lo, int c_hi, int x_lo, int x_hi, int *perm) {
    constexpr int LC = ls_cols<T>();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Cx<T> *vals = reinterpret_cast<Cx<T> *>(smem_raw);  // [moves][LC]
    __shared__ int sp[LS_MAX], root[2][LS_MAX], xs[LS_MAX], msrc[2 * LS_MAX], mdst[2 * LS_MAX], pv[2 * LS_MAX];
    __shared__ int nmove;
    const int tid = threadIdx.x;
    const int jmax = min(min(nsw, n - k), LS_MAX);
    if (tid == 0) nmove = 0;
    for (int j = tid; j < jmax; j += 256) {
        const int p = ipiv[k + j];
        sp[j] = (p > k + j && p < n) ? p : k + j;  // out-of-range entries are no interchange, as in laswp_range_kernel
    }
    __syncthreads();
    int prev_x = -1, last_p = -1;
    bool has_next = false;
    const int j = tid;
    if (j < jmax) {
        const int pj = sp[j];
        for (int i = 0; i < jmax; ++i) {
            const int pi = sp[i];
            if (i < j) {
                if (pi == k + j) prev_x = i;
                if (pi == pj && pj != k + j) last_p = i;
            } else if (i > j && pi == pj) {
                has_next = true;
            }
        }
        root[0][j] = prev_x < 0 ? j : prev_x;
    }
    __syncthreads();
    int b = 0;
    for (int step = 1; step < LS_MAX; step *= 2) {  // log2(LS_MAX) rounds
        if (j < jmax) root[b ^ 1][j] = root[b][root[b][j]];
        b ^= 1;
        __syncthreads();
    }
    if (j < jmax) xs[j] = k + root[b][j];
    __syncthreads();
    if (j < jmax) {
        const int pj = sp[j], xj = xs[j];
        const int vj = pj == k + j ? xj : (last_p >= 0 ? xs[last_p] : pj);
        if (vj != k + j) {
            const int m = atomicAdd(&nmove, 1);
            msrc[m] = vj;
            mdst[m] = k + j;
        }
        if (pj >= k + jmax && !has_next) {
            const int m = atomicAdd(&nmove, 1);
            msrc[m] = xj;
            mdst[m] = pj;
        }
    }
    __syncthreads();
    const int nm = nmove;
    const int cbase = c_lo + (int)blockIdx.x * LC;
    for (int i = tid; i < nm * LC; i += 256) {
        const int c = cbase + i % LC;
        if (c < c_hi && (c < x_lo || c >= x_hi)) vals[i] = A[(int64_t)msrc[i / LC] * ld + c];
    }
    if (perm && blockIdx.x == 0)
        for (int m = tid; m < nm; m += 256) pv[m] = perm[msrc[m]];
    __syncthreads();
    for (int i = tid; i < nm * LC; i += 256) {
        const int c = cbase + i % LC;
        if (c < c_hi && (c < x_lo || c >= x_hi)) A[(int64_t)mdst[i / LC] * ld + c] = vals[i];
    }
    if (perm && blockIdx.x == 0)
        for (int m = tid; m < nm; m += 256) perm[mdst[m]] = pv[m];
}

__global__ void iota_kernel(int *perm, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) perm[i] = i;
}

// A[k:k+kb, c_begin:c_end] = L^-1 A[...] with L = A[k:k+kb, k:k+kb] unit
// lower (nb = allocated width of the triangle); 32 columns per CTA
constexpr int TRSM_COLS = 32;
template <typename T>
__global__ void __launch_bounds__(256) trsm_kernel(Cx<T> *A, int64_t ld, int n, int k, int nb, int c_begin, int c_end) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Cx<T> *L = reinterpret_cast<Cx<T> *>(smem_raw);  // nb x nb
    Cx<T> *X = L + nb * nb;                           // nb x TRSM_COLS
    const int c0 = c_begin + blockIdx.x * TRSM_COLS;
    const int nc = min(TRSM_COLS, c_end - c0);
    const int kb = min(nb, n - k);
    batched_copy<256, 16, Cx<T>>(
        kb * kb, [&](int i) { return A[(int64_t)(k + i / kb) * ld + k + i % kb]; },
        [&](int i, Cx<T> v) { L[(i / kb) * nb + i % kb] = v; });
    batched_copy<256, 8, Cx<T>>(
        kb * TRSM_COLS,
        [&](int i) {
            const int c = i % TRSM_COLS;
            return c < nc ? A[(int64_t)(k + i / TRSM_COLS) * ld + c0 + c] : Cx<T>{T(0), T(0)};
        },
        [&](int i, Cx<T> v) { X[i] = v; });
    __syncthreads();
    for (int j = 0; j < kb - 1; ++j) {
        for (int idx = threadIdx.x; idx < (kb - 1 - j) * TRSM_COLS; idx += blockDim.x) {
            const int i = j + 1 + idx / TRSM_COLS, c = idx % TRSM_COLS;
            const Cx<T> l = L[i * nb + j], x = X[j * TRSM_COLS + c];
            Cx<T> &d = X[i * TRSM_COLS + c];
            d.re -= l.re * x.re - l.im * x.im;
            d.im -= l.re * x.im + l.im * x.re;
        }
        __syncthreads();
    }
    for (int i = threadIdx.x; i < kb * TRSM_COLS; i += blockDim.x) {
        const int r = i / TRSM_COLS, c = i % TRSM_COLS;
        if (c < nc) A[(int64_t)(k + r) * ld + c0 + c] = X[r * TRSM_COLS + c];
    }
}

// Inverse of a unit lower triangular kb x kb block (kb <= W <= 32), by one
// warp: lane c forward-substitutes column c of the inverse with four partial
// sums per row.  L holds the strictly lower part (row stride ldl), Y is W x
// (W + 1) scratch, D receives the W x W inverse row-major (identity past kb).
template <typename T>
__device__ __forceinline__ void warp_unit_lower_inverse(const Cx<T> *L, int ldl, int kb, int W, Cx<T> *Y, Cx<T> *D) {
    const int c = threadIdx.x & 31, ldy = W + 1;
    if (c < W) {
        for (int i = 0; i < W; ++i) {
            Cx<T> s0{T(i == c), T(0)}, s1{T(0), T(0)}, s2{T(0), T(0)}, s3{T(0), T(0)};
            if (i > c && i < kb) {
                int t = c;
                for (; t + 4 <= i; t += 4) {
                    s0 = cms(s0, L[i * ldl + t], Y[t * ldy + c]);
                    s1 = cms(s1, L[i * ldl + t + 1], Y[(t + 1) * ldy + c]);
                    s2 = cms(s2, L[i * ldl + t + 2], Y[(t + 2) * ldy + c]);
                    s3 = cms(s3, L[i * ldl + t + 3], Y[(t + 3) * ldy + c]);
                }
                for (; t < i; ++t) s0 = cms(s0, L[i * ldl + t], Y[t * ldy + c]);
            }
            Y[i * ldy + c] = Cx<T>{(s0.re + s1.re) + (s2.re + s3.re), (s0.im + s1.im) + (s2.im + s3.im)};
        }
        for (int i = 0; i < W; ++i) D[(size_t)i * W + c] = Y[i * ldy + c];
    }
}

// The same for the diagonal block A[k:k+kb, k:k+kb] (kb = min(W, n - k)) of
// a sub-panel factored by the grid-wide panel kernel.
template <typename T>
__global__ void __launch_bounds__(32) diag_block_inverse_kernel(const Cx<T> *A, int64_t ld, int n, int k, int W, Cx<T> *D) {
    __shared__ Cx<T> L[32 * 33];
    __shared__ Cx<T> Y[32 * 33];
    const int kb = min(W, n - k);
    batched_copy<32, 32, Cx<T>>(
        kb * kb, [&](int i) { return A[(int64_t)(k + i / kb) * ld + k + i % kb]; },
        [&](int i, Cx<T> v) { L[(i / kb) * 33 + i % kb] = v; });
    __syncwarp();
    warp_unit_lower_inverse(L, 33, kb, W, Y, D);
}

// Blocked U12 = L11^-1 A12 for L11 = A[k:k+kb, k:k+kb] (kb = S W) with the
// inverses D_s of its W x W diagonal blocks:  X_s = D_s (A_s - sum_{t<s}
// L_st X_t), s = 0..S-1.  32 columns per CTA, 256 threads, each thread W/8
// complex outputs of a W x 32 block per product; one barrier per block step
// instead of one per row.
constexpr int TB_COLS = 32;
// With bhi non-null (FP32, the tensor-core path) the solved block is also
// written in the trailing update's B-operand layout (the staging of
// tc_gemm.cu: rows 2j and 2j + 1 of B_s hold (Ur, -Ui) 2^s and (Ui, Ur) 2^s at
// K = 2kk for column j = c - j0 and row kk of the block, s from the column's
// largest |re| or |im|, as FP16 high parts and, when split == 3, FP16
// remainders; bscale[j] = 2^-(s + L_SHIFT)), so no separate staging pass
// rereads U12.  stage_u_block does it for a block of COLS columns in shared
// memory (X[row * COLS + column]); all 256 threads of the CTA call it.
template <int COLS>
__device__ void stage_u_block(const Cx<float> *X, int kb, int nc, int c0, int j0, __half *bhi, __half *blo,
                              float *bscale, int split) {
    __shared__ unsigned cmax[COLS];  // largest |re| or |im| of each column, as ordered bits
    const int tid = threadIdx.x;
    if (tid < COLS) cmax[tid] = 0u;
    __syncthreads();
    {
        const int c = tid % COLS;
        float mx = 0.f;
        for (int r = tid / COLS; r < kb; r += 256 / COLS) {
            const Cx<float> u = X[r * COLS + c];
            mx = fmaxf(mx, fmaxf(fabsf(u.re), fabsf(u.im)));
        }
        atomicMax(&cmax[c], __float_as_uint(mx));
    }
    __syncthreads();
    if (tid < nc) bscale[c0 + tid - j0] = pow2f(-stage_exp(__uint_as_float(cmax[tid])) - L_SHIFT);
    // consecutive threads: consecutive K (rows kk of the block) of one B_s row
    for (int i = tid; i < 2 * COLS * kb; i += 256) {
        const int row = i / kb, kk = i % kb, c = row >> 1;
        if (c >= nc) continue;
        const float sc = pow2f(stage_exp(__uint_as_float(cmax[c])));
        const Cx<float> u = X[kk * COLS + c];
        const float vx = ((row & 1) ? u.im : u.re) * sc, vy = ((row & 1) ? u.re : -u.im) * sc;
        const int64_t at = (int64_t)(2 * (c0 + c - j0) + (row & 1)) * 2 * kb + 2 * kk;
        __half hx, hy, lx, ly;
        split_f16(vx, hx, lx);
        split_f16(vy, hy, ly);
        *reinterpret_cast<__half2 *>(bhi + at) = __halves2half2(hx, hy);
        if (split == 3) *reinterpret_cast<__half2 *>(blo + at) = __halves2half2(lx, ly);
    }
}
template <typename T, int W>
__global__ void __launch_bounds__(256) trsm_blocked_kernel(Cx<T> *A, int64_t ld, int k, int S, const Cx<T> *D,
                                                            int c_begin, int c_end, __half *bhi = nullptr,
                                                            __half *blo = nullptr, float *bscale = nullptr,
                                                            int j0 = 0, int split = 3) {
    constexpr int OPT = W * TB_COLS / 256;  // outputs per thread: 4 (W = 32) or 2 (W = 16)
    constexpr int CG = TB_COLS / OPT;       // column groups
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int kb = S * W;
    Cx<T> *X = reinterpret_cast<Cx<T> *>(smem_raw);  // kb x TB_COLS
    Cx<T> *Dt = X + (size_t)kb * TB_COLS;             // W x (W + 1)
    Cx<T> *Lt = Dt + W * (W + 1);                     // W x (r0 + 1), r0 <= kb - W
    const int tid = threadIdx.x, r = tid / CG, cg = tid % CG;
    const int c0 = c_begin + blockIdx.x * TB_COLS;
    const int nc = min(TB_COLS, c_end - c0);
    batched_copy<256, 8, Cx<T>>(
        kb * TB_COLS,
        [&](int i) {
            const int c = i % TB_COLS;
            return c < nc ? A[(int64_t)(k + i / TB_COLS) * ld + c0 + c] : Cx<T>{T(0), T(0)};
        },
        [&](int i, Cx<T> v) { X[i] = v; });
    for (int s = 0; s < S; ++s) {
        const int r0 = s * W;
        batched_copy<256, 4, Cx<T>>(
            W * W, [&](int i) { return D[(size_t)s * W * W + i]; },
            [&](int i, Cx<T> v) { Dt[(i / W) * (W + 1) + i % W] = v; });
        if (s > 0)
            batched_copy<256, 8, Cx<T>>(
                W * r0, [&](int i) { return A[(int64_t)(k + r0 + i / r0) * ld + k + i % r0]; },
                [&](int i, Cx<T> v) { Lt[(i / r0) * (r0 + 1) + i % r0] = v; });
        __syncthreads();
        Cx<T> acc[OPT];
#pragma unroll
        for (int o = 0; o < OPT; ++o) acc[o] = X[(r0 + r) * TB_COLS + cg * OPT + o];
        for (int t = 0; t < r0; ++t) {  // A_s - L_s,<s X_<s
            const Cx<T> l = Lt[r * (r0 + 1) + t];
#pragma unroll
            for (int o = 0; o < OPT; ++o) {
                const Cx<T> x = X[t * TB_COLS + cg * OPT + o];
                acc[o].re -= l.re * x.re - l.im * x.im;
                acc[o].im -= l.re * x.im + l.im * x.re;
            }
        }
        __syncthreads();  // every thread has read block s of X
#pragma unroll
        for (int o = 0; o < OPT; ++o) X[(r0 + r) * TB_COLS + cg * OPT + o] = acc[o];
        __syncthreads();
        Cx<T> y[OPT];
#pragma unroll
        for (int o = 0; o < OPT; ++o) y[o] = Cx<T>{T(0), T(0)};
        for (int t = 0; t <= r; ++t) {  // D_s is lower triangular
            const Cx<T> d = Dt[r * (W + 1) + t];
#pragma unroll
            for (int o = 0; o < OPT; ++o) {
                const Cx<T> x = X[(r0 + t) * TB_COLS + cg * OPT + o];
                y[o].re += d.re * x.re - d.im * x.im;
                y[o].im += d.re * x.im + d.im * x.re;
            }
        }
        __syncthreads();
#pragma unroll
        for (int o = 0; o < OPT; ++o) X[(r0 + r) * TB_COLS + cg * OPT + o] = y[o];
        // the next block step's loads of Dt / Lt follow the next barrier
        __syncthreads();
    }
    for (int i = tid; i < kb * TB_COLS; i += 256) {
        const int rr = i / TB_COLS, c = i % TB_COLS;
        if (c < nc) A[(int64_t)(k + rr) * ld + c0 + c] = X[rr * TB_COLS + c];
    }
    if constexpr (sizeof(T) == 4) {
        if (bhi) stage_u_block<TB_COLS>(X, kb, nc, c0, j0, bhi, blo, bscale, split);
    }
}

// one complex element, global -> shared, through the asynchronous copy unit
template <typename T> __device__ __forceinline__ void cp_async_cx(Cx<T> *smem, const Cx<T> *gmem) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(smem);
    if constexpr (sizeof(Cx<T>) == 8)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(gmem) : "memory");
    else
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(gmem) : "memory");
}

// The same solve for the launches on the factorisation's critical path (the
// next panel's columns, the rest of a panel after each sub-panel).  256 / W
// columns per CTA, one entry of a W-row block per thread, so that the columns
// spread over 4 times more CTAs; the right-hand sides, every diagonal-block
// inverse and every off-diagonal L block of the triangle are in flight
// together before the first block step, so the S dependent steps wait on no
// global load.  Two partial sums per product.  The same optional B-operand
// staging as trsm_blocked_kernel.
template <int W> __host__ __device__ constexpr int narrow_cols() { return 256 / W; }
template <typename T, int W, int NC = narrow_cols<W>()> static size_t trsm_narrow_smem(int S) {
    return sizeof(Cx<T>) * ((size_t)S * W * NC + (size_t)S * W * (W + 1) +
                            (size_t)W * ((size_t)W * S * (S - 1) / 2 + (S - 1)) + (size_t)W * NC);
}
// NC columns per CTA (a multiple of 256 / W): each thread holds OPT = NC W / 256
// entries of a W-row block, row tid / (256 / W), columns tid % (256 / W) + (256 / W) o.
template <typename T, int W, int NC = narrow_cols<W>()>
__global__ void __launch_bounds__(256) trsm_narrow_kernel(Cx<T> *A, int64_t ld, int k, int S, const Cx<T> *D,
                                                          int c_begin, int c_end, __half *bhi, __half *blo,
                                                          float *bscale, int j0, int split) {
    constexpr int CG = narrow_cols<W>(), OPT = NC / CG;
    static_assert(OPT >= 1 && NC % CG == 0, "NC: a multiple of 256 / W");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int kb = S * W;
    Cx<T> *X = reinterpret_cast<Cx<T> *>(smem_raw);  // kb x NC
    Cx<T> *Ds = X + (size_t)kb * NC;                  // S blocks of W x (W + 1)
    Cx<T> *Ls = Ds + (size_t)S * W * (W + 1);         // block row s >= 1: W x (s W + 1)
    Cx<T> *Z = Ls + (size_t)W * ((size_t)W * S * (S - 1) / 2 + (S - 1));  // W x NC
    const int tid = threadIdx.x, r = tid / CG, cg = tid % CG;
    const int c0 = c_begin + blockIdx.x * NC;
    const int nc = min(NC, c_end - c0);
    for (int i = tid; i < kb * NC; i += 256) {
        const int c = i % NC;
        if (c < nc)
            cp_async_cx(&X[i], &A[(int64_t)(k + i / NC) * ld + c0 + c]);
        else
            X[i] = Cx<T>{T(0), T(0)};
    }
    for (int i = tid; i < S * W * W; i += 256) {
        const int s = i / (W * W), e = i % (W * W);
        cp_async_cx(&Ds[(size_t)s * W * (W + 1) + (e / W) * (W + 1) + e % W], &D[i]);
    }
    for (int s = 1; s < S; ++s) {  // L rows [s W, s W + W) x columns [0, s W)
        const int r0 = s * W;
        Cx<T> *Lb = Ls + (size_t)W * ((size_t)W * s * (s - 1) / 2 + (s - 1));
        for (int i = tid; i < W * r0; i += 256)
            cp_async_cx(&Lb[(i / r0) * (r0 + 1) + i % r0], &A[(int64_t)(k + r0 + i / r0) * ld + k + i % r0]);
    }
    asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
    __syncthreads();
    for (int s = 0; s < S; ++s) {
        const int r0 = s * W;
        Cx<T> a0[OPT], a1[OPT];
#pragma unroll
        for (int o = 0; o < OPT; ++o) {
            a0[o] = X[(r0 + r) * NC + cg + CG * o];
            a1[o] = Cx<T>{T(0), T(0)};
        }
        if (s > 0) {  // A_s - L_s,<s X_<s
            const Cx<T> *Lr = Ls + (size_t)W * ((size_t)W * s * (s - 1) / 2 + (s - 1)) + (size_t)r * (r0 + 1);
            for (int t = 0; t < r0; t += 2) {  // r0 is a multiple of W, so even
                const Cx<T> l0 = Lr[t], l1 = Lr[t + 1];
#pragma unroll
                for (int o = 0; o < OPT; ++o) {
                    a0[o] = cms(a0[o], l0, X[t * NC + cg + CG * o]);
                    a1[o] = cms(a1[o], l1, X[(t + 1) * NC + cg + CG * o]);
                }
            }
        }
#pragma unroll
        for (int o = 0; o < OPT; ++o) Z[r * NC + cg + CG * o] = Cx<T>{a0[o].re + a1[o].re, a0[o].im + a1[o].im};
        __syncthreads();
        const Cx<T> *Dr = Ds + (size_t)s * W * (W + 1) + (size_t)r * (W + 1);
        Cx<T> y0[OPT], y1[OPT];
#pragma unroll
        for (int o = 0; o < OPT; ++o) y0[o] = y1[o] = Cx<T>{T(0), T(0)};
        int t = 0;
        for (; t + 1 <= r; t += 2) {  // D_s is lower triangular
            const Cx<T> d0 = Dr[t], d1 = Dr[t + 1];
#pragma unroll
            for (int o = 0; o < OPT; ++o) {
                const Cx<T> z0 = Z[t * NC + cg + CG * o], z1 = Z[(t + 1) * NC + cg + CG * o];
                y0[o] = Cx<T>{y0[o].re + (d0.re * z0.re - d0.im * z0.im), y0[o].im + (d0.re * z0.im + d0.im * z0.re)};
                y1[o] = Cx<T>{y1[o].re + (d1.re * z1.re - d1.im * z1.im), y1[o].im + (d1.re * z1.im + d1.im * z1.re)};
            }
        }
        if (t == r) {
            const Cx<T> d0 = Dr[t];
#pragma unroll
            for (int o = 0; o < OPT; ++o) {
                const Cx<T> z0 = Z[t * NC + cg + CG * o];
                y0[o] = Cx<T>{y0[o].re + (d0.re * z0.re - d0.im * z0.im), y0[o].im + (d0.re * z0.im + d0.im * z0.re)};
            }
        }
#pragma unroll
        for (int o = 0; o < OPT; ++o)
            X[(r0 + r) * NC + cg + CG * o] = Cx<T>{y0[o].re + y1[o].re, y0[o].im + y1[o].im};
        __syncthreads();  // block s of X is complete; Z is free again
    }
    for (int i = tid; i < kb * NC; i += 256) {
        const int c = i % NC;
        if (c < nc) A[(int64_t)(k + i / NC) * ld + c0 + c] = X[i];
    }
    if constexpr (sizeof(T) == 4) {
        if (bhi) stage_u_block<NC>(X, kb, nc, c0, j0, bhi, blo, bscale, split);
    }
}

// ---------------------------------------------------------------------------
// SIMT complex GEMM for the trailing update: C[m0.., n0..] -= L U
// L = A[r, k:k+kk], U = A[k:k+kk, c]; 64 x 64 output tile, 256 threads,
// 4 x 4 complex accumulators per thread.
// ---------------------------------------------------------------------------
constexpr int GT = 64, GKC = 16;
template <typename T>
__global__ void __launch_bounds__(256, 2) gemm_update_kernel(Cx<T> *A, int64_t ld, int n, int k, int kk, int row0,
                                                          int col0, int col_end) {
    __shared__ Cx<T> sL[GKC][GT + 1];
    __shared__ Cx<T> sU[GKC][GT];
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    const int r0 = row0 + blockIdx.y * GT, c0 = col0 + blockIdx.x * GT;
    T acc[4][4][2];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = T(0);
    for (int kc = 0; kc < kk; kc += GKC) {
        {
            constexpr int PER = GT * GKC / 256;
            Cx<T> vl[PER], vu[PER];
#pragma unroll
            for (int u = 0; u < PER; ++u) {
                const int idx = threadIdx.x + u * 256;
                const int i = idx / GKC, q = idx % GKC, r = r0 + i, kq = kc + q;
                vl[u] = (r < n && kq < kk) ? A[(int64_t)r * ld + k + kq] : Cx<T>{T(0), T(0)};
                const int q2 = idx / GT, j = idx % GT, c = c0 + j, kq2 = kc + q2;
                vu[u] = (c < col_end && kq2 < kk) ? A[(int64_t)(k + kq2) * ld + c] : Cx<T>{T(0), T(0)};
            }
#pragma unroll
            for (int u = 0; u < PER; ++u) {
                const int idx = threadIdx.x + u * 256;
                sL[idx % GKC][idx / GKC] = vl[u];
                sU[idx / GT][idx % GT] = vu[u];
            }
        }
        __syncthreads();
#pragma unroll 4
        for (int q = 0; q < GKC; ++q) {
            Cx<T> a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) a[i] = sL[q][ty + 16 * i];
#pragma unroll
            for (int j = 0; j < 4; ++j) b[j] = sU[q][tx + 16 * j];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    acc[i][j][0] += a[i].re * b[j].re - a[i].im * b[j].im;
                    acc[i][j][1] += a[i].re * b[j].im + a[i].im * b[j].re;
                }
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int r = r0 + ty + 16 * i, c = c0 + tx + 16 * j;
            if (r < n && c < col_end) {
                Cx<T> &d = A[(int64_t)r * ld + c];
                d.re -= acc[i][j][0];
                d.im -= acc[i][j][1];
            }
        }
}

// ---------------------------------------------------------------------------
// FP64 tensor-core (DMMA) complex GEMM for the FP64 form's updates:
// C[r0.., c0..] -= L U on the same 64 x 64 complex output tiles as
// gemm_update_kernel.  Eight warps as 2 x 4, each a 32 x 16 complex warp tile
// of 8 x 8 blocks computed with mma.sync.m8n8k4.f64 (4 real products per
// complex block: re += Lr Ur - Li Ui, im += Lr Ui + Li Ur).  L and U are
// staged as separate real / imaginary planes, K in chunks of 16, with row
// paddings that keep each fragment load to its two 128-byte wavefronts.
// Fragments (PTX ISA, m8n8k4 .f64): A a0 at (lane / 4, lane % 4); B b0 at
// (lane % 4, lane / 4); C c0, c1 at (lane / 4, 2 (lane % 4) + 0, 1).
// ---------------------------------------------------------------------------
constexpr int DM_KC = 16, DM_LP = DM_KC + 4, DM_UP = GT + 4;

__device__ __forceinline__ void dmma884(double (&c)[2], double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(c[0]), "+d"(c[1])
                 : "d"(a), "d"(b));
}

// Persistent over the output tiles (tiles_x per row of tiles, ntiles in all):
// CTA b takes tiles b, b + gridDim.x, ... so a capped grid leaves SMs free
// for the kernels running beside it (the LU's panel on the other stream).
__global__ void __launch_bounds__(256, 2) dmma_update_kernel(Cx<double> *A, int64_t ld, int n, int k, int kk,
                                                            int row0, int col0, int col_end, int tiles_x,
                                                            int ntiles) {
    __shared__ double sLr[GT][DM_LP], sLi[GT][DM_LP];  // L chunk: 64 rows x 16
    __shared__ double sUr[DM_KC][DM_UP], sUi[DM_KC][DM_UP];  // U chunk: 16 x 64 columns
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wr = warp >> 2, wc = warp & 3;  // warp tile: rows 32 wr .., columns 16 wc ..
    const int g = lane >> 2, t = lane & 3;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int r0 = row0 + (tile / tiles_x) * GT, c0 = col0 + (tile % tiles_x) * GT;
    double cr[4][2][2], ci[4][2][2];  // [row block][column block][fragment]
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 2; ++j) cr[i][j][0] = cr[i][j][1] = ci[i][j][0] = ci[i][j][1] = 0.0;
    for (int kc = 0; kc < kk; kc += DM_KC) {
        // stage the chunk: 64 x 16 of L and 16 x 64 of U, four complex entries each per thread
#pragma unroll
        for (int u = 0; u < GT * DM_KC / 256; ++u) {
            const int idx = tid + u * 256;
            const int i = idx / DM_KC, q = idx % DM_KC, r = r0 + i, kq = kc + q;
            const Cx<double> vl = (r < n && kq < kk) ? A[(int64_t)r * ld + k + kq] : Cx<double>{0.0, 0.0};
            sLr[i][q] = vl.re;
            sLi[i][q] = vl.im;
            const int q2 = idx / GT, j = idx % GT, c = c0 + j, kq2 = kc + q2;
            const Cx<double> vu = (c < col_end && kq2 < kk) ? A[(int64_t)(k + kq2) * ld + c] : Cx<double>{0.0, 0.0};
            sUr[q2][j] = vu.re;
            sUi[q2][j] = vu.im;
        }
        __syncthreads();
#pragma unroll
        for (int k4 = 0; k4 < DM_KC; k4 += 4) {
            double ar[4], ai[4], nai[4], br[2], bi[2];
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                ar[i] = sLr[32 * wr + 8 * i + g][k4 + t];
                ai[i] = sLi[32 * wr + 8 * i + g][k4 + t];
                nai[i] = -ai[i];
            }
#pragma unroll
            for (int j = 0; j < 2; ++j) {
                br[j] = sUr[k4 + t][16 * wc + 8 * j + g];
                bi[j] = sUi[k4 + t][16 * wc + 8 * j + g];
            }
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 2; ++j) {
                    dmma884(cr[i][j], ar[i], br[j]);
                    dmma884(cr[i][j], nai[i], bi[j]);
                    dmma884(ci[i][j], ar[i], bi[j]);
                    dmma884(ci[i][j], ai[i], br[j]);
                }
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 2; ++j)
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                const int r = r0 + 32 * wr + 8 * i + g, c = c0 + 16 * wc + 8 * j + 2 * t + e;
                if (r < n && c < col_end) {
                    Cx<double> &d = A[(int64_t)r * ld + c];
                    d.re -= cr[i][j][e];
                    d.im -= ci[i][j][e];
                }
            }
    }
}

// the trailing / in-panel update C -= L U over rows row0.. and columns
// [col0, col_end): tensor cores (DMMA) in FP64, SIMT in FP32.  max_ctas
// (0: no cap) bounds the persistent DMMA grid.
template <typename T>
static void launch_update(cudaStream_t st, dim3 grid, Cx<T> *A, int64_t ld, int n, int k, int kk, int row0, int col0,
                          int col_end, int max_ctas = 0) {
    if constexpr (sizeof(T) == 8) {
        const int ntiles = (int)(grid.x * grid.y);
        const int g = max_ctas > 0 ? std::min(ntiles, max_ctas) : ntiles;
        if (g > 0)
            dmma_update_kernel<<<g, 256, 0, st>>>(A, ld, n, k, kk, row0, col0, col_end, (int)grid.x, ntiles);
    } else {
        gemm_update_kernel<T><<<grid, 256, 0, st>>>(A, ld, n, k, kk, row0, col0, col_end);
    }
}

// ---------------------------------------------------------------------------
// FP32 update inside a panel, after each of its sub-panels: C[row0.., col0 ..
// col_end) -= L U with L = A[r, k:k+kk], U = A[k:k+kk, c], kk <= 32.  The
// update is 32, 64 or 96 columns wide, so the tiles are 128 x 32 complex: the
// whole K is staged at once by the asynchronous copy unit while each thread
// prefetches its 4 x 4 outputs, then one barrier and kk rank-1 steps from
// shared memory.  (The square 64 x 64 tiles of gemm_update_kernel left half of
// each tile idle on the 32-column updates and staged K in two synchronised
// chunks.)  C never overlaps L or U: rows >= row0 > k + kk, columns >= col0.
// ---------------------------------------------------------------------------
constexpr int PU_ROWS = 128, PU_COLS = 32, PU_K = 32;
__global__ void __launch_bounds__(256, 2) panel_update_kernel(Cx<float> *A, int64_t ld, int n, int k, int kk, int row0,
                                                             int col0, int col_end) {
    __shared__ __align__(16) Cx<float> sL[PU_ROWS][PU_K + 1];
    __shared__ __align__(16) Cx<float> sU[PU_K][PU_COLS];
    const int tid = threadIdx.x, tx = tid % 8, ty = tid / 8;  // outputs: rows ty + 32 i, columns tx + 8 j
    const int r0 = row0 + blockIdx.y * PU_ROWS, c0 = col0 + blockIdx.x * PU_COLS;
    for (int i = tid; i < PU_ROWS * PU_K; i += 256) {
        const int rr = i / PU_K, q = i % PU_K, r = r0 + rr;
        if (r < n && q < kk)
            cp_async_cx(&sL[rr][q], &A[(int64_t)r * ld + k + q]);
        else
            sL[rr][q] = Cx<float>{0.f, 0.f};
    }
    for (int i = tid; i < PU_K * PU_COLS; i += 256) {
        const int q = i / PU_COLS, cc = i % PU_COLS, c = c0 + cc;
        if (c < col_end && q < kk)
            cp_async_cx(&sU[q][cc], &A[(int64_t)(k + q) * ld + c]);
        else
            sU[q][cc] = Cx<float>{0.f, 0.f};
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
    Cx<float> cur[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int r = r0 + ty + 32 * i, c = c0 + tx + 8 * j;
            cur[i][j] = (r < n && c < col_end) ? A[(int64_t)r * ld + c] : Cx<float>{0.f, 0.f};
        }
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    __syncthreads();
    float acc[4][4][2];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.f;
#pragma unroll 4
    for (int q = 0; q < PU_K; ++q) {
        Cx<float> a[4], b[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) a[i] = sL[ty + 32 * i][q];
#pragma unroll
        for (int j = 0; j < 4; ++j) b[j] = sU[q][tx + 8 * j];
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                acc[i][j][0] += a[i].re * b[j].re - a[i].im * b[j].im;
                acc[i][j][1] += a[i].re * b[j].im + a[i].im * b[j].re;
            }
    }
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int r = r0 + ty + 32 * i, c = c0 + tx + 8 * j;
            if (r < n && c < col_end)
                A[(int64_t)r * ld + c] = Cx<float>{cur[i][j].re - acc[i][j][0], cur[i][j].im - acc[i][j][1]};
        }
}

// ---------------------------------------------------------------------------
// Sub-panel factorisation on one thread-block cluster.  CP_CTAS CTAs hold all
// rows of a w-column sub-panel (256-byte rows) in shared memory; rows never
// move: each row carries its logical position, and an interchange only swaps
// two positions.  Per column j:
//   1. wait on this CTA's mbarrier until every CTA's candidate for column j
//      (magnitude, position, and the whole candidate row, finished through
//      step j - 1) has landed in this CTA's shared memory;
//   2. every warp picks the same winner from the CP_CTAS candidates
//      (redux.sync on the magnitude bits, then the smallest position);
//   3. look-ahead: multipliers of column j and column j + 1 of every
//      remaining row, each thread's best row, each warp's best row finished
//      through step j into a staging buffer by the warp's lanes;
//   4. one CTA barrier, the CTA's best row among the warps' rows, and warp q
//      pushes it to CTA q (one 16-byte st.async per lane, complete_tx on the
//      receiver's mbarrier);
//   5. the remaining columns of step j are eliminated while the pushes fly.
// Candidate slots and mbarriers rotate over three columns: a CTA still
// eliminating column j - 1 reads that column's slot after it has pushed its
// candidate for column j, so a peer that holds every candidate for j may push
// j + 1, but never j + 2, before the slot of j - 1 is free.  The staging
// buffers and the warp results alternate with the column parity: the one CTA
// barrier of a column separates their writers from the previous readers.
// Every wait is bounded.
// ---------------------------------------------------------------------------
constexpr int CP_CTAS = 16, CP_THREADS = 512, CP_WARPS = CP_THREADS / 32, CP_RMAX = 2, CP_ROW_BYTES = 272,
              CP_SLOTS = 3;
static_assert(CP_WARPS == CP_CTAS, "warp q pushes to CTA q");
constexpr int CP_NONE = 0x7fffffff;  // position of "no candidate"

struct alignas(16) PivKey {
    uint32_t w[4];  // magnitude bits (lo, hi), position, unused
};

__device__ __forceinline__ uint32_t cl_rank() {
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}
__device__ __forceinline__ uint32_t sm_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ uint32_t cl_map(uint32_t a, uint32_t rank) {
    uint32_t r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(rank));
    return r;
}
__device__ __forceinline__ void cl_sync() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}
__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
__device__ __forceinline__ void mb_init(uint64_t *b, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(sm_addr(b)), "r"(count) : "memory");
}
__device__ __forceinline__ void mb_init_fence() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void mb_arrive_expect(uint64_t *b, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(sm_addr(b)), "r"(bytes) : "memory");
}
// true once the phase of the given parity completed (the thread may be
// suspended inside until the phase completes or a time limit of the system
// passes; with a suspend-time hint of 1 us the panels measured 3 % slower)
__device__ __forceinline__ bool mb_try(uint64_t *b, unsigned parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(sm_addr(b)), "r"(parity)
        : "memory");
    return ok != 0;
}
// one row of 16-byte-aligned bytes between global and shared memory by the
// bulk-copy engine (no multicast); the load completes on an mbarrier
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void *src, uint32_t bytes, uint32_t bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
}
__device__ __forceinline__ void bulk_s2g(void *dst, uint32_t src, uint32_t bytes) {
    asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst), "r"(src), "r"(bytes) : "memory");
}
__device__ __forceinline__ void bulk_commit_wait_all() {
    asm volatile("cp.async.bulk.commit_group;\n\tcp.async.bulk.wait_group 0;" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void st_async16(uint32_t addr, uint4 v, uint32_t bar) {
    asm volatile("st.async.shared::cluster.mbarrier::complete_tx::bytes.v4.b32 [%0], {%1, %2, %3, %4}, [%5];" ::"r"(
                     addr),
                 "r"(v.x), "r"(v.y), "r"(v.z), "r"(v.w), "r"(bar)
                 : "memory");
}

// ordered bits of a non-negative magnitude (0 also stands for "none")
__device__ __forceinline__ uint64_t mag_bits(float v) { return (uint64_t)__float_as_uint(v); }
__device__ __forceinline__ uint64_t mag_bits(double v) { return (uint64_t)__double_as_longlong(v); }
template <typename T> __device__ __forceinline__ T mag_value(uint64_t b);
template <> __device__ __forceinline__ float mag_value<float>(uint64_t b) { return __uint_as_float((uint32_t)b); }
template <> __device__ __forceinline__ double mag_value<double>(uint64_t b) { return __longlong_as_double((long long)b); }

// lane holding the largest magnitude, the smallest position among equals
// (all 32 lanes take part; the result is the same in every lane)
template <typename T> __device__ __forceinline__ int warp_argbest(uint64_t m, int pos) {
    bool tie;
    if (sizeof(T) == 8) {
        const uint32_t hi = (uint32_t)(m >> 32), lo = (uint32_t)m;
        const uint32_t mhi = __reduce_max_sync(0xffffffffu, hi);
        const uint32_t mlo = __reduce_max_sync(0xffffffffu, hi == mhi ? lo : 0u);
        tie = hi == mhi && lo == mlo;
    } else {
        const uint32_t mm = __reduce_max_sync(0xffffffffu, (uint32_t)m);
        tie = (uint32_t)m == mm;
    }
    const unsigned ties = __ballot_sync(0xffffffffu, tie);
    if (__popc(ties) == 1) return __ffs(ties) - 1;  // one largest magnitude: no position to compare
    const int mpos = __reduce_min_sync(0xffffffffu, tie ? pos : CP_NONE);
    return __ffs(__ballot_sync(0xffffffffu, tie && pos == mpos)) - 1;
}

// 16 bytes of a row: 2 c64 or 1 c128 entries
__device__ __forceinline__ float4 v16_ld(const Cx<float> *p) { return *reinterpret_cast<const float4 *>(p); }
__device__ __forceinline__ double2 v16_ld(const Cx<double> *p) { return *reinterpret_cast<const double2 *>(p); }
__device__ __forceinline__ void v16_st(Cx<float> *p, float4 v) { *reinterpret_cast<float4 *>(p) = v; }
__device__ __forceinline__ void v16_st(Cx<double> *p, double2 v) { *reinterpret_cast<double2 *>(p) = v; }
__device__ __forceinline__ float4 v16_cms(float4 x, Cx<float> l, float4 u) {
    const Cx<float> a = cms(Cx<float>{x.x, x.y}, l, Cx<float>{u.x, u.y});
    const Cx<float> b = cms(Cx<float>{x.z, x.w}, l, Cx<float>{u.z, u.w});
    return make_float4(a.re, a.im, b.re, b.im);
}
__device__ __forceinline__ double2 v16_cms(double2 x, Cx<double> l, double2 u) {
    const Cx<double> a = cms(Cx<double>{x.x, x.y}, l, Cx<double>{u.x, u.y});
    return make_double2(a.re, a.im);
}

// row[c] -= l prow[c] for c in [c0, w); row and prow 16-byte aligned, w even
// for c64 entries
template <typename T> __device__ __forceinline__ void row_update(Cx<T> *row, const Cx<T> *prow, Cx<T> l, int c0, int w) {
    constexpr int E = 16 / sizeof(Cx<T>);
    int c = c0;
    if (E == 2 && (c & 1) && c < w) {
        row[c] = cms(row[c], l, prow[c]);
        ++c;
    }
    for (; c < w; c += 4 * E) {
        decltype(v16_ld(row)) x[4], u[4];
#pragma unroll
        for (int t = 0; t < 4; ++t)
            if (c + t * E < w) {
                x[t] = v16_ld(row + c + t * E);
                u[t] = v16_ld(prow + c + t * E);
            }
#pragma unroll
        for (int t = 0; t < 4; ++t)
            if (c + t * E < w) v16_st(row + c + t * E, v16_cms(x[t], l, u[t]));
    }
}

template <typename T> struct ClusterPanelArgs {
    Cx<T> *A;
    int64_t ld;
    int n, k, w;  // sub-panel: rows [k, n), columns [k, k + w)
    int rpc;      // rows per CTA
    int *ipiv;
    int *status;
    Cx<T> *dinv;  // inverse of the unit lower w x w diagonal block (nullptr: not wanted)
    int xc0, xc1; // the panel's columns: the interchanges go to [xc0, xc1) outside [k, k + w) as well
                  // (xc0 == xc1: the caller swaps the other columns itself)
    uint64_t timeout_ns;
};

// values per thread that the interchange of the panel's other columns holds
// between its read and write phases: moved rows (<= 2 w) x columns (< nb)
template <typename T> struct CpMove { static constexpr int V = sizeof(T) == 4 ? 12 : 8; };
constexpr int CP_MAXMOVED = 64;

template <typename T>
__global__ void __launch_bounds__(CP_THREADS) cluster_panel_kernel(ClusterPanelArgs<T> a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr int RS = CP_ROW_BYTES / sizeof(Cx<T>);  // padded row stride (entries)
    const int w = a.w, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    Cx<T> *P = reinterpret_cast<Cx<T> *>(smem_raw);                                    // rpc x RS
    Cx<T> *slot_row = P + (size_t)a.rpc * RS;                                           // [CP_SLOTS][CP_CTAS][w]
    Cx<T> *wbuf = slot_row + CP_SLOTS * CP_CTAS * w;                                    // [2][CP_WARPS][w]
    Cx<T> *ublk = wbuf + 2 * CP_WARPS * w;                                              // w x (w + 1): L11^-1 (CTA 0)
    PivKey *slot_key = reinterpret_cast<PivKey *>(ublk + w * (w + 1));                 // [CP_SLOTS][CP_CTAS]
    __shared__ uint64_t mbar[CP_SLOTS];
    __shared__ uint64_t ldbar;  // the sub-panel's rows landed in shared memory
    __shared__ uint64_t red_m[2][CP_WARPS];
    __shared__ int red_pos[2][CP_WARPS];
    __shared__ int s_abort[2];
    const uint32_t rank = cl_rank();
    const int gr0 = a.k + (int)rank * a.rpc;
    const int nrows = max(0, min(a.rpc, a.n - gr0));
    const int jmax = min(w, a.n - a.k);
    const int nd = w * (int)sizeof(Cx<T>) / 16;  // data lanes of a push
    const unsigned step_bytes = CP_CTAS * (unsigned)(w * sizeof(Cx<T>) + sizeof(PivKey));
    const uint32_t row_bytes = (uint32_t)(w * sizeof(Cx<T>));
    if (tid == 0) {
        mb_init(&ldbar, 1);
        for (int b = 0; b < CP_SLOTS; ++b) mb_init(&mbar[b], 1);
        mb_init_fence();
        mb_arrive_expect(&ldbar, (unsigned)nrows * row_bytes);
        for (int b = 0; b < CP_SLOTS; ++b) mb_arrive_expect(&mbar[b], step_bytes);  // columns 0, 1, 2
        s_abort[0] = s_abort[1] = 0;
    }
    __syncthreads();
    for (int i = tid; i < nrows; i += CP_THREADS)  // rows in flight all at once
        bulk_g2s(sm_addr(P + (size_t)i * RS), a.A + (int64_t)(gr0 + i) * a.ld + a.k, row_bytes, sm_addr(&ldbar));
    if (!mb_try(&ldbar, 0u)) {
        const uint64_t t0 = global_ns();
        while (!mb_try(&ldbar, 0u))
            if (global_ns() - t0 > a.timeout_ns) {
                atomicOr(a.status, (int)DEV_BARRIER_TIMEOUT);
                break;
            }
    }
    int mp[CP_RMAX];  // logical position of local rows tid + r * CP_THREADS (-1: none)
#pragma unroll
    for (int r = 0; r < CP_RMAX; ++r) {
        const int i = tid + r * CP_THREADS;
        mp[r] = i < nrows ? gr0 + i : -1;
    }

    // the warp's best row (given each thread's best) into the staging buffer
    // `pb`, finished through step jprev (multiplier in column jprev, written by
    // its owner lane), and the warp's result into red_*[pb]
    auto warp_stage = [&](uint64_t m, int pos, int li, int pb, int jprev, const Cx<T> *prow_prev) -> int {
        const int wl = warp_argbest<T>(m, pos);
        const int wpos = __shfl_sync(0xffffffffu, pos, wl);
        const int wli = __shfl_sync(0xffffffffu, li, wl);
        const uint64_t wm = __shfl_sync(0xffffffffu, m, wl);
        __syncwarp();
        if (wpos != CP_NONE) {
            Cx<T> *row = P + (size_t)wli * RS;
            Cx<T> *dst = wbuf + (size_t)(pb * CP_WARPS + warp) * w;
            for (int c = lane; c < w; c += 32) {
                Cx<T> x = row[c];
                if (jprev >= 0 && c >= jprev + 2) {
                    x = cms(x, row[jprev], prow_prev[c]);
                    row[c] = x;
                }
                dst[c] = x;
            }
        }
        if (lane == 0) {
            red_m[pb][warp] = wm;
            red_pos[pb][warp] = wpos;
        }
        return wpos != CP_NONE ? wli : -1;
    };
    // after the CTA barrier: the CTA's best among the warps' rows; warp q
    // pushes it (slot of column s) to CTA q
    auto push = [&](int s, int pb) {
        const uint64_t m = lane < CP_WARPS ? red_m[pb][lane] : 0ull;
        const int pos = lane < CP_WARPS ? red_pos[pb][lane] : CP_NONE;
        const int bw = warp_argbest<T>(m, pos);
        const uint64_t cm = __shfl_sync(0xffffffffu, m, bw);
        const int cpos = __shfl_sync(0xffffffffu, pos, bw);
        const int ps = s % CP_SLOTS;
        uint4 v = make_uint4(0u, 0u, 0u, 0u);
        uint32_t dst = 0;
        if (lane < nd) {
            if (cpos != CP_NONE) v = reinterpret_cast<const uint4 *>(wbuf + (size_t)(pb * CP_WARPS + bw) * w)[lane];
            dst = sm_addr(slot_row + (size_t)(ps * CP_CTAS + rank) * w) + 16u * lane;
        } else if (lane == nd) {
            v = make_uint4((uint32_t)cm, (uint32_t)(cm >> 32), (uint32_t)cpos, 0u);
            dst = sm_addr(&slot_key[ps * CP_CTAS + rank]);
        }
        if (lane <= nd) st_async16(cl_map(dst, warp), v, cl_map(sm_addr(&mbar[ps]), warp));
    };

    // candidate of column 0
    {
        uint64_t m = 0;
        int pos = CP_NONE, li = -1;
#pragma unroll
        for (int r = 0; r < CP_RMAX; ++r) {
            const int i = tid + r * CP_THREADS;
            if (mp[r] >= 0) {
                const uint64_t mr = mag_bits(cabs1(P[i * RS]));
                if (pos == CP_NONE || mr > m || (mr == m && mp[r] < pos)) {
                    m = mr;
                    pos = mp[r];
                    li = i;
                }
            }
        }
        warp_stage(m, pos, li, 1, -1, nullptr);
        __syncthreads();
        cl_sync();  // every CTA's mbarriers are initialised before any remote store
        if (jmax > 0) push(0, 1);
    }

    for (int j = 0; j < jmax; ++j) {
        const int jr = a.k + j, par = j % CP_SLOTS, pb = j & 1;
        if (!mb_try(&mbar[par], (unsigned)(j / CP_SLOTS) & 1u)) {
            const uint64_t t0 = global_ns();
            while (!mb_try(&mbar[par], (unsigned)(j / CP_SLOTS) & 1u)) {
                if (global_ns() - t0 > a.timeout_ns) {
                    s_abort[pb] = 1;
                    atomicOr(a.status, (int)DEV_BARRIER_TIMEOUT);
                    break;
                }
            }
        }
        if (tid == 0 && !s_abort[pb]) mb_arrive_expect(&mbar[par], step_bytes);  // next phase: column j + 3
        // the same winner in every warp
        int p, wc;
        T wv;
        {
            const PivKey kq = slot_key[par * CP_CTAS + (lane & (CP_CTAS - 1))];
            const uint64_t m = lane < CP_CTAS ? ((uint64_t)kq.w[1] << 32 | kq.w[0]) : 0ull;
            const int pos = lane < CP_CTAS ? (int)kq.w[2] : CP_NONE;
            wc = warp_argbest<T>(m, pos) & (CP_CTAS - 1);
            p = __shfl_sync(0xffffffffu, pos, wc);
            wv = mag_value<T>(__shfl_sync(0xffffffffu, m, wc));
        }
        if (p < jr || p >= a.n) {  // no candidate (or a damaged slot): keep the row in place
            p = jr;
            wv = T(0);
        }
        const Cx<T> *prow = slot_row + (size_t)(par * CP_CTAS + wc) * w;
        if (tid == 0) {
            if (!(wv > T(0))) atomicOr(a.status, (int)DEV_ZERO_PIVOT);
            if (rank == 0) a.ipiv[jr] = p;
        }
        const Cx<T> pv = prow[j];
        const T den = pv.re * pv.re + pv.im * pv.im;
        const T rd = den > T(0) ? rcp_rn(den) : T(0);
        const Cx<T> inv{pv.re * rd, -pv.im * rd};
        // interchange of positions jr and p; the pivot row retires at jr
#pragma unroll
        for (int r = 0; r < CP_RMAX; ++r) {
            if (mp[r] == p)
                mp[r] = jr;
            else if (mp[r] == jr)
                mp[r] = p;
        }
        // look-ahead: multipliers and column j + 1, with each thread's best row
        const bool more = j + 1 < jmax;
        uint64_t m = 0;
        int pos = CP_NONE, li = -1;
        {
            Cx<T> xj[CP_RMAX], xn[CP_RMAX];
#pragma unroll
            for (int r = 0; r < CP_RMAX; ++r)
                if (mp[r] > jr) {
                    const Cx<T> *row = P + (size_t)(tid + r * CP_THREADS) * RS;
                    xj[r] = row[j];
                    if (more) xn[r] = row[j + 1];
                }
            const Cx<T> u = more ? prow[j + 1] : Cx<T>{T(0), T(0)};
#pragma unroll
            for (int r = 0; r < CP_RMAX; ++r)
                if (mp[r] > jr) {
                    const int i = tid + r * CP_THREADS;
                    Cx<T> *row = P + (size_t)i * RS;
                    const Cx<T> l = cmul(xj[r], inv);
                    row[j] = l;
                    if (more) {
                        const Cx<T> y = cms(xn[r], l, u);
                        row[j + 1] = y;
                        const uint64_t mr = mag_bits(cabs1(y));
                        if (pos == CP_NONE || mr > m || (mr == m && mp[r] < pos)) {
                            m = mr;
                            pos = mp[r];
                            li = i;
                        }
                    }
                }
        }
        int staged = -1;  // local row finished by this warp for the push
        if (more) staged = warp_stage(m, pos, li, pb, j, prow);
        __syncthreads();
        if (s_abort[pb]) break;  // read after the barrier: uniform
        if (more) push(j + 1, pb);
        // rest of step j
        const int c0 = more ? j + 2 : j + 1;
#pragma unroll
        for (int r = 0; r < CP_RMAX; ++r) {
            const int i = tid + r * CP_THREADS;
            if (mp[r] > jr && i != staged) {
                Cx<T> *row = P + (size_t)i * RS;
                row_update(row, prow, row[j], c0, w);
            }
        }
        if (rank == 0 && warp == CP_WARPS - 1 && a.dinv && lane < w) {
            // row j of the inverse of the unit lower diagonal block, whose row
            // j is prow[0:j]:  Y[j][c] = delta_jc - sum_{t<j} prow[t] Y[t][c]
            Cx<T> s0{T(lane == j), T(0)}, s1{T(0), T(0)}, s2{T(0), T(0)}, s3{T(0), T(0)};
            int t = 0;
            for (; t + 4 <= j; t += 4) {
                s0 = cms(s0, prow[t], ublk[t * (w + 1) + lane]);
                s1 = cms(s1, prow[t + 1], ublk[(t + 1) * (w + 1) + lane]);
                s2 = cms(s2, prow[t + 2], ublk[(t + 2) * (w + 1) + lane]);
                s3 = cms(s3, prow[t + 3], ublk[(t + 3) * (w + 1) + lane]);
            }
            for (; t < j; ++t) s0 = cms(s0, prow[t], ublk[t * (w + 1) + lane]);
            ublk[j * (w + 1) + lane] = Cx<T>{(s0.re + s1.re) + (s2.re + s3.re), (s0.im + s1.im) + (s2.im + s3.im)};
        }
    }
    // each row to its final position, by the bulk-copy engine
    fence_proxy_async_smem();
    __syncthreads();
#pragma unroll
    for (int r = 0; r < CP_RMAX; ++r) {
        const int i = tid + r * CP_THREADS;
        if (i < nrows && mp[r] >= a.k && mp[r] < a.n)
            bulk_s2g(a.A + (int64_t)mp[r] * a.ld + a.k, sm_addr(P + (size_t)i * RS), row_bytes);
    }
    // the same interchanges on the panel's other columns: every CTA reads its
    // moved rows there before the cluster barrier and writes them at their
    // final positions after it (a permutation: every destination is some moved
    // row's origin, read before the barrier)
    __shared__ int mv_src[CP_MAXMOVED], mv_dst[CP_MAXMOVED], mv_n;
    constexpr int MV = CpMove<T>::V;
    Cx<T> mvv[MV];
    const int nleft = a.k - a.xc0, nother = (a.xc1 > a.xc0) ? nleft + (a.xc1 - a.k - w) : 0;
    int nitems = 0;
    if (nother > 0) {
        if (tid == 0) mv_n = 0;
        __syncthreads();
#pragma unroll
        for (int r = 0; r < CP_RMAX; ++r) {
            const int i = tid + r * CP_THREADS;
            if (i < nrows && mp[r] >= a.k && mp[r] < a.n && mp[r] != gr0 + i) {
                const int slot = atomicAdd(&mv_n, 1);
                if (slot < CP_MAXMOVED) {
                    mv_src[slot] = gr0 + i;
                    mv_dst[slot] = mp[r];
                }
            }
        }
        __syncthreads();
        nitems = min(mv_n, CP_MAXMOVED) * nother;
        if (mv_n > CP_MAXMOVED || nitems > MV * CP_THREADS) {  // the host sizes the panel so that this cannot happen
            if (tid == 0) atomicOr(a.status, (int)DEV_BARRIER_TIMEOUT);
            nitems = 0;
        }
#pragma unroll
        for (int u = 0; u < MV; ++u) {
            const int it = tid + u * CP_THREADS;
            if (it < nitems) {
                const int row = it / nother, cc = it % nother;
                const int col = cc < nleft ? a.xc0 + cc : a.k + w + (cc - nleft);
                mvv[u] = a.A[(int64_t)mv_src[row] * a.ld + col];
            }
        }
    }
    bulk_commit_wait_all();
    if (rank == 0 && warp == 0 && a.dinv && lane < w)  // the inverse, identity past jmax
        for (int i = 0; i < w; ++i)
            a.dinv[(size_t)i * w + lane] = i < jmax ? ublk[i * (w + 1) + lane] : Cx<T>{T(i == lane), T(0)};
    cl_sync();  // every CTA's reads are done; no CTA leaves while a peer may still store into its shared memory
#pragma unroll
    for (int u = 0; u < MV; ++u) {
        const int it = tid + u * CP_THREADS;
        if (it < nitems) {
            const int row = it / nother, cc = it % nother;
            const int col = cc < nleft ? a.xc0 + cc : a.k + w + (cc - nleft);
            a.A[(int64_t)mv_dst[row] * a.ld + col] = mvv[u];
        }
    }
}

// shared memory of the cluster kernel for rpc rows of width w
template <typename T> static size_t cluster_panel_smem(int rpc, int w) {
    return (size_t)rpc * CP_ROW_BYTES + sizeof(Cx<T>) * ((CP_SLOTS * CP_CTAS + 2 * CP_WARPS) * (size_t)w + w * (w + 1)) +
           sizeof(PivKey) * CP_SLOTS * CP_CTAS;
}

// Launches the cluster kernel for a sub-panel; false when the rows do not fit
// the cluster's shared memory or no cluster of CP_CTAS can be scheduled.
template <typename T>
static bool cluster_panel(beat_b200_ctx *c, Cx<T> *A, int64_t ld, int n, int k, int w, int *ipiv, Cx<T> *dinv,
                          int xc0 = 0, int xc1 = 0) {
    const int m = n - k;
    const int rpc = (m + CP_CTAS - 1) / CP_CTAS;
    constexpr size_t cap = 220 * 1024;
    if (w * sizeof(Cx<T>) > 256 || (w * sizeof(Cx<T>)) % 16 != 0 || rpc > CP_RMAX * CP_THREADS || n >= (1 << 30))
        return false;
    const size_t smem = cluster_panel_smem<T>(rpc, w);
    if (smem > cap) return false;
    static std::atomic<bool> attr_done[2] = {false, false};  // sweep lanes call this from several threads
    const int ti = sizeof(T) == 8;
    if (!attr_done[ti]) {
        BB_CUDA(cudaFuncSetAttribute(cluster_panel_kernel<T>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
        BB_CUDA(cudaFuncSetAttribute(cluster_panel_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cap));
        attr_done[ti] = true;
    }
    ClusterPanelArgs<T> a;
    a.A = A;
    a.ld = ld;
    a.n = n;
    a.k = k;
    a.w = w;
    a.rpc = rpc;
    a.ipiv = ipiv;
    a.status = c->status.as<int>();
    a.dinv = dinv;
    a.xc0 = xc0;
    a.xc1 = xc1;
    a.timeout_ns = 100000000ull;  // 0.1 s per column wait
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(CP_CTAS);
    cfg.blockDim = dim3(CP_THREADS);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = c->stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = CP_CTAS;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    if (!c->cluster_checked) {
        int nclusters = 0;
        cfg.dynamicSmemBytes = cap;  // the largest request any sub-panel makes
        cudaError_t e = cudaOccupancyMaxActiveClusters(&nclusters, (void *)cluster_panel_kernel<T>, &cfg);
        cfg.dynamicSmemBytes = smem;
        c->cluster_ok = (e == cudaSuccess && nclusters >= 1);
        cudaGetLastError();
        c->cluster_checked = true;
    }
    if (!c->cluster_ok) return false;
    BB_CUDA(cudaLaunchKernelEx(&cfg, cluster_panel_kernel<T>, a));
    return true;
}

// FP32 form trailing update on the tensor cores (tc_gemm.cu)
bool tc_update_supported(int nb);
void tc_stage_l(beat_b200_ctx *c, int k, int nb, int split_terms, cudaStream_t st);
void tc_stage_u(beat_b200_ctx *c, int k, int nb, int split_terms, int col_lo, int col_hi, cudaStream_t st);
void tc_stage_u_buffers(beat_b200_ctx *c, int k, int nb, __half **bhi, __half **blo, float **bscale);
void tc_update_cols(beat_b200_ctx *c, int k, int nb, int split_terms, int col_lo, int col_hi, cudaStream_t st,
                    int max_ctas);

// ---------------------------------------------------------------------------
// host driver
// ---------------------------------------------------------------------------
template <typename T> static void lu_factor_t(beat_b200_ctx *c, int nb, int split_terms) {
    Workspace &w = c->ws;
    const int n = c->V;
    const int64_t ld = w.ld;
    Cx<T> *A = w.A.as<Cx<T>>();
    int G = c->sm_count;
    // shared memory per CTA for the panel: rows x nb + 2 nb + rows
    const size_t smem_cap = 200 * 1024;
    int rpc = (n + G - 1) / G;
    size_t smem = sizeof(Cx<T>) * ((size_t)rpc * nb + 2 * nb + rpc);
    BB_REQUIRE(smem <= smem_cap, BEAT_B200_INVALID_ARG,
               "LU: system of order " + std::to_string(n) + " exceeds the shared-memory panel limit");
    // scratch: [2][G] pivot records, [2][G][nb] candidate rows, [2][nb] diagonal rows
    // and the inverses of the sub-panels' W x W diagonal blocks
    const int W = std::min(nb, (int)(256 / sizeof(Cx<T>)));
    const size_t rec_bytes = sizeof(PivotRec) * 2 * (size_t)G;
    const size_t scratch = rec_bytes + sizeof(Cx<T>) * (2 * (size_t)G * nb + 2 * nb);
    const size_t dinv_off = (scratch + 255) / 256 * 256;
    const size_t dinv_bytes = sizeof(Cx<T>) * (size_t)W * W * ((n + W - 1) / W);
    w.panel_scratch.alloc(dinv_off + dinv_bytes);
    PivotRec *recs = w.panel_scratch.as<PivotRec>();
    Cx<T> *pub_rows = reinterpret_cast<Cx<T> *>(recs + 2 * G);
    Cx<T> *pub_diag = pub_rows + 2 * (size_t)G * nb;
    Cx<T> *dinv = reinterpret_cast<Cx<T> *>(w.panel_scratch.as<unsigned char>() + dinv_off);
    // blocked U12 solves need whole W-column sub-panels of 256-byte rows
    constexpr int WF = 256 / sizeof(Cx<T>);
    const bool blocked = W == WF && nb % W == 0;
    const size_t tb_smem = sizeof(Cx<T>) * ((size_t)nb * TB_COLS + (size_t)W * (W + 1) + (size_t)W * (nb - W + 1));
    if (blocked)
        BB_CUDA(cudaFuncSetAttribute(trsm_blocked_kernel<T, WF>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)tb_smem));
    // the critical-path solves take the narrow kernel when its whole triangle fits
    constexpr int NC = narrow_cols<WF>();
    const bool narrow = blocked && trsm_narrow_smem<T, WF>(nb / W) <= 227 * 1024;
    if (narrow)
        BB_CUDA(cudaFuncSetAttribute(trsm_narrow_kernel<T, WF>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)trsm_narrow_smem<T, WF>(nb / W)));
    // the side stream's solve of the remaining columns: the same kernel with 16 columns per CTA
    // (two entries per thread in FP32), two CTAs per SM
    constexpr int NCS = NC > 16 ? NC : 16;
    const bool wide = blocked && trsm_narrow_smem<T, WF, NCS>(nb / W) <= 110 * 1024;
    if (wide)
        BB_CUDA(cudaFuncSetAttribute(trsm_narrow_kernel<T, WF, NCS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)trsm_narrow_smem<T, WF, NCS>(nb / W)));
    c->barrier.alloc(sizeof(unsigned) * 4096);
    BB_CUDA(cudaFuncSetAttribute(panel_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_cap));
    // the unblocked U12 solve (used only when the blocked one does not apply)
    const size_t trsm_smem = sizeof(Cx<T>) * ((size_t)nb * nb + (size_t)nb * TRSM_COLS);
    if (!blocked) {
        BB_REQUIRE(trsm_smem <= 227 * 1024, BEAT_B200_INVALID_ARG,
                   "LU: lu_block " + std::to_string(nb) + " is too wide for the unblocked U12 solve");
        BB_CUDA(cudaFuncSetAttribute(trsm_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)trsm_smem));
    }
    constexpr int LC = ls_cols<T>();
    BB_CUDA(cudaFuncSetAttribute(laswp_panel_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)laswp_panel_smem<T>(std::min(nb, LS_MAX))));
    iota_kernel<<<(n + 255) / 256, 256, 0, c->stream>>>(w.perm.as<int>(), n);
    BB_CUDA(cudaMemsetAsync(c->status.p, 0, sizeof(int), c->stream));
    const size_t trsm_w_smem = sizeof(Cx<T>) * ((size_t)W * W + (size_t)W * TRSM_COLS);
    int *ipiv = w.ipiv.as<int>();
    int *perm = w.perm.as<int>();
    cudaStream_t s0 = c->stream, s1 = c->side_stream;
    const bool tc = sizeof(T) == 4 && tc_update_supported(nb);
    // SMs the look-ahead update leaves to the panel factorisation beside it: one
    // 16-CTA cluster, and as many again for the panel's own updates and solves
    // between its sub-panels (measured at N = 10,242: mixed LU 46.4 ms with one
    // cluster's SMs left, 44.5 with two, 44.0 with three, where the sweep slows);
    // the grid-wide panel fallback waits for its own SMs
    const int side_cap = std::max(1, G - 2 * CP_CTAS);
    // U12 = L11^-1 A12 of panel k for the columns [c_lo, c_hi), on stream st
    // with the tensor-core update (blocked) the same launch stages U12 as the update's B operand
    const bool fused_stage = tc && blocked;
    // (crit: the next panel's columns, on the critical path)
    auto u_solve = [&](int k, int c_lo, int c_hi, cudaStream_t st, bool crit) {
        const int cols = c_hi - c_lo;
        if (cols <= 0) return;
        __half *bhi = nullptr, *blo = nullptr;
        float *bsc = nullptr;
        if (fused_stage) tc_stage_u_buffers(c, k, nb, &bhi, &blo, &bsc);
        if (crit && narrow)
            trsm_narrow_kernel<T, WF><<<(cols + NC - 1) / NC, 256, trsm_narrow_smem<T, WF>(nb / W), st>>>(
                A, ld, k, nb / W, dinv + (size_t)(k / W) * W * W, c_lo, c_hi, bhi, blo, bsc, k + nb, split_terms);
        else if (wide)
            trsm_narrow_kernel<T, WF, NCS><<<(cols + NCS - 1) / NCS, 256, trsm_narrow_smem<T, WF, NCS>(nb / W), st>>>(
                A, ld, k, nb / W, dinv + (size_t)(k / W) * W * W, c_lo, c_hi, bhi, blo, bsc, k + nb, split_terms);
        else if (blocked)
            trsm_blocked_kernel<T, WF><<<(cols + TB_COLS - 1) / TB_COLS, 256, tb_smem, st>>>(
                A, ld, k, nb / W, dinv + (size_t)(k / W) * W * W, c_lo, c_hi, bhi, blo, bsc, k + nb, split_terms);
        else
            trsm_kernel<T><<<(cols + TRSM_COLS - 1) / TRSM_COLS, 256, trsm_smem, st>>>(A, ld, n, k, nb, c_lo, c_hi);
        BB_CUDA(cudaGetLastError());
    };
    // A[k+nb.., c_lo..c_hi) -= L21 U12 of panel k, on stream st
    auto update = [&](int k, int c_lo, int c_hi, cudaStream_t st, int cap) {
        if (c_hi <= c_lo || k + nb >= n) return;
        if (tc) {
            if (!fused_stage) tc_stage_u(c, k, nb, split_terms, c_lo, c_hi, st);
            tc_update_cols(c, k, nb, split_terms, c_lo, c_hi, st, cap);
        } else {
            // one CTA per tile: capping this grid as the tensor-core one is capped
            // measured slower at N = 10,242 (154 against 136 ms for the FP64 LU)
            dim3 grid((c_hi - c_lo + GT - 1) / GT, (n - k - nb + GT - 1) / GT);
            launch_update<T>(st, grid, A, ld, n, k, nb, k + nb, c_lo, c_hi, 0);
            BB_CUDA(cudaGetLastError());
        }
    };
    // Right-looking LU with a look-ahead of one panel.  For panel k (columns
    // [k, pe)):
    //   1. factor its sub-panels on s0, swapping rows inside the panel only;
    //   2. wait for the side stream (the previous panel's update of the
    //      columns right of this panel);
    //   3. the panel's interchanges on every other column and the permutation;
    //   4. U12 and the update of the next panel's columns on s0 (they are all
    //      the next panel needs);
    //   5. U12 and the update of the remaining columns on s1, which then runs
    //      beside the next panel's factorisation (step 1 of panel k + nb).
    // The next panel touches only its own columns and rows >= pe until its
    // step 3, which follows the join: the streams never touch the same entries.
    bool side_pending = false;
    for (int k = 0; k < n; k += nb) {
        const int pe = std::min(k + nb, n);  // end of this panel
        for (int ks = k; ks < pe; ks += W) {
            const int m = n - ks;
            Cx<T> *dinv_s = blocked ? dinv + (size_t)(ks / W) * W * W : nullptr;
            // the cluster kernel also swaps the panel's other columns when they fit its
            // registers: moved rows (<= 2 W) x other columns (< nb) per CTA_THREADS x CpMove::V
            const bool own_swaps = pe - k > W && 2 * W * (pe - k - W) <= CpMove<T>::V * CP_THREADS &&
                                   2 * W <= CP_MAXMOVED;
            const bool on_cluster =
                cluster_panel<T>(c, A, ld, n, ks, W, ipiv, dinv_s, own_swaps ? k : 0, own_swaps ? pe : 0);
            if (!on_cluster) {
                // grid-wide panel kernel on the sub-panel
                int g = std::min(G, std::max(1, (m + 15) / 16));
                int rows = (m + g - 1) / g;
                PanelArgs<T> a;
                a.A = A;
                a.ld = ld;
                a.n = n;
                a.k = ks;
                a.nb = W;
                a.rpc = rows;
                a.ipiv = ipiv;
                a.pub_rows = pub_rows;
                a.pub_diag = pub_diag;
                a.recs = recs;
                a.counter = c->barrier.as<unsigned>();
                a.status = c->status.as<int>();
                a.spin_limit = 1u << 22;
                const size_t ps = sizeof(Cx<T>) * ((size_t)rows * W + 2 * W + rows);
                BB_CUDA(cudaMemsetAsync(c->barrier.p, 0, sizeof(unsigned), s0));
                void *args[] = {&a};
                BB_CUDA(cudaLaunchCooperativeKernel((void *)panel_kernel<T>, dim3(g), dim3(PANEL_THREADS), args, ps,
                                                    s0));
            }
            // this sub-panel's interchanges on the rest of the panel (unless the cluster kernel did them)
            if (pe - k > W && !(on_cluster && own_swaps)) {
                if (W <= LS_MAX)
                    laswp_panel_kernel<T><<<(pe - k + LC - 1) / LC, 256, laswp_panel_smem<T>(W), s0>>>(
                        A, ld, n, ks, W, ipiv, k, pe, ks, ks + W, nullptr);
                else
                    laswp_range_kernel<T><<<(pe - k + 1 + 255) / 256, 256, 0, s0>>>(A, ld, n, ks, W, ipiv, k, pe, ks,
                                                                                    ks + W, nullptr);
                BB_CUDA(cudaGetLastError());
            }
            if (blocked && !on_cluster) {
                diag_block_inverse_kernel<T><<<1, 32, 0, s0>>>(A, ld, n, ks, W, dinv_s);
                BB_CUDA(cudaGetLastError());
            }
            if (ks + W < pe) {
                // rest of this panel: U row block, then the panel's own trailing update
                const int cols = pe - ks - W;
                if (narrow)
                    trsm_narrow_kernel<T, WF><<<(cols + NC - 1) / NC, 256, trsm_narrow_smem<T, WF>(1), s0>>>(
                        A, ld, ks, 1, dinv + (size_t)(ks / W) * W * W, ks + W, pe, nullptr, nullptr, nullptr, 0,
                        split_terms);
                else if (blocked)
                    trsm_blocked_kernel<T, WF><<<(cols + TB_COLS - 1) / TB_COLS, 256, tb_smem, s0>>>(
                        A, ld, ks, 1, dinv + (size_t)(ks / W) * W * W, ks + W, pe);
                else
                    trsm_kernel<T><<<(cols + TRSM_COLS - 1) / TRSM_COLS, 256, trsm_w_smem, s0>>>(
                        A, ld, n, ks, W, ks + W, pe);
                if constexpr (sizeof(T) == 4) {
                    dim3 grid((cols + PU_COLS - 1) / PU_COLS, (n - ks - W + PU_ROWS - 1) / PU_ROWS);
                    panel_update_kernel<<<grid, 256, 0, s0>>>(A, ld, n, ks, W, ks + W, ks + W, pe);
                } else {
                    dim3 grid((cols + GT - 1) / GT, (n - ks - W + GT - 1) / GT);
                    launch_update<T>(s0, grid, A, ld, n, ks, W, ks + W, ks + W, pe);
                }
                BB_CUDA(cudaGetLastError());
            }
        }
        if (side_pending) {
            BB_CUDA(cudaStreamWaitEvent(s0, c->la_join, 0));
            side_pending = false;
        }
        // the panel's interchanges on every column outside it, and on perm
        if (pe - k <= LS_MAX)
            laswp_panel_kernel<T><<<(n + LC - 1) / LC, 256, laswp_panel_smem<T>(pe - k), s0>>>(A, ld, n, k, pe - k, ipiv,
                                                                                            0, n, k, pe, perm);
        else
            laswp_range_kernel<T><<<(n + 1 + 255) / 256, 256, 0, s0>>>(A, ld, n, k, pe - k, ipiv, 0, n, k, pe, perm);
        BB_CUDA(cudaGetLastError());
        if (pe >= n) break;
        const int ne = std::min(pe + nb, n);  // end of the next panel
        if (tc) {
            // L21's staging reads rows >= pe, the U12 solve writes rows < pe: the staging runs on
            // the side stream (idle since the join) beside the solve
            BB_CUDA(cudaEventRecord(c->la_fork, s0));
            BB_CUDA(cudaStreamWaitEvent(s1, c->la_fork, 0));
            tc_stage_l(c, k, nb, split_terms, s1);
            BB_CUDA(cudaEventRecord(c->la_join, s1));
        }
        u_solve(k, pe, ne, s0, true);
        if (tc) BB_CUDA(cudaStreamWaitEvent(s0, c->la_join, 0));
        update(k, pe, ne, s0, 0);
        if (ne < n) {
            BB_CUDA(cudaEventRecord(c->la_fork, s0));
            BB_CUDA(cudaStreamWaitEvent(s1, c->la_fork, 0));
            u_solve(k, ne, n, s1, false);
            update(k, ne, n, s1, side_cap);
            BB_CUDA(cudaEventRecord(c->la_join, s1));
            side_pending = true;
        }
    }
    if (side_pending) BB_CUDA(cudaStreamWaitEvent(s0, c->la_join, 0));
}



// ---------------------------------------------------------------------------
// triangular solves with R right-hand sides (X column-major N x R, FP64)
// ---------------------------------------------------------------------------
__global__ void permute_rows_kernel(const double2 *in, double2 *out, const int *perm, int n, int R) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int src = perm[i];
    for (int r = 0; r < R; ++r) out[(size_t)r * n + i] = in[(size_t)r * n + src];
}

constexpr int SB = 64, SRC = 16, SBP = SB + 1;

template <typename T> __device__ __forceinline__ Cx<double> to_d(Cx<T> v) {
    return Cx<double>{(double)v.re, (double)v.im};
}

// Inverse of every 64 x 64 diagonal block of L (unit lower, blockIdx.y = 0)
// and U (upper, blockIdx.y = 1), FP64, one CTA per block: column c of the
// inverse by substitution on e_c (64 threads, one column each).
template <typename T>
__global__ void __launch_bounds__(SB) diag_inverse_kernel(const Cx<T> *A, int64_t ld, int n, Cx<double> *Dinv) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Cx<double>(*D)[SBP] = reinterpret_cast<Cx<double>(*)[SBP]>(smem_raw);
    Cx<double>(*X)[SBP] = reinterpret_cast<Cx<double>(*)[SBP]>(smem_raw + sizeof(Cx<double>) * SB * SBP);
    const int b = blockIdx.x, upper = blockIdx.y;
    const int rb = b * SB, rows = min(SB, n - rb), c = threadIdx.x;
    for (int i = 0; i < SB; ++i)
        D[i][c] = (i < rows && c < rows) ? to_d(A[(int64_t)(rb + i) * ld + rb + c]) : Cx<double>{i == c ? 1.0 : 0.0, 0.0};
    __syncthreads();
    if (!upper) {
        for (int i = 0; i < SB; ++i) {
            Cx<double> s{i == c ? 1.0 : 0.0, 0.0};
            for (int q = 0; q < i; ++q) {
                const Cx<double> l = D[i][q], x = X[q][c];
                s.re -= l.re * x.re - l.im * x.im;
                s.im -= l.re * x.im + l.im * x.re;
            }
            X[i][c] = s;
        }
    } else {
        for (int i = SB - 1; i >= 0; --i) {
            Cx<double> s{i == c ? 1.0 : 0.0, 0.0};
            for (int q = i + 1; q < SB; ++q) {
                const Cx<double> u = D[i][q], x = X[q][c];
                s.re -= u.re * x.re - u.im * x.im;
                s.im -= u.re * x.im + u.im * x.re;
            }
            const Cx<double> u = D[i][i];
            const double den = u.re * u.re + u.im * u.im;
            X[i][c] = den > 0 ? Cx<double>{(s.re * u.re + s.im * u.im) / den, (s.im * u.re - s.re * u.im) / den}
                              : Cx<double>{0.0, 0.0};
        }
    }
    Cx<double> *out = Dinv + ((size_t)upper * gridDim.x + b) * SB * SB;
    for (int i = 0; i < SB; ++i) out[i * SB + c] = X[i][c];
}

// H_b^(d) = D_b^-1 M_b for the two blocks nearest the diagonal on the solve's
// critical path: M_b = L[b, b-d] (lower) or U[b, b+d] (upper), d = 1, 2
// (blockIdx.y = 2 (d - 1) + upper; stored in slot 2 + blockIdx.y).  With them,
// X_b = Z_b - H^(2)_b X_{b-+2} - H^(1)_b X_{b-+1}, where Z_b holds everything
// else and is formed while the two neighbouring blocks are solved.
template <typename T>
__global__ void __launch_bounds__(256) offdiag_product_kernel(const Cx<T> *A, int64_t ld, int n, Cx<double> *Dinv) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Cx<double> *Dt = reinterpret_cast<Cx<double> *>(smem_raw);  // SB x SBP
    Cx<double> *Mt = Dt + SB * SBP;                               // SB x SBP
    const int nblk = gridDim.x, b = blockIdx.x, upper = blockIdx.y & 1, dist = 1 + (blockIdx.y >> 1);
    const int nb2 = upper ? b + dist : b - dist;
    Cx<double> *H = Dinv + ((size_t)(2 + blockIdx.y) * nblk + b) * SB * SB;
    if (nb2 < 0 || nb2 >= nblk) {
        for (int i = threadIdx.x; i < SB * SB; i += blockDim.x) H[i] = Cx<double>{0.0, 0.0};
        return;
    }
    const Cx<double> *D = Dinv + ((size_t)upper * nblk + b) * SB * SB;
    const int rb = b * SB, rows = min(SB, n - rb), cb = nb2 * SB, cols = min(SB, n - cb);
    batched_copy<256, 8, Cx<double>>(SB * SB, [&](int i) { return D[i]; },
                                     [&](int i, Cx<double> v) { Dt[(i / SB) * SBP + i % SB] = v; });
    batched_copy<256, 8, Cx<double>>(
        SB * SB,
        [&](int i) {
            const int a = i / SB, q = i % SB;
            return (a < rows && q < cols) ? to_d(A[(int64_t)(rb + a) * ld + cb + q]) : Cx<double>{0.0, 0.0};
        },
        [&](int i, Cx<double> v) { Mt[(i / SB) * SBP + i % SB] = v; });
    __syncthreads();
    for (int o = threadIdx.x; o < SB * SB; o += blockDim.x) {
        const int r = o / SB, c = o % SB;
        double sr = 0, si = 0;
        for (int q = 0; q < SB; ++q) {
            const Cx<double> d = Dt[r * SBP + q], m = Mt[q * SBP + c];
            sr += d.re * m.re - d.im * m.im;
            si += d.re * m.im + d.im * m.re;
        }
        H[o] = Cx<double>{sr, si};
    }
}

// Block substitution in one kernel.  The solution is cut into 64-row blocks;
// each CTA claims the next block from a counter (so it only ever waits on
// blocks already claimed by running CTAs).  For block b it folds in
// L_bj X_j (or U_bj X_j) for every finished block j at distance 3 or more,
// forms Z_b = D_b^-1 (B_b - that sum), subtracts H^(2)_b X_{b-+2} once that
// block is done, and then X_b = Z_b - H^(1)_b X_{b-+1}: the chain from one
// block to the next is a single 64 x 64 x R product, run by the whole CTA.
// Waits are bounded: on expiry the kernel sets a status bit and continues, so
// it always terminates.
//
// Arithmetic is in the factors' type: FP64 for the FP64 form, FP32 for the
// mixed form's factors (there the substitution is the preconditioner of the
// FP64 refinement).  The folded-in products are shared by NG warp groups of
// 128 threads (4 for FP32, 2 for FP64), group g taking steps g, g + NG, ...
// with its own factor tile (cp.async, zero-filled past the matrix edge) and
// X block, synchronised by its own named barrier, so that one SM always has
// several independent tile products in flight; each thread keeps a 2-row x
// 4-column block of the 64 x 16 product in registers.  The groups' partial
// sums meet in shared memory for the tail.
template <typename T> struct SubstTile {
    // padded row length: rows start on 16-byte boundaries (cp.async) and a
    // warp's 8 rows fall on distinct banks
    static constexpr int LP = SB + (sizeof(Cx<T>) == 16 ? 1 : 2);
    // the X block column-major with a padded column: the loads (consecutive
    // rows) and the product's reads (four columns at one row) spread over banks
    static constexpr int XP = SB + 1;
    static constexpr int NG = sizeof(Cx<T>) == 16 ? 2 : 4;
    static constexpr int THREADS = 128 * NG;
    static constexpr int GROUP = SB * LP + SRC * XP;  // complex entries per group
    static constexpr size_t smem() { return sizeof(Cx<T>) * (size_t)NG * GROUP; }
};

__device__ __forceinline__ bool wait_flag(const int *flag, int epoch, int *status, unsigned spin_limit) {
    unsigned it = 0;
    while (true) {
        int v;
        asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(flag) : "memory");
        if (v == epoch) return true;
        if ((*(volatile int *)status & DEV_BARRIER_TIMEOUT) || ++it > spin_limit) {
            atomicOr(status, (int)DEV_BARRIER_TIMEOUT);
            return false;
        }
    }
}

__device__ __forceinline__ void cp_async16(void *dst, const void *src, int src_bytes) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(d), "l"(src), "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }
// barrier of one 128-thread warp group (ids 1.. ; 0 is __syncthreads)
__device__ __forceinline__ void group_bar(int grp) {
    asm volatile("bar.sync %0, 128;" ::"r"(grp + 1) : "memory");
}

// acc[2][4] += M[rows rp, rp + 32][:] V[:][4 cg .. 4 cg + 3], V column-major
// with column stride XP
template <typename C, int LP, int XP>
__device__ __forceinline__ void subst_product(const Cx<C> *M, const Cx<C> *V, int rp, int cg, C (&ar)[2][4],
                                              C (&ai)[2][4]) {
#pragma unroll 8
    for (int q = 0; q < SB; ++q) {
        const Cx<C> m0 = M[rp * LP + q], m1 = M[(rp + 32) * LP + q];
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const Cx<C> v = V[(4 * cg + e) * XP + q];
            ar[0][e] += m0.re * v.re - m0.im * v.im;
            ai[0][e] += m0.re * v.im + m0.im * v.re;
            ar[1][e] += m1.re * v.re - m1.im * v.im;
            ai[1][e] += m1.re * v.im + m1.im * v.re;
        }
    }
}

template <typename T, bool LOWER>
__global__ void __launch_bounds__(SubstTile<T>::THREADS, 1) block_subst_kernel(const Cx<T> *A, int64_t ld, int n,
                                                                           const Cx<double> *Dinv, double2 *X, int R,
                                                                           int r0, int *counter, int *flags,
                                                                           int epoch, int *status,
                                                                           unsigned spin_limit) {
    using C = T;
    using ST = SubstTile<T>;
    constexpr int LP = ST::LP, XP = ST::XP, NG = ST::NG;
    constexpr int CH = 16 / sizeof(Cx<T>);  // complex entries per 16-byte chunk
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Cx<C> *base = reinterpret_cast<Cx<C> *>(smem_raw);
    __shared__ int s_blk;
    const int nblk = (n + SB - 1) / SB;
    // persistent: a CTA claims the next block when it has released its last one
    for (;;) {
    if (threadIdx.x == 0) s_blk = atomicAdd(counter, 1);
    __syncthreads();
    const int claim = s_blk;
    if (claim >= nblk) return;
    const int tid = threadIdx.x, grp = tid >> 7, gt = tid & 127;
    Cx<C> *Lg = base + (size_t)grp * ST::GROUP;  // this group's factor tile [SB][LP]
    Cx<C> *Xg = Lg + SB * LP;                    // this group's X block [SRC][XP]
    const int b = LOWER ? claim : nblk - 1 - claim;
    const int rb = b * SB, rows = min(SB, n - rb);
    const int rc = min(SRC, R - r0);
    const int rp = gt >> 2, cg = gt & 3;  // rows rp, rp + 32; columns 4 cg .. 4 cg + 3
    // the factor tile of block row b, block column j, into dst (cp.async)
    auto issue_tile = [&](int j, Cx<C> *dst) {
        const int cj = j * SB, cols = min(SB, n - cj);
        for (int i = gt; i < SB * (SB / CH); i += 128) {
            const int a = i / (SB / CH), q = (i % (SB / CH)) * CH;
            const int valid = (a < rows) ? max(0, min(CH, cols - q)) : 0;
            const Cx<T> *src = valid > 0 ? A + (int64_t)(rb + a) * ld + cj + q : A;
            cp_async16(dst + a * LP + q, src, valid * (int)sizeof(Cx<T>));
        }
        cp_async_commit();
    };
    // X_j (FP64, columns r0 .. r0 + rc) into dst in the compute type
    auto load_x = [&](int j, Cx<C> *dst) {
        const int cj = j * SB, cols = min(SB, n - cj);
        for (int i = gt; i < SB * SRC; i += 128) {
            const int q = i / SB, a = i % SB;  // consecutive threads: consecutive rows of one column
            const double2 v = (a < cols && q < rc) ? __ldcg(&X[(size_t)(r0 + q) * n + cj + a]) : make_double2(0, 0);
            dst[q * XP + a] = Cx<C>{(C)v.x, (C)v.y};
        }
    };
    // an FP64 64 x 64 block (D_b^-1 or H_b) into dst in the compute type
    auto load_block = [&](const Cx<double> *src, Cx<C> *dst) {
        for (int i = gt; i < SB * SB; i += 128) {
            const Cx<double> v = src[i];
            dst[(i / SB) * LP + i % SB] = Cx<C>{(C)v.re, (C)v.im};
        }
    };
    C ar[2][4], ai[2][4];
#pragma unroll
    for (int h = 0; h < 2; ++h)
#pragma unroll
        for (int e = 0; e < 4; ++e) ar[h][e] = ai[h][e] = C(0);
    // every finished block at distance >= 3, shared round-robin by the groups
    const int nsteps = claim > 2 ? claim - 2 : 0;
    for (int step = grp; step < nsteps; step += NG) {
        const int j = LOWER ? step : nblk - 1 - step;
        issue_tile(j, Lg);
        if (gt == 0) wait_flag(flags + j, epoch, status, spin_limit);
        group_bar(grp);
        load_x(j, Xg);
        cp_async_wait_all();
        group_bar(grp);
        subst_product<C, LP, XP>(Lg, Xg, rp, cg, ar, ai);
        group_bar(grp);
    }
    // the groups' partial sums meet in shared memory (each in its own X block)
#pragma unroll
    for (int h = 0; h < 2; ++h)
#pragma unroll
        for (int e = 0; e < 4; ++e) Xg[(4 * cg + e) * XP + rp + 32 * h] = Cx<C>{ar[h][e], ai[h][e]};
    __syncthreads();

    // tail, the whole CTA.  Thread tid owns rows tr, tr + 32 and columns tc,
    // tc + 1 of the 64 x 16 block; with 512 threads the 64-term sums are split
    // between the two lanes of a pair (even and odd terms, so that the pair's
    // loads fall on distinct banks) and combined by one shuffle.
    constexpr int THREADS = ST::THREADS, QS = THREADS / 256;  // lanes per 2 x 2 block
    const int tile = tid / QS, qh = tid % QS;
    const int tr = tile >> 3, tc = (tile & 7) * 2;
    Cx<C> *T0 = base, *T1 = base + ST::GROUP;  // groups 0 and 1's tiles
    // H^(1)_b: group 2's tile when there is one (loaded with D and H^(2)),
    // else group 0's after the D product
    Cx<C> *TH1 = NG >= 3 ? base + 2 * ST::GROUP : T0;
    Cx<C> *X0 = base + SB * LP;                // group 0's X block
    auto load_block_all = [&](const Cx<double> *src, Cx<C> *dst) {
        for (int i = tid; i < SB * SB; i += THREADS) {
            const Cx<double> v = src[i];
            dst[(i / SB) * LP + i % SB] = Cx<C>{(C)v.re, (C)v.im};
        }
    };
    auto load_x_all = [&](int j) {
        const int cj = j * SB, cols = min(SB, n - cj);
        for (int i = tid; i < SB * SRC; i += THREADS) {
            const int q = i / SB, a = i % SB;
            const double2 v = (a < cols && q < rc) ? __ldcg(&X[(size_t)(r0 + q) * n + cj + a]) : make_double2(0, 0);
            X0[q * XP + a] = Cx<C>{(C)v.x, (C)v.y};
        }
    };
    // o[h][e] = M[tr + 32 h, :] X0[:, tc + e]
    auto tail_product = [&](const Cx<C> *M, C (&orr)[2][2], C (&oi)[2][2]) {
#pragma unroll
        for (int h = 0; h < 2; ++h)
#pragma unroll
            for (int e = 0; e < 2; ++e) orr[h][e] = oi[h][e] = C(0);
#pragma unroll 8
        for (int i = 0; i < SB / QS; ++i) {
            const int q = QS * i + qh;
            const Cx<C> m0 = M[tr * LP + q], m1 = M[(tr + 32) * LP + q];
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                const Cx<C> v = X0[(tc + e) * XP + q];
                orr[0][e] += m0.re * v.re - m0.im * v.im;
                oi[0][e] += m0.re * v.im + m0.im * v.re;
                orr[1][e] += m1.re * v.re - m1.im * v.im;
                oi[1][e] += m1.re * v.im + m1.im * v.re;
            }
        }
        if (QS == 2) {
#pragma unroll
            for (int h = 0; h < 2; ++h)
#pragma unroll
                for (int e = 0; e < 2; ++e) {
                    orr[h][e] += __shfl_xor_sync(0xffffffffu, orr[h][e], 1);
                    oi[h][e] += __shfl_xor_sync(0xffffffffu, oi[h][e], 1);
                }
        }
    };
    const Cx<double> *Di = Dinv + ((size_t)(LOWER ? 0 : 1) * nblk + b) * SB * SB;
    const Cx<double> *H1 = Dinv + ((size_t)(LOWER ? 2 : 3) * nblk + b) * SB * SB;
    const Cx<double> *H2 = Dinv + ((size_t)(LOWER ? 4 : 5) * nblk + b) * SB * SB;
    // B_b - sum of the partials
    C vr[2][2], vi[2][2];
#pragma unroll
    for (int h = 0; h < 2; ++h)
#pragma unroll
        for (int e = 0; e < 2; ++e) {
            const int r = tr + 32 * h, cc = tc + e;
            C sr = C(0), si = C(0);
#pragma unroll
            for (int g = 0; g < NG; ++g) {
                const Cx<C> v = base[(size_t)g * ST::GROUP + SB * LP + cc * XP + r];
                sr += v.re;
                si += v.im;
            }
            double2 v = make_double2(0, 0);
            if (r < rows && cc < rc) v = X[(size_t)(r0 + cc) * n + rb + r];
            vr[h][e] = (C)v.x - sr;
            vi[h][e] = (C)v.y - si;
        }
    __syncthreads();  // partials read: the groups' buffers are free
    if (qh == 0)
#pragma unroll
        for (int h = 0; h < 2; ++h)
#pragma unroll
            for (int e = 0; e < 2; ++e) X0[(tc + e) * XP + tr + 32 * h] = Cx<C>{vr[h][e], vi[h][e]};
    load_block_all(Di, T0);
    if (claim >= 2) load_block_all(H2, T1);
    if (NG >= 3 && claim >= 1) load_block_all(H1, TH1);
    __syncthreads();
    // Z_b = D_b^-1 (B_b - sum)
    C zr[2][2], zi[2][2], hr[2][2], hi[2][2];
    tail_product(T0, zr, zi);
    __syncthreads();  // T0 and X0 free
    if (NG < 3 && claim >= 1) load_block_all(H1, TH1);  // overlaps the waits below
    auto subtract = [&]() {
#pragma unroll
        for (int h = 0; h < 2; ++h)
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                zr[h][e] -= hr[h][e];
                zi[h][e] -= hi[h][e];
            }
    };
    if (claim >= 2) {
        // Z_b -= H^(2)_b X_{b-+2}
        if (tid == 0) wait_flag(flags + (LOWER ? b - 2 : b + 2), epoch, status, spin_limit);
        __syncthreads();
        load_x_all(LOWER ? b - 2 : b + 2);
        __syncthreads();
        tail_product(T1, hr, hi);
        subtract();
        __syncthreads();  // X0 free
    }
    if (claim >= 1) {
        // X_b = Z_b - H^(1)_b X_{b-+1}
        if (tid == 0) wait_flag(flags + (LOWER ? b - 1 : b + 1), epoch, status, spin_limit);
        __syncthreads();
        load_x_all(LOWER ? b - 1 : b + 1);
        __syncthreads();
        tail_product(TH1, hr, hi);
        subtract();
    }
    {  // lane qh of a pair stores row tr + 32 qh (with one lane per block, both rows)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            if (QS == 2 && h != qh) continue;
            const int r = tr + 32 * h;
#pragma unroll
            for (int e = 0; e < 2; ++e)
                if (r < rows && tc + e < rc)
                    X[(size_t)(r0 + tc + e) * n + rb + r] = make_double2(zr[h][e], zi[h][e]);
        }
    }
    // the CTA barrier orders every thread's stores before thread 0's release
    // (release is cumulative), and consumers acquire the flag before a barrier
    // and their loads
    __syncthreads();
    if (tid == 0) asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(flags + b), "r"(epoch) : "memory");
    }
}

// Persistent CTAs of a block substitution: half the SMs.  A CTA holds about 58 K
// registers, so each one keeps its SM from every other kernel while the chain
// of blocks waits on its flags; at N = 10,242 one triangle takes the same time
// on 74 CTAs as on 148 (2.00 against 2.02 ms for the solve's two), 2.26 ms on 48,
// and the six-lane sweep's best of 8 runs read 18.7-19.1 freq-solves/s with 74
// against 18.3 with 148.
#define SUBST_CTAS_CAP(c) (std::max(1, (c)->sm_count / 2))
// CTAs of a substitution launch: every block's folded-in sum must be under
// way well before the chain reaches it, but a CTA spinning on a flag holds its
// SM, which the other lanes of a sweep could use
static int subst_grid(const beat_b200_ctx *c, int nblk) { return std::min(nblk, SUBST_CTAS_CAP(c)); }

template <typename T> static void diag_inverses(beat_b200_ctx *c) {
    Workspace &w = c->ws;
    const int n = c->V, nblk = (n + SB - 1) / SB;
    w.dinv.alloc(sizeof(Cx<double>) * 6 * (size_t)nblk * SB * SB);  // D (L, U), H^(1) (L, U), H^(2) (L, U)
    const size_t smem = 2 * sizeof(Cx<double>) * SB * SBP;
    BB_CUDA(cudaFuncSetAttribute(diag_inverse_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    diag_inverse_kernel<T><<<dim3(nblk, 2), SB, smem, c->stream>>>(w.A.as<Cx<T>>(), w.ld, n, w.dinv.as<Cx<double>>());
    BB_CUDA(cudaFuncSetAttribute(offdiag_product_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    offdiag_product_kernel<T><<<dim3(nblk, 4), 256, smem, c->stream>>>(w.A.as<Cx<T>>(), w.ld, n,
                                                                     w.dinv.as<Cx<double>>());
    BB_CUDA(cudaGetLastError());
}

template <typename T> static void lu_solve_t(beat_b200_ctx *c, int R, const double *in, double *out) {
    Workspace &w = c->ws;
    const int n = c->V;
    const Cx<T> *A = w.A.as<Cx<T>>();
    double2 *X = reinterpret_cast<double2 *>(out);
    const int nblk = (n + SB - 1) / SB;
    // counters: [0] claim counter, then nblk flags
    w.small_solve.alloc(sizeof(int) * (size_t)(nblk + 64));
    int *counter = w.small_solve.as<int>();
    int *flags = counter + 32;
    if (w.solve_epoch == 0) BB_CUDA(cudaMemsetAsync(flags, 0, sizeof(int) * nblk, c->stream));
    const size_t smem = SubstTile<T>::smem();
    BB_CUDA(cudaFuncSetAttribute(block_subst_kernel<T, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    BB_CUDA(cudaFuncSetAttribute(block_subst_kernel<T, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    permute_rows_kernel<<<(n + 255) / 256, 256, 0, c->stream>>>(reinterpret_cast<const double2 *>(in), X,
                                                                w.perm.as<int>(), n, R);
    const Cx<double> *Dinv = w.dinv.as<Cx<double>>();
    for (int r0 = 0; r0 < R; r0 += SRC) {
        for (int pass = 0; pass < 2; ++pass) {
            const int epoch = ++w.solve_epoch;
            BB_CUDA(cudaMemsetAsync(counter, 0, sizeof(int), c->stream));
            if (pass == 0)
                block_subst_kernel<T, true><<<subst_grid(c, nblk), SubstTile<T>::THREADS, smem, c->stream>>>(
                    A, w.ld, n, Dinv, X, R, r0, counter, flags, epoch, c->status.as<int>(), 1u << 22);
            else
                block_subst_kernel<T, false><<<subst_grid(c, nblk), SubstTile<T>::THREADS, smem, c->stream>>>(
                    A, w.ld, n, Dinv, X, R, r0, counter, flags, epoch, c->status.as<int>(), 1u << 22);
        }
    }
    BB_CUDA(cudaGetLastError());
}

static void lu_factor_eager(beat_b200_ctx *c, int precision, int nb, int split_terms) {
    if (precision == BEAT_B200_FP64) {
        lu_factor_t<double>(c, nb, split_terms);
        diag_inverses<double>(c);
    } else {
        lu_factor_t<float>(c, nb, split_terms);
        diag_inverses<float>(c);
    }
}

void lu_graph_release(beat_b200_ctx *c) {
    if (c->lu_graph) cudaGraphExecDestroy(c->lu_graph);
    c->lu_graph = nullptr;
    c->lu_graph_state = 0;
}

// The factorisation is about 1,300 launches on two streams whose arguments
// depend only on the sizes, the options and the workspace's buffers.  The
// first factorisation with a given key runs eagerly (allocating what it
// needs) and is then captured, without running, into a CUDA graph that later
// factorisations with the same key replay.  The graph keeps each kernel's
// stream priority (the look-ahead's side stream stays below the panels').  A
// capture that fails leaves the eager path in place for that key.
static void lu_key(const beat_b200_ctx *c, int precision, int nb, int split_terms, uint64_t (&key)[12]) {
    const Workspace &w = c->ws;
    const uint64_t k[12] = {(uint64_t)precision, (uint64_t)nb, (uint64_t)split_terms, (uint64_t)c->V,
                            (uint64_t)w.ld, (uint64_t)(uintptr_t)w.A.p, (uint64_t)(uintptr_t)w.ipiv.p,
                            (uint64_t)(uintptr_t)w.perm.p, (uint64_t)(uintptr_t)w.panel_scratch.p,
                            (uint64_t)(uintptr_t)w.stage.p, (uint64_t)(uintptr_t)w.dinv.p,
                            (uint64_t)(uintptr_t)c->status.p};
    std::memcpy(key, k, sizeof(k));
}

void lu_factor(beat_b200_ctx *c, int precision, int nb, int split_terms) {
    uint64_t key[12];
    lu_key(c, precision, nb, split_terms, key);
    const bool same = std::memcmp(key, c->lu_graph_key, sizeof(key)) == 0;
    if (same && c->lu_graph_state == 2) {
        BB_CUDA(cudaGraphLaunch(c->lu_graph, c->stream));
        return;
    }
    if (same && c->lu_graph_state == 3) {
        lu_factor_eager(c, precision, nb, split_terms);
        return;
    }
    lu_graph_release(c);
    lu_factor_eager(c, precision, nb, split_terms);
    // the buffers exist now: capture the same sequence for the next time
    lu_key(c, precision, nb, split_terms, key);
    std::memcpy(c->lu_graph_key, key, sizeof(key));
    c->lu_graph_state = 3;
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return;
    }
    try {
        lu_factor_eager(c, precision, nb, split_terms);
    } catch (...) {
        cudaStreamEndCapture(c->stream, &g);
        if (g) cudaGraphDestroy(g);
        cudaGetLastError();
        return;  // the eager factorisation above stands; this key stays eager
    }
    e = cudaStreamEndCapture(c->stream, &g);
    if (e == cudaSuccess && g) e = cudaGraphInstantiateWithFlags(&c->lu_graph, g, cudaGraphInstantiateFlagUseNodePriority);
    if (g) cudaGraphDestroy(g);
    // upload now, so that the first replay does not pay for it
    if (e == cudaSuccess && c->lu_graph) e = cudaGraphUpload(c->lu_graph, c->stream);
    if (e == cudaSuccess && c->lu_graph) {
        c->lu_graph_state = 2;
    } else {
        if (c->lu_graph) cudaGraphExecDestroy(c->lu_graph);
        c->lu_graph = nullptr;
        cudaGetLastError();
    }
}

void lu_solve_fp64(beat_b200_ctx *c, int R, double *x_dev) {
    // x_dev holds b on entry (N x R), solution on exit; uses ws.x as scratch
    BB_CUDA(cudaMemcpyAsync(c->ws.x.p, x_dev, (size_t)c->V * R * 16, cudaMemcpyDeviceToDevice, c->stream));
    lu_solve_t<double>(c, R, c->ws.x.as<double>(), x_dev);
}

void lu_precond_fp32(beat_b200_ctx *c, int R, const double *in, double *out) {
    lu_solve_t<float>(c, R, in, out);
}

// The same permutation and block substitutions as lu_solve_t, with the claim
// counter and per-block flags in caller-provided device memory (`scratch`,
// at least nblk + 32 ints): x = (L U)^-1 P b with the context's factors.
template <typename T>
static void lu_resolve_into_t(beat_b200_ctx *c, int R, const double *b, double *x, int *scratch) {
    Workspace &w = c->ws;
    const int n = c->V;
    const Cx<T> *A = w.A.as<Cx<T>>();
    double2 *X = reinterpret_cast<double2 *>(x);
    const int nblk = (n + SB - 1) / SB;
    int *counter = scratch;
    int *flags = scratch + 32;
    BB_CUDA(cudaMemsetAsync(scratch, 0, sizeof(int) * (size_t)(nblk + 32), c->stream));
    const size_t smem = SubstTile<T>::smem();
    BB_CUDA(cudaFuncSetAttribute(block_subst_kernel<T, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    BB_CUDA(cudaFuncSetAttribute(block_subst_kernel<T, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    permute_rows_kernel<<<(n + 255) / 256, 256, 0, c->stream>>>(reinterpret_cast<const double2 *>(b), X,
                                                                w.perm.as<int>(), n, R);
    const Cx<double> *Dinv = w.dinv.as<Cx<double>>();
    int epoch = 0;
    for (int r0 = 0; r0 < R; r0 += SRC) {
        for (int pass = 0; pass < 2; ++pass) {
            ++epoch;
            BB_CUDA(cudaMemsetAsync(counter, 0, sizeof(int), c->stream));
            if (pass == 0)
                block_subst_kernel<T, true><<<subst_grid(c, nblk), SubstTile<T>::THREADS, smem, c->stream>>>(
                    A, w.ld, n, Dinv, X, R, r0, counter, flags, epoch, c->status.as<int>(), 1u << 22);
            else
                block_subst_kernel<T, false><<<subst_grid(c, nblk), SubstTile<T>::THREADS, smem, c->stream>>>(
                    A, w.ld, n, Dinv, X, R, r0, counter, flags, epoch, c->status.as<int>(), 1u << 22);
        }
    }
    BB_CUDA(cudaGetLastError());
}

void lu_resolve_into(beat_b200_ctx *c, int R, const double *b, double *x, int *scratch) {
    if (c->ws.precision == BEAT_B200_FP64)
        lu_resolve_into_t<double>(c, R, b, x, scratch);
    else
        lu_resolve_into_t<float>(c, R, b, x, scratch);
}

}  // namespace bb
