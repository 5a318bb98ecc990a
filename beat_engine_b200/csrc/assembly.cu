// assembly.cu -- fused Burton-Miller system assembly on sm_100a.
//
//   A = 0.5 M_p1p1 - D + eta H            (N x N, row = test vertex)
//   B = -S - eta (K' + 0.5 M_p1dp0)       (N x F, column = trial face)
//   b = B q                               (N x R, FP64)
//
// Reference (paths relative to src/beat_engine/julia_local/src/):
//   per point pair combination   BeatEngineCpuBurtonMiller.jl:53-112 (regular),
//                                :116-167 (Duffy), green BeatEngineCpuAssembly.jl:1-6
//   CUDA element-pair kernel      BeatEngineCudaRegular.jl:18-383
//   Duffy block kernel + scatter  BeatEngineCudaSingular.jl:359-588,
//                                 BeatEngineCudaBurtonMiller.jl:97-162,273-329
//   identity kernel               BeatEngineCudaBurtonMiller.jl:21-69
//   cached RHS operator  b = B Q  BeatEngineCudaBurtonMiller.jl:774-830
//
// Design (no reference counterpart): elements are sorted along a Morton curve
// and cut into tiles of consecutive elements with few distinct vertices.  One
// CTA integrates a (test tile x trial tile) block of element pairs; each
// pair's 3x3 block and 3-vector land in shared-memory accumulators indexed by
// tile-local vertex numbers, and the CTA flushes them to HBM once with
// red.global.add.  The Duffy kernel runs one warp per touching pair, lanes
// over the Duffy points, in FP64 in both precision forms.
#include <cuda_runtime.h>

#include "internal.cuh"
#include "phase.cuh"

namespace bb {

constexpr int TT = 64, VT = 80;  // test tile: faces, distinct vertices (context.cu)
constexpr int TS = 16, VS = 32;  // trial tile
constexpr int REG_S = 3 * TS;    // slot-face indices of a trial tile
constexpr int REG_INC = VS + 1 + REG_S;  // Tiling::inc_stride() of the trial tiles
constexpr int REG_THREADS = 256;

// rule tables: index 0 -> 1-point, 1 -> 3-point, 2 -> 6-point (order 4)
__constant__ double c_rw64[3][6];
__constant__ double c_rb64[3][6][3];
__constant__ float c_rw32[3][6];
__constant__ float c_rb32[3][6][3];
__constant__ float2 c_rb32x2[3][6][3];  // (b, b): the packed-pair operand of the same basis value

template <typename T> struct RuleRef;
template <> struct RuleRef<double> {
    static __device__ __forceinline__ double w(int r, int q) { return c_rw64[r][q]; }
    static __device__ __forceinline__ double b(int r, int q, int a) { return c_rb64[r][q][a]; }
};
template <> struct RuleRef<float> {
    static __device__ __forceinline__ float w(int r, int q) { return c_rw32[r][q]; }
    static __device__ __forceinline__ float b(int r, int q, int a) { return c_rb32[r][q][a]; }
};

void upload_rule_tables(const std::vector<double> &pts, const std::vector<double> &w, int Q) {
    double w64[3][6] = {}, b64[3][6][3] = {};
    float w32[3][6] = {}, b32[3][6][3] = {};
    BB_CUDA(cudaMemcpyFromSymbol(w64, c_rw64, sizeof(w64)));
    BB_CUDA(cudaMemcpyFromSymbol(b64, c_rb64, sizeof(b64)));
    const int r = Q == 1 ? 0 : Q == 3 ? 1 : 2;
    for (int q = 0; q < Q; ++q) {
        w64[r][q] = w[q];
        b64[r][q][0] = 1.0 - pts[2 * q] - pts[2 * q + 1];
        b64[r][q][1] = pts[2 * q];
        b64[r][q][2] = pts[2 * q + 1];
    }
    for (int i = 0; i < 3; ++i)
        for (int q = 0; q < 6; ++q) {
            w32[i][q] = (float)w64[i][q];
            for (int a = 0; a < 3; ++a) b32[i][q][a] = (float)b64[i][q][a];
        }
    BB_CUDA(cudaMemcpyToSymbol(c_rw64, w64, sizeof(w64)));
    BB_CUDA(cudaMemcpyToSymbol(c_rb64, b64, sizeof(b64)));
    BB_CUDA(cudaMemcpyToSymbol(c_rw32, w32, sizeof(w32)));
    BB_CUDA(cudaMemcpyToSymbol(c_rb32, b32, sizeof(b32)));
    float2 b32x2[3][6][3];
    for (int i = 0; i < 3; ++i)
        for (int q = 0; q < 6; ++q)
            for (int a = 0; a < 3; ++a) b32x2[i][q][a] = make_float2(b32[i][q][a], b32[i][q][a]);
    BB_CUDA(cudaMemcpyToSymbol(c_rb32x2, b32x2, sizeof(b32x2)));
}

__device__ __forceinline__ void sincos_t(double x, double *s, double *c) { sincos_cw(x, s, c); }
// FP32 phase: reduced to [-pi, pi] by a two-part 2 pi (6.2831854820251465 is
// 2 pi rounded to float, -1.7484555e-7 the remainder), then the hardware
// approximation, whose absolute error on [-pi, pi] (about 2^-21.4) is below
// the rounding error of the FP32 phase k r itself.
__device__ __forceinline__ void sincos_t(float x, float *s, float *c) {
    const float n = rintf(x * 0.15915493667125702f);
    float r = fmaf(-n, 6.2831854820251465f, x);
    r = fmaf(-n, -1.7484555314695172e-07f, r);
    __sincosf(r, s, c);
}
// The same phase given in revolutions, t = x / (2 pi): t - rint(t) is exact,
// so the reduction to [-1/2, 1/2] is one rounding and one subtraction.  The
// multiply back to radians adds at most about 2^-22 absolute on [-pi, pi],
// below the hardware approximation's own error there (about 2^-21.4); for
// large phases the rounding of t itself (relative 2^-24) dominates.
__device__ __forceinline__ void sincos_rev(float t, float *s, float *c) {
    __sincosf((t - rintf(t)) * 6.2831854820251465f, s, c);
}
__device__ __forceinline__ double rsqrt_t(double x) { return rsqrt(x); }
__device__ __forceinline__ float rsqrt_t(float x) { return rsqrtf(x); }

__device__ __forceinline__ void red_add(double *p, double v) { atomicAdd(p, v); }
__device__ __forceinline__ void red_add(float *p, float v) { atomicAdd(p, v); }
// Packed FP32 pairs (sm_100 f32x2 arithmetic): two lanes of one instruction,
// (re, im) of a complex value or one value twice.
using F2 = unsigned long long;
__device__ __forceinline__ F2 pk2(float lo, float hi) {
    F2 r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
    return r;
}
__device__ __forceinline__ void up2(F2 v, float &lo, float &hi) {
    asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}
__device__ __forceinline__ F2 fma2(F2 a, F2 b, F2 c) {
    F2 d;
    asm("fma.rn.ftz.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}
__device__ __forceinline__ F2 mul2(F2 a, F2 b) {
    F2 d;
    asm("mul.rn.ftz.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ F2 add2(F2 a, F2 b) {
    F2 d;
    asm("add.rn.ftz.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ F2 rule_b2(int r, int q, int a) {
    return *reinterpret_cast<const F2 *>(&c_rb32x2[r][q][a]);
}

// Adds v[i] to base[off[i]] for every i, atomically.  Shared-memory float
// adds are compare-and-swap loops, each a dependent load -> add -> swap
// chain; here the loads, then the swaps, of all N adds are in flight
// together, and only a swap that lost to another warp's add is redone as an
// ordinary atomic add.  (ABA is harmless: the swap writes old + v over old.)
template <int N>
__device__ __forceinline__ void batch_add(float *base, const int (&off)[N], const float (&v)[N]) {
    static_assert(N <= 32, "one failure bit per add");
    unsigned old[N];
#pragma unroll
    for (int i = 0; i < N; ++i) old[i] = *reinterpret_cast<volatile unsigned *>(base + off[i]);
    unsigned fail = 0;
#pragma unroll
    for (int i = 0; i < N; ++i) {
        const unsigned got =
            atomicCAS(reinterpret_cast<unsigned *>(base + off[i]), old[i], __float_as_uint(__uint_as_float(old[i]) + v[i]));
        fail |= (got != old[i] ? 1u : 0u) << i;
    }
    if (fail) {
#pragma unroll
        for (int i = 0; i < N; ++i)
            if (fail >> i & 1u) atomicAdd(base + off[i], v[i]);
    }
}
// the same for double words (64-bit compare-and-swap)
template <int N>
__device__ __forceinline__ void batch_add(double *base, const int (&off)[N], const double (&v)[N]) {
    static_assert(N <= 32, "one failure bit per add");
    using U = unsigned long long;
    U old[N];
#pragma unroll
    for (int i = 0; i < N; ++i) old[i] = *reinterpret_cast<volatile U *>(base + off[i]);
    unsigned fail = 0;
#pragma unroll
    for (int i = 0; i < N; ++i) {
        const double sum = __longlong_as_double((long long)old[i]) + v[i];
        const U got = atomicCAS(reinterpret_cast<U *>(base + off[i]), old[i], (U)__double_as_longlong(sum));
        fail |= (got != old[i] ? 1u : 0u) << i;
    }
    if (fail) {
#pragma unroll
        for (int i = 0; i < N; ++i)
            if (fail >> i & 1u) atomicAdd(base + off[i], v[i]);
    }
}
// 4-byte global -> shared copy through the asynchronous copy unit: a CTA's
// tile arrays are all in flight at once and waited for together
__device__ __forceinline__ void cp_async4(void *smem, const void *gmem) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"((unsigned)__cvta_generic_to_shared(smem)), "l"(gmem)
                 : "memory");
}
// the same for one 4- or 8-byte element
template <typename E> __device__ __forceinline__ void cp_async_el(E *smem, const E *gmem) {
    static_assert(sizeof(E) == 4 || sizeof(E) == 8, "cp.async element of 4 or 8 bytes");
    if constexpr (sizeof(E) == 4)
        cp_async4(smem, gmem);
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"((unsigned)__cvta_generic_to_shared(smem)),
                     "l"(gmem)
                     : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
    asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
}

__device__ __forceinline__ void red_add_cx(Cx<double> *p, double re, double im) {
    atomicAdd(&p->re, re);
    atomicAdd(&p->im, im);
}
__device__ __forceinline__ void red_add_cx(Cx<float> *p, float re, float im) {
    atomicAdd(reinterpret_cast<float2 *>(p), make_float2(re, im));
}

// Where the right-hand-side operator goes.  Cached (B set): the N x F
// mapping B, b = B q formed afterwards by one tall product.  Matrix-free (B
// null): b = B q directly for the R columns of q, so no N x F array exists
// (exterior_rhs_policy.jl restated, one pass for every column where the
// reference's matrix_free path integrates once per column).
template <typename T> struct RhsOut {
    Cx<T> *B = nullptr;             // N x F, row-major
    const Cx<double> *q = nullptr;  // F x R, column-major (matrix-free)
    Cx<double> *b = nullptr;        // N x R, column-major (matrix-free)
    int F = 0, N = 0, R = 0;
};

template <typename T>
__device__ __forceinline__ void rhs_add(const RhsOut<T> &o, int row, int face, T re, T im) {
    if (o.B) {
        red_add_cx(&o.B[(int64_t)row * o.F + face], re, im);
        return;
    }
    for (int r = 0; r < o.R; ++r) {
        const Cx<double> qq = o.q[(size_t)r * o.F + face];
        red_add_cx(&o.b[(size_t)r * o.N + row], (double)re * qq.re - (double)im * qq.im,
                   (double)re * qq.im + (double)im * qq.re);
    }
}

// columns of q per staged chunk in the matrix-free tile epilogues
constexpr int MF_RC = 8;

template <typename T> struct RegArgs {
    const T *qpts;      // by position: F x Q x 3
    const T *normal;    // F x 3
    const T *curl;      // F x 9
    const T *area;      // F
    const T *plane = nullptr;  // F: plane offset . normal (FP32 symmetric kernel)
    const int *gvert;   // F x 3
    const int *face_id; // F
    const int *t_fstart, *t_vstart, *t_verts, *t_local;
    const int *s_fstart, *s_vstart, *s_verts;
    const int *t_inc = nullptr, *s_inc = nullptr;  // per-tile vertex incidences (Tiling::incidence)
    Cx<T> *A;
    Cx<T> *B;
    int64_t ld;         // row stride of A (complex entries)
    int F;
    T k, eta, k2;
    // image pass: trial elements reflected by these signs (curls also by det),
    // touching pairs kept (their Duffy delta comes from image_delta_kernel)
    int image = 0;
    T xs[3] = {T(1), T(1), T(1)};
    T xdet = T(1);
    // matrix-free right-hand sides (B null): b (N x R) += B-tile x q (F x R)
    const Cx<double> *q = nullptr;
    Cx<double> *b = nullptr;
    int N = 0, R = 0;
};

// Element-pair kernel.  grid = (trial tiles, test tiles), 256 threads.
template <typename T, int Q>
__global__ void __launch_bounds__(REG_THREADS, sizeof(T) == 4 ? 3 : 2) regular_pairs_kernel(RegArgs<T> g) {
    constexpr int RI = Q == 1 ? 0 : Q == 3 ? 1 : 2;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    // test vertex x trial vertex *slot* (s = b * TS + trial face): lanes that
    // share a test vertex never add to one word together (see the symmetric
    // kernel below); folded onto the trial tile's vertices at the flush
    Cx<T> *sC = reinterpret_cast<Cx<T> *>(smem_raw);  // VT x REG_S
    Cx<T> *sB = sC + VT * REG_S;                      // VT x TS
    T *tq = reinterpret_cast<T *>(sB + VT * TS);      // TT x Q x 3
    T *tn = tq + TT * Q * 3;                          // TT x 3
    T *tc = tn + TT * 3;                              // TT x 9
    T *ta = tc + TT * 9;                              // TT
    T *sq = ta + TT;                                  // (Q*3) x TS (trial, transposed)
    T *sn = sq + TS * Q * 3;                          // 3 x TS
    T *sc = sn + TS * 3;                              // 9 x TS
    T *sa = sc + TS * 9;                              // TS
    T *tpl = sa + TS;                                 // TT: plane offset x . n of each test face
    T *spl = tpl + TT;                                // TS: plane offset y . n of each trial face
    int *tgv = reinterpret_cast<int *>(spl + TS);     // TT x 3
    int *tlv = tgv + TT * 3;                          // TT x 3
    int *sgv = tlv + TT * 3;                          // 3 x TS
    int *inc_start = sgv + TS * 3;                    // VS + 1: trial vertex -> its slot-face indices
    int *inc_list = inc_start + VS + 1;               // REG_S

    const int tid = threadIdx.x;
    const int t0 = g.t_fstart[blockIdx.y], nt = g.t_fstart[blockIdx.y + 1] - t0;
    const int s0 = g.s_fstart[blockIdx.x], ns = g.s_fstart[blockIdx.x + 1] - s0;
    const int tv0 = g.t_vstart[blockIdx.y], nvt = g.t_vstart[blockIdx.y + 1] - tv0;
    const int sv0 = g.s_vstart[blockIdx.x], nvs = g.s_vstart[blockIdx.x + 1] - sv0;

    for (int i = tid; i < VT * REG_S; i += REG_THREADS) sC[i] = Cx<T>{T(0), T(0)};
    for (int i = tid; i < VT * TS; i += REG_THREADS) sB[i] = Cx<T>{T(0), T(0)};
    // the tile arrays: every copy in flight at once, one wait
    for (int i = tid; i < nt * Q * 3; i += REG_THREADS) cp_async_el(&tq[i], &g.qpts[(size_t)t0 * Q * 3 + i]);
    for (int i = tid; i < nt * 3; i += REG_THREADS) {
        cp_async_el(&tn[i], &g.normal[(size_t)t0 * 3 + i]);
        cp_async_el(&tgv[i], &g.gvert[(size_t)t0 * 3 + i]);
        cp_async_el(&tlv[i], &g.t_local[(size_t)t0 * 3 + i]);
    }
    for (int i = tid; i < nt * 9; i += REG_THREADS) cp_async_el(&tc[i], &g.curl[(size_t)t0 * 9 + i]);
    for (int i = tid; i < nt; i += REG_THREADS) cp_async_el(&ta[i], &g.area[t0 + i]);
    for (int i = tid; i < ns * Q * 3; i += REG_THREADS) {
        int s = i / (Q * 3), j = i % (Q * 3);
        cp_async_el(&sq[j * TS + s], &g.qpts[(size_t)s0 * Q * 3 + i]);
    }
    for (int i = tid; i < ns * 3; i += REG_THREADS) {
        int s = i / 3, j = i % 3;
        cp_async_el(&sn[j * TS + s], &g.normal[(size_t)s0 * 3 + i]);
        cp_async_el(&sgv[j * TS + s], &g.gvert[(size_t)s0 * 3 + i]);
    }
    for (int i = tid; i < ns * 9; i += REG_THREADS) {
        int s = i / 9, j = i % 9;
        cp_async_el(&sc[j * TS + s], &g.curl[(size_t)s0 * 9 + i]);
    }
    for (int i = tid; i < ns; i += REG_THREADS) cp_async_el(&sa[i], &g.area[s0 + i]);
    for (int i = tid; i < REG_INC; i += REG_THREADS)
        cp_async_el(&inc_start[i], &g.s_inc[(size_t)blockIdx.x * REG_INC + i]);
    cp_async_wait_all();
    __syncthreads();
    // every point y of a flat face has the same y . n
    for (int i = tid; i < nt; i += REG_THREADS)
        tpl[i] = tq[i * Q * 3] * tn[3 * i] + tq[i * Q * 3 + 1] * tn[3 * i + 1] + tq[i * Q * 3 + 2] * tn[3 * i + 2];
    if (tid < ns) {  // one thread per trial face: its image reflection, then its plane offset
        if (g.image) {
            // an image pass reflects the trial tile (signs xs, curls also by det)
            for (int j = 0; j < Q * 3; ++j) sq[j * TS + tid] *= g.xs[j % 3];
            for (int j = 0; j < 3; ++j) sn[j * TS + tid] *= g.xs[j];
            for (int j = 0; j < 9; ++j) sc[j * TS + tid] *= g.xdet * g.xs[j % 3];
        }
        spl[tid] = sq[tid] * sn[tid] + sq[TS + tid] * sn[TS + tid] + sq[2 * TS + tid] * sn[2 * TS + tid];
    }
    __syncthreads();

    const T k = g.k, eta = g.eta;
    const T inv4pi = T(0.07957747154594767);  // 1 / (4 pi)
    const int npairs = nt * TS;
    for (int p = tid; p < npairs; p += REG_THREADS) {
        const int tl = p / TS, sl = p % TS;
        if (sl >= ns) continue;
        const int ga = tgv[3 * tl], gb = tgv[3 * tl + 1], gc = tgv[3 * tl + 2];
        const int ha = sgv[sl], hb = sgv[TS + sl], hc = sgv[2 * TS + sl];
        if (!g.image && (ga == ha || ga == hb || ga == hc || gb == ha || gb == hb || gb == hc || gc == ha ||
                         gc == hb || gc == hc))
            continue;  // touching pair: the Duffy kernel integrates it
        const T ntx = tn[3 * tl], nty = tn[3 * tl + 1], ntz = tn[3 * tl + 2];
        const T nsx = sn[sl], nsy = sn[TS + sl], nsz = sn[2 * TS + sl];
        const T k2n = eta * g.k2 * (ntx * nsx + nty * nsy + ntz * nsz);
        // with r = y - x:  r . n_s = ds - x . n_s  and  -r . n_t = dt - y . n_t
        const T ds = spl[sl], dt = tpl[tl];
        T L[9][2], Rv[3][2], cr = T(0), ci = T(0);
#pragma unroll
        for (int i = 0; i < 9; ++i) L[i][0] = L[i][1] = T(0);
#pragma unroll
        for (int i = 0; i < 3; ++i) Rv[i][0] = Rv[i][1] = T(0);
#pragma unroll 1
        for (int qt = 0; qt < Q; ++qt) {
            const T x0 = tq[(tl * Q + qt) * 3], x1 = tq[(tl * Q + qt) * 3 + 1], x2 = tq[(tl * Q + qt) * 3 + 2];
            const T wt = RuleRef<T>::w(RI, qt) * inv4pi;
            const T xns = ds - (x0 * nsx + x1 * nsy + x2 * nsz);
            T S0r = 0, S0i = 0, S1r = 0, S1i = 0, S2r = 0, S2i = 0, Gr = 0, Gi = 0, Wr = 0, Wi = 0;
#pragma unroll
            for (int qs = 0; qs < Q; ++qs) {
                const T y0 = sq[(qs * 3) * TS + sl], y1 = sq[(qs * 3 + 1) * TS + sl], y2 = sq[(qs * 3 + 2) * TS + sl];
                const T rx = y0 - x0, ry = y1 - x1, rz = y2 - x2;
                const T r2 = rx * rx + ry * ry + rz * rz;
                const T ir = rsqrt_t(r2);
                T sn_, cs_;
                sincos_t(k * (r2 * ir), &sn_, &cs_);
                const T scl = ir * (wt * RuleRef<T>::w(RI, qs));
                const T gr = cs_ * scl, gi = sn_ * scl;           // weighted green
                const T gsr = -gr * ir - gi * k;                  // weighted d green / d r
                const T gsi = gr * k - gi * ir;
                const T dns = xns * ir, dnt = (dt - (y0 * ntx + y1 * nty + y2 * ntz)) * ir;
                const T lr = k2n * gi - gsr * dns;                // -grad*dn_s - i k2n g
                const T li = -(gsi * dns + k2n * gr);
                Gr += gr;
                Gi += gi;
                Wr += dnt * gsr;
                Wi += dnt * gsi;
                const T b0 = RuleRef<T>::b(RI, qs, 0), b1 = RuleRef<T>::b(RI, qs, 1), b2 = RuleRef<T>::b(RI, qs, 2);
                S0r += b0 * lr;
                S0i += b0 * li;
                S1r += b1 * lr;
                S1i += b1 * li;
                S2r += b2 * lr;
                S2i += b2 * li;
            }
            // sum over the trial points of -g - i eta grad*dn_t
            const T Ur = -Gr + eta * Wi, Ui = -Gi - eta * Wr;
            cr += Gr;
            ci += Gi;
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                const T ba = RuleRef<T>::b(RI, qt, a);
                L[3 * a + 0][0] += ba * S0r;
                L[3 * a + 0][1] += ba * S0i;
                L[3 * a + 1][0] += ba * S1r;
                L[3 * a + 1][1] += ba * S1i;
                L[3 * a + 2][0] += ba * S2r;
                L[3 * a + 2][1] += ba * S2i;
                Rv[a][0] += ba * Ur;
                Rv[a][1] += ba * Ui;
            }
        }
        // hypersingular curl term: eta * sum(g w) * curl_t . curl_s
        const T ccr = -eta * ci, cci = eta * cr;
        const T jac = T(4) * ta[tl] * sa[sl];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const int row = tlv[3 * tl + a];
            int off[8];  // this vertex's 8 adds, in T words from sC
            T val[8];
#pragma unroll
            for (int b = 0; b < 3; ++b) {
                const T d = tc[9 * tl + 3 * a] * sc[(3 * b) * TS + sl] +
                            tc[9 * tl + 3 * a + 1] * sc[(3 * b + 1) * TS + sl] +
                            tc[9 * tl + 3 * a + 2] * sc[(3 * b + 2) * TS + sl];
                const int o = 2 * (row * REG_S + b * TS + sl);
                off[2 * b] = o;
                val[2 * b] = (L[3 * a + b][0] + d * ccr) * jac;
                off[2 * b + 1] = o + 1;
                val[2 * b + 1] = (L[3 * a + b][1] + d * cci) * jac;
            }
            off[6] = 2 * (VT * REG_S + row * TS + sl);
            val[6] = Rv[a][0] * jac;
            off[7] = off[6] + 1;
            val[7] = Rv[a][1] * jac;
            batch_add<8>(reinterpret_cast<T *>(sC), off, val);
        }
    }
    __syncthreads();
    for (int i = tid; i < nvt * nvs; i += REG_THREADS) {
        const int lt = i / nvs, ls = i % nvs;
        Cx<T> v{T(0), T(0)};
        for (int e = inc_start[ls]; e < inc_start[ls + 1]; ++e) {
            const Cx<T> c = sC[lt * REG_S + inc_list[e]];
            v.re += c.re;
            v.im += c.im;
        }
        if (v.re != T(0) || v.im != T(0))
            red_add_cx(&g.A[(int64_t)g.t_verts[tv0 + lt] * g.ld + g.s_verts[sv0 + ls]], v.re, v.im);
    }
    if (g.B) {
        for (int i = tid; i < nvt * ns; i += REG_THREADS) {
            const int lt = i / ns, sl = i % ns;
            const Cx<T> v = sB[lt * TS + sl];
            if (v.re != T(0) || v.im != T(0))
                red_add_cx(&g.B[(int64_t)g.t_verts[tv0 + lt] * g.F + g.face_id[s0 + sl]], v.re, v.im);
        }
        return;
    }
    // matrix-free: the tile's rows of b += sB (test vertices x trial faces) q,
    // q staged MF_RC columns at a time over the (now unused) geometry region
    Cx<T> *qs = reinterpret_cast<Cx<T> *>(tq);  // [TS][MF_RC]
    for (int r0 = 0; r0 < g.R; r0 += MF_RC) {
        const int rc = min(MF_RC, g.R - r0);
        __syncthreads();
        for (int i = tid; i < TS * MF_RC; i += REG_THREADS) {
            const int f = i / MF_RC, r = i % MF_RC;
            Cx<T> v{T(0), T(0)};
            if (f < ns && r < rc) {
                const Cx<double> qq = g.q[(size_t)(r0 + r) * g.F + g.face_id[s0 + f]];
                v = Cx<T>{(T)qq.re, (T)qq.im};
            }
            qs[i] = v;
        }
        __syncthreads();
        for (int i = tid; i < nvt * rc; i += REG_THREADS) {
            const int lt = i / rc, r = i % rc;
            T sr = T(0), si = T(0);
            for (int f = 0; f < ns; ++f) {
                const Cx<T> bv = sB[lt * TS + f], qv = qs[f * MF_RC + r];
                sr += bv.re * qv.re - bv.im * qv.im;
                si += bv.re * qv.im + bv.im * qv.re;
            }
            if (sr != T(0) || si != T(0))
                red_add_cx(&g.b[(size_t)(r0 + r) * g.N + g.t_verts[tv0 + lt]], (double)sr, (double)si);
        }
    }
}

template <typename T, int Q> static size_t regular_smem_bytes() {
    return sizeof(Cx<T>) * (VT * REG_S + VT * TS) + sizeof(T) * (TT * (Q * 3 + 3 + 9 + 2) + TS * (Q * 3 + 3 + 9 + 2)) +
           sizeof(int) * (TT * 6 + TS * 3 + REG_INC);
}

// ---------------------------------------------------------------------------
// Symmetric element-pair kernel (FP32 form).  G(x, y) = G(y, x), so the two
// ordered pairs (tau, sigma) and (sigma, tau) of two elements share r, the
// phase, e^{ikr}/r and dG/dr at every point pair; only the normal
// derivatives swap roles: with r = y - x,
//   order 1 (test tau at x, trial sigma at y): dn_s =  r.n_sigma / r = a,
//                                               dn_t = -r.n_tau / r   = c,
//   order 2 (test sigma at y, trial tau at x): dn_s = c, dn_t = a.
// One CTA integrates an unordered pair of square tiles (I <= J; pairs of
// elements tau < sigma inside a diagonal tile) for both orders; each order
// has its own shared-memory accumulators, flushed like the one-order kernel.
// ---------------------------------------------------------------------------
constexpr int SYM_F = 32, SYM_V = 40;  // square tile: faces, distinct vertices (context.cu)
// Accumulators.  A warp takes one tau and 32 sigma (one per lane), so the
// entries a lane adds to are keyed by sigma's vertex *slot* (s = b * SYM_F +
// sigma, the slot-face index) rather than by sigma's vertex: two lanes whose
// faces share a vertex would otherwise add to the same word in the same
// instruction, and shared-memory float atomics retry once per colliding lane.
// The slot-face entries are folded onto tile J's vertices at the flush.
//   C1 [vI][s]      order 1, test vertex of tau x trial slot of sigma
//   C2 [s][vI]      order 2, test slot of sigma x trial vertex of tau
//   B1 [vI][sigma]  order 1 right-hand side (test vertex of tau x face sigma)
//   D2 [s][tau]     order 2 right-hand side (test slot of sigma x face tau)
// Re / im planes; a warp's lanes step 1 or an odd stride through each, so
// they spread over all banks.
constexpr int SYM_S = 3 * SYM_F;                  // slot-face indices of a tile
constexpr int SYM_C2S = SYM_V + 1, SYM_BS = SYM_F + 1;
constexpr int SYM_C1 = 0;
constexpr int SYM_C2 = SYM_C1 + SYM_V * SYM_S;
constexpr int SYM_B1 = SYM_C2 + SYM_S * SYM_C2S;
constexpr int SYM_D2 = SYM_B1 + SYM_V * SYM_BS;
constexpr int SYM_ACC = SYM_D2 + SYM_S * SYM_BS;  // floats per plane

constexpr int SYM_INC = SYM_V + 1 + SYM_S;  // Tiling::inc_stride() of the square tiles

template <int Q> static size_t sym_smem_bytes() {
    return sizeof(float) * 2 * SYM_ACC + sizeof(float) * 2 * SYM_F * (Q * 3 + 3 + 9 + 2) +
           sizeof(int) * (3 * 3 * SYM_F + SYM_INC);
}

template <int Q>
__global__ void __launch_bounds__(REG_THREADS, 2) sym_pairs_kernel(RegArgs<float> g) {
    using T = float;
    constexpr int RI = Q == 1 ? 0 : Q == 3 ? 1 : 2;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *acc_re = reinterpret_cast<T *>(smem_raw), *acc_im = acc_re + SYM_ACC;
    T *xq = acc_im + SYM_ACC;                  // tile I: [tau][Q][3]
    T *xn = xq + SYM_F * Q * 3;                // [tau][3]
    T *xc = xn + SYM_F * 3;                    // [tau][9]
    T *xa = xc + SYM_F * 9;                    // [tau]
    T *xp = xa + SYM_F;                        // [tau]: plane offset x . n_tau
    T *yq = xp + SYM_F;                        // tile J, transposed: [Q * 3][sigma]
    T *yn = yq + SYM_F * Q * 3;                // [3][sigma]
    T *yc = yn + 3 * SYM_F;                    // [9][sigma]
    T *ya = yc + 9 * SYM_F;                    // [sigma]
    T *yp = ya + SYM_F;                        // [sigma]: plane offset y . n_sigma (a reflection keeps it)
    int *xgv = reinterpret_cast<int *>(yp + SYM_F);  // [tau][3] global vertex ids
    int *xlv = xgv + 3 * SYM_F;                      // [tau][3] tile-local vertex ids
    int *ygv = xlv + 3 * SYM_F;                      // [3][sigma]
    int *inc_start = ygv + 3 * SYM_F;                // [vJ + 1]: slot-face indices of tile J's vertex vJ
    int *inc_list = inc_start + SYM_V + 1;           //   are inc_list[inc_start[vJ] .. inc_start[vJ + 1])

    // unordered tile pair (I, J), I <= J, from the linear block index
    const int64_t bi = blockIdx.x;
    int J = (int)((sqrt(8.0 * (double)bi + 1.0) - 1.0) * 0.5);
    while ((int64_t)J * (J + 1) / 2 > bi) --J;
    while ((int64_t)(J + 1) * (J + 2) / 2 <= bi) ++J;
    const int I = (int)(bi - (int64_t)J * (J + 1) / 2);
    const bool diag = I == J;

    const int tid = threadIdx.x;
    const int t0 = g.t_fstart[I], nI = g.t_fstart[I + 1] - t0;
    const int s0 = g.t_fstart[J], nJ = g.t_fstart[J + 1] - s0;
    const int tv0 = g.t_vstart[I], nvI = g.t_vstart[I + 1] - tv0;
    const int sv0 = g.t_vstart[J], nvJ = g.t_vstart[J + 1] - sv0;

    static_assert((2 * SYM_ACC) % 4 == 0, "accumulators are zeroed as float4");
    for (int i = tid; i < 2 * SYM_ACC / 4; i += REG_THREADS)
        reinterpret_cast<float4 *>(acc_re)[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    // the tile arrays: every copy in flight at once, one wait
    for (int i = tid; i < nI * Q * 3; i += REG_THREADS) cp_async4(&xq[i], &g.qpts[(size_t)t0 * Q * 3 + i]);
    for (int i = tid; i < nI * 3; i += REG_THREADS) {
        cp_async4(&xn[i], &g.normal[(size_t)t0 * 3 + i]);
        cp_async4(&xgv[i], &g.gvert[(size_t)t0 * 3 + i]);
        cp_async4(&xlv[i], &g.t_local[(size_t)t0 * 3 + i]);
    }
    for (int i = tid; i < nI * 9; i += REG_THREADS) cp_async4(&xc[i], &g.curl[(size_t)t0 * 9 + i]);
    for (int i = tid; i < nI; i += REG_THREADS) {
        cp_async4(&xa[i], &g.area[t0 + i]);
        cp_async4(&xp[i], &g.plane[t0 + i]);
    }
    for (int i = tid; i < nJ * Q * 3; i += REG_THREADS) {
        const int s = i / (Q * 3), j = i % (Q * 3);
        cp_async4(&yq[j * SYM_F + s], &g.qpts[(size_t)s0 * Q * 3 + i]);
    }
    for (int i = tid; i < nJ * 3; i += REG_THREADS) {
        const int s = i / 3, j = i % 3;
        cp_async4(&yn[j * SYM_F + s], &g.normal[(size_t)s0 * 3 + i]);
        cp_async4(&ygv[j * SYM_F + s], &g.gvert[(size_t)s0 * 3 + i]);
    }
    for (int i = tid; i < nJ * 9; i += REG_THREADS) {
        const int s = i / 9, j = i % 9;
        cp_async4(&yc[j * SYM_F + s], &g.curl[(size_t)s0 * 9 + i]);
    }
    for (int i = tid; i < nJ; i += REG_THREADS) {
        cp_async4(&ya[i], &g.area[s0 + i]);
        cp_async4(&yp[i], &g.plane[s0 + i]);
    }
    for (int i = tid; i < SYM_INC; i += REG_THREADS) cp_async4(&inc_start[i], &g.t_inc[(size_t)J * SYM_INC + i]);
    cp_async_wait_all();
    __syncthreads();
    if (g.image) {
        // an image pass reflects tile J: pairs (tau, S sigma) and (sigma, S tau)
        // have the same distances, |x - Sy| = |Sx - y|, and swap dn_s / dn_t
        for (int i = tid; i < nJ * Q * 3; i += REG_THREADS) {
            const int s = i / (Q * 3), j = i % (Q * 3);
            yq[j * SYM_F + s] *= g.xs[j % 3];
        }
        for (int i = tid; i < nJ * 3; i += REG_THREADS) {
            const int s = i / 3, j = i % 3;
            yn[j * SYM_F + s] *= g.xs[j];
        }
        for (int i = tid; i < nJ * 9; i += REG_THREADS) {
            const int s = i / 9, j = i % 9;
            yc[j * SYM_F + s] *= g.xdet * g.xs[j % 3];
        }
        __syncthreads();
    }

    const T k = g.k, eta = g.eta;
    const T kr = k * T(0.15915494309189535);  // k / (2 pi): the phase k r in revolutions
    const T inv4pi = T(0.07957747154594767);  // 1 / (4 pi)
    for (int p = tid; p < SYM_F * SYM_F; p += REG_THREADS) {
        const int ti = p / SYM_F, sj = p % SYM_F;  // a warp: one tau, every sigma
        // (an image pass keeps tau == sigma: the element and its own image,
        // whose two orders coincide and are taken at half weight)
        if (ti >= nI || sj >= nJ || (diag && (g.image ? sj < ti : sj <= ti))) continue;
        const int ga = xgv[3 * ti], gb = xgv[3 * ti + 1], gc = xgv[3 * ti + 2];
        const int ha = ygv[sj], hb = ygv[SYM_F + sj], hc = ygv[2 * SYM_F + sj];
        if (!g.image && (ga == ha || ga == hb || ga == hc || gb == ha || gb == hb || gb == hc || gc == ha ||
                         gc == hb || gc == hc))
            continue;  // touching pair: the Duffy kernel integrates both orders
        const T ntx = xn[3 * ti], nty = xn[3 * ti + 1], ntz = xn[3 * ti + 2];
        const T nsx = yn[sj], nsy = yn[SYM_F + sj], nsz = yn[2 * SYM_F + sj];
        const T k2n = eta * g.k2 * (ntx * nsx + nty * nsy + ntz * nsz);
        const T dtau = xp[ti], dsig = yp[sj];
        // r . n_tau = y . n_tau - x . n_tau is the same for every test point x
        // on the flat face tau: one value per trial point
        T ync[Q];
#pragma unroll
        for (int qs = 0; qs < Q; ++qs)
            ync[qs] = yq[(qs * 3) * SYM_F + sj] * ntx + yq[(qs * 3 + 1) * SYM_F + sj] * nty +
                      yq[(qs * 3 + 2) * SYM_F + sj] * ntz - dtau;
        // L1 / L2: the two orders' 3 x 3 blocks; R1: order 1's right-hand-side
        // 3-vector; TC_b: sum over both faces' points of w phi_b(y) G, which
        // gives the Green sum of the curl term and order 2's right-hand side
        T L1[9][2], L2[9][2], R1[3][2], TC[3][2];
#pragma unroll
        for (int i = 0; i < 9; ++i) L1[i][0] = L1[i][1] = L2[i][0] = L2[i][1] = T(0);
#pragma unroll
        for (int i = 0; i < 3; ++i) R1[i][0] = R1[i][1] = TC[i][0] = TC[i][1] = T(0);
#pragma unroll 1
        for (int qt = 0; qt < Q; ++qt) {
            const T x0 = xq[(ti * Q + qt) * 3], x1 = xq[(ti * Q + qt) * 3 + 1], x2 = xq[(ti * Q + qt) * 3 + 2];
            const T wt = RuleRef<T>::w(RI, qt) * inv4pi;
            const T xns = dsig - (x0 * nsx + x1 * nsy + x2 * nsz);  // r . n_sigma for every y on sigma
            // Per trial point (the test point's weight wt applied below):
            //   g = w_s exp(ikr) / r,  h = g (ik - 1/r) / r  (dG/dr / r),
            //   C_b += phi_b(y) g,  H_b += phi_b(y) h,  P_b += phi_b(y) (r . n_tau) h.
            // Order 1's kernel value -g' (r . n_sigma) / r - i k2n g sums to
            // -xns H_b - i k2n C_b, order 2's (r . n_tau) g' / r - i k2n g to
            // P_b - i k2n C_b; each sum a packed (re, im) pair.
            F2 C0 = 0, C1 = 0, C2 = 0, H0 = 0, H1 = 0, H2 = 0, P0 = 0, P1 = 0, P2 = 0;
#pragma unroll
            for (int qs = 0; qs < Q; ++qs) {
                const T rx = yq[(qs * 3) * SYM_F + sj] - x0, ry = yq[(qs * 3 + 1) * SYM_F + sj] - x1,
                        rz = yq[(qs * 3 + 2) * SYM_F + sj] - x2;
                const T r2 = rx * rx + ry * ry + rz * rz;
                const T ir = rsqrt_t(r2);
                T sn_, cs_;
                sincos_rev(kr * (r2 * ir), &sn_, &cs_);
                const T scl = ir * RuleRef<T>::w(RI, qs);
                const T gr = cs_ * scl, gi = sn_ * scl;
                const T hr = (-gr * ir - gi * k) * ir;
                const T hi = (gr * k - gi * ir) * ir;
                const F2 g2 = pk2(gr, gi), h2 = pk2(hr, hi);
                const F2 b0 = rule_b2(RI, qs, 0), b1 = rule_b2(RI, qs, 1), b2 = rule_b2(RI, qs, 2);
                C0 = fma2(b0, g2, C0);
                C1 = fma2(b1, g2, C1);
                C2 = fma2(b2, g2, C2);
                H0 = fma2(b0, h2, H0);
                H1 = fma2(b1, h2, H1);
                H2 = fma2(b2, h2, H2);
                const F2 p2 = mul2(pk2(ync[qs], ync[qs]), h2);
                P0 = fma2(b0, p2, P0);
                P1 = fma2(b1, p2, P1);
                P2 = fma2(b2, p2, P2);
            }
            T Cr[3], Ci[3], Hr[3], Hi[3], Pr[3], Pi[3];
            up2(C0, Cr[0], Ci[0]);
            up2(C1, Cr[1], Ci[1]);
            up2(C2, Cr[2], Ci[2]);
            up2(H0, Hr[0], Hi[0]);
            up2(H1, Hr[1], Hi[1]);
            up2(H2, Hr[2], Hi[2]);
            up2(P0, Pr[0], Pi[0]);
            up2(P1, Pr[1], Pi[1]);
            up2(P2, Pr[2], Pi[2]);
            // order 1's right-hand-side value -G + i eta W, W = sum (r . n_tau) g' / r
            const T Gr = Cr[0] + Cr[1] + Cr[2], Gi = Ci[0] + Ci[1] + Ci[2];
            const T Wr = Pr[0] + Pr[1] + Pr[2], Wi = Pi[0] + Pi[1] + Pi[2];
            const T Ur = -Gr - eta * Wi, Ui = -Gi + eta * Wr;
            T Sr[3], Si[3];
#pragma unroll
            for (int b = 0; b < 3; ++b) {
                Sr[b] = -xns * Hr[b] + k2n * Ci[b];
                Si[b] = -xns * Hi[b] - k2n * Cr[b];
                Pr[b] += k2n * Ci[b];
                Pi[b] -= k2n * Cr[b];
                TC[b][0] += wt * Cr[b];
                TC[b][1] += wt * Ci[b];
            }
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                const T ba = RuleRef<T>::b(RI, qt, a) * wt;
#pragma unroll
                for (int b = 0; b < 3; ++b) {
                    L1[3 * a + b][0] += ba * Sr[b];
                    L1[3 * a + b][1] += ba * Si[b];
                    // order 2: row = test vertex of sigma (b), column = trial vertex of tau (a)
                    L2[3 * b + a][0] += ba * Pr[b];
                    L2[3 * b + a][1] += ba * Pi[b];
                }
                R1[a][0] += ba * Ur;
                R1[a][1] += ba * Ui;
            }
        }
        // Order 2's right-hand-side value at (x, y) is -(1 + eta k2n) g + i eta
        // times order 1's kernel value, so its sum against phi_b(y) is
        // -(1 + eta k2n) TC_b + i eta sum_a L1[a][b] (the test basis sums to 1).
        const T cr = TC[0][0] + TC[1][0] + TC[2][0], ci = TC[0][1] + TC[1][1] + TC[2][1];
        const T ce = -(T(1) + eta * k2n);
        T R2[3][2];
#pragma unroll
        for (int b = 0; b < 3; ++b) {
            const T lr = L1[b][0] + L1[3 + b][0] + L1[6 + b][0], li = L1[b][1] + L1[3 + b][1] + L1[6 + b][1];
            R2[b][0] = ce * TC[b][0] - eta * li;
            R2[b][1] = ce * TC[b][1] + eta * lr;
        }
        // hypersingular curl term: eta * sum(g w) * curl_test . curl_trial (same sum for both orders)
        const T ccr = -eta * ci, cci = eta * cr;
        const T jac = T(4) * xa[ti] * ya[sj] * ((g.image && diag && sj == ti) ? T(0.5) : T(1));
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const int ra = xlv[3 * ti + a];  // vertex a of tau, tile I local
            int off[14];  // this vertex's 14 adds (re and im planes)
            float val[14];
#pragma unroll
            for (int b = 0; b < 3; ++b) {
                const T d = xc[9 * ti + 3 * a] * yc[(3 * b) * SYM_F + sj] +
                            xc[9 * ti + 3 * a + 1] * yc[(3 * b + 1) * SYM_F + sj] +
                            xc[9 * ti + 3 * a + 2] * yc[(3 * b + 2) * SYM_F + sj];  // curl_tau[a] . curl_sigma[b]
                const int o1 = SYM_C1 + ra * SYM_S + b * SYM_F + sj;
                off[4 * b] = o1;
                val[4 * b] = (L1[3 * a + b][0] + d * ccr) * jac;
                off[4 * b + 1] = o1 + SYM_ACC;
                val[4 * b + 1] = (L1[3 * a + b][1] + d * cci) * jac;
                // order 2 entry (sigma vertex b, tau vertex a) uses curl_sigma[b] . curl_tau[a] = d
                const int o2 = SYM_C2 + (b * SYM_F + sj) * SYM_C2S + ra;
                off[4 * b + 2] = o2;
                val[4 * b + 2] = (L2[3 * b + a][0] + d * ccr) * jac;
                off[4 * b + 3] = o2 + SYM_ACC;
                val[4 * b + 3] = (L2[3 * b + a][1] + d * cci) * jac;
            }
            off[12] = SYM_B1 + ra * SYM_BS + sj;
            val[12] = R1[a][0] * jac;
            off[13] = off[12] + SYM_ACC;
            val[13] = R1[a][1] * jac;
            // tau's other elements in flight on other warps may share vertex a
            batch_add<14>(acc_re, off, val);
            // (sigma slot a, face tau) belongs to this element pair alone: a plain store
            const int e2 = SYM_D2 + (a * SYM_F + sj) * SYM_BS + ti;
            acc_re[e2] = R2[a][0] * jac;
            acc_im[e2] = R2[a][1] * jac;
        }
    }
    __syncthreads();
    // fold the slot-face entries onto tile J's vertices and flush
    for (int i = tid; i < nvI * nvJ; i += REG_THREADS) {
        const int li = i / nvJ, lj = i % nvJ;
        Cx<T> v{T(0), T(0)}, u{T(0), T(0)};
        for (int e = inc_start[lj]; e < inc_start[lj + 1]; ++e) {
            const int s = inc_list[e];
            v.re += acc_re[SYM_C1 + li * SYM_S + s];
            v.im += acc_im[SYM_C1 + li * SYM_S + s];
            u.re += acc_re[SYM_C2 + s * SYM_C2S + li];
            u.im += acc_im[SYM_C2 + s * SYM_C2S + li];
        }
        const int gi_ = g.t_verts[tv0 + li], gj_ = g.t_verts[sv0 + lj];
        if (v.re != T(0) || v.im != T(0)) red_add_cx(&g.A[(int64_t)gi_ * g.ld + gj_], v.re, v.im);
        if (u.re != T(0) || u.im != T(0)) red_add_cx(&g.A[(int64_t)gj_ * g.ld + gi_], u.re, u.im);
    }
    if (g.B) {
        for (int i = tid; i < nvI * nJ; i += REG_THREADS) {
            const int li = i / nJ, sj = i % nJ;
            const Cx<T> v{acc_re[SYM_B1 + li * SYM_BS + sj], acc_im[SYM_B1 + li * SYM_BS + sj]};
            if (v.re != T(0) || v.im != T(0))
                red_add_cx(&g.B[(int64_t)g.t_verts[tv0 + li] * g.F + g.face_id[s0 + sj]], v.re, v.im);
        }
        for (int i = tid; i < nvJ * nI; i += REG_THREADS) {
            const int lj = i / nI, ti = i % nI;
            Cx<T> v{T(0), T(0)};
            for (int e = inc_start[lj]; e < inc_start[lj + 1]; ++e) {
                const int s = inc_list[e];
                v.re += acc_re[SYM_D2 + s * SYM_BS + ti];
                v.im += acc_im[SYM_D2 + s * SYM_BS + ti];
            }
            if (v.re != T(0) || v.im != T(0))
                red_add_cx(&g.B[(int64_t)g.t_verts[sv0 + lj] * g.F + g.face_id[t0 + ti]], v.re, v.im);
        }
        return;
    }
    // matrix-free: rows of b += B1 q (tile I vertices x tile J faces) and
    // B2 q (tile J vertices x tile I faces); q of both tiles' faces staged
    // MF_RC columns at a time over the (now unused) geometry region
    float2 *qs = reinterpret_cast<float2 *>(xq);  // [2][SYM_F][MF_RC]: tile I faces, then tile J faces
    // order 2 rows folded onto tile J's vertices, over the (read) C1 block
    constexpr int B2V = SYM_C1;  // [vJ][tau]
    __syncthreads();
    for (int i = tid; i < nvJ * nI; i += REG_THREADS) {
        const int lj = i / nI, ti = i % nI;
        T vr = T(0), vi = T(0);
        for (int e = inc_start[lj]; e < inc_start[lj + 1]; ++e) {
            vr += acc_re[SYM_D2 + inc_list[e] * SYM_BS + ti];
            vi += acc_im[SYM_D2 + inc_list[e] * SYM_BS + ti];
        }
        acc_re[B2V + lj * SYM_BS + ti] = vr;
        acc_im[B2V + lj * SYM_BS + ti] = vi;
    }
    for (int r0 = 0; r0 < g.R; r0 += MF_RC) {
        const int rc = min(MF_RC, g.R - r0);
        __syncthreads();
        for (int i = tid; i < 2 * SYM_F * MF_RC; i += REG_THREADS) {
            const int h = i / (SYM_F * MF_RC), f = (i / MF_RC) % SYM_F, r = i % MF_RC;
            float2 v = make_float2(0.f, 0.f);
            if (f < (h ? nJ : nI) && r < rc) {
                const Cx<double> qq = g.q[(size_t)(r0 + r) * g.F + g.face_id[(h ? s0 : t0) + f]];
                v = make_float2((float)qq.re, (float)qq.im);
            }
            qs[i] = v;
        }
        __syncthreads();
        for (int i = tid; i < (nvI + nvJ) * rc; i += REG_THREADS) {
            const int row = i / rc, r = i % rc;
            const bool first = row < nvI;
            const int base = first ? SYM_B1 + row * SYM_BS : B2V + (row - nvI) * SYM_BS;
            const int nf = first ? nJ : nI;
            const float2 *qh = qs + (first ? SYM_F * MF_RC : 0);
            T sr = T(0), si = T(0);
            for (int f = 0; f < nf; ++f) {
                const T br = acc_re[base + f], bi = acc_im[base + f];
                const float2 qv = qh[f * MF_RC + r];
                sr += br * qv.x - bi * qv.y;
                si += br * qv.y + bi * qv.x;
            }
            const int gv = first ? g.t_verts[tv0 + row] : g.t_verts[sv0 + row - nvI];
            if (sr != T(0) || si != T(0)) red_add_cx(&g.b[(size_t)(r0 + r) * g.N + gv], (double)sr, (double)si);
        }
    }
}

// ---------------------------------------------------------------------------
// touching pairs: one warp per pair, FP64, Duffy points over the lanes
// ---------------------------------------------------------------------------
template <typename T> struct SingArgs {
    const int *test, *trial, *rule;
    const double *jac, *nn;
    const int *rule_start;
    const double *rule_data;  // 5 per point
    const double *verts;      // V x 3
    const int *faces;         // F x 3
    const double *normals;    // F x 3
    const double *curls;      // F x 9
    Cx<T> *A;
    RhsOut<T> rhs;
    int64_t ld;
    int64_t npairs;
    double k, eta;
};

template <typename T>
__global__ void __launch_bounds__(256, 2) singular_pairs_kernel(SingArgs<T> g) {
    const int lane = threadIdx.x & 31;
    const int64_t pair = (int64_t)blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
    if (pair >= g.npairs) return;
    const int t = g.test[pair], s = g.trial[pair], r = g.rule[pair];
    const int *ft = g.faces + 3 * t, *fs = g.faces + 3 * s;
    double tv[3][3], sv[3][3];
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            tv[a][c] = g.verts[3 * ft[a] + c];
            sv[a][c] = g.verts[3 * fs[a] + c];
        }
    const double ntx = g.normals[3 * t], nty = g.normals[3 * t + 1], ntz = g.normals[3 * t + 2];
    const double nsx = g.normals[3 * s], nsy = g.normals[3 * s + 1], nsz = g.normals[3 * s + 2];
    const double k = g.k, eta = g.eta;
    const double k2n = eta * (k * k * g.nn[pair]);
    double acc[26];
#pragma unroll
    for (int i = 0; i < 26; ++i) acc[i] = 0.0;  // L[9] re/im, R[3] re/im, curl re/im
    const int q1 = g.rule_start[r + 1];
    for (int q = g.rule_start[r] + lane; q < q1; q += 32) {
        const double *d = g.rule_data + 5 * (size_t)q;
        const double xi = d[0], et = d[1], yi = d[2], ye = d[3], w = d[4];
        const double bt[3] = {1.0 - xi - et, xi, et}, bs[3] = {1.0 - yi - ye, yi, ye};
        double x[3], y[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            x[c] = bt[0] * tv[0][c] + bt[1] * tv[1][c] + bt[2] * tv[2][c];
            y[c] = bs[0] * sv[0][c] + bs[1] * sv[1][c] + bs[2] * sv[2][c];
        }
        const double rx = y[0] - x[0], ry = y[1] - x[1], rz = y[2] - x[2];
        const double r2 = rx * rx + ry * ry + rz * rz;
        if (r2 == 0.0) continue;
        const double ir = rsqrt(r2), rad = r2 * ir;  // one reciprocal square root, no divide
        double sn_, cs_;
        sincos_cw(k * rad, &sn_, &cs_);
        const double scl = ir * (0.07957747154594767 * w);
        const double gr = cs_ * scl, gi = sn_ * scl;
        const double gsr = -gr * ir - gi * k, gsi = gr * k - gi * ir;
        const double dns = (rx * nsx + ry * nsy + rz * nsz) * ir;
        const double dnt = -(rx * ntx + ry * nty + rz * ntz) * ir;
        const double lr = -gsr * dns + k2n * gi, li = -gsi * dns - k2n * gr;
        const double rr = -gr + eta * (gsi * dnt), ri = -gi - eta * (gsr * dnt);
#pragma unroll
        for (int a = 0; a < 3; ++a) {
#pragma unroll
            for (int b = 0; b < 3; ++b) {
                const double bp = bt[a] * bs[b];
                acc[2 * (3 * a + b)] += bp * lr;
                acc[2 * (3 * a + b) + 1] += bp * li;
            }
            acc[18 + 2 * a] += bt[a] * rr;
            acc[18 + 2 * a + 1] += bt[a] * ri;
        }
        acc[24] += gr;
        acc[25] += gi;
    }
#pragma unroll
    for (int i = 0; i < 26; ++i) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc[i] += __shfl_xor_sync(0xffffffffu, acc[i], o);
    }
    const double jac = g.jac[pair];
    const double ccr = -eta * acc[25], cci = eta * acc[24];
    if (lane < 9) {
        const int a = lane / 3, b = lane % 3;
        const double *cta = g.curls + 9 * t + 3 * a, *csb = g.curls + 9 * s + 3 * b;
        const double d = cta[0] * csb[0] + cta[1] * csb[1] + cta[2] * csb[2];
        double vr = 0, vi = 0;
#pragma unroll
        for (int i = 0; i < 9; ++i)
            if (i == lane) {
                vr = acc[2 * i];
                vi = acc[2 * i + 1];
            }
        red_add_cx(&g.A[(int64_t)ft[a] * g.ld + fs[b]], (T)((vr + d * ccr) * jac), (T)((vi + d * cci) * jac));
    } else if (lane < 12) {
        const int a = lane - 9;
        double vr = 0, vi = 0;
#pragma unroll
        for (int i = 0; i < 3; ++i)
            if (i == a) {
                vr = acc[18 + 2 * i];
                vi = acc[18 + 2 * i + 1];
            }
        rhs_add(g.rhs, ft[a], s, (T)(vr * jac), (T)(vi * jac));
    }
}

// ---------------------------------------------------------------------------
// touching image pairs (test t, trial s reflected by image x): the remapped
// Duffy integral minus the regular-rule integral the image pass added
// (_cuda_image_singular_delta_blocks_kernel!, BeatEngineCudaSingular.jl:590-897).
// One warp per pair, FP64, lanes over the Duffy points, then over the Q x Q
// regular points.
// ---------------------------------------------------------------------------
struct ImgXf {
    double s[3][3];  // per image: signs
    double det[3];
};

template <typename T> struct ImgArgs {
    const int *test, *trial, *rule, *img;
    const double *jac, *nn;
    const int *rule_start;
    const double *rule_data;  // 5 per point
    const double *verts;
    const int *faces;
    const double *normals, *curls;
    int Q, RI;
    Cx<T> *A;
    RhsOut<T> rhs;
    int64_t ld;
    int64_t npairs;
    double k, eta;
    ImgXf xf;
};

__device__ __forceinline__ void bm_point_d(const double *x, const double *y, const double *bt, const double *bs,
                                           double w, const double *nt, const double *ns, double k, double eta,
                                           double k2n, double sign, double *acc) {
    const double rx = y[0] - x[0], ry = y[1] - x[1], rz = y[2] - x[2];
    const double r2 = rx * rx + ry * ry + rz * rz;
    if (r2 == 0.0) return;
    const double ir = rsqrt(r2), rad = r2 * ir;
    double sn_, cs_;
    sincos_cw(k * rad, &sn_, &cs_);
    const double scl = sign * ir * (0.07957747154594767 * w);
    const double gr = cs_ * scl, gi = sn_ * scl;
    const double gsr = -gr * ir - gi * k, gsi = gr * k - gi * ir;
    const double dns = (rx * ns[0] + ry * ns[1] + rz * ns[2]) * ir;
    const double dnt = -(rx * nt[0] + ry * nt[1] + rz * nt[2]) * ir;
    const double lr = -gsr * dns + k2n * gi, li = -gsi * dns - k2n * gr;
    const double rr = -gr + eta * (gsi * dnt), ri = -gi - eta * (gsr * dnt);
#pragma unroll
    for (int a = 0; a < 3; ++a) {
#pragma unroll
        for (int b = 0; b < 3; ++b) {
            const double bp = bt[a] * bs[b];
            acc[2 * (3 * a + b)] += bp * lr;
            acc[2 * (3 * a + b) + 1] += bp * li;
        }
        acc[18 + 2 * a] += bt[a] * rr;
        acc[18 + 2 * a + 1] += bt[a] * ri;
    }
    acc[24] += gr;
    acc[25] += gi;
}

template <typename T>
__global__ void __launch_bounds__(256, 2) image_delta_kernel(ImgArgs<T> g) {
    const int lane = threadIdx.x & 31;
    const int64_t pair = (int64_t)blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
    if (pair >= g.npairs) return;
    const int t = g.test[pair], s = g.trial[pair], r = g.rule[pair], ix = g.img[pair];
    const double *sg = g.xf.s[ix];
    const int *ft = g.faces + 3 * t, *fs = g.faces + 3 * s;
    double tv[3][3], sv[3][3], nt[3], ns[3];
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            tv[a][c] = g.verts[3 * ft[a] + c];
            sv[a][c] = sg[c] * g.verts[3 * fs[a] + c];
        }
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        nt[c] = g.normals[3 * t + c];
        ns[c] = sg[c] * g.normals[3 * s + c];
    }
    const double k = g.k, eta = g.eta;
    const double k2n = eta * (k * k * g.nn[pair]);
    double acc[26];
#pragma unroll
    for (int i = 0; i < 26; ++i) acc[i] = 0.0;
    // + Duffy
    for (int q = g.rule_start[r] + lane; q < g.rule_start[r + 1]; q += 32) {
        const double *d = g.rule_data + 5 * (size_t)q;
        const double bt[3] = {1.0 - d[0] - d[1], d[0], d[1]}, bs[3] = {1.0 - d[2] - d[3], d[2], d[3]};
        double x[3], y[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            x[c] = bt[0] * tv[0][c] + bt[1] * tv[1][c] + bt[2] * tv[2][c];
            y[c] = bs[0] * sv[0][c] + bs[1] * sv[1][c] + bs[2] * sv[2][c];
        }
        bm_point_d(x, y, bt, bs, d[4], nt, ns, k, eta, k2n, 1.0, acc);
    }
    // - regular rule
    for (int pq = lane; pq < g.Q * g.Q; pq += 32) {
        const int qt = pq / g.Q, qs = pq % g.Q;
        const double bt[3] = {c_rb64[g.RI][qt][0], c_rb64[g.RI][qt][1], c_rb64[g.RI][qt][2]};
        const double bs[3] = {c_rb64[g.RI][qs][0], c_rb64[g.RI][qs][1], c_rb64[g.RI][qs][2]};
        double x[3], y[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            x[c] = bt[0] * tv[0][c] + bt[1] * tv[1][c] + bt[2] * tv[2][c];
            y[c] = bs[0] * sv[0][c] + bs[1] * sv[1][c] + bs[2] * sv[2][c];
        }
        bm_point_d(x, y, bt, bs, c_rw64[g.RI][qt] * c_rw64[g.RI][qs], nt, ns, k, eta, k2n, -1.0, acc);
    }
#pragma unroll
    for (int i = 0; i < 26; ++i) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc[i] += __shfl_xor_sync(0xffffffffu, acc[i], o);
    }
    const double jac = g.jac[pair];
    const double ccr = -eta * acc[25], cci = eta * acc[24];
    const double cdet = g.xf.det[ix];
    if (lane < 9) {
        const int a = lane / 3, b = lane % 3;
        const double *cta = g.curls + 9 * t + 3 * a, *csb = g.curls + 9 * s + 3 * b;
        const double d = cdet * (cta[0] * sg[0] * csb[0] + cta[1] * sg[1] * csb[1] + cta[2] * sg[2] * csb[2]);
        double vr = 0, vi = 0;
#pragma unroll
        for (int i = 0; i < 9; ++i)
            if (i == lane) {
                vr = acc[2 * i];
                vi = acc[2 * i + 1];
            }
        red_add_cx(&g.A[(int64_t)ft[a] * g.ld + fs[b]], (T)((vr + d * ccr) * jac), (T)((vi + d * cci) * jac));
    } else if (lane < 12) {
        const int a = lane - 9;
        double vr = 0, vi = 0;
#pragma unroll
        for (int i = 0; i < 3; ++i)
            if (i == a) {
                vr = acc[18 + 2 * i];
                vi = acc[18 + 2 * i + 1];
            }
        rhs_add(g.rhs, ft[a], s, (T)(vr * jac), (T)(vi * jac));
    }
}

// orbit row weights (p1_symmetry_orbit_weights, BeatEngineCore.jl:563-582):
// the rows of A and B of vertices on a symmetry plane, times 2 per plane
// (the rows of b instead of B in the matrix-free mode: b = B q is linear in B)
template <typename T>
__global__ void row_weight_kernel(const int *verts, const double *weights, int nw, Cx<T> *A, int64_t ld, int n,
                                  RhsOut<T> rhs) {
    const int v = blockIdx.y;
    if (v >= nw) return;
    const int row = verts[v];
    const double w = weights[v];
    const int cols = rhs.B ? rhs.F : rhs.R;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n + cols; j += gridDim.x * blockDim.x) {
        if (j < n || rhs.B) {
            Cx<T> &e = j < n ? A[(int64_t)row * ld + j] : rhs.B[(int64_t)row * rhs.F + (j - n)];
            e.re *= (T)w;
            e.im *= (T)w;
        } else {
            Cx<double> &e = rhs.b[(size_t)(j - n) * rhs.N + row];
            e.re *= w;
            e.im *= w;
        }
    }
}

// ---------------------------------------------------------------------------
// identity terms: A += 0.5 M_p1p1, B += -0.5 eta M_p1dp0
// ---------------------------------------------------------------------------
template <typename T>
__global__ void identity_kernel(const int *faces, const double *areas, int F, int Q, double eta, Cx<T> *A,
                                int64_t ld, RhsOut<T> rhs) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= F) return;
    const int ri = Q == 1 ? 0 : Q == 3 ? 1 : 2;
    const double jac = 2.0 * areas[f];
    double blk[9] = {0}, col[3] = {0};
    for (int q = 0; q < Q; ++q) {
        const double w = c_rw64[ri][q];
        for (int a = 0; a < 3; ++a) {
            const double pa = c_rb64[ri][q][a];
            col[a] += pa * w * jac;
            for (int b = 0; b < 3; ++b) blk[3 * a + b] += pa * c_rb64[ri][q][b] * w * jac;
        }
    }
    const int *fc = faces + 3 * f;
    for (int a = 0; a < 3; ++a) {
        for (int b = 0; b < 3; ++b) red_add(&A[(int64_t)fc[a] * ld + fc[b]].re, (T)(0.5 * blk[3 * a + b]));
        rhs_add(rhs, fc[a], f, T(0), (T)(-0.5 * eta * col[a]));
    }
}

// ---------------------------------------------------------------------------
// host driver
// ---------------------------------------------------------------------------
template <typename T> static RhsOut<T> rhs_out(beat_b200_ctx *c, int R, const Cx<double> *q) {
    RhsOut<T> o;
    o.B = c->ws.rhs_cached ? c->ws.B.as<Cx<T>>() : nullptr;
    o.q = q;
    o.b = c->ws.b.as<Cx<double>>();
    o.F = c->F;
    o.N = c->V;
    o.R = R;
    return o;
}

template <typename T, int Q>
static void launch_regular(beat_b200_ctx *c, double k, double eta, int img, int R, const Cx<double> *q) {
    RegArgs<T> g;
    const bool d = sizeof(T) == 8;
    g.qpts = (const T *)(d ? c->pos_qpts64.p : c->pos_qpts32.p);
    g.normal = (const T *)(d ? c->pos_normal64.p : c->pos_normal32.p);
    g.curl = (const T *)(d ? c->pos_curl64.p : c->pos_curl32.p);
    g.area = (const T *)(d ? c->pos_area64.p : c->pos_area32.p);
    g.gvert = c->pos_gvert.as<int>();
    g.face_id = c->pos_face.as<int>();
    g.t_fstart = c->test_tiles.face_start.as<int>();
    g.t_vstart = c->test_tiles.vert_start.as<int>();
    g.t_verts = c->test_tiles.verts.as<int>();
    g.t_local = c->test_tiles.local_vert.as<int>();
    g.s_fstart = c->trial_tiles.face_start.as<int>();
    g.s_vstart = c->trial_tiles.vert_start.as<int>();
    g.s_verts = c->trial_tiles.verts.as<int>();
    g.s_inc = c->trial_tiles.incidence.as<int>();
    BB_REQUIRE(c->trial_tiles.inc_stride() == REG_INC, BEAT_B200_STATE, "assembly: trial tile shape mismatch");
    g.A = c->ws.A.as<Cx<T>>();
    g.B = c->ws.rhs_cached ? c->ws.B.as<Cx<T>>() : nullptr;
    g.q = q;
    g.b = c->ws.b.as<Cx<double>>();
    g.N = c->V;
    g.R = R;
    g.ld = c->ws.ld;
    g.F = c->F;
    g.k = (T)k;
    g.eta = (T)eta;
    g.k2 = (T)(k * k);
    if (img >= 0) {
        g.image = 1;
        for (int i = 0; i < 3; ++i) g.xs[i] = (T)c->img_sign[img][i];
        g.xdet = (T)c->img_det[img];
    }
    const size_t smem = regular_smem_bytes<T, Q>();
    BB_CUDA(cudaFuncSetAttribute(regular_pairs_kernel<T, Q>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    BB_CUDA(cudaFuncSetAttribute(regular_pairs_kernel<T, Q>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                 cudaSharedmemCarveoutMaxShared));
    dim3 grid(c->trial_tiles.ntiles, c->test_tiles.ntiles);
    regular_pairs_kernel<T, Q><<<grid, REG_THREADS, smem, c->stream>>>(g);
    BB_CUDA(cudaGetLastError());
}

// FP32 form: the symmetric kernel over unordered pairs of square tiles
template <int Q>
static void launch_sym(beat_b200_ctx *c, double k, double eta, int img, int R, const Cx<double> *q) {
    RegArgs<float> g;
    g.qpts = c->pos_qpts32.as<float>();
    g.normal = c->pos_normal32.as<float>();
    g.curl = c->pos_curl32.as<float>();
    g.area = c->pos_area32.as<float>();
    g.plane = c->pos_plane32.as<float>();
    g.gvert = c->pos_gvert.as<int>();
    g.face_id = c->pos_face.as<int>();
    g.t_fstart = c->sym_tiles.face_start.as<int>();
    g.t_vstart = c->sym_tiles.vert_start.as<int>();
    g.t_verts = c->sym_tiles.verts.as<int>();
    g.t_local = c->sym_tiles.local_vert.as<int>();
    g.t_inc = c->sym_tiles.incidence.as<int>();
    BB_REQUIRE(c->sym_tiles.inc_stride() == SYM_INC, BEAT_B200_STATE, "assembly: square tile shape mismatch");
    g.s_fstart = g.s_vstart = g.s_verts = nullptr;
    g.A = c->ws.A.as<Cx<float>>();
    g.B = c->ws.rhs_cached ? c->ws.B.as<Cx<float>>() : nullptr;
    g.q = q;
    g.b = c->ws.b.as<Cx<double>>();
    g.N = c->V;
    g.R = R;
    g.ld = c->ws.ld;
    g.F = c->F;
    g.k = (float)k;
    g.eta = (float)eta;
    g.k2 = (float)(k * k);
    if (img >= 0) {
        g.image = 1;
        for (int i = 0; i < 3; ++i) g.xs[i] = c->img_sign[img][i];
        g.xdet = c->img_det[img];
    }
    const size_t smem = sym_smem_bytes<Q>();
    BB_CUDA(cudaFuncSetAttribute(sym_pairs_kernel<Q>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    BB_CUDA(cudaFuncSetAttribute(sym_pairs_kernel<Q>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                 cudaSharedmemCarveoutMaxShared));  // two CTAs per SM
    const int64_t nt = c->sym_tiles.ntiles;
    const int64_t blocks = nt * (nt + 1) / 2;
    BB_REQUIRE(blocks < (1ll << 31), BEAT_B200_INVALID_ARG, "assembly: mesh too large for the tile-pair grid");
    sym_pairs_kernel<Q><<<(unsigned)blocks, REG_THREADS, smem, c->stream>>>(g);
    BB_CUDA(cudaGetLastError());
}

template <typename T> static void assemble_t(beat_b200_ctx *c, double k, double eta, int R, const Cx<double> *q,
                                             float *ms_total, float *ms_singular) {
    Workspace &w = c->ws;
    const int N = c->V, F = c->F;
    BB_CUDA(cudaEventRecord(c->ev[0], c->stream));
    BB_CUDA(cudaMemsetAsync(w.A.p, 0, (size_t)N * w.ld * sizeof(Cx<T>), c->stream));
    if (w.rhs_cached)
        BB_CUDA(cudaMemsetAsync(w.B.p, 0, (size_t)N * F * sizeof(Cx<T>), c->stream));
    else  // matrix-free: the kernels add into b directly
        BB_CUDA(cudaMemsetAsync(w.b.p, 0, sizeof(Cx<double>) * (size_t)N * R, c->stream));
    BB_CUDA(cudaEventRecord(c->ev[8], c->stream));
    for (int img = -1; img < c->nimg; ++img) {  // the mesh itself, then one pass per symmetry image
        if (sizeof(T) == 4) {
            switch (c->Q) {
                case 1: launch_sym<1>(c, k, eta, img, R, q); break;
                case 3: launch_sym<3>(c, k, eta, img, R, q); break;
                default: launch_sym<6>(c, k, eta, img, R, q); break;
            }
        } else {
            switch (c->Q) {
                case 1: launch_regular<T, 1>(c, k, eta, img, R, q); break;
                case 3: launch_regular<T, 3>(c, k, eta, img, R, q); break;
                default: launch_regular<T, 6>(c, k, eta, img, R, q); break;
            }
        }
    }
    BB_CUDA(cudaEventRecord(c->ev[1], c->stream));
    if (c->npairs > 0) {
        SingArgs<T> s;
        s.test = c->sp_test.as<int>();
        s.trial = c->sp_trial.as<int>();
        s.rule = c->sp_rule.as<int>();
        s.jac = c->sp_jac.as<double>();
        s.nn = c->sp_nn.as<double>();
        s.rule_start = c->rule_start.as<int>();
        s.rule_data = c->rule_data.as<double>();
        s.verts = c->d_verts.as<double>();
        s.faces = c->d_faces.as<int>();
        s.normals = c->d_normals.as<double>();
        s.curls = c->d_curls.as<double>();
        s.A = w.A.as<Cx<T>>();
        s.rhs = rhs_out<T>(c, R, q);
        s.ld = w.ld;
        s.npairs = c->npairs;
        s.k = k;
        s.eta = eta;
        const int wpb = 8;
        singular_pairs_kernel<T><<<(unsigned)((c->npairs + wpb - 1) / wpb), 32 * wpb, 0, c->stream>>>(s);
        BB_CUDA(cudaGetLastError());
    }
    if (c->nimg_pairs > 0) {
        ImgArgs<T> d;
        d.test = c->ip_test.as<int>();
        d.trial = c->ip_trial.as<int>();
        d.rule = c->ip_rule.as<int>();
        d.img = c->ip_img.as<int>();
        d.jac = c->ip_jac.as<double>();
        d.nn = c->ip_nn.as<double>();
        d.rule_start = c->rule_start.as<int>();
        d.rule_data = c->rule_data.as<double>();
        d.verts = c->d_verts.as<double>();
        d.faces = c->d_faces.as<int>();
        d.normals = c->d_normals.as<double>();
        d.curls = c->d_curls.as<double>();
        d.Q = c->Q;
        d.RI = c->Q == 1 ? 0 : c->Q == 3 ? 1 : 2;
        d.A = w.A.as<Cx<T>>();
        d.rhs = rhs_out<T>(c, R, q);
        d.ld = w.ld;
        d.npairs = c->nimg_pairs;
        d.k = k;
        d.eta = eta;
        for (int i = 0; i < 3; ++i) {
            for (int j = 0; j < 3; ++j) d.xf.s[i][j] = c->img_sign[i][j];
            d.xf.det[i] = c->img_det[i];
        }
        image_delta_kernel<T><<<(unsigned)((c->nimg_pairs + 7) / 8), 256, 0, c->stream>>>(d);
        BB_CUDA(cudaGetLastError());
    }
    BB_CUDA(cudaEventRecord(c->ev[2], c->stream));
    identity_kernel<T><<<(F + 255) / 256, 256, 0, c->stream>>>(c->d_faces.as<int>(), c->d_areas.as<double>(), F,
                                                               c->Q, eta, w.A.as<Cx<T>>(), w.ld, rhs_out<T>(c, R, q));
    BB_CUDA(cudaGetLastError());
    if (c->nweighted > 0) {
        row_weight_kernel<T><<<dim3(32, c->nweighted), 256, 0, c->stream>>>(
            c->rw_vert.as<int>(), c->rw_weight.as<double>(), c->nweighted, w.A.as<Cx<T>>(), w.ld, N,
            rhs_out<T>(c, R, q));
        BB_CUDA(cudaGetLastError());
    }
    if (w.rhs_cached) {
        BB_CUDA(cudaMemsetAsync(w.b.p, 0, sizeof(Cx<double>) * (size_t)N * R, c->stream));
        tall_gemm<T>(c->stream, c->sm_count, w.B.as<Cx<T>>(), F, N, F, reinterpret_cast<const double *>(q),
                     w.b.as<double>(), R, 1.0);
    }
    BB_CUDA(cudaEventRecord(c->ev[3], c->stream));
    if (ms_total || ms_singular) {
        BB_CUDA(cudaEventSynchronize(c->ev[3]));
        if (ms_total) BB_CUDA(cudaEventElapsedTime(ms_total, c->ev[0], c->ev[3]));
        if (ms_singular) BB_CUDA(cudaEventElapsedTime(ms_singular, c->ev[1], c->ev[2]));
        BB_CUDA(cudaEventElapsedTime(&c->last_regular_ms, c->ev[8], c->ev[1]));
    }
}

void assemble(beat_b200_ctx *c, double k, double eta, int precision, int R, const void *q_dev, float *ms_total,
              float *ms_singular) {
    BB_REQUIRE(c->F > 0, BEAT_B200_STATE, "no mesh: call beat_b200_set_mesh first");
    BB_REQUIRE(std::isfinite(k) && k != 0.0 && std::isfinite(eta), BEAT_B200_INVALID_ARG,
               "assemble: wavenumber must be finite and nonzero");
    if (precision == BEAT_B200_FP64)
        assemble_t<double>(c, k, eta, R, (const Cx<double> *)q_dev, ms_total, ms_singular);
    else
        assemble_t<float>(c, k, eta, R, (const Cx<double> *)q_dev, ms_total, ms_singular);
}

}  // namespace bb
