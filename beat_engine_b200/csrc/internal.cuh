// internal.cuh -- shared declarations of libbeatb200 (not part of the ABI).
#pragma once

#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/beat_b200.h"

namespace bb {

// ---------------------------------------------------------------------------
// errors
// ---------------------------------------------------------------------------
struct Error {
    int32_t code;
    std::string msg;
};

#define BB_CUDA(call)                                                                       \
    do {                                                                                    \
        cudaError_t e_ = (call);                                                            \
        if (e_ != cudaSuccess)                                                              \
            throw ::bb::Error{e_ == cudaErrorMemoryAllocation ? BEAT_B200_OOM               \
                                                              : BEAT_B200_CUDA_ERROR,       \
                              std::string(#call) + ": " + cudaGetErrorString(e_)};          \
    } while (0)

#define BB_REQUIRE(cond, code, text)                    \
    do {                                                \
        if (!(cond)) throw ::bb::Error{(code), (text)}; \
    } while (0)

// device-side status words (one int per context, read by the host after a
// stage that can give up)
enum DeviceStatus : int {
    DEV_OK = 0,
    DEV_BARRIER_TIMEOUT = 1,  // a grid barrier ran out of its spin budget
    DEV_ZERO_PIVOT = 2,
    DEV_BAD_INDEX = 4,
};

// ---------------------------------------------------------------------------
// device buffers (plain cudaMalloc, owned by the context)
// ---------------------------------------------------------------------------
struct DevBuf {
    void *p = nullptr;
    size_t bytes = 0;
    void alloc(size_t n);
    void free_();
    template <typename T> T *as() const { return reinterpret_cast<T *>(p); }
};

// ---------------------------------------------------------------------------
// complex helpers
// ---------------------------------------------------------------------------
template <typename T> struct alignas(2 * sizeof(T)) Cx {
    T re, im;
};

template <typename T> __host__ __device__ __forceinline__ Cx<T> cmul(Cx<T> a, Cx<T> b) {
    return Cx<T>{a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}

#ifdef __CUDACC__
// Operand staging of the FP32 LU's tensor-core update (tc_gemm.cu): L is
// staged times 2^L_SHIFT, a complex column of U times 2^s with s =
// stage_exp(its largest |re| or |im|), each value as an FP16 high part and the
// FP16 rounding of the remainder.
constexpr int L_SHIFT = 12;
constexpr int B_SCALE_EXP = 14;
// s with m 2^s in [2^13, 2^14) for a normal m > 0 (m = f 2^e, f in [0.5, 1):
// s = 14 - e), clamped to [-100, 100]; 0 for m = 0
__device__ __forceinline__ int stage_exp(float m) {
    const unsigned bits = __float_as_uint(m);
    if (!(m > 0.f)) return 0;
    const int e = (int)((bits >> 23) & 0xffu) - 126;
    return max(-100, min(100, B_SCALE_EXP - e));
}
__device__ __forceinline__ float pow2f(int s) { return __int_as_float((127 + s) << 23); }  // |s| <= 126
// x as an FP16 high part and the FP16 rounding of x - high (exact in FP32)
__device__ __forceinline__ void split_f16(float x, __half &hi, __half &lo) {
    hi = __float2half_rn(x);
    lo = __float2half_rn(x - __half2float(hi));
}
// Cooperative copy of `total` items by NT threads, BATCH loads in flight per
// thread before any store: load(i) returns item i, store(i, v) writes it.
// (A plain `for (i = tid; ...) dst = src` loop waits for each load before the
// next one is issued when the store may alias the source.)
template <int NT, int BATCH, typename V, typename Load, typename Store>
__device__ __forceinline__ void batched_copy(int total, Load load, Store store) {
    for (int base = 0; base < total; base += NT * BATCH) {
        V v[BATCH];
#pragma unroll
        for (int u = 0; u < BATCH; ++u) {
            const int i = base + u * NT + (int)threadIdx.x;
            if (i < total) v[u] = load(i);
        }
#pragma unroll
        for (int u = 0; u < BATCH; ++u) {
            const int i = base + u * NT + (int)threadIdx.x;
            if (i < total) store(i, v[u]);
        }
    }
}
#endif

// ---------------------------------------------------------------------------
// mesh-derived tables for the element-pair kernel
// ---------------------------------------------------------------------------
struct Tiling {
    int tile_faces = 0;   // max faces per tile
    int tile_verts = 0;   // max distinct vertices per tile
    int ntiles = 0;
    DevBuf face_start;    // ntiles + 1 (positions in the sorted face order)
    DevBuf vert_start;    // ntiles + 1
    DevBuf verts;         // concatenated global vertex ids per tile
    DevBuf local_vert;    // F x 3 (by sorted position): index of each face vertex in its tile
    // per tile, inc_stride() ints: start[tile_verts + 1] then list[3 tile_faces]; the
    // slot-face indices s = b * tile_faces + f (vertex slot b of the tile's face f)
    // of local vertex v are list[start[v] .. start[v + 1]), in increasing s
    DevBuf incidence;
    int inc_stride() const { return tile_verts + 1 + 3 * tile_faces; }
};

struct Workspace {
    int precision = -1;
    int N = 0, F = 0, R = 0;
    int64_t ld = 0;       // leading dimension (row stride, in complex entries) of A
    DevBuf A;             // N x ld system matrix (row-major); FP64 or FP32 complex
    DevBuf Aop;           // mixed form: FP32 copy kept as the refinement operator
    DevBuf B;             // N x F RHS operator (row-major), same precision as A
    DevBuf b;             // N x R FP64 right-hand sides (column-major)
    DevBuf x;             // N x R FP64 solution (column-major)
    DevBuf ipiv;          // N int
    DevBuf perm;          // N int (row permutation of the factorisation)
    DevBuf panel_scratch; // pivot candidates, published rows
    DevBuf stage;         // tensor-core staging (expanded operands)
    DevBuf krylov;        // GMRES bases
    DevBuf small;         // GMRES small vectors
    DevBuf q;             // F x R FP64 Neumann data (column-major)
    DevBuf small_solve;   // block-substitution claim counter and per-block flags
    DevBuf dinv;          // FP64 inverses of the 64 x 64 diagonal blocks of L and U
    DevBuf field;         // field sources and evaluation points (grow-only)
    DevBuf io;            // device staging of the host-buffer entry points (grow-only)
    DevBuf qeff;          // Neumann data with the admittance term, for the field (grow-only)
    DevBuf grad;          // field gradient: near (point, face) pairs and error word (grow-only)
    int rhs_cached = 1;   // B (N x F) assembled and resident, else matrix-free right-hand sides
    int solve_epoch = 0;  // flag value of the latest substitution launch
    int lu_valid = 0;     // factors match the current operator
};

}  // namespace bb

// ---------------------------------------------------------------------------
// the opaque context
// ---------------------------------------------------------------------------
struct beat_b200_ctx {
    int device = 0;
    int sm_count = 0;
    cudaStream_t stream = nullptr;
    std::string last_error;

    // mesh (host copies)
    int V = 0, F = 0, Q = 0, quad_order = 4, sing_order = 4;
    std::vector<double> verts;    // V x 3
    std::vector<int> faces;       // F x 3, 0-based
    std::vector<double> normals;  // F x 3
    std::vector<double> areas;    // F
    std::vector<double> rule_pts; // Q x 2
    std::vector<double> rule_w;   // Q

    // device mesh data indexed by sorted position (Morton order of centroids)
    bb::DevBuf pos_face;          // F: original face id at each position
    bb::DevBuf pos_qpts64;        // F x Q x 3
    bb::DevBuf pos_qpts32;
    bb::DevBuf pos_normal64;      // F x 3
    bb::DevBuf pos_normal32;
    bb::DevBuf pos_curl64;        // F x 9
    bb::DevBuf pos_curl32;
    bb::DevBuf pos_area64;        // F
    bb::DevBuf pos_area32;
    bb::DevBuf pos_plane32;       // F: plane offset (first rule point) . normal, FP32
    bb::DevBuf pos_gvert;         // F x 3 global vertex ids
    bb::Tiling test_tiles, trial_tiles;
    bb::Tiling sym_tiles;         // square tiles of the symmetric element-pair kernel

    // device mesh data by original face id
    bb::DevBuf d_verts;           // V x 3 double
    bb::DevBuf d_faces;           // F x 3 int (0-based)
    bb::DevBuf d_normals;         // F x 3 double
    bb::DevBuf d_areas;           // F double
    bb::DevBuf d_curls;           // F x 9 double
    bb::DevBuf d_qpts;            // F x Q x 3 double (field sources)
    bb::DevBuf vf_start, vf_face; // vertex -> incident faces (CSR: V + 1 offsets, 3F face ids)

    // symmetry images (0 off, 1 x, 2 xy, 3 ground): the mesh is the
    // fundamental domain, every image reflects the trial elements
    int sym_mode = 0;
    int nimg = 0;
    float img_sign[3][3] = {};    // per image: sign of x, y, z
    float img_det[3] = {};        // per image: determinant (curl factor)
    std::vector<double> in_verts; // set_mesh input as given (re-run on a symmetry change)
    std::vector<int32_t> in_faces;
    int64_t nimg_pairs = 0;       // touching (test, reflected trial) pairs
    bb::DevBuf ip_test, ip_trial, ip_rule, ip_img;   // int per pair
    bb::DevBuf ip_jac, ip_nn;                        // double per pair
    int nweighted = 0;            // vertices on a symmetry plane
    bb::DevBuf rw_vert, rw_weight;  // their ids and orbit weights (2 or 4)

    // admittance boundary condition q = q0 - a (P p), P = face average of P1 p
    bb::DevBuf adm;               // F complex FP64 coefficients a_f
    bool adm_set = false;
    double last_k = 0.0;          // signed wavenumber of the factors in the workspace
    double last_eta = 0.0;        // Burton-Miller coupling (imaginary part) of that solve

    // singular (touching) pairs
    int64_t npairs = 0;
    int nrules = 0;
    bb::DevBuf sp_test, sp_trial, sp_rule;  // int per pair (original face ids)
    bb::DevBuf sp_jac, sp_nn;               // double per pair
    bb::DevBuf rule_start;                  // nrules + 1
    bb::DevBuf rule_data;                   // per point: test xi, eta, trial xi, eta, weight

    int64_t regular_pairs = 0;
    bb::DevBuf status;            // device status word(s)
    bb::DevBuf barrier;           // grid-barrier counters
    bb::Workspace ws;

    cudaEvent_t ev[10] = {};
    // the LU's look-ahead: the trailing update of panel k runs on side_stream
    // (lower priority) while panel k + 1 is factored on `stream`
    cudaStream_t side_stream = nullptr;
    cudaEvent_t la_fork = nullptr, la_join = nullptr;
    // the factorisation's launch sequence as a CUDA graph, replayed while its
    // key (sizes, options and every buffer it touches) stays the same
    cudaGraphExec_t lu_graph = nullptr;
    uint64_t lu_graph_key[12] = {};
    int lu_graph_state = 0;  // 0: none, 2: graph of lu_graph_key ready, 3: that key runs eagerly
    float last_regular_ms = 0.f;
    bool cluster_checked = false;  // can a 16-CTA cluster of the panel kernel be scheduled?
    bool cluster_ok = false;

    // extra solve lanes of a frequency sweep: each a full context (own stream,
    // workspace and status words) over a copy of this mesh
    std::vector<beat_b200_ctx *> lanes;
};

namespace bb {

// context.cu
void set_mesh(beat_b200_ctx *c, int V, const double *verts, int F, const int32_t *faces,
              int quad_order, int sing_order);
// allocates the per-solve buffers and decides the right-hand-side mode
// (BEAT_B200_RHS_*) for the next assembly: ws.rhs_cached
void ensure_workspace(beat_b200_ctx *c, int precision, int R, int rhs_request = BEAT_B200_RHS_AUTO);
// exterior_use_rhs_operator: 1 cached, 0 matrix-free, -1 unknown mode
int rhs_use_operator(int mode, int excitations, int64_t matrix_bytes, int64_t operator_bytes,
                     int64_t available_bytes);
void release_workspace(beat_b200_ctx *c);
int64_t device_bytes(const beat_b200_ctx *c);
int read_status(beat_b200_ctx *c);

// assembly.cu: rule tables in constant memory (fixed per rule size)
void upload_rule_tables(const std::vector<double> &pts, const std::vector<double> &w, int Q);
// context.cu: triangle_rule(T, order) of the reference (weights sum to 1/2)
int triangle_rule(int order, std::vector<double> &pts, std::vector<double> &w);
// assembly.cu: A (row-major N x ld) and B (N x F) in the workspace precision,
// then b = B q (FP64, N x R column-major).  q_dev is F x R FP64 complex.
void assemble(beat_b200_ctx *c, double k, double eta, int precision, int R, const void *q_dev,
              float *ms_total, float *ms_singular);

// lu.cu
void lu_factor(beat_b200_ctx *c, int precision, int nb, int split_terms);
void lu_graph_release(beat_b200_ctx *c);  // drops the captured factorisation (buffers about to change)
void lu_solve_fp64(beat_b200_ctx *c, int R, double *x_dev);          // in place, N x R col-major
void lu_precond_fp32(beat_b200_ctx *c, int R, const double *in, double *out);

// gmres.cu: Y += alpha * M X (M complex row-major rows x K, X/Y FP64 column-major)
template <typename T>
void tall_gemm(cudaStream_t st, int sm_count, const Cx<T> *M, int64_t ld, int rows, int K, const double *X, double *Y,
               int R, double alpha);
struct IrResult {
    int iterations;
    int converged;
    double residual;
};
IrResult gmres_refine(beat_b200_ctx *c, int R, double *x_dev, const double *b_dev, int restart,
                      int max_iters, double rtol);

// adjoint.cu
void apply_admittance_lhs(beat_b200_ctx *c, int precision);  // A += B diag(a) P
// q_eff = q - a (P p) (F x R, FP64 column-major); a copy of q when no admittance is set
void effective_neumann(beat_b200_ctx *c, int R, const double *p_dev, const double *q_dev, double *q_eff);
void lu_solve_adjoint(beat_b200_ctx *c, int R, const double *in, double *out);  // out = A^-H in (stored factors)
void adjoint(beat_b200_ctx *c, double k, int M, const double *dirs_host, int R, const double *p_dev,
             const double *g_dev, double *w_dev, double *ga_dev, const beat_b200_opts &o, IrResult *ir,
             const double **z_out = nullptr);
// shape.cu: gradient with respect to the vertices (V x 3) from the adjoint
// solution z, the solve's p, its effective Neumann data q and g (device)
void shape_gradient(beat_b200_ctx *c, double k, double eta, int M, const double *dirs_dev, int R,
                    const double *p_dev, const double *q_dev, const double *g_dev, const double *z_dev,
                    double *gX_dev);
// gmres.cu: Y (cols x R) += alpha M^H X (X: rows x R); M complex row-major rows x cols
template <typename T>
void tall_gemm_h(cudaStream_t st, int sm_count, const Cx<T> *M, int64_t ld, int rows, int cols, const double *X,
                 double *Y, int R, double alpha);
IrResult gmres_refine_adjoint(beat_b200_ctx *c, int R, double *x_dev, const double *b_dev, int restart,
                              int max_iters, double rtol);

// field.cu
void farfield(beat_b200_ctx *c, double k, int M, const double *dirs_host, int R, const double *p_dev,
              const double *q_dev, double *out_dev, bool far);
// coupled.cu: the coupled FEM-BEM path's combined operators (column-major
// device buffers; element type by precision) and their block products
void assemble_coupled(beat_b200_ctx *c, double k, int precision, void *d_A, void *d_C);
void coupled_blocks(beat_b200_ctx *c, int precision, const void *d_C, int ncols, const int *colptr,
                    const int *rowval, const void *nzval, int64_t nnz, void *d_interface, int nm,
                    const void *d_motion, void *d_motion_out, int np, const void *d_prescribed,
                    void *d_prescribed_out);
// pressure and its gradient, M x 4 x R complex (value, d/dx, d/dy, d/dz)
void field_gradient(beat_b200_ctx *c, double k, int M, const double *pts_host, int R, const double *p_dev,
                    const double *q_dev, double *out_dev);

}  // namespace bb
