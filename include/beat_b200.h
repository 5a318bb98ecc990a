/*
 * beat_b200.h -- C ABI of libbeatb200.so, the B200 (sm_100a) exterior
 * Burton-Miller direct-system solver.
 *
 * Every entry point is extern "C", takes plain pointers and sizes, and returns
 * an int32 status (BEAT_B200_OK = 0).  Nothing here traps or aborts; on error
 * beat_b200_last_error() describes what failed.  A context is not thread safe:
 * one context per request/mesh, called from one host thread (the reference's
 * worker runs one job at a time).
 *
 * Layout conventions (Julia's, so the reference can pass its arrays as is):
 *   vertices  V x 3 float64, one (x,y,z) triple per vertex
 *             (Vector{SVector{3,Float64}} in memory)
 *   faces     F x 3 int32, 1-based vertex numbers, one triple per face
 *   complex   interleaved (re, im) float64 pairs (ComplexF64)
 *   q, p, out column-major: q[f + r*F], p[i + r*N], out[m + r*M]
 *
 * Reference interfaces replaced (paths relative to src/beat_engine/julia_local/):
 *   solve_exterior_direct_cuda            BeatEngineCompiledDriver.jl:870-915
 *   assemble_burton_miller_neumann_system_cuda  src/BeatEngineCudaBurtonMiller.jl:396-580
 *   lu!(system.matrix); factorization \ rhs     BeatEngineCompiledDriver.jl:902-903
 *   evaluate_galerkin_field_cuda          src/BeatEngineCudaField.jl:329-389
 *   build_cuda_regular_assembly_cache /
 *   build_singular_correction_cache       src/BeatEngineCudaRegular.jl:827-893,
 *                                         src/BeatEngineCore.jl:994-1089
 *   reclaim_accelerator_memory!           BeatEngineCompiledDriver.jl:3951
 */
#ifndef BEAT_B200_H
#define BEAT_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define BEAT_B200_ABI_VERSION 2 /* 2: beat_b200_opts.sweep_lanes, beat_b200_sweep_batch */

/* status codes */
#define BEAT_B200_OK 0
#define BEAT_B200_INVALID_ARG 1
#define BEAT_B200_OOM 2
#define BEAT_B200_CUDA_ERROR 3
#define BEAT_B200_NOT_CONVERGED 4 /* iterative refinement missed its tolerance */
#define BEAT_B200_TIMEOUT 5       /* a device-side wait ran out of its budget */
#define BEAT_B200_NO_DEVICE 6
#define BEAT_B200_STATE 7         /* call order (e.g. solve before set_mesh) */
#define BEAT_B200_SINGULAR 8      /* exact zero pivot */

/* precision forms */
#define BEAT_B200_FP64 0          /* FP64 assembly, FP64 LU, FP64 solve */
#define BEAT_B200_MIXED_FP32_IR 1 /* FP32 regular assembly (FP64 singular),
                                     FP32 complex LU with TF32 tensor-core
                                     trailing updates, FP64 GMRES refinement */

typedef struct beat_b200_ctx beat_b200_ctx;

typedef struct {
    int32_t precision;      /* BEAT_B200_FP64 or BEAT_B200_MIXED_FP32_IR */
    int32_t ir_restart;     /* GMRES restart length (20) */
    int32_t ir_max_iters;   /* total GMRES iterations allowed (200) */
    int32_t lu_split_terms; /* split products per trailing update: 3 (FP16 high x high + high x low +
                               low x high, about FP32 accuracy) or 1 (FP16 high parts only) (3) */
    double ir_rtol;         /* relative residual target of the refinement (1e-10) */
    int32_t lu_block;       /* LU panel width; 0 = tuned default */
    int32_t flags;          /* BEAT_B200_FLAG_* bits, 0 by default */
    int32_t sweep_lanes;    /* solve lanes of a sweep (1..16); 0 = default: 6 in the mixed
                               form, 4 in FP64 (always capped by free device memory) */
} beat_b200_opts;

/* opts.flags: return the mixed form's direct FP32-LU solution without the
 * GMRES refinement (diagnostics; the result is then FP32-LU accurate only) */
#define BEAT_B200_FLAG_NO_REFINE 1

/* Right-hand-side modes (exterior_rhs_policy.jl:15-44).  Cached: the P1 x DP0
 * mapping B (N x F) is assembled with the system and b = B q is one tall
 * product; B stays resident for the admittance term and the adjoint.
 * Matrix-free: the element-pair kernels add B-tile x q straight into b, so
 * no N x F array exists; unlike the reference's matrix_free path (one pair
 * integration per excitation) this is one pass for every column.  Auto: the
 * reference's rule, cached from two excitations on when the system matrix,
 * B and a 512 MiB margin fit in the free device memory plus what the context
 * already holds; an admittance always needs B.  If B cannot be allocated the
 * solve falls back to matrix-free, as the reference does. */
#define BEAT_B200_RHS_AUTO 0
#define BEAT_B200_RHS_MATRIX_FREE 1
#define BEAT_B200_RHS_CACHED 2
/* opts.flags bits 1-2 request a mode (both clear = auto, both set = invalid) */
#define BEAT_B200_FLAG_RHS_MATRIX_FREE 2
#define BEAT_B200_FLAG_RHS_CACHED 4
/* opts.flags: a mixed-form solve whose refinement misses its tolerance
 * returns BEAT_B200_NOT_CONVERGED instead of falling back.  By default the
 * frequency is then solved again in the FP64 form (the reference's dense solve
 * does the same: BeatEngineDenseSolve.jl:1067-1085, non-convergence is
 * reported, never raised) and diag.precision reports BEAT_B200_FP64 with
 * diag.ir_converged = 0 and the failed refinement's iterations and residual. */
#define BEAT_B200_FLAG_NO_FALLBACK 8

/* Test hook (environment, read at every device allocation):
 * BEAT_B200_FAULT_OOM_BYTES=n makes each allocation of n bytes or more fail
 * as out of memory, to exercise the out-of-memory paths (the right-hand-side
 * mapping's fallback, BEAT_B200_OOM) without exhausting the device. */

typedef struct {
    double assembly_ms;     /* regular + singular + identity + RHS */
    double singular_ms;     /* Duffy pass alone (part of assembly_ms) */
    double regular_ms;      /* element-pair kernel alone (part of assembly_ms) */
    double lu_ms;
    double solve_ms;        /* triangular solves of the direct solve */
    double ir_ms;           /* GMRES refinement (mixed form) */
    double field_ms;
    int32_t ir_iterations;
    int32_t ir_converged;
    double ir_residual;     /* final max over columns of ||b - A x|| / ||b|| */
    int64_t regular_pairs;
    int64_t singular_pairs;
    int32_t precision;
    int32_t lu_block;
    int32_t lu_split_terms;
    int32_t rhs_mode;       /* BEAT_B200_RHS_MATRIX_FREE or _CACHED: the mode that ran (the
                               mapping then held N x F x 8 (mixed) or 16 (FP64) bytes) */
} beat_b200_diag;

/* ABI check: returns BEAT_B200_ABI_VERSION. */
int32_t beat_b200_abi_version(void);

/* Fill opts with the defaults listed above. */
void beat_b200_default_opts(beat_b200_opts *opts);

/* One context per mesh: device buffers, streams, tuned tile choices. */
int32_t beat_b200_create(int32_t device, beat_b200_ctx **out);
int32_t beat_b200_destroy(beat_b200_ctx *ctx);
const char *beat_b200_last_error(const beat_b200_ctx *ctx);

/* Upload a mesh and build everything that depends only on it: element
 * geometry, the order-`quad_order` triangle rule (triangle_rule), touching
 * pairs with orientation-remapped Duffy rules of order `singular_order`
 * (build_singular_correction_cache), tiles for the element-pair kernel and
 * the field source cache.  Host arrays are copied. */
int32_t beat_b200_set_mesh(beat_b200_ctx *ctx, int32_t V, const double *vertices, int32_t F,
                           const int32_t *faces, int32_t quad_order, int32_t singular_order);

/* Assemble, factor once, solve all R right-hand sides (and refine in the
 * mixed form).  k_signed = outgoing_wavenumber(k), eta_im = imag of
 * burton_miller_coupling(k).  q: F x R Neumann data; p_out: N x R pressures.
 * opts may be NULL (defaults), diag may be NULL.  The factors and the
 * operator stay on the device for beat_b200_field / beat_b200_farfield. */
int32_t beat_b200_solve(beat_b200_ctx *ctx, double k_signed, double eta_im, int32_t R,
                        const double *q, const beat_b200_opts *opts, double *p_out,
                        beat_b200_diag *diag);

/* As beat_b200_solve with q and p_out in device memory (same layouts). */
int32_t beat_b200_solve_device(beat_b200_ctx *ctx, double k_signed, double eta_im, int32_t R,
                               const void *d_q, const beat_b200_opts *opts, void *d_p_out,
                               beat_b200_diag *diag);

/* Pressure at M observation points (M x 3) for R columns of boundary
 * pressure p (N x R) and Neumann data q (F x R): out is M x R. */
int32_t beat_b200_field(beat_b200_ctx *ctx, double k_signed, int32_t M, const double *points,
                        int32_t R, const double *p, const double *q, double *out);

/* Far-field pattern p_inf(d) = lim r exp(-i k r) p(r d) at M directions. */
int32_t beat_b200_farfield(beat_b200_ctx *ctx, double k_signed, int32_t M, const double *dirs,
                           int32_t R, const double *p, const double *q, double *out);

/* Pressure and its gradient at M observation points (pressure_gradient_v1):
 * out is M x 4 x R complex, column-major, component d (0 = value, 1..3 =
 * d/dx, d/dy, d/dz) of column r at out[m + M (d + 4 r)].  The regular
 * quadrature sum is corrected, for every face (and symmetry image) whose
 * centroid lies within 3 face diameters of a point, by adaptive subdivision
 * with the fourth-order rule down to depth 12; a point closer to the boundary
 * than that resolves gives BEAT_B200_INVALID_ARG.  Replaces
 * evaluate_galerkin_field_gradient_cuda (src/BeatEngineCudaFieldGradient.jl:
 * 20-38) with correct_field_gradient! (src/BeatEngineFieldGradient.jl:45-71),
 * which the reference runs on host threads; here both parts run on the GPU.
 * The reference requires the fourth-order rule for gradients
 * (BeatEngineCompiledDriver.jl:4168-4170): set_mesh with quad_order 4. */
int32_t beat_b200_field_gradient(beat_b200_ctx *ctx, double k_signed, int32_t M, const double *points,
                                 int32_t R, const double *p, const double *q, double *out);

/* As beat_b200_field_gradient with p, q and out in device memory. */
int32_t beat_b200_field_gradient_device(beat_b200_ctx *ctx, double k_signed, int32_t M,
                                        const double *points, int32_t R, const void *d_p,
                                        const void *d_q, void *d_out);

/* Device-pointer variants of the two evaluators (points/dirs stay host). */
int32_t beat_b200_farfield_device(beat_b200_ctx *ctx, double k_signed, int32_t M,
                                  const double *dirs, int32_t R, const void *d_p,
                                  const void *d_q, void *d_out);

/* Assemble only and copy the system out (N x N column-major A, N x R b) in
 * FP64, whatever the precision form; A_out or b_out may be NULL. */
int32_t beat_b200_assemble(beat_b200_ctx *ctx, double k_signed, double eta_im, int32_t R,
                           const double *q, int32_t precision, double *A_out, double *b_out);

/* Free the per-solve workspaces (system matrix, factors, Krylov vectors);
 * the mesh stays.  The next solve reallocates them. */
int32_t beat_b200_release_workspace(beat_b200_ctx *ctx);

/* Coupled FEM-BEM combined BEM operators, replacing
 * assemble_coupled_burton_miller_cuda (src/BeatEngineCudaCoupledBurtonMiller.jl:
 * 537-593): A = 1/2 M - D + alpha H (N x N) and C = S + alpha (K' + 1/2 M_p1dp0)
 * (N x F), alpha = i / k_signed (burton_miller_coupling), with the context's
 * symmetry images and orbit row weights; no admittance term (the coupled
 * path's admittance lives on the FEM side).  Written column-major into the
 * caller's device buffers d_A and d_C (either may be NULL), complex float in
 * the mixed form (FP32 regular quadrature, FP64 touching pairs) or complex
 * double in the FP64 form.  Overwrites the context's system (a later adjoint
 * needs a new solve). */
int32_t beat_b200_assemble_coupled_device(beat_b200_ctx *ctx, double k_signed, int32_t precision,
                                          void *d_A, void *d_C);

/* build_cuda_combined_bem_blocks (src/BeatEngineCudaCoupledBurtonMiller.jl:
 * 595-640) on a column-major C (N x F) from beat_b200_assemble_coupled_device:
 * interface = C Q for the F x ncols sparse interface map Q in CSC form
 * (colptr: ncols + 1 entries, rowval / nzval: nnz entries, 1-based as Julia
 * stores them), motion_out = C motion (F x nmotion), prescribed_out =
 * -C prescribed (F x nprescribed).  All device buffers, column-major, of the
 * precision's complex type; an index outside the map gives
 * BEAT_B200_INVALID_ARG. */
int32_t beat_b200_coupled_blocks_device(beat_b200_ctx *ctx, int32_t precision, const void *d_C,
                                        int32_t ncols, const int32_t *d_colptr,
                                        const int32_t *d_rowval, const void *d_nzval, int64_t nnz,
                                        void *d_interface, int32_t nmotion, const void *d_motion,
                                        void *d_motion_out, int32_t nprescribed,
                                        const void *d_prescribed, void *d_prescribed_out);

/* exterior_use_rhs_operator (exterior_rhs_policy.jl:31-44): 1 when the
 * cached mapping is used for `excitations` right-hand sides with a system
 * matrix of matrix_bytes, a mapping of operator_bytes and available_bytes of
 * device memory, 0 when matrix-free, -1 for an unknown mode.  Pure host
 * logic: needs no device and no context. */
int32_t beat_b200_rhs_use_operator(int32_t mode, int32_t excitations, int64_t matrix_bytes,
                                   int64_t operator_bytes, int64_t available_bytes);

/* Bytes of device memory the context holds right now. */
int64_t beat_b200_device_bytes(const beat_b200_ctx *ctx);

/* No counterpart in the reference.  Solve R more right-hand sides with the
 * factors of the last beat_b200_solve on this context, allocating no memory:
 * for callers whose device memory belongs to their own pool (so a
 * library-side cudaMalloc would bypass its accounting) or that cannot afford
 * cudaMalloc/cudaFree on their thread.  d_b (input) and d_x (output) are
 * non-overlapping device buffers of N x R complex doubles, column-major.
 * The factors must come from beat_b200_solve or beat_b200_solve_device:
 * after a sweep (whose lanes leave no factors the caller can name), a failed
 * solve or a change of mesh, symmetry or admittance the call returns
 * BEAT_B200_STATE.  The FP64
 * form gives the exact LU solution; the mixed form gives its FP32-LU
 * solution without the GMRES refinement.  Limit: N <= 262144.  Its scratch
 * is a 16 KB static device array that every GPU loading the library holds
 * until exit, shared by all calls on that device: calls whose work overlaps
 * on the GPU race and must be serialised by the caller.  The first call on a
 * device looks up that array's address and keeps it for the life of the
 * process; a cudaDeviceReset of that device invalidates it, so do not call
 * this entry point on a device after resetting it.  Make the first call on a
 * device before any stream capture.  Synchronises the context's stream
 * before returning. */
int32_t beat_b200_resolve_noalloc(beat_b200_ctx *ctx, int32_t R, const void *d_b, void *d_x);

/* Frequency sweep: nfreq independent solves of this mesh, each followed by
 * its far field at M directions (M = 0: none).  Replaces the per-frequency
 * loop of solve_exterior_request (BeatEngineCompiledDriver.jl:1269-1592),
 * which calls solve_exterior_direct_cuda once per frequency (:1338) and
 * overlaps the next frequency's assembly with the current solve only on its
 * Metal path (start_sweep_assembly_pipeline, :1265).  Frequencies are
 * pipelined over up to six solve lanes, four in the FP64 form (each with its
 * own stream and workspace, the further ones created on first use with a
 * copy of the mesh;
 * no more lanes than frequencies, nor than have room for a system matrix in
 * the free device memory), one host thread per lane: one frequency's
 * assembly runs beside the others' factorisations.
 * Frequency f uses k_signed[f], eta_im[f], q + f F R, p_out + f N R and
 * ff_out + f M R (complex doubles, column-major slices as in
 * beat_b200_solve); diags (NULL or nfreq entries) receives each solve's
 * diagnostics.  The first failing frequency's status is returned. */
int32_t beat_b200_sweep(beat_b200_ctx *ctx, int32_t nfreq, const double *k_signed,
                        const double *eta_im, int32_t R, const double *q,
                        const beat_b200_opts *opts, double *p_out, int32_t M, const double *dirs,
                        double *ff_out, beat_b200_diag *diags);

/* As beat_b200_sweep with q, p_out and ff_out in device memory (dirs, k and
 * eta stay host). */
int32_t beat_b200_sweep_device(beat_b200_ctx *ctx, int32_t nfreq, const double *k_signed,
                               const double *eta_im, int32_t R, const void *d_q,
                               const beat_b200_opts *opts, void *d_p, int32_t M,
                               const double *dirs, void *d_ff, beat_b200_diag *diags);

/* Batched sweep: the frequency sweeps of nmesh meshes (meshes of uneven
 * size, e.g. the variants of a design) as one job list over one set of solve
 * lanes.  The reference runs its meshes' sweeps one after another, each
 * overlapping assembly and solve only on Metal (start_sweep_assembly_pipeline
 * / take_sweep_assembly!, src/BeatEngineCore.jl:1451-1599, called from
 * BeatEngineCompiledDriver.jl:1222-1268).  Here mesh m (context ctxs[m], on
 * one device, each with its mesh set) has nfreq[m] frequencies with
 * k_signed[m][f], eta_im[m][f], R[m] columns, q[m] + f F_m R_m, p_out[m] +
 * f N_m R_m and ff_out[m] + f M R_m (layouts as in beat_b200_sweep), options
 * opts[m] (opts NULL: defaults), diagnostics diags[m][f] (diags or diags[m]
 * may be NULL).  Every (mesh, frequency) is one job; the lanes (opts[0]'s
 * sweep_lanes, capped by the free memory for every mesh) take the jobs in
 * decreasing order of N^3, the factorisation's cost, each the next one when
 * it finishes one.  Errors are reported on ctxs[0]; the first failing job in
 * mesh-major numbering gives the status. */
int32_t beat_b200_sweep_batch(int32_t nmesh, beat_b200_ctx *const *ctxs, const int32_t *nfreq,
                              const double *const *k_signed, const double *const *eta_im,
                              const int32_t *R, const double *const *q,
                              const beat_b200_opts *opts, double *const *p_out, int32_t M,
                              const double *dirs, double *const *ff_out,
                              beat_b200_diag *const *diags);

/* As beat_b200_sweep_batch with every mesh's q, p and far field in device
 * memory. */
int32_t beat_b200_sweep_batch_device(int32_t nmesh, beat_b200_ctx *const *ctxs,
                                     const int32_t *nfreq, const double *const *k_signed,
                                     const double *const *eta_im, const int32_t *R,
                                     const void *const *d_q, const beat_b200_opts *opts,
                                     void *const *d_p, int32_t M, const double *dirs,
                                     void *const *d_ff, beat_b200_diag *const *diags);

/* Symmetry images (the reference's symmetry_mode: normalized_symmetry_mode,
 * symmetry_transforms, BeatEngineCore.jl:448-482; image passes and
 * image-singular deltas, src/BeatEngineCudaBurtonMiller.jl:475-493,
 * src/BeatEngineCudaSingular.jl:140-278,590-897; orbit row weights,
 * BeatEngineCore.jl:563-582): 0 off, 1 x (mesh in x >= 0, mirror x), 2 xy
 * (mesh in x, y >= 0), 3 ground (rigid ground plane y = 0).  The mesh is the
 * fundamental domain: vertices within max(1e-9, 1e-6 x bounding-box
 * diagonal) of an active plane are snapped onto it, a vertex on the negative
 * side is an error.  Solves, fields, sweeps and the adjoint include the
 * images.  May be called before or after beat_b200_set_mesh (after: the mesh
 * set-up is rebuilt). */
int32_t beat_b200_set_symmetry(beat_b200_ctx *ctx, int32_t mode);

/* Admittance boundary condition (row a19 of the path; the reference's
 * exterior solve has none, its admittance is a coupled-FEM wall model,
 * BeatEngineCoupled.jl:594-623).  With coefficients a (F complex, one per
 * face) every later solve on this context uses q = q0 - a (P p), where P is
 * the face average of the P1 pressure:  (A + B diag(a) P) p = B q0, and the
 * field evaluators apply the same q.  For a normal-velocity admittance Y
 * (v = v0 - Y p, exp(-i omega t)) pass a = neumann_scale * Y.  a = NULL
 * clears it (the reference's solve). */
int32_t beat_b200_set_admittance(beat_b200_ctx *ctx, const double *a);

/* Adjoint gradients of a real far-field functional J after a solve on this
 * context with the same k_signed (row a19; no reference counterpart):
 * g = dJ/d conj(p_inf) at the M directions (M x R), p the solve's pressures
 * (N x R).  Returns w_out = dJ/d conj(q0) (F x R: the gradient with respect
 * to the Neumann data; dJ = 2 Re sum conj(w) dq0) and, if ga_out is not NULL,
 * ga_out = dJ/d conj(a) (F).  The conjugate-transposed system uses the
 * stored factors (FP64 form) or the FP32 factors plus FP64 GMRES refinement
 * on the stored operator (mixed form, opts' tolerances).  Gradients with
 * respect to the vertices are not provided. */
int32_t beat_b200_adjoint(beat_b200_ctx *ctx, double k_signed, int32_t M, const double *dirs,
                          int32_t R, const double *p, const double *g, const beat_b200_opts *opts,
                          double *w_out, double *ga_out);

/* beat_b200_adjoint plus the gradient with respect to the vertex positions:
 * gX_out (V x 3 doubles, the layout of set_mesh's vertices) is dJ/dX of the
 * same real functional, by reverse-mode differentiation of the discrete
 * assembly (regular and Duffy element pairs, identity), the far field and,
 * with an admittance, its Neumann term.  q is the Neumann data (F x R) of the
 * last solve, which the shape derivative needs besides p; w_out and ga_out
 * are as in beat_b200_adjoint and may be NULL.  With symmetry images the
 * image passes, touching image pairs and image far-field sources are
 * differentiated too; in the x and xy modes a vertex on a symmetry plane must
 * stay on it, so the component of its gradient normal to that plane is zero.
 * No counterpart in the reference. */
int32_t beat_b200_adjoint_shape(beat_b200_ctx *ctx, double k_signed, int32_t M, const double *dirs,
                                int32_t R, const double *p, const double *q, const double *g,
                                const beat_b200_opts *opts, double *w_out, double *ga_out,
                                double *gX_out);

/* The CUDA stream (cudaStream_t) every kernel of this context is launched
 * on, so a caller can order its own work or record timing events on it.
 * Entry points return only after their work on it has completed. */
void *beat_b200_stream(const beat_b200_ctx *ctx);

#ifdef __cplusplus
}
#endif
#endif /* BEAT_B200_H */
