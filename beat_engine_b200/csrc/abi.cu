// abi.cu -- the extern "C" entry points of libbeatb200.so (include/beat_b200.h).
//
// The solve entry replaces solve_exterior_direct_cuda
// (BeatEngineCompiledDriver.jl:870-915): assemble the fused Burton-Miller
// system for all R excitations, factor once, solve every column; the field
// entries replace evaluate_galerkin_field_cuda (src/BeatEngineCudaField.jl:329-389).
// Every entry converts exceptions to a status code and keeps the message for
// beat_b200_last_error; nothing here aborts.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <algorithm>
#include <atomic>
#include <new>
#include <thread>

#include "internal.cuh"

using namespace bb;

namespace {

template <typename F> int32_t guarded(beat_b200_ctx *c, F &&fn) {
    if (!c) return BEAT_B200_INVALID_ARG;
    try {
        BB_CUDA(cudaSetDevice(c->device));
        fn();
        c->last_error.clear();
        return BEAT_B200_OK;
    } catch (const Error &e) {
        c->last_error = e.msg;
        cudaGetLastError();
        return e.code;
    } catch (const std::bad_alloc &) {
        c->last_error = "host allocation failed";
        return BEAT_B200_OOM;
    } catch (...) {
        c->last_error = "unexpected exception";
        return BEAT_B200_CUDA_ERROR;
    }
}

constexpr int MAX_SWEEP_LANES = 16;

beat_b200_opts resolve_opts(const beat_b200_opts *o) {
    beat_b200_opts r;
    beat_b200_default_opts(&r);
    if (o) r = *o;
    if (r.ir_restart <= 0) r.ir_restart = 20;
    if (r.ir_max_iters <= 0) r.ir_max_iters = 200;
    if (!(r.ir_rtol > 0)) r.ir_rtol = 1e-10;
    if (r.lu_split_terms != 1 && r.lu_split_terms != 3) r.lu_split_terms = 3;
    BB_REQUIRE(r.precision == BEAT_B200_FP64 || r.precision == BEAT_B200_MIXED_FP32_IR, BEAT_B200_INVALID_ARG,
               "unknown precision form");
    BB_REQUIRE(r.sweep_lanes >= 0 && r.sweep_lanes <= MAX_SWEEP_LANES, BEAT_B200_INVALID_ARG,
               "sweep_lanes must be 0 (default) or 1.." + std::to_string(MAX_SWEEP_LANES));
    if (r.lu_block <= 0) r.lu_block = 128;  // measured best for both forms at N = 10,242
    BB_REQUIRE(r.lu_block == 32 || r.lu_block == 64 || r.lu_block == 128 || r.lu_block == 256,
               BEAT_B200_INVALID_ARG, "lu_block must be 32, 64, 128 or 256");
    BB_REQUIRE((r.flags & (BEAT_B200_FLAG_RHS_MATRIX_FREE | BEAT_B200_FLAG_RHS_CACHED)) !=
                   (BEAT_B200_FLAG_RHS_MATRIX_FREE | BEAT_B200_FLAG_RHS_CACHED),
               BEAT_B200_INVALID_ARG, "flags request both right-hand-side modes");
    return r;
}

// the right-hand-side mode the flags request (BEAT_B200_RHS_*)
static int rhs_request(const beat_b200_opts &o) {
    if (o.flags & BEAT_B200_FLAG_RHS_MATRIX_FREE) return BEAT_B200_RHS_MATRIX_FREE;
    if (o.flags & BEAT_B200_FLAG_RHS_CACHED) return BEAT_B200_RHS_CACHED;
    return BEAT_B200_RHS_AUTO;
}

// row-major (ld) -> column-major N x N FP64
template <typename T>
__global__ void export_matrix_kernel(const Cx<T> *A, int64_t ld, int n, double2 *out) {
    __shared__ double2 tile[32][33];
    const int bx = blockIdx.x * 32, by = blockIdx.y * 32;
    for (int i = threadIdx.y; i < 32; i += blockDim.y) {
        const int r = by + i, cc = bx + threadIdx.x;
        if (r < n && cc < n) {
            const Cx<T> v = A[(int64_t)r * ld + cc];
            tile[i][threadIdx.x] = make_double2((double)v.re, (double)v.im);
        }
    }
    __syncthreads();
    for (int i = threadIdx.y; i < 32; i += blockDim.y) {
        const int cc = bx + i, r = by + threadIdx.x;
        if (r < n && cc < n) out[(size_t)cc * n + r] = tile[threadIdx.x][i];
    }
}

void solve_core(beat_b200_ctx *c, double k, double eta, int R, const double *d_q, const beat_b200_opts &o,
                double *d_x, beat_b200_diag *diag) {
    BB_REQUIRE(c->F > 0, BEAT_B200_STATE, "no mesh: call beat_b200_set_mesh first");
    BB_REQUIRE(R >= 1, BEAT_B200_INVALID_ARG, "R must be >= 1");
    BB_REQUIRE(std::isfinite(k) && k != 0.0 && std::isfinite(eta), BEAT_B200_INVALID_ARG,
               "wavenumber must be finite and nonzero");
    // the factors are overwritten from here on (a workspace change may free
    // them): they count as current again only once this factorisation has
    // finished without a timeout or a zero pivot
    c->ws.lu_valid = 0;
    ensure_workspace(c, o.precision, R, rhs_request(o));
    Workspace &w = c->ws;
    const int n = c->V;
    float ms_asm = 0, ms_sing = 0, ms_lu = 0, ms_solve = 0, ms_ir = 0;
    assemble(c, k, eta, o.precision, R, d_q, &ms_asm, &ms_sing);
    apply_admittance_lhs(c, o.precision);  // A += B diag(a) P when an admittance is set
    if (o.precision != BEAT_B200_FP64)
        BB_CUDA(cudaMemcpyAsync(w.Aop.p, w.A.p, (size_t)n * w.ld * 8, cudaMemcpyDeviceToDevice, c->stream));
    BB_CUDA(cudaEventRecord(c->ev[4], c->stream));
    lu_factor(c, o.precision, o.lu_block, o.lu_split_terms);
    BB_CUDA(cudaEventRecord(c->ev[5], c->stream));
    const int st = read_status(c);
    c->last_k = k;
    c->last_eta = eta;
    BB_REQUIRE(!(st & DEV_BARRIER_TIMEOUT), BEAT_B200_TIMEOUT, "LU panel: grid barrier ran out of its wait budget");
    BB_REQUIRE(!(st & DEV_ZERO_PIVOT), BEAT_B200_SINGULAR, "LU: exact zero pivot (singular system)");
    w.lu_valid = 1;
    IrResult ir{0, 1, 0.0};
    if (o.precision == BEAT_B200_FP64) {
        BB_CUDA(cudaMemcpyAsync(d_x, w.b.p, (size_t)n * R * 16, cudaMemcpyDeviceToDevice, c->stream));
        lu_solve_fp64(c, R, d_x);
        BB_CUDA(cudaEventRecord(c->ev[6], c->stream));
        BB_CUDA(cudaEventRecord(c->ev[7], c->stream));
    } else {
        lu_precond_fp32(c, R, w.b.as<double>(), d_x);
        BB_CUDA(cudaEventRecord(c->ev[6], c->stream));
        if (o.flags & BEAT_B200_FLAG_NO_REFINE)
            ir = IrResult{0, 0, -1.0};
        else
            ir = gmres_refine(c, R, d_x, w.b.as<double>(), o.ir_restart, o.ir_max_iters, o.ir_rtol);
        BB_CUDA(cudaEventRecord(c->ev[7], c->stream));
    }
    BB_CUDA(cudaEventSynchronize(c->ev[7]));
    const int st2 = read_status(c);
    BB_REQUIRE(!(st2 & DEV_BARRIER_TIMEOUT), BEAT_B200_TIMEOUT,
               "triangular solve: a block wait ran out of its budget");
    BB_CUDA(cudaEventElapsedTime(&ms_lu, c->ev[4], c->ev[5]));
    BB_CUDA(cudaEventElapsedTime(&ms_solve, c->ev[5], c->ev[6]));
    BB_CUDA(cudaEventElapsedTime(&ms_ir, c->ev[6], c->ev[7]));
    if (diag) {
        diag->assembly_ms = ms_asm;
        diag->singular_ms = ms_sing;
        diag->regular_ms = c->last_regular_ms;
        diag->lu_ms = ms_lu;
        diag->solve_ms = ms_solve;
        diag->ir_ms = ms_ir;
        diag->field_ms = 0;
        diag->ir_iterations = ir.iterations;
        diag->ir_converged = ir.converged;
        diag->ir_residual = ir.residual;
        diag->regular_pairs = c->regular_pairs;
        diag->singular_pairs = c->npairs;
        diag->precision = o.precision;
        diag->lu_block = o.lu_block;
        diag->lu_split_terms = o.lu_split_terms;
        diag->rhs_mode = w.rhs_cached ? BEAT_B200_RHS_CACHED : BEAT_B200_RHS_MATRIX_FREE;
    }
    if (ir.converged || o.precision == BEAT_B200_FP64 || (o.flags & BEAT_B200_FLAG_NO_REFINE)) return;
    BB_REQUIRE(!(o.flags & BEAT_B200_FLAG_NO_FALLBACK), BEAT_B200_NOT_CONVERGED,
               "GMRES refinement missed its tolerance (worst relative residual " + std::to_string(ir.residual) + ")");
    // the refinement did not converge: solve this frequency in the FP64 form
    // (non-convergence reported in diag, not raised)
    beat_b200_opts o64 = o;
    o64.precision = BEAT_B200_FP64;
    o64.lu_block = 128;
    solve_core(c, k, eta, R, d_q, o64, d_x, diag);
    if (diag) {
        diag->ir_iterations = ir.iterations;
        diag->ir_converged = 0;
        diag->ir_residual = ir.residual;
    }
}

// ---------------------------------------------------------------------------
// frequency sweep over solve lanes
// ---------------------------------------------------------------------------
// lanes per sweep, measured on B200 at F = 20,480, R = 16, 24 frequencies:
// mixed form 4 lanes 14.5, 6 lanes 15.0, 8 lanes 14.8 freq-solves/s (the
// end-to-end sweep 15.0, 15.8, 15.9); FP64 form 4 lanes 4.19, 6 lanes 3.49
// (its lanes are twice the size and its assembly alone fills the GPU)
constexpr int SWEEP_LANES = 6, SWEEP_LANES_FP64 = 4;

// lane i of c (lane 0 is c itself); created on first use with c's mesh
beat_b200_ctx *sweep_lane(beat_b200_ctx *c, int i) {
    if (i == 0) return c;
    while ((int)c->lanes.size() < i) {
        beat_b200_ctx *l = nullptr;
        const int32_t st = beat_b200_create(c->device, &l);
        BB_REQUIRE(st == BEAT_B200_OK, st, "sweep: could not create a solve lane");
        c->lanes.push_back(l);
        l->sym_mode = c->sym_mode;
        std::vector<int32_t> faces1(c->faces.size());
        for (size_t j = 0; j < faces1.size(); ++j) faces1[j] = c->faces[j] + 1;
        BB_CUDA(cudaSetDevice(c->device));
        set_mesh(l, c->V, c->verts.data(), c->F, faces1.data(), c->quad_order, c->sing_order);
    }
    return c->lanes[i - 1];
}

static int64_t held_matrix_bytes(const beat_b200_ctx *l) {
    return (int64_t)(l->ws.A.bytes + l->ws.Aop.bytes + l->ws.B.bytes);
}

// device bytes one lane of context c needs for a solve with these options
static int64_t lane_bytes(const beat_b200_ctx *c, const beat_b200_opts &o, int R) {
    const bool fp64 = o.precision == BEAT_B200_FP64;
    const int64_t ld = ((int64_t)c->V + 127) / 128 * 128;
    const int64_t csz = fp64 ? 16 : 8;
    const int req = rhs_request(o);
    const bool may_cache = c->adm_set || req == BEAT_B200_RHS_CACHED || (req == BEAT_B200_RHS_AUTO && R >= 2);
    return (int64_t)c->V * ld * csz * (fp64 ? 1 : 2) + (may_cache ? (int64_t)c->V * c->F * csz : 0);
}

static int default_lanes(const beat_b200_opts &o) {
    if (o.sweep_lanes > 0) return o.sweep_lanes;
    return o.precision == BEAT_B200_FP64 ? SWEEP_LANES_FP64 : SWEEP_LANES;
}

// How many lanes a sweep over the contexts cs (one per mesh) runs: the
// requested count (default_lanes of the first mesh's options), no more than
// there are jobs, and only as many as can hold every mesh's system matrix
// (with the FP32 operator copy in the mixed form, and the N x F mapping when
// the right-hand sides may be cached) beside a 512 MiB margin in the free
// device memory; buffers a lane already holds count as available.  Lane 0
// always runs.
static int lane_count(const std::vector<beat_b200_ctx *> &cs, const std::vector<int> &R, int njobs,
                      const beat_b200_opts *o) {
    const int want = std::min(default_lanes(o[0]), njobs);
    if (want <= 1) return 1;
    size_t free_b = 0, total_b = 0;
    BB_CUDA(cudaMemGetInfo(&free_b, &total_b));
    const int64_t margin = 512ll << 20;
    int64_t avail = (int64_t)free_b;
    for (size_t m = 0; m < cs.size(); ++m)  // lane 0 is the contexts themselves
        avail -= std::max<int64_t>(0, lane_bytes(cs[m], o[m], R[m]) - held_matrix_bytes(cs[m]));
    int lanes = 1;
    for (int i = 1; i < want; ++i) {
        int64_t need = margin;
        for (size_t m = 0; m < cs.size(); ++m) {
            const beat_b200_ctx *l = i - 1 < (int)cs[m]->lanes.size() ? cs[m]->lanes[i - 1] : nullptr;
            need += std::max<int64_t>(0, lane_bytes(cs[m], o[m], R[m]) - (l ? held_matrix_bytes(l) : 0));
        }
        if (need > avail) break;
        avail -= need;
        ++lanes;
    }
    return lanes;
}

static int sweep_lane_count(beat_b200_ctx *c, int nfreq, const beat_b200_opts &o, int R) {
    return lane_count({c}, {R}, nfreq, &o);
}

// Runs work(lane, job) for the jobs in `order`, one host thread per lane (lane
// 0 on the calling thread).  Each lane takes the next unclaimed job from a
// shared counter when it finishes one, so a lane that drew cheap jobs does
// not idle while another still holds a queue.  After a failure no lane starts
// another job; the first error (by job number, named `what` in the message)
// is rethrown after every lane has stopped, with stream_of(lane, job)
// synchronised for the failed job.
template <typename W, typename S>
void run_jobs(beat_b200_ctx *c, int L, const std::vector<int> &order, const char *what, W &&work, S &&stream_of) {
    const int njobs = (int)order.size();
    std::vector<Error> err(L);
    std::vector<int> err_job(L, -1);
    std::atomic<int> next{0};
    std::atomic<bool> failed{false};
    auto body = [&](int i) {
        try {
            BB_CUDA(cudaSetDevice(c->device));
            for (int t = next.fetch_add(1); t < njobs && !failed.load(); t = next.fetch_add(1)) {
                err_job[i] = order[t];
                work(i, order[t]);
            }
            err_job[i] = -1;
        } catch (const Error &e) {
            err[i] = e;
        } catch (const std::bad_alloc &) {
            err[i] = Error{BEAT_B200_OOM, "host allocation failed"};
        } catch (...) {
            err[i] = Error{BEAT_B200_CUDA_ERROR, "unexpected exception"};
        }
        if (err_job[i] >= 0) {
            failed.store(true);
            cudaStream_t st = stream_of(i, err_job[i]);
            if (st) cudaStreamSynchronize(st);
        }
    };
    std::vector<std::thread> th;
    for (int i = 1; i < L; ++i) th.emplace_back(body, i);
    body(0);
    for (auto &t : th) t.join();
    int first = -1;
    for (int i = 0; i < L; ++i)
        if (err_job[i] >= 0 && (first < 0 || err_job[i] < err_job[first])) first = i;
    if (first >= 0)
        throw Error{err[first].code, std::string(what) + " " + std::to_string(err_job[first]) + ": " + err[first].msg};
}

// The lanes of context c for a sweep of L lanes (lane 0 is c itself), with
// c's admittance copied to the others.
static std::vector<beat_b200_ctx *> prepare_lanes(beat_b200_ctx *c, int L) {
    std::vector<beat_b200_ctx *> lane(L);
    for (int i = 0; i < L; ++i) lane[i] = sweep_lane(c, i);
    for (int i = 1; i < L; ++i) {  // the lanes solve with this context's admittance
        lane[i]->adm_set = c->adm_set;
        if (c->adm_set) {
            lane[i]->adm.alloc(c->adm.bytes);
            BB_CUDA(cudaMemcpy(lane[i]->adm.p, c->adm.p, c->adm.bytes, cudaMemcpyDeviceToDevice));
        }
        lane[i]->ws.lu_valid = 0;
    }
    return lane;
}

// Runs work(lane_ctx, f) for f = 0..nfreq-1 over L lanes of c.  Afterwards no
// lane offers its factors: lane 0 is this context, and its factors belong to
// whichever frequency it solved last, which the caller cannot name, so
// beat_b200_resolve_noalloc and beat_b200_adjoint refuse them.
template <typename W> void run_sweep(beat_b200_ctx *c, int nfreq, int lanes, W &&work) {
    const int L = std::max(1, std::min(lanes, nfreq));
    std::vector<beat_b200_ctx *> lane = prepare_lanes(c, L);
    std::vector<int> order(nfreq);
    for (int f = 0; f < nfreq; ++f) order[f] = f;
    try {
        run_jobs(
            c, L, order, "frequency", [&](int i, int f) { work(lane[i], f); },
            [&](int i, int) { return lane[i]->stream; });
    } catch (...) {
        for (beat_b200_ctx *l : lane) l->ws.lu_valid = 0;
        throw;
    }
    for (beat_b200_ctx *l : lane) l->ws.lu_valid = 0;
}

// Several meshes' sweeps as one job list over L lanes: job (m, f) is mesh m
// at its frequency f, on lane i's context of mesh m.  Jobs are taken in
// decreasing order of cost (N^3, the factorisation), so the lanes finish
// together instead of one lane ending on the largest mesh alone.
template <typename W>
void run_batch(const std::vector<beat_b200_ctx *> &cs, const std::vector<int> &nfreq, int lanes, W &&work) {
    const int nm = (int)cs.size();
    std::vector<int> base(nm + 1, 0);
    for (int m = 0; m < nm; ++m) base[m + 1] = base[m] + nfreq[m];
    const int njobs = base[nm];
    if (njobs == 0) return;
    const int L = std::max(1, std::min(lanes, njobs));
    std::vector<std::vector<beat_b200_ctx *>> lane(nm);
    for (int m = 0; m < nm; ++m) lane[m] = prepare_lanes(cs[m], L);
    std::vector<int> order(njobs), mesh_of(njobs);
    for (int m = 0; m < nm; ++m)
        for (int f = 0; f < nfreq[m]; ++f) mesh_of[base[m] + f] = m;
    for (int j = 0; j < njobs; ++j) order[j] = j;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
        const double na = cs[mesh_of[a]]->V, nb = cs[mesh_of[b]]->V;
        return na * na * na > nb * nb * nb;
    });
    auto clear = [&] {
        for (auto &v : lane)
            for (beat_b200_ctx *l : v) l->ws.lu_valid = 0;
    };
    try {
        run_jobs(
            cs[0], L, order, "job (mesh-major numbering)",
            [&](int i, int j) {
                const int m = mesh_of[j];
                work(lane[m][i], m, j - base[m]);
            },
            [&](int i, int j) { return lane[mesh_of[j]][i]->stream; });
    } catch (...) {
        clear();
        throw;
    }
    clear();
}

}  // namespace

extern "C" {

int32_t beat_b200_abi_version(void) { return BEAT_B200_ABI_VERSION; }

void beat_b200_default_opts(beat_b200_opts *o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->precision = BEAT_B200_MIXED_FP32_IR;
    o->ir_restart = 20;
    o->ir_max_iters = 200;
    o->lu_split_terms = 3;
    o->ir_rtol = 1e-10;
    o->lu_block = 0;
    o->flags = 0;
}

int32_t beat_b200_create(int32_t device, beat_b200_ctx **out) {
    if (!out) return BEAT_B200_INVALID_ARG;
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count <= 0) {
        cudaGetLastError();
        return BEAT_B200_NO_DEVICE;
    }
    if (device < 0 || device >= count) return BEAT_B200_INVALID_ARG;
    beat_b200_ctx *c = new (std::nothrow) beat_b200_ctx();
    if (!c) return BEAT_B200_OOM;
    c->device = device;
    const int32_t st = guarded(c, [&] {
        cudaDeviceProp prop;
        BB_CUDA(cudaGetDeviceProperties(&prop, device));
        BB_REQUIRE(prop.major >= 10, BEAT_B200_NO_DEVICE,
                   std::string("libbeatb200 is built for sm_100a; device is ") + prop.name);
        c->sm_count = prop.multiProcessorCount;
        // the context's stream carries the LU's critical path (its panels) at the
        // highest priority; the look-ahead trailing updates run on the side stream
        int prio_least = 0, prio_greatest = 0;
        BB_CUDA(cudaDeviceGetStreamPriorityRange(&prio_least, &prio_greatest));
        BB_CUDA(cudaStreamCreateWithPriority(&c->stream, cudaStreamNonBlocking, prio_greatest));
        BB_CUDA(cudaStreamCreateWithPriority(&c->side_stream, cudaStreamNonBlocking, prio_least));
        BB_CUDA(cudaEventCreateWithFlags(&c->la_fork, cudaEventDisableTiming));
        BB_CUDA(cudaEventCreateWithFlags(&c->la_join, cudaEventDisableTiming));
        for (auto &e : c->ev) BB_CUDA(cudaEventCreate(&e));
        c->status.alloc(256);
        BB_CUDA(cudaMemset(c->status.p, 0, 256));
        c->barrier.alloc(sizeof(unsigned) * 4096);
        BB_CUDA(cudaMemset(c->barrier.p, 0, sizeof(unsigned) * 4096));
    });
    if (st != BEAT_B200_OK) {
        beat_b200_destroy(c);
        return st;
    }
    *out = c;
    return BEAT_B200_OK;
}

int32_t beat_b200_destroy(beat_b200_ctx *c) {
    if (!c) return BEAT_B200_OK;
    for (beat_b200_ctx *l : c->lanes) beat_b200_destroy(l);
    c->lanes.clear();
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    release_workspace(c);
    for (DevBuf *b : {&c->pos_face, &c->pos_qpts64, &c->pos_qpts32, &c->pos_normal64, &c->pos_normal32,
                      &c->pos_curl64, &c->pos_curl32, &c->pos_area64, &c->pos_area32, &c->pos_plane32,
                      &c->pos_gvert, &c->d_verts,
                      &c->d_faces, &c->d_normals, &c->d_areas, &c->d_curls, &c->d_qpts, &c->vf_start, &c->vf_face,
                      &c->adm, &c->ip_test, &c->ip_trial, &c->ip_rule, &c->ip_img, &c->ip_jac, &c->ip_nn,
                      &c->rw_vert, &c->rw_weight, &c->sp_test, &c->sp_trial,
                      &c->sp_rule, &c->sp_jac, &c->sp_nn, &c->rule_start, &c->rule_data, &c->status, &c->barrier})
        b->free_();
    for (Tiling *t : {&c->test_tiles, &c->trial_tiles, &c->sym_tiles}) {
        t->face_start.free_();
        t->vert_start.free_();
        t->verts.free_();
        t->local_vert.free_();
    }
    for (auto &e : c->ev)
        if (e) cudaEventDestroy(e);
    if (c->side_stream) cudaStreamSynchronize(c->side_stream);
    for (cudaEvent_t e : {c->la_fork, c->la_join})
        if (e) cudaEventDestroy(e);
    if (c->side_stream) cudaStreamDestroy(c->side_stream);
    if (c->stream) cudaStreamDestroy(c->stream);
    cudaGetLastError();
    delete c;
    return BEAT_B200_OK;
}

const char *beat_b200_last_error(const beat_b200_ctx *c) { return c ? c->last_error.c_str() : "null context"; }

int32_t beat_b200_set_mesh(beat_b200_ctx *c, int32_t V, const double *vertices, int32_t F, const int32_t *faces,
                           int32_t quad_order, int32_t singular_order) {
    return guarded(c, [&] {
        for (beat_b200_ctx *l : c->lanes) beat_b200_destroy(l);  // lanes hold the previous mesh
        c->lanes.clear();
        set_mesh(c, V, vertices, F, faces, quad_order, singular_order);
    });
}

int32_t beat_b200_solve_device(beat_b200_ctx *c, double k, double eta, int32_t R, const void *d_q,
                               const beat_b200_opts *opts, void *d_p, beat_b200_diag *diag) {
    return guarded(c, [&] {
        BB_REQUIRE(d_q && d_p, BEAT_B200_INVALID_ARG, "null device pointer");
        const beat_b200_opts o = resolve_opts(opts);
        solve_core(c, k, eta, R, (const double *)d_q, o, (double *)d_p, diag);
    });
}

int32_t beat_b200_solve(beat_b200_ctx *c, double k, double eta, int32_t R, const double *q,
                        const beat_b200_opts *opts, double *p_out, beat_b200_diag *diag) {
    return guarded(c, [&] {
        BB_REQUIRE(q && p_out && R >= 1, BEAT_B200_INVALID_ARG, "null pointer or R < 1");
        BB_REQUIRE(c->F > 0, BEAT_B200_STATE, "no mesh: call beat_b200_set_mesh first");
        const beat_b200_opts o = resolve_opts(opts);
        c->ws.lu_valid = 0;  // the workspace may change below; solve_core sets it once the factors are good
        ensure_workspace(c, o.precision, R, rhs_request(o));
        Workspace &w = c->ws;
        BB_CUDA(cudaMemcpyAsync(w.q.p, q, (size_t)c->F * R * 16, cudaMemcpyHostToDevice, c->stream));
        DevBuf &out = w.io;
        out.alloc((size_t)c->V * R * 16);
        try {
            solve_core(c, k, eta, R, w.q.as<double>(), o, out.as<double>(), diag);
            BB_CUDA(cudaMemcpyAsync(p_out, out.p, (size_t)c->V * R * 16, cudaMemcpyDeviceToHost, c->stream));
            BB_CUDA(cudaStreamSynchronize(c->stream));
        } catch (...) {
            if (c->stream) cudaStreamSynchronize(c->stream);
            throw;
        }
    });
}

static int32_t field_common(beat_b200_ctx *c, double k, int32_t M, const double *pts, int32_t R, const double *p,
                            const double *q, double *out, bool far) {
    return guarded(c, [&] {
        BB_REQUIRE(c->F > 0, BEAT_B200_STATE, "no mesh: call beat_b200_set_mesh first");
        BB_REQUIRE(M >= 0 && R >= 1 && (M == 0 || (pts && p && q && out)), BEAT_B200_INVALID_ARG,
                   "field: bad arguments");
        if (M == 0) return;
        DevBuf &buf = c->ws.io;
        buf.alloc(16 * ((size_t)c->V * R + (size_t)c->F * R + (size_t)M * R));
        try {
            double *dp = buf.as<double>(), *dq = dp + 2 * (size_t)c->V * R, *dout = dq + 2 * (size_t)c->F * R;
            BB_CUDA(cudaMemcpyAsync(dp, p, (size_t)c->V * R * 16, cudaMemcpyHostToDevice, c->stream));
            BB_CUDA(cudaMemcpyAsync(dq, q, (size_t)c->F * R * 16, cudaMemcpyHostToDevice, c->stream));
            farfield(c, k, M, pts, R, dp, dq, dout, far);
            BB_CUDA(cudaMemcpyAsync(out, dout, (size_t)M * R * 16, cudaMemcpyDeviceToHost, c->stream));
            BB_CUDA(cudaStreamSynchronize(c->stream));
        } catch (...) {
            if (c->stream) cudaStreamSynchronize(c->stream);
            throw;
        }
    });
}

int32_t beat_b200_field(beat_b200_ctx *c, double k, int32_t M, const double *points, int32_t R, const double *p,
                        const double *q, double *out) {
    return field_common(c, k, M, points, R, p, q, out, false);
}

int32_t beat_b200_farfield(beat_b200_ctx *c, double k, int32_t M, const double *dirs, int32_t R, const double *p,
                           const double *q, double *out) {
    return field_common(c, k, M, dirs, R, p, q, out, true);
}

int32_t beat_b200_field_gradient(beat_b200_ctx *c, double k, int32_t M, const double *points, int32_t R,
                                 const double *p, const double *q, double *out) {
    return guarded(c, [&] {
        BB_REQUIRE(c->F > 0, BEAT_B200_STATE, "no mesh: call beat_b200_set_mesh first");
        BB_REQUIRE(M >= 0 && R >= 1 && (M == 0 || (points && p && q && out)), BEAT_B200_INVALID_ARG,
                   "field gradient: bad arguments");
        if (M == 0) return;
        DevBuf &buf = c->ws.io;
        buf.alloc(16 * ((size_t)c->V * R + (size_t)c->F * R + 4 * (size_t)M * R));
        try {
            double *dp = buf.as<double>(), *dq = dp + 2 * (size_t)c->V * R, *dout = dq + 2 * (size_t)c->F * R;
            BB_CUDA(cudaMemcpyAsync(dp, p, (size_t)c->V * R * 16, cudaMemcpyHostToDevice, c->stream));
            BB_CUDA(cudaMemcpyAsync(dq, q, (size_t)c->F * R * 16, cudaMemcpyHostToDevice, c->stream));
            field_gradient(c, k, M, points, R, dp, dq, dout);
            BB_CUDA(cudaMemcpyAsync(out, dout, 4 * (size_t)M * R * 16, cudaMemcpyDeviceToHost, c->stream));
            BB_CUDA(cudaStreamSynchronize(c->stream));
        } catch (...) {
            if (c->stream) cudaStreamSynchronize(c->stream);
            throw;
        }
    });
}

int32_t beat_b200_field_gradient_device(beat_b200_ctx *c, double k, int32_t M, const double *points, int32_t R,
                                        const void *d_p, const void *d_q, void *d_out) {
    return guarded(c, [&] {
        BB_REQUIRE(M == 0 || (points && d_p && d_q && d_out), BEAT_B200_INVALID_ARG, "null pointer");
        field_gradient(c, k, M, points, R, (const double *)d_p, (const double *)d_q, (double *)d_out);
    });
}

int32_t beat_b200_assemble_coupled_device(beat_b200_ctx *c, double k, int32_t precision, void *d_A, void *d_C) {
    return guarded(c, [&] { assemble_coupled(c, k, precision, d_A, d_C); });
}

int32_t beat_b200_coupled_blocks_device(beat_b200_ctx *c, int32_t precision, const void *d_C, int32_t ncols,
                                        const int32_t *d_colptr, const int32_t *d_rowval, const void *d_nzval,
                                        int64_t nnz, void *d_interface, int32_t nmotion, const void *d_motion,
                                        void *d_motion_out, int32_t nprescribed, const void *d_prescribed,
                                        void *d_prescribed_out) {
    return guarded(c, [&] {
        coupled_blocks(c, precision, d_C, ncols, d_colptr, d_rowval, d_nzval, nnz, d_interface, nmotion, d_motion,
                       d_motion_out, nprescribed, d_prescribed, d_prescribed_out);
    });
}

int32_t beat_b200_rhs_use_operator(int32_t mode, int32_t excitations, int64_t matrix_bytes, int64_t operator_bytes,
                                   int64_t available_bytes) {
    return rhs_use_operator(mode, excitations, matrix_bytes, operator_bytes, available_bytes);
}

int32_t beat_b200_farfield_device(beat_b200_ctx *c, double k, int32_t M, const double *dirs, int32_t R,
                                  const void *d_p, const void *d_q, void *d_out) {
    return guarded(c, [&] {
        BB_REQUIRE(dirs && d_p && d_q && d_out, BEAT_B200_INVALID_ARG, "null pointer");
        farfield(c, k, M, dirs, R, (const double *)d_p, (const double *)d_q, (double *)d_out, true);
    });
}

int32_t beat_b200_assemble(beat_b200_ctx *c, double k, double eta, int32_t R, const double *q, int32_t precision,
                           double *A_out, double *b_out) {
    return guarded(c, [&] {
        BB_REQUIRE(c->F > 0, BEAT_B200_STATE, "no mesh: call beat_b200_set_mesh first");
        BB_REQUIRE(R >= 0 && (R == 0 || q), BEAT_B200_INVALID_ARG, "assemble: bad arguments");
        BB_REQUIRE(precision == BEAT_B200_FP64 || precision == BEAT_B200_MIXED_FP32_IR, BEAT_B200_INVALID_ARG,
                   "unknown precision form");
        const int Rr = std::max(R, 1);
        ensure_workspace(c, precision, Rr);
        Workspace &w = c->ws;
        const int n = c->V;
        if (R > 0)
            BB_CUDA(cudaMemcpyAsync(w.q.p, q, (size_t)c->F * R * 16, cudaMemcpyHostToDevice, c->stream));
        else
            BB_CUDA(cudaMemsetAsync(w.q.p, 0, (size_t)c->F * 16, c->stream));
        assemble(c, k, eta, precision, Rr, w.q.p, nullptr, nullptr);
        w.lu_valid = 0;
        if (A_out) {
            DevBuf tmp;
            tmp.alloc((size_t)n * n * 16);
            dim3 grid((n + 31) / 32, (n + 31) / 32), block(32, 8);
            if (precision == BEAT_B200_FP64)
                export_matrix_kernel<double><<<grid, block, 0, c->stream>>>(w.A.as<Cx<double>>(), w.ld, n,
                                                                            tmp.as<double2>());
            else
                export_matrix_kernel<float><<<grid, block, 0, c->stream>>>(w.A.as<Cx<float>>(), w.ld, n,
                                                                           tmp.as<double2>());
            BB_CUDA(cudaGetLastError());
            BB_CUDA(cudaMemcpyAsync(A_out, tmp.p, (size_t)n * n * 16, cudaMemcpyDeviceToHost, c->stream));
            BB_CUDA(cudaStreamSynchronize(c->stream));
            tmp.free_();
        }
        if (b_out && R > 0) {
            BB_CUDA(cudaMemcpyAsync(b_out, w.b.p, (size_t)n * R * 16, cudaMemcpyDeviceToHost, c->stream));
        }
        BB_CUDA(cudaStreamSynchronize(c->stream));
    });
}

int32_t beat_b200_release_workspace(beat_b200_ctx *c) {
    return guarded(c, [&] {
        BB_CUDA(cudaStreamSynchronize(c->stream));
        release_workspace(c);
        for (beat_b200_ctx *l : c->lanes) {
            BB_CUDA(cudaStreamSynchronize(l->stream));
            release_workspace(l);
        }
    });
}

int64_t beat_b200_device_bytes(const beat_b200_ctx *c) {
    if (!c) return 0;
    int64_t s = device_bytes(c);
    for (const beat_b200_ctx *l : c->lanes) s += device_bytes(l);
    return s;
}

int32_t beat_b200_sweep_device(beat_b200_ctx *c, int32_t nfreq, const double *k_signed, const double *eta_im,
                               int32_t R, const void *d_q, const beat_b200_opts *opts, void *d_p, int32_t M,
                               const double *dirs, void *d_ff, beat_b200_diag *diags) {
    return guarded(c, [&] {
        BB_REQUIRE(nfreq >= 0 && R >= 1, BEAT_B200_INVALID_ARG, "sweep: nfreq must be >= 0 and R >= 1");
        if (nfreq == 0) return;
        BB_REQUIRE(k_signed && eta_im && d_q && d_p, BEAT_B200_INVALID_ARG, "sweep: null pointer");
        BB_REQUIRE(M >= 0 && (M == 0 || (dirs && d_ff)), BEAT_B200_INVALID_ARG, "sweep: bad far-field arguments");
        BB_REQUIRE(c->F > 0, BEAT_B200_STATE, "no mesh: call beat_b200_set_mesh first");
        const beat_b200_opts o = resolve_opts(opts);
        const size_t qs = (size_t)c->F * R * 2, ps = (size_t)c->V * R * 2, fs = (size_t)M * R * 2;
        run_sweep(c, nfreq, sweep_lane_count(c, nfreq, o, R), [&](beat_b200_ctx *l, int f) {
            const double *q = (const double *)d_q + f * qs;
            double *p = (double *)d_p + f * ps;
            solve_core(l, k_signed[f], eta_im[f], R, q, o, p, diags ? diags + f : nullptr);
            if (M > 0) farfield(l, k_signed[f], M, dirs, R, p, q, (double *)d_ff + f * fs, true);
        });
    });
}

int32_t beat_b200_sweep(beat_b200_ctx *c, int32_t nfreq, const double *k_signed, const double *eta_im, int32_t R,
                        const double *q, const beat_b200_opts *opts, double *p_out, int32_t M, const double *dirs,
                        double *ff_out, beat_b200_diag *diags) {
    return guarded(c, [&] {
        BB_REQUIRE(nfreq >= 0 && R >= 1, BEAT_B200_INVALID_ARG, "sweep: nfreq must be >= 0 and R >= 1");
        if (nfreq == 0) return;
        BB_REQUIRE(k_signed && eta_im && q && p_out, BEAT_B200_INVALID_ARG, "sweep: null pointer");
        BB_REQUIRE(M >= 0 && (M == 0 || (dirs && ff_out)), BEAT_B200_INVALID_ARG, "sweep: bad far-field arguments");
        BB_REQUIRE(c->F > 0, BEAT_B200_STATE, "no mesh: call beat_b200_set_mesh first");
        const beat_b200_opts o = resolve_opts(opts);
        const size_t qs = (size_t)c->F * R * 2, ps = (size_t)c->V * R * 2, fs = (size_t)M * R * 2;
        run_sweep(c, nfreq, sweep_lane_count(c, nfreq, o, R), [&](beat_b200_ctx *l, int f) {
            ensure_workspace(l, o.precision, R, rhs_request(o));
            Workspace &w = l->ws;
            BB_CUDA(cudaMemcpyAsync(w.q.p, q + f * qs, qs * sizeof(double), cudaMemcpyHostToDevice, l->stream));
            w.io.alloc((ps + fs) * sizeof(double));
            double *dp = w.io.as<double>(), *dff = dp + ps;
            solve_core(l, k_signed[f], eta_im[f], R, w.q.as<double>(), o, dp, diags ? diags + f : nullptr);
            if (M > 0) farfield(l, k_signed[f], M, dirs, R, dp, w.q.as<double>(), dff, true);
            BB_CUDA(cudaMemcpyAsync(p_out + f * ps, dp, ps * sizeof(double), cudaMemcpyDeviceToHost, l->stream));
            if (M > 0)
                BB_CUDA(cudaMemcpyAsync(ff_out + f * fs, dff, fs * sizeof(double), cudaMemcpyDeviceToHost, l->stream));
            BB_CUDA(cudaStreamSynchronize(l->stream));
        });
    });
}

// the contexts, options and column counts of a batched sweep, checked
static void batch_inputs(int32_t nmesh, beat_b200_ctx *const *ctxs, const int32_t *nfreq, const int32_t *R,
                         const beat_b200_opts *opts, std::vector<beat_b200_ctx *> &cs, std::vector<int> &nf,
                         std::vector<int> &rr, std::vector<beat_b200_opts> &o) {
    BB_REQUIRE(nmesh >= 1 && ctxs && nfreq && R, BEAT_B200_INVALID_ARG, "batched sweep: bad arguments");
    for (int m = 0; m < nmesh; ++m) {
        beat_b200_ctx *c = ctxs[m];
        BB_REQUIRE(c, BEAT_B200_INVALID_ARG, "batched sweep: null context");
        BB_REQUIRE(c->device == ctxs[0]->device, BEAT_B200_INVALID_ARG,
                   "batched sweep: every context must be on the same device");
        for (int j = 0; j < m; ++j)
            BB_REQUIRE(ctxs[j] != c, BEAT_B200_INVALID_ARG, "batched sweep: a context appears twice");
        BB_REQUIRE(c->F > 0, BEAT_B200_STATE, "batched sweep: a context has no mesh");
        BB_REQUIRE(nfreq[m] >= 0 && R[m] >= 1, BEAT_B200_INVALID_ARG, "batched sweep: nfreq >= 0 and R >= 1");
        cs.push_back(c);
        nf.push_back(nfreq[m]);
        rr.push_back(R[m]);
        o.push_back(resolve_opts(opts ? opts + m : nullptr));
    }
}

int32_t beat_b200_sweep_batch(int32_t nmesh, beat_b200_ctx *const *ctxs, const int32_t *nfreq,
                              const double *const *k_signed, const double *const *eta_im, const int32_t *R,
                              const double *const *q, const beat_b200_opts *opts, double *const *p_out, int32_t M,
                              const double *dirs, double *const *ff_out, beat_b200_diag *const *diags) {
    if (nmesh < 1 || !ctxs || !ctxs[0]) return BEAT_B200_INVALID_ARG;
    return guarded(ctxs[0], [&] {
        std::vector<beat_b200_ctx *> cs;
        std::vector<int> nf, rr;
        std::vector<beat_b200_opts> o;
        batch_inputs(nmesh, ctxs, nfreq, R, opts, cs, nf, rr, o);
        BB_REQUIRE(k_signed && eta_im && q && p_out, BEAT_B200_INVALID_ARG, "batched sweep: null pointer");
        BB_REQUIRE(M >= 0 && (M == 0 || (dirs && ff_out)), BEAT_B200_INVALID_ARG,
                   "batched sweep: bad far-field arguments");
        int njobs = 0;
        for (int m = 0; m < nmesh; ++m) {
            BB_REQUIRE(nf[m] == 0 || (k_signed[m] && eta_im[m] && q[m] && p_out[m] && (M == 0 || ff_out[m])),
                       BEAT_B200_INVALID_ARG, "batched sweep: null pointer for mesh " + std::to_string(m));
            njobs += nf[m];
        }
        run_batch(cs, nf, lane_count(cs, rr, njobs, o.data()), [&](beat_b200_ctx *l, int m, int f) {
            const int Rm = rr[m];
            const size_t qs = (size_t)cs[m]->F * Rm * 2, ps = (size_t)cs[m]->V * Rm * 2, fs = (size_t)M * Rm * 2;
            ensure_workspace(l, o[m].precision, Rm, rhs_request(o[m]));
            Workspace &w = l->ws;
            BB_CUDA(cudaMemcpyAsync(w.q.p, q[m] + f * qs, qs * sizeof(double), cudaMemcpyHostToDevice, l->stream));
            w.io.alloc((ps + fs) * sizeof(double));
            double *dp = w.io.as<double>(), *dff = dp + ps;
            solve_core(l, k_signed[m][f], eta_im[m][f], Rm, w.q.as<double>(), o[m], dp,
                       diags && diags[m] ? diags[m] + f : nullptr);
            if (M > 0) farfield(l, k_signed[m][f], M, dirs, Rm, dp, w.q.as<double>(), dff, true);
            BB_CUDA(cudaMemcpyAsync(p_out[m] + f * ps, dp, ps * sizeof(double), cudaMemcpyDeviceToHost, l->stream));
            if (M > 0)
                BB_CUDA(cudaMemcpyAsync(ff_out[m] + f * fs, dff, fs * sizeof(double), cudaMemcpyDeviceToHost,
                                        l->stream));
            BB_CUDA(cudaStreamSynchronize(l->stream));
        });
    });
}

int32_t beat_b200_sweep_batch_device(int32_t nmesh, beat_b200_ctx *const *ctxs, const int32_t *nfreq,
                                     const double *const *k_signed, const double *const *eta_im, const int32_t *R,
                                     const void *const *d_q, const beat_b200_opts *opts, void *const *d_p, int32_t M,
                                     const double *dirs, void *const *d_ff, beat_b200_diag *const *diags) {
    if (nmesh < 1 || !ctxs || !ctxs[0]) return BEAT_B200_INVALID_ARG;
    return guarded(ctxs[0], [&] {
        std::vector<beat_b200_ctx *> cs;
        std::vector<int> nf, rr;
        std::vector<beat_b200_opts> o;
        batch_inputs(nmesh, ctxs, nfreq, R, opts, cs, nf, rr, o);
        BB_REQUIRE(k_signed && eta_im && d_q && d_p, BEAT_B200_INVALID_ARG, "batched sweep: null pointer");
        BB_REQUIRE(M >= 0 && (M == 0 || (dirs && d_ff)), BEAT_B200_INVALID_ARG,
                   "batched sweep: bad far-field arguments");
        int njobs = 0;
        for (int m = 0; m < nmesh; ++m) {
            BB_REQUIRE(nf[m] == 0 || (k_signed[m] && eta_im[m] && d_q[m] && d_p[m] && (M == 0 || d_ff[m])),
                       BEAT_B200_INVALID_ARG, "batched sweep: null pointer for mesh " + std::to_string(m));
            njobs += nf[m];
        }
        run_batch(cs, nf, lane_count(cs, rr, njobs, o.data()), [&](beat_b200_ctx *l, int m, int f) {
            const int Rm = rr[m];
            const size_t qs = (size_t)cs[m]->F * Rm * 2, ps = (size_t)cs[m]->V * Rm * 2, fs = (size_t)M * Rm * 2;
            const double *qd = (const double *)d_q[m] + f * qs;
            double *pd = (double *)d_p[m] + f * ps;
            solve_core(l, k_signed[m][f], eta_im[m][f], Rm, qd, o[m], pd, diags && diags[m] ? diags[m] + f : nullptr);
            if (M > 0) farfield(l, k_signed[m][f], M, dirs, Rm, pd, qd, (double *)d_ff[m] + f * fs, true);
        });
    });
}

int32_t beat_b200_set_symmetry(beat_b200_ctx *c, int32_t mode) {
    return guarded(c, [&] {
        BB_REQUIRE(mode >= 0 && mode <= 3, BEAT_B200_INVALID_ARG, "symmetry mode must be 0 (off), 1 (x), 2 (xy) or 3 (ground)");
        BB_CUDA(cudaStreamSynchronize(c->stream));
        for (beat_b200_ctx *l : c->lanes) beat_b200_destroy(l);  // lanes hold the previous set-up
        c->lanes.clear();
        const int old = c->sym_mode;
        c->sym_mode = mode;
        if (c->F > 0 && mode != old) {
            const bool adm = c->adm_set;
            DevBuf keep;
            if (adm) {  // set_mesh clears the admittance: carry it over
                keep.alloc(c->adm.bytes);
                BB_CUDA(cudaMemcpy(keep.p, c->adm.p, c->adm.bytes, cudaMemcpyDeviceToDevice));
            }
            try {
                set_mesh(c, c->V, c->in_verts.data(), c->F, c->in_faces.data(), c->quad_order, c->sing_order);
            } catch (...) {
                c->sym_mode = old;
                keep.free_();
                set_mesh(c, c->V, c->in_verts.data(), c->F, c->in_faces.data(), c->quad_order, c->sing_order);
                throw;
            }
            if (adm) {
                c->adm.alloc(keep.bytes);
                BB_CUDA(cudaMemcpy(c->adm.p, keep.p, keep.bytes, cudaMemcpyDeviceToDevice));
                c->adm_set = true;
                keep.free_();
            }
        }
        c->ws.lu_valid = 0;
    });
}

int32_t beat_b200_set_admittance(beat_b200_ctx *c, const double *a) {
    return guarded(c, [&] {
        BB_REQUIRE(c->F > 0, BEAT_B200_STATE, "no mesh: call beat_b200_set_mesh first");
        BB_CUDA(cudaStreamSynchronize(c->stream));
        if (!a) {
            c->adm_set = false;
        } else {
            for (size_t i = 0; i < 2 * (size_t)c->F; ++i)
                BB_REQUIRE(std::isfinite(a[i]), BEAT_B200_INVALID_ARG, "admittance: non-finite coefficient");
            c->adm.alloc(sizeof(double) * 2 * (size_t)c->F);
            BB_CUDA(cudaMemcpy(c->adm.p, a, sizeof(double) * 2 * (size_t)c->F, cudaMemcpyHostToDevice));
            c->adm_set = true;
        }
        c->ws.lu_valid = 0;  // the factors belong to the previous operator
    });
}

int32_t beat_b200_adjoint(beat_b200_ctx *c, double k_signed, int32_t M, const double *dirs, int32_t R,
                          const double *p, const double *g, const beat_b200_opts *opts, double *w_out,
                          double *ga_out) {
    return guarded(c, [&] {
        BB_REQUIRE(dirs && p && g && w_out, BEAT_B200_INVALID_ARG, "adjoint: null pointer");
        BB_REQUIRE(c->F > 0, BEAT_B200_STATE, "no mesh: call beat_b200_set_mesh first");
        BB_REQUIRE(M >= 1 && R >= 1, BEAT_B200_INVALID_ARG, "adjoint: M and R must be >= 1");
        const beat_b200_opts o = resolve_opts(opts);
        const size_t np = (size_t)c->V * R, ng = (size_t)M * R, nw = (size_t)c->F * R;
        DevBuf &io = c->ws.io;
        io.alloc(sizeof(double2) * (np + ng + nw + c->F));
        double2 *dp = io.as<double2>(), *dg = dp + np, *dw = dg + ng, *dga = dw + nw;
        BB_CUDA(cudaMemcpyAsync(dp, p, sizeof(double2) * np, cudaMemcpyHostToDevice, c->stream));
        BB_CUDA(cudaMemcpyAsync(dg, g, sizeof(double2) * ng, cudaMemcpyHostToDevice, c->stream));
        IrResult ir{0, 1, 0.0};
        adjoint(c, k_signed, M, dirs, R, (const double *)dp, (const double *)dg, (double *)dw,
                ga_out ? (double *)dga : nullptr, o, &ir);
        BB_CUDA(cudaMemcpyAsync(w_out, dw, sizeof(double2) * nw, cudaMemcpyDeviceToHost, c->stream));
        if (ga_out)
            BB_CUDA(cudaMemcpyAsync(ga_out, dga, sizeof(double2) * c->F, cudaMemcpyDeviceToHost, c->stream));
        BB_CUDA(cudaStreamSynchronize(c->stream));
        BB_REQUIRE(ir.converged, BEAT_B200_NOT_CONVERGED,
                   "adjoint refinement missed its tolerance (worst relative residual " + std::to_string(ir.residual) +
                       ")");
    });
}

int32_t beat_b200_adjoint_shape(beat_b200_ctx *c, double k_signed, int32_t M, const double *dirs, int32_t R,
                                const double *p, const double *q, const double *g, const beat_b200_opts *opts,
                                double *w_out, double *ga_out, double *gX_out) {
    return guarded(c, [&] {
        BB_REQUIRE(dirs && p && q && g && gX_out, BEAT_B200_INVALID_ARG, "adjoint: null pointer");
        BB_REQUIRE(c->F > 0, BEAT_B200_STATE, "no mesh: call beat_b200_set_mesh first");
        BB_REQUIRE(M >= 1 && R >= 1, BEAT_B200_INVALID_ARG, "adjoint: M and R must be >= 1");
        const beat_b200_opts o = resolve_opts(opts);
        const int N = c->V, F = c->F;
        const size_t np = (size_t)N * R, ng = (size_t)M * R, nw = (size_t)F * R;
        DevBuf &io = c->ws.io;
        // p, q, g, w, ga (complex), then gX (3N) and the directions (3M), doubles
        io.alloc(sizeof(double2) * (np + 2 * nw + ng + F) + sizeof(double) * (3 * (size_t)N + 3 * (size_t)M));
        double2 *dp = io.as<double2>(), *dq = dp + np, *dg = dq + nw, *dw = dg + ng, *dga = dw + nw;
        double *dgx = reinterpret_cast<double *>(dga + F), *ddirs = dgx + 3 * (size_t)N;
        BB_CUDA(cudaMemcpyAsync(dp, p, sizeof(double2) * np, cudaMemcpyHostToDevice, c->stream));
        BB_CUDA(cudaMemcpyAsync(dq, q, sizeof(double2) * nw, cudaMemcpyHostToDevice, c->stream));
        BB_CUDA(cudaMemcpyAsync(dg, g, sizeof(double2) * ng, cudaMemcpyHostToDevice, c->stream));
        BB_CUDA(cudaMemcpyAsync(ddirs, dirs, sizeof(double) * 3 * M, cudaMemcpyHostToDevice, c->stream));
        IrResult ir{0, 1, 0.0};
        const double *z = nullptr;
        adjoint(c, k_signed, M, dirs, R, (const double *)dp, (const double *)dg, (double *)dw, (double *)dga, o, &ir,
                &z);
        BB_REQUIRE(ir.converged, BEAT_B200_NOT_CONVERGED,
                   "adjoint refinement missed its tolerance (worst relative residual " + std::to_string(ir.residual) +
                       ")");
        // the boundary's Neumann data: q0 - diag(a) P p with an admittance
        c->ws.qeff.alloc(sizeof(double2) * nw);
        effective_neumann(c, R, (const double *)dp, (const double *)dq, c->ws.qeff.as<double>());
        shape_gradient(c, k_signed, c->last_eta, M, ddirs, R, (const double *)dp, c->ws.qeff.as<double>(),
                       (const double *)dg, z, dgx);
        if (w_out) BB_CUDA(cudaMemcpyAsync(w_out, dw, sizeof(double2) * nw, cudaMemcpyDeviceToHost, c->stream));
        if (ga_out) BB_CUDA(cudaMemcpyAsync(ga_out, dga, sizeof(double2) * F, cudaMemcpyDeviceToHost, c->stream));
        BB_CUDA(cudaMemcpyAsync(gX_out, dgx, sizeof(double) * 3 * (size_t)N, cudaMemcpyDeviceToHost, c->stream));
        BB_CUDA(cudaStreamSynchronize(c->stream));
    });
}

void *beat_b200_stream(const beat_b200_ctx *c) { return c ? (void *)c->stream : nullptr; }

}  // extern "C"
