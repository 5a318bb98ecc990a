// context.cu -- mesh set-up on the host (geometry, rules, touching pairs,
// element tiles) and device workspace management.
//
// Host restatements of the reference's mesh-only set-up (paths relative to
// src/beat_engine/julia_local/src/):
//   BoundaryMesh constructor           BeatEngineCore.jl:344-364
//   surface_gradients / surface_curls  BeatEngineCore.jl:856-873
//   triangle_rule                      BeatEngineCore.jl:660-692
//   gauss_rule_1d / duffy_rule         BeatEngineCore.jl:713-802
//   remap_shared_vertex / _edge        BeatEngineCore.jl:810-826
//   adjacency_info                     BeatEngineCore.jl:596-622
//   build_singular_correction_cache    BeatEngineCore.jl:994-1089
//   _cuda_geometry_arrays              BeatEngineCudaRegular.jl:827-893
// The tiling (Morton order of centroids, tiles of consecutive elements with
// a cap on distinct vertices) has no reference counterpart: it exists so the
// element-pair kernel can reduce its 3x3 blocks in shared memory.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <map>
#include <numeric>

#include "internal.cuh"

namespace bb {

// BEAT_B200_FAULT_OOM_BYTES (test hook): allocations of at least that many bytes fail
static size_t injected_oom_bytes() {
    const char *e = getenv("BEAT_B200_FAULT_OOM_BYTES");
    return e ? (size_t)strtoull(e, nullptr, 10) : 0;
}

void DevBuf::alloc(size_t n) {
    if (n <= bytes && p) return;
    free_();
    if (n == 0) return;
    const size_t lim = injected_oom_bytes();
    if (lim && n >= lim)
        throw Error{BEAT_B200_OOM, "cudaMalloc of " + std::to_string(n) +
                                       " bytes failed: injected by BEAT_B200_FAULT_OOM_BYTES"};
    cudaError_t e = cudaMalloc(&p, n);
    if (e != cudaSuccess) {
        p = nullptr;
        bytes = 0;
        cudaGetLastError();
        throw Error{BEAT_B200_OOM, "cudaMalloc of " + std::to_string(n) + " bytes failed: " +
                                       cudaGetErrorString(e)};
    }
    bytes = n;
}

void DevBuf::free_() {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
}

template <typename T> static void upload(DevBuf &d, const std::vector<T> &h) {
    d.alloc(std::max<size_t>(h.size() * sizeof(T), 16));
    if (!h.empty()) BB_CUDA(cudaMemcpy(d.p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice));
}

// ---------------------------------------------------------------------------
// rules
// ---------------------------------------------------------------------------
int triangle_rule(int order, std::vector<double> &pts, std::vector<double> &w) {
    if (order <= 1) {
        pts = {1.0 / 3.0, 1.0 / 3.0};
        w = {0.5};
    } else if (order == 4) {
        pts = {0.4459484909159651, 0.4459484909159651, 0.0915762135097710, 0.0915762135097700,
               0.1081030181680700, 0.4459484909159651, 0.4459484909159651, 0.1081030181680700,
               0.8168475729804590, 0.0915762135097700, 0.0915762135097710, 0.8168475729804580};
        const double ww[6] = {0.2233815896780110, 0.1099517436553220, 0.2233815896780110,
                              0.2233815896780110, 0.1099517436553220, 0.1099517436553220};
        w.resize(6);
        for (int i = 0; i < 6; ++i) w[i] = 0.5 * ww[i];
    } else {
        pts = {1.0 / 6.0, 1.0 / 6.0, 2.0 / 3.0, 1.0 / 6.0, 1.0 / 6.0, 2.0 / 3.0};
        w = {1.0 / 6.0, 1.0 / 6.0, 1.0 / 6.0};
    }
    return (int)w.size();
}

static void gauss01(int order, std::vector<double> &x, std::vector<double> &w) {
    x.assign(order, 0.0);
    w.assign(order, 0.0);
    if (order == 1) {
        x[0] = 0.5;
        w[0] = 1.0;
    } else if (order == 2) {
        double a = 0.5 / std::sqrt(3.0);
        x = {0.5 - a, 0.5 + a};
        w = {0.5, 0.5};
    } else if (order == 3) {
        double a = std::sqrt(3.0 / 5.0) / 2.0;
        x = {0.5 - a, 0.5, 0.5 + a};
        w = {5.0 / 18.0, 4.0 / 9.0, 5.0 / 18.0};
    } else if (order == 4) {
        double x1 = std::sqrt(3.0 / 7.0 - 2.0 / 7.0 * std::sqrt(6.0 / 5.0)) / 2.0;
        double x2 = std::sqrt(3.0 / 7.0 + 2.0 / 7.0 * std::sqrt(6.0 / 5.0)) / 2.0;
        double w1 = (18.0 + std::sqrt(30.0)) / 72.0, w2 = (18.0 - std::sqrt(30.0)) / 72.0;
        x = {0.5 - x2, 0.5 - x1, 0.5 + x1, 0.5 + x2};
        w = {w2, w1, w1, w2};
    } else {
        // Gauss-Legendre nodes by Newton iteration on the three-term recurrence
        for (int i = 0; i < order; ++i) {
            double t = -std::cos(M_PI * (i + 0.75) / (order + 0.5)), dp = 1.0;
            for (int it = 0; it < 100; ++it) {
                double p0 = 1.0, p1 = t;
                for (int n = 2; n <= order; ++n) {
                    double p2 = ((2.0 * n - 1.0) * t * p1 - (n - 1.0) * p0) / n;
                    p0 = p1;
                    p1 = p2;
                }
                dp = order * (t * p1 - p0) / (t * t - 1.0);
                double dt = p1 / dp;
                t -= dt;
                if (std::fabs(dt) < 1e-16) break;
            }
            double p0 = 1.0, p1 = t;
            for (int n = 2; n <= order; ++n) {
                double p2 = ((2.0 * n - 1.0) * t * p1 - (n - 1.0) * p0) / n;
                p0 = p1;
                p1 = p2;
            }
            dp = order * (t * p1 - p0) / (t * t - 1.0);
            x[i] = (t + 1.0) / 2.0;
            w[i] = 1.0 / ((1.0 - t * t) * dp * dp);
        }
    }
}

struct DuffyPt {
    double tx, ty, sx, sy, w;
};

enum { COINCIDENT = 1, EDGE = 2, VERTEX = 3 };

// Duffy-transformed tensor rule of a touching pair: the point pairs the
// reference's duffy_rule emits, in the same order.
static std::vector<DuffyPt> duffy(int order, int kind) {
    std::vector<double> xr, wr;
    gauss01(order, xr, wr);
    const int m = order, nt = m * m;
    std::vector<double> px(nt), py(nt), pw(nt);
    for (int i = 0, c = 0; i < m; ++i)
        for (int j = 0; j < m; ++j, ++c) {
            px[c] = xr[j];
            py[c] = xr[i];
            pw[c] = wr[i] * wr[j];
        }
    std::vector<DuffyPt> out;
    auto add = [&](double tx, double ty, double sx, double sy, double w) {
        out.push_back(DuffyPt{tx - ty, ty, sx - sy, sy, w});
    };
    for (int a = 0; a < nt; ++a)
        for (int b = 0; b < nt; ++b) {
            const double xsi = px[a], e1 = py[a], e2 = px[b], e3 = py[b];
            const double e12 = e1 * e2, e123 = e12 * e3, bw = pw[a] * pw[b];
            if (kind == COINCIDENT) {
                double w = bw * xsi * xsi * xsi * e1 * e1 * e2;
                add(xsi, xsi * (1 - e1 + e12), xsi * (1 - e123), xsi * (1 - e1), w);
                add(xsi * (1 - e123), xsi * (1 - e1), xsi, xsi * (1 - e1 + e12), w);
                add(xsi, xsi * (e1 - e12 + e123), xsi * (1 - e12), xsi * (e1 - e12), w);
                add(xsi * (1 - e12), xsi * (e1 - e12), xsi, xsi * (e1 - e12 + e123), w);
                add(xsi * (1 - e123), xsi * (e1 - e123), xsi, xsi * (e1 - e12), w);
                add(xsi, xsi * (e1 - e12), xsi * (1 - e123), xsi * (e1 - e123), w);
            } else if (kind == EDGE) {
                double w = bw * xsi * xsi * xsi * e1 * e1;
                add(xsi, xsi * e1 * e3, xsi * (1 - e12), xsi * e1 * (1 - e2), w);
                add(xsi, xsi * e1, xsi * (1 - e123), xsi * e1 * e2 * (1 - e3), w * e2);
                add(xsi * (1 - e12), xsi * e1 * (1 - e2), xsi, xsi * e123, w * e2);
                add(xsi * (1 - e123), xsi * e12 * (1 - e3), xsi, xsi * e1, w * e2);
                add(xsi * (1 - e123), xsi * e1 * (1 - e2 * e3), xsi, xsi * e12, w * e2);
            } else {
                double w = bw * xsi * xsi * xsi * e2;
                add(xsi, xsi * e1, xsi * e2, xsi * e2 * e3, w);
                add(xsi * e2, xsi * e2 * e3, xsi, xsi * e1, w);
            }
        }
    return out;
}

// map a point of the canonical Duffy configuration onto the element's own
// vertex numbering (va, vb are 1-based shared-vertex ids)
static void remap(int kind, int va, int vb, double x, double y, double &ox, double &oy) {
    if (kind == EDGE) {
        static const double ref[3][2] = {{0, 0}, {1, 0}, {0, 1}};
        const double *v0 = ref[va - 1], *v1 = ref[vb - 1], *v2 = ref[6 - va - vb - 1];
        ox = v0[0] + x * (v1[0] - v0[0]) + y * (v2[0] - v0[0]);
        oy = v0[1] + x * (v1[1] - v0[1]) + y * (v2[1] - v0[1]);
    } else if (kind == VERTEX) {
        if (va == 1) {
            ox = x;
            oy = y;
        } else if (va == 2) {
            ox = 1 - x - y;
            oy = y;
        } else {
            ox = x;
            oy = 1 - x - y;
        }
    } else {
        ox = x;
        oy = y;
    }
}

// ---------------------------------------------------------------------------
// Morton order and tiles
// ---------------------------------------------------------------------------
static uint64_t spread3(uint64_t v) {
    v &= 0x1fffff;
    v = (v | v << 32) & 0x1f00000000ffffULL;
    v = (v | v << 16) & 0x1f0000ff0000ffULL;
    v = (v | v << 8) & 0x100f00f00f00f00fULL;
    v = (v | v << 4) & 0x10c30c30c30c30c3ULL;
    v = (v | v << 2) & 0x1249249249249249ULL;
    return v;
}

static void build_tiling(Tiling &t, int max_faces, int max_verts, const std::vector<int> &pos_gv,
                         int F) {
    std::vector<int> fstart{0}, vstart{0}, verts, local(3 * (size_t)F);
    std::vector<int> tile_vs;
    int count = 0;
    auto close = [&]() {
        fstart.push_back(fstart.back() + count);
        verts.insert(verts.end(), tile_vs.begin(), tile_vs.end());
        vstart.push_back((int)verts.size());
        tile_vs.clear();
        count = 0;
    };
    for (int p = 0; p < F; ++p) {
        int add = 0;
        for (int a = 0; a < 3; ++a)
            if (std::find(tile_vs.begin(), tile_vs.end(), pos_gv[3 * p + a]) == tile_vs.end()) ++add;
        if (count == max_faces || (int)tile_vs.size() + add > max_verts) close();
        for (int a = 0; a < 3; ++a) {
            int g = pos_gv[3 * p + a];
            auto it = std::find(tile_vs.begin(), tile_vs.end(), g);
            int li;
            if (it == tile_vs.end()) {
                li = (int)tile_vs.size();
                tile_vs.push_back(g);
            } else {
                li = (int)(it - tile_vs.begin());
            }
            local[3 * (size_t)p + a] = li;
        }
        ++count;
    }
    if (count) close();
    t.tile_faces = max_faces;
    t.tile_verts = max_verts;
    t.ntiles = (int)fstart.size() - 1;
    // vertex -> slot-face incidences of every tile (counting sort, s increasing)
    const int stride = t.inc_stride();
    std::vector<int> inc((size_t)t.ntiles * stride, 0);
    for (int ti = 0; ti < t.ntiles; ++ti) {
        const int f0 = fstart[ti], nf = fstart[ti + 1] - f0, nv = vstart[ti + 1] - vstart[ti];
        int *start = &inc[(size_t)ti * stride], *list = start + max_verts + 1;
        for (int b = 0; b < 3; ++b)
            for (int f = 0; f < nf; ++f) ++start[local[3 * (size_t)(f0 + f) + b] + 1];
        for (int v = 0; v < nv; ++v) start[v + 1] += start[v];
        std::vector<int> fill(start, start + nv);
        for (int b = 0; b < 3; ++b)
            for (int f = 0; f < nf; ++f) list[fill[local[3 * (size_t)(f0 + f) + b]]++] = b * max_faces + f;
        for (int v = nv + 1; v <= max_verts; ++v) start[v] = start[nv];
    }
    upload(t.face_start, fstart);
    upload(t.vert_start, vstart);
    upload(t.verts, verts);
    upload(t.local_vert, local);
    upload(t.incidence, inc);
}

// element-pair kernel tile shapes (must match assembly.cu)
constexpr int TEST_TILE_FACES = 64, TEST_TILE_VERTS = 80;
constexpr int TRIAL_TILE_FACES = 16, TRIAL_TILE_VERTS = 32;
constexpr int SYM_TILE_FACES = 32, SYM_TILE_VERTS = 40;  // both roles of the symmetric kernel

void set_mesh(beat_b200_ctx *c, int V, const double *verts, int F, const int32_t *faces,
              int quad_order, int sing_order) {
    BB_REQUIRE(V >= 3 && F >= 1 && verts && faces, BEAT_B200_INVALID_ARG, "set_mesh: empty mesh");
    BB_REQUIRE(quad_order >= 1 && quad_order <= 10, BEAT_B200_INVALID_ARG,
               "set_mesh: quadrature order must be in 1..10");
    BB_REQUIRE(sing_order >= 1 && sing_order <= 8, BEAT_B200_INVALID_ARG,
               "set_mesh: singular order must be in 1..8");
    BB_REQUIRE(F <= (1 << 24) && V <= (1 << 24), BEAT_B200_INVALID_ARG, "set_mesh: mesh too large");
    release_workspace(c);
    if (c->in_verts.data() != verts) c->in_verts.assign(verts, verts + 3 * (size_t)V);
    if (c->in_faces.data() != faces) c->in_faces.assign(faces, faces + 3 * (size_t)F);
    c->V = V;
    c->F = F;
    c->quad_order = quad_order;
    c->sing_order = sing_order;
    c->verts.assign(verts, verts + 3 * (size_t)V);
    // symmetry: images, plane snapping, fundamental-domain check
    // (symmetry_transforms, snap_symmetry_plane_vertices,
    // validate_symmetry_fundamental_domain!, BeatEngineCore.jl:463-548)
    c->nimg = 0;
    {
        auto add = [&](float sx, float sy, float sz, float det) {
            c->img_sign[c->nimg][0] = sx;
            c->img_sign[c->nimg][1] = sy;
            c->img_sign[c->nimg][2] = sz;
            c->img_det[c->nimg] = det;
            ++c->nimg;
        };
        if (c->sym_mode == 1 || c->sym_mode == 2) add(-1, 1, 1, -1);
        if (c->sym_mode == 2) {
            add(1, -1, 1, -1);
            add(-1, -1, 1, 1);
        }
        if (c->sym_mode == 3) add(1, -1, 1, -1);
    }
    std::vector<int> rw_v;
    std::vector<double> rw_w;
    if (c->sym_mode == 1 || c->sym_mode == 2) {
        double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
        for (int v = 0; v < V; ++v)
            for (int i = 0; i < 3; ++i) {
                lo[i] = std::min(lo[i], verts[3 * v + i]);
                hi[i] = std::max(hi[i], verts[3 * v + i]);
            }
        const double diag = std::sqrt((hi[0] - lo[0]) * (hi[0] - lo[0]) + (hi[1] - lo[1]) * (hi[1] - lo[1]) +
                                      (hi[2] - lo[2]) * (hi[2] - lo[2]));
        const double tol = std::max(1e-9, diag * 1e-6);
        const int naxes = c->sym_mode == 2 ? 2 : 1;
        for (int v = 0; v < V; ++v) {
            double w = 1.0;
            for (int ax = 0; ax < naxes; ++ax) {
                double &x = c->verts[3 * v + ax];
                BB_REQUIRE(x >= -tol, BEAT_B200_INVALID_ARG,
                           std::string("set_mesh: vertex ") + std::to_string(v + 1) +
                               " lies outside the positive fundamental domain of the symmetry");
                if (std::fabs(x) <= tol) {
                    x = 0.0;
                    w *= 2.0;
                }
            }
            if (w != 1.0) {
                rw_v.push_back(v);
                rw_w.push_back(w);
            }
        }
    }
    c->nweighted = (int)rw_v.size();
    upload(c->rw_vert, rw_v);
    upload(c->rw_weight, rw_w);
    c->faces.resize(3 * (size_t)F);
    for (size_t i = 0; i < 3 * (size_t)F; ++i) {
        BB_REQUIRE(faces[i] >= 1 && faces[i] <= V, BEAT_B200_INVALID_ARG,
                   "set_mesh: face vertex number out of 1..V at entry " + std::to_string(i));
        c->faces[i] = faces[i] - 1;
    }
    for (int i = 0; i < 3 * V; ++i)
        BB_REQUIRE(std::isfinite(verts[i]), BEAT_B200_INVALID_ARG, "set_mesh: non-finite vertex");
    c->Q = triangle_rule(quad_order, c->rule_pts, c->rule_w);
    const int Q = c->Q;
    upload_rule_tables(c->rule_pts, c->rule_w, Q);

    // geometry by original face id
    c->normals.resize(3 * (size_t)F);
    c->areas.resize(F);
    std::vector<double> curls(9 * (size_t)F), qpts(3 * (size_t)F * Q), cent(3 * (size_t)F);
    for (int f = 0; f < F; ++f) {
        const double *a = &c->verts[3 * c->faces[3 * f]], *b = &c->verts[3 * c->faces[3 * f + 1]],
                     *d = &c->verts[3 * c->faces[3 * f + 2]];
        double e1[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]};
        double e2[3] = {d[0] - a[0], d[1] - a[1], d[2] - a[2]};
        double cr[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2],
                        e1[0] * e2[1] - e1[1] * e2[0]};
        double nr = std::sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]);
        BB_REQUIRE(nr > 0, BEAT_B200_INVALID_ARG, "set_mesh: degenerate face " + std::to_string(f));
        double n[3] = {cr[0] / nr, cr[1] / nr, cr[2] / nr};
        c->areas[f] = nr / 2.0;
        for (int i = 0; i < 3; ++i) {
            c->normals[3 * f + i] = n[i];
            cent[3 * f + i] = (a[i] + b[i] + d[i]) / 3.0;
        }
        double g11 = e1[0] * e1[0] + e1[1] * e1[1] + e1[2] * e1[2];
        double g12 = e1[0] * e2[0] + e1[1] * e2[1] + e1[2] * e2[2];
        double g22 = e2[0] * e2[0] + e2[1] * e2[1] + e2[2] * e2[2];
        double det = g11 * g22 - g12 * g12;
        double i11 = g22 / det, i12 = -g12 / det, i22 = g11 / det;
        double l1[3], l2[3], gr[3][3];
        for (int i = 0; i < 3; ++i) {
            l1[i] = e1[i] * i11 + e2[i] * i12;
            l2[i] = e1[i] * i12 + e2[i] * i22;
            gr[0][i] = -l1[i] - l2[i];
            gr[1][i] = l1[i];
            gr[2][i] = l2[i];
        }
        for (int v = 0; v < 3; ++v) {
            curls[9 * f + 3 * v + 0] = n[1] * gr[v][2] - n[2] * gr[v][1];
            curls[9 * f + 3 * v + 1] = n[2] * gr[v][0] - n[0] * gr[v][2];
            curls[9 * f + 3 * v + 2] = n[0] * gr[v][1] - n[1] * gr[v][0];
        }
        for (int q = 0; q < Q; ++q) {
            double xi = c->rule_pts[2 * q], et = c->rule_pts[2 * q + 1], l0 = 1.0 - xi - et;
            for (int i = 0; i < 3; ++i) qpts[3 * ((size_t)f * Q + q) + i] = l0 * a[i] + xi * b[i] + et * d[i];
        }
    }

    // Morton order of centroids
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    for (int f = 0; f < F; ++f)
        for (int i = 0; i < 3; ++i) {
            lo[i] = std::min(lo[i], cent[3 * f + i]);
            hi[i] = std::max(hi[i], cent[3 * f + i]);
        }
    double span = std::max({hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2], 1e-300});
    std::vector<uint64_t> code(F);
    for (int f = 0; f < F; ++f) {
        uint64_t m = 0;
        for (int i = 0; i < 3; ++i) {
            double u = (cent[3 * f + i] - lo[i]) / span;
            uint64_t q = (uint64_t)std::min(2097151.0, std::max(0.0, u * 2097151.0));
            m |= spread3(q) << i;
        }
        code[f] = m;
    }
    std::vector<int> order(F);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return code[a] < code[b]; });

    std::vector<int> pos_gv(3 * (size_t)F);
    std::vector<double> pq64(3 * (size_t)F * Q), pn64(3 * (size_t)F), pc64(9 * (size_t)F), pa64(F);
    std::vector<float> pq32(3 * (size_t)F * Q), pn32(3 * (size_t)F), pc32(9 * (size_t)F), pa32(F), pp32(F);
    for (int p = 0; p < F; ++p) {
        int f = order[p];
        for (int i = 0; i < 3; ++i) {
            pos_gv[3 * p + i] = c->faces[3 * f + i];
            pn64[3 * p + i] = c->normals[3 * f + i];
            pn32[3 * p + i] = (float)c->normals[3 * f + i];
        }
        for (int i = 0; i < 9; ++i) {
            pc64[9 * p + i] = curls[9 * f + i];
            pc32[9 * p + i] = (float)curls[9 * f + i];
        }
        for (int i = 0; i < 3 * Q; ++i) {
            pq64[3 * (size_t)p * Q + i] = qpts[3 * (size_t)f * Q + i];
            pq32[3 * (size_t)p * Q + i] = (float)qpts[3 * (size_t)f * Q + i];
        }
        pa64[p] = c->areas[f];
        pa32[p] = (float)c->areas[f];
        // every point y of a flat face has the same y . n (FP32, multiply then two fused adds)
        const float *q0 = &pq32[3 * (size_t)p * Q], *n = &pn32[3 * (size_t)p];
        pp32[p] = std::fmaf(q0[2], n[2], std::fmaf(q0[1], n[1], q0[0] * n[0]));
    }
    upload(c->pos_face, order);
    upload(c->pos_qpts64, pq64);
    upload(c->pos_qpts32, pq32);
    upload(c->pos_normal64, pn64);
    upload(c->pos_normal32, pn32);
    upload(c->pos_curl64, pc64);
    upload(c->pos_curl32, pc32);
    upload(c->pos_area64, pa64);
    upload(c->pos_area32, pa32);
    upload(c->pos_plane32, pp32);
    upload(c->pos_gvert, pos_gv);
    build_tiling(c->test_tiles, TEST_TILE_FACES, TEST_TILE_VERTS, pos_gv, F);
    build_tiling(c->trial_tiles, TRIAL_TILE_FACES, TRIAL_TILE_VERTS, pos_gv, F);
    build_tiling(c->sym_tiles, SYM_TILE_FACES, SYM_TILE_VERTS, pos_gv, F);

    upload(c->d_verts, c->verts);
    upload(c->d_faces, c->faces);
    {
        // vertex -> incident faces (CSR), for the admittance terms
        std::vector<int> vstart(V + 1, 0), vface(3 * (size_t)F);
        for (int f = 0; f < F; ++f)
            for (int a = 0; a < 3; ++a) ++vstart[c->faces[3 * f + a] + 1];
        for (int v = 0; v < V; ++v) vstart[v + 1] += vstart[v];
        std::vector<int> fill(vstart.begin(), vstart.end() - 1);
        for (int f = 0; f < F; ++f)
            for (int a = 0; a < 3; ++a) vface[fill[c->faces[3 * f + a]]++] = f;
        upload(c->vf_start, vstart);
        upload(c->vf_face, vface);
    }
    c->adm.free_();
    c->adm_set = false;
    upload(c->d_normals, c->normals);
    upload(c->d_areas, c->areas);
    upload(c->d_curls, curls);
    upload(c->d_qpts, qpts);

    // touching pairs, found per test element with the trial candidates in the
    // vertex -> element order of adjacent_trial_indices_by_test (reordered by
    // rule size once the rules are built, below)
    std::vector<int> vstart(V + 1, 0), vlist(3 * (size_t)F), fill(V, 0);
    for (int f = 0; f < F; ++f)
        for (int a = 0; a < 3; ++a) vstart[c->faces[3 * f + a] + 1]++;
    for (int v = 0; v < V; ++v) vstart[v + 1] += vstart[v];
    for (int f = 0; f < F; ++f)
        for (int a = 0; a < 3; ++a) {
            int v = c->faces[3 * f + a];
            vlist[vstart[v] + fill[v]++] = f;
        }
    std::vector<int> sp_t, sp_s, sp_r, seen(F, -1);
    std::vector<double> sp_j, sp_n;
    std::map<int, int> key_rule;
    std::vector<std::array<int, 5>> keys;
    for (int t = 0; t < F; ++t) {
        const int *ft = &c->faces[3 * t];
        for (int a = 0; a < 3; ++a) {
            int v = ft[a];
            for (int e = vstart[v]; e < vstart[v + 1]; ++e) {
                int s = vlist[e];
                if (seen[s] == t) continue;
                seen[s] = t;
                const int *fs = &c->faces[3 * s];
                int sa[3], sb[3], n = 0;
                for (int i = 0; i < 3; ++i)
                    for (int j = 0; j < 3; ++j)
                        if (ft[i] == fs[j]) {
                            sa[n] = i + 1;
                            sb[n] = j + 1;
                            ++n;
                        }
                if (n == 0) continue;
                int kind = n == 3 ? COINCIDENT : n == 2 ? EDGE : VERTEX;
                std::array<int, 5> key{kind, 0, 0, 0, 0};
                if (kind == EDGE) {
                    if (sb[1] < sb[0]) {
                        std::swap(sa[0], sa[1]);
                        std::swap(sb[0], sb[1]);
                    }
                    key = {kind, sa[0], sa[1], sb[0], sb[1]};
                } else if (kind == VERTEX) {
                    key = {kind, sa[0], 0, sb[0], 0};
                }
                int kc = (((key[0] * 4 + key[1]) * 4 + key[2]) * 4 + key[3]) * 4 + key[4];
                auto it = key_rule.find(kc);
                int r;
                if (it == key_rule.end()) {
                    r = (int)keys.size();
                    key_rule[kc] = r;
                    keys.push_back(key);
                } else {
                    r = it->second;
                }
                sp_t.push_back(t);
                sp_s.push_back(s);
                sp_r.push_back(r);
                sp_j.push_back((2.0 * c->areas[t]) * (2.0 * c->areas[s]));
                sp_n.push_back(c->normals[3 * t] * c->normals[3 * s] + c->normals[3 * t + 1] * c->normals[3 * s + 1] +
                               c->normals[3 * t + 2] * c->normals[3 * s + 2]);
            }
        }
    }
    c->npairs = (int64_t)sp_t.size();
    c->regular_pairs = (int64_t)F * F * (1 + c->nimg) - c->npairs;

    // touching image pairs: test element t and reflected trial element s
    // sharing vertex positions (image_singular_candidates and
    // geometric_adjacency_info, BeatEngineCore.jl:624-650,1152-1180; tolerance
    // 1e-8 as there); their rules join the same remapped-rule table
    std::vector<int> ip_t, ip_s, ip_r, ip_x;
    std::vector<double> ip_j, ip_n;
    if (c->nimg > 0) {
        const double tol = 1e-8;
        auto key_of = [&](double x, double y, double z) {
            return std::array<long long, 3>{(long long)std::llround(x / tol), (long long)std::llround(y / tol),
                                            (long long)std::llround(z / tol)};
        };
        std::map<std::array<long long, 3>, std::vector<int>> by_key;
        for (int t = 0; t < F; ++t)
            for (int a = 0; a < 3; ++a) {
                const double *p = &c->verts[3 * c->faces[3 * t + a]];
                by_key[key_of(p[0], p[1], p[2])].push_back(t);
            }
        for (int ix = 0; ix < c->nimg; ++ix) {
            const float *sg = c->img_sign[ix];
            std::map<std::pair<int, int>, int> seen_pair;
            for (int s = 0; s < F; ++s) {
                double sv[3][3];
                for (int b = 0; b < 3; ++b)
                    for (int i = 0; i < 3; ++i) sv[b][i] = sg[i] * c->verts[3 * c->faces[3 * s + b] + i];
                for (int b = 0; b < 3; ++b) {
                    auto it = by_key.find(key_of(sv[b][0], sv[b][1], sv[b][2]));
                    if (it == by_key.end()) continue;
                    for (int t : it->second) {
                        if (seen_pair.count({t, s})) continue;
                        seen_pair[{t, s}] = 1;
                        int sa[3], sb[3], n = 0;
                        for (int i = 0; i < 3; ++i)
                            for (int j = 0; j < 3; ++j) {
                                const double *tp = &c->verts[3 * c->faces[3 * t + i]];
                                const double d0 = tp[0] - sv[j][0], d1 = tp[1] - sv[j][1], d2 = tp[2] - sv[j][2];
                                if (std::sqrt(d0 * d0 + d1 * d1 + d2 * d2) <= tol && n < 3) {
                                    sa[n] = i + 1;
                                    sb[n] = j + 1;
                                    ++n;
                                }
                            }
                        if (n == 0) continue;
                        int kind = n == 3 ? COINCIDENT : n == 2 ? EDGE : VERTEX;
                        std::array<int, 5> key{kind, 0, 0, 0, 0};
                        if (kind == EDGE) {
                            if (sb[1] < sb[0]) {
                                std::swap(sa[0], sa[1]);
                                std::swap(sb[0], sb[1]);
                            }
                            key = {kind, sa[0], sa[1], sb[0], sb[1]};
                        } else if (kind == VERTEX) {
                            key = {kind, sa[0], 0, sb[0], 0};
                        }
                        int kc = (((key[0] * 4 + key[1]) * 4 + key[2]) * 4 + key[3]) * 4 + key[4];
                        auto kr = key_rule.find(kc);
                        int r;
                        if (kr == key_rule.end()) {
                            r = (int)keys.size();
                            key_rule[kc] = r;
                            keys.push_back(key);
                        } else {
                            r = kr->second;
                        }
                        ip_t.push_back(t);
                        ip_s.push_back(s);
                        ip_r.push_back(r);
                        ip_x.push_back(ix);
                        ip_j.push_back((2.0 * c->areas[t]) * (2.0 * c->areas[s]));
                        double nn = 0;
                        for (int i = 0; i < 3; ++i) nn += c->normals[3 * t + i] * sg[i] * c->normals[3 * s + i];
                        ip_n.push_back(nn);
                    }
                }
            }
        }
    }
    c->nimg_pairs = (int64_t)ip_t.size();
    c->nrules = (int)keys.size();
    std::vector<DuffyPt> base[4];
    for (int k = 1; k <= 3; ++k) base[k] = duffy(sing_order, k);
    std::vector<int> rstart{0};
    std::vector<double> rdata;
    for (auto &key : keys) {
        const auto &b = base[key[0]];
        for (const auto &pt : b) {
            double tx, ty, sx, sy;
            remap(key[0], key[1], key[2], pt.tx, pt.ty, tx, ty);
            remap(key[0], key[3], key[4], pt.sx, pt.sy, sx, sy);
            rdata.insert(rdata.end(), {tx, ty, sx, sy, pt.w});
        }
        rstart.push_back(rstart.back() + (int)b.size());
    }
    // Pairs in increasing order of their rule's point count (vertex, edge,
    // coincident at the same order), stably: the Duffy kernels give each pair
    // one warp, and a CTA's warps then hold pairs of one size and finish
    // together instead of idling beside its longest pair.  Increasing, so that
    // the mixed form's FP32 entries take their small vertex- and edge-pair
    // terms before the large self terms.
    auto by_rule_size = [&](std::vector<int> &t, std::vector<int> &s, std::vector<int> &r, std::vector<double> &j,
                            std::vector<double> &n, std::vector<int> *x) {
        std::vector<size_t> order(t.size());
        std::iota(order.begin(), order.end(), size_t(0));
        std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) {
            return rstart[r[a] + 1] - rstart[r[a]] < rstart[r[b] + 1] - rstart[r[b]];
        });
        auto apply = [&](auto &v) {
            auto w = v;
            for (size_t i = 0; i < order.size(); ++i) w[i] = v[order[i]];
            v.swap(w);
        };
        apply(t);
        apply(s);
        apply(r);
        apply(j);
        apply(n);
        if (x) apply(*x);
    };
    by_rule_size(sp_t, sp_s, sp_r, sp_j, sp_n, nullptr);
    by_rule_size(ip_t, ip_s, ip_r, ip_j, ip_n, &ip_x);
    upload(c->ip_test, ip_t);
    upload(c->ip_trial, ip_s);
    upload(c->ip_rule, ip_r);
    upload(c->ip_img, ip_x);
    upload(c->ip_jac, ip_j);
    upload(c->ip_nn, ip_n);
    upload(c->sp_test, sp_t);
    upload(c->sp_trial, sp_s);
    upload(c->sp_rule, sp_r);
    upload(c->sp_jac, sp_j);
    upload(c->sp_nn, sp_n);
    upload(c->rule_start, rstart);
    upload(c->rule_data, rdata);
}

// ---------------------------------------------------------------------------
// workspaces
// ---------------------------------------------------------------------------
// exterior_use_rhs_operator, exterior_rhs_policy.jl:25-44: the system matrix
// and the mapping are resident together, with 512 MiB for the transients
int rhs_use_operator(int mode, int excitations, int64_t matrix_bytes, int64_t operator_bytes,
                     int64_t available_bytes) {
    if (mode != BEAT_B200_RHS_AUTO && mode != BEAT_B200_RHS_MATRIX_FREE && mode != BEAT_B200_RHS_CACHED) return -1;
    if (mode == BEAT_B200_RHS_MATRIX_FREE) return 0;
    if (excitations < 1) return 0;
    if (mode == BEAT_B200_RHS_AUTO && excitations < 2) return 0;
    const int64_t margin = 512ll << 20;
    return operator_bytes > 0 && matrix_bytes >= 0 && matrix_bytes + operator_bytes + margin <= available_bytes;
}

void ensure_workspace(beat_b200_ctx *c, int precision, int R, int rhs_request) {
    BB_REQUIRE(c->F > 0, BEAT_B200_STATE, "no mesh: call beat_b200_set_mesh first");
    BB_REQUIRE(rhs_request >= BEAT_B200_RHS_AUTO && rhs_request <= BEAT_B200_RHS_CACHED, BEAT_B200_INVALID_ARG,
               "unknown right-hand-side mode");
    BB_REQUIRE(!(c->adm_set && rhs_request == BEAT_B200_RHS_MATRIX_FREE), BEAT_B200_INVALID_ARG,
               "an admittance needs the cached right-hand-side mapping B; the matrix-free mode was requested");
    Workspace &w = c->ws;
    const int N = c->V, F = c->F;
    const int64_t ld = ((int64_t)N + 127) / 128 * 128;
    const size_t csz = precision == BEAT_B200_FP64 ? 16 : 8;
    if (w.precision != precision || w.N != N) {
        w.A.free_();
        w.Aop.free_();
        w.B.free_();
        w.stage.free_();
        w.lu_valid = 0;
    }
    w.precision = precision;
    w.N = N;
    w.F = F;
    w.ld = ld;
    // the mode: free device memory plus what this context's matrix buffers hold
    const int64_t matrix_bytes = (int64_t)N * ld * (int64_t)csz * (precision == BEAT_B200_FP64 ? 1 : 2);
    const int64_t operator_bytes = (int64_t)N * F * (int64_t)csz;
    size_t free_b = 0, total_b = 0;
    BB_CUDA(cudaMemGetInfo(&free_b, &total_b));
    const int64_t available = (int64_t)free_b + (int64_t)(w.A.bytes + w.Aop.bytes + w.B.bytes);
    bool cached;
    if (c->adm_set) {
        cached = true;  // the admittance term A += B diag(a) P needs B
        BB_REQUIRE(rhs_use_operator(BEAT_B200_RHS_CACHED, std::max(R, 1), matrix_bytes, operator_bytes, available) ==
                       1,
                   BEAT_B200_OOM, "an admittance needs the right-hand-side mapping B, which does not fit in memory");
    } else {
        cached = rhs_use_operator(rhs_request, R, matrix_bytes, operator_bytes, available) == 1;
    }
    if (!cached) w.B.free_();
    w.A.alloc((size_t)N * ld * csz);
    if (precision != BEAT_B200_FP64) w.Aop.alloc((size_t)N * ld * csz);
    if (cached) {
        try {
            w.B.alloc((size_t)N * F * csz);
        } catch (const Error &e) {
            if (e.code != BEAT_B200_OOM || c->adm_set) throw;
            cached = false;  // the mapping did not fit after all: integrate the columns instead
        }
    }
    w.rhs_cached = cached ? 1 : 0;
    if (R > w.R || !w.b.p) {
        w.R = std::max(R, 1);
        w.b.free_();
        w.x.free_();
        w.q.free_();
    }
    w.b.alloc((size_t)N * w.R * 16);
    w.x.alloc((size_t)N * w.R * 16);
    w.q.alloc((size_t)F * w.R * 16);
    w.ipiv.alloc((size_t)(N + 256) * sizeof(int));
    w.perm.alloc((size_t)(N + 256) * sizeof(int));
}

void release_workspace(beat_b200_ctx *c) {
    lu_graph_release(c);
    Workspace &w = c->ws;
    for (DevBuf *b : {&w.A, &w.Aop, &w.B, &w.b, &w.x, &w.ipiv, &w.perm, &w.panel_scratch, &w.stage, &w.krylov,
                      &w.small, &w.q, &w.small_solve, &w.dinv, &w.field, &w.io, &w.qeff, &w.grad})
        b->free_();
    w.precision = -1;
    w.N = w.F = w.R = 0;
    w.lu_valid = 0;
    w.solve_epoch = 0;
}

int64_t device_bytes(const beat_b200_ctx *c) {
    int64_t s = 0;
    const Workspace &w = c->ws;
    for (const DevBuf *b : {&w.A, &w.Aop, &w.B, &w.b, &w.x, &w.ipiv, &w.perm, &w.panel_scratch, &w.stage, &w.krylov,
                            &w.small, &w.q, &w.small_solve, &w.dinv, &w.field, &w.io, &w.qeff, &w.grad})
        s += (int64_t)b->bytes;
    for (const DevBuf *b : {&c->pos_face, &c->pos_qpts64, &c->pos_qpts32, &c->pos_normal64, &c->pos_normal32,
                            &c->pos_curl64, &c->pos_curl32, &c->pos_area64, &c->pos_area32, &c->pos_plane32,
                            &c->pos_gvert,
                            &c->d_verts, &c->d_faces, &c->d_normals, &c->d_areas, &c->d_curls, &c->d_qpts,
                            &c->vf_start, &c->vf_face, &c->adm, &c->ip_test, &c->ip_trial, &c->ip_rule,
                            &c->ip_img, &c->ip_jac, &c->ip_nn, &c->rw_vert, &c->rw_weight,
                            &c->sp_test, &c->sp_trial, &c->sp_rule, &c->sp_jac, &c->sp_nn, &c->rule_start,
                            &c->rule_data, &c->status, &c->barrier})
        s += (int64_t)b->bytes;
    for (const Tiling *t : {&c->test_tiles, &c->trial_tiles, &c->sym_tiles})
        s += (int64_t)(t->face_start.bytes + t->vert_start.bytes + t->verts.bytes + t->local_vert.bytes +
                       t->incidence.bytes);
    return s;
}

int read_status(beat_b200_ctx *c) {
    int s = 0;
    BB_CUDA(cudaMemcpyAsync(&s, c->status.p, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    BB_CUDA(cudaStreamSynchronize(c->stream));
    return s;
}

}  // namespace bb
