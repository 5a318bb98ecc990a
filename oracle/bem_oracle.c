/*
 * bem_oracle.c -- FP64 CPU restatement of BEAT Engine's exterior Burton-Miller
 * direct-system path (fused regular + Duffy singular + identity assembly, one
 * partial-pivot complex LU for all right-hand sides, Galerkin field evaluation).
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the oracle: the parity tests, the
 * smoke check and the CPU-baseline leg of bench.py call it as the checker.  The
 * product library (beat_engine_b200/libbeatb200.so) never links, loads or runs
 * it.
 *
 * Pinned against the reference's own known answers (see tests/test_oracle_golden.py):
 *   - the Julia-produced per-frequency pressure and field norms of
 *     src/beat_engine/julia_local/results/baseline_sweep_cpu.json (sample.msh,
 *     order 2/2, 8 frequencies), compared at the reference CI's 1e-3;
 *   - the closed-form pulsating sphere gate (<= 0.05 dB, <= 0.5 deg) of
 *     julia_local/tests/analytical_exterior_tests.jl:122-155;
 *   - the oscillating-sphere (dipole) gate (< 8 %, halving under refinement)
 *     of julia_local/tests/axial_source_tests.jl:95-160.
 *
 * Reference files are cited relative to src/beat_engine/julia_local/.
 *
 * Conventions of this file:
 *   vertices  V x 3 doubles, row-major (x,y,z per vertex)
 *   faces     F x 3 ints, 0-based vertex indices, row-major
 *   complex   interleaved (re, im) doubles
 *   matrices  column-major like Julia: A[i + j*N], b[i + r*N], q[f + r*F]
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define BO_MAXQ 16
#define BO_OK 0
#define BO_EINVAL 1
#define BO_ENOMEM 2
#define BO_ESINGULAR 3
#define BO_ETOOCLOSE 4 /* a field point too close to the boundary for the adaptive correction */

#define BO_SKIP_REGULAR 1
#define BO_SKIP_SINGULAR 2
#define BO_SKIP_IDENTITY 4
#define BO_NO_CLEAR 8 /* accumulate into A and b as given (a slice of a larger assembly) */

static const double BO_PI = 3.14159265358979323846;

/* ------------------------------------------------------------------------ */
/* small vector helpers                                                      */
/* ------------------------------------------------------------------------ */
typedef struct { double x, y, z; } v3;
static inline v3 v3make(const double *p) { v3 r = {p[0], p[1], p[2]}; return r; }
static inline v3 v3sub(v3 a, v3 b) { v3 r = {a.x - b.x, a.y - b.y, a.z - b.z}; return r; }
static inline double v3dot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline v3 v3cross(v3 a, v3 b) {
    v3 r = {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
    return r;
}
static inline double v3norm(v3 a) { return sqrt(v3dot(a, a)); }

/* ------------------------------------------------------------------------ */
/* quadrature rules                                                          */
/* ------------------------------------------------------------------------ */

/* triangle_rule(T, order), BeatEngineCore.jl:660-692.  Weights include the
 * reference triangle's 1/2.  Orders other than <=1 and 4 fall to the 3-point
 * rule, exactly as the reference does. */
int bo_triangle_rule(int order, double *pts, double *w)
{
    if (order <= 1) {
        pts[0] = 1.0 / 3.0; pts[1] = 1.0 / 3.0; w[0] = 0.5;
        return 1;
    }
    if (order == 4) {
        static const double p[12] = {
            0.4459484909159651, 0.4459484909159651,
            0.0915762135097710, 0.0915762135097700,
            0.1081030181680700, 0.4459484909159651,
            0.4459484909159651, 0.1081030181680700,
            0.8168475729804590, 0.0915762135097700,
            0.0915762135097710, 0.8168475729804580};
        static const double ww[6] = {0.2233815896780110, 0.1099517436553220, 0.2233815896780110,
                                     0.2233815896780110, 0.1099517436553220, 0.1099517436553220};
        for (int i = 0; i < 12; ++i) pts[i] = p[i];
        for (int i = 0; i < 6; ++i) w[i] = 0.5 * ww[i];
        return 6;
    }
    pts[0] = 1.0 / 6.0; pts[1] = 1.0 / 6.0;
    pts[2] = 2.0 / 3.0; pts[3] = 1.0 / 6.0;
    pts[4] = 1.0 / 6.0; pts[5] = 2.0 / 3.0;
    w[0] = w[1] = w[2] = 1.0 / 6.0;
    return 3;
}

/* gauss_rule_1d(T, order) on [0,1], BeatEngineCore.jl:713-740.  Orders above
 * 4 use Newton iteration on the Legendre recurrence, which converges to the
 * same nodes the reference's Golub-Welsch eigen-decomposition returns. */
int bo_gauss_rule_1d(int order, double *x, double *w)
{
    if (order == 1) { x[0] = 0.5; w[0] = 1.0; return 1; }
    if (order == 2) {
        double a = 0.5 / sqrt(3.0);
        x[0] = 0.5 - a; x[1] = 0.5 + a; w[0] = w[1] = 0.5;
        return 2;
    }
    if (order == 3) {
        double a = sqrt(3.0 / 5.0) / 2.0;
        x[0] = 0.5 - a; x[1] = 0.5; x[2] = 0.5 + a;
        w[0] = 5.0 / 18.0; w[1] = 4.0 / 9.0; w[2] = 5.0 / 18.0;
        return 3;
    }
    if (order == 4) {
        double x1 = sqrt(3.0 / 7.0 - 2.0 / 7.0 * sqrt(6.0 / 5.0)) / 2.0;
        double x2 = sqrt(3.0 / 7.0 + 2.0 / 7.0 * sqrt(6.0 / 5.0)) / 2.0;
        double w1 = (18.0 + sqrt(30.0)) / 72.0;
        double w2 = (18.0 - sqrt(30.0)) / 72.0;
        x[0] = 0.5 - x2; x[1] = 0.5 - x1; x[2] = 0.5 + x1; x[3] = 0.5 + x2;
        w[0] = w2; w[1] = w1; w[2] = w1; w[3] = w2;
        return 4;
    }
    if (order < 1) return 0;
    /* Legendre roots on [-1,1], ascending, mapped to [0,1] (weights halved). */
    for (int i = 0; i < order; ++i) {
        double t = -cos(BO_PI * (i + 0.75) / (order + 0.5));
        for (int it = 0; it < 100; ++it) {
            double p0 = 1.0, p1 = t;
            for (int n = 2; n <= order; ++n) {
                double p2 = ((2.0 * n - 1.0) * t * p1 - (n - 1.0) * p0) / n;
                p0 = p1; p1 = p2;
            }
            double dp = order * (t * p1 - p0) / (t * t - 1.0);
            double dt = p1 / dp;
            t -= dt;
            if (fabs(dt) < 1e-16) break;
        }
        double p0 = 1.0, p1 = t;
        for (int n = 2; n <= order; ++n) {
            double p2 = ((2.0 * n - 1.0) * t * p1 - (n - 1.0) * p0) / n;
            p0 = p1; p1 = p2;
        }
        double dp = order * (t * p1 - p0) / (t * t - 1.0);
        x[i] = (t + 1.0) / 2.0;
        w[i] = 1.0 / ((1.0 - t * t) * dp * dp);
    }
    return order;
}

/* Duffy kinds, numbered as singular_kind_code, BeatEngineCore.jl:958-963. */
#define BO_COINCIDENT 1
#define BO_EDGE 2
#define BO_VERTEX 3

static int duffy_append(double *tp, double *sp, double *w, int n,
                        double tx, double ty, double sx, double sy, double wt)
{
    /* append_duffy_point!, BeatEngineCore.jl:804-808 */
    tp[2 * n] = tx - ty; tp[2 * n + 1] = ty;
    sp[2 * n] = sx - sy; sp[2 * n + 1] = sy;
    w[n] = wt;
    return n + 1;
}

/* duffy_rule(T, order, adjacency), BeatEngineCore.jl:742-802.  Returns the
 * number of point pairs; buffers must hold order^4 * 6 entries. */
int bo_duffy_rule(int order, int kind, double *tp, double *sp, double *w)
{
    double xr[64], wr[64];
    int m = bo_gauss_rule_1d(order, xr, wr);
    if (m <= 0 || m > 64) return 0;
    int nt = m * m, n = 0;
    double *tpx = malloc(sizeof(double) * nt * 2), *tw = malloc(sizeof(double) * nt);
    int c = 0;
    for (int i = 0; i < m; ++i)
        for (int j = 0; j < m; ++j) {
            tpx[2 * c] = xr[j]; tpx[2 * c + 1] = xr[i];
            tw[c] = wr[i] * wr[j];
            ++c;
        }
    for (int a = 0; a < nt; ++a)
        for (int b = 0; b < nt; ++b) {
            double xsi = tpx[2 * a], e1 = tpx[2 * a + 1], e2 = tpx[2 * b], e3 = tpx[2 * b + 1];
            double e12 = e1 * e2, e123 = e12 * e3;
            double bw = tw[a] * tw[b];
            if (kind == BO_COINCIDENT) {
                double wt = bw * xsi * xsi * xsi * e1 * e1 * e2;
                n = duffy_append(tp, sp, w, n, xsi, xsi * (1.0 - e1 + e12), xsi * (1.0 - e123), xsi * (1.0 - e1), wt);
                n = duffy_append(tp, sp, w, n, xsi * (1.0 - e123), xsi * (1.0 - e1), xsi, xsi * (1.0 - e1 + e12), wt);
                n = duffy_append(tp, sp, w, n, xsi, xsi * (e1 - e12 + e123), xsi * (1.0 - e12), xsi * (e1 - e12), wt);
                n = duffy_append(tp, sp, w, n, xsi * (1.0 - e12), xsi * (e1 - e12), xsi, xsi * (e1 - e12 + e123), wt);
                n = duffy_append(tp, sp, w, n, xsi * (1.0 - e123), xsi * (e1 - e123), xsi, xsi * (e1 - e12), wt);
                n = duffy_append(tp, sp, w, n, xsi, xsi * (e1 - e12), xsi * (1.0 - e123), xsi * (e1 - e123), wt);
            } else if (kind == BO_EDGE) {
                double wt = bw * xsi * xsi * xsi * e1 * e1;
                n = duffy_append(tp, sp, w, n, xsi, xsi * e1 * e3, xsi * (1.0 - e12), xsi * e1 * (1.0 - e2), wt);
                n = duffy_append(tp, sp, w, n, xsi, xsi * e1, xsi * (1.0 - e123), xsi * e1 * e2 * (1.0 - e3), wt * e2);
                n = duffy_append(tp, sp, w, n, xsi * (1.0 - e12), xsi * e1 * (1.0 - e2), xsi, xsi * e123, wt * e2);
                n = duffy_append(tp, sp, w, n, xsi * (1.0 - e123), xsi * e12 * (1.0 - e3), xsi, xsi * e1, wt * e2);
                n = duffy_append(tp, sp, w, n, xsi * (1.0 - e123), xsi * e1 * (1.0 - e2 * e3), xsi, xsi * e12, wt * e2);
            } else if (kind == BO_VERTEX) {
                double wt = bw * xsi * xsi * xsi * e2;
                n = duffy_append(tp, sp, w, n, xsi, xsi * e1, xsi * e2, xsi * e2 * e3, wt);
                n = duffy_append(tp, sp, w, n, xsi * e2, xsi * e2 * e3, xsi, xsi * e1, wt);
            }
        }
    free(tpx); free(tw);
    return n;
}

/* remap_shared_vertex / remap_shared_edge, BeatEngineCore.jl:810-826
 * (vertex ids 1-based as in the reference). */
static void remap_point(int kind, int va, int vb, const double *p, double *out)
{
    if (kind == BO_EDGE) {
        static const double ref[3][2] = {{0.0, 0.0}, {1.0, 0.0}, {0.0, 1.0}};
        int rem = 6 - va - vb;
        const double *v0 = ref[va - 1], *v1 = ref[vb - 1], *v2 = ref[rem - 1];
        out[0] = v0[0] + p[0] * (v1[0] - v0[0]) + p[1] * (v2[0] - v0[0]);
        out[1] = v0[1] + p[0] * (v1[1] - v0[1]) + p[1] * (v2[1] - v0[1]);
    } else if (kind == BO_VERTEX) {
        if (va == 1) { out[0] = p[0]; out[1] = p[1]; }
        else if (va == 2) { out[0] = 1.0 - p[0] - p[1]; out[1] = p[1]; }
        else { out[0] = p[0]; out[1] = 1.0 - p[0] - p[1]; }
    } else {
        out[0] = p[0]; out[1] = p[1];
    }
}

/* ------------------------------------------------------------------------ */
/* mesh data                                                                 */
/* ------------------------------------------------------------------------ */
typedef struct {
    int V, F, Q;
    const double *verts;
    const int *faces;
    double *normals; /* F x 3 */
    double *areas;   /* F */
    double *curls;   /* F x 9: curl of basis a at [9f + 3a + c] */
    double *qpts;    /* F x Q x 3 global rule points */
    double rpts[2 * BO_MAXQ], rw[BO_MAXQ], basis[3 * BO_MAXQ];
} bo_mesh;

/* BoundaryMesh constructor, BeatEngineCore.jl:344-364, and surface_curls,
 * BeatEngineCore.jl:856-873. */
static int mesh_init(bo_mesh *m, int V, const double *verts, int F, const int *faces, int order)
{
    memset(m, 0, sizeof(*m));
    m->V = V; m->F = F; m->verts = verts; m->faces = faces;
    m->Q = bo_triangle_rule(order, m->rpts, m->rw);
    m->normals = malloc(sizeof(double) * 3 * F);
    m->areas = malloc(sizeof(double) * F);
    m->curls = malloc(sizeof(double) * 9 * F);
    m->qpts = malloc(sizeof(double) * 3 * F * m->Q);
    if (!m->normals || !m->areas || !m->curls || !m->qpts) return BO_ENOMEM;
    for (int q = 0; q < m->Q; ++q) {
        m->basis[3 * q] = 1.0 - m->rpts[2 * q] - m->rpts[2 * q + 1];
        m->basis[3 * q + 1] = m->rpts[2 * q];
        m->basis[3 * q + 2] = m->rpts[2 * q + 1];
    }
    for (int f = 0; f < F; ++f) {
        const int *fc = faces + 3 * f;
        if (fc[0] < 0 || fc[0] >= V || fc[1] < 0 || fc[1] >= V || fc[2] < 0 || fc[2] >= V) return BO_EINVAL;
        v3 a = v3make(verts + 3 * fc[0]), b = v3make(verts + 3 * fc[1]), c = v3make(verts + 3 * fc[2]);
        v3 e1 = v3sub(b, a), e2 = v3sub(c, a);
        v3 cr = v3cross(e1, e2);
        double nrm = v3norm(cr);
        if (!(nrm > 0.0)) return BO_EINVAL;
        m->areas[f] = nrm / 2.0;
        v3 n = {cr.x / nrm, cr.y / nrm, cr.z / nrm};
        m->normals[3 * f] = n.x; m->normals[3 * f + 1] = n.y; m->normals[3 * f + 2] = n.z;
        /* lift = [e1 e2] * inv(gram) */
        double g11 = v3dot(e1, e1), g12 = v3dot(e1, e2), g22 = v3dot(e2, e2);
        double det = g11 * g22 - g12 * g12;
        double i11 = g22 / det, i12 = -g12 / det, i22 = g11 / det;
        v3 l1 = {e1.x * i11 + e2.x * i12, e1.y * i11 + e2.y * i12, e1.z * i11 + e2.z * i12};
        v3 l2 = {e1.x * i12 + e2.x * i22, e1.y * i12 + e2.y * i22, e1.z * i12 + e2.z * i22};
        v3 g[3] = {{-l1.x - l2.x, -l1.y - l2.y, -l1.z - l2.z}, l1, l2};
        for (int i = 0; i < 3; ++i) {
            v3 cu = v3cross(n, g[i]);
            m->curls[9 * f + 3 * i] = cu.x; m->curls[9 * f + 3 * i + 1] = cu.y; m->curls[9 * f + 3 * i + 2] = cu.z;
        }
        for (int q = 0; q < m->Q; ++q) {
            double xi = m->rpts[2 * q], et = m->rpts[2 * q + 1], l0 = 1.0 - xi - et;
            m->qpts[3 * (f * m->Q + q)] = l0 * a.x + xi * b.x + et * c.x;
            m->qpts[3 * (f * m->Q + q) + 1] = l0 * a.y + xi * b.y + et * c.y;
            m->qpts[3 * (f * m->Q + q) + 2] = l0 * a.z + xi * b.z + et * c.z;
        }
    }
    return BO_OK;
}

static void mesh_free(bo_mesh *m)
{
    free(m->normals); free(m->areas); free(m->curls); free(m->qpts);
}

int bo_mesh_geometry(int V, const double *verts, int F, const int *faces,
                     double *normals, double *areas, double *curls)
{
    bo_mesh m;
    int st = mesh_init(&m, V, verts, F, faces, 4);
    if (st == BO_OK) {
        memcpy(normals, m.normals, sizeof(double) * 3 * F);
        memcpy(areas, m.areas, sizeof(double) * F);
        memcpy(curls, m.curls, sizeof(double) * 9 * F);
    }
    mesh_free(&m);
    return st;
}

/* vertex -> incident elements, in increasing element order (the insertion
 * order of adjacent_trial_indices_by_test, BeatEngineCore.jl:925-945). */
typedef struct { int *start, *list; } bo_v2e;
static int v2e_build(const bo_mesh *m, bo_v2e *g)
{
    g->start = calloc(m->V + 1, sizeof(int));
    g->list = malloc(sizeof(int) * 3 * m->F);
    if (!g->start || !g->list) return BO_ENOMEM;
    for (int f = 0; f < m->F; ++f)
        for (int a = 0; a < 3; ++a) g->start[m->faces[3 * f + a] + 1]++;
    for (int v = 0; v < m->V; ++v) g->start[v + 1] += g->start[v];
    int *fill = calloc(m->V, sizeof(int));
    for (int f = 0; f < m->F; ++f)
        for (int a = 0; a < 3; ++a) {
            int v = m->faces[3 * f + a];
            g->list[g->start[v] + fill[v]++] = f;
        }
    free(fill);
    return BO_OK;
}

static inline int faces_adjacent(const int *a, const int *b)
{
    /* elements_are_adjacent, BeatEngineCore.jl:584-594 */
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            if (a[i] == b[j]) return 1;
    return 0;
}

/* adjacency_info, BeatEngineCore.jl:596-622: kind and 1-based shared local
 * vertex ids (test a,b; trial a,b). */
static int adjacency_info(const int *fa, const int *fb, int *ta, int *tb, int *sa, int *sb)
{
    int sh_a[3], sh_b[3], n = 0;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            if (fa[i] == fb[j]) { sh_a[n] = i + 1; sh_b[n] = j + 1; ++n; }
    *ta = *tb = *sa = *sb = 0;
    if (n == 3) return BO_COINCIDENT;
    if (n == 2) {
        if (sh_b[1] < sh_b[0]) {
            int t = sh_a[0]; sh_a[0] = sh_a[1]; sh_a[1] = t;
            t = sh_b[0]; sh_b[0] = sh_b[1]; sh_b[1] = t;
        }
        *ta = sh_a[0]; *tb = sh_a[1]; *sa = sh_b[0]; *sb = sh_b[1];
        return BO_EDGE;
    }
    if (n == 1) { *ta = sh_a[0]; *sa = sh_b[0]; return BO_VERTEX; }
    return 0;
}

/* ------------------------------------------------------------------------ */
/* singular correction cache (build_singular_correction_cache,               */
/* BeatEngineCore.jl:994-1089)                                               */
/* ------------------------------------------------------------------------ */
typedef struct {
    int npairs;
    int *test, *trial, *rule;    /* per pair */
    double *jac, *nn;            /* per pair */
    int *by_test_start;          /* F + 1: pairs are stored grouped by test */
    int nrules;
    int *rule_start;             /* nrules + 1 */
    double *rt, *rs, *rw;        /* concatenated remapped rules */
} bo_singular;

static void singular_free(bo_singular *s)
{
    free(s->test); free(s->trial); free(s->rule); free(s->jac); free(s->nn);
    free(s->by_test_start); free(s->rule_start); free(s->rt); free(s->rs); free(s->rw);
}

static int singular_build(const bo_mesh *m, int order, bo_singular *s)
{
    memset(s, 0, sizeof(*s));
    bo_v2e g;
    if (v2e_build(m, &g) != BO_OK) return BO_ENOMEM;
    int F = m->F;
    int cap = 16 * F + 64;
    s->test = malloc(sizeof(int) * cap); s->trial = malloc(sizeof(int) * cap);
    s->rule = malloc(sizeof(int) * cap);
    s->jac = malloc(sizeof(double) * cap); s->nn = malloc(sizeof(double) * cap);
    s->by_test_start = calloc(F + 1, sizeof(int));
    int key_to_rule[4 * 4 * 4 * 4 * 4];
    for (int i = 0; i < 1024; ++i) key_to_rule[i] = -1;
    int keys[64][5];
    int *seen = malloc(sizeof(int) * F);
    for (int i = 0; i < F; ++i) seen[i] = -1;
    int np = 0;
    for (int t = 0; t < F; ++t) {
        const int *ft = m->faces + 3 * t;
        s->by_test_start[t] = np;
        for (int a = 0; a < 3; ++a) {
            int v = ft[a];
            for (int e = g.start[v]; e < g.start[v + 1]; ++e) {
                int sidx = g.list[e];
                if (seen[sidx] == t) continue;
                seen[sidx] = t;
                int ta, tb, sa, sb;
                int kind = adjacency_info(ft, m->faces + 3 * sidx, &ta, &tb, &sa, &sb);
                if (kind == 0) continue;
                int key = (((kind * 4 + ta) * 4 + tb) * 4 + sa) * 4 + sb;
                if (key_to_rule[key] < 0) {
                    keys[s->nrules][0] = kind; keys[s->nrules][1] = ta; keys[s->nrules][2] = tb;
                    keys[s->nrules][3] = sa; keys[s->nrules][4] = sb;
                    key_to_rule[key] = s->nrules++;
                }
                if (np >= cap) {
                    cap *= 2;
                    s->test = realloc(s->test, sizeof(int) * cap); s->trial = realloc(s->trial, sizeof(int) * cap);
                    s->rule = realloc(s->rule, sizeof(int) * cap);
                    s->jac = realloc(s->jac, sizeof(double) * cap); s->nn = realloc(s->nn, sizeof(double) * cap);
                }
                s->test[np] = t; s->trial[np] = sidx; s->rule[np] = key_to_rule[key];
                s->jac[np] = (2.0 * m->areas[t]) * (2.0 * m->areas[sidx]);
                s->nn[np] = m->normals[3 * t] * m->normals[3 * sidx] + m->normals[3 * t + 1] * m->normals[3 * sidx + 1] +
                            m->normals[3 * t + 2] * m->normals[3 * sidx + 2];
                ++np;
            }
        }
    }
    s->by_test_start[F] = np;
    s->npairs = np;
    free(seen); free(g.start); free(g.list);

    /* base rules and their orientation remaps (remapped_duffy_rule,
     * BeatEngineCore.jl:965-985) */
    int nb = order * order * order * order * 6;
    double *bt[4], *bs[4], *bw[4];
    int bn[4] = {0, 0, 0, 0};
    for (int k = 1; k <= 3; ++k) {
        bt[k] = malloc(sizeof(double) * 2 * nb); bs[k] = malloc(sizeof(double) * 2 * nb);
        bw[k] = malloc(sizeof(double) * nb);
        bn[k] = bo_duffy_rule(order, k, bt[k], bs[k], bw[k]);
    }
    s->rule_start = malloc(sizeof(int) * (s->nrules + 1));
    int tot = 0;
    for (int r = 0; r < s->nrules; ++r) { s->rule_start[r] = tot; tot += bn[keys[r][0]]; }
    s->rule_start[s->nrules] = tot;
    s->rt = malloc(sizeof(double) * 2 * (tot + 1)); s->rs = malloc(sizeof(double) * 2 * (tot + 1));
    s->rw = malloc(sizeof(double) * (tot + 1));
    for (int r = 0; r < s->nrules; ++r) {
        int k = keys[r][0], o = s->rule_start[r];
        for (int q = 0; q < bn[k]; ++q) {
            remap_point(k, keys[r][1], keys[r][2], bt[k] + 2 * q, s->rt + 2 * (o + q));
            remap_point(k, keys[r][3], keys[r][4], bs[k] + 2 * q, s->rs + 2 * (o + q));
            s->rw[o + q] = bw[k][q];
        }
    }
    for (int k = 1; k <= 3; ++k) { free(bt[k]); free(bs[k]); free(bw[k]); }
    return BO_OK;
}

/* Exposed for host-logic tests: counts and the (test, trial, kind) list. */
int bo_singular_pairs(int V, const double *verts, int F, const int *faces, int order,
                      int capacity, int *test, int *trial, int *rule, int *nrules_out, int *npoints_out)
{
    bo_mesh m;
    int st = mesh_init(&m, V, verts, F, faces, 4);
    if (st != BO_OK) { mesh_free(&m); return -st; }
    bo_singular s;
    singular_build(&m, order, &s);
    int np = s.npairs;
    for (int i = 0; i < np && i < capacity; ++i) { test[i] = s.test[i]; trial[i] = s.trial[i]; rule[i] = s.rule[i]; }
    if (nrules_out) *nrules_out = s.nrules;
    if (npoints_out) {
        long tot = 0;
        for (int i = 0; i < np; ++i) tot += s.rule_start[s.rule[i] + 1] - s.rule_start[s.rule[i]];
        *npoints_out = (int)(tot > 2147483647L ? 2147483647L : tot);
    }
    singular_free(&s);
    mesh_free(&m);
    return np;
}

/* ------------------------------------------------------------------------ */
/* Burton-Miller pair blocks                                                 */
/* ------------------------------------------------------------------------ */

/* One point pair of _beat_cpu_bm_regular_pair_blocks / _beat_cpu_bm_pair_blocks,
 * BeatEngineCpuBurtonMiller.jl:62-167, with the green function of
 * BeatEngineCpuAssembly.jl:1-6.  Accumulates lhs_scale and rhs_scale into the
 * 3x3 / 3 blocks with the given basis values, and green*weight into curl. */
static inline void bm_point(v3 x, v3 y, const double *bt, const double *bs, double weight,
                            v3 nt, v3 ns, double k, double eta, double k2n_im,
                            double *lhs, double *rhs, double *curl)
{
    v3 r = v3sub(y, x);
    double radius = v3norm(r);
    if (radius == 0.0) return;
    double inv_r = 1.0 / radius;
    double phase = k * radius;
    double scale = (1.0 / (4.0 * BO_PI)) * inv_r;
    double sn = sin(phase), cs = cos(phase);
    double g_re = cs * scale, g_im = sn * scale;
    /* grad_scale = green * (-inv_r + i k) */
    double gs_re = g_re * (-inv_r) - g_im * k;
    double gs_im = g_re * k + g_im * (-inv_r);
    double wg_re = g_re * weight, wg_im = g_im * weight;
    double dn_s = v3dot(r, ns) * inv_r;
    double dn_t = -v3dot(r, nt) * inv_r;
    /* lhs_scale = -grad_scale*dn_s*weight - k2n*wg, with k2n = i*k2n_im */
    double ls_re = -gs_re * dn_s * weight + k2n_im * wg_im;
    double ls_im = -gs_im * dn_s * weight - k2n_im * wg_re;
    /* rhs_scale = -wg - eta*grad_scale*dn_t*weight, with eta = i*eta */
    double t_re = gs_re * dn_t * weight, t_im = gs_im * dn_t * weight;
    double rs_re = -wg_re + eta * t_im;
    double rs_im = -wg_im - eta * t_re;
    curl[0] += wg_re; curl[1] += wg_im;
    for (int a = 0; a < 3; ++a) {
        rhs[2 * a] += bt[a] * rs_re; rhs[2 * a + 1] += bt[a] * rs_im;
        for (int b = 0; b < 3; ++b) {
            double bp = bt[a] * bs[b];
            lhs[2 * (3 * a + b)] += bp * ls_re;
            lhs[2 * (3 * a + b) + 1] += bp * ls_im;
        }
    }
}

static inline void bm_finish(const double *ct, const double *cs, double eta, const double *curl, double *lhs)
{
    /* curl_total *= coupling; lhs += dot(curl_t, curl_s) * curl_total */
    double c_re = -eta * curl[1], c_im = eta * curl[0];
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) {
            double d = ct[3 * a] * cs[3 * b] + ct[3 * a + 1] * cs[3 * b + 1] + ct[3 * a + 2] * cs[3 * b + 2];
            lhs[2 * (3 * a + b)] += d * c_re;
            lhs[2 * (3 * a + b) + 1] += d * c_im;
        }
}

static void regular_pair(const bo_mesh *m, int t, int s, double k, double eta, double *lhs, double *rhs)
{
    v3 nt = v3make(m->normals + 3 * t), ns = v3make(m->normals + 3 * s);
    double np = v3dot(nt, ns);
    double jac = 4.0 * m->areas[t] * m->areas[s];
    double k2n_im = eta * (k * k * np);
    double curl[2] = {0.0, 0.0};
    memset(lhs, 0, sizeof(double) * 18); memset(rhs, 0, sizeof(double) * 6);
    int Q = m->Q;
    for (int a = 0; a < Q; ++a) {
        v3 x = v3make(m->qpts + 3 * (t * Q + a));
        for (int b = 0; b < Q; ++b) {
            v3 y = v3make(m->qpts + 3 * (s * Q + b));
            bm_point(x, y, m->basis + 3 * a, m->basis + 3 * b, m->rw[a] * m->rw[b] * jac,
                     nt, ns, k, eta, k2n_im, lhs, rhs, curl);
        }
    }
    bm_finish(m->curls + 9 * t, m->curls + 9 * s, eta, curl, lhs);
}

static void singular_pair(const bo_mesh *m, const bo_singular *sc, int p, double k, double eta, double *lhs, double *rhs)
{
    int t = sc->test[p], s = sc->trial[p], r = sc->rule[p];
    v3 nt = v3make(m->normals + 3 * t), ns = v3make(m->normals + 3 * s);
    double k2n_im = eta * (k * k * sc->nn[p]);
    double jac = sc->jac[p];
    double curl[2] = {0.0, 0.0};
    memset(lhs, 0, sizeof(double) * 18); memset(rhs, 0, sizeof(double) * 6);
    const int *ft = m->faces + 3 * t, *fs = m->faces + 3 * s;
    v3 ta = v3make(m->verts + 3 * ft[0]), tb = v3make(m->verts + 3 * ft[1]), tc = v3make(m->verts + 3 * ft[2]);
    v3 sa = v3make(m->verts + 3 * fs[0]), sb = v3make(m->verts + 3 * fs[1]), sc3 = v3make(m->verts + 3 * fs[2]);
    for (int q = sc->rule_start[r]; q < sc->rule_start[r + 1]; ++q) {
        double xi = sc->rt[2 * q], et = sc->rt[2 * q + 1];
        double yi = sc->rs[2 * q], ye = sc->rs[2 * q + 1];
        double bt[3] = {1.0 - xi - et, xi, et}, bs[3] = {1.0 - yi - ye, yi, ye};
        v3 x = {bt[0] * ta.x + bt[1] * tb.x + bt[2] * tc.x, bt[0] * ta.y + bt[1] * tb.y + bt[2] * tc.y,
                bt[0] * ta.z + bt[1] * tb.z + bt[2] * tc.z};
        v3 y = {bs[0] * sa.x + bs[1] * sb.x + bs[2] * sc3.x, bs[0] * sa.y + bs[1] * sb.y + bs[2] * sc3.y,
                bs[0] * sa.z + bs[1] * sb.z + bs[2] * sc3.z};
        bm_point(x, y, bt, bs, sc->rw[q] * jac, nt, ns, k, eta, k2n_im, lhs, rhs, curl);
    }
    bm_finish(m->curls + 9 * t, m->curls + 9 * s, eta, curl, lhs);
}

/* _beat_cpu_bm_scatter!, BeatEngineCpuBurtonMiller.jl:26-51 */
static void scatter(const bo_mesh *m, int t, int s, const double *lhs, const double *rhs,
                    int R, const double *q, double *A, double *b)
{
    int N = m->V, F = m->F;
    const int *ft = m->faces + 3 * t, *fs = m->faces + 3 * s;
    for (int a = 0; a < 3; ++a) {
        int row = ft[a];
        for (int d = 0; d < R; ++d) {
            double qr = q[2 * (s + (size_t)d * F)], qi = q[2 * (s + (size_t)d * F) + 1];
            b[2 * (row + (size_t)d * N)] += rhs[2 * a] * qr - rhs[2 * a + 1] * qi;
            b[2 * (row + (size_t)d * N) + 1] += rhs[2 * a] * qi + rhs[2 * a + 1] * qr;
        }
        for (int c = 0; c < 3; ++c) {
            size_t col = fs[c];
            A[2 * (row + col * N)] += lhs[2 * (3 * a + c)];
            A[2 * (row + col * N) + 1] += lhs[2 * (3 * a + c) + 1];
        }
    }
}

/* greedy vertex colouring, _beat_cpu_element_color_groups,
 * BeatEngineCpuAssembly.jl:102-130.  Returns the number of colours; order[]
 * lists elements grouped by colour, start[] the group offsets. */
static int colour_groups(const bo_mesh *m, int *order, int *start)
{
    int F = m->F, V = m->V;
    uint64_t *vmask = calloc(V, sizeof(uint64_t));
    int *col = malloc(sizeof(int) * F);
    int ncol = 0;
    for (int f = 0; f < F; ++f) {
        uint64_t used = 0;
        for (int a = 0; a < 3; ++a) used |= vmask[m->faces[3 * f + a]];
        int c = 0;
        while (c < 63 && (used >> c) & 1ull) ++c;
        col[f] = c;
        if (c + 1 > ncol) ncol = c + 1;
        for (int a = 0; a < 3; ++a) vmask[m->faces[3 * f + a]] |= 1ull << c;
    }
    int pos = 0;
    for (int c = 0; c < ncol; ++c) {
        start[c] = pos;
        for (int f = 0; f < F; ++f)
            if (col[f] == c) order[pos++] = f;
    }
    start[ncol] = pos;
    free(vmask); free(col);
    return ncol;
}

/* assemble_burton_miller_neumann_system_cpu, BeatEngineCpuBurtonMiller.jl:276-469
 * (symmetry off).  A (N x N) and b (N x R) are overwritten.  k is the signed
 * wavenumber outgoing_wavenumber(k); eta the imaginary part of
 * burton_miller_coupling(k) (BeatEnginePhasor.jl:8-12).
 * test_begin/test_end restrict the regular and singular passes to a range of
 * test elements (the CPU-baseline sample); pass 0, F for the full system. */
int bo_assemble_range(int V, const double *verts, int F, const int *faces,
                      int quad_order, int sing_order, double k, double eta,
                      int R, const double *q, double *A, double *b,
                      int nthreads, int flags, int test_begin, int test_end)
{
    if (V <= 0 || F <= 0 || R < 0 || !verts || !faces || !A || (R > 0 && (!b || !q))) return BO_EINVAL;
    bo_mesh m;
    int st = mesh_init(&m, V, verts, F, faces, quad_order);
    if (st != BO_OK) { mesh_free(&m); return st; }
    int N = V;
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
    if (!(flags & BO_NO_CLEAR)) {
        memset(A, 0, sizeof(double) * 2 * (size_t)N * N);
        if (R > 0) memset(b, 0, sizeof(double) * 2 * (size_t)N * R);
    }
    if (test_begin < 0) test_begin = 0;
    if (test_end > F) test_end = F;

    int *order = malloc(sizeof(int) * F), *start = malloc(sizeof(int) * 65);
    int ncol = colour_groups(&m, order, start);

    if (!(flags & BO_SKIP_REGULAR)) {
        for (int c = 0; c < ncol; ++c) {
#pragma omp parallel for schedule(dynamic, 1)
            for (int i = start[c]; i < start[c + 1]; ++i) {
                int t = order[i];
                if (t < test_begin || t >= test_end) continue;
                double lhs[18], rhs[6];
                for (int s = 0; s < F; ++s) {
                    if (faces_adjacent(faces + 3 * t, faces + 3 * s)) continue;
                    regular_pair(&m, t, s, k, eta, lhs, rhs);
                    scatter(&m, t, s, lhs, rhs, R, q, A, b);
                }
            }
        }
    }
    if (!(flags & BO_SKIP_SINGULAR)) {
        bo_singular sc;
        singular_build(&m, sing_order, &sc);
        for (int c = 0; c < ncol; ++c) {
#pragma omp parallel for schedule(dynamic, 4)
            for (int i = start[c]; i < start[c + 1]; ++i) {
                int t = order[i];
                if (t < test_begin || t >= test_end) continue;
                double lhs[18], rhs[6];
                for (int p = sc.by_test_start[t]; p < sc.by_test_start[t + 1]; ++p) {
                    singular_pair(&m, &sc, p, k, eta, lhs, rhs);
                    scatter(&m, t, sc.trial[p], lhs, rhs, R, q, A, b);
                }
            }
        }
        singular_free(&sc);
    }
    if (!(flags & BO_SKIP_IDENTITY)) {
        /* lhs += 0.5 M_p1p1; rhs += -0.5 eta M_p1dp0 q  (l2_identity_element_matrix,
         * BeatEngineCore.jl:905-923; assemble_l2_identity_matrix, :1187-1214) */
        for (int f = 0; f < F; ++f) {
            double jac = 2.0 * m.areas[f];
            double blk[9] = {0}, col[3] = {0};
            for (int qq = 0; qq < m.Q; ++qq) {
                const double *ph = m.basis + 3 * qq;
                for (int a = 0; a < 3; ++a) {
                    col[a] += ph[a] * m.rw[qq] * jac;
                    for (int c = 0; c < 3; ++c) blk[3 * a + c] += ph[a] * ph[c] * m.rw[qq] * jac;
                }
            }
            const int *fc = faces + 3 * f;
            for (int a = 0; a < 3; ++a) {
                for (int c = 0; c < 3; ++c) A[2 * (fc[a] + (size_t)fc[c] * N)] += 0.5 * blk[3 * a + c];
                for (int d = 0; d < R; ++d) {
                    double qr = q[2 * (f + (size_t)d * F)], qi = q[2 * (f + (size_t)d * F) + 1];
                    /* (-0.5 * i*eta) * col * q */
                    b[2 * (fc[a] + (size_t)d * N)] += 0.5 * eta * col[a] * qi;
                    b[2 * (fc[a] + (size_t)d * N) + 1] += -0.5 * eta * col[a] * qr;
                }
            }
        }
    }
    free(order); free(start);
    mesh_free(&m);
    return BO_OK;
}

int bo_assemble(int V, const double *verts, int F, const int *faces,
                int quad_order, int sing_order, double k, double eta,
                int R, const double *q, double *A, double *b, int nthreads, int flags)
{
    return bo_assemble_range(V, verts, F, faces, quad_order, sing_order, k, eta, R, q, A, b,
                             nthreads, flags, 0, F);
}

/* ------------------------------------------------------------------------ */
/* dense LU with partial pivoting (what LinearAlgebra.lu! computes through   */
/* LAPACK zgetrf, BeatEngineDenseSolve.jl:1104-1110): pivot = first maximum  */
/* of |re| + |im| as izamax chooses.  Column-major, in place.                */
/* ------------------------------------------------------------------------ */
int bo_lu_factor(int N, double *A, int *piv, int nthreads)
{
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
    for (int j = 0; j < N; ++j) {
        int p = j;
        double best = -1.0;
        for (int i = j; i < N; ++i) {
            double v = fabs(A[2 * (i + (size_t)j * N)]) + fabs(A[2 * (i + (size_t)j * N) + 1]);
            if (v > best) { best = v; p = i; }
        }
        piv[j] = p;
        if (best == 0.0) return BO_ESINGULAR;
        if (p != j) {
            for (int c = 0; c < N; ++c) {
                size_t a = 2 * (j + (size_t)c * N), bb = 2 * (p + (size_t)c * N);
                double t0 = A[a], t1 = A[a + 1];
                A[a] = A[bb]; A[a + 1] = A[bb + 1]; A[bb] = t0; A[bb + 1] = t1;
            }
        }
        double pr = A[2 * (j + (size_t)j * N)], pi = A[2 * (j + (size_t)j * N) + 1];
        double den = pr * pr + pi * pi;
        double ir = pr / den, ii = -pi / den;
        for (int i = j + 1; i < N; ++i) {
            double ar = A[2 * (i + (size_t)j * N)], ai = A[2 * (i + (size_t)j * N) + 1];
            A[2 * (i + (size_t)j * N)] = ar * ir - ai * ii;
            A[2 * (i + (size_t)j * N) + 1] = ar * ii + ai * ir;
        }
#pragma omp parallel for schedule(static) if (N - j > 256)
        for (int c = j + 1; c < N; ++c) {
            double ur = A[2 * (j + (size_t)c * N)], ui = A[2 * (j + (size_t)c * N) + 1];
            if (ur == 0.0 && ui == 0.0) continue;
            double *colc = A + 2 * (size_t)c * N;
            const double *colj = A + 2 * (size_t)j * N;
            for (int i = j + 1; i < N; ++i) {
                double lr = colj[2 * i], li = colj[2 * i + 1];
                colc[2 * i] -= lr * ur - li * ui;
                colc[2 * i + 1] -= lr * ui + li * ur;
            }
        }
    }
    return BO_OK;
}

int bo_lu_solve(int N, const double *LU, const int *piv, int R, double *B)
{
    for (int d = 0; d < R; ++d) {
        double *x = B + 2 * (size_t)d * N;
        for (int j = 0; j < N; ++j)
            if (piv[j] != j) {
                double t0 = x[2 * j], t1 = x[2 * j + 1];
                x[2 * j] = x[2 * piv[j]]; x[2 * j + 1] = x[2 * piv[j] + 1];
                x[2 * piv[j]] = t0; x[2 * piv[j] + 1] = t1;
            }
        for (int j = 0; j < N; ++j) {
            double xr = x[2 * j], xi = x[2 * j + 1];
            const double *col = LU + 2 * (size_t)j * N;
            for (int i = j + 1; i < N; ++i) {
                x[2 * i] -= col[2 * i] * xr - col[2 * i + 1] * xi;
                x[2 * i + 1] -= col[2 * i] * xi + col[2 * i + 1] * xr;
            }
        }
        for (int j = N - 1; j >= 0; --j) {
            const double *col = LU + 2 * (size_t)j * N;
            double pr = col[2 * j], pi = col[2 * j + 1], den = pr * pr + pi * pi;
            double xr = x[2 * j], xi = x[2 * j + 1];
            double yr = (xr * pr + xi * pi) / den, yi = (xi * pr - xr * pi) / den;
            x[2 * j] = yr; x[2 * j + 1] = yi;
            for (int i = 0; i < j; ++i) {
                x[2 * i] -= col[2 * i] * yr - col[2 * i + 1] * yi;
                x[2 * i + 1] -= col[2 * i] * yi + col[2 * i + 1] * yr;
            }
        }
    }
    return BO_OK;
}

/* ------------------------------------------------------------------------ */
/* field evaluation: evaluate_galerkin_field_cpu, BeatEngineCpuField.jl:1-49, */
/* with the source cache of build_field_evaluation_cache,                    */
/* BeatEngineCore.jl:1770-1810 (symmetry off).                               */
/* p (N x R) and q (F x R) column-major; out (M x R).                        */
/* ------------------------------------------------------------------------ */
int bo_field(int V, const double *verts, int F, const int *faces, int quad_order, double k,
             int M, const double *points, int R, const double *p, const double *q, double *out, int nthreads)
{
    bo_mesh m;
    int st = mesh_init(&m, V, verts, F, faces, quad_order);
    if (st != BO_OK) { mesh_free(&m); return st; }
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
    int N = V, Q = m.Q;
#pragma omp parallel for schedule(dynamic, 4)
    for (int i = 0; i < M; ++i) {
        v3 x = v3make(points + 3 * i);
        for (int d = 0; d < R; ++d) { out[2 * (i + (size_t)d * M)] = 0.0; out[2 * (i + (size_t)d * M) + 1] = 0.0; }
        for (int f = 0; f < F; ++f) {
            const int *fc = faces + 3 * f;
            v3 n = v3make(m.normals + 3 * f);
            double jac = 2.0 * m.areas[f];
            for (int qq = 0; qq < Q; ++qq) {
                v3 y = v3make(m.qpts + 3 * (f * Q + qq));
                v3 r = v3sub(y, x);
                double radius = v3norm(r);
                if (radius == 0.0) continue;
                double phase = k * radius;
                double gsc = 1.0 / (4.0 * BO_PI * radius);
                double g_re = cos(phase) * gsc, g_im = sin(phase) * gsc;
                double proj = v3dot(r, n) / radius;
                /* double_layer = green * (i k - 1/r) * proj */
                double fr = -1.0 / radius, fi = k;
                double dl_re = (g_re * fr - g_im * fi) * proj, dl_im = (g_re * fi + g_im * fr) * proj;
                double w = m.rw[qq] * jac;
                const double *ph = m.basis + 3 * qq;
                for (int d = 0; d < R; ++d) {
                    const double *pd = p + 2 * (size_t)d * N;
                    double ps_re = (ph[0] * pd[2 * fc[0]] + ph[1] * pd[2 * fc[1]] + ph[2] * pd[2 * fc[2]]) * w;
                    double ps_im = (ph[0] * pd[2 * fc[0] + 1] + ph[1] * pd[2 * fc[1] + 1] + ph[2] * pd[2 * fc[2] + 1]) * w;
                    double qs_re = q[2 * (f + (size_t)d * F)] * w, qs_im = q[2 * (f + (size_t)d * F) + 1] * w;
                    out[2 * (i + (size_t)d * M)] += dl_re * ps_re - dl_im * ps_im - (g_re * qs_re - g_im * qs_im);
                    out[2 * (i + (size_t)d * M) + 1] += dl_re * ps_im + dl_im * ps_re - (g_re * qs_im + g_im * qs_re);
                }
            }
        }
    }
    mesh_free(&m);
    return BO_OK;
}

/* Far-field pattern p_inf(d) = lim_{r->inf} r exp(-i k r) p(r d) of the field
 * representation above (no counterpart in the reference; it is the r -> inf
 * limit of BeatEngineCpuField.jl:23-44 with the same signed k):
 *   p_inf(d) = sum_src exp(-i k d.y)/(4 pi) * [(-i k)(d.n) p_src - q_src]. */
int bo_farfield(int V, const double *verts, int F, const int *faces, int quad_order, double k,
                int M, const double *dirs, int R, const double *p, const double *q, double *out, int nthreads)
{
    bo_mesh m;
    int st = mesh_init(&m, V, verts, F, faces, quad_order);
    if (st != BO_OK) { mesh_free(&m); return st; }
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
    int N = V, Q = m.Q;
#pragma omp parallel for schedule(dynamic, 4)
    for (int i = 0; i < M; ++i) {
        v3 dv = v3make(dirs + 3 * i);
        double dn = v3norm(dv);
        v3 d = {dv.x / dn, dv.y / dn, dv.z / dn};
        for (int c = 0; c < R; ++c) { out[2 * (i + (size_t)c * M)] = 0.0; out[2 * (i + (size_t)c * M) + 1] = 0.0; }
        for (int f = 0; f < F; ++f) {
            const int *fc = faces + 3 * f;
            v3 n = v3make(m.normals + 3 * f);
            double jac = 2.0 * m.areas[f];
            double dnrm = v3dot(d, n);
            for (int qq = 0; qq < Q; ++qq) {
                v3 y = v3make(m.qpts + 3 * (f * Q + qq));
                double ph_ = -k * v3dot(d, y);
                double e_re = cos(ph_) / (4.0 * BO_PI), e_im = sin(ph_) / (4.0 * BO_PI);
                /* a = e * (-i k dn) */
                double a_re = e_im * k * dnrm, a_im = -e_re * k * dnrm;
                double w = m.rw[qq] * jac;
                const double *ph = m.basis + 3 * qq;
                for (int c = 0; c < R; ++c) {
                    const double *pd = p + 2 * (size_t)c * N;
                    double ps_re = (ph[0] * pd[2 * fc[0]] + ph[1] * pd[2 * fc[1]] + ph[2] * pd[2 * fc[2]]) * w;
                    double ps_im = (ph[0] * pd[2 * fc[0] + 1] + ph[1] * pd[2 * fc[1] + 1] + ph[2] * pd[2 * fc[2] + 1]) * w;
                    double qs_re = q[2 * (f + (size_t)c * F)] * w, qs_im = q[2 * (f + (size_t)c * F) + 1] * w;
                    out[2 * (i + (size_t)c * M)] += a_re * ps_re - a_im * ps_im - (e_re * qs_re - e_im * qs_im);
                    out[2 * (i + (size_t)c * M) + 1] += a_re * ps_im + a_im * ps_re - (e_re * qs_im + e_im * qs_re);
                }
            }
        }
    }
    mesh_free(&m);
    return BO_OK;
}

/* ------------------------------------------------------------------------ */
/* symmetry images (symmetry_transforms, BeatEngineCore.jl:463-482;          */
/* reflect_point / reflect_normal / reflect_curl, :487-496; plane snapping   */
/* and orbit weights, :504-582; image passes and image-singular deltas,      */
/* BeatEngineCudaBurtonMiller.jl:475-493 and BeatEngineCudaSingular.jl:140-  */
/* 278, 590-897).  Modes: 0 off, 1 x, 2 xy, 3 ground.                        */
/* ------------------------------------------------------------------------ */
typedef struct { double s[3]; double det; } bo_xf;

static int sym_images(int mode, bo_xf *out)
{
    int n = 0;
    if (mode == 1 || mode == 2) { out[n].s[0] = -1; out[n].s[1] = 1; out[n].s[2] = 1; out[n].det = -1; ++n; }
    if (mode == 2) {
        out[n].s[0] = 1; out[n].s[1] = -1; out[n].s[2] = 1; out[n].det = -1; ++n;
        out[n].s[0] = -1; out[n].s[1] = -1; out[n].s[2] = 1; out[n].det = 1; ++n;
    }
    if (mode == 3) { out[n].s[0] = 1; out[n].s[1] = -1; out[n].s[2] = 1; out[n].det = -1; ++n; }
    return n;
}

/* symmetry_plane_tolerance: max(1e-9, 1e-6 x bounding-box diagonal) */
static double sym_plane_tol(int V, const double *verts)
{
    double lo[3] = {verts[0], verts[1], verts[2]}, hi[3] = {verts[0], verts[1], verts[2]};
    for (int v = 1; v < V; ++v)
        for (int c = 0; c < 3; ++c) {
            if (verts[3 * v + c] < lo[c]) lo[c] = verts[3 * v + c];
            if (verts[3 * v + c] > hi[c]) hi[c] = verts[3 * v + c];
        }
    double d = sqrt((hi[0] - lo[0]) * (hi[0] - lo[0]) + (hi[1] - lo[1]) * (hi[1] - lo[1]) + (hi[2] - lo[2]) * (hi[2] - lo[2]));
    double t = d * 1e-6;
    return t > 1e-9 ? t : 1e-9;
}

static inline v3 reflect(const bo_xf *x, v3 p) { v3 r = {x->s[0] * p.x, x->s[1] * p.y, x->s[2] * p.z}; return r; }

/* regular pair with the trial element reflected by x (all pairs, touching or not) */
static void regular_pair_x(const bo_mesh *m, int t, int s, const bo_xf *x, double k, double eta, double *lhs, double *rhs)
{
    v3 nt = v3make(m->normals + 3 * t), ns = reflect(x, v3make(m->normals + 3 * s));
    double jac = 4.0 * m->areas[t] * m->areas[s];
    double k2n_im = eta * (k * k * v3dot(nt, ns));
    double curl[2] = {0.0, 0.0}, cs[9];
    for (int a = 0; a < 3; ++a)
        for (int c = 0; c < 3; ++c) cs[3 * a + c] = x->det * x->s[c] * m->curls[9 * s + 3 * a + c];
    memset(lhs, 0, sizeof(double) * 18); memset(rhs, 0, sizeof(double) * 6);
    int Q = m->Q;
    for (int a = 0; a < Q; ++a) {
        v3 xp = v3make(m->qpts + 3 * (t * Q + a));
        for (int b = 0; b < Q; ++b) {
            v3 y = reflect(x, v3make(m->qpts + 3 * (s * Q + b)));
            bm_point(xp, y, m->basis + 3 * a, m->basis + 3 * b, m->rw[a] * m->rw[b] * jac, nt, ns, k, eta, k2n_im,
                     lhs, rhs, curl);
        }
    }
    bm_finish(m->curls + 9 * t, cs, eta, curl, lhs);
}

/* geometric_adjacency_info, BeatEngineCore.jl:624-650, on vertex positions */
static int geometric_adjacency(const v3 *tv, const v3 *sv, double tol, int *ta, int *tb, int *sa, int *sb)
{
    int sh_a[3], sh_b[3], n = 0;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            if (v3norm(v3sub(tv[i], sv[j])) <= tol && n < 3) { sh_a[n] = i + 1; sh_b[n] = j + 1; ++n; }
    *ta = *tb = *sa = *sb = 0;
    if (n == 3) return BO_COINCIDENT;
    if (n == 2) {
        if (sh_b[1] < sh_b[0]) {
            int t = sh_a[0]; sh_a[0] = sh_a[1]; sh_a[1] = t;
            t = sh_b[0]; sh_b[0] = sh_b[1]; sh_b[1] = t;
        }
        *ta = sh_a[0]; *tb = sh_a[1]; *sa = sh_b[0]; *sb = sh_b[1];
        return BO_EDGE;
    }
    if (n == 1) { *ta = sh_a[0]; *sa = sh_b[0]; return BO_VERTEX; }
    return 0;
}

/* image-singular delta of a touching (test, reflected trial) pair: the
 * remapped Duffy integral minus the regular-rule integral the image pass
 * already added (_cuda_image_singular_delta_blocks_kernel!) */
static void image_delta_pair(const bo_mesh *m, int t, int s, const bo_xf *x, int kind, int ta, int tb, int sa, int sb,
                             int sing_order, double k, double eta, double *lhs, double *rhs)
{
    int nb = sing_order * sing_order * sing_order * sing_order * 6;
    double *bt = malloc(sizeof(double) * 2 * nb), *bs = malloc(sizeof(double) * 2 * nb), *bw = malloc(sizeof(double) * nb);
    int nq = bo_duffy_rule(sing_order, kind, bt, bs, bw);
    const int *ft = m->faces + 3 * t, *fs = m->faces + 3 * s;
    v3 tv[3], sv[3];
    for (int a = 0; a < 3; ++a) { tv[a] = v3make(m->verts + 3 * ft[a]); sv[a] = reflect(x, v3make(m->verts + 3 * fs[a])); }
    v3 nt = v3make(m->normals + 3 * t), ns = reflect(x, v3make(m->normals + 3 * s));
    double jac = (2.0 * m->areas[t]) * (2.0 * m->areas[s]);
    double k2n_im = eta * (k * k * v3dot(nt, ns));
    double curl[2] = {0.0, 0.0}, cs[9];
    for (int a = 0; a < 3; ++a)
        for (int c = 0; c < 3; ++c) cs[3 * a + c] = x->det * x->s[c] * m->curls[9 * s + 3 * a + c];
    memset(lhs, 0, sizeof(double) * 18); memset(rhs, 0, sizeof(double) * 6);
    for (int q = 0; q < nq; ++q) {
        double pt[2], ps[2];
        remap_point(kind, ta, tb, bt + 2 * q, pt);
        remap_point(kind, sa, sb, bs + 2 * q, ps);
        double b1[3] = {1.0 - pt[0] - pt[1], pt[0], pt[1]}, b2[3] = {1.0 - ps[0] - ps[1], ps[0], ps[1]};
        v3 xp = {b1[0] * tv[0].x + b1[1] * tv[1].x + b1[2] * tv[2].x, b1[0] * tv[0].y + b1[1] * tv[1].y + b1[2] * tv[2].y,
                 b1[0] * tv[0].z + b1[1] * tv[1].z + b1[2] * tv[2].z};
        v3 y = {b2[0] * sv[0].x + b2[1] * sv[1].x + b2[2] * sv[2].x, b2[0] * sv[0].y + b2[1] * sv[1].y + b2[2] * sv[2].y,
                b2[0] * sv[0].z + b2[1] * sv[1].z + b2[2] * sv[2].z};
        bm_point(xp, y, b1, b2, bw[q] * jac, nt, ns, k, eta, k2n_im, lhs, rhs, curl);
    }
    bm_finish(m->curls + 9 * t, cs, eta, curl, lhs);
    double rl[18], rr[6];
    regular_pair_x(m, t, s, x, k, eta, rl, rr);
    for (int i = 0; i < 18; ++i) lhs[i] -= rl[i];
    for (int i = 0; i < 6; ++i) rhs[i] -= rr[i];
    free(bt); free(bs); free(bw);
}

/* Snap vertices within the plane tolerance onto the active symmetry planes
 * (snap_symmetry_plane_vertices); returns BO_EINVAL when a vertex lies on the
 * negative side (validate_symmetry_fundamental_domain!). */
int bo_symmetry_snap(int V, double *verts, int mode)
{
    double tol = sym_plane_tol(V, verts);
    int axes[2], na = 0;
    if (mode == 1 || mode == 2) axes[na++] = 0;
    if (mode == 2) axes[na++] = 1;
    for (int v = 0; v < V; ++v)
        for (int i = 0; i < na; ++i) {
            double *c = verts + 3 * v + axes[i];
            if (*c < -tol) return BO_EINVAL;
            if (fabs(*c) <= tol) *c = 0.0;
        }
    return BO_OK;
}

/* The system with symmetry images: the one-copy assembly, one reflected-trial
 * pass per image, the image-singular deltas, then the orbit row weights
 * (2 per active plane a row's vertex lies on; p1_symmetry_orbit_weights).
 * verts must already be snapped (bo_symmetry_snap). */
int bo_assemble_sym(int V, const double *verts, int F, const int *faces, int quad_order, int sing_order, double k,
                    double eta, int R, const double *q, double *A, double *b, int nthreads, int mode)
{
    int st = bo_assemble_range(V, verts, F, faces, quad_order, sing_order, k, eta, R, q, A, b, nthreads, 0, 0, F);
    if (st != BO_OK || mode == 0) return st;
    bo_mesh m;
    st = mesh_init(&m, V, verts, F, faces, quad_order);
    if (st != BO_OK) { mesh_free(&m); return st; }
    bo_xf xf[4];
    int nimg = sym_images(mode, xf);
    int *order = malloc(sizeof(int) * F), *start = malloc(sizeof(int) * 65);
    int ncol = colour_groups(&m, order, start);
    const double tol_pair = 1e-8;
    for (int ix = 0; ix < nimg; ++ix) {
        for (int c = 0; c < ncol; ++c) {
#pragma omp parallel for schedule(dynamic, 1)
            for (int i = start[c]; i < start[c + 1]; ++i) {
                int t = order[i];
                double lhs[18], rhs[6];
                v3 tv[3];
                for (int a = 0; a < 3; ++a) tv[a] = v3make(verts + 3 * faces[3 * t + a]);
                for (int s = 0; s < F; ++s) {
                    regular_pair_x(&m, t, s, &xf[ix], k, eta, lhs, rhs);
                    scatter(&m, t, s, lhs, rhs, R, q, A, b);
                    v3 sv[3];
                    for (int a = 0; a < 3; ++a) sv[a] = reflect(&xf[ix], v3make(verts + 3 * faces[3 * s + a]));
                    int ta, tb, sa, sb;
                    int kind = geometric_adjacency(tv, sv, tol_pair, &ta, &tb, &sa, &sb);
                    if (kind == 0) continue;
                    image_delta_pair(&m, t, s, &xf[ix], kind, ta, tb, sa, sb, sing_order, k, eta, lhs, rhs);
                    scatter(&m, t, s, lhs, rhs, R, q, A, b);
                }
            }
        }
    }
    free(order); free(start);
    double tol = sym_plane_tol(V, verts);
    int N = V;
    for (int v = 0; v < V; ++v) {
        double w = 1.0;
        if ((mode == 1 || mode == 2) && fabs(verts[3 * v]) <= tol) w *= 2.0;
        if (mode == 2 && fabs(verts[3 * v + 1]) <= tol) w *= 2.0;
        if (w == 1.0) continue;
        for (int c = 0; c < N; ++c) { A[2 * (v + (size_t)c * N)] *= w; A[2 * (v + (size_t)c * N) + 1] *= w; }
        for (int d = 0; d < R; ++d) { b[2 * (v + (size_t)d * N)] *= w; b[2 * (v + (size_t)d * N) + 1] *= w; }
    }
    mesh_free(&m);
    return BO_OK;
}

/* Field and far field with the image sources (reflected positions and
 * normals, the same p and q). */
int bo_field_sym(int V, const double *verts, int F, const int *faces, int quad_order, double k, int M,
                 const double *points, int R, const double *p, const double *q, double *out, int nthreads, int mode,
                 int far)
{
    bo_mesh m;
    int st = mesh_init(&m, V, verts, F, faces, quad_order);
    if (st != BO_OK) { mesh_free(&m); return st; }
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
    bo_xf xf[5];
    xf[0].s[0] = xf[0].s[1] = xf[0].s[2] = 1.0; xf[0].det = 1.0;
    int nx = 1 + sym_images(mode, xf + 1);
    int N = V, Q = m.Q;
#pragma omp parallel for schedule(dynamic, 4)
    for (int i = 0; i < M; ++i) {
        v3 xo = v3make(points + 3 * i);
        if (far) { double nn = v3norm(xo); xo.x /= nn; xo.y /= nn; xo.z /= nn; }
        for (int d = 0; d < R; ++d) { out[2 * (i + (size_t)d * M)] = 0.0; out[2 * (i + (size_t)d * M) + 1] = 0.0; }
        for (int ix = 0; ix < nx; ++ix)
            for (int f = 0; f < F; ++f) {
                const int *fc = faces + 3 * f;
                v3 n = reflect(&xf[ix], v3make(m.normals + 3 * f));
                double jac = 2.0 * m.areas[f];
                for (int qq = 0; qq < Q; ++qq) {
                    v3 y = reflect(&xf[ix], v3make(m.qpts + 3 * (f * Q + qq)));
                    double g_re, g_im, dl_re, dl_im;
                    if (far) {
                        double ph_ = -k * v3dot(xo, y);
                        g_re = cos(ph_) / (4.0 * BO_PI); g_im = sin(ph_) / (4.0 * BO_PI);
                        double dnrm = v3dot(xo, n);
                        dl_re = g_im * k * dnrm; dl_im = -g_re * k * dnrm;
                    } else {
                        v3 r = v3sub(y, xo);
                        double radius = v3norm(r);
                        if (radius == 0.0) continue;
                        double phase = k * radius, gsc = 1.0 / (4.0 * BO_PI * radius);
                        g_re = cos(phase) * gsc; g_im = sin(phase) * gsc;
                        double proj = v3dot(r, n) / radius, fr = -1.0 / radius, fi = k;
                        dl_re = (g_re * fr - g_im * fi) * proj; dl_im = (g_re * fi + g_im * fr) * proj;
                    }
                    double w = m.rw[qq] * jac;
                    const double *ph = m.basis + 3 * qq;
                    for (int d = 0; d < R; ++d) {
                        const double *pd = p + 2 * (size_t)d * N;
                        double ps_re = (ph[0] * pd[2 * fc[0]] + ph[1] * pd[2 * fc[1]] + ph[2] * pd[2 * fc[2]]) * w;
                        double ps_im = (ph[0] * pd[2 * fc[0] + 1] + ph[1] * pd[2 * fc[1] + 1] + ph[2] * pd[2 * fc[2] + 1]) * w;
                        double qs_re = q[2 * (f + (size_t)d * F)] * w, qs_im = q[2 * (f + (size_t)d * F) + 1] * w;
                        out[2 * (i + (size_t)d * M)] += dl_re * ps_re - dl_im * ps_im - (g_re * qs_re - g_im * qs_im);
                        out[2 * (i + (size_t)d * M) + 1] += dl_re * ps_im + dl_im * ps_re - (g_re * qs_im + g_im * qs_re);
                    }
                }
            }
    }
    mesh_free(&m);
    return BO_OK;
}

/* ------------------------------------------------------------------------ */
/* pressure and its gradient at observation points (pressure_gradient_v1):   */
/* field_value_gradient, _gradient_triangle, _adaptive_gradient_triangle,    */
/* correct_field_gradient!, evaluate_galerkin_field_gradient_cpu,            */
/* BeatEngineFieldGradient.jl:1-88.  out is M x 4 x R complex, column-major: */
/* (value, d/dx, d/dy, d/dz) of column r at out[i + M (d + 4 r)].            */
/* ------------------------------------------------------------------------ */
static void fvg(v3 x, v3 y, v3 n, const double *p, const double *q, int R, double k, double w, double *acc)
{
    v3 r = v3sub(y, x);
    double rad = v3norm(r);
    if (rad == 0.0) return;
    v3 u = {r.x / rad, r.y / rad, r.z / rad};
    double gsc = w / (4.0 * BO_PI * rad);
    double g_re = cos(k * rad) * gsc, g_im = sin(k * rad) * gsc;
    double a_re = -1.0 / rad, a_im = k;
    double b_re = 3.0 / (rad * rad) - k * k, b_im = -3.0 * k / rad;
    double proj = v3dot(u, n);
    double ua[3] = {u.x, u.y, u.z}, na[3] = {n.x, n.y, n.z};
    for (int c = 0; c < R; ++c) {
        double pr = p[2 * c], pi = p[2 * c + 1], qr = q[2 * c], qi = q[2 * c + 1];
        /* value = G (a proj p - q) */
        double t_re = (a_re * pr - a_im * pi) * proj - qr, t_im = (a_re * pi + a_im * pr) * proj - qi;
        acc[8 * c] += g_re * t_re - g_im * t_im;
        acc[8 * c + 1] += g_re * t_im + g_im * t_re;
        /* gradient = G (a q u - p (b proj u + (a / r) n)) */
        double aq_re = a_re * qr - a_im * qi, aq_im = a_re * qi + a_im * qr;
        double bp_re = (b_re * pr - b_im * pi) * proj, bp_im = (b_re * pi + b_im * pr) * proj;
        double ap_re = (a_re * pr - a_im * pi) / rad, ap_im = (a_re * pi + a_im * pr) / rad;
        for (int d = 0; d < 3; ++d) {
            double v_re = aq_re * ua[d] - (bp_re * ua[d] + ap_re * na[d]);
            double v_im = aq_im * ua[d] - (bp_im * ua[d] + ap_im * na[d]);
            acc[8 * c + 2 + 2 * d] += g_re * v_re - g_im * v_im;
            acc[8 * c + 3 + 2 * d] += g_re * v_im + g_im * v_re;
        }
    }
}

/* one triangle with the rule (rpts, rw, nq); pv: 3 x R complex vertex values */
static void grad_triangle(v3 x, const v3 *v, v3 n, const double *pv, const double *q, int R, double k,
                          const double *rpts, const double *rw, int nq, double *acc)
{
    double jac = v3norm(v3cross(v3sub(v[1], v[0]), v3sub(v[2], v[0])));
    double *ps = malloc(sizeof(double) * 2 * R);
    for (int j = 0; j < nq; ++j) {
        double xi = rpts[2 * j], et = rpts[2 * j + 1], b[3] = {1.0 - xi - et, xi, et};
        v3 y = {b[0] * v[0].x + b[1] * v[1].x + b[2] * v[2].x, b[0] * v[0].y + b[1] * v[1].y + b[2] * v[2].y,
                b[0] * v[0].z + b[1] * v[1].z + b[2] * v[2].z};
        for (int c = 0; c < R; ++c) {
            ps[2 * c] = b[0] * pv[2 * c] + b[1] * pv[2 * (R + c)] + b[2] * pv[2 * (2 * R + c)];
            ps[2 * c + 1] = b[0] * pv[2 * c + 1] + b[1] * pv[2 * (R + c) + 1] + b[2] * pv[2 * (2 * R + c) + 1];
        }
        fvg(x, y, n, ps, q, R, k, jac * rw[j], acc);
    }
    free(ps);
}

static int grad_adaptive(v3 x, const v3 *v, v3 n, const double *pv, const double *q, int R, double k,
                         const double *rpts, const double *rw, int nq, int depth, double *acc)
{
    v3 c = {(v[0].x + v[1].x + v[2].x) / 3, (v[0].y + v[1].y + v[2].y) / 3, (v[0].z + v[1].z + v[2].z) / 3};
    double d01 = v3norm(v3sub(v[0], v[1])), d12 = v3norm(v3sub(v[1], v[2])), d20 = v3norm(v3sub(v[2], v[0]));
    double diam = d01 > d12 ? (d01 > d20 ? d01 : d20) : (d12 > d20 ? d12 : d20);
    double dist = v3norm(v3sub(x, c));
    if (diam <= 0.4 * dist && fabs(k) * diam <= 0.7) {
        grad_triangle(x, v, n, pv, q, R, k, rpts, rw, nq, acc);
        return BO_OK;
    }
    if (depth >= 12) return BO_ETOOCLOSE;
    v3 ab = {(v[0].x + v[1].x) / 2, (v[0].y + v[1].y) / 2, (v[0].z + v[1].z) / 2};
    v3 bc = {(v[1].x + v[2].x) / 2, (v[1].y + v[2].y) / 2, (v[1].z + v[2].z) / 2};
    v3 ca = {(v[2].x + v[0].x) / 2, (v[2].y + v[0].y) / 2, (v[2].z + v[0].z) / 2};
    double *mid = malloc(sizeof(double) * 6 * R), *sub = malloc(sizeof(double) * 6 * R);
    /* midpoint values pab, pbc, pca */
    for (int c2 = 0; c2 < 2 * R; ++c2) {
        mid[c2] = (pv[c2] + pv[2 * R + c2]) / 2;              /* ab */
        mid[2 * R + c2] = (pv[2 * R + c2] + pv[4 * R + c2]) / 2;  /* bc */
        mid[4 * R + c2] = (pv[4 * R + c2] + pv[c2]) / 2;      /* ca */
    }
    const v3 tri[4][3] = {{v[0], ab, ca}, {ab, v[1], bc}, {ca, bc, v[2]}, {ab, bc, ca}};
    const double *src[4][3] = {{pv, mid, mid + 4 * R}, {mid, pv + 2 * R, mid + 2 * R},
                               {mid + 4 * R, mid + 2 * R, pv + 4 * R}, {mid, mid + 2 * R, mid + 4 * R}};
    int st = BO_OK;
    for (int t = 0; t < 4 && st == BO_OK; ++t) {
        for (int a = 0; a < 3; ++a) memcpy(sub + 2 * R * a, src[t][a], sizeof(double) * 2 * R);
        st = grad_adaptive(x, tri[t], n, sub, q, R, k, rpts, rw, nq, depth + 1, acc);
    }
    free(mid); free(sub);
    return st;
}

int bo_field_gradient(int V, const double *verts, int F, const int *faces, int quad_order, double k, int M,
                      const double *points, int R, const double *p, const double *q, double *out, int nthreads,
                      int mode)
{
    bo_mesh m;
    int st = mesh_init(&m, V, verts, F, faces, quad_order);
    if (st != BO_OK) { mesh_free(&m); return st; }
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
    bo_xf xf[5];
    xf[0].s[0] = xf[0].s[1] = xf[0].s[2] = 1.0; xf[0].det = 1.0;
    int nx = 1 + sym_images(mode, xf + 1);
    double fine_pts[2 * BO_MAXQ], fine_w[BO_MAXQ];
    int nfine = bo_triangle_rule(4, fine_pts, fine_w);
    int N = V, Q = m.Q, status = BO_OK;
#pragma omp parallel for schedule(dynamic, 1)
    for (int i = 0; i < M; ++i) {
        v3 x = v3make(points + 3 * i);
        double *acc = calloc(8 * (size_t)R, sizeof(double));
        double *pv = malloc(sizeof(double) * 6 * R), *qf = malloc(sizeof(double) * 2 * R);
        for (int ix = 0; ix < nx; ++ix)
            for (int f = 0; f < F; ++f) {
                const int *fc = faces + 3 * f;
                v3 v[3];
                for (int a = 0; a < 3; ++a) v[a] = reflect(&xf[ix], v3make(verts + 3 * fc[a]));
                v3 n = reflect(&xf[ix], v3make(m.normals + 3 * f));
                for (int a = 0; a < 3; ++a)
                    for (int c = 0; c < R; ++c) {
                        pv[2 * (a * R + c)] = p[2 * (fc[a] + (size_t)c * N)];
                        pv[2 * (a * R + c) + 1] = p[2 * (fc[a] + (size_t)c * N) + 1];
                    }
                for (int c = 0; c < R; ++c) { qf[2 * c] = q[2 * (f + (size_t)c * F)]; qf[2 * c + 1] = q[2 * (f + (size_t)c * F) + 1]; }
                /* regular sum (evaluate_galerkin_field_gradient_cpu) */
                grad_triangle(x, v, n, pv, qf, R, k, m.rpts, m.rw, Q, acc);
                /* near-panel correction: adaptive - regular (correct_field_gradient!) */
                v3 cen = {(v[0].x + v[1].x + v[2].x) / 3, (v[0].y + v[1].y + v[2].y) / 3, (v[0].z + v[1].z + v[2].z) / 3};
                double d01 = v3norm(v3sub(v[0], v[1])), d12 = v3norm(v3sub(v[1], v[2])), d20 = v3norm(v3sub(v[2], v[0]));
                double diam = d01 > d12 ? (d01 > d20 ? d01 : d20) : (d12 > d20 ? d12 : d20);
                if (v3norm(v3sub(x, cen)) > 3.0 * diam) continue;
                double *fine = calloc(8 * (size_t)R, sizeof(double)), *coarse = calloc(8 * (size_t)R, sizeof(double));
                int s2 = grad_adaptive(x, v, n, pv, qf, R, k, fine_pts, fine_w, nfine, 0, fine);
                if (s2 != BO_OK) {
#pragma omp critical
                    status = s2;
                }
                grad_triangle(x, v, n, pv, qf, R, k, m.rpts, m.rw, Q, coarse);
                for (size_t e = 0; e < 8 * (size_t)R; ++e) acc[e] += fine[e] - coarse[e];
                free(fine); free(coarse);
            }
        for (int c = 0; c < R; ++c)
            for (int d = 0; d < 4; ++d) {
                out[2 * (i + (size_t)M * (d + 4 * c))] = acc[8 * c + 2 * d];
                out[2 * (i + (size_t)M * (d + 4 * c)) + 1] = acc[8 * c + 2 * d + 1];
            }
        free(acc); free(pv); free(qf);
    }
    mesh_free(&m);
    return status;
}

int bo_version(void) { return 1; }
