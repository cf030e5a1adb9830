/*
 * gvc_oracle.c -- CPU restatement of the reference algorithm for the Gaussian-mixture
 * volume path.  TEST INFRASTRUCTURE ONLY: imported by tests/, by the smoke check and
 * by bench.py's cpu_baseline / reference arm.  Never linked into the product library.
 *
 * Parity status:
 *   - The reference's CUDA extension cannot be built here (its BVH library cuBQL, its
 *     matrix library glm and its sampler library Viskores are not vendored), so the
 *     kernels' floating-point semantics are restated from source and are "parity
 *     unpinned" against the reference binary.  The Python-side orderings (21-bit
 *     Morton sort of Gaussians and samples) are pinned by fixtures generated from the
 *     reference's own Python source (tests/golden/make_golden.py).
 *   - Integer / ordering work (30-bit Morton keys, stable key sort, Karras hierarchy,
 *     min/max refit, tet location with the lowest-containing-cell tie-break) is a
 *     declared specification; the CUDA product must match it bit for bit.
 *
 * Every function cites the reference file:line it follows (paths inside the
 * reference project).  Compile with -ffp-contract=off so that the double-precision
 * predicates match the GPU's explicitly rounded arithmetic bit for bit.
 */
#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_WEIGHT_CUTOFF 1e-2  /* diff-gaussian-rasterization/cuda_rasterizer/config.h:9 */
#define ORC_POWER_FLOOR (-14.0) /* forward.cu:166, forward.cu:235, backward.cu:258 */
#define ORC_COND_FP64 1.0e2f    /* condition estimate above which the conic is inverted in FP64 */

static int orc_nthreads(int req) {
#ifdef _OPENMP
    if (req > 0) return req;
    return omp_get_max_threads();
#else
    (void)req;
    return 1;
#endif
}

int orc_openmp_enabled(void) {
#ifdef _OPENMP
    return 1;
#else
    return 0;
#endif
}

/* ------------------------------------------------------------------------------------
 * Preprocess: covariance -> conic and the per-Gaussian AABB.
 * Follows diff-gaussian-rasterization/cuda_rasterizer/forward.cu:23-113.
 *   R is built from the raw quaternion (r,x,y,z) = rot[0..3] without normalisation
 *   (forward.cu:33-44).  glm's 9-scalar constructor fills columns, so the glm matrix
 *   is the transpose of the textbook rotation R_std; Sigma = (S Rg)^T (S Rg) =
 *   R_std S^2 R_std^T.  The AABB corners walk the glm COLUMNS R[k], i.e. the rows of
 *   R_std (the reference's transposed-box quirk, forward.cu:91-112), scaled by
 *   m = sqrt(-2 ln(1e-3 / w)) (forward.cu:79).  min/max follow CUDA fminf/fmaxf,
 *   which ignore a NaN operand: for w < 1e-3 the box collapses to the mean.
 * ------------------------------------------------------------------------------------ */
static void rot_glm_cols(const float q[4], float Rc[3][3]) {
    /* Rc[col][row], same expression order as forward.cu:40-44 */
    float r = q[0], x = q[1], y = q[2], z = q[3];
    Rc[0][0] = 1.f - 2.f * (y * y + z * z);
    Rc[0][1] = 2.f * (x * y - r * z);
    Rc[0][2] = 2.f * (x * z + r * y);
    Rc[1][0] = 2.f * (x * y + r * z);
    Rc[1][1] = 1.f - 2.f * (x * x + z * z);
    Rc[1][2] = 2.f * (y * z - r * x);
    Rc[2][0] = 2.f * (x * z - r * y);
    Rc[2][1] = 2.f * (y * z + r * x);
    Rc[2][2] = 1.f - 2.f * (x * x + y * y);
}

static float fminf_nan(float a, float b) { return fminf(a, b); }
static float fmaxf_nan(float a, float b) { return fmaxf(a, b); }

/* AABB of one Gaussian, float arithmetic in the reference's expression order. */
static void aabb_one(const float mu[3], const float s[3], const float q[4], float w, float sm,
                     float lo[3], float hi[3]) {
    float Rc[3][3];
    rot_glm_cols(q, Rc);
    float S0 = sm * s[0], S1 = sm * s[1], S2 = sm * s[2];
    /* forward.cu:79: (0.1 * WEIGHT_CUTOFF) is a double and the quotient is rounded to
       float as in the reference; the logarithm and square root are evaluated in double
       and rounded once (declared: reproducible on CPU and GPU, within 1 ulp of logf) */
    float arg = (float)((0.1 * ORC_WEIGHT_CUTOFF) / (double)w);
    float m = (float)sqrt(-2.0 * log((double)arg));
    float ss0 = S0 * m, ss1 = S1 * m, ss2 = S2 * m;
    const float n[2] = {-1.0f, 1.0f};
    for (int a = 0; a < 3; a++) { lo[a] = mu[a]; hi[a] = mu[a]; }
    for (int i = 0; i < 2; i++)
        for (int j = 0; j < 2; j++)
            for (int k = 0; k < 2; k++) {
                for (int a = 0; a < 3; a++) {
                    float t0 = n[i] * Rc[0][a];
                    t0 = t0 * ss0;
                    float t1 = n[j] * Rc[1][a];
                    t1 = t1 * ss1;
                    float t2 = n[k] * Rc[2][a];
                    t2 = t2 * ss2;
                    float c = mu[a] + t0;
                    c = c + t1;
                    c = c + t2;
                    lo[a] = fminf_nan(lo[a], c);
                    hi[a] = fmaxf_nan(hi[a], c);
                }
            }
}

/* Sigma in double from float scales / raw quaternion (forward.cu:27-49). */
static void sigma_f64(const float s_in[3], const float q_in[4], float sm, double Sg[3][3]) {
    double r = q_in[0], x = q_in[1], y = q_in[2], z = q_in[3];
    double Rg[3][3]; /* Rg[i][j] = row i col j of the glm matrix = R_std[j][i] */
    double Rs[3][3] = {
        {1.0 - 2.0 * (y * y + z * z), 2.0 * (x * y - r * z), 2.0 * (x * z + r * y)},
        {2.0 * (x * y + r * z), 1.0 - 2.0 * (x * x + z * z), 2.0 * (y * z - r * x)},
        {2.0 * (x * z - r * y), 2.0 * (y * z + r * x), 1.0 - 2.0 * (x * x + y * y)}};
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) Rg[i][j] = Rs[j][i];
    double sv[3] = {(double)(sm * s_in[0]), (double)(sm * s_in[1]), (double)(sm * s_in[2])};
    /* M = diag(s) Rg ; Sigma = M^T M */
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            double acc = 0.0;
            for (int k = 0; k < 3; k++) acc += (sv[k] * Rg[k][i]) * (sv[k] * Rg[k][j]);
            Sg[i][j] = acc;
        }
}

/* conic = adj(Sigma + eps I) / det, eps = 1e-5 max|diag| (forward.cu:52-76), in double. */
static void conic_from_sigma_f64(const double Sg[3][3], double c[6]) {
    double eps = fmax(fmax(fabs(Sg[0][0]), fabs(Sg[1][1])), fabs(Sg[2][2])) * 1e-5;
    double a = Sg[0][0] + eps, b = Sg[0][1], cc = Sg[0][2];
    double d = Sg[1][1] + eps, e = Sg[1][2], f = Sg[2][2] + eps;
    double det = a * (d * f - e * e) - b * (b * f - cc * e) + cc * (b * e - cc * d);
    double inv = 1.0 / det;
    c[0] = (d * f - e * e) * inv;
    c[1] = (cc * e - b * f) * inv;
    c[2] = (b * e - cc * d) * inv;
    c[3] = (a * f - cc * cc) * inv;
    c[4] = (b * cc - a * e) * inv;
    c[5] = (a * d - b * b) * inv;
}

/* Float conic in the reference's float arithmetic (forward.cu:46-76). */
static void conic_f32(const float s_in[3], const float q_in[4], float sm, float c[6]) {
    float Rc[3][3];
    rot_glm_cols(q_in, Rc);
    float sv[3] = {sm * s_in[0], sm * s_in[1], sm * s_in[2]};
    /* M[col][row] = sv[row] * Rc[col][row]; Sigma[col][row] = sum_k M[col][k] M[row][k] */
    float M[3][3];
    for (int cidx = 0; cidx < 3; cidx++)
        for (int r = 0; r < 3; r++) M[cidx][r] = sv[r] * Rc[cidx][r];
    float Sg[3][3];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            float acc = M[i][0] * M[j][0];
            acc = acc + M[i][1] * M[j][1];
            acc = acc + M[i][2] * M[j][2];
            Sg[i][j] = acc;
        }
    float eps = (float)((double)fmaxf(fmaxf(fabsf(Sg[0][0]), fabsf(Sg[1][1])), fabsf(Sg[2][2])) * 1e-5);
    float a = Sg[0][0] + eps, b = Sg[0][1], cc = Sg[0][2];
    float d = Sg[1][1] + eps, e = Sg[1][2], f = Sg[2][2] + eps;
    float det = a * (d * f - e * e) - b * (b * f - cc * e) + cc * (b * e - cc * d);
    float inv = (float)(1.0 / (double)det);
    c[0] = (d * f - e * e) * inv;
    c[1] = (cc * e - b * f) * inv;
    c[2] = (b * e - cc * d) * inv;
    c[3] = (a * f - cc * cc) * inv;
    c[4] = (b * cc - a * e) * inv;
    c[5] = (a * d - b * b) * inv;
    /* Frobenius condition estimate ||Sigma'||_F ||conic||_F; above ORC_COND_FP64 the
       inverse is recomputed in double and rounded once (declared; the reference always
       inverts in float) */
    float nS = a * a;
    nS = nS + d * d;
    nS = nS + f * f;
    float oS = b * b;
    oS = oS + cc * cc;
    oS = oS + e * e;
    nS = nS + 2.f * oS;
    float nC = c[0] * c[0];
    nC = nC + c[3] * c[3];
    nC = nC + c[5] * c[5];
    float oC = c[1] * c[1];
    oC = oC + c[2] * c[2];
    oC = oC + c[4] * c[4];
    nC = nC + 2.f * oC;
    float cond2 = nS * nC;
    if (cond2 <= ORC_COND_FP64 * ORC_COND_FP64) return;
    double Sd[3][3], cd[6];
    sigma_f64(s_in, q_in, sm, Sd);
    conic_from_sigma_f64(Sd, cd);
    for (int k = 0; k < 6; k++) c[k] = (float)cd[k];
}


/* means/scales/rots/weights as the reference's tensors: [P,3],[P,3],[P,4],[P].
   conics64 may be NULL; conics32 may be NULL. aabbs: [P,6] = lo xyz, hi xyz. */
void orc_preprocess(int64_t P, const float* means, const float* scales, const float* rots,
                    const float* weights, float sm, float* conics32, double* conics64,
                    float* aabbs, int nthreads) {
    int nt = orc_nthreads(nthreads);
#pragma omp parallel for num_threads(nt) schedule(static)
    for (int64_t i = 0; i < P; i++) {
        if (aabbs) aabb_one(means + 3 * i, scales + 3 * i, rots + 4 * i, weights[i], sm,
                            aabbs + 6 * i, aabbs + 6 * i + 3);
        if (conics32) conic_f32(scales + 3 * i, rots + 4 * i, sm, conics32 + 6 * i);
        if (conics64) {
            double Sg[3][3];
            sigma_f64(scales + 3 * i, rots + 4 * i, sm, Sg);
            conic_from_sigma_f64(Sg, conics64 + 6 * i);
        }
    }
}

/* ------------------------------------------------------------------------------------
 * Uniform-grid binning (oracle-side candidate search; the reference uses cuBQL box
 * queries, forward.cu:150,209 -- only the candidate SET matters for the result).
 * ------------------------------------------------------------------------------------ */
typedef struct {
    double lo[3], inv_h;
    int64_t n[3];
    int64_t* start; /* ncell+1 */
    int32_t* items;
} orc_grid;

static int64_t clampi(int64_t v, int64_t lo, int64_t hi) { return v < lo ? lo : (v > hi ? hi : v); }

static void grid_cell_range(const orc_grid* g, const float* lo, const float* hi, int64_t c0[3], int64_t c1[3]) {
    for (int a = 0; a < 3; a++) {
        double l = ((double)lo[a] - g->lo[a]) * g->inv_h;
        double h = ((double)hi[a] - g->lo[a]) * g->inv_h;
        if (!(l == l)) l = 0; /* NaN guard */
        if (!(h == h)) h = 0;
        c0[a] = clampi((int64_t)floor(l), 0, g->n[a] - 1);
        c1[a] = clampi((int64_t)floor(h), 0, g->n[a] - 1);
    }
}

/* boxes: [n,6] lo/hi.  Builds a CSR grid over [glo, ghi] with cell size >= h.
   n_a = floor((ghi_a - glo_a) / h) + 1 computed with the same expression as the
   lookups, so every point inside [glo, ghi] maps to a valid cell. */
static void grid_build(orc_grid* g, int64_t n, const float* boxes, const double glo[3], const double ghi[3],
                       double h, int nt) {
    double hmax = 0;
    for (int a = 0; a < 3; a++) hmax = fmax(hmax, (ghi[a] - glo[a]) / 1000.0);
    if (!(h > hmax)) h = hmax;
    if (!(h > 0)) h = 1.0;
    /* at most ~64 grid cells per item (degenerate boxes would otherwise ask for 1e9) */
    for (;;) {
        g->inv_h = 1.0 / h;
        for (int a = 0; a < 3; a++) {
            g->lo[a] = glo[a];
            g->n[a] = (int64_t)floor((ghi[a] - glo[a]) * g->inv_h) + 1;
            if (g->n[a] < 1) g->n[a] = 1;
        }
        if ((double)g->n[0] * (double)g->n[1] * (double)g->n[2] <= 64.0 * (double)n + 4096.0) break;
        h *= 1.5;
    }
    int64_t ncell = g->n[0] * g->n[1] * g->n[2];
    int64_t* cnt = (int64_t*)calloc((size_t)ncell + 1, sizeof(int64_t));
    for (int64_t i = 0; i < n; i++) {
        int64_t c0[3], c1[3];
        grid_cell_range(g, boxes + 6 * i, boxes + 6 * i + 3, c0, c1);
        for (int64_t z = c0[2]; z <= c1[2]; z++)
            for (int64_t y = c0[1]; y <= c1[1]; y++)
                for (int64_t x = c0[0]; x <= c1[0]; x++) cnt[(z * g->n[1] + y) * g->n[0] + x + 1]++;
    }
    for (int64_t c = 0; c < ncell; c++) cnt[c + 1] += cnt[c];
    g->start = cnt;
    g->items = (int32_t*)malloc(sizeof(int32_t) * (size_t)(cnt[ncell] > 0 ? cnt[ncell] : 1));
    int64_t* fill = (int64_t*)malloc(sizeof(int64_t) * (size_t)ncell);
    memcpy(fill, cnt, sizeof(int64_t) * (size_t)ncell);
    for (int64_t i = 0; i < n; i++) { /* insertion in index order -> lists sorted by id */
        int64_t c0[3], c1[3];
        grid_cell_range(g, boxes + 6 * i, boxes + 6 * i + 3, c0, c1);
        for (int64_t z = c0[2]; z <= c1[2]; z++)
            for (int64_t y = c0[1]; y <= c1[1]; y++)
                for (int64_t x = c0[0]; x <= c1[0]; x++) g->items[fill[(z * g->n[1] + y) * g->n[0] + x]++] = (int32_t)i;
    }
    free(fill);
    (void)nt;
}

/* cell of a point, or -1 when the point lies outside the grid */
static int64_t grid_cell_of_point(const orc_grid* g, const float* p) {
    int64_t ci[3];
    for (int a = 0; a < 3; a++) {
        double l = ((double)p[a] - g->lo[a]) * g->inv_h;
        if (!(l >= 0)) return -1;
        ci[a] = (int64_t)floor(l);
        if (ci[a] >= g->n[a]) return -1;
    }
    return (ci[2] * g->n[1] + ci[1]) * g->n[0] + ci[0];
}

static void grid_free(orc_grid* g) {
    free(g->start);
    free(g->items);
}

static void boxes_bounds(int64_t n, const float* boxes, double lo[3], double hi[3]) {
    for (int a = 0; a < 3; a++) { lo[a] = INFINITY; hi[a] = -INFINITY; }
    for (int64_t i = 0; i < n; i++)
        for (int a = 0; a < 3; a++) {
            double l = boxes[6 * i + a], h = boxes[6 * i + 3 + a];
            if (l < lo[a]) lo[a] = l;
            if (h > hi[a]) hi[a] = h;
        }
    for (int a = 0; a < 3; a++)
        if (!(lo[a] <= hi[a])) { lo[a] = 0; hi[a] = 1; }
}

static double median_extent(int64_t n, const float* boxes) {
    /* a cheap robust size estimate: mean extent over a strided subset */
    int64_t step = n > 4096 ? n / 4096 : 1, k = 0;
    double acc = 0;
    for (int64_t i = 0; i < n; i += step) {
        double e = 0;
        for (int a = 0; a < 3; a++) e = fmax(e, (double)boxes[6 * i + 3 + a] - boxes[6 * i + a]);
        if (e == e && e < 1e30) { acc += e; k++; }
    }
    return k ? acc / (double)k : 1.0;
}

static inline int in_box(const float* b, float x, float y, float z) {
    return b[0] <= x && x <= b[3] && b[1] <= y && y <= b[4] && b[2] <= z && z <= b[5];
}

/* Pair power in double, reference expression (forward.cu:224-234). */
static inline double pair_power(const double* c, double dx, double dy, double dz) {
    double qf = dx * (c[0] * dx + c[1] * dy + c[2] * dz) + dy * (c[1] * dx + c[3] * dy + c[4] * dz) +
                dz * (c[2] * dx + c[4] * dy + c[5] * dz);
    return -0.5 * qf;
}

/* ------------------------------------------------------------------------------------
 * Forward (formal spec of forward.cu:185-259 and forward.cu:116-182 + 261-274):
 *   candidates of sample x: Gaussians with x inside the closed AABB;
 *   contributing: -14 <= p <= 0; W = sum w e^p, V = sum w v e^p;
 *   out = V/W, outw = W if W > 0.01, else out = -1, outw = 0.
 * Pair math and accumulation in double (the FP64 oracle); d = x - mu in double.
 * counts (optional, int64[S]): number of contributing pairs per sample
 * (the reference's count_intersections, forward.cu:239).
 * ------------------------------------------------------------------------------------ */
void orc_forward(int64_t P, int64_t S, const float* means, const float* values, const float* weights,
                 const double* conics, const float* aabbs, const float* samples, double* out, double* outw,
                 int64_t* counts, int nthreads) {
    int nt = orc_nthreads(nthreads);
    if (P == 0) { /* rasterize_points.cu:51: P == 0 returns the zero-initialised outputs */
        for (int64_t s = 0; s < S; s++) { out[s] = 0; outw[s] = 0; if (counts) counts[s] = 0; }
        return;
    }
    double glo[3], ghi[3];
    boxes_bounds(P, aabbs, glo, ghi);
    double h = median_extent(P, aabbs);
    orc_grid g;
    grid_build(&g, P, aabbs, glo, ghi, h, nt);
#pragma omp parallel for num_threads(nt) schedule(dynamic, 256)
    for (int64_t s = 0; s < S; s++) {
        float x = samples[3 * s], y = samples[3 * s + 1], z = samples[3 * s + 2];
        double W = 0, V = 0;
        int64_t cnt = 0;
        const float* pp = samples + 3 * s;
        int64_t cell = grid_cell_of_point(&g, pp);
        if (cell >= 0) {
            for (int64_t k = g.start[cell]; k < g.start[cell + 1]; k++) {
                int32_t i = g.items[k];
                if (!in_box(aabbs + 6 * i, x, y, z)) continue;
                double dx = (double)x - means[3 * i], dy = (double)y - means[3 * i + 1], dz = (double)z - means[3 * i + 2];
                double p = pair_power(conics + 6 * i, dx, dy, dz);
                if (p < ORC_POWER_FLOOR || p > 0.0) continue;
                double wt = (double)weights[i] * exp(p);
                W += wt;
                V += wt * (double)values[i];
                cnt++;
            }
        }
        if (W <= ORC_WEIGHT_CUTOFF) { out[s] = -1.0; outw[s] = 0.0; }
        else { out[s] = V / W; outw[s] = W; }
        if (counts) counts[s] = cnt;
    }
    grid_free(&g);
}

/* Candidate and contributing pair counts (sample in AABB; and additionally in the
   power window), the pair-count definition used for the work-per-step figures. */
void orc_pair_counts(int64_t P, int64_t S, const float* means, const double* conics, const float* aabbs,
                     const float* samples, int64_t* n_cand, int64_t* n_contrib, int nthreads) {
    int nt = orc_nthreads(nthreads);
    *n_cand = 0;
    *n_contrib = 0;
    if (P == 0 || S == 0) return;
    double glo[3], ghi[3];
    boxes_bounds(P, aabbs, glo, ghi);
    orc_grid g;
    grid_build(&g, P, aabbs, glo, ghi, median_extent(P, aabbs), nt);
    int64_t tc = 0, tk = 0;
#pragma omp parallel for num_threads(nt) schedule(dynamic, 256) reduction(+ : tc, tk)
    for (int64_t s = 0; s < S; s++) {
        float x = samples[3 * s], y = samples[3 * s + 1], z = samples[3 * s + 2];
        int64_t cell = grid_cell_of_point(&g, samples + 3 * s);
        if (cell < 0) continue;
        for (int64_t k = g.start[cell]; k < g.start[cell + 1]; k++) {
            int32_t i = g.items[k];
            if (!in_box(aabbs + 6 * i, x, y, z)) continue;
            tc++;
            double p = pair_power(conics + 6 * i, (double)x - means[3 * i], (double)y - means[3 * i + 1],
                                  (double)z - means[3 * i + 2]);
            if (p < ORC_POWER_FLOOR || p > 0.0) continue;
            tk++;
        }
    }
    *n_cand = tc;
    *n_contrib = tk;
    grid_free(&g);
}

/* Contributing pair list (sample, gaussian) for W > 0.01 samples, up to cap entries.
   Returns the total number of pairs (may exceed cap). Used by the FP64 autograd/FD
   tests to freeze the candidate set. */
int64_t orc_pair_list(int64_t P, int64_t S, const float* means, const double* conics, const float* aabbs,
                      const float* samples, const double* outw, int64_t cap, int64_t* ps, int64_t* pg) {
    if (P == 0 || S == 0) return 0;
    double glo[3], ghi[3];
    boxes_bounds(P, aabbs, glo, ghi);
    orc_grid g;
    grid_build(&g, P, aabbs, glo, ghi, median_extent(P, aabbs), 1);
    int64_t n = 0;
    for (int64_t s = 0; s < S; s++) {
        if (outw && !(outw[s] > ORC_WEIGHT_CUTOFF)) continue;
        float x = samples[3 * s], y = samples[3 * s + 1], z = samples[3 * s + 2];
        int64_t cell = grid_cell_of_point(&g, samples + 3 * s);
        if (cell < 0) continue;
        for (int64_t k = g.start[cell]; k < g.start[cell + 1]; k++) {
            int32_t i = g.items[k];
            if (!in_box(aabbs + 6 * i, x, y, z)) continue;
            double p = pair_power(conics + 6 * i, (double)x - means[3 * i], (double)y - means[3 * i + 1],
                                  (double)z - means[3 * i + 2]);
            if (p < ORC_POWER_FLOOR || p > 0.0) continue;
            if (n < cap) { ps[n] = s; pg[n] = i; }
            n++;
        }
    }
    grid_free(&g);
    return n;
}

/* ------------------------------------------------------------------------------------
 * Backward per-pair adjoint, Gaussian-owned (backward.cu:252-298, the sample-BVH
 * variant's math; the Gaussian-BVH variant backward.cu:437-481 is the same formula).
 *   out/outw are the forward's saved outputs (float), gout/gw the incoming grads.
 *   Pairs with outw <= 0.01 are skipped (backward.cu:263).
 * Outputs (double): dmeans[3P], dvalues[P], dweights[P], dconics[6P] (unique-parameter
 * convention: the off-diagonal entries carry the factor 2, backward.cu:294-297).
 * ------------------------------------------------------------------------------------ */
void orc_backward(int64_t P, int64_t S, const float* means, const float* values, const float* weights,
                  const double* conics, const float* aabbs, const float* samples, const float* out_cells,
                  const float* out_weights, const float* gout, const float* gw, double* dmeans, double* dvalues,
                  double* dweights, double* dconics, int nthreads) {
    int nt = orc_nthreads(nthreads);
    memset(dmeans, 0, sizeof(double) * 3 * (size_t)P);
    memset(dvalues, 0, sizeof(double) * (size_t)P);
    memset(dweights, 0, sizeof(double) * (size_t)P);
    memset(dconics, 0, sizeof(double) * 6 * (size_t)P);
    if (P == 0 || S == 0) return;
    /* bin samples as degenerate boxes */
    float* sboxes = (float*)malloc(sizeof(float) * 6 * (size_t)S);
    for (int64_t s = 0; s < S; s++)
        for (int a = 0; a < 3; a++) sboxes[6 * s + a] = sboxes[6 * s + 3 + a] = samples[3 * s + a];
    double glo[3], ghi[3];
    boxes_bounds(S, sboxes, glo, ghi);
    double h = median_extent(P, aabbs) * 0.5;
    if (!(h > 0)) h = 1.0;
    orc_grid g;
    grid_build(&g, S, sboxes, glo, ghi, h, nt);
#pragma omp parallel for num_threads(nt) schedule(dynamic, 64)
    for (int64_t i = 0; i < P; i++) {
        const float* b = aabbs + 6 * i;
        int64_t c0[3], c1[3];
        grid_cell_range(&g, b, b + 3, c0, c1);
        /* skip Gaussians whose box misses the sample bounds entirely */
        int miss = 0;
        for (int a = 0; a < 3; a++)
            if (!((double)b[3 + a] >= glo[a] && (double)b[a] <= ghi[a])) miss = 1;
        if (miss) continue;
        const double* c = conics + 6 * i;
        double mx = means[3 * i], my = means[3 * i + 1], mz = means[3 * i + 2];
        double w = weights[i], v = values[i];
        double a_v = 0, a_w = 0, a_mx = 0, a_my = 0, a_mz = 0, a_c[6] = {0, 0, 0, 0, 0, 0};
        for (int64_t z = c0[2]; z <= c1[2]; z++)
            for (int64_t y = c0[1]; y <= c1[1]; y++)
                for (int64_t x = c0[0]; x <= c1[0]; x++) {
                    int64_t cell = (z * g.n[1] + y) * g.n[0] + x;
                    for (int64_t k = g.start[cell]; k < g.start[cell + 1]; k++) {
                        int32_t s = g.items[k];
                        float sx = samples[3 * s], sy = samples[3 * s + 1], sz = samples[3 * s + 2];
                        if (!in_box(b, sx, sy, sz)) continue;
                        double dx = (double)sx - mx, dy = (double)sy - my, dz = (double)sz - mz;
                        double p = pair_power(c, dx, dy, dz);
                        if (p < ORC_POWER_FLOOR || p > 0.0) continue;
                        double W = out_weights[s];
                        if (W <= ORC_WEIGHT_CUTOFF) continue;
                        double go = gout[s], gww = gw[s];
                        double e = exp(p);
                        double wt = w * e;
                        a_v += go * wt / W;
                        double dLv_dwt = go * (v / W - (double)out_cells[s] / W);
                        double dwt_dq = -0.5 * wt;
                        a_w += dLv_dwt * e + gww * e;
                        double dq = dLv_dwt * dwt_dq + gww * dwt_dq;
                        a_mx += dq * -2.0 * (c[0] * dx + c[1] * dy + c[2] * dz);
                        a_my += dq * -2.0 * (c[1] * dx + c[3] * dy + c[4] * dz);
                        a_mz += dq * -2.0 * (c[2] * dx + c[4] * dy + c[5] * dz);
                        a_c[0] += dq * dx * dx;
                        a_c[1] += dq * 2.0 * dx * dy;
                        a_c[2] += dq * 2.0 * dx * dz;
                        a_c[3] += dq * dy * dy;
                        a_c[4] += dq * 2.0 * dy * dz;
                        a_c[5] += dq * dz * dz;
                    }
                }
        dvalues[i] = a_v;
        dweights[i] = a_w;
        dmeans[3 * i] = a_mx;
        dmeans[3 * i + 1] = a_my;
        dmeans[3 * i + 2] = a_mz;
        for (int k = 0; k < 6; k++) dconics[6 * i + k] = a_c[k];
    }
    grid_free(&g);
    free(sboxes);
}

/* ------------------------------------------------------------------------------------
 * Covariance adjoint: dconic (unique-parameter) -> dscales, drots (raw quaternion).
 * Mode 0 (true gradient, derived from the forward at forward.cu:27-76):
 *   G   = symmetric-matrix gradient (off-diagonals halved),
 *   H   = -C G C (gradient wrt Sigma + eps I),
 *   dSigma = H + tr(H) * deps/dSigma (eps = 1e-5 max|Sigma_kk|, first argmax),
 *   dM  = 2 M dSigma, M = diag(s) Rg,
 *   ds_k = sum_j dM[k][j] Rg[k][j] * scale_modifier, dRg[k][j] = s_k dM[k][j],
 *   dq  = chain rule through R_std(q) = Rg^T.
 * Mode 1 (reference-compatible): restates backward.cu:50-124 literally, including
 *   its un-halved off-diagonals, dL/dM = 2 dSigma M and the column scaling.
 * ------------------------------------------------------------------------------------ */
static void cov_backward_true_one(const float s_in[3], const float q_in[4], float sm, const double* dc,
                                  double ds_out[3], double dq_out[4]) {
    double r = q_in[0], x = q_in[1], y = q_in[2], z = q_in[3];
    double Rs[3][3] = {
        {1.0 - 2.0 * (y * y + z * z), 2.0 * (x * y - r * z), 2.0 * (x * z + r * y)},
        {2.0 * (x * y + r * z), 1.0 - 2.0 * (x * x + z * z), 2.0 * (y * z - r * x)},
        {2.0 * (x * z - r * y), 2.0 * (y * z + r * x), 1.0 - 2.0 * (x * x + y * y)}};
    double Rg[3][3];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) Rg[i][j] = Rs[j][i];
    double sv[3] = {(double)(sm * s_in[0]), (double)(sm * s_in[1]), (double)(sm * s_in[2])};
    double M[3][3], Sg[3][3];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) M[i][j] = sv[i] * Rg[i][j];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            double acc = 0;
            for (int k = 0; k < 3; k++) acc += M[k][i] * M[k][j];
            Sg[i][j] = acc;
        }
    double c6[6];
    conic_from_sigma_f64(Sg, c6);
    double C[3][3] = {{c6[0], c6[1], c6[2]}, {c6[1], c6[3], c6[4]}, {c6[2], c6[4], c6[5]}};
    double G[3][3] = {{dc[0], 0.5 * dc[1], 0.5 * dc[2]}, {0.5 * dc[1], dc[3], 0.5 * dc[4]}, {0.5 * dc[2], 0.5 * dc[4], dc[5]}};
    double T[3][3], H[3][3];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            double acc = 0;
            for (int k = 0; k < 3; k++) acc += G[i][k] * C[k][j];
            T[i][j] = acc;
        }
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            double acc = 0;
            for (int k = 0; k < 3; k++) acc += C[i][k] * T[k][j];
            H[i][j] = -acc;
        }
    /* eps derivative: first index attaining max |Sigma_kk| */
    double a0 = fabs(Sg[0][0]), a1 = fabs(Sg[1][1]), a2 = fabs(Sg[2][2]);
    int kmax = 0;
    if (a1 > a0) kmax = 1;
    if (a2 > (kmax == 0 ? a0 : a1)) kmax = 2;
    double trH = H[0][0] + H[1][1] + H[2][2];
    double sgn = Sg[kmax][kmax] > 0 ? 1.0 : (Sg[kmax][kmax] < 0 ? -1.0 : 0.0);
    H[kmax][kmax] += trH * 1e-5 * sgn;
    double dM[3][3];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            double acc = 0;
            for (int k = 0; k < 3; k++) acc += M[i][k] * H[k][j];
            dM[i][j] = 2.0 * acc;
        }
    double dRg[3][3];
    for (int k = 0; k < 3; k++) {
        double acc = 0;
        for (int j = 0; j < 3; j++) acc += dM[k][j] * Rg[k][j];
        ds_out[k] = acc * (double)sm;
        for (int j = 0; j < 3; j++) dRg[k][j] = sv[k] * dM[k][j];
    }
    double GR[3][3]; /* gradient wrt R_std */
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) GR[i][j] = dRg[j][i];
    dq_out[0] = 2.0 * (-z * GR[0][1] + y * GR[0][2] + z * GR[1][0] - x * GR[1][2] - y * GR[2][0] + x * GR[2][1]);
    dq_out[1] = 2.0 * (y * GR[0][1] + z * GR[0][2] + y * GR[1][0] - 2.0 * x * GR[1][1] - r * GR[1][2] + z * GR[2][0] +
                       r * GR[2][1] - 2.0 * x * GR[2][2]);
    dq_out[2] = 2.0 * (-2.0 * y * GR[0][0] + x * GR[0][1] + r * GR[0][2] + x * GR[1][0] + z * GR[1][2] - r * GR[2][0] +
                       z * GR[2][1] - 2.0 * y * GR[2][2]);
    dq_out[3] = 2.0 * (-2.0 * z * GR[0][0] - r * GR[0][1] + x * GR[0][2] + r * GR[1][0] - 2.0 * z * GR[1][1] +
                       y * GR[1][2] + x * GR[2][0] + y * GR[2][1]);
}

/* backward.cu:9-125 restated with glm column-major semantics, in double. */
static void cov_backward_ref_one(const float s_in[3], const float q_in[4], float sm, const float* conic,
                                 const double* dc, double ds_out[3], double dq_out[4]) {
    double r = q_in[0], x = q_in[1], y = q_in[2], z = q_in[3];
    /* glm matrices stored [col][row] */
    double Rc[3][3] = {{1.0 - 2.0 * (y * y + z * z), 2.0 * (x * y - r * z), 2.0 * (x * z + r * y)},
                       {2.0 * (x * y + r * z), 1.0 - 2.0 * (x * x + z * z), 2.0 * (y * z - r * x)},
                       {2.0 * (x * z - r * y), 2.0 * (y * z + r * x), 1.0 - 2.0 * (x * x + y * y)}};
    double sv[3] = {(double)(sm * s_in[0]), (double)(sm * s_in[1]), (double)(sm * s_in[2])};
    /* glm product A*B: (A*B)[c][r] = sum_k A[k][r] * B[c][k] */
#define GLM_MUL(A, B, OUT)                                                          \
    for (int cc_ = 0; cc_ < 3; cc_++)                                               \
        for (int rr_ = 0; rr_ < 3; rr_++) {                                         \
            double acc_ = 0;                                                        \
            for (int kk_ = 0; kk_ < 3; kk_++) acc_ += (A)[kk_][rr_] * (B)[cc_][kk_]; \
            (OUT)[cc_][rr_] = acc_;                                                 \
        }
    double Sm[3][3] = {{sv[0], 0, 0}, {0, sv[1], 0}, {0, 0, sv[2]}};
    double M[3][3], Mt[3][3], Sigma[3][3];
    GLM_MUL(Sm, Rc, M);
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) Mt[i][j] = M[j][i];
    GLM_MUL(Mt, M, Sigma);
    double C[3][3] = {{conic[0], conic[1], conic[2]}, {conic[1], conic[3], conic[4]}, {conic[2], conic[4], conic[5]}};
    double G[3][3] = {{dc[0], dc[1], dc[2]}, {dc[1], dc[3], dc[4]}, {dc[2], dc[4], dc[5]}};
    double negC[3][3], T1[3][3], dS[3][3];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) negC[i][j] = -C[i][j];
    GLM_MUL(negC, G, T1);
    GLM_MUL(T1, C, dS);
    double dcov[6] = {dS[0][0], dS[0][1], dS[0][2], dS[1][1], dS[1][2], dS[2][2]};
    double a0 = fabs(Sigma[0][0]), a1 = fabs(Sigma[1][1]), a2 = fabs(Sigma[2][2]);
#define SGN(v) ((v) > 0 ? 1.0 : ((v) < 0 ? -1.0 : 0.0))
    double de0 = (a0 >= a1 && a0 >= a2) ? 1e-5 * SGN(Sigma[0][0]) : 0.0;
    double de1 = (a1 >= a0 && a1 >= a2) ? 1e-5 * SGN(Sigma[1][1]) : 0.0;
    double de2 = (a2 >= a0 && a2 >= a1) ? 1e-5 * SGN(Sigma[2][2]) : 0.0;
    double tr = dcov[0] + dcov[3] + dcov[5];
    double dLdSigma[3][3] = {{dcov[0] + tr * de0, dcov[1], dcov[2]},
                             {dcov[1], dcov[3] + tr * de1, dcov[4]},
                             {dcov[2], dcov[4], dcov[5] + tr * de2}};
    double dM[3][3], Rt[3][3], dSm[3][3];
    GLM_MUL(dLdSigma, M, dM);
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) dM[i][j] *= 2.0;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) Rt[i][j] = Rc[j][i];
    GLM_MUL(dM, Rt, dSm);
    ds_out[0] = dSm[0][0] * sm;
    ds_out[1] = dSm[1][1] * sm;
    ds_out[2] = dSm[2][2] * sm;
    for (int k = 0; k < 3; k++)
        for (int rr = 0; rr < 3; rr++) dM[k][rr] *= sv[k]; /* dL_dM[k] *= s_k scales glm column k */
    dq_out[0] = 2 * z * (dM[1][0] - dM[0][1]) + 2 * y * (dM[0][2] - dM[2][0]) + 2 * x * (dM[2][1] - dM[1][2]);
    dq_out[1] = 2 * y * (dM[0][1] + dM[1][0]) + 2 * z * (dM[0][2] + dM[2][0]) + 2 * r * (dM[2][1] - dM[1][2]) -
                4 * x * (dM[2][2] + dM[1][1]);
    dq_out[2] = 2 * x * (dM[0][1] + dM[1][0]) + 2 * r * (dM[0][2] - dM[2][0]) + 2 * z * (dM[2][1] + dM[1][2]) -
                4 * y * (dM[2][2] + dM[0][0]);
    dq_out[3] = 2 * r * (dM[1][0] - dM[0][1]) + 2 * x * (dM[0][2] + dM[2][0]) + 2 * y * (dM[2][1] + dM[1][2]) -
                4 * z * (dM[1][1] + dM[0][0]);
#undef GLM_MUL
#undef SGN
}

void orc_cov_backward(int64_t P, const float* scales, const float* rots, const float* conics32, float sm,
                      const double* dconics, int ref_compat, double* dscales, double* drots, int nthreads) {
    int nt = orc_nthreads(nthreads);
#pragma omp parallel for num_threads(nt) schedule(static)
    for (int64_t i = 0; i < P; i++) {
        if (ref_compat)
            cov_backward_ref_one(scales + 3 * i, rots + 4 * i, sm, conics32 + 6 * i, dconics + 6 * i, dscales + 3 * i,
                                 drots + 4 * i);
        else
            cov_backward_true_one(scales + 3 * i, rots + 4 * i, sm, dconics + 6 * i, dscales + 3 * i, drots + 4 * i);
    }
}

/* ------------------------------------------------------------------------------------
 * LBVH specification (declared; the reference delegates to cuBQL's radixBuilder,
 * rasterizer_impl.cu:78-83 and ext.cu:50-54, whose ordering is not vendored).
 *   key  = 30-bit Morton code (10 bits/axis, x in the lowest bit of each triple)
 *          of the box centroid c = (lo + hi) * 0.5f, quantised over the float
 *          bounds [blo, bhi] of all centroids: q = (c - blo) * (1024 / (bhi - blo)),
 *          all in float with single roundings, clamped to [0, 1023] (NaN -> 0);
 *   order = stable sort by key (ties keep the input index order);
 *   tree = Karras 2012 radix tree over the sorted keys, equal keys disambiguated by
 *          the sorted position (delta = 32 + clz(i ^ j));
 *   child encoding: internal node k >= 0, leaf i encoded as (i | 0x80000000);
 *   boxes = min/max refit (order independent, exact).
 * ------------------------------------------------------------------------------------ */
static uint32_t expand10(uint32_t v) {
    v &= 0x3ffu;
    v = (v | (v << 16)) & 0x030000FFu;
    v = (v | (v << 8)) & 0x0300F00Fu;
    v = (v | (v << 4)) & 0x030C30C3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}

static uint32_t quant10(float c, float lo, float scale) {
    float t = (c - lo) * scale;
    if (!(t >= 0.0f)) return 0;
    if (t >= 1023.0f) return 1023;
    return (uint32_t)t;
}

void orc_centroid_bounds(int64_t n, const float* boxes, float blo[3], float bhi[3]) {
    for (int a = 0; a < 3; a++) { blo[a] = INFINITY; bhi[a] = -INFINITY; }
    for (int64_t i = 0; i < n; i++)
        for (int a = 0; a < 3; a++) {
            float c = (boxes[6 * i + a] + boxes[6 * i + 3 + a]) * 0.5f;
            blo[a] = fminf(blo[a], c);
            bhi[a] = fmaxf(bhi[a], c);
        }
}

void orc_morton_keys(int64_t n, const float* boxes, const float blo[3], const float bhi[3], uint32_t* keys) {
    float scale[3];
    for (int a = 0; a < 3; a++) {
        float ext = bhi[a] - blo[a];
        scale[a] = ext > 0.0f ? 1024.0f / ext : 0.0f;
    }
    for (int64_t i = 0; i < n; i++) {
        uint32_t q[3];
        for (int a = 0; a < 3; a++) {
            float c = (boxes[6 * i + a] + boxes[6 * i + 3 + a]) * 0.5f;
            q[a] = quant10(c, blo[a], scale[a]);
        }
        keys[i] = expand10(q[0]) | (expand10(q[1]) << 1) | (expand10(q[2]) << 2);
    }
}

/* Stable LSD counting sort on 32-bit keys, values = input index. */
void orc_sort_keys(int64_t n, const uint32_t* keys_in, uint32_t* keys_out, int32_t* perm) {
    uint32_t* k0 = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)(n ? n : 1));
    uint32_t* k1 = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)(n ? n : 1));
    int32_t* v0 = (int32_t*)malloc(sizeof(int32_t) * (size_t)(n ? n : 1));
    int32_t* v1 = (int32_t*)malloc(sizeof(int32_t) * (size_t)(n ? n : 1));
    for (int64_t i = 0; i < n; i++) { k0[i] = keys_in[i]; v0[i] = (int32_t)i; }
    for (int pass = 0; pass < 4; pass++) {
        int64_t cnt[257] = {0};
        int sh = pass * 8;
        for (int64_t i = 0; i < n; i++) cnt[((k0[i] >> sh) & 255u) + 1]++;
        for (int d = 0; d < 256; d++) cnt[d + 1] += cnt[d];
        for (int64_t i = 0; i < n; i++) {
            int64_t dst = cnt[(k0[i] >> sh) & 255u]++;
            k1[dst] = k0[i];
            v1[dst] = v0[i];
        }
        uint32_t* tk = k0; k0 = k1; k1 = tk;
        int32_t* tv = v0; v0 = v1; v1 = tv;
    }
    memcpy(keys_out, k0, sizeof(uint32_t) * (size_t)n);
    memcpy(perm, v0, sizeof(int32_t) * (size_t)n);
    free(k0); free(k1); free(v0); free(v1);
}

static int delta_fn(const uint32_t* k, int64_t n, int64_t i, int64_t j) {
    if (j < 0 || j >= n) return -1;
    uint32_t a = k[i], b = k[j];
    if (a == b) return 32 + __builtin_clz((uint32_t)(i ^ j)); /* i != j on every call */
    return __builtin_clz(a ^ b);
}

/* Karras 2012, "Maximizing parallelism in the construction of BVHs, octrees and k-d trees",
   Fig. 4: internal node i of n-1 finds its key range and split. */
void orc_karras(int64_t n, const uint32_t* skeys, int32_t* left, int32_t* right, int32_t* parent_int,
                int32_t* parent_leaf) {
    if (n < 2) { if (n == 1) parent_leaf[0] = -1; return; }
    for (int64_t i = 0; i < n - 1; i++) {
        int d = (delta_fn(skeys, n, i, i + 1) - delta_fn(skeys, n, i, i - 1)) >= 0 ? 1 : -1;
        int dmin = delta_fn(skeys, n, i, i - d);
        int64_t lmax = 2;
        while (delta_fn(skeys, n, i, i + lmax * d) > dmin) lmax *= 2;
        int64_t l = 0;
        for (int64_t t = lmax / 2; t >= 1; t /= 2)
            if (delta_fn(skeys, n, i, i + (l + t) * d) > dmin) l += t;
        int64_t j = i + l * d;
        int dnode = delta_fn(skeys, n, i, j);
        int64_t s = 0;
        int64_t t = l;
        do {
            t = (t + 1) / 2;
            if (delta_fn(skeys, n, i, i + (s + t) * d) > dnode) s += t;
        } while (t > 1);
        int64_t gamma = i + s * d + (d < 0 ? d : 0);
        int64_t lo = i < j ? i : j, hi = i < j ? j : i;
        if (lo == gamma) { left[i] = (int32_t)(gamma | 0x80000000u); parent_leaf[gamma] = (int32_t)i; }
        else { left[i] = (int32_t)gamma; parent_int[gamma] = (int32_t)i; }
        if (hi == gamma + 1) { right[i] = (int32_t)((gamma + 1) | 0x80000000u); parent_leaf[gamma + 1] = (int32_t)i; }
        else { right[i] = (int32_t)(gamma + 1); parent_int[gamma + 1] = (int32_t)i; }
    }
    parent_int[0] = -1;
}

/* Refit: node boxes (internal) from leaf boxes given in SORTED order. */
static void refit_rec(int32_t node, const int32_t* left, const int32_t* right, const float* leaf_boxes,
                      float* node_boxes, float out[6]) {
    /* iterative post-order would avoid deep recursion; LBVH depth is bounded (<= 64 + log n) */
    int32_t ch[2] = {left[node], right[node]};
    float b[2][6];
    for (int c = 0; c < 2; c++) {
        if (ch[c] < 0) {
            int32_t li = ch[c] & 0x7fffffff;
            memcpy(b[c], leaf_boxes + 6 * (int64_t)li, sizeof(float) * 6);
        } else {
            refit_rec(ch[c], left, right, leaf_boxes, node_boxes, b[c]);
        }
    }
    for (int a = 0; a < 3; a++) {
        out[a] = fminf(b[0][a], b[1][a]);
        out[3 + a] = fmaxf(b[0][3 + a], b[1][3 + a]);
    }
    memcpy(node_boxes + 6 * (int64_t)node, out, sizeof(float) * 6);
}

void orc_refit(int64_t n, const int32_t* left, const int32_t* right, const float* leaf_boxes_sorted,
               float* node_boxes) {
    if (n < 2) return;
    float root[6];
    refit_rec(0, left, right, leaf_boxes_sorted, node_boxes, root);
}

/* Full build: boxes [n,6] in input order -> sorted keys, perm, children, node boxes. */
void orc_lbvh_build(int64_t n, const float* boxes, uint32_t* skeys, int32_t* perm, int32_t* left, int32_t* right,
                    float* node_boxes) {
    float blo[3], bhi[3];
    uint32_t* keys = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)(n ? n : 1));
    orc_centroid_bounds(n, boxes, blo, bhi);
    orc_morton_keys(n, boxes, blo, bhi, keys);
    orc_sort_keys(n, keys, skeys, perm);
    int32_t* pi = (int32_t*)malloc(sizeof(int32_t) * (size_t)(n ? n : 1));
    int32_t* pl = (int32_t*)malloc(sizeof(int32_t) * (size_t)(n ? n : 1));
    orc_karras(n, skeys, left, right, pi, pl);
    float* sb = (float*)malloc(sizeof(float) * 6 * (size_t)(n ? n : 1));
    for (int64_t i = 0; i < n; i++) memcpy(sb + 6 * i, boxes + 6 * (int64_t)perm[i], sizeof(float) * 6);
    orc_refit(n, left, right, sb, node_boxes);
    free(sb); free(pi); free(pl); free(keys);
}

/* ------------------------------------------------------------------------------------
 * Mesh sampling oracle (gpu_sampling/sample_mesh.cu:26-240 uniform, :242-414 explicit;
 * the reference delegates location and interpolation to Viskores' Probe filter with
 * invalid value -1, sample_mesh.cu:155-167,380-390).  Declared semantics:
 *   uniform: f = (x - o) / sp per axis in double; inside iff 0 <= f <= n-1 on every
 *            axis; cell i = min(floor(f), n-2) (0 for n == 1); t = f - i;
 *            trilinear with lerp(a, b, t) = a + t * (b - a), x first, then y, then z.
 *   tets:    orient(a,b,c,d) = det[b-a, c-a, d-a] in double, left-to-right;
 *            inside (closed) iff every sub-volume has the sign of the full volume or
 *            is zero; degenerate tets (volume 0) never contain a point;
 *            ties -> the lowest containing cell id; value = sum_k (V_k / V) f_k.
 * ------------------------------------------------------------------------------------ */
static inline double lerp_d(double a, double b, double t) { return a + t * (b - a); }

/* values given as double (converted by the caller from the source dtype) */
void orc_sample_uniform(const int64_t dims[3], const float origin[3], const float spacing[3], const double* values,
                        int64_t N, const float* samples, double* out, int8_t* valid, int nthreads) {
    int nt = orc_nthreads(nthreads);
    int64_t nx = dims[0], ny = dims[1], nz = dims[2];
#pragma omp parallel for num_threads(nt) schedule(static)
    for (int64_t s = 0; s < N; s++) {
        int64_t ci[3];
        double t[3];
        int ok = 1;
        for (int a = 0; a < 3; a++) {
            double f = ((double)samples[3 * s + a] - (double)origin[a]) / (double)spacing[a];
            int64_t n = dims[a];
            if (!(f >= 0.0) || !(f <= (double)(n - 1))) { ok = 0; break; }
            if (n == 1) { ci[a] = 0; t[a] = 0.0; continue; }
            int64_t i = (int64_t)floor(f);
            if (i > n - 2) i = n - 2;
            ci[a] = i;
            t[a] = f - (double)i;
        }
        if (!ok) { out[s] = -1.0; valid[s] = 0; continue; }
        int64_t sx = nx > 1 ? 1 : 0, sy = ny > 1 ? nx : 0, sz = nz > 1 ? nx * ny : 0;
        int64_t b = ci[0] + nx * (ci[1] + ny * ci[2]);
        double v000 = values[b], v100 = values[b + sx], v010 = values[b + sy], v110 = values[b + sx + sy];
        double v001 = values[b + sz], v101 = values[b + sx + sz], v011 = values[b + sy + sz],
               v111 = values[b + sx + sy + sz];
        double c00 = lerp_d(v000, v100, t[0]), c10 = lerp_d(v010, v110, t[0]);
        double c01 = lerp_d(v001, v101, t[0]), c11 = lerp_d(v011, v111, t[0]);
        double c0 = lerp_d(c00, c10, t[1]), c1 = lerp_d(c01, c11, t[1]);
        out[s] = lerp_d(c0, c1, t[2]);
        valid[s] = 1;
    }
}

static inline double det3(double ux, double uy, double uz, double vx, double vy, double vz, double wx, double wy,
                          double wz) {
    double m0 = vy * wz - vz * wy;
    double m1 = vx * wz - vz * wx;
    double m2 = vx * wy - vy * wx;
    double r = ux * m0;
    r = r - uy * m1;
    r = r + uz * m2;
    return r;
}

static inline double orient(const float* a, const float* b, const float* c, const float* d) {
    double ax = a[0], ay = a[1], az = a[2];
    return det3((double)b[0] - ax, (double)b[1] - ay, (double)b[2] - az, (double)c[0] - ax, (double)c[1] - ay,
                (double)c[2] - az, (double)d[0] - ax, (double)d[1] - ay, (double)d[2] - az);
}

/* returns 1 and fills lambda[4] if p is inside tet (a,b,c,d) */
static int tet_contains(const float* a, const float* b, const float* c, const float* d, const float* p,
                        double lam[4]) {
    double V = orient(a, b, c, d);
    if (V == 0.0) return 0;
    double Va = orient(p, b, c, d), Vb = orient(a, p, c, d), Vc = orient(a, b, p, d), Vd = orient(a, b, c, p);
    if (V > 0) {
        if (Va < 0 || Vb < 0 || Vc < 0 || Vd < 0) return 0;
    } else {
        if (Va > 0 || Vb > 0 || Vc > 0 || Vd > 0) return 0;
    }
    lam[0] = Va / V; lam[1] = Vb / V; lam[2] = Vc / V; lam[3] = Vd / V;
    return 1;
}

void orc_tet_boxes(int64_t C, const float* pts, const int64_t* conn4, float* boxes) {
    for (int64_t c = 0; c < C; c++) {
        for (int a = 0; a < 3; a++) { boxes[6 * c + a] = INFINITY; boxes[6 * c + 3 + a] = -INFINITY; }
        for (int k = 0; k < 4; k++) {
            const float* v = pts + 3 * conn4[4 * c + k];
            for (int a = 0; a < 3; a++) {
                boxes[6 * c + a] = fminf(boxes[6 * c + a], v[a]);
                boxes[6 * c + 3 + a] = fmaxf(boxes[6 * c + 3 + a], v[a]);
            }
        }
    }
}

/* conn4: [C,4] vertex ids; values: [npts] double. out: value or -1; cell: id or -1. */
void orc_sample_tets(int64_t npts, const float* pts, int64_t C, const int64_t* conn4, const double* values,
                     int64_t N, const float* samples, double* out, int64_t* cell, int nthreads) {
    int nt = orc_nthreads(nthreads);
    (void)npts;
    float* boxes = (float*)malloc(sizeof(float) * 6 * (size_t)(C ? C : 1));
    orc_tet_boxes(C, pts, conn4, boxes);
    double glo[3], ghi[3];
    boxes_bounds(C, boxes, glo, ghi);
    orc_grid g;
    grid_build(&g, C, boxes, glo, ghi, median_extent(C, boxes), nt);
#pragma omp parallel for num_threads(nt) schedule(dynamic, 1024)
    for (int64_t s = 0; s < N; s++) {
        const float* p = samples + 3 * s;
        out[s] = -1.0;
        cell[s] = -1;
        if (C == 0) continue;
        int64_t cl = grid_cell_of_point(&g, p);
        if (cl < 0) continue;
        for (int64_t k = g.start[cl]; k < g.start[cl + 1]; k++) { /* ids ascending: first hit is lowest */
            int32_t c = g.items[k];
            const float* bx = boxes + 6 * (int64_t)c;
            if (!in_box(bx, p[0], p[1], p[2])) continue;
            double lam[4];
            const int64_t* cv = conn4 + 4 * (int64_t)c;
            if (tet_contains(pts + 3 * cv[0], pts + 3 * cv[1], pts + 3 * cv[2], pts + 3 * cv[3], p, lam)) {
                double v = lam[0] * values[cv[0]];
                v = v + lam[1] * values[cv[1]];
                v = v + lam[2] * values[cv[2]];
                v = v + lam[3] * values[cv[3]];
                out[s] = v;
                cell[s] = c;
                break;
            }
        }
    }
    grid_free(&g);
    free(boxes);
}

/* ------------------------------------------------------------------------------------
 * General explicit cells (gpu_sampling/sample_mesh.cu:300-336 maps VTK types 1,3,5,9,10,
 * 12,13,14 to Viskores shapes).  Declared semantics:
 *   10 tetra: as orc_sample_tets;
 *   12 hexahedron, 13 wedge, 14 pyramid: isoparametric shape functions in VTK node order
 *      hex:   N = (1-r)(1-s)(1-t), r(1-s)(1-t), rs(1-t), (1-r)s(1-t), (1-r)(1-s)t, r(1-s)t, rst, (1-r)st
 *      wedge: N = (1-r-s)(1-t), r(1-t), s(1-t), (1-r-s)t, rt, st
 *      pyram: N = (1-r)(1-s)(1-t), r(1-s)(1-t), rs(1-t), (1-r)s(1-t), t
 *      the point is mapped to (r,s,t) by Newton's method in double (start at the cell's
 *      parametric centre, at most 20 iterations, stop when max|dr| < 1e-13, singular
 *      Jacobian -> outside), inside iff every parametric bound holds within 1e-9
 *      (hex: 0 <= r,s,t <= 1; wedge: r,s >= 0, r+s <= 1, 0 <= t <= 1; pyramid: 0 <= r,s,t <= 1);
 *   1 vertex, 3 line, 5 triangle, 9 quad: zero volume, never contain a probe point.
 *   Ties -> the lowest cell id; outside every cell -> -1.
 * The same expressions (no FMA contraction) run on the GPU.
 * ------------------------------------------------------------------------------------ */
#define ORC_NEWTON_ITERS 20
#define ORC_NEWTON_TOL 1e-13
#define ORC_INSIDE_EPS 1e-9

static int shape_eval(int type, double r, double s, double t, double N[8], double dN[8][3]) {
    switch (type) {
        case 12: {
            double rm = 1.0 - r, sm = 1.0 - s, tm = 1.0 - t;
            N[0] = rm * sm * tm; N[1] = r * sm * tm; N[2] = r * s * tm; N[3] = rm * s * tm;
            N[4] = rm * sm * t;  N[5] = r * sm * t;  N[6] = r * s * t;  N[7] = rm * s * t;
            dN[0][0] = -(sm * tm); dN[0][1] = -(rm * tm); dN[0][2] = -(rm * sm);
            dN[1][0] = sm * tm;    dN[1][1] = -(r * tm);  dN[1][2] = -(r * sm);
            dN[2][0] = s * tm;     dN[2][1] = r * tm;     dN[2][2] = -(r * s);
            dN[3][0] = -(s * tm);  dN[3][1] = rm * tm;    dN[3][2] = -(rm * s);
            dN[4][0] = -(sm * t);  dN[4][1] = -(rm * t);  dN[4][2] = rm * sm;
            dN[5][0] = sm * t;     dN[5][1] = -(r * t);   dN[5][2] = r * sm;
            dN[6][0] = s * t;      dN[6][1] = r * t;      dN[6][2] = r * s;
            dN[7][0] = -(s * t);   dN[7][1] = rm * t;     dN[7][2] = rm * s;
            return 8;
        }
        case 13: {
            double u = 1.0 - r - s, tm = 1.0 - t;
            N[0] = u * tm; N[1] = r * tm; N[2] = s * tm; N[3] = u * t; N[4] = r * t; N[5] = s * t;
            dN[0][0] = -tm; dN[0][1] = -tm; dN[0][2] = -u;
            dN[1][0] = tm;  dN[1][1] = 0.0; dN[1][2] = -r;
            dN[2][0] = 0.0; dN[2][1] = tm;  dN[2][2] = -s;
            dN[3][0] = -t;  dN[3][1] = -t;  dN[3][2] = u;
            dN[4][0] = t;   dN[4][1] = 0.0; dN[4][2] = r;
            dN[5][0] = 0.0; dN[5][1] = t;   dN[5][2] = s;
            return 6;
        }
        case 14: {
            double rm = 1.0 - r, sm = 1.0 - s, tm = 1.0 - t;
            N[0] = rm * sm * tm; N[1] = r * sm * tm; N[2] = r * s * tm; N[3] = rm * s * tm; N[4] = t;
            dN[0][0] = -(sm * tm); dN[0][1] = -(rm * tm); dN[0][2] = -(rm * sm);
            dN[1][0] = sm * tm;    dN[1][1] = -(r * tm);  dN[1][2] = -(r * sm);
            dN[2][0] = s * tm;     dN[2][1] = r * tm;     dN[2][2] = -(r * s);
            dN[3][0] = -(s * tm);  dN[3][1] = rm * tm;    dN[3][2] = -(rm * s);
            dN[4][0] = 0.0;        dN[4][1] = 0.0;        dN[4][2] = 1.0;
            return 5;
        }
    }
    return 0;
}

/* Newton inversion + inside test; on success writes the shape function values. */
static int iso_contains(int type, const float* pts, const int32_t* cv, const float* p, double Nout[8]) {
    double r, s, t;
    if (type == 12) { r = 0.5; s = 0.5; t = 0.5; }
    else if (type == 13) { r = 1.0 / 3.0; s = 1.0 / 3.0; t = 0.5; }
    else { r = 0.5; s = 0.5; t = 0.25; }
    double N[8], dN[8][3];
    int n = 0, converged = 0;
    for (int it = 0; it < ORC_NEWTON_ITERS; it++) {
        n = shape_eval(type, r, s, t, N, dN);
        double f[3] = {0.0, 0.0, 0.0}, J[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
        for (int k = 0; k < n; k++) {
            const float* x = pts + 3 * (int64_t)cv[k];
            for (int a = 0; a < 3; a++) {
                f[a] = f[a] + N[k] * (double)x[a];
                for (int b = 0; b < 3; b++) J[a][b] = J[a][b] + dN[k][b] * (double)x[a];
            }
        }
        for (int a = 0; a < 3; a++) f[a] = f[a] - (double)p[a];
        double det = det3(J[0][0], J[0][1], J[0][2], J[1][0], J[1][1], J[1][2], J[2][0], J[2][1], J[2][2]);
        if (det == 0.0 || det != det) return 0;
        /* Cramer's rule for J d = f */
        double d0 = det3(f[0], J[0][1], J[0][2], f[1], J[1][1], J[1][2], f[2], J[2][1], J[2][2]) / det;
        double d1 = det3(J[0][0], f[0], J[0][2], J[1][0], f[1], J[1][2], J[2][0], f[2], J[2][2]) / det;
        double d2 = det3(J[0][0], J[0][1], f[0], J[1][0], J[1][1], f[1], J[2][0], J[2][1], f[2]) / det;
        r = r - d0;
        s = s - d1;
        t = t - d2;
        double m = fabs(d0);
        if (fabs(d1) > m) m = fabs(d1);
        if (fabs(d2) > m) m = fabs(d2);
        if (!(m >= ORC_NEWTON_TOL)) {
            converged = 1;
            break;
        }
    }
    /* an unconverged iterate says nothing about the point: not contained */
    if (!converged) return 0;
    const double e = ORC_INSIDE_EPS;
    int inside;
    if (type == 13) inside = r >= -e && s >= -e && r + s <= 1.0 + e && t >= -e && t <= 1.0 + e;
    else inside = r >= -e && r <= 1.0 + e && s >= -e && s <= 1.0 + e && t >= -e && t <= 1.0 + e;
    if (!inside) return 0;
    n = shape_eval(type, r, s, t, N, dN);
    for (int k = 0; k < n; k++) Nout[k] = N[k];
    return n;
}

static int cell_npts(int type) {
    switch (type) {
        case 10: return 4;
        case 12: return 8;
        case 13: return 6;
        case 14: return 5;
    }
    return 0;
}

/* types[C] (VTK ids), offsets[C] (start of each cell in conn), conn int32. */
void orc_sample_cells(int64_t npts, const float* pts, int64_t C, const uint8_t* types, const int64_t* offsets,
                      const int32_t* conn, const double* values, int64_t N, const float* samples, double* out,
                      int64_t* cell, int nthreads) {
    int nt = orc_nthreads(nthreads);
    (void)npts;
    float* boxes = (float*)malloc(sizeof(float) * 6 * (size_t)(C ? C : 1));
    for (int64_t c = 0; c < C; c++) {
        int n = cell_npts(types[c]);
        for (int a = 0; a < 3; a++) { boxes[6 * c + a] = INFINITY; boxes[6 * c + 3 + a] = -INFINITY; }
        for (int k = 0; k < n; k++) {
            const float* v = pts + 3 * (int64_t)conn[offsets[c] + k];
            for (int a = 0; a < 3; a++) {
                boxes[6 * c + a] = fminf(boxes[6 * c + a], v[a]);
                boxes[6 * c + 3 + a] = fmaxf(boxes[6 * c + 3 + a], v[a]);
            }
        }
    }
    double glo[3], ghi[3];
    boxes_bounds(C, boxes, glo, ghi);
    orc_grid g;
    grid_build(&g, C, boxes, glo, ghi, median_extent(C, boxes), nt);
#pragma omp parallel for num_threads(nt) schedule(dynamic, 1024)
    for (int64_t s = 0; s < N; s++) {
        const float* p = samples + 3 * s;
        out[s] = -1.0;
        cell[s] = -1;
        if (C == 0) continue;
        int64_t cl = grid_cell_of_point(&g, p);
        if (cl < 0) continue;
        for (int64_t k = g.start[cl]; k < g.start[cl + 1]; k++) {
            int32_t c = g.items[k];
            if (!in_box(boxes + 6 * (int64_t)c, p[0], p[1], p[2])) continue;
            const int32_t* cv = conn + offsets[c];
            int type = types[c];
            if (type == 10) {
                double lam[4];
                if (tet_contains(pts + 3 * cv[0], pts + 3 * cv[1], pts + 3 * cv[2], pts + 3 * cv[3], p, lam)) {
                    double v = lam[0] * values[cv[0]];
                    v = v + lam[1] * values[cv[1]];
                    v = v + lam[2] * values[cv[2]];
                    v = v + lam[3] * values[cv[3]];
                    out[s] = v;
                    cell[s] = c;
                    break;
                }
            } else if (type == 12 || type == 13 || type == 14) {
                double Nf[8] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
                int n = iso_contains(type, pts, cv, p, Nf);
                if (n) {
                    double v = Nf[0] * values[cv[0]];
                    for (int q = 1; q < n; q++) v = v + Nf[q] * values[cv[q]];
                    out[s] = v;
                    cell[s] = c;
                    break;
                }
            }
        }
    }
    grid_free(&g);
    free(boxes);
}

/* ------------------------------------------------------------------------------------
 * Three-nearest-neighbour mean squared distance: the initial Gaussian scale rule of
 * scene/gaussian_model.py:175-179 (create_from_pcd) and :729-733 (densify_in_empty),
 * which call simple-knn's distCUDA2 (third-party, not in the reference tree).  Its
 * published behaviour: per point, the three smallest squared distances to any OTHER
 * index (duplicates count with distance 0), ascending, summed (b0 + b1) + b2 and
 * divided by 3 in float32; missing neighbours count as FLT_MAX.  The squared distance
 * is (dx*dx + dy*dy) + dz*dz in float32 with every operation rounded (no contraction).
 *
 * Search: exact, on a uniform grid of about n/2 cells (at most 1001 per axis); rings of
 * cells around the query's cell are scanned until the distance from the query to the
 * outside of the scanned block (in double, less a relative margin far above float
 * rounding) exceeds the current third-best distance.
 * ------------------------------------------------------------------------------------ */
static inline float knn_d2(const float* a, const float* b) {
    float dx = a[0] - b[0], dy = a[1] - b[1], dz = a[2] - b[2];
    float xx = dx * dx, yy = dy * dy, zz = dz * dz;
    float s = xx + yy;
    return s + zz;
}

static inline void knn_keep3(float d, float* b) {
    if (d < b[2]) {
        if (d < b[1]) {
            b[2] = b[1];
            if (d < b[0]) { b[1] = b[0]; b[0] = d; } else { b[1] = d; }
        } else {
            b[2] = d;
        }
    }
}

void orc_knn3_mean_dist2(int64_t n, const float* pts, float* out, int nthreads) {
    int nt = orc_nthreads(nthreads);
    if (n <= 0) return;
    double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int64_t i = 0; i < n; i++)
        for (int a = 0; a < 3; a++) {
            double v = pts[3 * i + a];
            if (v < lo[a]) lo[a] = v;
            if (v > hi[a]) hi[a] = v;
        }
    double ext = 0.0;
    for (int a = 0; a < 3; a++) ext = fmax(ext, hi[a] - lo[a]);
    if (!(ext > 0.0)) ext = 1.0;
    /* cubic cells of side h, about n/2 cells over the bounding box */
    double vol = 1.0;
    for (int a = 0; a < 3; a++) vol *= fmax(hi[a] - lo[a], ext * 1e-3);
    double h = cbrt(vol / fmax(1.0, 0.5 * (double)n));
    if (!(h > 0.0)) h = ext;
    for (int a = 0; a < 3; a++) h = fmax(h, (hi[a] - lo[a]) / 1000.0);
    int64_t dim[3];
    for (int a = 0; a < 3; a++) dim[a] = (int64_t)(floor((hi[a] - lo[a]) / h) + 1.0);
    int64_t ncell = dim[0] * dim[1] * dim[2];
    int64_t* start = (int64_t*)calloc((size_t)ncell + 1, sizeof(int64_t));
    int64_t* cellof = (int64_t*)malloc(sizeof(int64_t) * (size_t)n);
    int64_t* items = (int64_t*)malloc(sizeof(int64_t) * (size_t)n);
    for (int64_t i = 0; i < n; i++) {
        int64_t c[3];
        for (int a = 0; a < 3; a++) {
            double f = floor(((double)pts[3 * i + a] - lo[a]) / h);
            c[a] = clampi((int64_t)f, 0, dim[a] - 1);
        }
        cellof[i] = (c[2] * dim[1] + c[1]) * dim[0] + c[0];
        start[cellof[i] + 1]++;
    }
    for (int64_t c = 0; c < ncell; c++) start[c + 1] += start[c];
    {
        int64_t* fill = (int64_t*)malloc(sizeof(int64_t) * (size_t)ncell);
        memcpy(fill, start, sizeof(int64_t) * (size_t)ncell);
        for (int64_t i = 0; i < n; i++) items[fill[cellof[i]]++] = i;
        free(fill);
    }
    int64_t rmax = dim[0];
    if (dim[1] > rmax) rmax = dim[1];
    if (dim[2] > rmax) rmax = dim[2];
#pragma omp parallel for num_threads(nt) schedule(dynamic, 256)
    for (int64_t i = 0; i < n; i++) {
        const float* q = pts + 3 * i;
        int64_t c[3];
        c[0] = cellof[i] % dim[0];
        c[1] = (cellof[i] / dim[0]) % dim[1];
        c[2] = cellof[i] / (dim[0] * dim[1]);
        float b[3] = {FLT_MAX, FLT_MAX, FLT_MAX};
        for (int64_t r = 0; r <= rmax; r++) {
            for (int64_t z = c[2] - r; z <= c[2] + r; z++) {
                if (z < 0 || z >= dim[2]) continue;
                for (int64_t y = c[1] - r; y <= c[1] + r; y++) {
                    if (y < 0 || y >= dim[1]) continue;
                    int shell_zy = (z == c[2] - r || z == c[2] + r || y == c[1] - r || y == c[1] + r);
                    for (int64_t x = c[0] - r; x <= c[0] + r; x++) {
                        if (x < 0 || x >= dim[0]) continue;
                        if (!shell_zy && x != c[0] - r && x != c[0] + r) continue;
                        int64_t cl = (z * dim[1] + y) * dim[0] + x;
                        for (int64_t k = start[cl]; k < start[cl + 1]; k++) {
                            int64_t j = items[k];
                            if (j == i) continue;
                            knn_keep3(knn_d2(q, pts + 3 * j), b);
                        }
                    }
                }
            }
            /* distance from q to the outside of the scanned block of cells */
            double m = INFINITY;
            int covers = 1;
            for (int a = 0; a < 3; a++) {
                int64_t c0 = c[a] - r, c1 = c[a] + r;
                if (c0 > 0) { m = fmin(m, (double)q[a] - (lo[a] + (double)c0 * h)); covers = 0; }
                if (c1 < dim[a] - 1) { m = fmin(m, lo[a] + (double)(c1 + 1) * h - (double)q[a]); covers = 0; }
            }
            if (covers) break;
            if (m > 0.0 && (double)b[2] < m * m * (1.0 - 1e-5)) break;
        }
        float s = b[0] + b[1];
        s = s + b[2];
        out[i] = s / 3.0f;
    }
    free(start);
    free(cellof);
    free(items);
}

/* ------------------------------------------------------------------------------------
 * Training sample points (train.py:34-61 sample_mesh_points), with the device's
 * declared generator: Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC 2011), counter =
 * (point index lo, hi, block, 0), key = (seed lo, seed hi).  Block 0 gives the cell
 * (floor(r64 * C / 2^64), r64 = word0:word1) and two uniforms (words 2, 3), block 1
 * word 0 the third; a uniform is (r >> 8) * 2^-24.  The three are sorted and their gaps
 * (u0, u1 - u0, u2 - u1, 1 - u2) weight the tetrahedron's vertices, summed left to right
 * in float32 with every operation rounded.
 * ------------------------------------------------------------------------------------ */
void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3], k0 = key[0], k1 = key[1];
    for (int r = 0; r < 10; r++) {
        if (r) { k0 += 0x9E3779B9u; k1 += 0xBB67AE85u; }
        uint64_t p0 = (uint64_t)0xD2511F53u * c0, p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0, n1 = (uint32_t)p1;
        uint32_t n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1, n3 = (uint32_t)p0;
        c0 = n0; c1 = n1; c2 = n2; c3 = n3;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

static inline float unit24f(uint32_t r) { return (float)(r >> 8) * 5.9604644775390625e-8f; }

void orc_tet_points(int64_t N, uint64_t seed, const float* pts, const int64_t* conn4, int64_t C, float* out,
                    int nthreads) {
    int nt = orc_nthreads(nthreads);
    const uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
#pragma omp parallel for num_threads(nt) schedule(static)
    for (int64_t t = 0; t < N; t++) {
        uint32_t ca[4] = {(uint32_t)t, (uint32_t)((uint64_t)t >> 32), 0u, 0u}, a[4];
        uint32_t cb[4] = {(uint32_t)t, (uint32_t)((uint64_t)t >> 32), 1u, 0u}, b[4];
        orc_philox4x32_10(ca, key, a);
        orc_philox4x32_10(cb, key, b);
        uint64_t r64 = ((uint64_t)a[0] << 32) | a[1];
        int64_t cell = (int64_t)(((unsigned __int128)r64 * (unsigned __int128)(uint64_t)C) >> 64);
        float u[3] = {unit24f(a[2]), unit24f(a[3]), unit24f(b[0])};
        for (int i = 1; i < 3; i++)
            for (int j = i; j > 0 && u[j] < u[j - 1]; j--) { float tmp = u[j]; u[j] = u[j - 1]; u[j - 1] = tmp; }
        float w[4] = {u[0], u[1] - u[0], u[2] - u[1], 1.0f - u[2]};
        const int64_t* cv = conn4 + 4 * cell;
        for (int ax = 0; ax < 3; ax++) {
            float s = w[0] * pts[3 * cv[0] + ax];
            s = s + w[1] * pts[3 * cv[1] + ax];
            s = s + w[2] * pts[3 * cv[2] + ax];
            s = s + w[3] * pts[3 * cv[3] + ax];
            out[3 * t + ax] = s;
        }
    }
}
