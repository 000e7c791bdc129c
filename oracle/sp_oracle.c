/*
 * sp_oracle.c — CPU restatement of the reference's ePlace GP operators.
 *
 * TEST INFRASTRUCTURE: the checker of the CUDA path. Only tests/, the smoke check and the
 * CPU-baseline leg of bench.py load it; the product never does.
 *
 * Each function cites the reference lines it restates. Float expressions are written in
 * the reference's evaluation order and built with -ffp-contract=off, so the float results
 * are bit-identical to the reference built the same way (checked by tests/test_oracle.py
 * against oracle/_ref and the fixtures in tests/golden/). The Poisson solve is computed
 * in FP64 from FFTW's published r2r definitions and is the accuracy reference for the
 * device solvers.
 */
#include "sp_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define KMAX_BIN_DIM 1024 /* bin_grid.cpp:18 */
#define KREDUCE_CHUNKS 64 /* reduction.h:24 */

static int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }
static float minf_(float a, float b) { return (b < a) ? b : a; } /* std::min */
static float maxf_(float a, float b) { return (a < b) ? b : a; } /* std::max */

/* overlapArea (src/db/geometry.h:35-39). */
static float overlap_area(float alx, float aly, float ahx, float ahy, float blx, float bly,
                          float bhx, float bhy) {
    const float dx = minf_(ahx, bhx) - maxf_(alx, blx);
    const float dy = minf_(ahy, bhy) - maxf_(aly, bly);
    return (dx > 0.f && dy > 0.f) ? dx * dy : 0.f;
}

static int is_fixed(const spg_db_view* db, int i) { return (db->node_flags[i] & SPG_F_FIXED) != 0; }
static int is_ni(const spg_db_view* db, int i) { return (db->node_flags[i] & SPG_F_NI) != 0; }
static int is_macro(const spg_db_view* db, int i) { return (db->node_flags[i] & SPG_F_MACRO) != 0; }
static int is_filler(const spg_db_view* db, int i) { return (db->node_flags[i] & SPG_F_FILLER) != 0; }

/* ------------------------------------------------------------------ grid setup */
int spo_grid_setup(const spg_db_view* db, float target_density, int bin_dim, spo_grid* g) {
    /* bin_grid.cpp:66-107 */
    g->target_density = target_density;
    g->origin_x = db->core_lx;
    g->origin_y = db->core_ly;
    double cell_area = 0.0, macro_area = 0.0;
    for (int i = 0; i < db->num_movable; ++i) {
        if (is_fixed(db, i) || is_ni(db, i)) continue;
        const double a = (double)db->node_w[i] * (double)db->node_h[i];
        if (is_macro(db, i)) macro_area += a;
        else cell_area += a;
    }
    g->movable_area_scaled = cell_area + macro_area * (double)target_density;
    int dim;
    if (bin_dim > 0) {
        dim = bin_dim < KMAX_BIN_DIM ? bin_dim : KMAX_BIN_DIM;
    } else {
        const double avg = (db->num_movable > 0) ? (cell_area + macro_area) / db->num_movable : 1.0;
        double ideal_bin = avg / target_density;
        if (ideal_bin < 1e-9) ideal_bin = 1e-9;
        const float cw = db->core_hx - db->core_lx, ch = db->core_hy - db->core_ly;
        const double core_area = (double)cw * (double)ch;
        const double ideal_count = core_area / ideal_bin;
        dim = 4;
        while (dim * 2 <= KMAX_BIN_DIM && (double)(dim * 2) * (dim * 2) <= ideal_count) dim *= 2;
    }
    g->dim = dim;
    g->step_x = (db->core_hx - db->core_lx) / (float)dim;
    g->step_y = (db->core_hy - db->core_ly) / (float)dim;
    return 0;
}

typedef struct {
    float ly, hy, lx, hx;
} row_rect;

static int cmp_row(const void* a, const void* b) {
    const float x = ((const row_rect*)a)->ly, y = ((const row_rect*)b)->ly;
    return (x < y) ? -1 : (x > y) ? 1 : 0;
}

void spo_static_density(const spg_db_view* db, const spo_grid* g, float* terminal, float* base) {
    const int dim = g->dim;
    const size_t n = (size_t)dim * dim;
    memset(terminal, 0, n * sizeof(float));
    /* terminalDensity: bin_grid.cpp:120-137 */
    for (int i = 0; i < db->num_nodes; ++i) {
        if (!is_fixed(db, i)) continue;
        if (is_ni(db, i)) continue;
        const float blx0 = db->node_x[i] - 0.5f * db->node_w[i];
        const float bly0 = db->node_y[i] - 0.5f * db->node_h[i];
        const float bhx0 = db->node_x[i] + 0.5f * db->node_w[i];
        const float bhy0 = db->node_y[i] + 0.5f * db->node_h[i];
        const int bx0 = clampi((int)((blx0 - g->origin_x) / g->step_x), 0, dim - 1);
        const int bx1 = clampi((int)((bhx0 - g->origin_x) / g->step_x), 0, dim - 1);
        const int by0 = clampi((int)((bly0 - g->origin_y) / g->step_y), 0, dim - 1);
        const int by1 = clampi((int)((bhy0 - g->origin_y) / g->step_y), 0, dim - 1);
        for (int bx = bx0; bx <= bx1; ++bx) {
            const float blx = g->origin_x + bx * g->step_x;
            for (int by = by0; by <= by1; ++by) {
                const float bly = g->origin_y + by * g->step_y;
                terminal[(size_t)bx * dim + by] +=
                    g->target_density * overlap_area(blx, bly, blx + g->step_x, bly + g->step_y,
                                                     blx0, bly0, bhx0, bhy0);
            }
        }
    }
    /* baseDensity: bin_grid.cpp:144-173 (rows sorted by ly, binary search on hy) */
    const int nr = db->num_rows;
    row_rect* rows = (row_rect*)malloc((size_t)(nr > 0 ? nr : 1) * sizeof(row_rect));
    for (int r = 0; r < nr; ++r) {
        rows[r].ly = db->row_ly[r];
        rows[r].hy = db->row_ly[r] + db->row_height[r];
        rows[r].lx = db->row_lx[r];
        rows[r].hx = db->row_lx[r] + db->row_step[r] * (float)db->row_num_sites[r];
    }
    qsort(rows, (size_t)nr, sizeof(row_rect), cmp_row);
    for (int by = 0; by < dim; ++by) {
        const float bly = g->origin_y + by * g->step_y;
        const float bhy = bly + g->step_y;
        size_t lo = 0, hi = (size_t)nr;
        while (lo < hi) {
            const size_t mid = (lo + hi) / 2;
            if (rows[mid].hy <= bly) lo = mid + 1;
            else hi = mid;
        }
        for (int bx = 0; bx < dim; ++bx) {
            const float blx = g->origin_x + bx * g->step_x;
            const float bhx = blx + g->step_x;
            float covered = 0.f;
            for (size_t t = lo; t < (size_t)nr; ++t) {
                if (rows[t].ly >= bhy) break;
                covered += overlap_area(blx, bly, bhx, bhy, rows[t].lx, rows[t].ly, rows[t].hx,
                                        rows[t].hy);
            }
            const float area = (bhx - blx) * (bhy - bly);
            const float free_area = maxf_(0.f, area - covered);
            base[(size_t)bx * dim + by] = g->target_density * free_area;
        }
    }
    free(rows);
}

/* ------------------------------------------------------------------ footprint */
int spo_footprint(const spg_db_view* db, const spo_grid* g, int i, int* bx0, int* bx1, int* by0,
                  int* by1, float* lxo, float* lyo, float* hxo, float* hyo, float* weight) {
    if (is_fixed(db, i) || is_ni(db, i)) return 0;
    /* footprintOf: bin_grid.cpp:22-54 */
    float lx = db->node_x[i] - 0.5f * db->node_w[i], hx = db->node_x[i] + 0.5f * db->node_w[i];
    float ly = db->node_y[i] - 0.5f * db->node_h[i], hy = db->node_y[i] + 0.5f * db->node_h[i];
    float sx = 1.f, sy = 1.f;
    const float w = db->node_w[i], h = db->node_h[i];
    if (w < g->step_x) {
        sx = w / g->step_x;
        const float cx = db->node_x[i];
        lx = cx - 0.5f * g->step_x;
        hx = cx + 0.5f * g->step_x;
    }
    if (h < g->step_y) {
        sy = h / g->step_y;
        const float cy = db->node_y[i];
        ly = cy - 0.5f * g->step_y;
        hy = cy + 0.5f * g->step_y;
    }
    const float scale = sx * sy;
    const int dim = g->dim;
    *bx0 = clampi((int)((lx - g->origin_x) / g->step_x), 0, dim - 1);
    *bx1 = clampi((int)((hx - g->origin_x) / g->step_x), 0, dim - 1);
    *by0 = clampi((int)((ly - g->origin_y) / g->step_y), 0, dim - 1);
    *by1 = clampi((int)((hy - g->origin_y) / g->step_y), 0, dim - 1);
    *lxo = lx;
    *lyo = ly;
    *hxo = hx;
    *hyo = hy;
    /* chargeWeight: bin_grid.cpp:56-62 */
    if (is_filler(db, i)) *weight = scale;
    else if (is_macro(db, i)) *weight = scale * g->target_density;
    else *weight = scale;
    return 1;
}

float spo_bin_contribution(const spo_grid* g, int bx, int by, float lx, float ly, float hx,
                           float hy, float w) {
    const float blx = g->origin_x + bx * g->step_x;
    const float bly = g->origin_y + by * g->step_y;
    return overlap_area(blx, bly, blx + g->step_x, bly + g->step_y, lx, ly, hx, hy) * w;
}

void spo_accumulate_chunks(const spg_db_view* db, const spo_grid* g, int chunks, float* node,
                           float* filler) {
    /* bin_grid.cpp:191-251 */
    const int dim = g->dim;
    const size_t n = (size_t)dim * dim;
    const int nc = chunks > 0 ? chunks : 8;
    const int total = db->num_nodes + db->num_fillers;
    float* ln = (float*)calloc(n * (size_t)nc, sizeof(float));
    float* lf = (float*)calloc(n * (size_t)nc, sizeof(float));
    for (int c = 0; c < nc; ++c) {
        const int lo = (int)((int64_t)total * c / nc);
        const int hi = (int)((int64_t)total * (c + 1) / nc);
        float* cn = ln + (size_t)c * n;
        float* cf = lf + (size_t)c * n;
        for (int i = lo; i < hi; ++i) {
            int bx0, bx1, by0, by1;
            float lx, ly, hx, hy, w;
            if (!spo_footprint(db, g, i, &bx0, &bx1, &by0, &by1, &lx, &ly, &hx, &hy, &w)) continue;
            const int fil = is_filler(db, i);
            for (int bx = bx0; bx <= bx1; ++bx)
                for (int by = by0; by <= by1; ++by) {
                    const float ov = spo_bin_contribution(g, bx, by, lx, ly, hx, hy, w);
                    if (ov <= 0.f) continue;
                    const size_t idx = (size_t)bx * dim + by;
                    if (fil) cf[idx] += ov;
                    else cn[idx] += ov;
                }
        }
    }
    for (size_t b = 0; b < n; ++b) {
        float sn = 0.f, sf = 0.f;
        for (int c = 0; c < nc; ++c) {
            sn += ln[(size_t)c * n + b];
            sf += lf[(size_t)c * n + b];
        }
        node[b] = sn;
        filler[b] = sf;
    }
    free(ln);
    free(lf);
}

int spo_fixed_shift(const spg_db_view* db, const spo_grid* g) {
    const int total = db->num_nodes + db->num_fillers;
    const double tw = g->target_density > 1.f ? (double)g->target_density : 1.0;
    /* four partial sums, node i into acc[i % 4], combined as (0 + 1) + (2 + 3) */
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    for (int i = 0; i < total; ++i) {
        if (is_fixed(db, i) || is_ni(db, i)) continue;
        acc[i & 3] += (double)db->node_w[i] * (double)db->node_h[i];
    }
    double bound = (acc[0] + acc[1]) + (acc[2] + acc[3]);
    bound *= tw;
    if (!(bound > 0.0)) return 40;
    int e = 0;
    frexp(bound, &e); /* bound < 2^e */
    const int s = 62 - e;
    return s < 40 ? s : 40;
}

void spo_accumulate_fixed(const spg_db_view* db, const spo_grid* g, int shift, int64_t* node,
                          int64_t* filler) {
    const int dim = g->dim;
    const size_t n = (size_t)dim * dim;
    memset(node, 0, n * sizeof(int64_t));
    memset(filler, 0, n * sizeof(int64_t));
    const double scale = ldexp(1.0, shift);
    const int total = db->num_nodes + db->num_fillers;
    for (int i = 0; i < total; ++i) {
        int bx0, bx1, by0, by1;
        float lx, ly, hx, hy, w;
        if (!spo_footprint(db, g, i, &bx0, &bx1, &by0, &by1, &lx, &ly, &hx, &hy, &w)) continue;
        int64_t* dst = is_filler(db, i) ? filler : node;
        for (int bx = bx0; bx <= bx1; ++bx)
            for (int by = by0; by <= by1; ++by) {
                const float ov = spo_bin_contribution(g, bx, by, lx, ly, hx, hy, w);
                if (ov <= 0.f) continue;
                dst[(size_t)bx * dim + by] += (int64_t)llrint((double)ov * scale);
            }
    }
}

/* ------------------------------------------------------------------ reductions */
/* deterministicSum: reduction.h:28-31 chunking, :44-71 sum */
static double chunk_sum_fn(int64_t n, double (*f)(int64_t, const void*), const void* ctx) {
    if (n <= 0) return 0.0;
    double partial[KREDUCE_CHUNKS];
    for (int c = 0; c < KREDUCE_CHUNKS; ++c) {
        const int64_t lo = n * c / KREDUCE_CHUNKS, hi = n * (c + 1) / KREDUCE_CHUNKS;
        double s = 0.0;
        for (int64_t i = lo; i < hi; ++i) s += f(i, ctx);
        partial[c] = s;
    }
    double total = 0.0;
    for (int c = 0; c < KREDUCE_CHUNKS; ++c) total += partial[c];
    return total;
}

typedef struct {
    const float* a;
    int mode;
} arr_ctx;

static double arr_term(int64_t i, const void* p) {
    const arr_ctx* c = (const arr_ctx*)p;
    const double v = (double)c->a[i];
    return c->mode == 0 ? v : (c->mode == 1 ? v * v : fabs(v));
}

double spo_chunk_sum(const float* a, int64_t n, int mode) {
    arr_ctx c = {a, mode};
    return chunk_sum_fn(n, arr_term, &c);
}

typedef struct {
    const spo_grid* g;
    const float *node, *terminal, *base;
    double area, target;
} ovf_ctx;

static double ovf_term(int64_t b, const void* p) {
    const ovf_ctx* c = (const ovf_ctx*)p;
    /* bin_grid.cpp:276-283 */
    const double rho = ((double)c->node[b] + c->terminal[b] + c->base[b]) / c->area;
    const double d = rho - c->target;
    return d > 0.0 ? d * c->area : 0.0;
}

float spo_overflow(const spo_grid* g, const float* node, const float* terminal, const float* base) {
    /* bin_grid.cpp:265-285 */
    if (g->movable_area_scaled <= 0.0) return 0.f;
    ovf_ctx c = {g, node, terminal, base, (double)(g->step_x * g->step_y), (double)g->target_density};
    const double over = chunk_sum_fn((int64_t)g->dim * g->dim, ovf_term, &c);
    return (float)(over / g->movable_area_scaled);
}

void spo_rho(const spo_grid* g, const float* node, const float* filler, const float* terminal,
             const float* base, float* rho) {
    /* bin_grid.cpp:253-259 */
    const float inv_area = 1.0f / (g->step_x * g->step_y);
    const size_t n = (size_t)g->dim * g->dim;
    for (size_t b = 0; b < n; ++b) rho[b] = (node[b] + filler[b] + terminal[b] + base[b]) * inv_area;
}

/* ------------------------------------------------------------------ FP64 r2r transforms */
/* FFTW definitions (cpu_poisson.cpp:8-37):
 *   REDFT10: Y_k = 2 sum_j X_j cos(pi k (j+1/2)/n)
 *   REDFT01: Y_j = X_0 + 2 sum_{k>=1} X_k cos(pi k (j+1/2)/n)
 *   RODFT01: Y_j = (-1)^j X_{n-1} + 2 sum_{k=0}^{n-2} X_k sin(pi (k+1)(j+1/2)/n)
 * Power-of-two n uses a Makhoul reordering onto a radix-2 complex FFT; other n are summed
 * directly. */
typedef struct {
    double re, im;
} cplx;

static void fft_d(cplx* a, int n, int inverse) {
    for (int i = 1, j = 0; i < n; ++i) {
        int bit = n >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) {
            cplx t = a[i];
            a[i] = a[j];
            a[j] = t;
        }
    }
    for (int len = 2; len <= n; len <<= 1) {
        const double ang = (inverse ? 2.0 : -2.0) * M_PI / len;
        for (int s = 0; s < n; s += len) {
            for (int k = 0; k < len / 2; ++k) {
                const double wr = cos(ang * k), wi = sin(ang * k);
                cplx* u = &a[s + k];
                cplx* v = &a[s + k + len / 2];
                const double tr = v->re * wr - v->im * wi, ti = v->re * wi + v->im * wr;
                v->re = u->re - tr;
                v->im = u->im - ti;
                u->re += tr;
                u->im += ti;
            }
        }
    }
}

static int pow2(int n) { return n >= 4 && (n & (n - 1)) == 0; }

static void redft10_d(const double* in, double* out, int n, cplx* w) {
    if (!pow2(n)) {
        for (int k = 0; k < n; ++k) {
            double s = 0.0;
            for (int j = 0; j < n; ++j) s += in[j] * cos(M_PI * k * (j + 0.5) / n);
            out[k] = 2.0 * s;
        }
        return;
    }
    for (int j = 0; j < n / 2; ++j) {
        w[j].re = in[2 * j];
        w[j].im = 0.0;
        w[n - 1 - j].re = in[2 * j + 1];
        w[n - 1 - j].im = 0.0;
    }
    fft_d(w, n, 0);
    for (int k = 0; k < n; ++k) {
        const double a = -M_PI * k / (2.0 * n);
        out[k] = 2.0 * (w[k].re * cos(a) - w[k].im * sin(a));
    }
}

static void redft01_d(const double* in, double* out, int n, cplx* w) {
    if (!pow2(n)) {
        for (int j = 0; j < n; ++j) {
            double s = 0.0;
            for (int k = 1; k < n; ++k) s += in[k] * cos(M_PI * k * (j + 0.5) / n);
            out[j] = in[0] + 2.0 * s;
        }
        return;
    }
    w[0].re = in[0];
    w[0].im = 0.0;
    for (int k = 1; k < n; ++k) {
        const double a = M_PI * k / (2.0 * n);
        const double xr = in[k], xi = -in[n - k];
        w[k].re = xr * cos(a) - xi * sin(a);
        w[k].im = xr * sin(a) + xi * cos(a);
    }
    fft_d(w, n, 1);
    for (int m = 0; m < n / 2; ++m) {
        out[2 * m] = w[m].re;
        out[2 * m + 1] = w[n - 1 - m].re;
    }
}

static void rodft01_d(const double* in, double* out, int n, cplx* w, double* tmp) {
    for (int k = 0; k < n; ++k) tmp[k] = in[n - 1 - k];
    redft01_d(tmp, out, n, w);
    for (int j = 1; j < n; j += 2) out[j] = -out[j];
}

enum { R10, R01, O01 };

static void apply_d(int kind, const double* in, double* out, int n, cplx* w, double* tmp) {
    if (kind == R10) redft10_d(in, out, n, w);
    else if (kind == R01) redft01_d(in, out, n, w);
    else rodft01_d(in, out, n, w, tmp);
}

/* 2-D r2r with kind0 along x (slow axis) and kind1 along y (fast axis). */
static void r2r2d_d(int nx, int ny, const double* in, double* out, int k0, int k1) {
    const int m = nx > ny ? nx : ny;
    double* mid = (double*)malloc((size_t)nx * ny * sizeof(double));
    cplx* w = (cplx*)malloc((size_t)m * sizeof(cplx));
    double* tmp = (double*)malloc((size_t)m * sizeof(double));
    double* col = (double*)malloc((size_t)m * sizeof(double));
    double* res = (double*)malloc((size_t)m * sizeof(double));
    for (int x = 0; x < nx; ++x) apply_d(k1, in + (size_t)x * ny, mid + (size_t)x * ny, ny, w, tmp);
    for (int y = 0; y < ny; ++y) {
        for (int x = 0; x < nx; ++x) col[x] = mid[(size_t)x * ny + y];
        apply_d(k0, col, res, nx, w, tmp);
        for (int x = 0; x < nx; ++x) out[(size_t)x * ny + y] = res[x];
    }
    free(mid);
    free(w);
    free(tmp);
    free(col);
    free(res);
}

void spo_poisson_f64(int nx, int ny, double sx, double sy, const double* rho, double* phi,
                     double* ex, double* ey) {
    /* cpu_poisson.cpp:149-207 */
    const size_t n = (size_t)nx * ny;
    double* spec = (double*)malloc(n * sizeof(double));
    double* work = (double*)malloc(n * sizeof(double));
    r2r2d_d(nx, ny, rho, spec, R10, R10);
    const double inv_norm = 1.0 / (4.0 * nx * (double)ny);
    for (int j = 0; j < nx; ++j) {
        const double u = M_PI * j / (nx * sx);
        for (int k = 0; k < ny; ++k) {
            const double v = M_PI * k / (ny * sy);
            const double den = u * u + v * v;
            spec[(size_t)j * ny + k] = den > 0.0 ? spec[(size_t)j * ny + k] * inv_norm / den : 0.0;
        }
    }
    r2r2d_d(nx, ny, spec, phi, R01, R01);
    for (int j = 0; j < nx; ++j) {
        double* dst = work + (size_t)j * ny;
        if (j == nx - 1) {
            for (int k = 0; k < ny; ++k) dst[k] = 0.0;
        } else {
            const double u = M_PI * (j + 1) / (nx * sx);
            for (int k = 0; k < ny; ++k) dst[k] = spec[(size_t)(j + 1) * ny + k] * u;
        }
    }
    r2r2d_d(nx, ny, work, ex, O01, R01);
    for (int j = 0; j < nx; ++j) {
        double* dst = work + (size_t)j * ny;
        for (int k = 0; k < ny - 1; ++k) dst[k] = spec[(size_t)j * ny + k + 1] * (M_PI * (k + 1) / (ny * sy));
        dst[ny - 1] = 0.0;
    }
    r2r2d_d(nx, ny, work, ey, R01, O01);
    free(spec);
    free(work);
}

void spo_poisson(int nx, int ny, float sx, float sy, const float* rho, float* phi, float* ex,
                 float* ey) {
    const size_t n = (size_t)nx * ny;
    double* b = (double*)malloc(4 * n * sizeof(double));
    for (size_t i = 0; i < n; ++i) b[i] = rho[i];
    spo_poisson_f64(nx, ny, sx, sy, b, b + n, b + 2 * n, b + 3 * n);
    for (size_t i = 0; i < n; ++i) {
        phi[i] = (float)b[n + i];
        ex[i] = (float)b[2 * n + i];
        ey[i] = (float)b[3 * n + i];
    }
    free(b);
}

/* ------------------------------------------------------------------ gather */
void spo_gather(const spg_db_view* db, const spo_grid* g, const float* fx, const float* fy,
                float* force) {
    /* bin_grid.cpp:287-318 */
    const int total = db->num_nodes + db->num_fillers;
    memset(force, 0, 2 * (size_t)total * sizeof(float));
    for (int i = 0; i < total; ++i) {
        int bx0, bx1, by0, by1;
        float lx, ly, hx, hy, w;
        if (!spo_footprint(db, g, i, &bx0, &bx1, &by0, &by1, &lx, &ly, &hx, &hy, &w)) continue;
        float ax = 0.f, ay = 0.f;
        for (int bx = bx0; bx <= bx1; ++bx)
            for (int by = by0; by <= by1; ++by) {
                const float q = spo_bin_contribution(g, bx, by, lx, ly, hx, hy, w);
                if (q <= 0.f) continue;
                const size_t idx = (size_t)bx * g->dim + by;
                ax += q * fx[idx];
                ay += q * fy[idx];
            }
        force[i] = ax;
        force[total + i] = ay;
    }
}

double spo_total_charge(const spg_db_view* db, const spo_grid* g) {
    /* bin_grid.cpp:320-338 */
    const int total = db->num_nodes + db->num_fillers;
    double sum = 0.0;
    for (int i = 0; i < total; ++i) {
        int bx0, bx1, by0, by1;
        float lx, ly, hx, hy, w;
        if (!spo_footprint(db, g, i, &bx0, &bx1, &by0, &by1, &lx, &ly, &hx, &hy, &w)) continue;
        for (int bx = bx0; bx <= bx1; ++bx)
            for (int by = by0; by <= by1; ++by)
                sum += (double)spo_bin_contribution(g, bx, by, lx, ly, hx, hy, w);
    }
    return sum;
}

/* ------------------------------------------------------------------ schedules */
float spo_gamma(float tau, float bin_step) {
    /* wa_wirelength.cpp:18-29 */
    float gamma = 8.0f * bin_step;
    if (tau > 1.0f) gamma *= 10.0f;
    else if (tau < 0.1f) gamma *= 0.1f;
    else gamma *= powf(10.0f, (20.0f / 9.0f) * (tau - 0.1f) - 1.0f);
    return gamma > 1e-4f ? gamma : 1e-4f;
}

float spo_lambda_mu(double delta_hpwl, double reference) {
    /* lambda_schedule.h:22-25 */
    const double mu = pow(1.1, -delta_hpwl / reference + 1.0);
    return (float)(mu < 0.95 ? 0.95 : (mu > 1.05 ? 1.05 : mu));
}

/* ------------------------------------------------------------------ WA and HPWL */
static float pin_x(const spg_db_view* db, int p) { return db->node_x[db->pin2node[p]] + db->pin_offset_x[p]; }
static float pin_y(const spg_db_view* db, int p) { return db->node_y[db->pin2node[p]] + db->pin_offset_y[p]; }

typedef struct {
    const spg_db_view* db;
    float inv_g;
    int ignore;
    float *bpx, *bnx, *cpx, *cnx, *bpy, *bny, *cpy, *cny, *mxx, *mnx, *mxy, *mny;
    float *epx, *enx, *epy, *eny;
} wa_ctx;

static double wa_net(int64_t kk, const void* p) {
    /* wa_wirelength.cpp:74-126 */
    const wa_ctx* c = (const wa_ctx*)p;
    const spg_db_view* db = c->db;
    const int k = (int)kk;
    const int b = db->net2pin_start[k], e = db->net2pin_start[k + 1];
    const int deg = e - b;
    if (deg < 2 || deg > c->ignore) {
        c->bpx[k] = 0.f;
        c->bpy[k] = 0.f;
        return 0.0;
    }
    float mxX = -FLT_MAX, mnX = FLT_MAX, mxY = -FLT_MAX, mnY = FLT_MAX;
    for (int t = b; t < e; ++t) {
        const int q = db->flat_net2pin[t];
        const float px = pin_x(db, q), py = pin_y(db, q);
        mxX = maxf_(mxX, px);
        mnX = minf_(mnX, px);
        mxY = maxf_(mxY, py);
        mnY = minf_(mnY, py);
    }
    c->mxx[k] = mxX;
    c->mnx[k] = mnX;
    c->mxy[k] = mxY;
    c->mny[k] = mnY;
    float bpx = 0.f, bnx = 0.f, cpx = 0.f, cnx = 0.f, bpy = 0.f, bny = 0.f, cpy = 0.f, cny = 0.f;
    const float invG = c->inv_g;
    for (int t = b; t < e; ++t) {
        const int q = db->flat_net2pin[t];
        const float dxp = pin_x(db, q) - mxX;
        const float dxn = pin_x(db, q) - mnX;
        const float ap = expf(dxp * invG);
        const float an = expf(-dxn * invG);
        c->epx[q] = ap;
        c->enx[q] = an;
        bpx += ap;
        cpx += dxp * ap;
        bnx += an;
        cnx += dxn * an;
        const float dyp = pin_y(db, q) - mxY;
        const float dyn = pin_y(db, q) - mnY;
        const float bp = expf(dyp * invG);
        const float bn = expf(-dyn * invG);
        c->epy[q] = bp;
        c->eny[q] = bn;
        bpy += bp;
        cpy += dyp * bp;
        bny += bn;
        cny += dyn * bn;
    }
    c->bpx[k] = bpx;
    c->cpx[k] = cpx;
    c->bnx[k] = bnx;
    c->cnx[k] = cnx;
    c->bpy[k] = bpy;
    c->cpy[k] = cpy;
    c->bny[k] = bny;
    c->cny[k] = cny;
    return (double)((mxX - mnX) + cpx / bpx - cnx / bnx) + (double)((mxY - mnY) + cpy / bpy - cny / bny);
}

double spo_wa(const spg_db_view* db, float gamma, int ignore_net_degree, float* grad) {
    const int nn = db->num_nets, np = db->num_pins, nm = db->num_movable;
    const float g = gamma > 1e-4f ? gamma : 1e-4f;
    wa_ctx c;
    c.db = db;
    c.inv_g = 1.0f / g;
    c.ignore = ignore_net_degree;
    float* buf = (float*)calloc((size_t)12 * (nn > 0 ? nn : 1) + (size_t)4 * (np > 0 ? np : 1), sizeof(float));
    float** nets[12] = {&c.bpx, &c.bnx, &c.cpx, &c.cnx, &c.bpy, &c.bny, &c.cpy, &c.cny, &c.mxx, &c.mnx, &c.mxy, &c.mny};
    for (int t = 0; t < 12; ++t) *nets[t] = buf + (size_t)t * (nn > 0 ? nn : 1);
    float* pb = buf + (size_t)12 * (nn > 0 ? nn : 1);
    c.epx = pb;
    c.enx = pb + (np > 0 ? np : 1);
    c.epy = pb + 2 * (size_t)(np > 0 ? np : 1);
    c.eny = pb + 3 * (size_t)(np > 0 ? np : 1);
    const double wl = chunk_sum_fn(nn, wa_net, &c);
    const float invG = c.inv_g;
    /* pass 2: wa_wirelength.cpp:137-179 */
    for (int i = 0; i < nm; ++i) {
        float gx = 0.f, gy = 0.f;
        for (int t = db->node2pin_start[i]; t < db->node2pin_start[i + 1]; ++t) {
            const int p = db->flat_node2pin[t];
            const int k = db->pin2net[p];
            if (k < 0) continue;
            if (c.bpx[k] <= 0.f) continue;
            {
                const float bp = c.bpx[k], bn = c.bnx[k], cp = c.cpx[k], cn = c.cnx[k];
                const float ap = c.epx[p], an = c.enx[p];
                const float dp = pin_x(db, p) - c.mxx[k];
                const float dn = pin_x(db, p) - c.mnx[k];
                const float tmax = ap * (bp + (dp * bp - cp) * invG) / (bp * bp);
                const float tmin = an * (bn + (cn - dn * bn) * invG) / (bn * bn);
                gx += tmax - tmin;
            }
            {
                const float bp = c.bpy[k], bn = c.bny[k], cp = c.cpy[k], cn = c.cny[k];
                const float ap = c.epy[p], an = c.eny[p];
                const float dp = pin_y(db, p) - c.mxy[k];
                const float dn = pin_y(db, p) - c.mny[k];
                const float tmax = ap * (bp + (dp * bp - cp) * invG) / (bp * bp);
                const float tmin = an * (bn + (cn - dn * bn) * invG) / (bn * bn);
                gy += tmax - tmin;
            }
        }
        grad[i] = gx;
        grad[nm + i] = gy;
    }
    free(buf);
    return wl;
}

static double hpwl_net(int64_t kk, const void* p) {
    /* hpwl.cpp:18-32 */
    const spg_db_view* db = (const spg_db_view*)p;
    const int k = (int)kk;
    const int b = db->net2pin_start[k], e = db->net2pin_start[k + 1];
    if (e - b < 2) return 0.0;
    float lox = FLT_MAX, hix = -FLT_MAX, loy = FLT_MAX, hiy = -FLT_MAX;
    for (int t = b; t < e; ++t) {
        const int q = db->flat_net2pin[t];
        const float px = pin_x(db, q), py = pin_y(db, q);
        lox = minf_(lox, px);
        hix = maxf_(hix, px);
        loy = minf_(loy, py);
        hiy = maxf_(hiy, py);
    }
    return (double)(hix - lox) + (double)(hiy - loy);
}

double spo_hpwl(const spg_db_view* db) { return chunk_sum_fn(db->num_nets, hpwl_net, db); }
