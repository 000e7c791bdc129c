/*
 * sp_oracle.h — CPU restatement of the reference's ePlace GP operators, used ONLY as the
 * checker of the CUDA path (tests, smoke check, CPU-baseline leg of the benchmark).
 * The product never links or calls it.
 *
 * Pinned by: the reference's own tests (test/test_poisson.cpp, test/test_density.cpp,
 * test/test_wirelength.cpp, test/test_hpwl.cpp) restated in tests/test_oracle.py, and by
 * bit-level comparison against the reference's own code built from its sources
 * (oracle/_ref, fixtures in tests/golden/).
 *
 * Arrays follow include/spgpu.h: node SoA in centre coordinates, grid maps row-major
 * data[x * dim + y].
 */
#ifndef SP_ORACLE_H_
#define SP_ORACLE_H_

#include <stdint.h>

#include "spgpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct spo_grid {
    int dim;
    float step_x, step_y, origin_x, origin_y, target_density;
    double movable_area_scaled; /* tau denominator */
} spo_grid;

/* BinGrid::initialize dimension/step/denominator (src/gp/bin_grid.cpp:64-107). */
int spo_grid_setup(const spg_db_view* db, float target_density, int bin_dim, spo_grid* g);
/* terminalDensity (bin_grid.cpp:115-137) and baseDensity (bin_grid.cpp:139-173). */
void spo_static_density(const spg_db_view* db, const spo_grid* g, float* terminal, float* base);

/* Footprint + charge weight of node i (bin_grid.cpp:22-62). Returns 0 when the node is
 * skipped (fixed or NI). */
int spo_footprint(const spg_db_view* db, const spo_grid* g, int i, int* bx0, int* bx1, int* by0,
                  int* by1, float* lx, float* ly, float* hx, float* hy, float* weight);

/* One bin's contribution overlap(bin, rect) * w exactly as bin_grid.cpp:220-229 computes it. */
float spo_bin_contribution(const spo_grid* g, int bx, int by, float lx, float ly, float hx,
                           float hy, float w);

/* BinGrid::accumulate with the reference's fixed 8-chunk float semantics
 * (bin_grid.cpp:191-251): bit-identical to the reference. */
void spo_accumulate_chunks(const spg_db_view* db, const spo_grid* g, int chunks, float* node,
                           float* filler);
/* The engine's deterministic 64-bit fixed-point accumulation: every contribution is
 * rounded to round(c * 2^shift) and summed exactly. */
void spo_accumulate_fixed(const spg_db_view* db, const spo_grid* g, int shift, int64_t* node,
                          int64_t* filler);
/* Fixed-point shift used for a design: the largest s <= 40 with total_charge * 2^s < 2^62. */
int spo_fixed_shift(const spg_db_view* db, const spo_grid* g);

/* BinGrid::overflow (bin_grid.cpp:265-285) over float maps, FP64. */
float spo_overflow(const spo_grid* g, const float* node, const float* terminal, const float* base);
/* rho = (node + filler + terminal + base) / binArea (bin_grid.cpp:253-259). */
void spo_rho(const spo_grid* g, const float* node, const float* filler, const float* terminal,
             const float* base, float* rho);

/* Poisson solve in FP64 (cpu_poisson.cpp:149-207 math, FFTW r2r definitions): inputs and
 * outputs double. */
void spo_poisson_f64(int nx, int ny, double step_x, double step_y, const double* rho, double* phi,
                     double* ex, double* ey);
/* Float-in/float-out wrapper (computes in FP64). */
void spo_poisson(int nx, int ny, float step_x, float step_y, const float* rho, float* phi,
                 float* ex, float* ey);

/* BinGrid::gatherForce (bin_grid.cpp:287-318): force = q*xi for all non-fixed nodes,
 * 2*total floats [x..., y...]. */
void spo_gather(const spg_db_view* db, const spo_grid* g, const float* fx, const float* fy,
                float* force);
/* BinGrid::totalCharge (bin_grid.cpp:320-338). */
double spo_total_charge(const spg_db_view* db, const spo_grid* g);

/* computeGamma (src/gp/wa_wirelength.cpp:18-29). */
float spo_gamma(float tau, float bin_step);
/* lambdaMultiplier (src/gp/lambda_schedule.h:22-25). */
float spo_lambda_mu(double delta_hpwl, double reference);

/* WaWirelength::compute (src/gp/wa_wirelength.cpp:46-180): returns WA length, grad over
 * num_movable as [x..., y...]. */
double spo_wa(const spg_db_view* db, float gamma, int ignore_net_degree, float* grad);
/* computeHPWL (src/db/hpwl.cpp:13-39). */
double spo_hpwl(const spg_db_view* db);

/* deterministicSum's fixed 64-chunk FP64 sum of a float array's values, squares or
 * absolute values (src/numeric/reduction.h:44-71). mode 0 = x, 1 = x*x, 2 = |x|. */
double spo_chunk_sum(const float* a, int64_t n, int mode);

#ifdef __cplusplus
}
#endif

#endif
