// Poisson solve on the bin grid as dense cosine-matrix contractions (sm_100a).
//
// Math (FFTW r2r definitions, src/numeric/cpu/cpu_poisson.cpp:1-40): with rho[x][y]
// (x slow, y fast), Cx[j][x] = cos(pi j (x+1/2)/nx), Cy[k][y] = cos(pi k (y+1/2)/ny),
// c_0 = 1, c_{j>0} = 2, u_j = pi j/(nx sx), v_k = pi k/(ny sy):
//   P    = (Cx rho Cy^T) / (nx ny (u_j^2 + v_k^2)),  P[0][0] = 0
//   phi  = Ax P Ay^T             Ax[x][j] = c_j cos(pi j (x+1/2)/nx)
//   xi_x = Sx P Ay^T             Sx[x][j] = 2 u_j sin(pi j (x+1/2)/nx)
//   xi_y = Ax P Sy^T             Sy[y][k] = 2 v_k sin(pi k (y+1/2)/ny)
// The RODFT01 index shift of the reference (cpu_poisson.cpp:182-206) is folded into the
// sine bases, so no reorder or sign pass is needed.
//
// Every contraction is written C[m][n] = sum_k A[m][k] B[n][k] (both operands K-major):
//   G1  T0t  (ny x nx)  = Cy        . rho^T          K = ny
//   G2  P    (nx x ny)  = Cx        . T0t^T  (x S)   K = nx   (spectral divide epilogue)
//   G3  T12t (2ny x nx) = [Ay; Sy]  . P^T            K = ny
//   G4  [phi; xi_x]     = [Ax; Sx]  . T1t^T          K = nx
//       xi_y            = Ax        . T2t^T          K = nx
// 14 nx ny max(nx,ny) flops for a square grid (2+2+4+4+2 M^3).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

namespace spg {

struct PoissonPlan {
    int nx = 0, ny = 0, batch_cap = 1;
    float step_x = 1.f, step_y = 1.f;
    int precision = 0;
    std::string name;
    // FP32 bases
    float *cy = nullptr, *cx = nullptr, *bcat = nullptr, *acat = nullptr, *scale = nullptr;
    // FP32 work (sized for batch_cap grids)
    float *t0t = nullptr, *p = nullptr, *t12t = nullptr;
    float* dc = nullptr;  // DC-split row means and sums

    // FP64 bases and work (the FP64 reference form)
    double *cy64 = nullptr, *cx64 = nullptr, *bcat64 = nullptr, *acat64 = nullptr, *scale64 = nullptr;
    double *rho64 = nullptr, *t0t64 = nullptr, *p64 = nullptr, *t12t64 = nullptr;

    // split-BF16 bases and work: hi and lo planes, stored [hi | lo] per matrix
    uint16_t *cy_s = nullptr, *cx_s = nullptr, *bcat_s = nullptr, *acat_s = nullptr;
    uint16_t *rho_s = nullptr, *t0t_s = nullptr, *p_s = nullptr, *t12t_s = nullptr;
    void* tc = nullptr;  // tensor-core launch state (poisson_tc.cu)
    std::vector<double> sin_x, sin_y;  // host sine tables, for new bin steps (set_steps)
    size_t bytes = 0;    // device memory held
    cudaStream_t stream = nullptr;  // the stream its buffers' frees are ordered on
    // a one-grid split-BF16 solve may run as one persistent launch (tc_fused_kernel). Its grid
    // barriers need all its CTAs resident at once, so it is only for a plan whose solves do not
    // run beside another such launch on the device; off unless the owner asks for it
    bool single_launch = false;
};

// Allocates bases and work buffers for up to batch_cap grids. precision: SPG_POISSON_*.
void poisson_plan_create(PoissonPlan& pl, int nx, int ny, float step_x, float step_y,
                         int precision, int batch_cap);
void poisson_plan_destroy(PoissonPlan& pl);
// New bin steps for an existing plan: the tables are rebuilt on the host and written into the
// plan's buffers on its stream (no allocation; the tensor maps stay valid).
void poisson_plan_set_steps(PoissonPlan& pl, float step_x, float step_y);
// Device solve of `batch` grids stored back to back.
// rho_split_ready (tensor-core plans, one grid): the caller already wrote rho's RhoOperand
// (tc_rho_operand), so the solve starts at its first GEMM
void poisson_solve(PoissonPlan& pl, int batch, const float* rho, float* phi, float* ex, float* ey,
                   cudaStream_t s, bool rho_split_ready = false);

// ---- FP32 SIMT GEMM "TN": C[m][n] = sum_k A[m*lda+k] * (B[n*ldb+k] - boff[n])
// (optionally * S[m][n]). Rows m >= split go to C2 (row m - split) so one launch can fill
// two outputs.
//
// DC split: a forward cosine contraction over data with a large mean accumulates long
// partial sums that cancel, and FP32 sequential accumulation then loses the small
// low-frequency coefficients the 1/(u^2+v^2) divide amplifies. Subtracting each B row's
// mean (boff) removes that component; since sum_k cos(pi j (k+1/2)/n) = 0 for j >= 1 only
// output row 0 (the DC row, whose basis row is all ones) changes, and it is restored
// exactly from the row sums.
template <typename T, typename TO>
struct GemmArgsT {
    const T* A;
    const T* B;
    TO* C;
    TO* C2;
    const T* S;
    int M, N, K, split;
    int64_t lda, ldb, ldc, lds;
    int64_t sA, sB, sC;  // per-batch strides (blockIdx.z)
    const T* boff = nullptr;  // per-B-row offset, batch stride sBoff
    int64_t sBoff = 0;
};
using GemmArgs = GemmArgsT<float, float>;

// Row statistics for the DC split: for each row r (of `rows`, length `cols` each, leading
// dimension ld) and each segment of `seg` columns, mean and sum (accumulated in FP64).
// Output index: segment * rows + r.
void row_stats(const float* a, int rows, int cols, int64_t ld, int seg, float* mean, float* sum,
               cudaStream_t s);
// C[row 0][n] = vals[n] (* scale[n] when scale is given), for `batch` outputs.
void set_row0(float* C, int64_t sC, int n, const float* vals, int64_t sv, const float* scale,
              int batch, cudaStream_t s);
void sgemm_tn(const GemmArgs& g, int batch, cudaStream_t s);

// ---- tensor-core path (poisson_tc.cu)
bool tc_supported(int nx, int ny);
// split-BF16 planes of the FP32 bases (given as the host tables the plan uploaded), work
// buffers and tensor maps
void tc_plan_create(PoissonPlan& pl, const std::vector<float>& cy, const std::vector<float>& cx,
                    const std::vector<float>& bcat, const std::vector<float>& acat);
void tc_plan_destroy(PoissonPlan& pl);
// The plan's device error flag (0, or SPG_E_CUDA after a tensor-core solve gave up a bounded
// pipeline wait), or nullptr for plans without tensor-core GEMMs.
const int* tc_error_flag(const PoissonPlan& pl);
// Where a one-grid tensor-core solve takes its first operand: the split BF16 planes of the
// density rows minus their means (hi plane, lo plane at + plane_stride, row r at r * ld) and
// the exact FP32 row sums. False for plans without tensor-core GEMMs.
struct RhoOperand {
    uint16_t* planes;
    int64_t plane_stride;
    int64_t ld;
    float* sums;
};
bool tc_rho_operand(const PoissonPlan& pl, RhoOperand* out);
// rewrite the split-BF16 planes of the step-dependent rows in place: Sy (rows ny..2ny of
// [Ay; Sy]) and Sx (rows nx..2nx of [Ax; Sx]); same buffers, same tensor maps
void tc_plan_refill_sines(PoissonPlan& pl, const std::vector<float>& sy_rows, const std::vector<float>& sx_rows);
// rho_split_ready: the caller already wrote the RhoOperand of rho (one grid)
void tc_solve(PoissonPlan& pl, int batch, const float* rho, float* phi, float* ex, float* ey,
              cudaStream_t s, bool rho_split_ready = false);

}  // namespace spg
