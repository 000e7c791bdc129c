// Poisson plan, the plain-FP32 contraction path, and the solve driver.
// The math and the GEMM chain are described in poisson.h.
//
// The FP32 path is a register-tiled SIMT SGEMM (64x64 tile, 4x4 per thread, BK 16,
// register prefetch of the next K slab). It is the "plain FP32 GPU form" the split-BF16
// tensor-core path (poisson_tc.cu) is measured against, and the exact-enough reference
// for the parity tests at 1e-5. The FP64 path runs the same kernel in double: the accuracy
// reference of the precision study (potential, field and final HPWL against FP32 and
// split-BF16), not a production form.
#include <cmath>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "poisson.h"

namespace spg {

namespace {

constexpr int BM = 64, BN = 64, BK = 16, NT = 256;

// C[m][n] = sum_k A[m][k] (B[n][k] - boff[n]) (* S[m][n]) in T, stored as TO. The float4 load
// path serves the FP32 form; the FP64 form loads scalars.
template <typename T, typename TO>
__global__ void __launch_bounds__(NT) gemm_tn_kernel(GemmArgsT<T, TO> g, int vec_ok) {
    pdl_wait();
    pdl_trigger();
    __shared__ T As[BK][BM + 4];
    __shared__ T Bs[BK][BN + 4];
    const int z = blockIdx.z;
    const T* A = g.A + z * g.sA;
    const T* B = g.B + z * g.sB;
    const T* boff = g.boff ? g.boff + z * g.sBoff : nullptr;
    const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
    const int tid = threadIdx.x;
    const int tx = tid & 15, ty = tid >> 4;
    const int lr = tid >> 2, lk = (tid & 3) * 4;  // loader: row, k offset
    T acc[4][4] = {};
    T ra[4], rb[4];

    auto load = [&](int k0) {
        const int am = m0 + lr, bn = n0 + lr, k = k0 + lk;
        bool done = false;
        if constexpr (sizeof(T) == 4) {
            if (vec_ok && k + 3 < g.K) {
                if (am < g.M) {
                    const float4 v = *reinterpret_cast<const float4*>(A + am * g.lda + k);
                    ra[0] = v.x; ra[1] = v.y; ra[2] = v.z; ra[3] = v.w;
                } else {
                    ra[0] = ra[1] = ra[2] = ra[3] = T(0);
                }
                if (bn < g.N) {
                    const float4 v = *reinterpret_cast<const float4*>(B + bn * g.ldb + k);
                    rb[0] = v.x; rb[1] = v.y; rb[2] = v.z; rb[3] = v.w;
                } else {
                    rb[0] = rb[1] = rb[2] = rb[3] = T(0);
                }
                done = true;
            }
        }
        if (!done) {
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                ra[i] = (am < g.M && k + i < g.K) ? A[am * g.lda + k + i] : T(0);
                rb[i] = (bn < g.N && k + i < g.K) ? B[bn * g.ldb + k + i] : T(0);
            }
        }
        if (boff && bn < g.N) {  // DC split: B row minus its mean
            const T o = boff[bn];
#pragma unroll
            for (int i = 0; i < 4; ++i) rb[i] = (k + i < g.K) ? rb[i] - o : T(0);
        }
    };

    load(0);
    for (int k0 = 0; k0 < g.K; k0 += BK) {
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            As[lk + i][lr] = ra[i];
            Bs[lk + i][lr] = rb[i];
        }
        __syncthreads();
        if (k0 + BK < g.K) load(k0 + BK);
#pragma unroll
        for (int kk = 0; kk < BK; ++kk) {
            T av[4], bv[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                av[i] = As[kk][ty * 4 + i];
                bv[i] = Bs[kk][tx * 4 + i];
            }
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][j] = fma(av[i], bv[j], acc[i][j]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int m = m0 + ty * 4 + i;
        if (m >= g.M) continue;
        TO* crow = (m < g.split) ? g.C + z * g.sC + m * g.ldc : g.C2 + z * g.sC + (m - g.split) * g.ldc;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int n = n0 + tx * 4 + j;
            if (n >= g.N) continue;
            T v = acc[i][j];
            if (g.S) v *= g.S[m * g.lds + n];
            crow[n] = static_cast<TO>(v);
        }
    }
}

// FP32 -> FP64 copy of the density (the FP64 form's B operand of G1).
__global__ void widen_kernel(const float* src, double* dst, int64_t n) {
    pdl_wait();
    pdl_trigger();
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x)
        dst[i] = static_cast<double>(src[i]);
}

// One warp per (row, segment): FP64 sum of `seg` contiguous floats, fixed shuffle tree.
__global__ void row_stats_kernel(const float* a, int rows, int nseg, int64_t ld, int seg,
                                 float* mean, float* sum) {
    pdl_wait();
    pdl_trigger();
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (w >= rows * nseg) return;
    const int r = w % rows, sg = w / rows;
    const float* p = a + r * ld + static_cast<int64_t>(sg) * seg;
    double v = 0.0;
    for (int i = lane; i < seg; i += 32) v += static_cast<double>(p[i]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) {
        mean[w] = static_cast<float>(v / seg);
        sum[w] = static_cast<float>(v);
    }
}

__global__ void set_row0_kernel(float* C, int64_t sC, int n, const float* vals, int64_t sv,
                                const float* scale) {
    pdl_wait();
    pdl_trigger();
    const int z = blockIdx.y;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float v = vals[z * sv + i];
        if (scale) v *= scale[i];
        C[z * sC + i] = v;
    }
}

// Double-precision basis tables, rounded once to float.
double cospi_ratio(int64_t num, int64_t den) {
    // cos(pi * num / den) with exact argument reduction modulo 2
    const int64_t r = num % (2 * den);
    return std::cos(M_PI * static_cast<double>(r) / static_cast<double>(den));
}
double sinpi_ratio(int64_t num, int64_t den) {
    const int64_t r = num % (2 * den);
    return std::sin(M_PI * static_cast<double>(r) / static_cast<double>(den));
}

template <typename T>
T* dalloc(size_t n, PoissonPlan& pl) {
    T* p = static_cast<T*>(dev_alloc(n * sizeof(T), &pl.stream));
    pl.bytes += n * sizeof(T);
    return p;
}

// The basis tables of the chain (FFTW r2r definitions, poisson.h) in FP64.
struct Tables {
    std::vector<double> cy, cx, bcat, acat, sc;
    std::vector<double> sin_x, sin_y;  // sin(pi j (x+1/2)/nx) [j][x], sin(pi k (y+1/2)/ny) [k][y]
};

// The step-dependent tables from the cached sines: Sy (rows ny..2ny of [Ay; Sy]), Sx (rows
// nx..2nx of [Ax; Sx]) and the spectral scale, with the same expressions as make_tables.
void step_tables(int nx, int ny, float sx, float sy, const std::vector<double>& sin_x,
                 const std::vector<double>& sin_y, std::vector<double>& sy_rows, std::vector<double>& sx_rows,
                 std::vector<double>& sc) {
    const size_t X = nx, Y = ny;
    std::vector<double> u(X), v(Y);
    for (size_t j = 0; j < X; ++j) u[j] = M_PI * static_cast<double>(j) / (static_cast<double>(nx) * sx);
    for (size_t k = 0; k < Y; ++k) v[k] = M_PI * static_cast<double>(k) / (static_cast<double>(ny) * sy);
    sy_rows.resize(Y * Y);
    sx_rows.resize(X * X);
    sc.resize(X * Y);
    for (size_t k = 0; k < Y; ++k)
        for (size_t y = 0; y < Y; ++y) sy_rows[y * Y + k] = 2.0 * v[k] * sin_y[k * Y + y];
    for (size_t j = 0; j < X; ++j)
        for (size_t x = 0; x < X; ++x) sx_rows[x * X + j] = 2.0 * u[j] * sin_x[j * X + x];
    const double nn = static_cast<double>(nx) * static_cast<double>(ny);
    for (size_t j = 0; j < X; ++j)
        for (size_t k = 0; k < Y; ++k) {
            const double den = u[j] * u[j] + v[k] * v[k];
            sc[j * Y + k] = den > 0.0 ? 1.0 / (nn * den) : 0.0;
        }
}
Tables make_tables(int nx, int ny, float sx, float sy) {
    const size_t X = nx, Y = ny;
    Tables t;
    t.cy.resize(Y * Y);
    t.cx.resize(X * X);
    t.bcat.resize(2 * Y * Y);
    t.acat.resize(2 * X * X);
    t.sc.resize(X * Y);
    std::vector<double>&cy = t.cy, &cx = t.cx, &bcat = t.bcat, &acat = t.acat, &sc = t.sc;
    t.sin_x.resize(X * X);
    t.sin_y.resize(Y * Y);
    std::vector<double> u(X), v(Y);
    for (size_t j = 0; j < X; ++j) u[j] = M_PI * static_cast<double>(j) / (static_cast<double>(nx) * sx);
    for (size_t k = 0; k < Y; ++k) v[k] = M_PI * static_cast<double>(k) / (static_cast<double>(ny) * sy);
    for (size_t k = 0; k < Y; ++k)
        for (size_t y = 0; y < Y; ++y) {
            const int64_t num = static_cast<int64_t>(k) * (2 * static_cast<int64_t>(y) + 1);
            const double c = cospi_ratio(num, 2 * static_cast<int64_t>(ny));
            const double s = sinpi_ratio(num, 2 * static_cast<int64_t>(ny));
            cy[k * Y + y] = c;
            t.sin_y[k * Y + y] = s;
            bcat[y * Y + k] = (k == 0 ? 1.0 : 2.0) * c;      // Ay[y][k]
            bcat[(Y + y) * Y + k] = 2.0 * v[k] * s;          // Sy[y][k]
        }
    for (size_t j = 0; j < X; ++j)
        for (size_t x = 0; x < X; ++x) {
            const int64_t num = static_cast<int64_t>(j) * (2 * static_cast<int64_t>(x) + 1);
            const double c = cospi_ratio(num, 2 * static_cast<int64_t>(nx));
            const double s = sinpi_ratio(num, 2 * static_cast<int64_t>(nx));
            cx[j * X + x] = c;
            t.sin_x[j * X + x] = s;
            acat[x * X + j] = (j == 0 ? 1.0 : 2.0) * c;      // Ax[x][j]
            acat[(X + x) * X + j] = 2.0 * u[j] * s;          // Sx[x][j]
        }
    const double nn = static_cast<double>(nx) * static_cast<double>(ny);
    for (size_t j = 0; j < X; ++j)
        for (size_t k = 0; k < Y; ++k) {
            const double den = u[j] * u[j] + v[k] * v[k];
            sc[j * Y + k] = den > 0.0 ? 1.0 / (nn * den) : 0.0;
        }

    return t;
}

}  // namespace

void sgemm_tn(const GemmArgs& g, int batch, cudaStream_t s) {
    const bool aligned = (g.lda % 4 == 0) && (g.ldb % 4 == 0) &&
                         (reinterpret_cast<uintptr_t>(g.A) % 16 == 0) &&
                         (reinterpret_cast<uintptr_t>(g.B) % 16 == 0) && (g.sA % 4 == 0) &&
                         (g.sB % 4 == 0);
    dim3 grid(ceil_div(g.N, BN), ceil_div(g.M, BM), batch);
    launch_pdl(gemm_tn_kernel<float, float>, grid, dim3(NT), 0, s, g, aligned ? 1 : 0);
}

template <typename TO>
void dgemm_tn(const GemmArgsT<double, TO>& g, int batch, cudaStream_t s) {
    dim3 grid(ceil_div(g.N, BN), ceil_div(g.M, BM), batch);
    launch_pdl(gemm_tn_kernel<double, TO>, grid, dim3(NT), 0, s, g, 0);
}

void row_stats(const float* a, int rows, int cols, int64_t ld, int seg, float* mean, float* sum,
               cudaStream_t s) {
    const int nseg = cols / seg;
    const int warps = rows * nseg;
    launch_pdl(row_stats_kernel, dim3(ceil_div(warps, 8)), dim3(256), 0, s, a, rows, nseg, ld, seg, mean, sum);
}

void set_row0(float* C, int64_t sC, int n, const float* vals, int64_t sv, const float* scale,
              int batch, cudaStream_t s) {
    dim3 grid(ceil_div(n, 256), batch);
    launch_pdl(set_row0_kernel, grid, dim3(256), 0, s, C, sC, n, vals, sv, scale);
}

void poisson_plan_create(PoissonPlan& pl, int nx, int ny, float sx, float sy, int precision,
                         int batch_cap) {
    SPG_REQUIRE(nx >= 2 && ny >= 2, SPG_E_INVALID, "Poisson: grid must be at least 2x2");
    SPG_REQUIRE(sx > 0.f && sy > 0.f, SPG_E_INVALID, "Poisson: bin step must be positive");
    SPG_REQUIRE(precision == SPG_POISSON_FP32 || precision == SPG_POISSON_BF16X3 || precision == SPG_POISSON_FP64,
                SPG_E_INVALID, "Poisson: unknown precision");
    SPG_REQUIRE(batch_cap >= 1, SPG_E_INVALID, "Poisson: batch capacity must be positive");
    if (precision == SPG_POISSON_BF16X3)
        SPG_REQUIRE(tc_supported(nx, ny), SPG_E_INVALID,
                    "Poisson: split-BF16 path needs nx, ny multiples of 128");
    pl.nx = nx;
    pl.ny = ny;
    pl.step_x = sx;
    pl.step_y = sy;
    pl.precision = precision;
    pl.batch_cap = batch_cap;
    pl.name = precision == SPG_POISSON_FP32   ? "cuda-sm100a-fp32"
              : precision == SPG_POISSON_FP64 ? "cuda-sm100a-fp64"
                                              : "cuda-sm100a-bf16x3";

    const size_t X = nx, Y = ny;
    const Tables t = make_tables(nx, ny, sx, sy);
    const std::vector<double>&cy = t.cy, &cx = t.cx, &bcat = t.bcat, &acat = t.acat, &sc = t.sc;
    pl.sin_x = t.sin_x;
    pl.sin_y = t.sin_y;

    const size_t B = static_cast<size_t>(batch_cap);
    if (precision == SPG_POISSON_FP64) {
        auto up64 = [&](double*& dst, const std::vector<double>& h) {
            dst = dalloc<double>(h.size(), pl);
            upload_bytes(dst, h.data(), h.size() * 8, pl.stream);
        };
        up64(pl.cy64, cy);
        up64(pl.cx64, cx);
        up64(pl.bcat64, bcat);
        up64(pl.acat64, acat);
        up64(pl.scale64, sc);
        pl.rho64 = dalloc<double>(B * X * Y, pl);
        pl.t0t64 = dalloc<double>(B * X * Y, pl);
        pl.p64 = dalloc<double>(B * X * Y, pl);
        pl.t12t64 = dalloc<double>(2 * B * X * Y, pl);
        return;
    }
    // the FP32 forms: bases rounded once to float
    auto up32 = [&](float*& dst, const std::vector<double>& h) {
        std::vector<float> f(h.begin(), h.end());
        dst = dalloc<float>(f.size(), pl);
        upload_bytes(dst, f.data(), f.size() * 4, pl.stream);
        return f;
    };
    const std::vector<float> fcy = up32(pl.cy, cy), fcx = up32(pl.cx, cx);
    const std::vector<float> fbcat = up32(pl.bcat, bcat), facat = up32(pl.acat, acat);
    up32(pl.scale, sc);
    pl.dc = dalloc<float>(4 * B * std::max(X, Y), pl);  // row means / sums, both splits
    if (precision == SPG_POISSON_FP32) {
        pl.t0t = dalloc<float>(B * X * Y, pl);
        pl.p = dalloc<float>(B * X * Y, pl);
        pl.t12t = dalloc<float>(2 * B * X * Y, pl);
    } else {
        tc_plan_create(pl, fcy, fcx, fbcat, facat);
    }
}

void poisson_plan_set_steps(PoissonPlan& pl, float sx, float sy) {
    if (sx == pl.step_x && sy == pl.step_y) return;
    SPG_REQUIRE(sx > 0.f && sy > 0.f, SPG_E_INVALID, "Poisson: bin step must be positive");
    const size_t X = pl.nx, Y = pl.ny;
    std::vector<double> sy_rows, sx_rows, sc;
    step_tables(pl.nx, pl.ny, sx, sy, pl.sin_x, pl.sin_y, sy_rows, sx_rows, sc);
    if (pl.precision == SPG_POISSON_FP64) {
        upload_bytes(pl.bcat64 + Y * Y, sy_rows.data(), Y * Y * 8, pl.stream);
        upload_bytes(pl.acat64 + X * X, sx_rows.data(), X * X * 8, pl.stream);
        upload_bytes(pl.scale64, sc.data(), sc.size() * 8, pl.stream);
    } else {
        const std::vector<float> fsy(sy_rows.begin(), sy_rows.end()), fsx(sx_rows.begin(), sx_rows.end());
        const std::vector<float> fsc(sc.begin(), sc.end());
        upload_bytes(pl.bcat + Y * Y, fsy.data(), Y * Y * 4, pl.stream);
        upload_bytes(pl.acat + X * X, fsx.data(), X * X * 4, pl.stream);
        upload_bytes(pl.scale, fsc.data(), fsc.size() * 4, pl.stream);
        if (pl.precision == SPG_POISSON_BF16X3) tc_plan_refill_sines(pl, fsy, fsx);
    }
    pl.step_x = sx;
    pl.step_y = sy;
}

void poisson_plan_destroy(PoissonPlan& pl) {
    if (pl.precision == SPG_POISSON_BF16X3) tc_plan_destroy(pl);
    for (float* q : {pl.cy, pl.cx, pl.bcat, pl.acat, pl.scale, pl.t0t, pl.p, pl.t12t, pl.dc}) dev_free(q, pl.stream);
    pl.cy = pl.cx = pl.bcat = pl.acat = pl.scale = pl.t0t = pl.p = pl.t12t = pl.dc = nullptr;
    for (double* q : {pl.cy64, pl.cx64, pl.bcat64, pl.acat64, pl.scale64, pl.rho64, pl.t0t64, pl.p64, pl.t12t64})
        dev_free(q, pl.stream);
    pl.cy64 = pl.cx64 = pl.bcat64 = pl.acat64 = pl.scale64 = nullptr;
    pl.rho64 = pl.t0t64 = pl.p64 = pl.t12t64 = nullptr;
}

void poisson_solve(PoissonPlan& pl, int batch, const float* rho, float* phi, float* ex, float* ey,
                   cudaStream_t s, bool rho_split_ready) {
    SPG_REQUIRE(batch >= 1 && batch <= pl.batch_cap, SPG_E_CAPACITY, "Poisson: batch exceeds plan");
    SPG_REQUIRE(!rho_split_ready || (pl.precision == SPG_POISSON_BF16X3 && batch == 1), SPG_E_INVALID,
                "Poisson: a prepared density operand needs a one-grid tensor-core solve");
    if (pl.precision == SPG_POISSON_BF16X3) {
        tc_solve(pl, batch, rho, phi, ex, ey, s, rho_split_ready);
        return;
    }
    const int X = pl.nx, Y = pl.ny;
    if (pl.precision == SPG_POISSON_FP64) {
        // the same chain in FP64 (no DC split needed), results rounded once to float
        const int64_t BX = static_cast<int64_t>(batch) * X, XY = static_cast<int64_t>(X) * Y;
        launch_pdl(widen_kernel, dim3(std::min<int64_t>(ceil_div(BX * Y, 256), 4096)), dim3(256), 0, s, rho,
                   pl.rho64, BX * Y);
        dgemm_tn<double>({pl.cy64, pl.rho64, pl.t0t64, nullptr, nullptr, Y, static_cast<int>(BX), Y, Y, Y, Y, BX, 0,
                          0, 0, 0}, 1, s);
        dgemm_tn<double>({pl.cx64, pl.t0t64, pl.p64, nullptr, pl.scale64, X, Y, X, X, X, BX, Y, Y, 0, X, XY}, batch, s);
        dgemm_tn<double>({pl.bcat64, pl.p64, pl.t12t64, nullptr, nullptr, 2 * Y, static_cast<int>(BX), Y, 2 * Y, Y, Y,
                          BX, 0, 0, 0, 0}, 1, s);
        dgemm_tn<float>({pl.acat64, pl.t12t64, phi, ex, nullptr, 2 * X, Y, X, X, X, BX, Y, 0, 0, X, XY}, batch, s);
        dgemm_tn<float>({pl.acat64, pl.t12t64 + static_cast<int64_t>(Y) * BX, ey, nullptr, nullptr, X, Y, X, X, X, BX,
                         Y, 0, 0, X, XY}, batch, s);
        return;
    }
    const int64_t BX = static_cast<int64_t>(batch) * X;
    const int64_t XY = static_cast<int64_t>(X) * Y;
    const int64_t MXY = std::max(X, Y) * static_cast<int64_t>(batch);
    float* mean_r = pl.dc;
    float* sum_r = pl.dc + MXY;
    float* mean_t = pl.dc + 2 * MXY;
    float* sum_t = pl.dc + 3 * MXY;
    // G1: T0t (Y x B*X) = Cy . (rho_all - rowmean)^T, DC row from the exact row sums
    row_stats(rho, static_cast<int>(BX), Y, Y, Y, mean_r, sum_r, s);
    GemmArgs g1{pl.cy, rho, pl.t0t, nullptr, nullptr, Y, static_cast<int>(BX), Y, Y, Y, Y, BX, 0, 0, 0, 0};
    g1.boff = mean_r;
    sgemm_tn(g1, 1, s);
    set_row0(pl.t0t, 0, static_cast<int>(BX), sum_r, 0, nullptr, 1, s);
    // G2: P_g (X x Y) = Cx . (T0t[:, g] - rowmean)^T times the spectral scale; row 0 of P_g
    // (the x-DC row) from the exact sums
    row_stats(pl.t0t, Y, static_cast<int>(BX), BX, X, mean_t, sum_t, s);
    GemmArgs g2{pl.cx, pl.t0t, pl.p, nullptr, pl.scale, X, Y, X, X, X, BX, Y, Y, 0, X, XY};
    g2.boff = mean_t;
    g2.sBoff = Y;
    sgemm_tn(g2, batch, s);
    set_row0(pl.p, XY, Y, sum_t, Y, pl.scale, batch, s);
    // G3: T12t (2Y x B*X) = [Ay; Sy] . P_all^T
    sgemm_tn({pl.bcat, pl.p, pl.t12t, nullptr, nullptr, 2 * Y, static_cast<int>(BX), Y, 2 * Y, Y, Y, BX, 0, 0, 0, 0}, 1, s);
    // G4a: [phi_g; xi_x_g] = [Ax; Sx] . T1t[:, g]^T
    sgemm_tn({pl.acat, pl.t12t, phi, ex, nullptr, 2 * X, Y, X, X, X, BX, Y, 0, 0, X, XY}, batch, s);
    // G4b: xi_y_g = Ax . T2t[:, g]^T
    sgemm_tn({pl.acat, pl.t12t + static_cast<int64_t>(Y) * BX, ey, nullptr, nullptr, X, Y, X, X, X, BX, Y, 0, 0, X, XY},
             batch, s);
}

}  // namespace spg
