// Stand-in for the reference's FFTW-based CpuPoissonBackend, used ONLY to build the
// reference's own CPU GP path (oracle/_ref) in an image without FFTW.
//
// Test infrastructure: nothing in the product links this file.
//
// It implements the same factory symbol the reference declares in
// src/numeric/cpu/cpu_poisson.h:12 (sp::makeCpuPoissonBackend) and the same solve()
// contract as src/numeric/cpu/cpu_poisson.cpp:149-207:
//   F   = REDFT10 x REDFT10 (rho)
//   P   = F / (4 nx ny) / (u_j^2 + v_k^2),  P[0][0] = 0        (cpu_poisson.cpp:163-172)
//   phi = REDFT01 x REDFT01 (P)                                (cpu_poisson.cpp:176-179)
//   xi_x= RODFT01 x REDFT01 (P shifted down one in x, times u) (cpu_poisson.cpp:182-195)
//   xi_y= REDFT01 x RODFT01 (P shifted down one in y, times v) (cpu_poisson.cpp:198-206)
// The r2r kinds follow FFTW's published definitions (restated in cpu_poisson.cpp:8-37):
//   REDFT10: Y_k = 2 sum_j X_j cos(pi k (j+1/2)/n)
//   REDFT01: Y_k = X_0 + 2 sum_{j>=1} X_j cos(pi j (k+1/2)/n)
//   RODFT01: Y_k = (-1)^k X_{n-1} + 2 sum_{j=0}^{n-2} X_j sin(pi (j+1)(k+1/2)/n)
// Power-of-two lengths use a Makhoul reordering onto a radix-2 complex FFT computed in
// single precision (like FFTW's fftwf plans); other lengths use direct O(n^2) sums.
// The frequency tables are computed exactly as cpu_poisson.cpp:100-104 computes them.
#include "numeric/cpu/cpu_poisson.h"

#include <cmath>
#include <complex>
#include <cstring>
#include <stdexcept>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace sp {
namespace {

using cf = std::complex<float>;
constexpr float kPiF = 3.14159265358979323846f;
constexpr double kPiD = 3.14159265358979323846;

bool isPow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

// One-dimensional transform plan of length n (all three kinds share the tables).
struct Plan1D {
    int n = 0;
    bool fast = false;
    std::vector<int> bitrev;
    std::vector<cf> root;       // e^{-2 pi i k / n}, k < n/2
    std::vector<cf> tw;         // e^{-i pi k / (2n)}, k < n
    std::vector<float> cosTab;  // direct path: cos(pi k (j+1/2)/n) laid out [k*n+j]

    explicit Plan1D(int len) : n(len), fast(isPow2(len) && len >= 4) {
        tw.resize(static_cast<size_t>(n));
        for (int k = 0; k < n; ++k) {
            const double a = -kPiD * k / (2.0 * n);
            tw[static_cast<size_t>(k)] = cf(static_cast<float>(std::cos(a)), static_cast<float>(std::sin(a)));
        }
        if (fast) {
            int lg = 0;
            while ((1 << lg) < n) ++lg;
            bitrev.resize(static_cast<size_t>(n));
            for (int i = 0; i < n; ++i) {
                int r = 0;
                for (int b = 0; b < lg; ++b) r |= ((i >> b) & 1) << (lg - 1 - b);
                bitrev[static_cast<size_t>(i)] = r;
            }
            root.resize(static_cast<size_t>(n / 2));
            for (int k = 0; k < n / 2; ++k) {
                const double a = -2.0 * kPiD * k / n;
                root[static_cast<size_t>(k)] = cf(static_cast<float>(std::cos(a)), static_cast<float>(std::sin(a)));
            }
        } else {
            cosTab.resize(static_cast<size_t>(n) * n);
            for (int k = 0; k < n; ++k)
                for (int j = 0; j < n; ++j)
                    cosTab[static_cast<size_t>(k) * n + j] =
                        static_cast<float>(std::cos(kPiD * k * (j + 0.5) / n));
        }
    }

    // In-place forward complex FFT (sign -1), unnormalised.
    void fft(cf* a, bool inverse) const {
        for (int i = 0; i < n; ++i) {
            const int r = bitrev[static_cast<size_t>(i)];
            if (i < r) std::swap(a[i], a[r]);
        }
        for (int len = 2; len <= n; len <<= 1) {
            const int half = len >> 1, stride = n / len;
            for (int s = 0; s < n; s += len) {
                for (int k = 0; k < half; ++k) {
                    cf w = root[static_cast<size_t>(k * stride)];
                    if (inverse) w = std::conj(w);
                    const cf t = w * a[s + k + half];
                    a[s + k + half] = a[s + k] - t;
                    a[s + k] = a[s + k] + t;
                }
            }
        }
    }

    // REDFT10: out_k = 2 sum_j in_j cos(pi k (j+1/2)/n)
    void redft10(const float* in, float* out, cf* work) const {
        if (!fast) {
            for (int k = 0; k < n; ++k) {
                float s = 0.f;
                const float* c = &cosTab[static_cast<size_t>(k) * n];
                for (int j = 0; j < n; ++j) s += in[j] * c[j];
                out[k] = 2.f * s;
            }
            return;
        }
        for (int j = 0; j < n / 2; ++j) {
            work[j] = cf(in[2 * j], 0.f);
            work[n - 1 - j] = cf(in[2 * j + 1], 0.f);
        }
        fft(work, false);
        for (int k = 0; k < n; ++k) out[k] = 2.f * (tw[static_cast<size_t>(k)] * work[k]).real();
    }

    // REDFT01: out_j = in_0 + 2 sum_{k>=1} in_k cos(pi k (j+1/2)/n)
    void redft01(const float* in, float* out, cf* work) const {
        if (!fast) {
            for (int j = 0; j < n; ++j) {
                float s = 0.f;
                for (int k = 1; k < n; ++k) s += in[k] * cosTab[static_cast<size_t>(k) * n + j];
                out[j] = in[0] + 2.f * s;
            }
            return;
        }
        work[0] = cf(in[0], 0.f);
        for (int k = 1; k < n; ++k)
            work[k] = cf(in[k], -in[n - k]) * std::conj(tw[static_cast<size_t>(k)]);
        fft(work, true);
        for (int m = 0; m < n / 2; ++m) {
            out[2 * m] = work[m].real();
            out[2 * m + 1] = work[n - 1 - m].real();
        }
    }

    // RODFT01: out_j = (-1)^j in_{n-1} + 2 sum_{k=0}^{n-2} in_k sin(pi (k+1)(j+1/2)/n)
    //        = (-1)^j REDFT01(reversed in)_j
    void rodft01(const float* in, float* out, float* tmp, cf* work) const {
        for (int k = 0; k < n; ++k) tmp[k] = in[n - 1 - k];
        redft01(tmp, out, work);
        for (int j = 1; j < n; j += 2) out[j] = -out[j];
    }
};

enum Kind { kR10, kR01, kO01 };

class ShimPoissonBackend final : public PoissonBackend {
public:
    explicit ShimPoissonBackend(const BackendConfig& cfg)
        : nx_(cfg.nx), ny_(cfg.ny), step_x_(cfg.step_x), step_y_(cfg.step_y),
          px_(cfg.nx), py_(cfg.ny) {
        // Same argument checks as cpu_poisson.cpp:78-83.
        if (nx_ < 2 || ny_ < 2)
            throw std::runtime_error("CpuPoissonBackend: grid must be at least 2x2");
        if (!(step_x_ > 0.f) || !(step_y_ > 0.f))
            throw std::runtime_error("CpuPoissonBackend: bin step must be positive");
        if (cfg.fftw_threads < 1)
            throw std::runtime_error("CpuPoissonBackend: fftw_threads must be positive");
        const size_t n = static_cast<size_t>(nx_) * static_cast<size_t>(ny_);
        threads_ = n >= static_cast<size_t>(256 * 256) ? cfg.fftw_threads : 1;
        freq_u_.resize(static_cast<size_t>(nx_));
        freq_v_.resize(static_cast<size_t>(ny_));
        for (int j = 0; j < nx_; ++j)
            freq_u_[static_cast<size_t>(j)] = kPiF * static_cast<float>(j) / (static_cast<float>(nx_) * step_x_);
        for (int k = 0; k < ny_; ++k)
            freq_v_[static_cast<size_t>(k)] = kPiF * static_cast<float>(k) / (static_cast<float>(ny_) * step_y_);
        spec_.assign(n, 0.f);
        work_.assign(n, 0.f);
        tmp_.assign(n, 0.f);
    }

    // 2D r2r: kind0 along x (slow axis), kind1 along y (fast axis), like
    // fftwf_plan_r2r_2d(nx, ny, in, out, kind0, kind1).
    void r2r2d(const float* in, float* out, Kind k0, Kind k1) {
        const int nx = nx_, ny = ny_;
        // along y: rows are contiguous
#pragma omp parallel num_threads(threads_)
        {
            std::vector<cf> w(static_cast<size_t>(std::max(nx, ny)));
            std::vector<float> t(static_cast<size_t>(std::max(nx, ny)));
#pragma omp for schedule(static)
            for (int x = 0; x < nx; ++x) {
                const float* src = in + static_cast<size_t>(x) * ny;
                float* dst = tmp_.data() + static_cast<size_t>(x) * ny;
                apply(py_, k1, src, dst, t.data(), w.data());
            }
        }
        // along x: gather columns
#pragma omp parallel num_threads(threads_)
        {
            std::vector<cf> w(static_cast<size_t>(std::max(nx, ny)));
            std::vector<float> t(static_cast<size_t>(std::max(nx, ny)));
            std::vector<float> col(static_cast<size_t>(nx)), res(static_cast<size_t>(nx));
#pragma omp for schedule(static)
            for (int y = 0; y < ny; ++y) {
                for (int x = 0; x < nx; ++x) col[static_cast<size_t>(x)] = tmp_[static_cast<size_t>(x) * ny + y];
                apply(px_, k0, col.data(), res.data(), t.data(), w.data());
                for (int x = 0; x < nx; ++x) out[static_cast<size_t>(x) * ny + y] = res[static_cast<size_t>(x)];
            }
        }
    }

    static void apply(const Plan1D& p, Kind k, const float* in, float* out, float* t, cf* w) {
        if (k == kR10) p.redft10(in, out, w);
        else if (k == kR01) p.redft01(in, out, w);
        else p.rodft01(in, out, t, w);
    }

    void solve(BinGridSpan density, BinGridSpan phi, BinGridSpan field_x,
               BinGridSpan field_y) override {
        checkSpan(density);
        checkSpan(phi);
        checkSpan(field_x);
        checkSpan(field_y);
        r2r2d(density.data, spec_.data(), kR10, kR10);
        const float invNorm = 1.0f / (4.0f * static_cast<float>(nx_) * static_cast<float>(ny_));
        for (int j = 0; j < nx_; ++j) {
            const float u2 = freq_u_[static_cast<size_t>(j)] * freq_u_[static_cast<size_t>(j)];
            float* row = spec_.data() + static_cast<size_t>(j) * ny_;
            for (int k = 0; k < ny_; ++k) {
                const float v2 = freq_v_[static_cast<size_t>(k)] * freq_v_[static_cast<size_t>(k)];
                const float denom = u2 + v2;
                row[k] = (denom > 0.f) ? (row[k] * invNorm / denom) : 0.f;
            }
        }
        r2r2d(spec_.data(), phi.data, kR01, kR01);
        for (int j = 0; j < nx_; ++j) {
            float* dst = work_.data() + static_cast<size_t>(j) * ny_;
            if (j == nx_ - 1) {
                std::memset(dst, 0, static_cast<size_t>(ny_) * sizeof(float));
            } else {
                const float u = freq_u_[static_cast<size_t>(j + 1)];
                const float* src = spec_.data() + static_cast<size_t>(j + 1) * ny_;
                for (int k = 0; k < ny_; ++k) dst[k] = src[k] * u;
            }
        }
        r2r2d(work_.data(), field_x.data, kO01, kR01);
        for (int j = 0; j < nx_; ++j) {
            float* dst = work_.data() + static_cast<size_t>(j) * ny_;
            const float* src = spec_.data() + static_cast<size_t>(j) * ny_;
            for (int k = 0; k < ny_ - 1; ++k) dst[k] = src[k + 1] * freq_v_[static_cast<size_t>(k + 1)];
            dst[ny_ - 1] = 0.f;
        }
        r2r2d(work_.data(), field_y.data, kR01, kO01);
    }

    const char* name() const override { return "cpu-dct-shim"; }
    int cpuThreads() const override { return threads_; }

private:
    void checkSpan(const BinGridSpan& s) const {
        if (!s.valid() || s.nx != nx_ || s.ny != ny_)
            throw std::runtime_error("CpuPoissonBackend: grid span dimension mismatch");
    }

    int nx_, ny_;
    float step_x_, step_y_;
    int threads_ = 1;
    Plan1D px_, py_;
    std::vector<float> freq_u_, freq_v_;
    std::vector<float> spec_, work_, tmp_;
};

}  // namespace

std::unique_ptr<PoissonBackend> makeCpuPoissonBackend(const BackendConfig& cfg) {
    return std::make_unique<ShimPoissonBackend>(cfg);
}

}  // namespace sp
