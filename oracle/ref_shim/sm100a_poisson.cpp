// The reference-side Poisson adapter a maintainer adds to superPlace to use this repository's
// engine (the adapter INTEGRATION.md gives), compiled here against the reference's own
// headers to show the drop-in builds and behaves: sp::makeCudaPoissonBackend, the factory hook
// the reference declares in src/numeric/cuda/cuda_poisson.h and calls from
// src/numeric/poisson_factory.cpp:16-18 when ENABLE_CUDA is defined, returns a PoissonBackend
// (src/numeric/poisson_backend.h:20-46) whose solve() is spg_poisson_solve.
//
// Test infrastructure: oracle/Makefile links it with the reference's poisson_factory.cpp
// (-DENABLE_CUDA), the CPU backend stand-in and the reference's own test programs
// test/test_poisson.cpp and test/test_poisson_parity.cpp, unmodified, so those programs run
// their checks through PoissonBackend::solve on the device.
//
// Contract kept from the reference's CUDA factory (cuda_poisson.h): nullptr when no device is
// usable or a dimension is odd (the caller falls back to the CPU backend); std::runtime_error
// when a device exists but the plan cannot be built. solve() allocates nothing.
//
// Precision: the plain FP32 contraction form by default, the reference's own CUDA backend being
// an FP32 FFT held to 1e-5 of the CPU solve; SPG_POISSON_PRECISION=bf16x3 selects the split-BF16
// tensor-core form where both dimensions are multiples of 128.
#include <cstdlib>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>

#include "numeric/cuda/cuda_poisson.h"
#include "numeric/poisson_backend.h"
#include "spgpu.h"

namespace sp {
namespace {

class Sm100aPoissonBackend final : public PoissonBackend {
public:
    Sm100aPoissonBackend(const BackendConfig& c, int precision) {
        const int rc = spg_poisson_create(c.nx, c.ny, c.step_x, c.step_y, precision, &h_);
        if (rc != SPG_OK) throw std::runtime_error(std::string("sm100a Poisson backend: ") + spg_last_error());
    }
    ~Sm100aPoissonBackend() override { spg_poisson_destroy(h_); }
    void solve(BinGridSpan density, BinGridSpan phi, BinGridSpan field_x, BinGridSpan field_y) override {
        if (density.nx != phi.nx || density.ny != phi.ny || density.nx != field_x.nx ||
            density.ny != field_x.ny || density.nx != field_y.nx || density.ny != field_y.ny)
            throw std::runtime_error("sm100a Poisson backend: span dimensions differ");
        if (spg_poisson_solve(h_, density.data, phi.data, field_x.data, field_y.data) != SPG_OK)
            throw std::runtime_error(std::string("sm100a Poisson backend: ") + spg_last_error());
    }
    const char* name() const override { return spg_poisson_name(h_); }

private:
    spg_poisson* h_ = nullptr;
};

int requested_precision(const BackendConfig& c) {
    const char* e = std::getenv("SPG_POISSON_PRECISION");
    if (e && std::strcmp(e, "bf16x3") == 0 && c.nx % 128 == 0 && c.ny % 128 == 0) return SPG_POISSON_BF16X3;
    return SPG_POISSON_FP32;
}

}  // namespace

std::unique_ptr<PoissonBackend> makeCudaPoissonBackend(const BackendConfig& cfg) {
    if (spg_device_check() != SPG_OK) return nullptr;
    if (cfg.nx % 2 != 0 || cfg.ny % 2 != 0) return nullptr;
    return std::make_unique<Sm100aPoissonBackend>(cfg, requested_precision(cfg));
}

}  // namespace sp
