// The QP's BiCGSTAB on the device (qp_device.cu), and the summation order it shares with the
// host solver in qp.cpp.
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>

constexpr int kQpBlocks = 1024;   // fixed grid of every solver kernel
constexpr int kQpThreads = 256;
constexpr int64_t kQpGrid = int64_t(kQpBlocks) * kQpThreads;

// s[0..255] summed by a halving tree: s[t] += s[t + h] for h = 128, 64, ..., 1.
inline float qp_tree(float* s) {
    for (int h = kQpThreads / 2; h > 0; h >>= 1)
        for (int t = 0; t < h; ++t) s[t] += s[t + h];
    return s[0];
}

// The 1024 block sums: four folded into each of 256 slots, then the halving tree.
inline float qp_fold_blocks(const float* blk) {
    float s[kQpThreads];
    for (int t = 0; t < kQpThreads; ++t)
        s[t] = ((blk[t] + blk[t + 256]) + blk[t + 512]) + blk[t + 768];
    return qp_tree(s);
}

struct QpDevice;

// A failed device step; code is SPG_E_NO_DEVICE or SPG_E_CUDA.
struct QpDeviceError : std::runtime_error {
    int code;
    QpDeviceError(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

// Throws QpDeviceError when no usable device is present or a CUDA call fails.
QpDevice* qp_device_create();
void qp_device_destroy(QpDevice* d);

// Solves A x = b (CSR over n rows, columns ascending) from the guess in x, as the host
// bicgstab does; x is overwritten with the solution. Returns the iterations and the final
// relative residual in *iters and *err.
void qp_device_solve(QpDevice* d, int32_t n, int64_t nnz, const int32_t* row_start, const int32_t* col,
                     const float* val, const float* rhs, float* x, int32_t max_iter, float tol, int32_t* iters,
                     float* err);

// Kernel launches made by this library's QP solver so far (all devices, all solves).
int64_t qp_device_launches();
