// Common device/host helpers for libpgx (B200, sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdio>
#include <string>

#include "../../include/pgx.h"

namespace pgx {

// ---------------------------------------------------------------- complex
struct cd {
    double x, y;
};

__host__ __device__ __forceinline__ cd mk(double x, double y = 0.0) { return cd{x, y}; }
__host__ __device__ __forceinline__ cd operator+(cd a, cd b) { return cd{a.x + b.x, a.y + b.y}; }
__host__ __device__ __forceinline__ cd operator-(cd a, cd b) { return cd{a.x - b.x, a.y - b.y}; }
__host__ __device__ __forceinline__ cd operator*(cd a, cd b) {
    return cd{a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x};
}
__host__ __device__ __forceinline__ cd operator*(cd a, double s) { return cd{a.x * s, a.y * s}; }
__host__ __device__ __forceinline__ cd operator*(double s, cd a) { return cd{a.x * s, a.y * s}; }
__host__ __device__ __forceinline__ cd conj(cd a) { return cd{a.x, -a.y}; }
__host__ __device__ __forceinline__ double abs2(cd a) { return a.x * a.x + a.y * a.y; }
// 1/a as conj(a)/|a|^2 (one real division).
__host__ __device__ __forceinline__ cd inv(cd a) {
    double r = 1.0 / abs2(a);
    return cd{a.x * r, -a.y * r};
}
__host__ __device__ __forceinline__ cd div(cd a, cd b) { return a * inv(b); }

// Scalar-type helpers used by templated kernels (double or cd).
__host__ __device__ __forceinline__ cd tocd(double a) { return cd{a, 0.0}; }
__host__ __device__ __forceinline__ cd tocd(cd a) { return a; }
template <typename T> struct is_cd { static constexpr bool value = false; };
template <> struct is_cd<cd> { static constexpr bool value = true; };

// ------------------------------------------------------------ error plumbing
struct Error {
    int code;
    std::string msg;
};

#define PGX_CUDA(call)                                                                 \
    do {                                                                               \
        cudaError_t e_ = (call);                                                       \
        if (e_ != cudaSuccess)                                                         \
            throw ::pgx::Error{PGX_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)}; \
    } while (0)

#define PGX_CHECK(cond, code, text)                                 \
    do {                                                            \
        if (!(cond)) throw ::pgx::Error{(code), std::string(text)}; \
    } while (0)

// Kernel launches issued by this library (process-wide).
long long& launch_counter();

inline void check_launch(const char* what) {
    ++launch_counter();
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) throw Error{PGX_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e)};
}

inline int ceil_div(long a, long b) { return int((a + b - 1) / b); }

}  // namespace pgx
