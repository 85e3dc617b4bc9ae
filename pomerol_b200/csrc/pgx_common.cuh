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

#ifdef __CUDACC__
// 1/x for x > 0 by the Newton-Raphson iteration y <- y + y (1 - x y), which
// doubles the number of correct bits per step (Muller et al., "Handbook of
// Floating-Point Arithmetic", 2nd ed., sec. 4.7), seeded with the hardware
// single-precision approximation (PTX rcp.approx.ftz.f32, at most 1 ulp of
// single precision): two steps bring the error to the double rounding level.
// Outside [1e-30, 1e30] (where the seed could leave the single-precision
// range) the IEEE division is used.
// The iteration alone, valid for |x| in [1e-30, 1e30] (either sign); callers
// that test the range once for several values keep their arithmetic free of
// branches.
__device__ __forceinline__ double recip_newton(double x) {
    float xf = (float)x, yf;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(yf) : "f"(xf));
    double y = (double)yf;
    double e = fma(-x, y, 1.0);
    y = fma(y, e, y);
    e = fma(-x, y, 1.0);
    return fma(y, e, y);
}
__device__ __forceinline__ bool recip_in_range(double x) {
    const double a = fabs(x);
    return a > 1e-30 && a < 1e30;
}
__device__ __forceinline__ double recip_pos(double x) { return recip_in_range(x) ? recip_newton(x) : 1.0 / x; }
// 1/a = conj(a) / |a|^2 with recip_pos for the real reciprocal.
__device__ __forceinline__ cd inv_fast(cd a) {
    const double r = recip_pos(abs2(a));
    return cd{a.x * r, -a.y * r};
}
#endif

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
