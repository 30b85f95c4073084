// piv_common.cuh -- shared definitions for the sm_100a PIV correlation kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <type_traits>
#include <utility>

// Error codes of the reference C-ABI (pivtools_cli/lib/common.h:31-36).
#define PIV_ERROR_NONE 0
#define PIV_ERROR_NOMEM 1
#define PIV_ERROR_NOPLAN_FWD 2
#define PIV_ERROR_NOPLAN_BWD 4
#define PIV_ERROR_NOPLAN 8
#define PIV_ERROR_OUT_OF_BOUNDS 9
// Additional code of this library: a CUDA runtime call failed (no device, launch
// failure).  The reference never returns it; callers treat any non-zero as fatal.
#define PIV_ERROR_CUDA 16

#define PIV_EXPORT extern "C" __attribute__((visibility("default")))

#define PIV_CUDA_TRY(expr)                                  \
    do {                                                    \
        cudaError_t e_ = (expr);                            \
        if (e_ != cudaSuccess) return PIV_ERROR_CUDA;       \
    } while (0)

namespace piv {

// ----------------------------------------------------------------------------
// Compile-time unrolling helper: f(std::integral_constant<int, i>) for i < N.
// ----------------------------------------------------------------------------
template <int... Is, class F>
__host__ __device__ __forceinline__ void sfor_impl(std::integer_sequence<int, Is...>, F &&f)
{
    (f(std::integral_constant<int, Is>{}), ...);
}
template <int N, class F>
__host__ __device__ __forceinline__ void sfor(F &&f)
{
    sfor_impl(std::make_integer_sequence<int, N>{}, static_cast<F &&>(f));
}

// ----------------------------------------------------------------------------
// Compile-time trigonometry for FFT twiddles: cos / sin of 2*pi*m/n, evaluated
// in double by Taylor series on an argument reduced to [0, pi/4].
// ----------------------------------------------------------------------------
constexpr double kPi = 3.14159265358979323846264338327950288;

__host__ __device__ constexpr double cx_sin_small(double x)
{
    double x2 = x * x, term = x, sum = x;
    for (int k = 1; k < 14; ++k) {
        term *= -x2 / (double)((2 * k) * (2 * k + 1));
        sum += term;
    }
    return sum;
}
__host__ __device__ constexpr double cx_cos_small(double x)
{
    double x2 = x * x, term = 1.0, sum = 1.0;
    for (int k = 1; k < 14; ++k) {
        term *= -x2 / (double)((2 * k - 1) * (2 * k));
        sum += term;
    }
    return sum;
}
// (cos, sin) of 2*pi*m/n for integer m, n > 0.
struct cx_cs { double c, s; };
__host__ __device__ constexpr cx_cs cx_cossin(int m, int n)
{
    long mm = ((long)m % n + n) % n;
    long a = 4 * mm;
    long quad = a / n;            // quadrant 0..3
    long rem = a - quad * n;      // angle within quadrant = (pi/2) * rem/n
    double beta = (kPi / 2.0) * (double)rem / (double)n;
    double c0 = 0.0, s0 = 0.0;
    if (2 * rem <= n) {
        c0 = cx_cos_small(beta);
        s0 = cx_sin_small(beta);
    } else {
        double g = (kPi / 2.0) * (double)(n - rem) / (double)n;
        c0 = cx_sin_small(g);
        s0 = cx_cos_small(g);
    }
    if (quad == 0) return {c0, s0};
    if (quad == 1) return {-s0, c0};
    if (quad == 2) return {-c0, -s0};
    return {s0, -c0};
}

}  // namespace piv
