// Forward-mode dual numbers (value + one directional derivative) for the
// tangent kernels.  Instantiating the material and kinematics templates of
// mechanics.cuh on Dual gives, in one pass, P(F) and its derivative along a
// chosen direction: a displacement increment (the true tangent K(u) v) or a
// material constant (dR/dtheta).
#pragma once
#include <cuda_runtime.h>

namespace efem {

struct Dual {
    double v, d;
    __host__ __device__ constexpr Dual() : v(0), d(0) {}
    __host__ __device__ constexpr Dual(double x) : v(x), d(0) {}
    __host__ __device__ constexpr Dual(double x, double dx) : v(x), d(dx) {}
    __device__ Dual& operator+=(const Dual& o)
    {
        v += o.v;
        d += o.d;
        return *this;
    }
    __device__ Dual& operator-=(const Dual& o)
    {
        v -= o.v;
        d -= o.d;
        return *this;
    }
    __device__ Dual& operator*=(const Dual& o)
    {
        d = d * o.v + v * o.d;
        v *= o.v;
        return *this;
    }
};

__device__ __forceinline__ Dual operator+(Dual a, Dual b) { return Dual(a.v + b.v, a.d + b.d); }
__device__ __forceinline__ Dual operator-(Dual a, Dual b) { return Dual(a.v - b.v, a.d - b.d); }
__device__ __forceinline__ Dual operator-(Dual a) { return Dual(-a.v, -a.d); }
__device__ __forceinline__ Dual operator*(Dual a, Dual b) { return Dual(a.v * b.v, a.d * b.v + a.v * b.d); }
__device__ __forceinline__ Dual operator/(Dual a, Dual b)
{
    const double q = a.v / b.v;
    return Dual(q, (a.d - q * b.d) / b.v);
}
__device__ __forceinline__ Dual sqrt(Dual a)
{
    const double s = ::sqrt(a.v);
    return Dual(s, s > 0.0 ? a.d / (2.0 * s) : 0.0);
}

}  // namespace efem
