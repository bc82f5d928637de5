// Forward-mode dual numbers with N derivative directions, usable on host and
// device.  The discrete adjoint builds its local Jacobians with them (face
// fluxes with respect to the six stencil densities and velocities, cell
// chemistry with respect to the concentrations), and the CPU tangent-linear
// check propagates parameter directions through the same forward map.
#pragma once

#include "vd_defs.H"
#include <cmath>

namespace vd {

template <int N>
struct Dual
{
    double v;
    double d[N];

    VD_HD Dual() : v(0.0)
    {
        for (int i = 0; i < N; ++i) d[i] = 0.0;
    }
    VD_HD Dual(double x) : v(x)
    {
        for (int i = 0; i < N; ++i) d[i] = 0.0;
    }
    VD_HD static Dual var(double x, int k)
    {
        Dual r(x);
        r.d[k] = 1.0;
        return r;
    }
    // var() by one select per slot: with k known only at run time the slots
    // can stay in registers, where the indexed store puts the dual in memory
    VD_HD static Dual var_sel(double x, int k)
    {
        Dual r(x);
#ifdef __CUDA_ARCH__
#pragma unroll
#endif
        for (int i = 0; i < N; ++i) r.d[i] = (i == k) ? 1.0 : 0.0;
        return r;
    }
    VD_HD Dual& operator+=(const Dual& o)
    {
        v += o.v;
        for (int i = 0; i < N; ++i) d[i] += o.d[i];
        return *this;
    }
    VD_HD Dual& operator-=(const Dual& o)
    {
        v -= o.v;
        for (int i = 0; i < N; ++i) d[i] -= o.d[i];
        return *this;
    }
    VD_HD Dual& operator*=(const Dual& o)
    {
        for (int i = 0; i < N; ++i) d[i] = d[i] * o.v + v * o.d[i];
        v *= o.v;
        return *this;
    }
    VD_HD Dual& operator/=(const Dual& o)
    {
        const double inv = 1.0 / o.v;
        const double q = v * inv;
        for (int i = 0; i < N; ++i) d[i] = (d[i] - q * o.d[i]) * inv;
        v = q;
        return *this;
    }
};

template <int N> VD_HD inline Dual<N> operator+(Dual<N> a, const Dual<N>& b) { return a += b; }
template <int N> VD_HD inline Dual<N> operator-(Dual<N> a, const Dual<N>& b) { return a -= b; }
template <int N> VD_HD inline Dual<N> operator*(Dual<N> a, const Dual<N>& b) { return a *= b; }
template <int N> VD_HD inline Dual<N> operator/(Dual<N> a, const Dual<N>& b) { return a /= b; }
template <int N> VD_HD inline Dual<N> operator+(Dual<N> a, double b) { a.v += b; return a; }
template <int N> VD_HD inline Dual<N> operator+(double b, Dual<N> a) { a.v += b; return a; }
template <int N> VD_HD inline Dual<N> operator-(Dual<N> a, double b) { a.v -= b; return a; }
template <int N> VD_HD inline Dual<N> operator-(double b, const Dual<N>& a)
{
    Dual<N> r;
    r.v = b - a.v;
    for (int i = 0; i < N; ++i) r.d[i] = -a.d[i];
    return r;
}
template <int N> VD_HD inline Dual<N> operator-(const Dual<N>& a)
{
    Dual<N> r;
    r.v = -a.v;
    for (int i = 0; i < N; ++i) r.d[i] = -a.d[i];
    return r;
}
template <int N> VD_HD inline Dual<N> operator*(Dual<N> a, double b)
{
    a.v *= b;
    for (int i = 0; i < N; ++i) a.d[i] *= b;
    return a;
}
template <int N> VD_HD inline Dual<N> operator*(double b, Dual<N> a) { return a * b; }
template <int N> VD_HD inline Dual<N> operator/(Dual<N> a, double b) { return a * (1.0 / b); }
template <int N> VD_HD inline Dual<N> operator/(double b, const Dual<N>& a)
{
    return Dual<N>(b) / a;
}

template <int N> VD_HD inline bool operator<(const Dual<N>& a, const Dual<N>& b) { return a.v < b.v; }
template <int N> VD_HD inline bool operator>(const Dual<N>& a, const Dual<N>& b) { return a.v > b.v; }
template <int N> VD_HD inline bool operator<(const Dual<N>& a, double b) { return a.v < b; }
template <int N> VD_HD inline bool operator>(const Dual<N>& a, double b) { return a.v > b; }
template <int N> VD_HD inline bool operator>=(const Dual<N>& a, double b) { return a.v >= b; }
template <int N> VD_HD inline bool operator<=(const Dual<N>& a, double b) { return a.v <= b; }

template <int N> VD_HD inline Dual<N> exp(const Dual<N>& a)
{
    Dual<N> r;
    r.v = ::exp(a.v);
    for (int i = 0; i < N; ++i) r.d[i] = r.v * a.d[i];
    return r;
}
template <int N> VD_HD inline Dual<N> log(const Dual<N>& a)
{
    Dual<N> r;
    r.v = ::log(a.v);
    const double inv = 1.0 / a.v;
    for (int i = 0; i < N; ++i) r.d[i] = inv * a.d[i];
    return r;
}
template <int N> VD_HD inline Dual<N> sqrt(const Dual<N>& a)
{
    Dual<N> r;
    r.v = ::sqrt(a.v);
    const double h = (r.v > 0.0) ? 0.5 / r.v : 0.0;
    for (int i = 0; i < N; ++i) r.d[i] = h * a.d[i];
    return r;
}
template <int N> VD_HD inline Dual<N> tanh(const Dual<N>& a)
{
    Dual<N> r;
    r.v = ::tanh(a.v);
    const double s = 1.0 - r.v * r.v;
    for (int i = 0; i < N; ++i) r.d[i] = s * a.d[i];
    return r;
}
// |a| and copysign: derivative taken on the branch of a's sign (kinks are
// avoided by keeping states away from them)
template <int N> VD_HD inline Dual<N> fabs(const Dual<N>& a) { return a.v < 0.0 ? -a : a; }

VD_HD inline double value(double x) { return x; }
template <int N> VD_HD inline double value(const Dual<N>& x) { return x.v; }

} // namespace vd
