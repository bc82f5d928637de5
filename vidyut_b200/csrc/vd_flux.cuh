// Drift-flux numerics on the device: WENO5 (JS / M / Z) reconstruction with
// the local Lax-Friedrichs split, the second-order WAF flux with the MINBEE
// limiter, and first-order upwind.  Same schemes and constants as the
// reference (Source/compute_explicit_flux.H:16-214, including the Rathan &
// Naga Raju WENO-M/Z weights), arranged for FP64 throughput: the three
// 1/(beta_k + eps) from one reciprocal of their product, and one reciprocal
// for the weight normalisation (two per reconstruction, not four), each a
// refined hardware approximation instead of an IEEE division.
#pragma once

namespace vd {

// 1/x for the positive, finite, normal x of the WENO weights (a product of
// smoothness indicators each >= 1e-20, checked below 1e300; a sum of
// weights >= 0.1): the hardware's approximate reciprocal (PTX
// rcp.approx.ftz.f64) refined by two Newton-Raphson steps
// r <- r + r (1 - x r), each of which squares the relative error, to within
// an ulp or two of the correctly rounded quotient -- far below the parity
// tolerance (the explicit-source parity tests hold it to 1e-12 against the
// oracle's IEEE divisions) -- in fewer instructions than an IEEE division.
__device__ __forceinline__ double weno_rcp(double x)
{
    double r;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(x));
    double e = fma(-x, r, 1.0);
    r = fma(r, e, r);
    e = fma(-x, r, 1.0);
    return fma(r, e, r);
}

__device__ __forceinline__ double weno_gk(double w, double g)
{
    return w * (g + g * g - 3.0 * g * w + w * w) / (g * g + w * (1.0 - 2.0 * g));
}

// Fifth-order WENO value at the i+1/2 face from the five cells
// i-2 .. i+2 (a .. e), upwind-biased towards a.
__device__ __forceinline__ double weno5(double a, double b, double c, double d, double e,
                                        int scheme)
{
    const double eps = 1e-20;
    const double p1 = (1.0 / 3.0) * a - (7.0 / 6.0) * b + (11.0 / 6.0) * c;
    const double p2 = -(1.0 / 6.0) * b + (5.0 / 6.0) * c + (1.0 / 3.0) * d;
    const double p3 = (1.0 / 3.0) * c + (5.0 / 6.0) * d - (1.0 / 6.0) * e;
    const double s1 = a - 2.0 * b + c, s1b = a - 4.0 * b + 3.0 * c;
    const double s2 = b - 2.0 * c + d, s2b = b - d;
    const double s3 = c - 2.0 * d + e, s3b = 3.0 * c - 4.0 * d + e;
    const double b1 = (13.0 / 12.0) * s1 * s1 + 0.25 * s1b * s1b;
    const double b2 = (13.0 / 12.0) * s2 * s2 + 0.25 * s2b * s2b;
    const double b3 = (13.0 / 12.0) * s3 * s3 + 0.25 * s3b * s3b;
    double a1, a2, a3;
    const double q1 = b1 + eps, q2 = b2 + eps, q3 = b3 + eps;
    // one division for the three 1/q_k when the product is representable
    const double prod = q1 * q2 * q3;
    double i1, i2, i3;
    if (prod < 1e300)
    {
        const double ip = weno_rcp(prod);
        i1 = q2 * q3 * ip;
        i2 = q1 * q3 * ip;
        i3 = q1 * q2 * ip;
    } else
    {
        i1 = 1.0 / q1;
        i2 = 1.0 / q2;
        i3 = 1.0 / q3;
    }
    if (scheme == 3)
    {
        const double tau = fabs(b1 - b3);
        const double r1 = tau * i1, r2 = tau * i2, r3 = tau * i3;
        a1 = 0.1 * (1.0 + r1 * r1);
        a2 = 0.6 * (1.0 + r2 * r2);
        a3 = 0.3 * (1.0 + r3 * r3);
    } else
    {
        a1 = 0.1 * (i1 * i1);
        a2 = 0.6 * (i2 * i2);
        a3 = 0.3 * (i3 * i3);
        if (scheme == 2)
        {
            const double inv = 1.0 / (a1 + a2 + a3);
            const double w1 = a1 * inv, w2 = a2 * inv, w3 = a3 * inv;
            a1 = weno_gk(w1, 0.1);
            a2 = weno_gk(w2, 0.6);
            a3 = weno_gk(w3, 0.3);
        }
    }
    const double inv = weno_rcp(a1 + a2 + a3);
    return (a1 * p1 + a2 * p2 + a3 * p3) * inv;
}

__device__ __forceinline__ double minbee_lim(double c, double dl, double dm, double dr)
{
    const double heps = 1.0e-30;
    const double r = (c >= 0.0) ? dl / (dm + heps) : dr / (dm + heps);
    if (r <= 0.0) return 1.0;
    if (r <= 1.0) return 1.0 - (1.0 - fabs(c)) * r;
    return fabs(c);
}

__device__ __forceinline__ double waf_flux(double vL, double vR, double pLm1, double pL,
                                           double pR, double pRp1, double dxmin, double dt)
{
    const double vm = 0.5 * (vL + vR);
    const double sgn = copysign(1.0, vm);
    const double c = vm * dt / dxmin;
    const double fL = pL * vL, fR = pR * vR;
    const double lim = minbee_lim(c, pL - pLm1, pR - pL, pRp1 - pR);
    return 0.5 * (fL + fR) - 0.5 * sgn * lim * (fR - fL);
}

__device__ __forceinline__ double upwind_flux(double vL, double vR, double pL, double pR)
{
    const double vm = 0.5 * (vL + vR);
    const double sgn = copysign(1.0, vm);
    return pL * vL * 0.5 * (1.0 + sgn) + pR * vR * 0.5 * (1.0 - sgn);
}

// Face flux from the six cells around the face (u0..u5 = cells face-3 ..
// face+2, v0..v5 their drift velocities).  Inlined at its call sites: at 256^3
// the explicit kernel ran 9% faster inlined (80 registers, 3 CTAs of 256 per
// SM) than calling one shared out-of-line copy.  Defining
// VD_FACE_FLUX_NOINLINE restores the shared copy.
#ifdef VD_FACE_FLUX_NOINLINE
#define VD_FACE_FLUX_ATTR __noinline__
#else
#define VD_FACE_FLUX_ATTR __forceinline__
#endif
__device__ VD_FACE_FLUX_ATTR double face_flux_v(double u0, double u1, double u2, double u3,
                                           double u4, double u5, double v0, double v1,
                                           double v2, double v3, double v4, double v5,
                                           int hyp_order, int weno_scheme, double dxmin,
                                           double dt)
{
    if (hyp_order == 1) return upwind_flux(v2, v3, u2, u3);
    if (hyp_order == 2) return waf_flux(v2, v3, u1, u2, u3, u4, dxmin, dt);
    const double f0 = u0 * v0, f1 = u1 * v1, f2 = u2 * v2, f3 = u3 * v3, f4 = u4 * v4,
                 f5 = u5 * v5;
    const double lam = fabs(0.5 * (v2 + v3));
    const double fph = weno5(f0, f1, f2, f3, f4, weno_scheme);
    const double fmh = weno5(f5, f4, f3, f2, f1, weno_scheme);
    const double uph = weno5(u0, u1, u2, u3, u4, weno_scheme);
    const double umh = weno5(u5, u4, u3, u2, u1, weno_scheme);
    return 0.5 * (fph + lam * uph) + 0.5 * (fmh - lam * umh);
}

__device__ __forceinline__ double face_flux6(const double* u, const double* v, int hyp_order,
                                             int weno_scheme, double dxmin, double dt)
{
    return face_flux_v(u[0], u[1], u[2], u[3], u[4], u[5], v[0], v[1], v[2], v[3], v[4], v[5],
                       hyp_order, weno_scheme, dxmin, dt);
}

} // namespace vd
