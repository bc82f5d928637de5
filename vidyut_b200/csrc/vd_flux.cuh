// Drift-flux numerics on the device: WENO5 (JS / M / Z) reconstruction with
// the local Lax-Friedrichs split, the second-order WAF flux with the MINBEE
// limiter, and first-order upwind.  Same schemes and constants as the
// reference (Source/compute_explicit_flux.H:16-214, including the Rathan &
// Naga Raju WENO-M/Z weights), arranged for FP64 throughput: one reciprocal
// per weight normalisation instead of three divisions.
#pragma once

namespace vd {

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
    if (scheme == 3)
    {
        const double tau = fabs(b1 - b3);
        const double r1 = tau / (b1 + eps), r2 = tau / (b2 + eps), r3 = tau / (b3 + eps);
        a1 = 0.1 * (1.0 + r1 * r1);
        a2 = 0.6 * (1.0 + r2 * r2);
        a3 = 0.3 * (1.0 + r3 * r3);
    } else
    {
        const double q1 = b1 + eps, q2 = b2 + eps, q3 = b3 + eps;
        a1 = 0.1 / (q1 * q1);
        a2 = 0.6 / (q2 * q2);
        a3 = 0.3 / (q3 * q3);
        if (scheme == 2)
        {
            const double inv = 1.0 / (a1 + a2 + a3);
            const double w1 = a1 * inv, w2 = a2 * inv, w3 = a3 * inv;
            a1 = weno_gk(w1, 0.1);
            a2 = weno_gk(w2, 0.6);
            a3 = weno_gk(w3, 0.3);
        }
    }
    const double inv = 1.0 / (a1 + a2 + a3);
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

// Face flux from the six cells around the face (u[0..5] = cells face-3 ..
// face+2, v[] their drift velocities).
__device__ __forceinline__ double face_flux6(const double* u, const double* v, int hyp_order,
                                             int weno_scheme, double dxmin, double dt)
{
    if (hyp_order == 1) return upwind_flux(v[2], v[3], u[2], u[3]);
    if (hyp_order == 2) return waf_flux(v[2], v[3], u[1], u[2], u[3], u[4], dxmin, dt);
    const double f0 = u[0] * v[0], f1 = u[1] * v[1], f2 = u[2] * v[2], f3 = u[3] * v[3],
                 f4 = u[4] * v[4], f5 = u[5] * v[5];
    const double lam = fabs(0.5 * (v[2] + v[3]));
    const double fph = weno5(f0, f1, f2, f3, f4, weno_scheme);
    const double fmh = weno5(f5, f4, f3, f2, f1, weno_scheme);
    const double uph = weno5(u[0], u[1], u[2], u[3], u[4], weno_scheme);
    const double umh = weno5(u[5], u[4], u[3], u[2], u[1], weno_scheme);
    return 0.5 * (fph + lam * uph) + 0.5 * (fmh - lam * umh);
}

} // namespace vd
