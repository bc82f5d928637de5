// Discrete adjoint of N explicit flux + source steps (sm_100a, FP64).
//
// Forward map (per step, every transported species s, i.e. every species
// that is not a background species):
//     u_s <- u_s + dt * ( sum_d (F_d,lo - F_d,hi)/dx_d + N_A wdot_s(u; theta) )
// F is the drift flux of the main path (WENO5/WAF/upwind, the formulas of
// Source/compute_explicit_flux.H:16-214) with cell velocities
// v = mu_s(Te, n_total, |E|) E_d (electron mobility times the scale p_mob),
// ghost densities and velocities by clamping to the boundary cell (periodic
// wrap in periodic directions), and zero flux on walls whose species BC is
// IHNEUBC or AXISBC.  E and Te are frozen at their values in the state when
// the run starts; background species are frozen too.  wdot is the case's
// mechanism with the log pre-factors shifted by theta (A_r -> A_r e^theta_r).
// Objective J = sum over cells of n_e dV after the last step.
//
// The forward step runs as the chemistry (k_adj_chem_step) and one line
// march per direction (k_adj_flux_line: each face flux formed once); the
// one-kernel form k_adj_step is kept for comparison.
//
// Backward step k (lambda = dJ/du^{k+1}, states recomputed from checkpoints):
//     lambda <- lambda + dt (dR/du)^T lambda,   g <- g + dt (dR/dp)^T lambda
// evaluated at u^k.  WENO: one thread per segment of a line of faces and
// species marches the faces (k_adj_faces_line), differentiates each flux
// from the 5-slot dual gradient of each of its four reconstructions
// (weno_face_flux_grad) and writes each cell's sum of w dF/du_m once,
// w = dt (lambda_R - lambda_L)/dx.  Upwind and WAF: one thread per face
// (k_adj_faces), dual numbers, one pass for the stencil densities and one
// for the velocities, scattered with FP64 atomics.
// Stencil positions that clamp onto the same boundary cell are seeded as one
// direction: the WENO smoothness indicators of such a flat sub-stencil are
// zero only up to rounding, and per-position derivatives of that rounding
// residue (amplified by 1/(beta + eps)) swamp the true derivative, whereas
// moving the copies together keeps the residue's derivative exactly zero; the velocities' dependence on the total density goes through
// dmu/dn (a one-direction dual through the mobility hook); the chemistry
// Jacobian comes from one-direction dual evaluations of the mechanism per
// transported species; the pre-factor gradient uses dq_r/dtheta_r = q_r and
// the mechanism's transposed stoichiometry.
#pragma once

#include "vd_dual.H"
#include "vd_kernels.cuh"

namespace vd {

// ---- the flux formulas of vd_flux.cuh on a generic number type
template <class R>
__device__ __forceinline__ R weno5_T(const R& a, const R& b, const R& c, const R& d, const R& e,
                                     int scheme)
{
    const double eps = 1e-20;
    const R p1 = (1.0 / 3.0) * a - (7.0 / 6.0) * b + (11.0 / 6.0) * c;
    const R p2 = -(1.0 / 6.0) * b + (5.0 / 6.0) * c + (1.0 / 3.0) * d;
    const R p3 = (1.0 / 3.0) * c + (5.0 / 6.0) * d - (1.0 / 6.0) * e;
    const R s1 = a - 2.0 * b + c, s1b = a - 4.0 * b + 3.0 * c;
    const R s2 = b - 2.0 * c + d, s2b = b - d;
    const R s3 = c - 2.0 * d + e, s3b = 3.0 * c - 4.0 * d + e;
    const R b1 = (13.0 / 12.0) * s1 * s1 + 0.25 * s1b * s1b;
    const R b2 = (13.0 / 12.0) * s2 * s2 + 0.25 * s2b * s2b;
    const R b3 = (13.0 / 12.0) * s3 * s3 + 0.25 * s3b * s3b;
    R a1, a2, a3;
    if (scheme == 3)
    {
        const R tau = fabs(b1 - b3);
        const R r1 = tau / (b1 + eps), r2 = tau / (b2 + eps), r3 = tau / (b3 + eps);
        a1 = 0.1 * (1.0 + r1 * r1);
        a2 = 0.6 * (1.0 + r2 * r2);
        a3 = 0.3 * (1.0 + r3 * r3);
    } else
    {
        const R q1 = b1 + eps, q2 = b2 + eps, q3 = b3 + eps;
        a1 = 0.1 / (q1 * q1);
        a2 = 0.6 / (q2 * q2);
        a3 = 0.3 / (q3 * q3);
        if (scheme == 2)
        {
            const R sum = a1 + a2 + a3;
            const R w1 = a1 / sum, w2 = a2 / sum, w3 = a3 / sum;
            a1 = w1 * (0.1 + 0.01 - 0.3 * w1 + w1 * w1) / (0.01 + w1 * (1.0 - 0.2));
            a2 = w2 * (0.6 + 0.36 - 1.8 * w2 + w2 * w2) / (0.36 + w2 * (1.0 - 1.2));
            a3 = w3 * (0.3 + 0.09 - 0.9 * w3 + w3 * w3) / (0.09 + w3 * (1.0 - 0.6));
        }
    }
    return (a1 * p1 + a2 * p2 + a3 * p3) / (a1 + a2 + a3);
}

template <class R>
__device__ __forceinline__ R face_flux_T(const R* u, const R* v, int hyp_order,
                                         int weno_scheme, double dxmin, double dt)
{
    if (hyp_order == 1)
    {
        const double sgn = copysign(1.0, 0.5 * (value(v[2]) + value(v[3])));
        return u[2] * v[2] * (0.5 * (1.0 + sgn)) + u[3] * v[3] * (0.5 * (1.0 - sgn));
    }
    if (hyp_order == 2)
    {
        const R vm = 0.5 * (v[2] + v[3]);
        const double sgn = copysign(1.0, value(vm));
        const R c = vm * dt / dxmin;
        const R fL = u[2] * v[2], fR = u[3] * v[3];
        const R dl = u[2] - u[1], dm = u[3] - u[2], dr = u[4] - u[3];
        const R rr = (value(c) >= 0.0) ? dl / (dm + 1.0e-30) : dr / (dm + 1.0e-30);
        R lim;
        if (value(rr) <= 0.0)
            lim = R(1.0);
        else if (value(rr) <= 1.0)
            lim = 1.0 - (1.0 - fabs(c)) * rr;
        else
            lim = fabs(c);
        return 0.5 * (fL + fR) - 0.5 * sgn * lim * (fR - fL);
    }
    const R lam = fabs(0.5 * (v[2] + v[3]));
    const R fph = weno5_T(u[0] * v[0], u[1] * v[1], u[2] * v[2], u[3] * v[3], u[4] * v[4],
                          weno_scheme);
    const R fmh = weno5_T(u[5] * v[5], u[4] * v[4], u[3] * v[3], u[2] * v[2], u[1] * v[1],
                          weno_scheme);
    const R uph = weno5_T(u[0], u[1], u[2], u[3], u[4], weno_scheme);
    const R umh = weno5_T(u[5], u[4], u[3], u[2], u[1], weno_scheme);
    return 0.5 * (fph + lam * uph) + 0.5 * (fmh - lam * umh);
}

// Value and gradient of one WENO5 reconstruction with respect to its five
// cells (forward mode over 5 slots).  Arguments that are one cell (stencil
// positions clamped onto the same boundary cell) share the slot of the first
// of them, grp[k] <= k, so they move together: the smoothness indicator of a
// flat sub-stencil then has an exactly zero derivative, instead of
// per-position derivatives of its rounding residue, amplified by
// 1/(beta + eps)^2, that do not cancel.  g[k] is set for k == grp[k].
__device__ __forceinline__ double weno5_grad(const double* x, const int* grp, int scheme,
                                             double* g)
{
    const Dual<5> W = weno5_T(Dual<5>::var_sel(x[0], grp[0]), Dual<5>::var_sel(x[1], grp[1]),
                              Dual<5>::var_sel(x[2], grp[2]), Dual<5>::var_sel(x[3], grp[3]),
                              Dual<5>::var_sel(x[4], grp[4]), scheme);
#pragma unroll
    for (int k = 0; k < 5; ++k) g[k] = W.d[k];
    return W.v;
}

// Derivatives of the WENO face flux (face_flux_T, hyp_order > 2) with respect
// to the densities (du) and drift velocities (dv) of the cells of its
// stencil, accumulated at each cell's first stencil position (dir[m]: the
// first position clamped onto the cell of position m).  With f_m = u_m v_m
// and lam = |(v_2 + v_3)/2|:
//   F = (fph + lam uph)/2 + (fmh - lam umh)/2,
//   dF/du = dF/df v + lam (duph/du - dumh/du)/2,
//   dF/dv = dF/df u + (uph - umh)/2 dlam/dv   (dlam/dv only at positions 2, 3).
// Four 5-slot reconstructions instead of the two passes of four 6-slot ones
// that differentiate face_flux_T in dual numbers; the same derivatives up to
// rounding, with the same seeding of clamped positions.  ID: no position is
// clamped (dir[m] == m, an interior face), so every slot and output index is
// a compile-time constant and the duals stay in registers.
template <bool ID = false>
__device__ __forceinline__ void weno_face_flux_grad(const double* u, const double* v,
                                                    const int* dir, int scheme, double* du,
                                                    double* dv)
{
    // argument positions of the reconstructions: fph, uph over 0..4; fmh, umh
    // over 5, 4, 3, 2, 1; and each argument's slot (its group's first argument)
    const int pp[5] = {0, 1, 2, 3, 4}, pm[5] = {5, 4, 3, 2, 1};
    int gpp[5], gpm[5];
#pragma unroll
    for (int k = 0; k < 5; ++k)
    {
        gpp[k] = k;
        gpm[k] = k;
        for (int q = k - 1; q >= 0 && !ID; --q)
        {
            if (dir[pp[q]] == dir[pp[k]]) gpp[k] = gpp[q];
            if (dir[pm[q]] == dir[pm[k]]) gpm[k] = gpm[q];
        }
    }
    double xf[5], xu[5], yf[5], yu[5];
#pragma unroll
    for (int k = 0; k < 5; ++k)
    {
        xf[k] = u[pp[k]] * v[pp[k]];
        xu[k] = u[pp[k]];
        yf[k] = u[pm[k]] * v[pm[k]];
        yu[k] = u[pm[k]];
    }
    double gfp[5], gfm[5], gup[5], gum[5];
    weno5_grad(xf, gpp, scheme, gfp);
    weno5_grad(yf, gpm, scheme, gfm);
    const double uph = weno5_grad(xu, gpp, scheme, gup);
    const double umh = weno5_grad(yu, gpm, scheme, gum);
    const double vm = 0.5 * (v[2] + v[3]);
    const double lam = (vm < 0.0) ? -vm : vm, slam = (vm < 0.0) ? -1.0 : 1.0;
#pragma unroll
    for (int m = 0; m < 6; ++m) du[m] = dv[m] = 0.0;
#pragma unroll
    for (int k = 0; k < 5; ++k)
    {
        // output index c = dir[m] by a select per position (an indexed
        // update would put du, dv in local memory)
        if (ID || gpp[k] == k)
        {
            const int m = pp[k], c = ID ? m : dir[m];
            const double a = 0.5 * gfp[k] * v[m] + 0.5 * lam * gup[k], b = 0.5 * gfp[k] * u[m];
#pragma unroll
            for (int q = 0; q < 6; ++q)
                if (q == c)
                {
                    du[q] += a;
                    dv[q] += b;
                }
        }
        if (ID || gpm[k] == k)
        {
            const int m = pm[k], c = ID ? m : dir[m];
            const double a = 0.5 * gfm[k] * v[m] - 0.5 * lam * gum[k], b = 0.5 * gfm[k] * u[m];
#pragma unroll
            for (int q = 0; q < 6; ++q)
                if (q == c)
                {
                    du[q] += a;
                    dv[q] += b;
                }
        }
    }
    const double dl = 0.5 * (uph - umh) * slam * 0.5;
#pragma unroll
    for (int q = 0; q < 6; ++q)
    {
        if (q == (ID ? 2 : dir[2])) dv[q] += dl;
        if (q == (ID ? 3 : dir[3])) dv[q] += dl;
    }
}

#ifdef VD_HAS_MECH_ADJOINT

// columns of the chemistry Jacobian formed per dual pass (k_adj_chem_update):
// each pass recomputes the rate exponentials, more slots cost registers;
// measured at 128^3 / 50 steps (LMEA): 1, 2, 3 slots 545, 513, 513 ms per
// adjoint run (1, 2, 4, 8 slots 1033, 1002, 1048, 1038 ms with the earlier
// face and step kernels)
#ifndef VD_ADJ_CHEM_SLOTS
#define VD_ADJ_CHEM_SLOTS 2
#endif

struct AdjParams
{
    GridDev g; // natural layout
    double dx[3];
    double dt, dxmin, Tg, mob_scale;
    int hyp_order, weno_scheme;
    int nt;                // transported species
    int spec[NUM_SPECIES]; // their component indices, ascending
    int eslot;             // slot of the electrons among them
    int bclo[NUM_SPECIES][3], bchi[NUM_SPECIES][3];
    const double* S;     // frozen state: E, Te, background species
    const double* theta; // log pre-factor shifts (device, NUM_REACTIONS)
    double* mu;          // nt x N mobilities (times the scale for electrons)
    double* dmu;         // nt x N d mobility / d total density
};

__device__ __forceinline__ long long adj_cidx(const GridDev& g, int i, int j, int k)
{
    return g.idx(clampi(i, g.n[0], g.per[0]), clampi(j, g.n[1], g.per[1]),
                 clampi(k, g.n[2], g.per[2]));
}

__device__ __forceinline__ bool adj_wall(const AdjParams& P, int s, int d, bool hi)
{
    return !P.g.per[d] && wall_zero(hi ? P.bchi[s][d] : P.bclo[s][d]);
}

// Mobilities and their density derivatives of every transported species.
__global__ void __launch_bounds__(256) k_adj_props(AdjParams P, const double* __restrict__ u)
{
    VD_PDL_WAIT();
    const long long N = P.g.ncell();
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < N;
         q += (long long)gridDim.x * blockDim.x)
    {
        const double ex = P.S[EFX_ID * N + q], ey = P.S[EFY_ID * N + q], ez = P.S[EFZ_ID * N + q];
        const double em = ::sqrt(ex * ex + ey * ey + ez * ez);
        const double te = P.S[ETEMP_ID * N + q];
        double nd = 0.0;
        int slot = 0;
        for (int sp = 0; sp < NUM_SPECIES; ++sp)
        {
            if (slot < P.nt && P.spec[slot] == sp)
                nd += u[(slot++) * N + q];
            else
                nd += P.S[sp * N + q];
        }
        for (int s = 0; s < P.nt; ++s)
        {
            const Dual<1> m = specMob_T<Dual<1>>(P.spec[s], Dual<1>(te), Dual<1>::var(nd, 0),
                                                 Dual<1>(em), P.Tg);
            const double sc = (s == P.eslot) ? P.mob_scale : 1.0;
            P.mu[s * N + q] = m.v * sc;
            P.dmu[s * N + q] = m.d[0] * sc;
        }
    }
}

// One forward step: unew = u + dt R(u).
__global__ void __launch_bounds__(256) k_adj_step(AdjParams P, const double* __restrict__ u,
                                                  double* __restrict__ unew)
{
    VD_PDL_WAIT();
    const GridDev& g = P.g;
    const long long N = g.ncell();
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < N;
         t += (long long)gridDim.x * blockDim.x)
    {
        int c3[3];
        cell_of(g, t, c3[0], c3[1], c3[2]);
        double C[NUM_SPECIES], q[NUM_REACTIONS], W[NUM_SPECIES];
        int slot = 0;
        for (int sp = 0; sp < NUM_SPECIES; ++sp)
        {
            const bool tr = slot < P.nt && P.spec[slot] == sp;
            C[sp] = (tr ? u[slot * N + t] : P.S[sp * N + t]) / N_A;
            if (tr) ++slot;
        }
        mech_rates<double>(P.Tg, C, P.S[ETEMP_ID * N + t], P.theta, q);
        mech_wdot<double>(q, W);
        for (int s = 0; s < P.nt; ++s)
        {
            double acc = 0.0;
            for (int d = 0; d < g.dim; ++d)
            {
                double uu[7], vv[7];
                for (int m = 0; m < 7; ++m)
                {
                    int c[3] = {c3[0], c3[1], c3[2]};
                    c[d] += m - 3;
                    const long long qq = adj_cidx(g, c[0], c[1], c[2]);
                    uu[m] = u[s * N + qq];
                    vv[m] = P.mu[s * N + qq] * P.S[(EFX_ID + d) * N + qq];
                }
                double flo = face_flux6(uu, vv, P.hyp_order, P.weno_scheme, P.dxmin, P.dt);
                double fhi = face_flux6(uu + 1, vv + 1, P.hyp_order, P.weno_scheme, P.dxmin, P.dt);
                if (c3[d] == 0 && adj_wall(P, s, d, false)) flo = 0.0;
                if (c3[d] == g.n[d] - 1 && adj_wall(P, s, d, true)) fhi = 0.0;
                acc += (flo - fhi) / P.dx[d];
            }
            unew[s * N + t] = u[s * N + t] + P.dt * (acc + W[P.spec[s]] * N_A);
        }
    }
}

// The same step in two parts, each face flux computed once.  Part 1, the
// chemistry: unew = u + dt N_A wdot(u).
__global__ void __launch_bounds__(256) k_adj_chem_step(AdjParams P, const double* __restrict__ u,
                                                       double* __restrict__ unew)
{
    VD_PDL_WAIT();
    const long long N = P.g.ncell();
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < N;
         t += (long long)gridDim.x * blockDim.x)
    {
        double C[NUM_SPECIES], q[NUM_REACTIONS], W[NUM_SPECIES];
        int slot = 0;
        for (int sp = 0; sp < NUM_SPECIES; ++sp)
        {
            const bool tr = slot < P.nt && P.spec[slot] == sp;
            C[sp] = (tr ? u[slot * N + t] : P.S[sp * N + t]) / N_A;
            if (tr) ++slot;
        }
        mech_rates<double>(P.Tg, C, P.S[ETEMP_ID * N + t], P.theta, q);
        mech_wdot<double>(q, W);
        for (int s = 0; s < P.nt; ++s) unew[s * N + t] = u[s * N + t] + P.dt * (W[P.spec[s]] * N_A);
    }
}

// Part 2, direction d: unew += dt (F_lo - F_hi)/dx_d, one thread per
// segment of a line of cells along d and species (nseg segments a line, so
// that the launch fills its last wave), marching the faces with the six
// stencil cells' u, v in registers (ghost positions clamped or wrapped as in
// k_adj_step); each face's flux is formed once and closes the cell on its
// left.  A segment of cells c0..c1-1 forms faces c0..c1 (one face more than
// its cells, shared with the next segment) and is the only writer of its
// cells.
__global__ void __launch_bounds__(128) k_adj_flux_line(AdjParams P, int d, int nseg,
                                                       const double* __restrict__ u,
                                                       double* __restrict__ unew)
{
    VD_PDL_WAIT();
    const GridDev& g = P.g;
    const long long N = g.ncell();
    const int n = g.n[d], per = g.per[d];
    const int da = d == 0 ? 1 : 0, db = d == 2 ? 1 : 2;
    const long long sd = d == 0 ? 1LL : (d == 1 ? (long long)g.n[0] : (long long)g.n[0] * g.n[1]);
    const long long lines = (long long)g.n[da] * g.n[db];
    const double* __restrict__ E = P.S + (EFX_ID + d) * N;
    const double cdt = P.dt / P.dx[d];
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
         t < lines * nseg * P.nt; t += (long long)gridDim.x * blockDim.x)
    {
        const int s = (int)(t / (lines * nseg));
        const long long r = t - s * lines * nseg;
        const int seg = (int)(r / lines);
        const long long l = r - seg * lines;
        const int c0 = (int)((long long)seg * n / nseg), c1 = (int)((long long)(seg + 1) * n / nseg);
        int c[3];
        c[d] = 0;
        c[da] = (int)(l % g.n[da]);
        c[db] = (int)(l / g.n[da]);
        const long long base = g.idx(c[0], c[1], c[2]);
        const double* __restrict__ us = u + s * N;
        const double* __restrict__ ms = P.mu + s * N;
        double* __restrict__ un = unew + s * N;
        const bool wlo = adj_wall(P, s, d, false), whi = adj_wall(P, s, d, true);
        double wu[6], wv[6];
#pragma unroll
        for (int m = 0; m < 6; ++m)
        {
            const long long q = base + clampi(c0 - 3 + m, n, per) * sd;
            wu[m] = us[q];
            wv[m] = ms[q] * E[q];
        }
        double Fprev = 0.0;
        for (int f = c0; f <= c1; ++f)
        {
            double F = face_flux6(wu, wv, P.hyp_order, P.weno_scheme, P.dxmin, P.dt);
            if ((f == 0 && wlo) || (f == n && whi)) F = 0.0;
            if (f > c0)
            {
                const long long q = base + (long long)(f - 1) * sd;
                un[q] += cdt * (Fprev - F);
            }
            Fprev = F;
            if (f == c1) break;
#pragma unroll
            for (int m = 0; m < 5; ++m)
            {
                wu[m] = wu[m + 1];
                wv[m] = wv[m + 1];
            }
            const long long q = base + clampi(f + 3, n, per) * sd;
            wu[5] = us[q];
            wv[5] = ms[q] * E[q];
        }
    }
}

// Adjoint of the face fluxes of direction d: one thread per face.
__global__ void __launch_bounds__(128) k_adj_faces(AdjParams P, int d,
                                                   const double* __restrict__ u,
                                                   const double* __restrict__ lam,
                                                   double* __restrict__ adj,
                                                   double* __restrict__ adjnd, double* gmob)
{
    VD_PDL_WAIT();
    __shared__ double sh[32];
    const GridDev& g = P.g;
    const long long N = g.ncell();
    const int fn[3] = {g.n[0] + (d == 0), g.n[1] + (d == 1), g.n[2] + (d == 2)};
    const long long nf = (long long)fn[0] * fn[1] * fn[2];
    double gm = 0.0;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < nf;
         t += (long long)gridDim.x * blockDim.x)
    {
        int f3[3];
        f3[0] = (int)(t % fn[0]);
        f3[1] = (int)((t / fn[0]) % fn[1]);
        f3[2] = (int)(t / ((long long)fn[0] * fn[1]));
        if (g.per[d] && f3[d] == g.n[d]) continue; // the periodic wrap face is face 0
        // stencil cells; positions that clamp onto the same cell share one
        // derivative direction (dir[m] = first position of that cell)
        long long qm[6];
        int dir[6];
        for (int m = 0; m < 6; ++m)
        {
            int c[3] = {f3[0], f3[1], f3[2]};
            c[d] += m - 3;
            qm[m] = adj_cidx(g, c[0], c[1], c[2]);
            dir[m] = m;
            for (int q = m - 1; q >= 0; --q)
                if (qm[q] == qm[m]) dir[m] = dir[q];
        }
        const bool hasL = f3[d] > 0 || g.per[d];
        const bool hasR = f3[d] < g.n[d];
        for (int s = 0; s < P.nt; ++s)
        {
            if (f3[d] == 0 && adj_wall(P, s, d, false)) continue;
            if (f3[d] == g.n[d] && adj_wall(P, s, d, true)) continue;
            const double lL = hasL ? lam[s * N + qm[2]] : 0.0;
            const double lR = hasR ? lam[s * N + qm[3]] : 0.0;
            const double w = P.dt * (lR - lL) / P.dx[d];
            if (w == 0.0) continue;
            double uv[6], vv[6];
            for (int m = 0; m < 6; ++m)
            {
                uv[m] = u[s * N + qm[m]];
                vv[m] = P.mu[s * N + qm[m]] * P.S[(EFX_ID + d) * N + qm[m]];
            }
            if (P.hyp_order > 2)
            {
                // WENO: both derivative sets from one gradient per
                // reconstruction, at each cell's first stencil position
                double au[6], av[6];
                weno_face_flux_grad(uv, vv, dir, P.weno_scheme, au, av);
                for (int m = 0; m < 6; ++m)
                {
                    if (dir[m] != m) continue;
                    if (au[m] != 0.0) atomicAdd(&adj[s * N + qm[m]], w * au[m]);
                    if (av[m] == 0.0) continue;
                    const double e = P.S[(EFX_ID + d) * N + qm[m]];
                    const double dn = P.dmu[s * N + qm[m]] * e;
                    if (dn != 0.0) atomicAdd(&adjnd[qm[m]], w * av[m] * dn);
                    if (s == P.eslot) gm += w * av[m] * vv[m];
                }
                continue;
            }
            {
                Dual<6> U[6], V[6];
                for (int m = 0; m < 6; ++m)
                {
                    U[m] = Dual<6>::var(uv[m], dir[m]);
                    V[m] = Dual<6>(vv[m]);
                }
                const Dual<6> F = face_flux_T(U, V, P.hyp_order, P.weno_scheme, P.dxmin, P.dt);
                for (int m = 0; m < 6; ++m)
                    if (dir[m] == m && F.d[m] != 0.0) atomicAdd(&adj[s * N + qm[m]], w * F.d[m]);
            }
            {
                Dual<6> U[6], V[6];
                for (int m = 0; m < 6; ++m)
                {
                    U[m] = Dual<6>(uv[m]);
                    V[m] = Dual<6>::var(vv[m], dir[m]);
                }
                const Dual<6> F = face_flux_T(U, V, P.hyp_order, P.weno_scheme, P.dxmin, P.dt);
                for (int m = 0; m < 6; ++m)
                {
                    if (dir[m] != m || F.d[m] == 0.0) continue;
                    const double e = P.S[(EFX_ID + d) * N + qm[m]];
                    const double dn = P.dmu[s * N + qm[m]] * e;
                    if (dn != 0.0) atomicAdd(&adjnd[qm[m]], w * F.d[m] * dn);
                    if (s == P.eslot) gm += w * F.d[m] * vv[m];
                }
            }
        }
    }
    gm = block_sum(gm, sh);
    if (threadIdx.x == 0 && gm != 0.0) atomicAdd(gmob, gm / P.mob_scale);
}

// Adjoint of the WENO face fluxes of direction d (hyp_order > 2): one thread
// per line of faces along d and species.  The thread marches its line with
// the six stencil cells' u, v and their accumulated w dF/du, w dF/dv in
// registers (position m of face f is the virtual cell f-3+m; ghost positions
// read the clamped or wrapped cell, as k_adj_faces does) and writes each
// cell's totals once, when it leaves the stencil: adj by a plain add (no
// other thread of the launch reaches this species' cells of the line),
// adjnd, which every species shares, by an atomic add.  The derivatives are
// k_adj_faces' (weno_face_flux_grad with the same grouping of clamped
// positions), summed per cell before the product with dmu E; each new face
// loads one new cell instead of six.
__device__ __forceinline__ void adj_line_flush(double* __restrict__ as, double* __restrict__ adjnd,
                                               const double* __restrict__ dms,
                                               const double* __restrict__ E, long long q,
                                               double au, double av, double v, bool elec,
                                               bool seam, double& gm)
{
    if (au != 0.0)
    {
        if (seam)
            atomicAdd(&as[q], au);
        else
            as[q] += au;
    }
    if (av == 0.0) return;
    const double dn = dms[q] * E[q];
    if (dn != 0.0) atomicAdd(&adjnd[q], av * dn);
    if (elec) gm += av * v;
}

// Blocks per SM the face adjoint's registers are sized for: 3 (168
// registers, about 0.5 KB of spills) beats 2 (242, none) and 4 (128, 1.2 KB)
// at 128^3: 496, 510, 521 ms per adjoint run.
#ifndef VD_ADJ_FACES_MINB
#define VD_ADJ_FACES_MINB 3
#endif
__global__ void __launch_bounds__(128, VD_ADJ_FACES_MINB) k_adj_faces_line(AdjParams P, int d, int nseg,
                                                        const double* __restrict__ u,
                                                        const double* __restrict__ lam,
                                                        double* __restrict__ adj,
                                                        double* __restrict__ adjnd, double* gmob)
{
    VD_PDL_WAIT();
    __shared__ double sh[32];
    const GridDev& g = P.g;
    const long long N = g.ncell();
    const int n = g.n[d], per = g.per[d];
    // the line's other two axes: da varies fastest between threads (x for
    // d = y, z: coalesced)
    const int da = d == 0 ? 1 : 0, db = d == 2 ? 1 : 2;
    const long long sd = d == 0 ? 1LL : (d == 1 ? (long long)g.n[0] : (long long)g.n[0] * g.n[1]);
    const long long lines = (long long)g.n[da] * g.n[db];
    const double* __restrict__ E = P.S + (EFX_ID + d) * N;
    const int nf = per ? n : n + 1; // the periodic wrap face is face 0
    double gm = 0.0;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
         t < lines * nseg * P.nt; t += (long long)gridDim.x * blockDim.x)
    {
        const int s = (int)(t / (lines * nseg));
        const long long r = t - s * lines * nseg;
        const int seg = (int)(r / lines);
        const long long l = r - seg * lines;
        // faces f0..f1-1 of the line; the five cells at either end of the
        // segment also take contributions from the neighbouring segments
        // (through the wrap in periodic lines): atomic adds there
        const int f0 = (int)((long long)seg * nf / nseg), f1 = (int)((long long)(seg + 1) * nf / nseg);
        const bool seams = nseg > 1;
        int c[3];
        c[d] = 0;
        c[da] = (int)(l % g.n[da]);
        c[db] = (int)(l / g.n[da]);
        const long long base = g.idx(c[0], c[1], c[2]);
        const double* __restrict__ us = u + s * N;
        const double* __restrict__ ms = P.mu + s * N;
        const double* __restrict__ ls = lam + s * N;
        const double* __restrict__ dms = P.dmu + s * N;
        double* __restrict__ as = adj + s * N;
        const bool wlo = adj_wall(P, s, d, false), whi = adj_wall(P, s, d, true);
        const bool elec = s == P.eslot;
        double wu[6], wv[6], au[6], av[6];
#pragma unroll
        for (int m = 0; m < 6; ++m)
        {
            const long long q = base + clampi(f0 - 3 + m, n, per) * sd;
            wu[m] = us[q];
            wv[m] = ms[q] * E[q];
            au[m] = av[m] = 0.0;
        }
        // lambda of the cells left and right of face f (0 outside a wall)
        double lL = (f0 > 0 || per) ? ls[base + (long long)clampi(f0 - 1, n, per) * sd] : 0.0;
        double lR = (f0 < n) ? ls[base + (long long)f0 * sd] : 0.0;
        for (int f = f0; f < f1; ++f)
        {
            int rc[6], dir[6];
#pragma unroll
            for (int m = 0; m < 6; ++m)
            {
                rc[m] = clampi(f - 3 + m, n, per);
                dir[m] = m;
#pragma unroll
                for (int q = m - 1; q >= 0; --q)
                    if (rc[q] == rc[m]) dir[m] = dir[q];
            }
            const bool wall = (f == 0 && wlo) || (f == n && whi);
            const double w = P.dt * (lR - lL) / P.dx[d];
            // no stencil position clamped or wrapped onto another's cell: the
            // gradient with constant slots (its arrays stay in registers)
            const bool inner = per ? n >= 6 : (f >= 3 && f + 2 < n);
            if (!wall && w != 0.0 && inner)
            {
                double gu[6], gv[6];
                weno_face_flux_grad<true>(wu, wv, dir, P.weno_scheme, gu, gv);
#pragma unroll
                for (int m = 0; m < 6; ++m)
                {
                    au[m] += w * gu[m];
                    av[m] += w * gv[m];
                }
            } else if (!wall && w != 0.0)
            {
                double gu[6], gv[6];
                weno_face_flux_grad<false>(wu, wv, dir, P.weno_scheme, gu, gv);
#pragma unroll
                for (int m = 0; m < 6; ++m)
                    if (dir[m] == m)
                    {
                        au[m] += w * gu[m];
                        av[m] += w * gv[m];
                    }
            }
            // virtual cell f-3 leaves the stencil; f+3 enters
            adj_line_flush(as, adjnd, dms, E, base + rc[0] * sd, au[0], av[0], wv[0], elec,
                           seams && f - f0 < 5, gm);
#pragma unroll
            for (int m = 0; m < 5; ++m)
            {
                wu[m] = wu[m + 1];
                wv[m] = wv[m + 1];
                au[m] = au[m + 1];
                av[m] = av[m + 1];
            }
            const long long q = base + clampi(f + 3, n, per) * sd;
            wu[5] = us[q];
            wv[5] = ms[q] * E[q];
            au[5] = av[5] = 0.0;
            lL = lR;
            lR = (f + 1 < n) ? ls[base + (long long)(f + 1) * sd] : (per ? ls[base] : 0.0);
        }
        // virtual cells f1-3 .. f1+1 are still in the window
#pragma unroll
        for (int m = 0; m < 5; ++m)
            adj_line_flush(as, adjnd, dms, E, base + clampi(f1 - 3 + m, n, per) * sd, au[m],
                           av[m], wv[m], elec, seams, gm);
    }
    gm = block_sum(gm, sh);
    if (threadIdx.x == 0 && gm != 0.0) atomicAdd(gmob, gm / P.mob_scale);
}

// Adjoint of the chemistry, then the adjoint update of the step:
//   lambda_s <- lambda_s + dt (dW/dC)^T lambda + adj_s + adjnd
// (adj: the flux terms, adjnd: the density term of the mobilities, shared by
// every transported species since n_total sums them).
__global__ void __launch_bounds__(128) k_adj_chem_update(AdjParams P,
                                                         const double* __restrict__ u,
                                                         double* __restrict__ lam,
                                                         const double* __restrict__ adj,
                                                         const double* __restrict__ adjnd,
                                                         double* gtheta)
{
    VD_PDL_WAIT();
    __shared__ double sh[32];
    // the thread's pre-factor gradient sums, in shared memory: 30 registers
    // pairs fewer for the dual passes
    __shared__ double gl[NUM_REACTIONS][128];
    for (int r = 0; r < NUM_REACTIONS; ++r) gl[r][threadIdx.x] = 0.0;
    const long long N = P.g.ncell();
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < N;
         t += (long long)gridDim.x * blockDim.x)
    {
        const double te = P.S[ETEMP_ID * N + t];
        double Cv[NUM_SPECIES], lamc[NUM_SPECIES];
        int slot = 0;
        for (int sp = 0; sp < NUM_SPECIES; ++sp)
        {
            const bool tr = slot < P.nt && P.spec[slot] == sp;
            Cv[sp] = (tr ? u[slot * N + t] : P.S[sp * N + t]) / N_A;
            lamc[sp] = tr ? lam[slot * N + t] : 0.0;
            if (tr) ++slot;
        }
        // pre-factor gradient: dR_s/dtheta_r = N_A nu_sr q_r
        {
            double q[NUM_REACTIONS], ln[NUM_REACTIONS];
            mech_rates<double>(P.Tg, Cv, te, P.theta, q);
            mech_lam_nu(lamc, ln);
            for (int r = 0; r < NUM_REACTIONS; ++r) gl[r][threadIdx.x] += P.dt * N_A * q[r] * ln[r];
        }
        // dR_s/du_s2 = d wdot_s / d C_s2 (R = N_A wdot, C = u / N_A),
        // VD_ADJ_CHEM_SLOTS columns per pass
        const double nd = adjnd[t];
        constexpr int K = VD_ADJ_CHEM_SLOTS;
        for (int s0 = 0; s0 < P.nt; s0 += K)
        {
            Dual<K> C[NUM_SPECIES], q[NUM_REACTIONS], W[NUM_SPECIES];
            // seeds by selects (an index known only at run time would put
            // the duals in local memory)
#pragma unroll
            for (int sp = 0; sp < NUM_SPECIES; ++sp)
            {
                C[sp] = Dual<K>(Cv[sp]);
#pragma unroll
                for (int e = 0; e < K; ++e)
                    if (s0 + e < P.nt && P.spec[s0 + e] == sp) C[sp].d[e] = 1.0;
            }
            mech_rates<Dual<K>>(P.Tg, C, te, P.theta, q);
            mech_wdot<Dual<K>>(q, W);
            for (int e = 0; e < K && s0 + e < P.nt; ++e)
            {
                const int s2 = s0 + e;
                double a = 0.0;
                for (int sp = 0; sp < NUM_SPECIES; ++sp) a += lamc[sp] * W[sp].d[e];
                // lamc[P.spec[s2]], read back from memory (not yet rewritten)
                lam[s2 * N + t] = lam[s2 * N + t] + P.dt * a + adj[s2 * N + t] + nd;
            }
        }
    }
    for (int r = 0; r < NUM_REACTIONS; ++r)
    {
        const double v = block_sum(gl[r][threadIdx.x], sh);
        if (threadIdx.x == 0 && v != 0.0) atomicAdd(&gtheta[r], v);
    }
}

#endif // VD_HAS_MECH_ADJOINT

// The objective sum_cells n_e dV is taken in double-double arithmetic
// (Knuth's TwoSum on every addition) with a fixed reduction order: per-block
// partials (hi, lo) first, then one block adds them up.  The result is the
// exactly rounded sum up to a few units in the last place and the same on
// every run, which central differences of the objective at h = 1e-6 need:
// the objective reaches 1e10 while its sensitivities are 1e2, so one ulp of
// J is worth ~2 in a difference quotient.
__device__ __forceinline__ void dd_add(double& hi, double& lo, double b)
{
    const double s = hi + b;
    const double bb = s - hi;
    lo += (hi - (s - bb)) + (b - bb);
    hi = s;
}

__device__ __forceinline__ void dd_add_dd(double& hi, double& lo, double bh, double bl)
{
    dd_add(hi, lo, bh);
    lo += bl;
    const double s = hi + lo;
    lo = lo - (s - hi);
    hi = s;
}

// Block-wide double-double sum in a fixed order; thread 0 gets the result.
__device__ __forceinline__ void dd_block_sum(double& hi, double& lo, double* sh)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int o = 16; o > 0; o >>= 1)
    {
        const double oh = __shfl_down_sync(0xffffffffu, hi, o);
        const double ol = __shfl_down_sync(0xffffffffu, lo, o);
        if (lane < o) dd_add_dd(hi, lo, oh, ol);
    }
    __syncthreads();
    if (lane == 0)
    {
        sh[2 * wid] = hi;
        sh[2 * wid + 1] = lo;
    }
    __syncthreads();
    if (threadIdx.x == 0)
    {
        const int nw = (blockDim.x + 31) >> 5;
        for (int w = 1; w < nw; ++w) dd_add_dd(hi, lo, sh[2 * w], sh[2 * w + 1]);
    }
}

// Stage 1: per-block partial sums of ue into part[2b], part[2b+1].
__global__ void k_adj_objective(long long n, const double* __restrict__ ue,
                                double* __restrict__ part)
{
    VD_PDL_WAIT();
    __shared__ double sh[64];
    double hi = 0.0, lo = 0.0;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
         t += (long long)gridDim.x * blockDim.x)
        dd_add(hi, lo, ue[t]);
    dd_block_sum(hi, lo, sh);
    if (threadIdx.x == 0)
    {
        part[2 * blockIdx.x] = hi;
        part[2 * blockIdx.x + 1] = lo;
    }
}

// Stage 2 (one block): J = dv * sum of the nb partials.
__global__ void k_adj_objective_final(int nb, const double* __restrict__ part, double dv,
                                      double* J)
{
    VD_PDL_WAIT();
    __shared__ double sh[64];
    double hi = 0.0, lo = 0.0;
    for (int b = threadIdx.x; b < nb; b += blockDim.x) dd_add_dd(hi, lo, part[2 * b], part[2 * b + 1]);
    dd_block_sum(hi, lo, sh);
    if (threadIdx.x == 0) *J = (hi + lo) * dv;
}

} // namespace vd
