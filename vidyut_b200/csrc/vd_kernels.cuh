// Per-step kernels of the species-and-field update (sm_100a, FP64):
// Poisson right-hand side, boundary callbacks, electric field, the fused
// reaction + drift-flux + divergence kernel, diffusion-solve set-up, Joule
// heating, and the state write-back.  Each cites the reference function
// whose arithmetic it reproduces.
#pragma once

#include "vd_mg.cuh"
#include "vd_flux.cuh"

// A reference case directory's boundary hooks take three integrated-current
// arrays more (vidyut_b200/compat defines them); otherwise nothing.
#ifndef VD_CURRENT_ARGS
#define VD_CURRENT_ARGS
#endif

namespace vd {

#define VD_NT (NUM_SPECIES + 1)

__host__ __device__ inline Array4 state_view(double* S, const GridDev& g)
{
    Array4 a;
    a.p = S;
    for (int d = 0; d < 3; ++d)
    {
        a.lo[d] = 0;
        a.hi[d] = g.n[d] - 1;
        a.periodic[d] = g.per[d];
    }
    a.jstride = g.n[0];
    a.kstride = (long long)g.n[0] * g.n[1];
    a.nstride = g.ncell();
    a.clamp = 1;
    return a;
}

// A view over one boundary side's plane of values, addressed by the ghost
// cell index the reference's hooks write (face-1 low side, face high side).
__host__ __device__ inline Array4 side_view(double* v, const GridDev& g, int s)
{
    const int d = s % 3;
    Array4 a;
    a.p = v;
    for (int q = 0; q < 3; ++q)
    {
        a.lo[q] = 0;
        a.hi[q] = g.n[q] - 1;
    }
    a.lo[d] = a.hi[d] = (s / 3) ? g.n[d] : -1;
    a.jstride = a.hi[0] - a.lo[0] + 1;
    a.kstride = a.jstride * (a.hi[1] - a.lo[1] + 1);
    a.nstride = a.kstride * (a.hi[2] - a.lo[2] + 1);
    return a;
}

__host__ __device__ inline Array4 cell_view(double* v, int i, int j, int k)
{
    Array4 a;
    a.p = v;
    a.lo[0] = a.hi[0] = i;
    a.lo[1] = a.hi[1] = j;
    a.lo[2] = a.hi[2] = k;
    a.jstride = a.kstride = 1;
    a.nstride = 1;
    return a;
}

__device__ __forceinline__ int clampi(int i, int n, int per)
{
    if (i < 0) return per ? ((i % n) + n) % n : 0;
    if (i >= n) return per ? i % n : n - 1;
    return i;
}

__device__ __forceinline__ void cell_of(const GridDev& g, long long t, int& i, int& j, int& k)
{
    i = (int)(t % g.n[0]);
    const long long r = t / g.n[0];
    j = (int)(r % g.n[1]);
    k = (int)(r / g.n[1]);
}

struct Geo
{
    GridDev g;
    double dx[3];
    double plo[3];
    double phi[3];
};

__device__ __forceinline__ GpuArray<Real, 3> ga3(const double* v)
{
    GpuArray<Real, 3> a;
    a[0] = v[0];
    a[1] = v[1];
    a[2] = v[2];
    return a;
}

// ---------------- Poisson right-hand side (Source/PotentialSolve.cpp:252-277, :484)
__global__ void k_poisson_rhs(Geo G, GridDev gm, const double* __restrict__ Sold, double* Sv,
                              double* __restrict__ rhs, double* __restrict__ sol,
                              int do_spacechrg, int warm, double ps, double time,
                              const ProbParm* pp, const double* __restrict__ ephi)
{
    VD_PDL_WAIT();
    const long long N = G.g.ncell();
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < N;
         t += (long long)gridDim.x * blockDim.x)
    {
        int ci, cj, ck;
        cell_of(G.g, t, ci, cj, ck);
        const long long m = gm.idx(ci, cj, ck);
        double r = 0.0;
        if (do_spacechrg)
        {
#pragma unroll
            for (int sp = 0; sp < NUM_SPECIES; sp++)
            {
                const int q = plasmachem::get_charge(sp);
                if (abs(q) > 0) r += q * Sold[sp * N + t];
            }
            r *= (-ECHARGE / EPS0);
#ifndef VD_NO_USER_POTENTIAL_SOURCES
            Array4 sv = state_view(const_cast<double*>(Sold), G.g);
            Array4 rv = cell_view(&r, ci, cj, ck);
            user_sources::add_user_potential_sources(ci, cj, ck, sv, rv, ga3(G.plo), ga3(G.phi),
                                                     ga3(G.dx), time, *pp);
#endif
        }
        if (ephi) r = r + ephi[t]; // electron-Poisson coupling source
        rhs[m] = r * (1.0 / ps);
        sol[m] = warm ? Sv[POT_ID * N + t] / ps : 0.0;
    }
}

// ---------------- boundary callbacks (Source/PotentialSolve.cpp:350-434,
// Source/ScalarSolve.cpp:693-803): one thread per face of side s.
struct SideArrays
{
    double* val;
    double* ra;
    double* rb;
    double* rf;
    double* g;
    double* c0;
};

__global__ void k_bc_hook(Geo G, int s, int kind, int comp, double* S, SideArrays A,
                          double time, double app_voltage, int user_defined, double Tg,
                          double Pg, const ProbParm* pp)
{
    VD_PDL_WAIT();
    const int d = s % 3;
    const int ta = (d == 0) ? 1 : 0, tb = (d == 2) ? 1 : 2;
    const int np = G.g.n[ta] * G.g.n[tb];
    const int sgn = (s / 3) ? 1 : -1;
    const long long N = G.g.ncell();
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < np; q += gridDim.x * blockDim.x)
    {
        int c[3], f[3];
        c[d] = (s / 3) ? G.g.n[d] - 1 : 0;
        c[ta] = q % G.g.n[ta];
        c[tb] = q / G.g.n[ta];
        f[0] = c[0];
        f[1] = c[1];
        f[2] = c[2];
        f[d] = (s / 3) ? G.g.n[d] : 0;
        A.val[q] = S[comp * N + G.g.idx(c[0], c[1], c[2])];
        A.ra[q] = 0.0;
        A.rb[q] = 1.0;
        A.rf[q] = 0.0;
        Array4 sv = state_view(S, G.g);
        Array4 bv = side_view(A.val, G.g, s), av = side_view(A.ra, G.g, s),
               bbv = side_view(A.rb, G.g, s), fv = side_view(A.rf, G.g, s);
        if (kind == 0)
        {
#ifdef VD_HAS_USER_TRANSPORT
            if (user_defined)
                user_transport::potential_bc(f[0], f[1], f[2], d, sgn, sv, bv, av, bbv, fv,
                                             ga3(G.plo), ga3(G.phi), ga3(G.dx), time, *pp, Tg,
                                             Pg, app_voltage VD_CURRENT_ARGS);
            else
#endif
                plasmachem_transport::potential_bc(f[0], f[1], f[2], d, sgn, sv, bv, av, bbv,
                                                   fv, ga3(G.plo), ga3(G.phi), ga3(G.dx), time,
                                                   *pp, Tg, Pg, app_voltage);
        } else
        {
#ifdef VD_HAS_USER_TRANSPORT
            if (user_defined)
                user_transport::species_bc(f[0], f[1], f[2], d, sgn, comp, 0, sv, bv, av, bbv,
                                           fv, ga3(G.plo), ga3(G.phi), ga3(G.dx), time, *pp,
                                           Tg, Pg VD_CURRENT_ARGS);
            else
#endif
                plasmachem_transport::species_bc(f[0], f[1], f[2], d, sgn, comp, 0, sv, bv, av,
                                                 bbv, fv, ga3(G.plo), ga3(G.phi), ga3(G.dx),
                                                 time, *pp, Tg, Pg);
        }
    }
}

// Scale the hook values into the solver's units and turn them into the
// ghost affine form (g = inhomogeneous part, c0 = Robin interior factor).
__global__ void k_bc_finalize(int np, int type, int nx_d, int maxorder, double dx,
                              double scale, SideArrays A)
{
    VD_PDL_WAIT();
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < np; q += gridDim.x * blockDim.x)
    {
        A.val[q] *= scale;
        A.rf[q] *= scale;
        if (type == MG_DIR)
        {
            const int NX = min(nx_d + 1, maxorder);
            A.g[q] = (NX <= 2) ? 2.0 * A.val[q] : (8.0 / 3.0) * A.val[q];
        } else if (type == MG_ROBIN)
        {
            const double a = A.ra[q], b = A.rb[q], dxi = 1.0 / dx;
            const double den = 0.5 * a + b * dxi;
            A.c0[q] = (b * dxi - 0.5 * a) / den;
            A.g[q] = A.rf[q] / den;
        } else
        {
            A.g[q] = 0.0;
        }
    }
}

// Inhomogeneous Neumann: the face gradient enters the right-hand side.
__global__ void k_inneu_adjust(GridDev g, int s, const double* bface, double bconst,
                               double beta, double dx, const double* val,
                               double* __restrict__ rhs)
{
    VD_PDL_WAIT();
    const int d = s % 3;
    const int ta = (d == 0) ? 1 : 0, tb = (d == 2) ? 1 : 2;
    const int np = g.n[ta] * g.n[tb];
    const bool hi = (s / 3) != 0;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < np; q += gridDim.x * blockDim.x)
    {
        int c[3];
        c[d] = hi ? g.n[d] - 1 : 0;
        c[ta] = q % g.n[ta];
        c[tb] = q / g.n[ta];
        int f[3] = {c[0], c[1], c[2]};
        if (hi) f[d] += 1;
        const double b = bface ? bface[face_index(g, d, f[0], f[1], f[2])] : bconst;
        const double fac = beta / dx;
        rhs[g.idx(c[0], c[1], c[2])] += (hi ? 1.0 : -1.0) * fac * b * val[q];
    }
}

// Face gradient of a solved field with its boundary closure (MLMG
// getGradSolution); inhomogeneous-Neumann faces return their gradient.
struct GradCtx
{
    MGOp<double> op; // fine operator of the solve (boundary data)
    double dxi[3];
    const double* inneu_val[6];
};

__device__ __forceinline__ double grad_at_face(const GradCtx& C, const double* __restrict__ x,
                                               int d, int i, int j, int k)
{
    const GridDev& g = C.op.g;
    int c[3] = {i, j, k};
    const int fi = c[d];
    if (fi > 0 && fi < g.n[d])
    {
        int m[3] = {i, j, k};
        m[d] -= 1;
        return (x[g.idx(i, j, k)] - x[g.idx(m[0], m[1], m[2])]) * C.dxi[d];
    }
    if (g.per[d])
    {
        int m[3] = {i, j, k}, p[3] = {i, j, k};
        m[d] = g.n[d] - 1;
        p[d] = 0;
        return (x[g.idx(p[0], p[1], p[2])] - x[g.idx(m[0], m[1], m[2])]) * C.dxi[d];
    }
    const bool lo = (fi == 0);
    int in[3] = {i, j, k};
    if (!lo) in[d] -= 1;
    const int s = d + (lo ? 0 : 3);
    if (C.op.bct[s] == MG_INNEU) return C.inneu_val[s][plane_index(g, d, in[0], in[1], in[2])];
    const double x0 = x[g.idx(in[0], in[1], in[2])];
    double cf, gh;
    if (d == 0)
        gh = mg_nbr<0>(C.op, x, in[0], in[1], in[2], lo ? -1 : 1, true, x0, cf);
    else if (d == 1)
        gh = mg_nbr<1>(C.op, x, in[0], in[1], in[2], lo ? -1 : 1, true, x0, cf);
    else
        gh = mg_nbr<2>(C.op, x, in[0], in[1], in[2], lo ? -1 : 1, true, x0, cf);
    return lo ? (x0 - gh) * C.dxi[d] : (gh - x0) * C.dxi[d];
}

// ---------------- E field, reduced field, potential (Source/PotentialSolve.cpp:500-541)
// Grid: (row blocks, ny, nz).  Faces inside the domain are plain differences
// of the solution; boundary faces go through the solve's closure.
// E = -grad(phi) at cell (i,j,k) of the solution x0 = sol there: the mean of
// the two face gradients, boundary faces from the solve's ghost closure.
__device__ __forceinline__ void efield_cell(const GradCtx& C, const double* __restrict__ sol,
                                            int i, int j, int k, double x0, double ps,
                                            double* E)
{
    const GridDev& g = C.op.g;
    const int c3[3] = {i, j, k};
#pragma unroll
    for (int d = 0; d < 3; ++d)
    {
        E[d] = 0.0;
        if (d >= g.dim) break;
        int m[3] = {i, j, k}, p[3] = {i, j, k};
        m[d] -= 1;
        p[d] += 1;
        const double glo = (c3[d] > 0) ? (x0 - sol[g.idx(m[0], m[1], m[2])]) * C.dxi[d]
                                       : grad_at_face(C, sol, d, i, j, k);
        const double ghi = (c3[d] < g.n[d] - 1)
                               ? (sol[g.idx(p[0], p[1], p[2])] - x0) * C.dxi[d]
                               : grad_at_face(C, sol, d, p[0], p[1], p[2]);
        E[d] = 0.5 * (glo * (-1.0 * ps) + ghi * (-1.0 * ps));
    }
}

__global__ void __launch_bounds__(128) k_efield(GradCtx C, const double* __restrict__ sol,
                                                double* __restrict__ S, double ps)
{
    VD_PDL_WAIT();
    const GridDev& g = C.op.g;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.n[0]) return;
    const int j = blockIdx.y, k = blockIdx.z;
    const long long N = g.ncell();
    const long long t = i + (long long)g.n[0] * (j + (long long)g.n[1] * k);
    const double x0 = sol[g.idx(i, j, k)];
    double E[3];
    efield_cell(C, sol, i, j, k, x0, ps, E);
    for (int d = 0; d < g.dim; ++d) S[(EFX_ID + d) * N + t] = E[d];
    double Esum = 0.0, nd = 0.0;
#pragma unroll
    for (int sp = 0; sp < NUM_SPECIES; sp++) nd += S[sp * N + t];
    nd = nd - S[E_ID * N + t];
    for (int d = 0; d < g.dim; ++d) Esum += E[d] * E[d];
    S[REF_ID * N + t] = (sqrt(Esum) / nd) / 1.0e-21;
    S[POT_ID * N + t] = x0 * ps;
}

// The same for two adjacent cells i, i+1 per thread (nx even): the state
// components are read and written as 16-byte pairs.
__global__ void __launch_bounds__(128) k_efield2(GradCtx C, const double* __restrict__ sol,
                                                 double* __restrict__ S, double ps)
{
    VD_PDL_WAIT();
    const GridDev& g = C.op.g;
    const int i = 2 * (blockIdx.x * blockDim.x + threadIdx.x);
    if (i >= g.n[0]) return;
    const int j = blockIdx.y, k = blockIdx.z;
    const long long N = g.ncell();
    const long long t = i + (long long)g.n[0] * (j + (long long)g.n[1] * k);
    double x0[2], E[2][3];
    const int nx = g.n[0], ny = g.n[1], nz = g.n[2];
    if (g.rb && g.dim == 3 && i >= 2 && i + 2 < nx && j > 0 && j < ny - 1 && k > 0 && k < nz - 1)
    {
        // interior pair on the red-black split potential: cell i is of
        // colour c0 = (i+j+k) & 1 and cell i+1 of the other, both at
        // half-index h; every neighbour is a fixed offset from h in one of
        // the two halves (x: i-1 and i+2 at h-1 and h+1; y, z: +-row, +-plane)
        const int nxh = nx >> 1, c0 = (i + j + k) & 1;
        const long long half = g.ncell() >> 1, row = nxh, plane = (long long)nxh * ny;
        const long long h = (i >> 1) + nxh * (j + (long long)ny * k);
        const double* __restrict__ sa = sol + c0 * half;       // colour of cell i
        const double* __restrict__ sb = sol + (1 - c0) * half; // colour of cell i+1
        x0[0] = sa[h];
        x0[1] = sb[h];
        const double nA[6] = {sb[h - 1], x0[1], sb[h - row], sb[h + row], sb[h - plane],
                              sb[h + plane]};
        const double nB[6] = {x0[0], sa[h + 1], sa[h - row], sa[h + row], sa[h - plane],
                              sa[h + plane]};
#pragma unroll
        for (int d = 0; d < 3; ++d)
        {
            // efield_cell's interior arithmetic
            const double gla = (x0[0] - nA[2 * d]) * C.dxi[d];
            const double gha = (nA[2 * d + 1] - x0[0]) * C.dxi[d];
            E[0][d] = 0.5 * (gla * (-1.0 * ps) + gha * (-1.0 * ps));
            const double glb = (x0[1] - nB[2 * d]) * C.dxi[d];
            const double ghb = (nB[2 * d + 1] - x0[1]) * C.dxi[d];
            E[1][d] = 0.5 * (glb * (-1.0 * ps) + ghb * (-1.0 * ps));
        }
    } else
    {
#pragma unroll
        for (int e = 0; e < 2; ++e) x0[e] = sol[g.idx(i + e, j, k)];
#pragma unroll
        for (int e = 0; e < 2; ++e) efield_cell(C, sol, i + e, j, k, x0[e], ps, E[e]);
    }
    for (int d = 0; d < g.dim; ++d)
        *reinterpret_cast<double2*>(S + (EFX_ID + d) * N + t) = make_double2(E[0][d], E[1][d]);
    double nd[2] = {0.0, 0.0};
#pragma unroll
    for (int sp = 0; sp < NUM_SPECIES; sp++)
    {
        const double2 v = *reinterpret_cast<const double2*>(S + sp * N + t);
        nd[0] += v.x;
        nd[1] += v.y;
    }
    const double2 ne = *reinterpret_cast<const double2*>(S + E_ID * N + t);
    nd[0] = nd[0] - ne.x;
    nd[1] = nd[1] - ne.y;
    double r[2];
#pragma unroll
    for (int e = 0; e < 2; ++e)
    {
        double Esum = 0.0;
        for (int d = 0; d < g.dim; ++d) Esum += E[e][d] * E[e][d];
        r[e] = (sqrt(Esum) / nd[e]) / 1.0e-21;
    }
    *reinterpret_cast<double2*>(S + REF_ID * N + t) = make_double2(r[0], r[1]);
    *reinterpret_cast<double2*>(S + POT_ID * N + t) = make_double2(x0[0] * ps, x0[1] * ps);
}

// ---------------- fused reactions + drift flux + divergence
// (update_rxnsrc_at_all_levels, Source/ScalarSolve.cpp:181-209;
//  compute_scalar_transport_flux + compute_flux, Source/ScalarSolve.cpp:285-324,
//  Source/compute_explicit_flux.H:218-415; compute_dsdt, Source/ScalarSolve.cpp:50-78).
// Every transported component's explicit source in one pass over the cells.
struct ExplParams
{
    Geo G;
    const double* S;
    double* expl;
    double* rxn_een;
    double* rxn_e; // electron reaction source (electron-Poisson coupling), or null
    int eidx;
    double Tg, Pg, time, dt, dxmin;
    int hyp_order, weno_scheme, user_vel, do_transport, do_reactions, do_bg_rxn;
    int ntr;
    int comp[VD_NT];
    int bclo[VD_NT][3];
    int bchi[VD_NT][3];
    int bg[NUM_SPECIES];
    const ProbParm* pp;
    // multicomponent solves: background species' pure reaction sources,
    // slot bgslot[sp] of rxn_bg (null otherwise)
    double* rxn_bg;
    int bgslot[NUM_SPECIES];
};

__device__ __forceinline__ bool wall_zero(int code) { return code == IHNEUBC || code == AXISBC; }

// Streaming form of the same update.  A CTA owns an EX_TX x EX_TY column of
// cells and marches along z over a chunk of planes.  Each loaded plane
// (with a 3-cell xy halo) gives, per transported component of the group,
// n and the x/y drift velocities in shared memory; the x and y face fluxes
// of that plane are computed once per face.  The z stencil lives in a
// six-plane register queue per thread, so every z face is also computed
// once.  Output for plane z happens three planes after it is loaded.  The
// first group launch evaluates the chemistry once per cell and stores the
// reaction sources of every component; later group launches (components
// beyond the first EX_QB) read them back.  Accumulation order per cell is
// the reference's ((Fx + rxn) + Fy) + Fz.
// The block has EX_THREADS threads whatever the tile height: threads past
// the tile's EX_TX x EX_TY cells only share the face work.  Seven rows give
// 33x7 + 32x8 = 487 x/y faces per plane, two rounds of the 256 threads
// (eight rows: 552 faces, a third round for 40 of them): 4.82 -> 4.75 ms of
// explicit work per 256^3 step.
#define EX_TX 32
#ifndef EX_TY
#define EX_TY 7
#endif
#define EX_THREADS 256
#define EX_HX (EX_TX + 6)
#define EX_HY (EX_TY + 6)
#define EX_QB 1

__device__ __forceinline__ void ex_cell_vel(const ExplParams& P, int ci, int cj, int ck,
                                            int ui, int uj, int uk, int comp, double te,
                                            double nd, double em, double ex, double ey,
                                            double ez, double& vx, double& vy, double& vz)
{
#ifdef VD_HAS_USER_TRANSPORT
    if (P.user_vel)
    {
        Array4 sv = state_view(const_cast<double*>(P.S), P.G.g);
        const IntVect c{ui, uj, uk};
        vx = user_transport::compute_vel(c, 0, comp, sv, ga3(P.G.dx), P.time, *P.pp, P.Tg, P.Pg);
        vy = (P.G.g.dim > 1) ? user_transport::compute_vel(c, 1, comp, sv, ga3(P.G.dx), P.time,
                                                            *P.pp, P.Tg, P.Pg)
                             : 0.0;
        vz = (P.G.g.dim > 2) ? user_transport::compute_vel(c, 2, comp, sv, ga3(P.G.dx), P.time,
                                                            *P.pp, P.Tg, P.Pg)
                             : 0.0;
        return;
    }
#endif
    const double mu = specMob(comp, te, nd, em, P.Tg);
    vx = mu * ex;
    vy = mu * ey;
    vz = mu * ez;
}

#ifndef EX_ZC
#define EX_ZC 0 // planes per CTA in z (0: chosen per grid, explicit_zchunk)
#endif
#ifndef EX_MINB
#define EX_MINB 4 // CTAs per SM the register budget is sized for (64 registers; measured
                  // at 256^3 with the inlined face flux: 4.13 ms per step against
                  // 4.37 with 3 CTAs and 4.51 with 5)
#endif
__global__ void __launch_bounds__(256, EX_MINB) k_explicit_stream(ExplParams P, int q0, int zc)
{
    VD_PDL_WAIT();
    __shared__ double s_n[EX_QB][EX_HY][EX_HX];
    __shared__ double s_vx[EX_QB][EX_HY][EX_HX];
    __shared__ double s_vy[EX_QB][EX_HY][EX_HX];
    __shared__ double s_vz[EX_QB][EX_HY][EX_HX];
    __shared__ double s_fx[EX_QB][EX_TY][EX_TX + 1];
    __shared__ double s_fy[EX_QB][EX_TY + 1][EX_TX];
    const GridDev& g = P.G.g;
    const long long N = g.ncell();
    const double* __restrict__ S = P.S;
    const int dim = g.dim;
    const int tx = threadIdx.x % EX_TX, ty = threadIdx.x / EX_TX;
    const int i0 = blockIdx.x * EX_TX, j0 = blockIdx.y * EX_TY;
    const int i = i0 + tx, j = j0 + ty;
    const bool active = ty < EX_TY && i < g.n[0] && j < g.n[1];
    const int nq = min(EX_QB, P.ntr - q0);
    const int zb = blockIdx.z * zc;
    const int ze = min(zb + zc, g.n[2]);
    const int lag = (dim == 3) ? 3 : 0;
    const int pfirst = (dim == 3) ? zb - 3 : zb;
    const int plast = ze - 1 + lag;
    const double dxmin = P.dxmin;

    double qn[EX_QB][6], qv[EX_QB][6], qdx[EX_QB][4], qdy[EX_QB][4], fzlo[EX_QB];
#pragma unroll
    for (int s = 0; s < EX_QB; ++s)
    {
#pragma unroll
        for (int m = 0; m < 6; ++m) qn[s][m] = qv[s][m] = 0.0;
#pragma unroll
        for (int m = 0; m < 4; ++m) qdx[s][m] = qdy[s][m] = 0.0;
        fzlo[s] = 0.0;
    }

    for (int p = pfirst; p <= plast; ++p)
    {
        const int pz = clampi(p, g.n[2], g.per[2]);
        __syncthreads();
        // ---- load plane p with its xy halo
        if (P.do_transport)
            for (int c = threadIdx.x; c < EX_HX * EX_HY; c += blockDim.x)
            {
                const int hx = c % EX_HX, hy = c / EX_HX;
                const int ui = i0 + hx - 3, uj = j0 + hy - 3;
                const int ci = clampi(ui, g.n[0], g.per[0]);
                const int cj = (dim > 1) ? clampi(uj, g.n[1], g.per[1]) : 0;
                const long long q = g.idx(ci, cj, pz);
                const double ex = S[EFX_ID * N + q], ey = S[EFY_ID * N + q],
                             ez = S[EFZ_ID * N + q];
                const double em = sqrt(ex * ex + ey * ey + ez * ez);
                const double te = S[ETEMP_ID * N + q];
                double nd = 0.0;
#pragma unroll
                for (int sp = 0; sp < NUM_SPECIES; sp++) nd += S[sp * N + q];
#pragma unroll
                for (int s = 0; s < EX_QB; ++s)
                {
                    if (s >= nq) break;
                    const int comp = P.comp[q0 + s];
                    double vx, vy, vz;
                    ex_cell_vel(P, ci, cj, pz, ui, uj, p, comp, te, nd, em, ex, ey, ez, vx, vy,
                                vz);
                    s_n[s][hy][hx] = S[comp * N + q];
                    s_vx[s][hy][hx] = vx;
                    s_vy[s][hy][hx] = vy;
                    s_vz[s][hy][hx] = vz;
                }
            }
        __syncthreads();
        // ---- x and y face fluxes of plane p: the (EX_TX+1) x EX_TY x-faces and
        // EX_TX x (EX_TY+1) y-faces of the tile spread evenly over the threads
        if (P.do_transport)
        {
            constexpr int NFX = (EX_TX + 1) * EX_TY, NFY = EX_TX * (EX_TY + 1);
            const int nfy = (dim > 1) ? NFY : 0;
            for (int fid = threadIdx.x; fid < NFX + nfy; fid += blockDim.x)
            {
                const bool xf = fid < NFX;
                const int r = xf ? fid / (EX_TX + 1) : (fid - NFX) / EX_TX;
                const int c = xf ? fid - r * (EX_TX + 1) : (fid - NFX) - r * EX_TX;
                // face index along its direction, and whether it is needed
                const int fi = i0 + c, fj = j0 + r;
                const bool need = xf ? (fi <= g.n[0] && fi - 1 < g.n[0] && fj < g.n[1])
                                     : (fj <= g.n[1] && fj - 1 < g.n[1] && fi < g.n[0]);
                if (!need) continue;
#pragma unroll
                for (int s = 0; s < EX_QB; ++s)
                {
                    if (s >= nq) break;
                    const int qc = q0 + s;
                    double u[6], v[6];
#pragma unroll
                    for (int m = 0; m < 6; ++m)
                    {
                        u[m] = xf ? s_n[s][r + 3][c + m] : s_n[s][r + m][c + 3];
                        v[m] = xf ? s_vx[s][r + 3][c + m] : s_vy[s][r + m][c + 3];
                    }
                    double fl = face_flux6(u, v, P.hyp_order, P.weno_scheme, dxmin, P.dt);
                    if (xf)
                    {
                        if ((fi == 0 && wall_zero(P.bclo[qc][0])) ||
                            (fi == g.n[0] && wall_zero(P.bchi[qc][0])))
                            fl = 0.0;
                        s_fx[s][r][c] = fl;
                    } else
                    {
                        if ((fj == 0 && wall_zero(P.bclo[qc][1])) ||
                            (fj == g.n[1] && wall_zero(P.bchi[qc][1])))
                            fl = 0.0;
                        s_fy[s][r][c] = fl;
                    }
                }
            }
        }
        __syncthreads();
        // ---- queues: this plane's x/y divergences and z stencil values
#pragma unroll
        for (int s = 0; s < EX_QB; ++s)
        {
#pragma unroll
            for (int m = 0; m < 3; ++m)
            {
                qdx[s][m] = qdx[s][m + 1];
                qdy[s][m] = qdy[s][m + 1];
            }
#pragma unroll
            for (int m = 0; m < 5; ++m)
            {
                qn[s][m] = qn[s][m + 1];
                qv[s][m] = qv[s][m + 1];
            }
            if (s < nq && active && P.do_transport)
            {
                qdx[s][3] = (s_fx[s][ty][tx] - s_fx[s][ty][tx + 1]) / P.G.dx[0];
                qdy[s][3] = (dim > 1) ? (s_fy[s][ty][tx] - s_fy[s][ty + 1][tx]) / P.G.dx[1] : 0.0;
                qn[s][5] = s_n[s][ty + 3][tx + 3];
                qv[s][5] = s_vz[s][ty + 3][tx + 3];
            }
        }
        const int z = p - lag; // output plane
        double fzhi[EX_QB];
#pragma unroll
        for (int s = 0; s < EX_QB; ++s) fzhi[s] = 0.0;
        if (dim == 3 && P.do_transport && active && p >= zb + 2)
        {
#pragma unroll
            for (int s = 0; s < EX_QB; ++s)
            {
                if (s >= nq) break;
                double f = face_flux6(qn[s], qv[s], P.hyp_order, P.weno_scheme, dxmin, P.dt);
                if (z == g.n[2] - 1 && wall_zero(P.bchi[q0 + s][2])) f = 0.0;
                fzhi[s] = f;
            }
        }
        if (z >= zb && active)
        {
            const long long t = g.idx(i, j, z);
            double rx[EX_QB];
            if (q0 == 0)
            {
                // reactions (update_rxnsrc_at_all_levels) for every component
                double rxa[VD_NT];
#pragma unroll
                for (int c = 0; c < VD_NT; ++c) rxa[c] = 0.0;
                if (P.do_reactions)
                {
                    double C[NUM_SPECIES], W[NUM_SPECIES];
#pragma unroll
                    for (int sp = 0; sp < NUM_SPECIES; sp++) C[sp] = S[sp * N + t] / N_A;
                    double ee = 0.0;
                    CKWC(P.Tg, C, W, S[ETEMP_ID * N + t], S[REF_ID * N + t], &ee);
#pragma unroll
                    for (int sp = 0; sp < NUM_SPECIES; sp++) rxa[sp] = W[sp] * N_A;
                    rxa[NUM_SPECIES] = ee;
#ifndef VD_NO_USER_REACT_SOURCES
                    Array4 sv = state_view(const_cast<double*>(S), g);
                    Array4 rv = cell_view(rxa, i, j, z);
                    user_sources::add_user_react_sources(i, j, z, sv, rv, ga3(P.G.plo),
                                                         ga3(P.G.phi), ga3(P.G.dx), P.time,
                                                         *P.pp, P.Tg, P.Pg);
#endif
                }
                if (P.rxn_een) P.rxn_een[t] = rxa[NUM_SPECIES];
                if (P.rxn_e) P.rxn_e[t] = rxa[P.eidx];
#pragma unroll
                for (int sp = 0; sp < NUM_SPECIES; sp++)
                    if (P.bg[sp])
                    {
                        P.expl[sp * N + t] = P.do_bg_rxn ? rxa[sp] : 0.0;
                        if (P.rxn_bg) P.rxn_bg[P.bgslot[sp] * N + t] = rxa[sp];
                    }
                // reaction sources of components handled by later group launches
                for (int q = EX_QB; q < P.ntr; ++q)
                {
                    const int comp = P.comp[q];
#pragma unroll
                    for (int c = 0; c < VD_NT; ++c)
                        if (c == comp) P.expl[comp * N + t] = rxa[c];
                }
#pragma unroll
                for (int s = 0; s < EX_QB; ++s)
                {
                    rx[s] = 0.0;
                    if (s < nq)
                    {
                        const int comp = P.comp[s];
#pragma unroll
                        for (int c = 0; c < VD_NT; ++c)
                            if (c == comp) rx[s] = rxa[c];
                    }
                }
            } else
            {
#pragma unroll
                for (int s = 0; s < EX_QB; ++s)
                    rx[s] = (s < nq) ? P.expl[P.comp[q0 + s] * N + t] : 0.0;
            }
#pragma unroll
            for (int s = 0; s < EX_QB; ++s)
            {
                if (s >= nq) break;
                // divergences of plane z: three planes back in 3-D, this plane in 2-D
                double v = ((dim == 3) ? qdx[s][0] : qdx[s][3]) + rx[s];
                if (dim > 1) v += (dim == 3) ? qdy[s][0] : qdy[s][3];
                if (dim == 3)
                {
                    double flo = fzlo[s];
                    if (z == 0 && wall_zero(P.bclo[q0 + s][2])) flo = 0.0;
                    v += (flo - fzhi[s]) / P.G.dx[2];
                }
                P.expl[P.comp[q0 + s] * N + t] = P.do_transport ? v : rx[s];
            }
        }
#pragma unroll
        for (int s = 0; s < EX_QB; ++s) fzlo[s] = fzhi[s];
    }
}

// ---------------- diffusion-solve set-up (Source/ScalarSolve.cpp:587-690, :819-846)
__device__ __forceinline__ double cell_diff(const double* __restrict__ S, const GridDev& g,
                                            long long N, int spec, int i, int j, int k,
                                            double Tg)
{
    const long long q = g.idx(clampi(i, g.n[0], g.per[0]), clampi(j, g.n[1], g.per[1]),
                              clampi(k, g.n[2], g.per[2]));
    double Es = 0.0, nd = 0.0;
#pragma unroll
    for (int d = 0; d < 3; ++d)
    {
        const double e = S[(EFX_ID + d) * N + q];
        Es += e * e;
    }
    const double emag = sqrt(Es);
#pragma unroll
    for (int sp = 0; sp < NUM_SPECIES; sp++) nd += S[sp * N + q];
    return specDiff(spec, S[ETEMP_ID * N + q], nd, emag, Tg);
}

// Electron time scales (find_time_scales, Source/TimeStep.cpp:46-134): the
// max-norms of |mu_e| |E|, D_e and |mu_e| n_e over the cells, per block into
// part[3 b + q]; k_time_scales_final reduces them into out[0..2].
__global__ void __launch_bounds__(256) k_time_scales(GridDev g, const double* __restrict__ S,
                                                     int eidx, double Tg,
                                                     double* __restrict__ part)
{
    VD_PDL_WAIT();
    __shared__ double sh[32];
    const long long N = g.ncell();
    double m0 = 0.0, m1 = 0.0, m2 = 0.0;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < N;
         t += (long long)gridDim.x * blockDim.x)
    {
        const double etemp = S[ETEMP_ID * N + t];
        double Esum = 0.0;
        for (int d = 0; d < g.dim; ++d)
        {
            const double e = S[(EFX_ID + d) * N + t];
            Esum += e * e;
        }
        const double emag = sqrt(Esum);
        double nd = 0.0;
#pragma unroll
        for (int sp = 0; sp < NUM_SPECIES; sp++) nd += S[sp * N + t];
        const double dco = specDiff(eidx, etemp, nd, emag, Tg);
        const double mu = specMob(eidx, etemp, nd, emag, Tg);
        m0 = fmax(m0, fabs(fabs(mu) * emag));
        m1 = fmax(m1, fabs(dco));
        m2 = fmax(m2, fabs(fabs(mu) * S[eidx * N + t]));
    }
    m0 = block_max(m0, sh);
    m1 = block_max(m1, sh);
    m2 = block_max(m2, sh);
    if (threadIdx.x == 0)
    {
        part[3 * blockIdx.x] = m0;
        part[3 * blockIdx.x + 1] = m1;
        part[3 * blockIdx.x + 2] = m2;
    }
}

__global__ void __launch_bounds__(256) k_time_scales_final(const double* __restrict__ part,
                                                           int nb, double* __restrict__ out)
{
    VD_PDL_WAIT();
    __shared__ double sh[32];
    double m[3] = {0.0, 0.0, 0.0};
    for (int b = threadIdx.x; b < nb; b += blockDim.x)
#pragma unroll
        for (int q = 0; q < 3; ++q) m[q] = fmax(m[q], part[3 * b + q]);
#pragma unroll
    for (int q = 0; q < 3; ++q)
    {
        const double v = block_max(m[q], sh);
        if (threadIdx.x == 0) out[q] = v;
    }
}

// Electron-Poisson coupling (Source/PotentialSolve.cpp:272-347): the
// potential operator's cell coefficient b = -(1 + dt/tau_diel),
// tau_diel = |eps0 / (e mu_e n_e)| (-1 outside real cells), from the state
// with clamped (foextrap) or wrapped neighbours, harmonic-averaged onto the
// faces of direction d.
__device__ __forceinline__ double pot_bcell(const double* __restrict__ S, const GridDev& g,
                                            long long N, int eidx, int i, int j, int k,
                                            double Tg, double dt)
{
    const long long q = g.idx(clampi(i, g.n[0], g.per[0]), clampi(j, g.n[1], g.per[1]),
                              clampi(k, g.n[2], g.per[2]));
    if (S[CMASK_ID * N + q] != 1.0) return -1.0;
    double Es = 0.0, nd = 0.0;
    for (int d = 0; d < g.dim; ++d)
    {
        const double e = S[(EFX_ID + d) * N + q];
        Es += e * e;
    }
    const double emag = sqrt(Es);
#pragma unroll
    for (int sp = 0; sp < NUM_SPECIES; sp++) nd += S[sp * N + q];
    const double mu_e = specMob(eidx, S[ETEMP_ID * N + q], nd, emag, Tg);
    const double tau_diel = fabs(EPS0 / (ECHARGE * mu_e * S[eidx * N + q]));
    return -(1.0 + dt / tau_diel);
}

__global__ void k_pot_faces(GridDev g, int d, const double* __restrict__ S, int eidx, double Tg,
                            double dt, double* __restrict__ bf)
{
    VD_PDL_WAIT();
    const long long tot = face_count(g, d);
    const long long N = g.ncell();
    const int nx = g.n[0] + (d == 0), ny = g.n[1] + (d == 1);
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < tot;
         t += (long long)gridDim.x * blockDim.x)
    {
        const int i = (int)(t % nx);
        const long long r = t / nx;
        const int j = (int)(r % ny);
        const int k = (int)(r / ny);
        int m[3] = {i, j, k};
        m[d] -= 1;
        const double b0 = pot_bcell(S, g, N, eidx, m[0], m[1], m[2], Tg, dt);
        const double b1 = pot_bcell(S, g, N, eidx, i, j, k, Tg, dt);
        bf[t] = 2.0 * b0 * b1 / (b0 + b1);
    }
}

// After the coupled electron solve: the floored electron density into the
// state (as Vidyut::implicit_solve_scalar stores it, so the stages after it
// read it, Source/Evolve.cpp:305-343) and the coupling source
// ephi = ((n_e^new - n_e^old)/dt - S_expl + S_rxn) dt e / eps0.
__global__ void k_ephi(GridDev g, GridDev gm, double* __restrict__ S,
                       const double* __restrict__ Sold, const double* __restrict__ u,
                       double scale, const double* __restrict__ expl,
                       const double* __restrict__ rxn_e, int eidx, int bound, double min_e,
                       double dt, double* __restrict__ ephi)
{
    VD_PDL_WAIT();
    const long long N = g.ncell();
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < N;
         t += (long long)gridDim.x * blockDim.x)
    {
        int i, j, k;
        cell_of(g, t, i, j, k);
        double ne = u[gm.idx(i, j, k)] * scale;
        if (bound && ne < min_e) ne = min_e;
        S[eidx * N + t] = ne;
        double v = (1.0 / dt) * ne + (-1.0 / dt) * Sold[eidx * N + t];
        v = v + (-1.0) * expl[eidx * N + t];
        v = v + 1.0 * rxn_e[t];
        ephi[t] = v * (dt * ECHARGE / EPS0);
    }
}

// Harmonic face average of the cell diffusivity (0 where both cells are 0).
__global__ void k_species_faces(GridDev g, int d, const double* __restrict__ S, int spec,
                                double Tg, double* __restrict__ bf)
{
    VD_PDL_WAIT();
    const long long tot = face_count(g, d);
    const long long N = g.ncell();
    const int nx = g.n[0] + (d == 0), ny = g.n[1] + (d == 1);
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < tot;
         t += (long long)gridDim.x * blockDim.x)
    {
        const int i = (int)(t % nx);
        const long long r = t / nx;
        const int j = (int)(r % ny);
        const int k = (int)(r / ny);
        int m[3] = {i, j, k};
        m[d] -= 1;
        const double d0 = cell_diff(S, g, N, spec, m[0], m[1], m[2], Tg);
        const double d1 = cell_diff(S, g, N, spec, i, j, k, Tg);
        const double den = d0 + d1;
        bf[t] = (den != 0.0) ? 2.0 * d0 * d1 / den : 0.0;
    }
}

// The same face coefficients for every direction in one pass, each cell's
// diffusivity evaluated once (k_species_faces evaluates it at both cells of
// every face, once per direction: six times per cell, each with the state
// loads the hook needs).  A 32 x 8 block of cells marches over a chunk of
// planes; a plane's diffusivities go to shared memory with a one-cell halo
// on the low x and y sides (the lower neighbours of the block's first
// column and row), the previous plane's stays in a register for the z
// faces, and the faces past the last cell of a row, column or plane take
// the neighbour as cell_diff clamps (or wraps) it.  Same values and the same
// harmonic mean as k_species_faces, so the same bits.
__global__ void __launch_bounds__(256) k_species_faces3(GridDev g, const double* __restrict__ S,
                                                        int spec, double Tg, int kchunk,
                                                        double* __restrict__ bx,
                                                        double* __restrict__ by,
                                                        double* __restrict__ bz)
{
    VD_PDL_WAIT();
    __shared__ double sd[8][33]; // column 0: the halo i0-1, columns 1..32 the block
    __shared__ double sy[32];    // the halo row j0-1
    const long long N = g.ncell();
    const int nx = g.n[0], ny = g.n[1], nz = g.n[2], dim = g.dim;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    const int i = blockIdx.x * 32 + tx, j = blockIdx.y * 8 + ty;
    const bool act = i < nx && j < ny;
    const int kb = blockIdx.z * kchunk, ke = min(nz, kb + kchunk);
    auto hm = [](double d0, double d1) {
        const double den = d0 + d1;
        return (den != 0.0) ? 2.0 * d0 * d1 / den : 0.0;
    };
    double dprev = 0.0;
    if (act && dim > 2) dprev = cell_diff(S, g, N, spec, i, j, kb - 1, Tg);
    for (int k = kb; k < ke; ++k)
    {
        const double dc = act ? cell_diff(S, g, N, spec, i, j, k, Tg) : 0.0;
        sd[ty][tx + 1] = dc;
        if (tx == 0 && j < ny) sd[ty][0] = cell_diff(S, g, N, spec, i - 1, j, k, Tg);
        if (ty == 0 && i < nx && dim > 1) sy[tx] = cell_diff(S, g, N, spec, i, j - 1, k, Tg);
        __syncthreads();
        if (act)
        {
            const int nx1 = nx + 1;
            bx[i + (long long)nx1 * (j + (long long)ny * k)] = hm(sd[ty][tx], dc);
            if (i == nx - 1)
                bx[nx + (long long)nx1 * (j + (long long)ny * k)] =
                    hm(dc, cell_diff(S, g, N, spec, nx, j, k, Tg));
            if (dim > 1)
            {
                const int ny1 = ny + 1;
                const double dm = ty ? sd[ty - 1][tx + 1] : sy[tx];
                by[i + (long long)nx * (j + (long long)ny1 * k)] = hm(dm, dc);
                if (j == ny - 1)
                    by[i + (long long)nx * (ny + (long long)ny1 * k)] =
                        hm(dc, cell_diff(S, g, N, spec, i, ny, k, Tg));
            }
            if (dim > 2)
            {
                const long long t = i + (long long)nx * (j + (long long)ny * k);
                bz[t] = hm(dprev, dc);
                if (k == nz - 1)
                    bz[t + (long long)nx * ny] = hm(dc, cell_diff(S, g, N, spec, i, j, nz, Tg));
            }
        }
        dprev = dc;
        __syncthreads();
    }
}

__global__ void k_species_rhs(GridDev g, GridDev gm, const double* __restrict__ S,
                              const double* __restrict__ Sold, const double* __restrict__ expl,
                              int spec, double dt, double ts, double scale,
                              double* __restrict__ rhs, double* __restrict__ sol)
{
    VD_PDL_WAIT();
    const long long N = g.ncell();
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < N;
         t += (long long)gridDim.x * blockDim.x)
    {
        int i, j, k;
        cell_of(g, t, i, j, k);
        const long long m = gm.idx(i, j, k);
        const double r = (1.0 / dt) * Sold[spec * N + t] + 1.0 * expl[spec * N + t];
        rhs[m] = r * (ts / scale);
        sol[m] = S[spec * N + t] * (1.0 / scale);
    }
}

// ---------------- Joule heating (Source/ElecEnergySource.cpp:127-293)
struct JouleParams
{
    GradCtx pot;           // Poisson boundary data, for the face field
    const double* phi_sol; // scaled Poisson solution
    double ps;
    const double* ue;      // electron solution (scaled, before the floor)
    GridDev gm;            // layout of ue
    double escale;
    const double* S;
    double* expl;
    double* ejh;
    double dx[3];
    double Tg;
    int floor_jh;
    int eidx;
};

__device__ __forceinline__ double onesided_grad(const double* S, const GridDev& g, long long N,
                                                int comp, const int* face, int sgn, int d,
                                                double dx)
{
    int cell[3] = {face[0], face[1], face[2]};
    cell[d] += (sgn == 1) ? -1 : 0;
    int n1[3] = {cell[0], cell[1], cell[2]}, n2[3] = {cell[0], cell[1], cell[2]};
    n1[d] = cell[d] - sgn;
    n2[d] = n1[d] - sgn;
    auto at = [&](const int* c) {
        return S[comp * N + g.idx(clampi(c[0], g.n[0], g.per[0]), clampi(c[1], g.n[1], g.per[1]),
                                  clampi(c[2], g.n[2], g.per[2]))];
    };
    double g1, g2;
    if (sgn == -1)
    {
        g1 = (at(n1) - at(cell)) / dx;
        g2 = (at(n2) - at(n1)) / dx;
    } else
    {
        g1 = (at(cell) - at(n1)) / dx;
        g2 = (at(n1) - at(n2)) / dx;
    }
    return 2.0 * g1 - g2;
}

// The Joule term of one face (d, face): q (mu n_e E_f - D grad n_e) E_f with
// the face averages of Te, |E|, n_e and the total density, the face field
// from the potential and the face gradient of the electron solution (one-sided
// at the domain ends) -- a function of the face alone
// (Source/ElecEnergySource.cpp:149-273).
__device__ __forceinline__ double joule_face(const JouleParams& P, const GridDev& g, long long N,
                                             int d, const int* face)
{
    const double* __restrict__ S = P.S;
    const double charge = plasmachem::get_charge(P.eidx) * ECHARGE;
    int lc[3] = {face[0], face[1], face[2]};
    lc[d] -= 1;
    const long long ql = g.idx(clampi(lc[0], g.n[0], g.per[0]), clampi(lc[1], g.n[1], g.per[1]),
                               clampi(lc[2], g.n[2], g.per[2]));
    const long long qr = g.idx(clampi(face[0], g.n[0], g.per[0]),
                               clampi(face[1], g.n[1], g.per[1]),
                               clampi(face[2], g.n[2], g.per[2]));
    const double te = (S[ETEMP_ID * N + ql] + S[ETEMP_ID * N + qr]) / 2.0;
    double Esum = 0.0;
    for (int q = 0; q < g.dim; ++q)
    {
        const double e = (S[(EFX_ID + q) * N + ql] + S[(EFX_ID + q) * N + qr]) / 2.0;
        Esum += e * e;
    }
    const double emag = sqrt(Esum);
    const double ne = (S[P.eidx * N + ql] + S[P.eidx * N + qr]) / 2.0;
    const double ef = grad_at_face(P.pot, P.phi_sol, d, face[0], face[1], face[2]) * (-1.0 * P.ps);
    double nd = 0.0;
#pragma unroll
    for (int sp = 0; sp < NUM_SPECIES; sp++) nd += (S[sp * N + ql] + S[sp * N + qr]) / 2.0;
    const double mu = specMob(P.eidx, te, nd, emag, P.Tg);
    const double dc = specDiff(P.eidx, te, nd, emag, P.Tg);
    double gn;
    if (face[d] == 0 || face[d] == g.n[d])
    {
        const int sgn = (face[d] == 0) ? -1 : 1;
        gn = onesided_grad(S, g, N, P.eidx, face, sgn, d, P.dx[d]);
    } else
    {
        gn = (P.ue[P.gm.idx(face[0], face[1], face[2])] - P.ue[P.gm.idx(lc[0], lc[1], lc[2])]) *
             (1.0 / P.dx[d]) * P.escale;
    }
    const double cd = charge * (mu * ne * ef - dc * gn);
    return cd * ef;
}

// Joule heating of every cell (compute_elecenergy_source's jh: half the sum
// of its faces' terms, x-lo, x-hi, y-lo, y-hi, z-lo, z-hi, floored at zero
// when asked) in two passes: every face's term once into a face array --
// evaluated per cell, each interior face costs twice its ~30 state loads and
// two transport-hook calls -- then the per-cell sums in that order.  The
// product of a face term is rounded before the sum, as the oracle does.
__global__ void k_joule_faces(JouleParams P, int d, double* __restrict__ pf)
{
    VD_PDL_WAIT();
    GridDev g = P.pot.op.g;
    g.rb = 0;
    const long long N = g.ncell();
    const long long tot = face_count(g, d);
    const int nx = g.n[0] + (d == 0), ny = g.n[1] + (d == 1);
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < tot;
         t += (long long)gridDim.x * blockDim.x)
    {
        int face[3];
        face[0] = (int)(t % nx);
        const long long r = t / nx;
        face[1] = (int)(r % ny);
        face[2] = (int)(r / ny);
        pf[t] = joule_face(P, g, N, d, face);
    }
}

__global__ void k_joule_sum(JouleParams P, const double* __restrict__ px,
                            const double* __restrict__ py, const double* __restrict__ pz)
{
    VD_PDL_WAIT();
    GridDev g = P.pot.op.g;
    g.rb = 0;
    const long long N = g.ncell();
    const int nx = g.n[0], ny = g.n[1];
    const double* pfs[3] = {px, py, pz};
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < N;
         t += (long long)gridDim.x * blockDim.x)
    {
        int c3[3];
        cell_of(g, t, c3[0], c3[1], c3[2]);
        double jh = 0.0;
        for (int d = 0; d < g.dim; ++d)
        {
            const int fx = nx + (d == 0), fy = ny + (d == 1);
            const long long lo = c3[0] + (long long)fx * (c3[1] + (long long)fy * c3[2]);
            const long long step = (d == 0) ? 1 : ((d == 1) ? fx : (long long)fx * fy);
            jh += pfs[d][lo];
            jh += pfs[d][lo + step];
        }
        jh *= 0.5;
        if (P.floor_jh && jh < 0.0) jh = 0.0;
        P.expl[NUM_SPECIES * N + t] += jh;
        P.ejh[t] = jh;
    }
}

// ---------------- write-back of the solves into the state
// (Source/ScalarSolve.cpp:894-987, Source/ElecEnergySource.cpp:43-69,
//  Source/Evolve.cpp:432-456)
struct FinalParams
{
    GridDev g;
    double* S;
    int nsol;
    int comp[VD_NT];
    const double* u[VD_NT];
    double scale[VD_NT];
    int bound_specden;
    double min_e, min_s, min_te;
    int eidx;
    int een_solved;
    int heat_diag;
    int lfa;
    double Tg;
    const double* ejh;
    const double* rxn_een;
    const double* expl;
    int bg[NUM_SPECIES];
    int do_bg_rxn;
    double dt;
    GridDev gm; // layout of the solve outputs u[]
    // multicomponent solves (Source/Evolve.cpp:534-572): background species
    // go back to the step's starting value Sold, and their reactions use the
    // pure reaction source rxn_bg (slot bgslot[sp]); otherwise null
    const double* Sold;
    const double* rxn_bg;
    int bgslot[NUM_SPECIES];
};

__global__ void k_finalize(FinalParams P)
{
    VD_PDL_WAIT();
    const long long N = P.g.ncell();
    double* __restrict__ S = P.S;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < N;
         t += (long long)gridDim.x * blockDim.x)
    {
        int ci, cj, ck;
        cell_of(P.g, t, ci, cj, ck);
        const long long m = P.gm.idx(ci, cj, ck);
        // values of the iteration's starting state read before any write
        double spec_old[NUM_SPECIES];
#pragma unroll
        for (int sp = 0; sp < NUM_SPECIES; sp++) spec_old[sp] = S[sp * N + t];
        const double ref_old = S[REF_ID * N + t];
        const double cmask = S[CMASK_ID * N + t];
        for (int q = 0; q < P.nsol; ++q)
        {
            const int c = P.comp[q];
            double v = P.u[q][m] * P.scale[q];
            if (P.bound_specden && c != EEN_ID)
            {
                if (c == P.eidx)
                {
                    if (v < P.min_e) v = P.min_e;
                } else if (v < P.min_s)
                    v = P.min_s;
            }
            S[c * N + t] = v;
        }
        for (int sp = 0; sp < NUM_SPECIES; sp++)
            if (P.bg[sp] && (P.do_bg_rxn || P.Sold))
            {
                double v = P.Sold ? P.Sold[sp * N + t] : S[sp * N + t];
                if (P.do_bg_rxn)
                {
                    v += (P.rxn_bg ? P.rxn_bg[P.bgslot[sp] * N + t] : P.expl[sp * N + t]) * P.dt;
                    if (v < P.min_s && P.bound_specden) v = P.min_s;
                }
                S[sp * N + t] = v;
            }
        const double ne_new = S[P.eidx * N + t];
        if (P.een_solved)
        {
            const double te = twothird / K_B * S[EEN_ID * N + t] / spec_old[P.eidx];
            S[ETEMP_ID * N + t] = te;
            if (te < P.min_te)
            {
                S[ETEMP_ID * N + t] = P.min_te;
                S[EEN_ID * N + t] = 1.5 * K_B * ne_new * P.min_te;
            }
        }
        if (P.heat_diag)
        {
            S[EJH_ID * N + t] = P.ejh[t];
            S[EIH_ID * N + t] = P.rxn_een[t];
        }
        if (P.lfa && int(cmask))
        {
            double te = etempLFA(P.Tg, spec_old, ref_old);
            if (te < P.min_te) te = P.min_te;
            S[ETEMP_ID * N + t] = te;
            S[EEN_ID * N + t] = 1.5 * K_B * ne_new * P.min_te;
        }
    }
}

__global__ void k_midpoint(double* __restrict__ S, const double* __restrict__ Sold, long long n)
{
    VD_PDL_WAIT();
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
         t += (long long)gridDim.x * blockDim.x)
        S[t] = 0.5 * Sold[t] + 0.5 * S[t];
}

__global__ void k_nonfinite(const double* __restrict__ S, long long n, unsigned long long* cnt)
{
    VD_PDL_WAIT();
    unsigned long long c = 0;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
         t += (long long)gridDim.x * blockDim.x)
        if (!isfinite(S[t])) ++c;
    if (c) atomicAdd(cnt, c);
}

template <typename T>
__global__ void k_add_same(T* __restrict__ x, const T* __restrict__ e, long long n,
                           const int* stop)
{
    VD_PDL_WAIT();
    if (stop && *(volatile const int*)stop) return;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
         t += (long long)gridDim.x * blockDim.x)
        x[t] += e[t];
}

template <typename T>
__global__ void k_add_scaled(double* __restrict__ x, const T* __restrict__ e, double s, long long n)
{
    VD_PDL_WAIT();
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
         t += (long long)gridDim.x * blockDim.x)
        x[t] += (double)e[t] * s;
}

} // namespace vd
