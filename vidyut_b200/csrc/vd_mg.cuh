// Geometric multigrid for the cell-centred operator
//     L(x) = alpha a x - beta div(b grad x)
// (the operator of AMReX's MLABecLaplacian as the reference uses it,
// Source/ScalarSolve.cpp:431-446 and Source/PotentialSolve.cpp:61-72),
// written for sm_100a.  One V-cycle: red-black Gauss-Seidel smoothing,
// residual fused with 2x averaging restriction, piecewise-constant
// prolongation fused into the correction, and a single-CTA BiCGStab bottom
// solve on the coarsest level.  Templated on the working precision so the
// same kernels run the FP64 V-cycles and the FP32 V-cycles of the
// iterative-refinement form.
//
// Boundary closure: a ghost value next to the boundary cell x0 is
//     ghost = c0 * x0 + c1 * x1 + g
// with x1 the next interior cell and g the inhomogeneous part (fine level
// only).  Dirichlet: polynomial extrapolation through the face value and
// the first one or two interior cells; Neumann: reflection; Robin
// a x + b dx/dn = f: the centred two-point closure.  The Gauss-Seidel
// update absorbs c0 into the diagonal so a boundary cell is solved exactly.
#pragma once

#include "vd_common.cuh"
#include <cooperative_groups.h>
#include <vector>


namespace vd {

enum MGBCType
{
    MG_PER = 0,
    MG_DIR = 1,
    MG_NEU = 2,
    MG_INNEU = 3,
    MG_ROBIN = 4
};

template <typename T>
struct MGOp
{
    GridDev g;
    T dh[3];
    T aconst;
    const T* a;
    const T* b[3];
    T bconst;
    int bct[6];
    T c0s[6];
    T c1s[6];
    const T* c0[6];
    const T* gv[6];
    const int* stop; // set to non-zero on the device once the solve has converged
    int* err;        // device word a TMA-staged sweep sets when a wait gives up
    long long big_cells; // host only: levels of at least this many cells (0: 8 M) take the
                         // sweeps built for HBM-resident levels
    int tma;             // host only: those levels' constant-coefficient sweeps are TMA-staged
};

template <typename T>
__device__ __forceinline__ bool mg_stopped(const MGOp<T>& L)
{
    return L.stop && *(volatile const int*)L.stop;
}

__host__ __device__ inline int plane_index(const GridDev& g, int d, int i, int j, int k)
{
    if (d == 0) return j + g.n[1] * k;
    if (d == 1) return i + g.n[0] * k;
    return i + g.n[0] * j;
}

__host__ __device__ inline int plane_count(const GridDev& g, int d)
{
    if (d == 0) return g.n[1] * g.n[2];
    if (d == 1) return g.n[0] * g.n[2];
    return g.n[0] * g.n[1];
}

__host__ __device__ inline long long face_index(const GridDev& g, int d, int i, int j, int k)
{
    const int nx = g.n[0] + (d == 0), ny = g.n[1] + (d == 1);
    return i + (long long)nx * (j + (long long)ny * k);
}

__host__ __device__ inline long long face_count(const GridDev& g, int d)
{
    return (long long)(g.n[0] + (d == 0)) * (g.n[1] + (d == 1)) * (g.n[2] + (d == 2));
}

template <typename T>
__device__ __forceinline__ T mg_face_b(const MGOp<T>& L, int d, int i, int j, int k)
{
    if (!L.b[d]) return L.bconst;
    return L.b[d][face_index(L.g, d, i, j, k)];
}

// Value of the neighbour of cell (i,j,k) one step along D in direction sg,
// through the boundary closure when it falls outside the level; `cf`
// returns the coefficient of x0 inside a ghost value (0 for real cells).
template <int D, typename T>
__device__ __forceinline__ T mg_nbr(const MGOp<T>& L, const T* __restrict__ x, int i,
                                    int j, int k, int sg, bool inhomog, T x0, T& cf)
{
    int ii = i, jj = j, kk = k;
    int& c = (D == 0) ? ii : ((D == 1) ? jj : kk);
    c += sg;
    cf = T(0);
    const int n = L.g.n[D];
    if (c >= 0 && c < n) return x[L.g.idx(ii, jj, kk)];
    if (L.g.per[D])
    {
        c = (c + n) % n;
        return x[L.g.idx(ii, jj, kk)];
    }
    const int s = D + (sg > 0 ? 3 : 0);
    const int p = (D == 0) ? (j + L.g.n[1] * k) : ((D == 1) ? (i + L.g.n[0] * k) : (i + L.g.n[0] * j));
    const T c0 = L.c0[s] ? L.c0[s][p] : L.c0s[s];
    T gh = c0 * x0;
    if (L.c1s[s] != T(0))
    {
        int mi = i, mj = j, mk = k;
        int& m = (D == 0) ? mi : ((D == 1) ? mj : mk);
        m -= sg;
        gh += L.c1s[s] * x[L.g.idx(mi, mj, mk)];
    }
    if (inhomog && L.gv[s]) gh += L.gv[s][p];
    cf = c0;
    return gh;
}

template <int D, typename T>
__device__ __forceinline__ void mg_face_pair(const MGOp<T>& L, int i, int j, int k, T& blo,
                                             T& bhi)
{
    if (!L.b[D])
    {
        blo = bhi = L.bconst;
        return;
    }
    const long long f = face_index(L.g, D, i, j, k);
    const long long st = (D == 0) ? 1
                         : (D == 1) ? (long long)L.g.n[0]
                                    : (long long)L.g.n[0] * L.g.n[1];
    blo = L.b[D][f];
    bhi = L.b[D][f + st];
}

template <int D, typename T>
__device__ __forceinline__ void mg_term(const MGOp<T>& L, const T* __restrict__ x, int i,
                                        int j, int k, bool inhomog, T x0, T& y)
{
    T blo, bhi, cf;
    mg_face_pair<D>(L, i, j, k, blo, bhi);
    const T xm = mg_nbr<D>(L, x, i, j, k, -1, inhomog, x0, cf);
    const T xp = mg_nbr<D>(L, x, i, j, k, +1, inhomog, x0, cf);
    y -= L.dh[D] * (bhi * (xp - x0) - blo * (x0 - xm));
}

template <typename T>
__device__ __forceinline__ T mg_apply(const MGOp<T>& L, const T* __restrict__ x, int i,
                                      int j, int k, bool inhomog)
{
    const long long p = L.g.idx(i, j, k);
    const T x0 = x[p];
    T y = (L.a ? L.a[p] : L.aconst) * x0;
    mg_term<0>(L, x, i, j, k, inhomog, x0, y);
    if (L.g.dim > 1) mg_term<1>(L, x, i, j, k, inhomog, x0, y);
    if (L.g.dim > 2) mg_term<2>(L, x, i, j, k, inhomog, x0, y);
    return y;
}

template <int D, typename T>
__device__ __forceinline__ void mg_gs_term(const MGOp<T>& L, const T* __restrict__ x, int i,
                                           int j, int k, bool inhomog, T x0, T& gamma,
                                           T& rho, T& delta)
{
    T blo, bhi, cfm, cfp;
    mg_face_pair<D>(L, i, j, k, blo, bhi);
    gamma += L.dh[D] * (blo + bhi);
    const T xm = mg_nbr<D>(L, x, i, j, k, -1, inhomog, x0, cfm);
    const T xp = mg_nbr<D>(L, x, i, j, k, +1, inhomog, x0, cfp);
    rho += L.dh[D] * (blo * xm + bhi * xp);
    delta += L.dh[D] * (blo * cfm + bhi * cfp);
}

// Gauss-Seidel update of one cell in place.
template <typename T>
__device__ __forceinline__ void mg_gs_cell(const MGOp<T>& L, T* __restrict__ x,
                                           const T* __restrict__ f, int i, int j, int k,
                                           bool inhomog)
{
    const long long p = L.g.idx(i, j, k);
    const T x0 = x[p];
    T gamma = L.a ? L.a[p] : L.aconst;
    T rho = T(0), delta = T(0);
    mg_gs_term<0>(L, x, i, j, k, inhomog, x0, gamma, rho, delta);
    if (L.g.dim > 1) mg_gs_term<1>(L, x, i, j, k, inhomog, x0, gamma, rho, delta);
    if (L.g.dim > 2) mg_gs_term<2>(L, x, i, j, k, inhomog, x0, gamma, rho, delta);
    const T res = f[p] - (gamma * x0 - rho);
    x[p] = x0 + res / (gamma - delta);
}

__device__ __forceinline__ bool mg_interior(const GridDev& g, int i, int j, int k)
{
    return i > 0 && i < g.n[0] - 1 && (g.dim < 2 || (j > 0 && j < g.n[1] - 1)) &&
           (g.dim < 3 || (k > 0 && k < g.n[2] - 1));
}

// ---------------------------------------------------------------- kernels
template <typename T>
__global__ void k_mg_smooth_color(MGOp<T> L, T* __restrict__ x,
                                  const T* __restrict__ f, int color, int inhomog)
{
    VD_PDL_WAIT();
    if (mg_stopped(L)) return;
    const int nxh = (L.g.n[0] + 1) >> 1;
    const long long tot = (long long)nxh * L.g.n[1] * L.g.n[2];
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < tot;
         t += (long long)gridDim.x * blockDim.x)
    {
        const int ih = (int)(t % nxh);
        const long long r = t / nxh;
        const int j = (int)(r % L.g.n[1]);
        const int k = (int)(r / L.g.n[1]);
        const int i = 2 * ih + ((j + k + color) & 1);
        if (i >= L.g.n[0]) continue;
        mg_gs_cell(L, x, f, i, j, k, inhomog != 0);
    }
}

// One Gauss-Seidel colour on a red-black split level, launched on a grid
// (half-row blocks, ny, nz): the thread's cell and its six neighbours are
// unit-stride loads from the two colour halves.  Interior cells take the
// branch-free path (constant coefficients use the precomputed 1/diagonal);
// boundary cells the general one.
template <typename T, bool VARB>
__global__ void __launch_bounds__(128) k_mg_smooth_rb(MGOp<T> L, T* __restrict__ x,
                                                      const T* __restrict__ f, int color,
                                                      int inhomog, T inv_gamma)
{
    VD_PDL_WAIT();
    if (mg_stopped(L)) return;
    const GridDev& g = L.g;
    const int nxh = g.n[0] >> 1;
    const int ih = blockIdx.x * blockDim.x + threadIdx.x;
    if (ih >= nxh) return;
    const int j = blockIdx.y, k = blockIdx.z;
    const long long half = g.ncell() >> 1;
    const long long plane = (long long)nxh * g.n[1];
    const long long r = j + (long long)g.n[1] * k;
    const long long h = ih + (long long)nxh * r;
    const int q = (j + k + color) & 1;
    const int i = 2 * ih + q;
    if (!mg_interior(g, i, j, k))
    {
        mg_gs_cell(L, x, f, i, j, k, inhomog != 0);
        return;
    }
    T* __restrict__ xs = x + color * half;
    const T* __restrict__ xo = x + (1 - color) * half;
    const T x0 = xs[h];
    const T xm = xo[h - 1 + q], xp = xo[h + q];
    const T ym = xo[h - nxh], yp = xo[h + nxh];
    const T dhx = L.dh[0], dhy = L.dh[1], dhz = L.dh[2];
    const T fv = f[color * half + h];
    if (VARB)
    {
        const long long fx = i + (long long)(g.n[0] + 1) * r;
        const T bxl = L.b[0][fx], bxh = L.b[0][fx + 1];
        const long long fy = i + (long long)g.n[0] * (j + (long long)(g.n[1] + 1) * k);
        const T byl = L.b[1][fy], byh = L.b[1][fy + g.n[0]];
        T gamma = L.aconst;
        gamma += dhx * (bxl + bxh);
        gamma += dhy * (byl + byh);
        T rho = dhx * (bxl * xm + bxh * xp);
        rho += dhy * (byl * ym + byh * yp);
        if (g.dim == 3)
        {
            const long long fz = i + (long long)g.n[0] * r;
            const T bzl = L.b[2][fz], bzh = L.b[2][fz + (long long)g.n[0] * g.n[1]];
            const T zm = xo[h - plane], zp = xo[h + plane];
            gamma += dhz * (bzl + bzh);
            rho += dhz * (bzl * zm + bzh * zp);
        }
        const T res = fv - (gamma * x0 - rho);
        xs[h] = x0 + res / gamma;
    } else
    {
        const T b = L.bconst;
        T rho = dhx * (b * xm + b * xp);
        rho += dhy * (b * ym + b * yp);
        if (g.dim == 3) rho += dhz * (b * xo[h - plane] + b * xo[h + plane]);
        // x0 + (f - (gamma x0 - rho)) / gamma = (f + rho) / gamma
        xs[h] = (fv + rho) * inv_gamma;
    }
}

// One Gauss-Seidel colour on a 3-D red-black split level (nx, ny, nz >= 4),
// one cell per thread on a (half-row x rows x planes) grid.  Rows with j or
// k on the boundary take the general path (whole warps, no divergence);
// in every other row the two x-boundary cells are folded into the fast
// path: the ghost value c0 x0 + c1 x1 + g of the boundary side contributes
// c1 x1 + g to the neighbour sum and c0 to the diagonal, which is the same
// cell equation mg_gs_cell solves (x0 cancels out of the exact update), and
// periodic x wraps to the row's other end.
template <typename T, bool VARB>
__global__ void __launch_bounds__(256) k_mg_smooth_rb3(MGOp<T> L, T* __restrict__ x,
                                                       const T* __restrict__ f, int color,
                                                       int inhomog, T inv_gamma)
{
    VD_PDL_WAIT();
    if (mg_stopped(L)) return;
    const GridDev& g = L.g;
    const int nx = g.n[0], nxh = nx >> 1, ny = g.n[1], nz = g.n[2];
    const int ih = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z;
    if (ih >= nxh || j >= ny) return;
    const int q = (j + k + color) & 1;
    const int i = 2 * ih + q;
    if (j == 0 || j == ny - 1 || k == 0 || k == nz - 1)
    {
        mg_gs_cell(L, x, f, i, j, k, inhomog != 0);
        return;
    }
    const long long half = g.ncell() >> 1;
    const long long plane = (long long)nxh * ny;
    const long long r = j + (long long)ny * k;
    const long long row = (long long)nxh * r;
    const long long h = ih + row;
    T* __restrict__ xs = x + color * half;
    const T* __restrict__ xo = x + (1 - color) * half;
    const bool lo = (i == 0), hi = (i == nx - 1);
    // x neighbours in the other colour: h-1+q and h+q, wrapped or replaced at the ends
    long long im = h - 1 + q, ip = h + q;
    if (lo) im = g.per[0] ? row + nxh - 1 : ip;
    if (hi) ip = g.per[0] ? row : im;
    T xm = xo[im], xp = xo[ip];
    const T ym = xo[h - nxh], yp = xo[h + nxh];
    const T zm = xo[h - plane], zp = xo[h + plane];
    const T fv = f[color * half + h];
    const T dhx = L.dh[0], dhy = L.dh[1], dhz = L.dh[2];
    T bxl, bxh, byl, byh, bzl, bzh;
    if (VARB)
    {
        const long long fx = i + (long long)(nx + 1) * r;
        bxl = L.b[0][fx];
        bxh = L.b[0][fx + 1];
        const long long fy = i + (long long)nx * (j + (long long)(ny + 1) * k);
        byl = L.b[1][fy];
        byh = L.b[1][fy + nx];
        const long long fz = i + (long long)nx * r;
        bzl = L.b[2][fz];
        bzh = L.b[2][fz + (long long)nx * ny];
    } else
        bxl = bxh = byl = byh = bzl = bzh = L.bconst;
    T dsub = T(0); // boundary coefficient absorbed into the diagonal
    if ((lo || hi) && !g.per[0])
    {
        const int s = lo ? 0 : 3;
        const int p = j + ny * k;
        const T c0 = L.c0[s] ? L.c0[s][p] : L.c0s[s];
        T gh = L.c1s[s] * (lo ? xp : xm);
        if (inhomog && L.gv[s]) gh += L.gv[s][p];
        if (lo)
        {
            xm = gh;
            dsub = dhx * bxl * c0;
        } else
        {
            xp = gh;
            dsub = dhx * bxh * c0;
        }
    }
    T rho = dhx * (bxl * xm + bxh * xp);
    rho += dhy * (byl * ym + byh * yp);
    rho += dhz * (bzl * zm + bzh * zp);
    if (VARB || dsub != T(0))
    {
        T gamma = L.aconst;
        gamma += dhx * (bxl + bxh);
        gamma += dhy * (byl + byh);
        gamma += dhz * (bzl + bzh);
        xs[h] = (fv + rho) / (gamma - dsub);
    } else
        xs[h] = (fv + rho) * inv_gamma;
}

// ---------------------------------------------------------------------
// 3-D red-black split levels, several planes per thread.  A thread owns
// half-cell ih of row j in MG3_U consecutive planes and issues every load
// of those cells before any arithmetic (the loads of one sweep are the
// bytes in flight that HBM bandwidth needs); the stop flag is read in
// parallel with them and only gates the stores.  Every cell takes the same
// code: a neighbour outside the level is replaced by its ghost value
// c0 x0 + c1 x1 + g (x1 the neighbour on the opposite side, loaded in its
// place), so the cells next to the boundary cost a few selects instead of
// a divergent general path.  Warps with no such cell skip even those.

#define MG3_U 2

// Boundary data of side s = d + 3 (hi) at plane index p: c0, c1 and the
// inhomogeneous part g of the ghost closure.
template <typename T>
__device__ __forceinline__ void mg3_ghost(const MGOp<T>& L, int s, int p, bool inhomog, T& c0,
                                          T& c1, T& gv)
{
    c0 = L.c0[s] ? L.c0[s][p] : L.c0s[s];
    c1 = L.c1s[s];
    gv = (inhomog && L.gv[s]) ? L.gv[s][p] : T(0);
}

// Face coefficients b[0..5] = x-lo, x-hi, y-lo, y-hi, z-lo, z-hi of cell (i,j,k).
template <typename T, bool VARB>
__device__ __forceinline__ void mg3_faces(const MGOp<T>& L, int i, int j, int k, T* b)
{
    if (!VARB)
    {
#pragma unroll
        for (int m = 0; m < 6; ++m) b[m] = L.bconst;
        return;
    }
    const int nx = L.g.n[0], ny = L.g.n[1];
    const long long r = j + (long long)ny * k;
    const long long fx = i + (long long)(nx + 1) * r;
    b[0] = __ldg(L.b[0] + fx);
    b[1] = __ldg(L.b[0] + fx + 1);
    const long long fy = i + (long long)nx * (j + (long long)(ny + 1) * k);
    b[2] = __ldg(L.b[1] + fy);
    b[3] = __ldg(L.b[1] + fy + nx);
    const long long fz = i + (long long)nx * r;
    b[4] = __ldg(L.b[2] + fz);
    b[5] = __ldg(L.b[2] + fz + (long long)nx * ny);
}

// Offsets (relative to the cell's half-index h in the other colour) of
// the six neighbours x-lo, x-hi, y-lo, y-hi, z-lo, z-hi; a neighbour outside
// the level takes the offset of the opposite one (a valid address whose
// value the ghost closure needs anyway).  Returns the mask of outside sides.
__device__ __forceinline__ int mg3_offsets(const GridDev& g, int i, int j, int k, int q,
                                           long long* off)
{
    const long long nxh = g.n[0] >> 1, plane = nxh * g.n[1];
    const int out = (i == 0) | ((i == g.n[0] - 1) << 1) | ((j == 0) << 2) |
                    ((j == g.n[1] - 1) << 3) | ((k == 0) << 4) | ((k == g.n[2] - 1) << 5);
    off[0] = q - 1;
    off[1] = q;
    off[2] = -nxh;
    off[3] = nxh;
    off[4] = -plane;
    off[5] = plane;
#pragma unroll
    for (int d = 0; d < 3; ++d)
    {
        if (out & (1 << (2 * d))) off[2 * d] = off[2 * d + 1];
        if (out & (2 << (2 * d))) off[2 * d + 1] = off[2 * d];
    }
    return out;
}

// Replace the outside neighbours in nb by their ghost part c1 x1 + g and
// return sum_d dh_d b_side c0 (the ghost's share of x0, absorbed into the
// diagonal).  x1 of an outside side is the opposite neighbour.
template <typename T>
__device__ __forceinline__ T mg3_apply_ghosts(const MGOp<T>& L, int out, int i, int j, int k,
                                              bool inhomog, const T* b, T* nb)
{
    T delta = T(0);
#pragma unroll
    for (int s2 = 0; s2 < 6; ++s2)
    {
        if (!(out & (1 << s2))) continue;
        const int d = s2 >> 1, hi = s2 & 1;
        const int s = d + 3 * hi;
        const int p = (d == 0) ? (j + L.g.n[1] * k) : ((d == 1) ? (i + L.g.n[0] * k) : (i + L.g.n[0] * j));
        T c0, c1, gv;
        mg3_ghost(L, s, p, inhomog, c0, c1, gv);
        nb[s2] = c1 * nb[s2 ^ 1] + gv;
        delta += L.dh[d] * (b[s2] * c0);
    }
    return delta;
}

// One colour of Gauss-Seidel on a 3-D red-black split level (nx even, all
// sizes >= 4, no periodic direction); 256-thread blocks of 32 half-cells by
// 8 rows, grid z over plane groups of MG3_U.  With PROL the other colour is
// read as x + P e (e the coarse correction, P piecewise constant): the
// post-smoothing's first sweep takes the place of the separate
// prolongation pass, which is exact because a Gauss-Seidel value does not
// depend on the cell's own previous value.
//   interior:  x = (f + sum_d dh_d (b_lo x_lo + b_hi x_hi)) / gamma
//   boundary:  the same with ghost parts in the sum and gamma - delta.
template <typename T, bool VARB, bool PROL>
__global__ void __launch_bounds__(256, 4) k_mg_sweep3(const __grid_constant__ MGOp<T> L,
                                                      T* __restrict__ x,
                                                      const T* __restrict__ f, int color,
                                                      int inhomog, T inv_gamma, GridDev gc,
                                                      const T* __restrict__ xc)
{
    VD_PDL_WAIT();
    // the stop flag only changes between kernels: a read-only (cached) load
    const int stop = L.stop ? __ldg(L.stop) : 0;
    if (stop) return;
    const GridDev& g = L.g;
    const int nx = g.n[0], nxh = nx >> 1, ny = g.n[1], nz = g.n[2];
    const int ih = blockIdx.x * 32 + (threadIdx.x & 31);
    const int j = blockIdx.y * 8 + (threadIdx.x >> 5);
    const int k0 = blockIdx.z * MG3_U;
    const bool active = ih < nxh && j < ny;
    const long long half = g.ncell() >> 1;
    T* __restrict__ xs = x + color * half;
    const T* __restrict__ xo = x + (1 - color) * half;
    const T* __restrict__ fs = f + color * half;
    const T dhx = L.dh[0], dhy = L.dh[1], dhz = L.dh[2];
    // warps that touch no boundary cell (nor a partial row) take straight-line
    // code with fixed neighbour offsets (32-bit: half < 2^31 on these levels)
    // (the x ends of each row are in the fast path: their one outside
    // neighbour is the ghost of side x-lo / x-hi)
    const bool edge = active && (j == 0 || j == ny - 1 || k0 == 0 || k0 + MG3_U > nz - 1);
    if (!__any_sync(0xffffffffu, edge))
    {
        if (!active) return;
        const int plane = nxh * ny;
        const int hb = ih + nxh * (j + ny * k0);
        T v[MG3_U][7];
#pragma unroll
        for (int u = 0; u < MG3_U; ++u)
        {
            const int q = (j + k0 + u + color) & 1;
            const int h = hb + u * plane;
            const int i = 2 * ih + q;
            const int xlo = i == 0, xhi = i == nx - 1;
            v[u][0] = __ldg(xo + (h + q - 1 + xlo));
            v[u][1] = __ldg(xo + (h + q - xhi));
            v[u][2] = __ldg(xo + (h - nxh));
            v[u][3] = __ldg(xo + (h + nxh));
            v[u][4] = __ldg(xo + (h - plane));
            v[u][5] = __ldg(xo + (h + plane));
            v[u][6] = __ldg(fs + h);
            if (PROL)
            {
                const int k = k0 + u, I = i >> 1, J = j >> 1, K = k >> 1;
                v[u][0] += __ldg(xc + gc.idx((xlo ? i + 1 : i - 1) >> 1, J, K));
                v[u][1] += __ldg(xc + gc.idx((xhi ? i - 1 : i + 1) >> 1, J, K));
                v[u][2] += __ldg(xc + gc.idx(I, (j - 1) >> 1, K));
                v[u][3] += __ldg(xc + gc.idx(I, (j + 1) >> 1, K));
                v[u][4] += __ldg(xc + gc.idx(I, J, (k - 1) >> 1));
                v[u][5] += __ldg(xc + gc.idx(I, J, (k + 1) >> 1));
            }
        }
#pragma unroll
        for (int u = 0; u < MG3_U; ++u)
        {
            const int q = (j + k0 + u + color) & 1;
            const int i = 2 * ih + q;
            const int xo_ = (i == 0) ? 1 : ((i == nx - 1) ? 2 : 0);
            T b[6];
            mg3_faces<T, VARB>(L, i, j, k0 + u, b);
            T delta = T(0);
            if (xo_) delta = mg3_apply_ghosts(L, xo_, i, j, k0 + u, inhomog != 0, b, v[u]);
            T out;
            if (!VARB)
            {
                const T cb = L.bconst;
                T rho = (dhx * cb) * (v[u][0] + v[u][1]);
                rho = fma(dhy * cb, v[u][2] + v[u][3], rho);
                rho = fma(dhz * cb, v[u][4] + v[u][5], rho);
                if (!xo_)
                    out = (v[u][6] + rho) * inv_gamma;
                else
                {
                    T gamma = L.aconst;
                    gamma += dhx * (cb + cb);
                    gamma += dhy * (cb + cb);
                    gamma += dhz * (cb + cb);
                    out = (v[u][6] + rho) / (gamma - delta);
                }
            } else
            {
                T rho = dhx * (b[0] * v[u][0] + b[1] * v[u][1]);
                rho += dhy * (b[2] * v[u][2] + b[3] * v[u][3]);
                rho += dhz * (b[4] * v[u][4] + b[5] * v[u][5]);
                T gamma = L.aconst;
                gamma += dhx * (b[0] + b[1]);
                gamma += dhy * (b[2] + b[3]);
                gamma += dhz * (b[4] + b[5]);
                out = (v[u][6] + rho) / (gamma - delta);
            }
            if (!stop) xs[hb + u * (nxh * ny)] = out;
        }
        return;
    }
    if (!active) return;
    T v[MG3_U][7];
    int outm[MG3_U];
    long long hh[MG3_U];
#pragma unroll
    for (int u = 0; u < MG3_U; ++u)
    {
        const int k = min(k0 + u, nz - 1);
        const int q = (j + k + color) & 1;
        const int i = 2 * ih + q;
        long long off[6];
        outm[u] = mg3_offsets(g, i, j, k, q, off);
        const long long h = ih + (long long)nxh * (j + (long long)ny * k);
        hh[u] = h;
#pragma unroll
        for (int m = 0; m < 6; ++m) v[u][m] = __ldg(xo + h + off[m]);
        v[u][6] = __ldg(fs + h);
        if (PROL)
        {
            // coarse corrections of the neighbours' parent cells (the
            // coarse level may be in either layout)
            const int ci[6] = {i - 1, i + 1, i, i, i, i}, cj[6] = {j, j, j - 1, j + 1, j, j},
                      ck[6] = {k, k, k, k, k - 1, k + 1};
#pragma unroll
            for (int m = 0; m < 6; ++m)
            {
                const int mm = (outm[u] & (1 << m)) ? (m ^ 1) : m;
                v[u][m] += __ldg(xc + gc.idx(ci[mm] >> 1, cj[mm] >> 1, ck[mm] >> 1));
            }
        }
    }
#pragma unroll
    for (int u = 0; u < MG3_U; ++u)
    {
        const int k = k0 + u;
        if (k >= nz) break;
        const int q = (j + k + color) & 1;
        const int i = 2 * ih + q;
        T b[6];
        mg3_faces<T, VARB>(L, i, j, k, b);
        T delta = T(0);
        if (outm[u]) delta = mg3_apply_ghosts(L, outm[u], i, j, k, inhomog != 0, b, v[u]);
        T out;
        if (!VARB)
        {
            const T cb = L.bconst;
            T rho = (dhx * cb) * (v[u][0] + v[u][1]);
            rho = fma(dhy * cb, v[u][2] + v[u][3], rho);
            rho = fma(dhz * cb, v[u][4] + v[u][5], rho);
            if (delta == T(0))
                out = (v[u][6] + rho) * inv_gamma;
            else
            {
                T gamma = L.aconst; // as the host forms the interior diagonal
                gamma += dhx * (cb + cb);
                gamma += dhy * (cb + cb);
                gamma += dhz * (cb + cb);
                out = (v[u][6] + rho) / (gamma - delta);
            }
        } else
        {
            T rho = dhx * (b[0] * v[u][0] + b[1] * v[u][1]);
            rho += dhy * (b[2] * v[u][2] + b[3] * v[u][3]);
            rho += dhz * (b[4] * v[u][4] + b[5] * v[u][5]);
            T gamma = L.aconst;
            gamma += dhx * (b[0] + b[1]);
            gamma += dhy * (b[2] + b[3]);
            gamma += dhz * (b[4] + b[5]);
            out = (v[u][6] + rho) / (gamma - delta);
        }
        if (!stop) xs[hh[u]] = out;
    }
}

template <typename T>
struct Vec2;
template <>
struct Vec2<double>
{
    using type = double2;
};
template <>
struct Vec2<float>
{
    using type = float2;
};

// Gauss-Seidel value of one cell from its six neighbour values (outside
// ones still to be replaced by ghosts when `out` is non-zero) and f.
template <typename T, bool VARB>
__device__ __forceinline__ T mg3_gs_value(const MGOp<T>& L, int i, int j, int k, int out,
                                          bool inhomog, T inv_gamma, T fv, T* nb)
{
    T b[6];
    mg3_faces<T, VARB>(L, i, j, k, b);
    T delta = T(0);
    if (out) delta = mg3_apply_ghosts(L, out, i, j, k, inhomog, b, nb);
    const T dhx = L.dh[0], dhy = L.dh[1], dhz = L.dh[2];
    if (!VARB)
    {
        const T cb = L.bconst;
        T rho = (dhx * cb) * (nb[0] + nb[1]);
        rho = fma(dhy * cb, nb[2] + nb[3], rho);
        rho = fma(dhz * cb, nb[4] + nb[5], rho);
        if (!out) return (fv + rho) * inv_gamma;
        T gamma = L.aconst; // as the host forms the interior diagonal
        gamma += dhx * (cb + cb);
        gamma += dhy * (cb + cb);
        gamma += dhz * (cb + cb);
        return (fv + rho) / (gamma - delta);
    }
    T rho = dhx * (b[0] * nb[0] + b[1] * nb[1]);
    rho += dhy * (b[2] * nb[2] + b[3] * nb[3]);
    rho += dhz * (b[4] * nb[4] + b[5] * nb[5]);
    T gamma = L.aconst;
    gamma += dhx * (b[0] + b[1]);
    gamma += dhy * (b[2] + b[3]);
    gamma += dhz * (b[4] + b[5]);
    return (fv + rho) / (gamma - delta);
}

// One colour of Gauss-Seidel, two adjacent half-cells per thread with
// 16-byte (two-element) loads and stores: of a pair's x neighbours three
// are distinct (one vector and one scalar load), and its y, z neighbours
// and f are vectors.  Needs nx % 4 == 0 (pairs never straddle a row and
// rows start 16-byte aligned).  Blocks of 32 pairs by 8 rows, MG3_UV planes
// per thread (2 on the finest levels, 1 on smaller ones, where more CTAs
// matter more: measured); warps with a row or plane on the level boundary
// update their cells one by one with the ghost closure.
//
// NORM (a colour-0 sweep that starts a V-cycle): the kernel also forms the
// residual f - L(x) of each cell it updates from the values it already holds
// (the neighbours, f, and the cell's previous value, one more load), i.e.
// the colour-0 residual of the previous cycle's result, and writes the
// per-block max |r| to part[] -- the convergence norm of that cycle without a
// pass of its own (the colour-1 residuals are zero after the previous
// cycle's last sweep).  Same mg3_residual arithmetic as k_mg_resid3v.
// CTAs per SM the sweep's registers are sized for: 4 (64 registers) for
// constant coefficients; 3 for face coefficients, whose extra loads spill at
// 64 (measured at 256^3: 0.11 ms per step less).
#ifndef VD_SWEEP_VARB_MINB
#define VD_SWEEP_VARB_MINB 3
#endif
template <typename T, bool VARB, bool PROL, int MG3_UV, bool NORM = false>
// The norm-carrying sweep (one more load and the residual per cell) also
// at 3 CTAs per SM: 0.07 ms per 256^3 step.
#ifndef VD_SWEEP_NORM_MINB
#define VD_SWEEP_NORM_MINB 3
#endif
__global__ void __launch_bounds__(256, VARB ? VD_SWEEP_VARB_MINB : (NORM ? VD_SWEEP_NORM_MINB : 4))
    k_mg_sweep3v(const __grid_constant__ MGOp<T> L,
                                                       T* __restrict__ x,
                                                       const T* __restrict__ f, int color,
                                                       int inhomog, T inv_gamma, GridDev gc,
                                                       const T* __restrict__ xc,
                                                       double* __restrict__ part)
{
    VD_PDL_WAIT();
    __shared__ double shm[NORM ? 32 : 1];
    double mres = 0.0;
    using V2 = typename Vec2<T>::type;
    // the stop flag only changes between kernels: a read-only (cached) load
    const int stop = L.stop ? __ldg(L.stop) : 0;
    if (stop) return;
    const GridDev& g = L.g;
    const int nx = g.n[0], nxh = nx >> 1, ny = g.n[1], nz = g.n[2];
    const int pr = blockIdx.x * 32 + (threadIdx.x & 31); // pair index: half-cells 2pr, 2pr+1
    const int j = blockIdx.y * 8 + (threadIdx.x >> 5);
    const int k0 = blockIdx.z * MG3_UV;
    const bool active = 2 * pr < nxh && j < ny;
    const long long half = g.ncell() >> 1;
    T* __restrict__ xs = x + color * half;
    const T* __restrict__ xo = x + (1 - color) * half;
    const T* __restrict__ fs = f + color * half;
    const bool edge = active && (j == 0 || j == ny - 1 || k0 == 0 || k0 + MG3_UV > nz - 1);
    const bool fastw = !__any_sync(0xffffffffu, edge);
    if (fastw && active)
    {
        const int plane = nxh * ny;
        const int hb = 2 * pr + nxh * (j + ny * k0);
        V2 vx[MG3_UV], vym[MG3_UV], vyp[MG3_UV], vzm[MG3_UV], vzp[MG3_UV], vf[MG3_UV];
        V2 v0[NORM ? MG3_UV : 1];
        T sx[MG3_UV];
#pragma unroll
        for (int u = 0; u < MG3_UV; ++u)
        {
            const int q = (j + k0 + u + color) & 1;
            const int h = hb + u * plane;
            // the pair's outer x neighbour: 2pr-1 (q = 0) or 2pr+2 (q = 1);
            // at the ends of a row the ghost closure replaces it
            const bool xlo = q == 0 && pr == 0, xhi = q == 1 && 2 * pr + 2 == nxh;
            const int so = q ? (xhi ? 1 : 2) : (xlo ? 0 : -1);
            vx[u] = __ldg(reinterpret_cast<const V2*>(xo + h));
            sx[u] = __ldg(xo + h + so);
            vym[u] = __ldg(reinterpret_cast<const V2*>(xo + h - nxh));
            vyp[u] = __ldg(reinterpret_cast<const V2*>(xo + h + nxh));
            vzm[u] = __ldg(reinterpret_cast<const V2*>(xo + h - plane));
            vzp[u] = __ldg(reinterpret_cast<const V2*>(xo + h + plane));
            vf[u] = __ldg(reinterpret_cast<const V2*>(fs + h));
            if (NORM) v0[u] = __ldg(reinterpret_cast<const V2*>(xs + h));
        }
        // prolongation on the fly: an other-colour neighbour at half-index
        // h' of row j has coarse column h'; cells A, B (coarse columns 2pr,
        // 2pr+1) share their y and z neighbours' coarse rows and planes
        T cxv[MG3_UV][3], cyz[MG3_UV][8];
        if (PROL)
        {
#pragma unroll
            for (int u = 0; u < MG3_UV; ++u)
            {
                const int k = k0 + u;
                const int q = (j + k + color) & 1;
                const int J = j >> 1, K = k >> 1;
#pragma unroll
                for (int e = 0; e < 3; ++e)
                {
                    const int I = min(max(2 * pr - 1 + q + e, 0), nxh - 1);
                    cxv[u][e] = __ldg(xc + gc.idx(I, J, K));
                }
                const int Jm = (j - 1) >> 1, Jp = (j + 1) >> 1, Km = (k - 1) >> 1,
                          Kp = (k + 1) >> 1;
#pragma unroll
                for (int e = 0; e < 2; ++e)
                {
                    const int I = 2 * pr + e;
                    cyz[u][e] = __ldg(xc + gc.idx(I, Jm, K));
                    cyz[u][2 + e] = __ldg(xc + gc.idx(I, Jp, K));
                    cyz[u][4 + e] = __ldg(xc + gc.idx(I, J, Km));
                    cyz[u][6 + e] = __ldg(xc + gc.idx(I, J, Kp));
                }
            }
        }
#pragma unroll
        for (int u = 0; u < MG3_UV; ++u)
        {
            const int k = k0 + u;
            const int q = (j + k + color) & 1;
            const int iA = 4 * pr + q, iB = iA + 2;
            if (PROL)
            {
                // half-indices 2pr-1+q .. 2pr+1+q of the other colour
                if (q == 0)
                {
                    sx[u] += cxv[u][0];
                    vx[u].x += cxv[u][1];
                    vx[u].y += cxv[u][2];
                } else
                {
                    vx[u].x += cxv[u][0];
                    vx[u].y += cxv[u][1];
                    sx[u] += cxv[u][2];
                }
                vym[u].x += cyz[u][0];
                vym[u].y += cyz[u][1];
                vyp[u].x += cyz[u][2];
                vyp[u].y += cyz[u][3];
                vzm[u].x += cyz[u][4];
                vzm[u].y += cyz[u][5];
                vzp[u].x += cyz[u][6];
                vzp[u].y += cyz[u][7];
            }
            T nA[6], nB[6];
            if (q == 0)
            {
                nA[0] = sx[u];
                nA[1] = vx[u].x;
                nB[0] = vx[u].x;
                nB[1] = vx[u].y;
            } else
            {
                nA[0] = vx[u].x;
                nA[1] = vx[u].y;
                nB[0] = vx[u].y;
                nB[1] = sx[u];
            }
            nA[2] = vym[u].x;
            nB[2] = vym[u].y;
            nA[3] = vyp[u].x;
            nB[3] = vyp[u].y;
            nA[4] = vzm[u].x;
            nB[4] = vzm[u].y;
            nA[5] = vzp[u].x;
            nB[5] = vzp[u].y;
            const int oA = (iA == 0) ? 1 : 0, oB = (iB == nx - 1) ? 2 : 0;
            if (NORM)
            {
                T rA[6], rB[6], bA[6], bB[6];
#pragma unroll
                for (int m = 0; m < 6; ++m)
                {
                    rA[m] = nA[m];
                    rB[m] = nB[m];
                }
                mg3_faces<T, VARB>(L, iA, j, k, bA);
                mg3_faces<T, VARB>(L, iB, j, k, bB);
                const double ra = fabs((double)mg3_residual(L, vf[u].x, v0[u].x, rA, bA, oA, iA,
                                                            j, k, inhomog != 0));
                const double rb = fabs((double)mg3_residual(L, vf[u].y, v0[u].y, rB, bB, oB, iB,
                                                            j, k, inhomog != 0));
                mres = nanmax(mres, nanmax(ra, rb));
            }
            V2 o;
            o.x = mg3_gs_value<T, VARB>(L, iA, j, k, oA, inhomog != 0, inv_gamma, vf[u].x, nA);
            o.y = mg3_gs_value<T, VARB>(L, iB, j, k, oB, inhomog != 0, inv_gamma, vf[u].y, nB);
            if (!stop) *reinterpret_cast<V2*>(xs + hb + u * plane) = o;
        }
    }
    // boundary rows and planes: cell by cell
#pragma unroll 1
    for (int u = 0; u < ((!fastw && active) ? MG3_UV : 0); ++u)
    {
        const int k = k0 + u;
        if (k >= nz) break;
        for (int e = 0; e < 2; ++e)
        {
            const int ih = 2 * pr + e;
            const int q = (j + k + color) & 1;
            const int i = 2 * ih + q;
            long long off[6];
            const int out = mg3_offsets(g, i, j, k, q, off);
            const long long h = ih + (long long)nxh * (j + (long long)ny * k);
            T nb[6];
#pragma unroll
            for (int m = 0; m < 6; ++m) nb[m] = __ldg(xo + h + off[m]);
            if (PROL)
            {
                const int ci[6] = {i - 1, i + 1, i, i, i, i}, cj[6] = {j, j, j - 1, j + 1, j, j},
                          ck[6] = {k, k, k, k, k - 1, k + 1};
#pragma unroll
                for (int m = 0; m < 6; ++m)
                {
                    const int mm = (out & (1 << m)) ? (m ^ 1) : m;
                    nb[m] += __ldg(xc + gc.idx(ci[mm] >> 1, cj[mm] >> 1, ck[mm] >> 1));
                }
            }
            const T fv = __ldg(fs + h);
            if (NORM)
            {
                T rn[6], b[6];
#pragma unroll
                for (int m = 0; m < 6; ++m) rn[m] = nb[m];
                mg3_faces<T, VARB>(L, i, j, k, b);
                mres = nanmax(mres, fabs((double)mg3_residual(L, fv, __ldg(xs + h), rn, b, out, i,
                                                            j, k, inhomog != 0)));
            }
            const T v = mg3_gs_value<T, VARB>(L, i, j, k, out, inhomog != 0, inv_gamma, fv, nb);
            if (!stop) xs[h] = v;
        }
    }
    if (NORM)
    {
        mres = block_max(mres, shm);
        if (threadIdx.x == 0)
            part[blockIdx.x + (long long)gridDim.x * (blockIdx.y + (long long)gridDim.y * blockIdx.z)] =
                mres;
    }
}

// Prolongation for the post-smoothing: x += P e on the colour-1 cells only
// (the colour-0 cells are rewritten by the first sweep, colour 0, which
// does not read their previous values).  Pairs of half-cells per thread
// (nx % 4 == 0); colour-1 cells 4pr+q1 and 4pr+2+q1 of row j have coarse
// columns 2pr and 2pr+1.  Grid as k_mg_sweep3v.
template <typename T>
__global__ void __launch_bounds__(256) k_mg_prolong_c1(GridDev g, GridDev gc, T* __restrict__ x,
                                                       const T* __restrict__ xc,
                                                       const int* stop)
{
    VD_PDL_WAIT();
    using V2 = typename Vec2<T>::type;
    if (stop && *(volatile const int*)stop) return;
    const int nxh = g.n[0] >> 1, ny = g.n[1], nz = g.n[2];
    const int pr = blockIdx.x * 32 + (threadIdx.x & 31);
    const int j = blockIdx.y * 8 + (threadIdx.x >> 5);
    const int k0 = blockIdx.z * MG3_U;
    if (2 * pr >= nxh || j >= ny) return;
    T* __restrict__ x1 = x + (g.ncell() >> 1);
#pragma unroll
    for (int u = 0; u < MG3_U; ++u)
    {
        const int k = k0 + u;
        if (k >= nz) break;
        const long long h = 2 * pr + (long long)nxh * (j + (long long)ny * k);
        V2 v = *reinterpret_cast<const V2*>(x1 + h);
        v.x += __ldg(xc + gc.idx(2 * pr, j >> 1, k >> 1));
        v.y += __ldg(xc + gc.idx(2 * pr + 1, j >> 1, k >> 1));
        *reinterpret_cast<V2*>(x1 + h) = v;
    }
}

// Residual f - L(x) of one cell from its value x0 and neighbour values nb
// (outside ones replaced in place by their ghost parts; the ghost's c0 x0
// share enters through delta): mg_apply's operator.
template <typename T>
__device__ __forceinline__ T mg3_residual(const MGOp<T>& L, T fv, T x0, T* nb, const T* b,
                                          int out, int i, int j, int k, bool inhomog)
{
    if (out)
    {
#pragma unroll
        for (int s2 = 0; s2 < 6; ++s2)
        {
            if (!(out & (1 << s2))) continue;
            const int d = s2 >> 1, hi = s2 & 1;
            const int s = d + 3 * hi;
            const int p = (d == 0) ? (j + L.g.n[1] * k) : ((d == 1) ? (i + L.g.n[0] * k) : (i + L.g.n[0] * j));
            T c0, c1, gv;
            mg3_ghost(L, s, p, inhomog, c0, c1, gv);
            nb[s2] = c0 * x0 + (c1 * nb[s2 ^ 1] + gv);
        }
    }
    T y = L.aconst * x0;
    y -= L.dh[0] * (b[1] * (nb[1] - x0) - b[0] * (x0 - nb[0]));
    y -= L.dh[1] * (b[3] * (nb[3] - x0) - b[2] * (x0 - nb[2]));
    y -= L.dh[2] * (b[5] * (nb[5] - x0) - b[4] * (x0 - nb[4]));
    return fv - y;
}

// Residual f - L(x) at the 8 children of every coarse cell, averaged into
// the coarse right-hand side (order kk, jj, ii as k_mg_resid_restrict); the
// coarse unknown zeroed.  3-D red-black split fine level; blocks of 32
// coarse cells in x by 8 coarse rows, one coarse plane per grid z.
// C0ONLY: after pre-smoothing, whose last sweep is colour 1, the colour-1
// residuals are zero up to rounding, so only the four colour-0 children are
// summed (reads 12 instead of 16 B/cell: no colour-1 f).
// CTAs per SM for the restriction (measured at 256^3: 4 is 0.13 ms per step
// faster than 3 once only the colour-0 children are read).
#ifndef VD_RESTRICT_MINB
#define VD_RESTRICT_MINB 4
#endif
template <typename T, bool VARB, bool C0ONLY = false>
__global__ void __launch_bounds__(256, VD_RESTRICT_MINB) k_mg_restrict3(const __grid_constant__ MGOp<T> L,
                                                      const T* __restrict__ x,
                                                      const T* __restrict__ f, GridDev gc,
                                                      T* __restrict__ fc, T* __restrict__ xc,
                                                      int inhomog)
{
    VD_PDL_WAIT();
    // the stop flag only changes between kernels: a read-only (cached) load
    const int stop = L.stop ? __ldg(L.stop) : 0;
    if (stop) return;
    const GridDev& g = L.g;
    const int nxh = g.n[0] >> 1, ny = g.n[1];
    const int I = blockIdx.x * 32 + (threadIdx.x & 31);
    const int J = blockIdx.y * 8 + (threadIdx.x >> 5);
    const int K = blockIdx.z;
    const bool active = I < gc.n[0] && J < gc.n[1];
    const long long half = g.ncell() >> 1;
    T s = T(0);
    const bool edge = active && (J == 0 || J == gc.n[1] - 1 || K == 0 || K == gc.n[2] - 1);
    if (!__any_sync(0xffffffffu, edge))
    {
        if (!active) return;
        // no child on the level boundary: fixed offsets, 32-bit indices
        const int plane = nxh * ny;
#pragma unroll
        for (int kk = 0; kk < 2; ++kk)
        {
            T xv[4][8];
#pragma unroll
            for (int jj = 0; jj < 2; ++jj)
#pragma unroll
                for (int ii = 0; ii < 2; ++ii)
                {
                    const int m = ii + 2 * jj;
                    const int c = (ii + jj + kk) & 1;
                    if (C0ONLY && c) continue;
                    const int h = I + nxh * (2 * J + jj + ny * (2 * K + kk));
                    const T* xs = x + c * half;
                    const T* xo = x + (1 - c) * half;
                    const int i = 2 * I + ii;
                    const int xlo = i == 0, xhi = i == g.n[0] - 1;
                    xv[m][0] = __ldg(xo + (h + ii - 1 + xlo));
                    xv[m][1] = __ldg(xo + (h + ii - xhi));
                    xv[m][2] = __ldg(xo + (h - nxh));
                    xv[m][3] = __ldg(xo + (h + nxh));
                    xv[m][4] = __ldg(xo + (h - plane));
                    xv[m][5] = __ldg(xo + (h + plane));
                    xv[m][6] = __ldg(xs + h);
                    xv[m][7] = __ldg(f + c * half + h);
                }
#pragma unroll
            for (int jj = 0; jj < 2; ++jj)
#pragma unroll
                for (int ii = 0; ii < 2; ++ii)
                {
                    const int m = ii + 2 * jj;
                    if (C0ONLY && ((ii + jj + kk) & 1)) continue;
                    const int i = 2 * I + ii;
                    const int xo_ = (i == 0) ? 1 : ((i == g.n[0] - 1) ? 2 : 0);
                    T b[6];
                    mg3_faces<T, VARB>(L, i, 2 * J + jj, 2 * K + kk, b);
                    s += mg3_residual(L, xv[m][7], xv[m][6], xv[m], b, xo_, i, 2 * J + jj,
                                      2 * K + kk, inhomog != 0);
                }
        }
        if (stop) return;
        const long long pc = gc.idx(I, J, K);
        fc[pc] = s * T(0.125);
        xc[pc] = T(0);
        return;
    }
    if (!active) return;
#pragma unroll
    for (int kk = 0; kk < 2; ++kk)
    {
        // the four children of this plane: every load first
        T xv[4][8];
        int outm[4];
#pragma unroll
        for (int jj = 0; jj < 2; ++jj)
#pragma unroll
            for (int ii = 0; ii < 2; ++ii)
            {
                const int m = ii + 2 * jj;
                const int i = 2 * I + ii, j = 2 * J + jj, k = 2 * K + kk;
                const int c = (ii + jj + kk) & 1;
                if (C0ONLY && c) continue;
                long long off[6];
                outm[m] = mg3_offsets(g, i, j, k, ii, off);
                const long long h = I + (long long)nxh * (j + (long long)ny * k);
                const T* xs = x + c * half;
                const T* xo = x + (1 - c) * half;
                xv[m][6] = __ldg(xs + h);
#pragma unroll
                for (int d = 0; d < 6; ++d) xv[m][d] = __ldg(xo + h + off[d]);
                xv[m][7] = __ldg(f + c * half + h);
            }
#pragma unroll
        for (int jj = 0; jj < 2; ++jj)
#pragma unroll
            for (int ii = 0; ii < 2; ++ii)
            {
                const int m = ii + 2 * jj;
                if (C0ONLY && ((ii + jj + kk) & 1)) continue;
                const int i = 2 * I + ii, j = 2 * J + jj, k = 2 * K + kk;
                T b[6];
                mg3_faces<T, VARB>(L, i, j, k, b);
                s += mg3_residual(L, xv[m][7], xv[m][6], xv[m], b, outm[m], i, j, k,
                                  inhomog != 0);
            }
    }
    if (stop) return;
    const long long pc = gc.idx(I, J, K);
    fc[pc] = s * T(0.125);
    xc[pc] = T(0);
}

// The same residual max-norm with two adjacent half-cells per thread and
// 16-byte accesses (nx % 4 == 0), as k_mg_sweep3v; outputs and arguments as
// k_mg_resid3.  Blocks of 32 pairs by 8 rows, MG3_U planes per thread.
template <typename T, bool VARB>
// CTAs per SM the residual's registers are sized for: 3 (80 registers) for
// constant coefficients and 2 (128) for face coefficients; at 4 (64) both
// spilled 112-240 B (measured at 256^3: 18.78-18.82 -> 18.68 ms per step).
#ifndef VD_RESID_MINB
#define VD_RESID_MINB 3
#endif
#ifndef VD_RESID_VARB_MINB
#define VD_RESID_VARB_MINB 2
#endif
__global__ void __launch_bounds__(256, VARB ? VD_RESID_VARB_MINB : VD_RESID_MINB)
    k_mg_resid3v(const __grid_constant__ MGOp<T> L,
                                                       const T* __restrict__ x,
                                                       const T* __restrict__ f,
                                                       T* __restrict__ rout, int inhomog,
                                                       int both, int fnorm,
                                                       double* __restrict__ part,
                                                       float* __restrict__ r32 = nullptr,
                                                       float* __restrict__ x32 = nullptr,
                                                       const double* rscale = nullptr)
{
    VD_PDL_WAIT();
    using V2 = typename Vec2<T>::type;
    __shared__ double sh[32];
    const int stop = L.stop ? __ldg(L.stop) : 0;
    if (stop) return;
    const GridDev& g = L.g;
    const int nx = g.n[0], nxh = nx >> 1, ny = g.n[1], nz = g.n[2];
    const int pr = blockIdx.x * 32 + (threadIdx.x & 31);
    const int j = blockIdx.y * 8 + (threadIdx.x >> 5);
    const int k0 = blockIdx.z * MG3_U;
    const bool active = 2 * pr < nxh && j < ny;
    const long long half = g.ncell() >> 1;
    const bool edge = active && (j == 0 || j == ny - 1 || k0 == 0 || k0 + MG3_U > nz - 1);
    const bool fastw = !__any_sync(0xffffffffu, edge);
    const double rs = r32 ? *rscale : 0.0;
    double m = 0.0, mf = 0.0;
    auto emit = [&](long long o, T r, T fv, bool wr) {
        if (wr && rout) rout[o] = r;
        if (r32)
        {
            r32[o] = (float)((double)r * rs);
            x32[o] = 0.0f;
        }
        const double a = fabs((double)r);
        m = nanmax(m, a);
        if (fnorm)
        {
            const double af = fabs((double)fv);
            mf = nanmax(mf, af);
        }
    };
    for (int col = 0; col < (both ? 2 : 1); ++col)
    {
        const T* xs = x + col * half;
        const T* xo = x + (1 - col) * half;
        const T* fc = f + col * half;
        if (!active) continue;
        if (fastw)
        {
            const int plane = nxh * ny;
            const int hb = 2 * pr + nxh * (j + ny * k0);
            V2 vx[MG3_U], vym[MG3_U], vyp[MG3_U], vzm[MG3_U], vzp[MG3_U], vf[MG3_U], v0[MG3_U];
            T sx[MG3_U];
#pragma unroll
            for (int u = 0; u < MG3_U; ++u)
            {
                const int q = (j + k0 + u + col) & 1;
                const int h = hb + u * plane;
                const bool xlo = q == 0 && pr == 0, xhi = q == 1 && 2 * pr + 2 == nxh;
                const int so = q ? (xhi ? 1 : 2) : (xlo ? 0 : -1);
                v0[u] = __ldg(reinterpret_cast<const V2*>(xs + h));
                vx[u] = __ldg(reinterpret_cast<const V2*>(xo + h));
                sx[u] = __ldg(xo + h + so);
                vym[u] = __ldg(reinterpret_cast<const V2*>(xo + h - nxh));
                vyp[u] = __ldg(reinterpret_cast<const V2*>(xo + h + nxh));
                vzm[u] = __ldg(reinterpret_cast<const V2*>(xo + h - plane));
                vzp[u] = __ldg(reinterpret_cast<const V2*>(xo + h + plane));
                vf[u] = __ldg(reinterpret_cast<const V2*>(fc + h));
            }
#pragma unroll
            for (int u = 0; u < MG3_U; ++u)
            {
                const int k = k0 + u;
                const int q = (j + k + col) & 1;
                const int iA = 4 * pr + q, iB = iA + 2;
                T nA[6], nB[6];
                if (q == 0)
                {
                    nA[0] = sx[u];
                    nA[1] = vx[u].x;
                    nB[0] = vx[u].x;
                    nB[1] = vx[u].y;
                } else
                {
                    nA[0] = vx[u].x;
                    nA[1] = vx[u].y;
                    nB[0] = vx[u].y;
                    nB[1] = sx[u];
                }
                nA[2] = vym[u].x;
                nB[2] = vym[u].y;
                nA[3] = vyp[u].x;
                nB[3] = vyp[u].y;
                nA[4] = vzm[u].x;
                nB[4] = vzm[u].y;
                nA[5] = vzp[u].x;
                nB[5] = vzp[u].y;
                T bA[6], bB[6];
                mg3_faces<T, VARB>(L, iA, j, k, bA);
                mg3_faces<T, VARB>(L, iB, j, k, bB);
                const int oA = (iA == 0) ? 1 : 0, oB = (iB == nx - 1) ? 2 : 0;
                const T rA = mg3_residual(L, vf[u].x, v0[u].x, nA, bA, oA, iA, j, k, inhomog != 0);
                const T rB = mg3_residual(L, vf[u].y, v0[u].y, nB, bB, oB, iB, j, k, inhomog != 0);
                const long long o = col * half + hb + u * plane;
                if (rout)
                {
                    V2 w;
                    w.x = rA;
                    w.y = rB;
                    *reinterpret_cast<V2*>(rout + o) = w;
                }
                emit(o, rA, vf[u].x, false);
                emit(o + 1, rB, vf[u].y, false);
            }
            continue;
        }
        // boundary rows and planes: cell by cell
#pragma unroll 1
        for (int u = 0; u < MG3_U; ++u)
        {
            const int k = k0 + u;
            if (k >= nz) break;
            for (int e = 0; e < 2; ++e)
            {
                const int ih = 2 * pr + e;
                const int q = (j + k + col) & 1;
                const int i = 2 * ih + q;
                long long off[6];
                const int out = mg3_offsets(g, i, j, k, q, off);
                const long long h = ih + (long long)nxh * (j + (long long)ny * k);
                T nb[6];
#pragma unroll
                for (int d = 0; d < 6; ++d) nb[d] = __ldg(xo + h + off[d]);
                T b[6];
                mg3_faces<T, VARB>(L, i, j, k, b);
                const T fv = __ldg(fc + h);
                const T r = mg3_residual(L, fv, __ldg(xs + h), nb, b, out, i, j, k, inhomog != 0);
                emit(col * half + h, r, fv, true);
            }
        }
    }
    m = block_max(m, sh);
    if (fnorm) mf = block_max(mf, sh);
    if (threadIdx.x == 0)
    {
        const long long nb = (long long)gridDim.x * gridDim.y * gridDim.z;
        const long long b = blockIdx.x + (long long)gridDim.x * (blockIdx.y + (long long)gridDim.y * blockIdx.z);
        part[b] = m;
        if (fnorm) part[nb + b] = mf;
    }
}

// Residual max-norm on a 3-D red-black split level: cells of colour 0 only
// (after a sweep of colour 1 the colour-1 residuals vanish: each such cell
// was just solved exactly from its colour-0 neighbours) or of both colours;
// the residual itself into rout when given, |f| max with fnorm.  Grid as
// k_mg_sweep3; per-block maxima into part[b] (part[nb + b] for |f|).
template <typename T, bool VARB>
__global__ void __launch_bounds__(256, 4) k_mg_resid3(const __grid_constant__ MGOp<T> L,
                                                      const T* __restrict__ x,
                                                      const T* __restrict__ f,
                                                      T* __restrict__ rout, int inhomog, int both,
                                                      int fnorm, double* __restrict__ part,
                                                      float* __restrict__ r32 = nullptr,
                                                      float* __restrict__ x32 = nullptr,
                                                      const double* rscale = nullptr)
{
    VD_PDL_WAIT();
    __shared__ double sh[32];
    // the stop flag only changes between kernels: a read-only (cached) load
    const int stop = L.stop ? __ldg(L.stop) : 0;
    if (stop) return;
    const GridDev& g = L.g;
    const int nx = g.n[0], nxh = nx >> 1, ny = g.n[1], nz = g.n[2];
    const int ih = blockIdx.x * 32 + (threadIdx.x & 31);
    const int j = blockIdx.y * 8 + (threadIdx.x >> 5);
    const int k0 = blockIdx.z * MG3_U;
    const long long half = g.ncell() >> 1;
    const bool active = ih < nxh && j < ny;
    const bool edge = active && (j == 0 || j == ny - 1 || k0 == 0 || k0 + MG3_U > nz - 1);
    const bool fastw = !__any_sync(0xffffffffu, edge);
    // refinement form: r32 = r * rscale (the previous residual's 1/max), x32 = 0
    const double rs = r32 ? *rscale : 0.0;
    double m = 0.0, mf = 0.0;
    for (int col = 0; col < (both ? 2 : 1); ++col)
    {
        const T* xs = x + col * half;
        const T* xo = x + (1 - col) * half;
        const T* fc = f + col * half;
        if (fastw && !active) continue;
        if (fastw)
        {
            const int plane = nxh * ny;
            const int hb = ih + nxh * (j + ny * k0);
            T v[MG3_U][8];
#pragma unroll
            for (int u = 0; u < MG3_U; ++u)
            {
                const int q = (j + k0 + u + col) & 1;
                const int h = hb + u * plane;
                const int i = 2 * ih + q;
                const int xlo = i == 0, xhi = i == nx - 1;
                v[u][0] = __ldg(xo + (h + q - 1 + xlo));
                v[u][1] = __ldg(xo + (h + q - xhi));
                v[u][2] = __ldg(xo + (h - nxh));
                v[u][3] = __ldg(xo + (h + nxh));
                v[u][4] = __ldg(xo + (h - plane));
                v[u][5] = __ldg(xo + (h + plane));
                v[u][6] = __ldg(xs + h);
                v[u][7] = __ldg(fc + h);
            }
#pragma unroll
            for (int u = 0; u < MG3_U; ++u)
            {
                const int q = (j + k0 + u + col) & 1;
                const int i = 2 * ih + q;
                const int xo_ = (i == 0) ? 1 : ((i == nx - 1) ? 2 : 0);
                T b[6];
                mg3_faces<T, VARB>(L, i, j, k0 + u, b);
                const T r = mg3_residual(L, v[u][7], v[u][6], v[u], b, xo_, i, j, k0 + u,
                                         inhomog != 0);
                if (rout && !stop) rout[col * half + hb + u * plane] = r;
                if (r32 && !stop)
                {
                    r32[col * half + hb + u * plane] = (float)((double)r * rs);
                    x32[col * half + hb + u * plane] = 0.0f;
                }
                const double a = fabs((double)r);
                m = nanmax(m, a);
                if (fnorm)
                {
                    const double af = fabs((double)v[u][7]);
                    mf = nanmax(mf, af);
                }
            }
            continue;
        }
        if (!active) continue;
        T v[MG3_U][8];
        int outm[MG3_U];
#pragma unroll
        for (int u = 0; u < MG3_U; ++u)
        {
            const int k = min(k0 + u, nz - 1);
            const int q = (j + k + col) & 1;
            const int i = 2 * ih + q;
            long long off[6];
            outm[u] = mg3_offsets(g, i, j, k, q, off);
            const long long h = ih + (long long)nxh * (j + (long long)ny * k);
            v[u][6] = __ldg(xs + h);
#pragma unroll
            for (int d = 0; d < 6; ++d) v[u][d] = __ldg(xo + h + off[d]);
            v[u][7] = __ldg(fc + h);
        }
#pragma unroll
        for (int u = 0; u < MG3_U; ++u)
        {
            const int k = k0 + u;
            if (k >= nz) break;
            const int q = (j + k + col) & 1;
            const int i = 2 * ih + q;
            T b[6];
            mg3_faces<T, VARB>(L, i, j, k, b);
            const T r =
                mg3_residual(L, v[u][7], v[u][6], v[u], b, outm[u], i, j, k, inhomog != 0);
            if (rout && !stop) rout[col * half + ih + (long long)nxh * (j + (long long)ny * k)] = r;
            if (r32 && !stop)
            {
                const long long o = col * half + ih + (long long)nxh * (j + (long long)ny * k);
                r32[o] = (float)((double)r * rs);
                x32[o] = 0.0f;
            }
            const double a = fabs((double)r);
            m = nanmax(m, a);
            if (fnorm)
            {
                const double af = fabs((double)v[u][7]);
                mf = nanmax(mf, af);
            }
        }
    }
    m = block_max(m, sh);
    if (fnorm) mf = block_max(mf, sh);
    if (threadIdx.x == 0)
    {
        const long long nb = (long long)gridDim.x * gridDim.y * gridDim.z;
        const long long b = blockIdx.x + (long long)gridDim.x * (blockIdx.y + (long long)gridDim.y * blockIdx.z);
        part[b] = m;
        if (fnorm) part[nb + b] = mf;
    }
}

// L(x) at an interior cell of a red-black split level, neighbours addressed
// directly in the two colour halves (same arithmetic as mg_apply).
template <typename T>
__device__ __forceinline__ T mg_apply_rb(const MGOp<T>& L, const T* __restrict__ x, int i,
                                         int j, int k)
{
    const GridDev& g = L.g;
    const int nxh = g.n[0] >> 1;
    const long long half = g.ncell() >> 1;
    const int color = (i + j + k) & 1, q = i & 1;
    const long long r = j + (long long)g.n[1] * k;
    const long long h = (i >> 1) + (long long)nxh * r;
    const T* __restrict__ xs = x + color * half;
    const T* __restrict__ xo = x + (1 - color) * half;
    const T x0 = xs[h];
    const T xm = xo[h - 1 + q], xp = xo[h + q];
    const T ym = xo[h - nxh], yp = xo[h + nxh];
    T bxl, bxh, byl, byh;
    if (L.b[0])
    {
        const long long fx = i + (long long)(g.n[0] + 1) * r;
        bxl = L.b[0][fx];
        bxh = L.b[0][fx + 1];
        const long long fy = i + (long long)g.n[0] * (j + (long long)(g.n[1] + 1) * k);
        byl = L.b[1][fy];
        byh = L.b[1][fy + g.n[0]];
    } else
        bxl = bxh = byl = byh = L.bconst;
    T y = L.aconst * x0;
    y -= L.dh[0] * (bxh * (xp - x0) - bxl * (x0 - xm));
    y -= L.dh[1] * (byh * (yp - x0) - byl * (x0 - ym));
    if (g.dim == 3)
    {
        const long long plane = (long long)nxh * g.n[1];
        const T zm = xo[h - plane], zp = xo[h + plane];
        T bzl, bzh;
        if (L.b[2])
        {
            const long long fz = i + (long long)g.n[0] * r;
            bzl = L.b[2][fz];
            bzh = L.b[2][fz + (long long)g.n[0] * g.n[1]];
        } else
            bzl = bzh = L.bconst;
        y -= L.dh[2] * (bzh * (zp - x0) - bzl * (x0 - zm));
    }
    return y;
}

template <typename T>
__device__ __forceinline__ T mg_apply_any(const MGOp<T>& L, const T* __restrict__ x, int i,
                                          int j, int k, bool inhomog)
{
    if (L.g.rb && !L.a && mg_interior(L.g, i, j, k)) return mg_apply_rb(L, x, i, j, k);
    return mg_apply(L, x, i, j, k, inhomog);
}

// Residual f - L(x) at the 2^dim children of every coarse cell, averaged
// into the coarse right-hand side; the coarse unknown is zeroed.  Grid:
// (coarse-row blocks, coarse ny, coarse nz).
template <typename T>
__global__ void __launch_bounds__(128) k_mg_resid_restrict(MGOp<T> L, const T* __restrict__ x,
                                                           const T* __restrict__ f, GridDev gc,
                                                           T* __restrict__ fc,
                                                           T* __restrict__ xc, int inhomog)
{
    VD_PDL_WAIT();
    if (mg_stopped(L)) return;
    const int I = blockIdx.x * blockDim.x + threadIdx.x;
    if (I >= gc.n[0]) return;
    const int J = blockIdx.y, K = blockIdx.z;
    const int rz = (L.g.dim == 3) ? 2 : 1;
    const T w = (L.g.dim == 3) ? T(0.125) : T(0.25);
    T s = T(0);
    for (int kk = 0; kk < rz; ++kk)
        for (int jj = 0; jj < 2; ++jj)
            for (int ii = 0; ii < 2; ++ii)
            {
                const int i = 2 * I + ii, j = 2 * J + jj, k = rz * K + kk;
                s += f[L.g.idx(i, j, k)] - mg_apply_any(L, x, i, j, k, inhomog != 0);
            }
    const long long pc = gc.idx(I, J, K);
    fc[pc] = s * w;
    if (xc) xc[pc] = T(0);
}

// Max-norm of f - L(x) into mx[0] (and of f into mx[1] when `fnorm`); the
// residual itself into rout when given.  Grid: (row blocks, ny/rows, nz),
// each thread walking `rows` rows.
// With `part` given, each block stores its maxima in part[b] (and
// part[nblocks + b] for |f|) for k_mg_max_partials instead of using atomics.
template <typename T>
__global__ void __launch_bounds__(128) k_mg_resid_norm(MGOp<T> L, const T* __restrict__ x,
                                                       const T* __restrict__ f,
                                                       T* __restrict__ rout,
                                                       unsigned long long* mx, int inhomog,
                                                       int fnorm, int rows,
                                                       double* part = nullptr)
{
    VD_PDL_WAIT();
    if (mg_stopped(L)) return;
    __shared__ double sh[32];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int k = blockIdx.z;
    double m = 0.0, mf = 0.0;
    if (i < L.g.n[0])
#pragma unroll 4
        for (int jj = 0; jj < rows; ++jj)
        {
            const int j = blockIdx.y * rows + jj;
            if (j >= L.g.n[1]) break;
            const long long p = L.g.idx(i, j, k);
            const T rr = f[p] - mg_apply_any(L, x, i, j, k, inhomog != 0);
            if (rout) rout[p] = rr;
            const double a = fabs((double)rr);
            m = nanmax(m, a);
            if (fnorm)
            {
                const double af = fabs((double)f[p]);
                mf = nanmax(mf, af);
            }
        }
    m = block_max(m, sh);
    if (fnorm) mf = block_max(mf, sh);
    if (threadIdx.x == 0)
    {
        if (part)
        {
            const long long nb = (long long)gridDim.x * gridDim.y * gridDim.z;
            const long long b = blockIdx.x + (long long)gridDim.x * (blockIdx.y + (long long)gridDim.y * blockIdx.z);
            part[b] = m;
            if (fnorm) part[nb + b] = mf;
        } else
        {
            atomic_max_nonneg(mx, m);
            if (fnorm) atomic_max_nonneg(mx + 1, mf);
        }
    }
}

// Residual max-norm on a red-black split level: one thread per half-row
// position h = (i/2, j, k), i.e. per pair of cells 2(i/2) and 2(i/2)+1 (one
// of each colour, both at offset h of their colour half), grid-stride over
// the pairs.  Per-block maxima go to part[b] (and part[gridDim.x + b] for
// |f|) for k_mg_max_partials; the residual itself to rout when given.
template <typename T>
__global__ void __launch_bounds__(256) k_mg_resid_norm_rb(MGOp<T> L, const T* __restrict__ x,
                                                          const T* __restrict__ f,
                                                          T* __restrict__ rout, int inhomog,
                                                          int fnorm, double* __restrict__ part)
{
    VD_PDL_WAIT();
    if (mg_stopped(L)) return;
    __shared__ double sh[32];
    const GridDev& g = L.g;
    const int nxh = g.n[0] >> 1, ny = g.n[1];
    const long long half = g.ncell() >> 1;
    double m = 0.0, mf = 0.0;
    for (long long h = blockIdx.x * (long long)blockDim.x + threadIdx.x; h < half;
         h += (long long)gridDim.x * blockDim.x)
    {
        const int ih = (int)(h % nxh);
        const long long r = h / nxh;
        const int j = (int)(r % ny), k = (int)(r / ny);
#pragma unroll
        for (int s = 0; s < 2; ++s)
        {
            const int i = 2 * ih + s;
            const long long p = (long long)((i + j + k) & 1) * half + h;
            const T rr = f[p] - mg_apply_any(L, x, i, j, k, inhomog != 0);
            if (rout) rout[p] = rr;
            const double a = fabs((double)rr);
            m = nanmax(m, a);
            if (fnorm)
            {
                const double af = fabs((double)f[p]);
                mf = nanmax(mf, af);
            }
        }
    }
    m = block_max(m, sh);
    if (fnorm) mf = block_max(mf, sh);
    if (threadIdx.x == 0)
    {
        part[blockIdx.x] = m;
        if (fnorm) part[gridDim.x + blockIdx.x] = mf;
    }
}

// Second stage of the residual max-norm: one block reduces the per-block
// partial maxima and stores the bit patterns in mx[0] (and mx[1]).
template <typename T>
__global__ void __launch_bounds__(1024) k_mg_max_partials(MGOp<T> L, const double* part,
                                                          long long nb, int fnorm,
                                                          unsigned long long* mx)
{
    VD_PDL_WAIT();
    if (mg_stopped(L)) return;
    __shared__ double sh[32];
    double m = 0.0, mf = 0.0;
    for (long long b = threadIdx.x; b < nb; b += blockDim.x)
    {
        m = nanmax(m, part[b]);
        if (fnorm) mf = nanmax(mf, part[nb + b]);
    }
    m = block_max(m, sh);
    if (fnorm) mf = block_max(mf, sh);
    if (threadIdx.x == 0)
    {
        mx[0] = (unsigned long long)__double_as_longlong(m);
        if (fnorm) mx[1] = (unsigned long long)__double_as_longlong(mf);
    }
}

template <typename T>
__global__ void __launch_bounds__(128) k_mg_prolong_add(GridDev gf, GridDev gc,
                                                        T* __restrict__ xf,
                                                        const T* __restrict__ xc,
                                                        const int* stop)
{
    VD_PDL_WAIT();
    if (stop && *(volatile const int*)stop) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= gf.n[0]) return;
    const int j = blockIdx.y, k = blockIdx.z;
    const int rz = (gf.dim == 3) ? 2 : 1;
    xf[gf.idx(i, j, k)] += xc[gc.idx(i >> 1, j >> 1, k / rz)];
}

// BiCGStab on the coarsest level in one CTA (homogeneous boundaries),
// relative tolerance `rel` on the max-norm, `maxiter` iterations, then `nub`
// Gauss-Seidel smooths (or `nuf` when BiCGStab did not converge).  Every
// vector is addressed through the level's layout (L.g.idx), like x and b.
template <typename T>
__device__ void mg_bottom_block(const MGOp<T>& L, T* __restrict__ x, const T* __restrict__ b,
                                T* __restrict__ scr, T rel, int maxiter, int nub, int nuf,
                                int* status, T* sh)
{
    const long long n = L.g.ncell();
    T* r = scr;
    T* rh = scr + n;
    T* p = scr + 2 * n;
    T* v = scr + 3 * n;
    T* s = scr + 4 * n;
    T* tt = scr + 5 * n;
    const int tid = threadIdx.x, bs = blockDim.x;
    const int nx = L.g.n[0], ny = L.g.n[1];
    T m = T(0);
    for (long long q = tid; q < n; q += bs)
    {
        x[q] = T(0);
        r[q] = b[q];
        rh[q] = b[q];
        p[q] = T(0);
        v[q] = T(0);
        const T a = r[q] < T(0) ? -r[q] : r[q];
        m = nanmax(m, a);
    }
    const T rnorm0 = block_max(m, sh);
    int ret = 0;
    if (rnorm0 > T(0))
    {
        ret = 8;
        T rho_1 = T(1), alpha = T(1), omega = T(1);
        for (int iter = 1; iter <= maxiter; ++iter)
        {
            T acc = T(0);
            for (long long q = tid; q < n; q += bs) acc += rh[q] * r[q];
            const T rho = block_sum(acc, sh);
            if (rho == T(0))
            {
                ret = 1;
                break;
            }
            if (iter == 1)
            {
                for (long long q = tid; q < n; q += bs) p[q] = r[q];
            } else
            {
                const T beta = (rho / rho_1) * (alpha / omega);
                for (long long q = tid; q < n; q += bs)
                    p[q] = r[q] + beta * (p[q] - omega * v[q]);
            }
            __syncthreads();
            acc = T(0);
            for (long long c = tid; c < n; c += bs)
            {
                const int i = (int)(c % nx), j = (int)((c / nx) % ny), k = (int)(c / ((long long)nx * ny));
                const long long q = L.g.idx(i, j, k);
                v[q] = mg_apply(L, p, i, j, k, false);
                acc += rh[q] * v[q];
            }
            const T rhTv = block_sum(acc, sh);
            if (rhTv == T(0))
            {
                ret = 2;
                break;
            }
            alpha = rho / rhTv;
            m = T(0);
            for (long long q = tid; q < n; q += bs)
            {
                x[q] += alpha * p[q];
                s[q] = r[q] - alpha * v[q];
                const T a = s[q] < T(0) ? -s[q] : s[q];
                m = nanmax(m, a);
            }
            if (block_max(m, sh) <= rel * rnorm0)
            {
                ret = 0;
                break;
            }
            T a1 = T(0), a2 = T(0);
            for (long long c = tid; c < n; c += bs)
            {
                const int i = (int)(c % nx), j = (int)((c / nx) % ny), k = (int)(c / ((long long)nx * ny));
                const long long q = L.g.idx(i, j, k);
                tt[q] = mg_apply(L, s, i, j, k, false);
                a1 += tt[q] * tt[q];
                a2 += tt[q] * s[q];
            }
            const T ttt = block_sum(a1, sh);
            const T tts = block_sum(a2, sh);
            if (ttt == T(0))
            {
                ret = 3;
                break;
            }
            omega = tts / ttt;
            m = T(0);
            for (long long q = tid; q < n; q += bs)
            {
                x[q] += omega * s[q];
                r[q] = s[q] - omega * tt[q];
                const T a = r[q] < T(0) ? -r[q] : r[q];
                m = nanmax(m, a);
            }
            if (block_max(m, sh) <= rel * rnorm0)
            {
                ret = 0;
                break;
            }
            if (omega == T(0))
            {
                ret = 4;
                break;
            }
            rho_1 = rho;
        }
    }
    __syncthreads();
    const int nsm = (ret == 0) ? nub : nuf;
    for (int sm = 0; sm < nsm; ++sm)
        for (int color = 0; color < 2; ++color)
        {
            for (long long c = tid; c < n; c += bs)
            {
                const int i = (int)(c % nx), j = (int)((c / nx) % ny), k = (int)(c / ((long long)nx * ny));
                if (((i + j + k + color) & 1) == 0) mg_gs_cell(L, x, b, i, j, k, false);
            }
            __syncthreads();
        }
    if (tid == 0 && status) *status = ret;
    __syncthreads();
}

template <typename T>
__global__ void k_mg_bottom(MGOp<T> L, T* __restrict__ x, const T* __restrict__ b,
                            T* __restrict__ scr, T rel, int maxiter, int nub, int nuf,
                            int* status)
{
    VD_PDL_WAIT();
    if (mg_stopped(L)) return;
    __shared__ T sh[32];
    mg_bottom_block(L, x, b, scr, rel, maxiter, nub, nuf, status, sh);
}

// The coarse end of a V-cycle in one CTA: levels lc .. nl-1 (each at most a
// few thousand cells) are smoothed, restricted, bottom-solved, prolongated
// and smoothed again with block barriers between the sweeps, replacing
// about ten kernel launches per level.  Level lc's right-hand side is
// already restricted and its unknown zeroed.
#define VD_MG_MAXLEV 16
#define VD_MG_COARSE_SMEM (200 * 1024)
template <typename T>
struct MGCoarse
{
    int lc, nl;
    MGOp<T> op[VD_MG_MAXLEV];
    T* x[VD_MG_MAXLEV];
    T* f[VD_MG_MAXLEV];
};

template <typename T>
__device__ void mg_block_smooth(const MGOp<T>& L, T* __restrict__ x, const T* __restrict__ f,
                                int nsm)
{
    const int nx = L.g.n[0], ny = L.g.n[1], nz = L.g.n[2];
    const int nxh = (nx + 1) >> 1;
    const int tot = nxh * ny * nz;
    for (int sm = 0; sm < nsm; ++sm)
        for (int color = 0; color < 2; ++color)
        {
            for (int t = threadIdx.x; t < tot; t += blockDim.x)
            {
                const int ih = t % nxh, r = t / nxh;
                const int j = r % ny, k = r / ny;
                const int i = 2 * ih + ((j + k + color) & 1);
                if (i < nx) mg_gs_cell(L, x, f, i, j, k, false);
            }
            __syncthreads();
        }
}

// Bytes of shared memory the coarse cycle needs to keep the unknowns and
// right-hand sides of levels lc .. nl-1 and the bottom solver's six work
// vectors on chip.
template <typename T>
size_t mg_coarse_smem(const MGCoarse<T>& C)
{
    size_t n = 0;
    for (int l = C.lc; l < C.nl; ++l) n += 2 * (size_t)C.op[l].g.ncell();
    n += 6 * (size_t)C.op[C.nl - 1].g.ncell();
    return n * sizeof(T);
}

// With `on_chip`, every level's x and f live in dynamic shared memory (the
// layout of mg_coarse_smem): level lc's right-hand side is read once from
// global memory and its unknown written back once at the end.
template <typename T>
__global__ void __launch_bounds__(512) k_mg_coarse_vcycle(MGCoarse<T> C, T* __restrict__ scr,
                                                          T rel, int maxiter, int nu1, int nu2,
                                                          int nub, int nuf, int on_chip)
{
    VD_PDL_WAIT();
    extern __shared__ __align__(16) unsigned char mg_smem[];
    if (mg_stopped(C.op[C.lc])) return;
    __shared__ T sh[32];
    const int last = C.nl - 1;
    T* X[VD_MG_MAXLEV];
    T* F[VD_MG_MAXLEV];
    T* bscr = scr;
    if (on_chip)
    {
        T* p = reinterpret_cast<T*>(mg_smem);
        for (int l = C.lc; l <= last; ++l)
        {
            const long long n = C.op[l].g.ncell();
            X[l] = p;
            F[l] = p + n;
            p += 2 * n;
        }
        bscr = p;
        const long long n0 = C.op[C.lc].g.ncell();
        for (long long q = threadIdx.x; q < n0; q += blockDim.x)
        {
            F[C.lc][q] = C.f[C.lc][q];
            X[C.lc][q] = T(0);
        }
        __syncthreads();
    } else
        for (int l = C.lc; l <= last; ++l)
        {
            X[l] = C.x[l];
            F[l] = C.f[l];
        }
    for (int l = C.lc; l < last; ++l)
    {
        const MGOp<T>& L = C.op[l];
        mg_block_smooth(L, X[l], F[l], nu1);
        const GridDev& gc = C.op[l + 1].g;
        const int rz = (L.g.dim == 3) ? 2 : 1;
        const T w = (L.g.dim == 3) ? T(0.125) : T(0.25);
        for (long long c = threadIdx.x; c < gc.ncell(); c += blockDim.x)
        {
            const int I = (int)(c % gc.n[0]), J = (int)((c / gc.n[0]) % gc.n[1]),
                      K = (int)(c / ((long long)gc.n[0] * gc.n[1]));
            T s = T(0);
            for (int kk = 0; kk < rz; ++kk)
                for (int jj = 0; jj < 2; ++jj)
                    for (int ii = 0; ii < 2; ++ii)
                    {
                        const int i = 2 * I + ii, j = 2 * J + jj, k = rz * K + kk;
                        s += F[l][L.g.idx(i, j, k)] - mg_apply(L, X[l], i, j, k, false);
                    }
            const long long pc = gc.idx(I, J, K);
            F[l + 1][pc] = s * w;
            X[l + 1][pc] = T(0);
        }
        __syncthreads();
    }
    mg_bottom_block(C.op[last], X[last], F[last], bscr, rel, maxiter, nub, nuf, (int*)nullptr,
                    sh);
    for (int l = last - 1; l >= C.lc; --l)
    {
        const MGOp<T>& L = C.op[l];
        const GridDev& gc = C.op[l + 1].g;
        const int rz = (L.g.dim == 3) ? 2 : 1;
        for (long long c = threadIdx.x; c < L.g.ncell(); c += blockDim.x)
        {
            const int i = (int)(c % L.g.n[0]), j = (int)((c / L.g.n[0]) % L.g.n[1]),
                      k = (int)(c / ((long long)L.g.n[0] * L.g.n[1]));
            X[l][L.g.idx(i, j, k)] += X[l + 1][gc.idx(i >> 1, j >> 1, k / rz)];
        }
        __syncthreads();
        mg_block_smooth(L, X[l], F[l], nu2);
    }
    if (on_chip)
    {
        const long long n0 = C.op[C.lc].g.ncell();
        for (long long q = threadIdx.x; q < n0; q += blockDim.x) C.x[C.lc][q] = X[C.lc][q];
    }
}

// ---------------------------------------------------------------------
// The coarse end of a V-cycle on 3-D levels without periodic directions,
// one 1024-thread CTA, every level on chip in natural layout.  Per cell
// the operator is kept in the form the Gauss-Seidel update and the
// residual both use:
//     L x = G x0 - sum_n w_n x_n,   G = gamma - delta
// where an outside neighbour n (homogeneous ghost c0 x0 + c1 x1) moves its
// c0 share into G (delta) and its c1 share onto the opposite neighbour's
// weight (the same operator as mg_apply / mg_gs_cell, rearranged).  G and
// 1/G are formed once per launch; cell coordinates are decoded once.

#define MGC_THREADS 1024

template <typename T>
struct MGCLevel
{
    T* x;
    T* f;
    T* G;
    T* iG;
    int* crd; // i | j << 10 | k << 20; colour-0 cells first when nx is even
};

// Per-side weights of cell (i,j,k): w[s2] for the neighbour on side s2
// (x-lo, x-hi, y-lo, y-hi, z-lo, z-hi), the index offsets o[s2] (an outside
// neighbour points at the opposite one, weight 0) and G.
template <typename T, bool VARB>
__device__ __forceinline__ void mgc_weights(const MGOp<T>& L, int i, int j, int k, T* w,
                                            int* o, T& G)
{
    const int nx = L.g.n[0], ny = L.g.n[1], nz = L.g.n[2];
    T b[6];
    mg3_faces<T, VARB>(L, i, j, k, b);
    const int st[3] = {1, nx, nx * ny};
    const int c[3] = {i, j, k}, n[3] = {nx, ny, nz};
    G = L.aconst;
#pragma unroll
    for (int d = 0; d < 3; ++d)
    {
        const T dh = L.dh[d];
        G += dh * (b[2 * d] + b[2 * d + 1]);
        w[2 * d] = dh * b[2 * d];
        w[2 * d + 1] = dh * b[2 * d + 1];
        o[2 * d] = -st[d];
        o[2 * d + 1] = st[d];
    }
#pragma unroll
    for (int d = 0; d < 3; ++d)
#pragma unroll
        for (int hi = 0; hi < 2; ++hi)
        {
            const bool outside = hi ? (c[d] == n[d] - 1) : (c[d] == 0);
            if (!outside) continue;
            const int s2 = 2 * d + hi, s = d + 3 * hi;
            const int p = (d == 0) ? (j + ny * k) : ((d == 1) ? (i + nx * k) : (i + nx * j));
            const T c0 = L.c0[s] ? L.c0[s][p] : L.c0s[s];
            const T c1 = L.c1s[s];
            G -= w[s2] * c0;
            w[s2 ^ 1] += w[s2] * c1;
            w[s2] = T(0);
            o[s2] = o[s2 ^ 1];
        }
}

// sum_n w_n x_n of cell c with the weights of mgc_weights, formed with
// selects instead of branches (every warp of a coarse level holds row-end
// cells, so a branch per side would diverge in all of them): an outside
// side's weight is 0 and its index the opposite neighbour's, and the
// opposite weight gains w c1.  Same terms in the same order as mgc_weights
// gives them.
template <typename T, bool VARB>
__device__ __forceinline__ T mgc_sum(const MGOp<T>& L, const T* __restrict__ x, int c, int i,
                                     int j, int k)
{
    const int nx = L.g.n[0], ny = L.g.n[1], nz = L.g.n[2];
    T b[6];
    mg3_faces<T, VARB>(L, i, j, k, b);
    const int st[3] = {1, nx, nx * ny};
    const int cd[3] = {i, j, k}, n[3] = {nx, ny, nz};
    T s = T(0);
#pragma unroll
    for (int d = 0; d < 3; ++d)
    {
        const T dh = L.dh[d];
        const bool lo = cd[d] == 0, hi = cd[d] == n[d] - 1;
        const T wl = dh * b[2 * d], wh = dh * b[2 * d + 1];
        const T wl2 = lo ? T(0) : (hi ? wl + wh * L.c1s[d + 3] : wl);
        const T wh2 = hi ? T(0) : (lo ? wh + wl * L.c1s[d] : wh);
        const int ol = lo ? st[d] : -st[d], oh = hi ? -st[d] : st[d];
        s += wl2 * x[c + ol];
        s += wh2 * x[c + oh];
    }
    return s;
}

// nsm Gauss-Seidel iterations on a level held on chip.  With nx even the
// coordinate list holds each colour's cells contiguously, so a colour sweep
// visits only its own cells (no lane idles on the other colour).
template <typename T, bool VARB>
__device__ void mgc_smooth(const MGOp<T>& L, const MGCLevel<T> V, int nsm)
{
    const int nx = L.g.n[0], ny = L.g.n[1];
    const int n = (int)L.g.ncell();
    const bool sorted = (nx & 1) == 0;
    const int cnt = sorted ? n >> 1 : n;
    for (int sm = 0; sm < nsm; ++sm)
        for (int color = 0; color < 2; ++color)
        {
            const int* crd = V.crd + (sorted ? color * cnt : 0);
            for (int m = threadIdx.x; m < cnt; m += MGC_THREADS)
            {
                const int cr = crd[m];
                const int i = cr & 1023, j = (cr >> 10) & 1023, k = (cr >> 20) & 1023;
                if (!sorted && ((i + j + k) & 1) != color) continue;
                const int c = i + nx * (j + ny * k);
                V.x[c] = (V.f[c] + mgc_sum<T, VARB>(L, V.x, c, i, j, k)) *
                         V.iG[c];
            }
            __syncthreads();
        }
}

// mg_bottom_block (BiCGStab, then nub or nuf Gauss-Seidel iterations) for
// a bottom level of at most 32 cells, on warp 0 alone: one cell per lane,
// reductions by warp shuffles, no block barriers (the other warps wait at
// the caller's barrier).  The operator is the G x0 - sum w x form; p and s
// go through shared memory (scr) because the operator reads neighbours.
template <typename T, bool VARB>
__device__ void mgc_bottom_warp(const MGOp<T>& L, const MGCLevel<T> V, T* __restrict__ scr,
                                T rel, int maxiter, int nub, int nuf)
{
    const unsigned FULL = 0xffffffffu;
    const int n = (int)L.g.ncell();
    const int lane = threadIdx.x & 31;
    const bool act = lane < n;
    const int nx = L.g.n[0], ny = L.g.n[1];
    const int c = act ? lane : 0;
    const int i = c % nx, rr = c / nx, j = rr % ny, k = rr / ny;
    T w[6], G;
    int o[6];
    mgc_weights<T, VARB>(L, i, j, k, w, o, G);
    T* p = scr;
    T* sv = scr + n;
    auto wsum = [&](T v) {
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(FULL, v, off);
        return v;
    };
    auto wmax = [&](T v) {
#pragma unroll
        for (int off = 16; off > 0; off >>= 1)
        {
            const T u = __shfl_xor_sync(FULL, v, off);
            v = u > v ? u : v;
        }
        return v;
    };
    auto apply = [&](const T* u) {
        T s = T(0);
#pragma unroll
        for (int m = 0; m < 6; ++m) s += w[m] * u[c + o[m]];
        return G * u[c] - s;
    };
    auto absv = [](T a) { return a < T(0) ? -a : a; };
    T xv = T(0), rv = act ? V.f[c] : T(0);
    const T rh = rv;
    T pv = T(0), vv = T(0);
    const T rnorm0 = wmax(absv(rv));
    int ret = 0;
    if (rnorm0 > T(0))
    {
        ret = 8;
        T rho_1 = T(1), alpha = T(1), omega = T(1);
        for (int iter = 1; iter <= maxiter; ++iter)
        {
            const T rho = wsum(rh * rv);
            if (rho == T(0))
            {
                ret = 1;
                break;
            }
            if (iter == 1)
                pv = rv;
            else
            {
                const T beta = (rho / rho_1) * (alpha / omega);
                pv = rv + beta * (pv - omega * vv);
            }
            if (act) p[c] = pv;
            __syncwarp();
            vv = act ? apply(p) : T(0);
            __syncwarp();
            const T rhTv = wsum(rh * vv);
            if (rhTv == T(0))
            {
                ret = 2;
                break;
            }
            alpha = rho / rhTv;
            xv += alpha * pv;
            const T sval = rv - alpha * vv;
            if (wmax(absv(sval)) <= rel * rnorm0)
            {
                ret = 0;
                break;
            }
            if (act) sv[c] = sval;
            __syncwarp();
            const T tv = act ? apply(sv) : T(0);
            __syncwarp();
            const T ttt = wsum(tv * tv);
            const T tts = wsum(tv * sval);
            if (ttt == T(0))
            {
                ret = 3;
                break;
            }
            omega = tts / ttt;
            xv += omega * sval;
            rv = sval - omega * tv;
            if (wmax(absv(rv)) <= rel * rnorm0)
            {
                ret = 0;
                break;
            }
            if (omega == T(0))
            {
                ret = 4;
                break;
            }
            rho_1 = rho;
        }
    }
    if (act) V.x[c] = xv;
    __syncwarp();
    const int nsm = (ret == 0) ? nub : nuf;
    for (int sm = 0; sm < nsm; ++sm)
        for (int color = 0; color < 2; ++color)
        {
            if (act && ((i + j + k + color) & 1) == 0)
            {
                T s = T(0);
#pragma unroll
                for (int m = 0; m < 6; ++m) s += w[m] * V.x[c + o[m]];
                V.x[c] = (V.f[c] + s) * V.iG[c];
            }
            __syncwarp();
        }
}

// Joint bottom solve of a multicomponent system (MLMG with ncomp > 1):
// each CTA of a thread-block cluster holds one component's bottom level
// (at most 32 cells, in warp 0), and every inner product and max-norm of
// BiCGStab is reduced over the whole cluster through distributed shared
// memory, so the Krylov scalars rho, alpha, omega are those of the joint
// system (MLCGSolver's dot products run over all components).  Every CTA
// forms the same sums (partials added in rank order), so all take the same
// branches and the same number of cluster barriers.  Partials go to one of
// two slots per CTA by the parity of the reduction's sequence number: a
// slot is rewritten two reductions later, after a barrier that every
// reader of its previous value has passed.  All threads of the CTA call
// this; threads past warp 0 hold no cells.
template <typename T, bool VARB>
__device__ void mgc_bottom_joint(const MGOp<T>& L, const MGCLevel<T> V, T* __restrict__ scr,
                                 T rel, int maxiter, int nub, int nuf)
{
    namespace cg = cooperative_groups;
    cg::cluster_group cl = cg::this_cluster();
    const unsigned nblk = cl.num_blocks();
    __shared__ T red[2];
    const unsigned FULL = 0xffffffffu;
    const int n = (int)L.g.ncell();
    const bool w0 = threadIdx.x < 32;
    const int lane = threadIdx.x & 31;
    const bool act = w0 && lane < n;
    const int nx = L.g.n[0], ny = L.g.n[1];
    const int c = act ? lane : 0;
    const int i = c % nx, rr = c / nx, j = rr % ny, k = rr / ny;
    T w[6], G;
    int o[6];
    mgc_weights<T, VARB>(L, i, j, k, w, o, G);
    T* p = scr;
    T* sv = scr + n;
    int seq = 0;
    auto jred = [&](T v, bool mx) -> T {
        if (w0)
        {
#pragma unroll
            for (int off = 16; off > 0; off >>= 1)
            {
                const T u = __shfl_xor_sync(FULL, v, off);
                v = mx ? (u > v ? u : v) : v + u;
            }
            if (lane == 0) red[seq & 1] = v;
        }
        cl.sync();
        T acc = T(0);
        for (unsigned r = 0; r < nblk; ++r)
        {
            const T x = cl.map_shared_rank(red, r)[seq & 1];
            acc = mx ? (x > acc ? x : acc) : acc + x;
        }
        ++seq;
        return acc;
    };
    auto apply = [&](const T* u) {
        T s = T(0);
#pragma unroll
        for (int m = 0; m < 6; ++m) s += w[m] * u[c + o[m]];
        return G * u[c] - s;
    };
    auto absv = [](T a) { return a < T(0) ? -a : a; };
    T xv = T(0), rv = act ? V.f[c] : T(0);
    const T rh = rv;
    T pv = T(0), vv = T(0);
    const T rnorm0 = jred(absv(rv), true);
    int ret = 0;
    if (rnorm0 > T(0))
    {
        ret = 8;
        T rho_1 = T(1), alpha = T(1), omega = T(1);
        for (int iter = 1; iter <= maxiter; ++iter)
        {
            const T rho = jred(rh * rv, false);
            if (rho == T(0))
            {
                ret = 1;
                break;
            }
            if (iter == 1)
                pv = rv;
            else
            {
                const T beta = (rho / rho_1) * (alpha / omega);
                pv = rv + beta * (pv - omega * vv);
            }
            if (act) p[c] = pv;
            __syncthreads();
            vv = act ? apply(p) : T(0);
            __syncthreads();
            const T rhTv = jred(rh * vv, false);
            if (rhTv == T(0))
            {
                ret = 2;
                break;
            }
            alpha = rho / rhTv;
            xv += alpha * pv;
            const T sval = rv - alpha * vv;
            if (jred(absv(sval), true) <= rel * rnorm0)
            {
                ret = 0;
                break;
            }
            if (act) sv[c] = sval;
            __syncthreads();
            const T tv = act ? apply(sv) : T(0);
            __syncthreads();
            const T ttt = jred(tv * tv, false);
            const T tts = jred(tv * sval, false);
            if (ttt == T(0))
            {
                ret = 3;
                break;
            }
            omega = tts / ttt;
            xv += omega * sval;
            rv = sval - omega * tv;
            if (jred(absv(rv), true) <= rel * rnorm0)
            {
                ret = 0;
                break;
            }
            if (omega == T(0))
            {
                ret = 4;
                break;
            }
            rho_1 = rho;
        }
    }
    // no CTA leaves while another may still read its partials
    cl.sync();
    if (act) V.x[c] = xv;
    __syncthreads();
    const int nsm = (ret == 0) ? nub : nuf;
    for (int sm = 0; sm < nsm; ++sm)
        for (int color = 0; color < 2; ++color)
        {
            if (act && ((i + j + k + color) & 1) == 0)
            {
                T s = T(0);
#pragma unroll
                for (int m = 0; m < 6; ++m) s += w[m] * V.x[c + o[m]];
                V.x[c] = (V.f[c] + s) * V.iG[c];
            }
            __syncthreads();
        }
}

// The coarse part of a V-cycle (levels lc .. nl-1) in one CTA, every level
// in shared memory; JOINT: one component of a multicomponent system per CTA
// of a cluster, with the bottom solve joint over the cluster.
template <typename T, bool VARB, bool JOINT>
__device__ __forceinline__ void mgc_run(const MGCoarse<T>& C, T rel, int maxiter, int nu1,
                                        int nu2, int nub, int nuf)
{
    extern __shared__ __align__(16) unsigned char mgc_smem[];
    __shared__ T sh[32];
    if (mg_stopped(C.op[C.lc])) return;
    const int lc = C.lc, last = C.nl - 1;
    MGCLevel<T> V[VD_MG_MAXLEV];
    // carve the levels: x, f, G, 1/G (T) then the coordinates (int)
    T* p = reinterpret_cast<T*>(mgc_smem);
    for (int l = lc; l <= last; ++l)
    {
        const int n = (int)C.op[l].g.ncell();
        V[l].x = p;
        V[l].f = p + n;
        V[l].G = p + 2 * n;
        V[l].iG = p + 3 * n;
        p += 4 * n;
    }
    T* bscr = p;
    p += 6 * C.op[last].g.ncell();
    int* ip = reinterpret_cast<int*>(p);
    for (int l = lc; l <= last; ++l)
    {
        V[l].crd = ip;
        ip += C.op[l].g.ncell();
    }
    // coordinates, G and 1/G of every level; level lc's right-hand side
    for (int l = lc; l <= last; ++l)
    {
        const MGOp<T>& L = C.op[l];
        const int nx = L.g.n[0], ny = L.g.n[1], n = (int)L.g.ncell();
        for (int c = threadIdx.x; c < n; c += MGC_THREADS)
        {
            const int i = c % nx, r = c / nx, j = r % ny, k = r / ny;
            // with nx even every row holds nx/2 cells of each colour
            const int m = (nx & 1) ? c
                                   : ((i + j + k) & 1) * (n >> 1) + (j + ny * k) * (nx >> 1) +
                                         (i >> 1);
            V[l].crd[m] = i | (j << 10) | (k << 20);
            T w[6], G;
            int o[6];
            mgc_weights<T, VARB>(L, i, j, k, w, o, G);
            V[l].G[c] = G;
            V[l].iG[c] = T(1) / G;
            if (l == lc)
            {
                V[l].f[c] = C.f[l][L.g.idx(i, j, k)];
                V[l].x[c] = T(0);
            }
        }
    }
    __syncthreads();
    // descend
    for (int l = lc; l < last; ++l)
    {
        const MGOp<T>& L = C.op[l];
        mgc_smooth<T, VARB>(L, V[l], nu1);
        const MGCLevel<T> Vf = V[l], Vc = V[l + 1]; // in registers, not the local array
        const GridDev& gc = C.op[l + 1].g;
        const int nx = L.g.n[0], ny = L.g.n[1];
        const int ncx = gc.n[0], ncy = gc.n[1], nc = (int)gc.ncell();
        // g threads per coarse cell (the most that keep the level to one pass
        // of the block), each summing 8/g children; the g partial sums are
        // g aligned lanes of one warp, added by shuffles
        int g = 8;
        while (g > 1 && nc * g > MGC_THREADS) g >>= 1;
        const int per = 8 / g;
        for (int base = 0; base < g * nc; base += MGC_THREADS)
        {
            const int t = base + threadIdx.x;
            const bool valid = t < g * nc;
            const int cc = valid ? t / g : 0, sub = t & (g - 1);
            const int I = cc % ncx, R = cc / ncx, J = R % ncy, K = R / ncy;
            T r = T(0);
            if (valid)
                for (int q = 0; q < per; ++q)
                {
                    const int ch = sub * per + q;
                    const int i = 2 * I + (ch & 1), j = 2 * J + ((ch >> 1) & 1),
                              k = 2 * K + (ch >> 2);
                    const int c = i + nx * (j + ny * k);
                    r += Vf.f[c] - (Vf.G[c] * Vf.x[c] - mgc_sum<T, VARB>(L, Vf.x, c, i, j, k));
                }
            for (int off = 1; off < g; off <<= 1) r += __shfl_xor_sync(0xffffffffu, r, off);
            if (valid && sub == 0)
            {
                Vc.f[cc] = r * T(0.125);
                Vc.x[cc] = T(0);
            }
        }
        __syncthreads();
    }
    // bottom: BiCGStab (+ smoothing) in natural layout
    {
        MGOp<T> Lb = C.op[last];
        Lb.g.rb = 0;
        if constexpr (JOINT)
            mgc_bottom_joint<T, VARB>(Lb, V[last], bscr, rel, maxiter, nub, nuf);
        else if (Lb.g.ncell() <= 32)
        {
            if (threadIdx.x < 32) mgc_bottom_warp<T, VARB>(Lb, V[last], bscr, rel, maxiter, nub, nuf);
            __syncthreads();
        } else
            mg_bottom_block(Lb, V[last].x, V[last].f, bscr, rel, maxiter, nub, nuf,
                            (int*)nullptr, sh);
    }
    // ascend
    for (int l = last - 1; l >= lc; --l)
    {
        const MGOp<T>& L = C.op[l];
        const GridDev& gc = C.op[l + 1].g;
        const int n = (int)L.g.ncell();
        const int ncx = gc.n[0], ncy = gc.n[1];
        const int nx = L.g.n[0], ny = L.g.n[1];
        const MGCLevel<T> Vf = V[l], Vc = V[l + 1];
        for (int m = threadIdx.x; m < n; m += MGC_THREADS)
        {
            const int cr = Vf.crd[m];
            const int i = cr & 1023, j = (cr >> 10) & 1023, k = (cr >> 20) & 1023;
            Vf.x[i + nx * (j + ny * k)] += Vc.x[(i >> 1) + ncx * ((j >> 1) + ncy * (k >> 1))];
        }
        __syncthreads();
        mgc_smooth<T, VARB>(L, V[l], nu2);
    }
    {
        const MGOp<T>& L = C.op[lc];
        const int n = (int)L.g.ncell();
        const int nx = L.g.n[0], ny = L.g.n[1];
        for (int m = threadIdx.x; m < n; m += MGC_THREADS)
        {
            const int cr = V[lc].crd[m];
            const int i = cr & 1023, j = (cr >> 10) & 1023, k = (cr >> 20) & 1023;
            C.x[lc][L.g.idx(i, j, k)] = V[lc].x[i + nx * (j + ny * k)];
        }
    }
}

template <typename T, bool VARB>
__global__ void __launch_bounds__(MGC_THREADS) k_mg_coarse3(MGCoarse<T> C, T rel, int maxiter,
                                                            int nu1, int nu2, int nub, int nuf)
{
    VD_PDL_WAIT();
    mgc_run<T, VARB, false>(C, rel, maxiter, nu1, nu2, nub, nuf);
}

// Multicomponent form: CTA b of a cluster of nc CTAs runs component b's
// coarse cycle from Cs[b]; the bottom solve is joint over the cluster (the
// host checks that the bottom level holds at most 32 cells).
template <typename T, bool VARB>
__global__ void __launch_bounds__(MGC_THREADS) k_mg_coarse3_joint(const MGCoarse<T>* __restrict__ Cs,
                                                                  T rel, int maxiter, int nu1,
                                                                  int nu2, int nub, int nuf)
{
    VD_PDL_WAIT();
    mgc_run<T, VARB, true>(Cs[blockIdx.x], rel, maxiter, nu1, nu2, nub, nuf);
}

// Shared memory of k_mg_coarse3 for levels lc .. nl-1.
template <typename T>
size_t mg_coarse3_smem(const MGCoarse<T>& C)
{
    size_t nt = 0, nc = 0;
    for (int l = C.lc; l < C.nl; ++l)
    {
        nt += 4 * (size_t)C.op[l].g.ncell();
        nc += (size_t)C.op[l].g.ncell();
    }
    nt += 6 * (size_t)C.op[C.nl - 1].g.ncell();
    return nt * sizeof(T) + nc * sizeof(int);
}

// Mean of the coincident fine faces onto a coarse face.
template <typename T>
__global__ void k_mg_avg_faces(GridDev gf, GridDev gc, int d, const T* __restrict__ bf,
                               T* __restrict__ bc)
{
    VD_PDL_WAIT();
    const long long tot = face_count(gc, d);
    const int rz = (gf.dim == 3) ? 2 : 1;
    const int nx = gc.n[0] + (d == 0), ny = gc.n[1] + (d == 1);
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < tot;
         t += (long long)gridDim.x * blockDim.x)
    {
        const int i = (int)(t % nx);
        const long long r = t / nx;
        const int j = (int)(r % ny);
        const int k = (int)(r / ny);
        T s = T(0);
        int cnt = 0;
        for (int kk = 0; kk < (d == 2 ? 1 : rz); ++kk)
            for (int jj = 0; jj < (d == 1 ? 1 : 2); ++jj)
                for (int ii = 0; ii < (d == 0 ? 1 : 2); ++ii)
                {
                    const int fi = (d == 0) ? 2 * i : 2 * i + ii;
                    const int fj = (d == 1) ? 2 * j : 2 * j + jj;
                    const int fk = (d == 2) ? 2 * k : rz * k + kk;
                    s += bf[face_index(gf, d, fi, fj, fk)];
                    ++cnt;
                }
        bc[t] = s / T(cnt);
    }
}

// Robin coefficients on a coarse boundary side.  A face a*phi + b*dphi/dn = f
// closed by the two-point ghost over a cell of width h passes the
// homogeneous flux -kappa*phi_inside, kappa = a / (a h/2 + b) (2/h for
// Dirichlet, 0 for Neumann).  The coarse face keeps the mean conductance of
// its 2^(dim-1) fine faces (width dxf), capped at its own Dirichlet value
// 2/dxc, as the Dirichlet weight w = min(1, mean(kappa) dxc/2) stored as
// (a, b) = (w, (1 - w) dxc/2): uniform Dirichlet and Neumann sides coarsen
// to themselves exactly, a uniform weak Robin side keeps its conductance,
// and Dirichlet patches in a Neumann wall keep their share of the flux
// (averaging a and b apart turns such a wall nearly Neumann on the coarse
// levels and the V-cycle diverges); then c0 = (b/dx - a/2) / (a/2 + b/dx).
template <typename T>
__device__ __forceinline__ T robin_conductance(T a, T b, T h)
{
    const T den = T(0.5) * a * h + b;
    return den != T(0) ? a / den : T(0);
}

template <typename T>
__global__ void k_mg_robin_coarsen(GridDev gf, GridDev gc, int s, const T* ra_f,
                                   const T* rb_f, T* ra_c, T* rb_c, T* c0_c, T dxf, T dxc)
{
    VD_PDL_WAIT();
    const int d = s % 3;
    const int ta = (d == 0) ? 1 : 0, tb = (d == 2) ? 1 : 2;
    const int na = gc.n[ta], nb = gc.n[tb];
    const bool tb_active = tb < gf.dim;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < na * nb;
         q += gridDim.x * blockDim.x)
    {
        const int ia = q % na, ib = q / na;
        T sk = T(0);
        int cnt = 0;
        for (int u = 0; u < 2; ++u)
            for (int w = 0; w < (tb_active ? 2 : 1); ++w)
            {
                const int fa = 2 * ia + u;
                const int fb = tb_active ? 2 * ib + w : ib;
                const int fp = fa + gf.n[ta] * fb;
                sk += robin_conductance(ra_f[fp], rb_f[fp], dxf);
                ++cnt;
            }
        const T kd = (sk / T(cnt)) * (T(0.5) * dxc);
        const T a = kd < T(1) ? kd : T(1), b = (T(1) - a) * (T(0.5) * dxc);
        ra_c[q] = a;
        rb_c[q] = b;
        const T dxi = T(1) / dxc;
        c0_c[q] = (b * dxi - T(0.5) * a) / (T(0.5) * a + b * dxi);
    }
}

template <typename T>
__global__ void k_fill(T* p, T v, long long n)
{
    VD_PDL_WAIT();
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
         t += (long long)gridDim.x * blockDim.x)
        p[t] = v;
}

template <typename TO, typename TI>
__global__ void k_convert(TO* __restrict__ o, const TI* __restrict__ in, TI scale, long long n)
{
    VD_PDL_WAIT();
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
         t += (long long)gridDim.x * blockDim.x)
        o[t] = (TO)(in[t] * scale);
}

} // namespace vd

namespace vd {
// Convergence bookkeeping of an asynchronous solve, on the device.
struct MGDev
{
    unsigned long long rbits;      // max-norm of the latest residual
    unsigned long long fbits;
    unsigned long long final_bits; // residual after the last counted cycle
    int done;
    int iters;
    int refs;       // refinement passes of the FP32-refined form
    double sc_cur;  // scale of the FP32 right-hand side being solved for
    double sc_next; // 1 / max-norm of the latest residual
    int wait_err;   // a TMA-staged sweep gave up waiting for its copies
};

// After each V-cycle: count it and raise the stop flag once the residual
// meets the target (nothing happens once the flag is up).
__global__ void k_mg_check(MGDev* s, double target)
{
    VD_PDL_WAIT();
    if (s->done) return;
    s->iters += 1;
    s->final_bits = s->rbits;
    if (__longlong_as_double((long long)s->rbits) <= target) s->done = 1;
}

// FP32-refined form, on the device: after the FP64 residual of the current
// solution, stop once it meets the target, else keep its 1/max-norm as the
// next right-hand side scale.
__global__ void k_ref_check(MGDev* s, double target)
{
    VD_PDL_WAIT();
    if (s->done) return;
    s->final_bits = s->rbits;
    const double r = __longlong_as_double((long long)s->rbits);
    if (r <= target)
        s->done = 1;
    else
        s->sc_next = 1.0 / r;
}

// x += e / sc_cur (the correction of the scaled FP32 equation).
__global__ void k_ref_add(double* __restrict__ x, const float* __restrict__ e, const MGDev* s,
                          long long n)
{
    VD_PDL_WAIT();
    if (*(volatile const int*)&s->done) return;
    const double inv = 1.0 / s->sc_cur;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
         t += (long long)gridDim.x * blockDim.x)
        x[t] += (double)e[t] * inv;
}

// One refinement pass completed: count it and move to the next scale.
__global__ void k_ref_rotate(MGDev* s, int inner)
{
    VD_PDL_WAIT();
    if (s->done) return;
    s->refs += 1;
    s->iters += inner;
    s->sc_cur = s->sc_next;
}
} // namespace vd
