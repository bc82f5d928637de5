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
};

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

// Value of the neighbour of boundary-adjacent cell (i,j,k) one step along d
// in direction sg; `cf` returns the coefficient of x0 inside a ghost value.
template <typename T>
__device__ __forceinline__ T mg_nbr(const MGOp<T>& L, const T* __restrict__ x, int i,
                                    int j, int k, int d, int sg, bool inhomog, T x0,
                                    T& cf)
{
    int c[3] = {i, j, k};
    c[d] += sg;
    cf = T(0);
    if (c[d] >= 0 && c[d] < L.g.n[d]) return x[L.g.idx(c[0], c[1], c[2])];
    if (L.g.per[d])
    {
        c[d] = (c[d] + L.g.n[d]) % L.g.n[d];
        return x[L.g.idx(c[0], c[1], c[2])];
    }
    const int s = d + (sg > 0 ? 3 : 0);
    const int p = plane_index(L.g, d, i, j, k);
    const T c0 = L.c0[s] ? L.c0[s][p] : L.c0s[s];
    T gh = c0 * x0;
    if (L.c1s[s] != T(0))
    {
        int m[3] = {i, j, k};
        m[d] -= sg;
        gh += L.c1s[s] * x[L.g.idx(m[0], m[1], m[2])];
    }
    if (inhomog && L.gv[s]) gh += L.gv[s][p];
    cf = c0;
    return gh;
}

template <typename T>
__device__ __forceinline__ T mg_apply(const MGOp<T>& L, const T* __restrict__ x, int i,
                                      int j, int k, bool inhomog)
{
    const long long p = L.g.idx(i, j, k);
    const T x0 = x[p];
    T y = (L.a ? L.a[p] : L.aconst) * x0;
    for (int d = 0; d < L.g.dim; ++d)
    {
        int c[3] = {i, j, k};
        const T blo = mg_face_b(L, d, c[0], c[1], c[2]);
        c[d] += 1;
        const T bhi = mg_face_b(L, d, c[0], c[1], c[2]);
        T cf;
        const T xm = mg_nbr(L, x, i, j, k, d, -1, inhomog, x0, cf);
        const T xp = mg_nbr(L, x, i, j, k, d, +1, inhomog, x0, cf);
        y -= L.dh[d] * (bhi * (xp - x0) - blo * (x0 - xm));
    }
    return y;
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
    for (int d = 0; d < L.g.dim; ++d)
    {
        int c[3] = {i, j, k};
        const T blo = mg_face_b(L, d, c[0], c[1], c[2]);
        c[d] += 1;
        const T bhi = mg_face_b(L, d, c[0], c[1], c[2]);
        gamma += L.dh[d] * (blo + bhi);
        T cfm, cfp;
        const T xm = mg_nbr(L, x, i, j, k, d, -1, inhomog, x0, cfm);
        const T xp = mg_nbr(L, x, i, j, k, d, +1, inhomog, x0, cfp);
        rho += L.dh[d] * (blo * xm + bhi * xp);
        delta += L.dh[d] * (blo * cfm + bhi * cfp);
    }
    const T res = f[p] - (gamma * x0 - rho);
    x[p] = x0 + res / (gamma - delta);
}

// ---------------------------------------------------------------- kernels
template <typename T>
__global__ void k_mg_smooth_color(MGOp<T> L, T* __restrict__ x,
                                  const T* __restrict__ f, int color, int inhomog)
{
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

// Residual f - L(x) at the 2^dim children of every coarse cell, averaged
// into the coarse right-hand side; the coarse unknown is zeroed.
template <typename T>
__global__ void k_mg_resid_restrict(MGOp<T> L, const T* __restrict__ x,
                                    const T* __restrict__ f, GridDev gc,
                                    T* __restrict__ fc, T* __restrict__ xc, int inhomog)
{
    const long long tot = gc.ncell();
    const int rz = (L.g.dim == 3) ? 2 : 1;
    const T w = (L.g.dim == 3) ? T(0.125) : T(0.25);
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < tot;
         t += (long long)gridDim.x * blockDim.x)
    {
        const int I = (int)(t % gc.n[0]);
        const long long r = t / gc.n[0];
        const int J = (int)(r % gc.n[1]);
        const int K = (int)(r / gc.n[1]);
        T s = T(0);
        for (int kk = 0; kk < rz; ++kk)
            for (int jj = 0; jj < 2; ++jj)
                for (int ii = 0; ii < 2; ++ii)
                {
                    const int i = 2 * I + ii, j = 2 * J + jj, k = rz * K + kk;
                    s += f[L.g.idx(i, j, k)] - mg_apply(L, x, i, j, k, inhomog != 0);
                }
        fc[t] = s * w;
        if (xc) xc[t] = T(0);
    }
}

// Max-norm of f - L(x) into mx[0] (and of f into mx[1] when `fnorm`).
template <typename T>
__global__ void k_mg_resid_norm(MGOp<T> L, const T* __restrict__ x,
                                const T* __restrict__ f, T* __restrict__ rout,
                                unsigned long long* mx, int inhomog, int fnorm = 0)
{
    __shared__ double sh[32];
    const long long tot = L.g.ncell();
    double m = 0.0, mf = 0.0;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < tot;
         t += (long long)gridDim.x * blockDim.x)
    {
        const int i = (int)(t % L.g.n[0]);
        const long long r = t / L.g.n[0];
        const int j = (int)(r % L.g.n[1]);
        const int k = (int)(r / L.g.n[1]);
        const T rr = f[t] - mg_apply(L, x, i, j, k, inhomog != 0);
        if (rout) rout[t] = rr;
        const double a = fabs((double)rr);
        m = a > m ? a : m;
        if (fnorm)
        {
            const double af = fabs((double)f[t]);
            mf = af > mf ? af : mf;
        }
    }
    m = block_max(m, sh);
    if (threadIdx.x == 0) atomic_max_nonneg(mx, m);
    if (fnorm)
    {
        mf = block_max(mf, sh);
        if (threadIdx.x == 0) atomic_max_nonneg(mx + 1, mf);
    }
}

template <typename T>
__global__ void k_mg_prolong_add(GridDev gf, GridDev gc, T* __restrict__ xf,
                                 const T* __restrict__ xc)
{
    const long long tot = gf.ncell();
    const int rz = (gf.dim == 3) ? 2 : 1;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < tot;
         t += (long long)gridDim.x * blockDim.x)
    {
        const int i = (int)(t % gf.n[0]);
        const long long r = t / gf.n[0];
        const int j = (int)(r % gf.n[1]);
        const int k = (int)(r / gf.n[1]);
        xf[t] += xc[gc.idx(i >> 1, j >> 1, k / rz)];
    }
}

// BiCGStab on the coarsest level in one CTA (homogeneous boundaries),
// relative tolerance `rel` on the max-norm, `maxiter` iterations, then `nub`
// Gauss-Seidel smooths (or `nuf` when BiCGStab did not converge).
template <typename T>
__global__ void k_mg_bottom(MGOp<T> L, T* __restrict__ x, const T* __restrict__ b,
                            T* __restrict__ scr, T rel, int maxiter, int nub, int nuf,
                            int* status)
{
    __shared__ T sh[32];
    const long long n = L.g.ncell();
    T* r = scr;
    T* rh = scr + n;
    T* p = scr + 2 * n;
    T* v = scr + 3 * n;
    T* s = scr + 4 * n;
    T* tt = scr + 5 * n;
    const int tid = threadIdx.x, bs = blockDim.x;
    auto cell = [&](long long q, int& i, int& j, int& k) {
        i = (int)(q % L.g.n[0]);
        const long long rr = q / L.g.n[0];
        j = (int)(rr % L.g.n[1]);
        k = (int)(rr / L.g.n[1]);
    };
    T m = T(0);
    for (long long q = tid; q < n; q += bs)
    {
        x[q] = T(0);
        r[q] = b[q];
        rh[q] = b[q];
        p[q] = T(0);
        v[q] = T(0);
        const T a = r[q] < T(0) ? -r[q] : r[q];
        m = a > m ? a : m;
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
            for (long long q = tid; q < n; q += bs)
            {
                int i, j, k;
                cell(q, i, j, k);
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
                m = a > m ? a : m;
            }
            if (block_max(m, sh) <= rel * rnorm0)
            {
                ret = 0;
                break;
            }
            T a1 = T(0), a2 = T(0);
            for (long long q = tid; q < n; q += bs)
            {
                int i, j, k;
                cell(q, i, j, k);
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
                m = a > m ? a : m;
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
            for (long long q = tid; q < n; q += bs)
            {
                int i, j, k;
                cell(q, i, j, k);
                if (((i + j + k + color) & 1) == 0) mg_gs_cell(L, x, b, i, j, k, false);
            }
            __syncthreads();
        }
    if (tid == 0 && status) *status = ret;
}

// Mean of the coincident fine faces onto a coarse face.
template <typename T>
__global__ void k_mg_avg_faces(GridDev gf, GridDev gc, int d, const T* __restrict__ bf,
                               T* __restrict__ bc)
{
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

// Robin coefficients on a coarse boundary side: mean of the fine a,b over
// the 2^(dim-1) fine faces, then c0 = (b/dx - a/2) / (a/2 + b/dx).
template <typename T>
__global__ void k_mg_robin_coarsen(GridDev gf, GridDev gc, int s, const T* ra_f,
                                   const T* rb_f, T* ra_c, T* rb_c, T* c0_c, T dxc)
{
    const int d = s % 3;
    const int ta = (d == 0) ? 1 : 0, tb = (d == 2) ? 1 : 2;
    const int na = gc.n[ta], nb = gc.n[tb];
    const bool tb_active = tb < gf.dim;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < na * nb;
         q += gridDim.x * blockDim.x)
    {
        const int ia = q % na, ib = q / na;
        T sa = T(0), sb = T(0);
        int cnt = 0;
        for (int u = 0; u < 2; ++u)
            for (int w = 0; w < (tb_active ? 2 : 1); ++w)
            {
                const int fa = 2 * ia + u;
                const int fb = tb_active ? 2 * ib + w : ib;
                const int fp = fa + gf.n[ta] * fb;
                sa += ra_f[fp];
                sb += rb_f[fp];
                ++cnt;
            }
        const T a = sa / T(cnt), b = sb / T(cnt);
        ra_c[q] = a;
        rb_c[q] = b;
        const T dxi = T(1) / dxc;
        c0_c[q] = (b * dxi - T(0.5) * a) / (T(0.5) * a + b * dxi);
    }
}

template <typename T>
__global__ void k_fill(T* p, T v, long long n)
{
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
         t += (long long)gridDim.x * blockDim.x)
        p[t] = v;
}

template <typename TO, typename TI>
__global__ void k_convert(TO* __restrict__ o, const TI* __restrict__ in, TI scale, long long n)
{
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
         t += (long long)gridDim.x * blockDim.x)
        o[t] = (TO)(in[t] * scale);
}

} // namespace vd
