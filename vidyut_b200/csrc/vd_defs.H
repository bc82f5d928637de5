// Plugin-surface types shared by the CUDA library and by case headers.
//
// A Vidyut case is a directory of device-inline hook headers (Chemistry.H,
// UserFunctions.H, UserSources.H, Prob.H, ProbParm.H), exactly as in the
// reference (docs/README.md:33-40, test/Make.vidyut:13-18).  The reference
// writes those hooks against AMReX types (Array4, IntVect, GpuArray).  This
// header provides small stand-ins with the same call syntax so that a case
// header ports by replacing `amrex::` with `vd::`:
//
//   Array4      phi(i,j,k,n) / phi(IntVect,n) element access.  A state view
//               clamps (first-order extrapolation, the reference's
//               `foextrap` ghost fill, Source/Vidyut.cpp:116-130) or wraps
//               (periodic, `int_dir`) out-of-domain reads, which replaces the
//               reference's FillPatch ghost cells (Source/GridWork.cpp:135-149).
//   IntVect     three ints, operator[].
//   GpuArray    fixed-size array passed by value to device code.
//
// Component indices (EEN_ID ... DCURZ_ID) and boundary-condition codes follow
// Source/VarDefines.H:5-45; physical constants follow Source/UnivConstants.H.
#pragma once

#include <cmath>
#include <cstdint>
#include <cstddef>

#if defined(__CUDACC__)
#define VD_HD __host__ __device__
#define VD_D __device__
#else
#define VD_HD
#define VD_D
#endif
#define VD_INLINE inline

// AMReX-spelling shims so that reference case headers port with minimal edits.
#define AMREX_GPU_HOST_DEVICE VD_HD
#define AMREX_GPU_DEVICE VD_HD
#define AMREX_FORCE_INLINE inline
#define AMREX_INLINE inline
#define AMREX_SPACEDIM 3
#define AMREX_D_DECL(a, b, c) a, b, c

namespace vd {

using Real = double;

struct IntVect
{
    int v[3];
    VD_HD IntVect() : v{0, 0, 0} {}
    VD_HD IntVect(int i, int j, int k) : v{i, j, k} {}
    VD_HD int& operator[](int d) { return v[d]; }
    VD_HD const int& operator[](int d) const { return v[d]; }
};

template <class T, int N>
struct GpuArray
{
    T arr[N];
    VD_HD T& operator[](int i) { return arr[i]; }
    VD_HD const T& operator[](int i) const { return arr[i]; }
};

// A strided 4-D view (x fastest, then y, z, component), the layout of an
// AMReX Array4.  `bx_lo/bx_hi` is the box the storage covers; with
// `clamp != 0`, indices outside [dom_lo, dom_hi] are mapped back into the
// domain (clamp = first-order extrapolation, or wrap where `periodic[d]`).
struct Array4
{
    Real* p = nullptr;
    int lo[3] = {0, 0, 0};
    int hi[3] = {0, 0, 0};
    long long jstride = 0, kstride = 0, nstride = 0;
    int clamp = 0;
    int periodic[3] = {0, 0, 0};

    VD_HD int fix(int i, int d) const
    {
        if (!clamp) return i;
        const int n = hi[d] - lo[d] + 1;
        if (i < lo[d]) return periodic[d] ? hi[d] - ((lo[d] - i - 1) % n) : lo[d];
        if (i > hi[d]) return periodic[d] ? lo[d] + ((i - hi[d] - 1) % n) : hi[d];
        return i;
    }
    VD_HD Real& operator()(int i, int j, int k, int n = 0) const
    {
        i = fix(i, 0);
        j = fix(j, 1);
        k = fix(k, 2);
        return p[(i - lo[0]) + (j - lo[1]) * jstride + (k - lo[2]) * kstride +
                 n * nstride];
    }
    VD_HD Real& operator()(const IntVect& iv, int n = 0) const
    {
        return (*this)(iv[0], iv[1], iv[2], n);
    }
};

// Geometry handed to initdomaindata (the reference's GeometryData).
struct GeometryData
{
    Real prob_lo[3];
    Real prob_hi[3];
    Real dx[3];
    int n_cell[3];
    VD_HD const Real* ProbLo() const { return prob_lo; }
    VD_HD const Real* ProbHi() const { return prob_hi; }
    VD_HD const Real* CellSize() const { return dx; }
};

struct Box
{
    int lo[3];
    int hi[3];
};

template <class T>
VD_HD VD_INLINE T vmax(T a, T b) { return a > b ? a : b; }
template <class T>
VD_HD VD_INLINE T vmin(T a, T b) { return a < b ? a : b; }

namespace Math {
template <int N>
VD_HD VD_INLINE Real powi(Real x)
{
    Real r = 1.0;
    for (int i = 0; i < N; ++i) r *= x;
    return r;
}
VD_HD VD_INLINE Real abs(Real x) { return std::fabs(x); }
} // namespace Math

} // namespace vd

// ---- physical constants: values of Source/UnivConstants.H:4-20 ----------
#define N_A 6.02214076e23
#define K_B 1.380649e-23
#define PI 3.14159265358979323846264338327950288
#define P_NTP 101325.0
#define T_NTP 293.15
#define N_NTP (P_NTP / K_B / T_NTP)
#define FARADCONST 96485.332
#define GASCONST 8.31446261815324
#define ECHARGE 1.60217662e-19
#define EPS0 8.854187817e-12
#define eV (ECHARGE / K_B)
#define FBYR (FARADCONST / GASCONST)
#define ME 9.10938188e-31
#define M_AMU 1.66054e-27
#define TDUNIT 1e-21
#define fivebythree (5.0 / 3.0)
#define twothird (2.0 / 3.0)

// ---- boundary-condition codes: Source/VarDefines.H:40-45 -----------------
#define PERBC 0
#define DIRCBC 1
#define HNEUBC 2
#define IHNEUBC 3
#define ROBINBC 4
#define AXISBC 5

#define MAX_CURRENT_LOCS 10
