// Compatibility layer that lets a reference case directory (Chemistry.H,
// Chemistry.cpp, UserFunctions.H, UserSources.H, Prob.H, ProbParm.H of
// test/verification/* or test/models/*) compile unchanged against this
// library and its oracle.  The reference writes its hooks against AMReX
// (AMReX_REAL.H, AMReX_Geometry.H, AMReX_FArrayBox.H, AMReX_Gpu.H,
// AMReX_ParmParse.H, AMReX_GpuMemory.H, AMReX_Box.H, UnivConstants.H,
// VarDefines.H); the headers of those names in this directory all include
// this file, which maps the names the hooks use onto the library's own
// plugin types (vd_defs.H) and parameter reader (vd_parmparse.H):
//
//   amrex::Real, IntVect, GpuArray, Box, GeometryData   the vd:: types
//   amrex::Array4<T>                                    vd::Array4
//   amrex::Vector<T>                                    std::vector<T>
//   amrex::Math::powi / abs                             vd::Math
//   amrex::lbound / ubound                              box corners
//   amrex::ParmParse("prob")                            the `prob.*` table
//                                                       vd_init_domain parses
//   amrex::Gpu::htod_memcpy                             host copy (the
//                                                       library uploads
//                                                       ProbParm itself)
//   amrex::literals (_rt)                               FP64 literals
//
// and defines VD_REFERENCE_CASE, which makes the library call the hooks
// with the reference's own signatures: potential_bc / species_bc with the
// three integrated-current arrays (passed as zeros: current tracking is out
// of scope), amrex_probinit(ProbParm&, ProbParm&) reading through
// amrex::ParmParse, initdomaindata with a non-const ProbParm*.  Reference
// hooks that need AMReX's runtime (ParallelFor, The_Arena, embedded
// boundaries, Print) are outside what a case on this path needs and are not
// provided.
#pragma once

#include "vd_defs.H"
#include "vd_parmparse.H"
#include "vd_ids.H"

#include <cstring>
#include <string>
#include <vector>

#ifndef VD_REFERENCE_CASE
#define VD_REFERENCE_CASE 1
#endif
// a reference UserFunctions.H always defines the user_transport hooks
#ifndef VD_HAS_USER_TRANSPORT
#define VD_HAS_USER_TRANSPORT 1
#endif

// device-side constant tables of generated mechanisms (global_imw, ...)
#define AMREX_USE_GPU 1
#ifdef __CUDA_ARCH__
#define AMREX_DEVICE_COMPILE 1
#else
#define AMREX_DEVICE_COMPILE 0
#endif
#if defined(__CUDACC__)
#define AMREX_GPU_CONSTANT __constant__
#else
#define AMREX_GPU_CONSTANT
#endif
#define AMREX_PRAGMA_SIMD
#define AMREX_RESTRICT __restrict__

namespace amrex {
using vd::Box;
using vd::GeometryData;
using vd::GpuArray;
using vd::IntVect;
using vd::Real;
template <class T>
using Array4 = vd::Array4;
template <class T>
using Vector = std::vector<T>;
namespace Math = vd::Math;

struct Dim3
{
    int x, y, z;
};
VD_HD inline Dim3 lbound(const Box& b) { return {b.lo[0], b.lo[1], b.lo[2]}; }
VD_HD inline Dim3 ubound(const Box& b) { return {b.hi[0], b.hi[1], b.hi[2]}; }

// ParmParse over the parameter table the library hands to amrex_probinit
// (set for the duration of that call by vd_probinit, vd_probinit.H).
class ParmParse
{
public:
    explicit ParmParse(const std::string& prefix = "") : m_pp(table(), prefix) {}
    static const vd::ParmParse::Table*& table()
    {
        static thread_local const vd::ParmParse::Table* t = nullptr;
        return t;
    }
    template <class T>
    bool query(const char* name, T& out) const
    {
        return m_pp.query(name, out);
    }
    template <class T>
    void get(const char* name, T& out) const
    {
        m_pp.query(name, out);
    }
    template <class T>
    bool queryarr(const char* name, std::vector<T>& out) const
    {
        const auto* v = m_pp.find(name);
        if (!v) return false;
        out.clear();
        for (const auto& s : *v)
        {
            T x{};
            std::istringstream is(s);
            is >> x;
            out.push_back(x);
        }
        return true;
    }
    template <class T>
    void getarr(const char* name, std::vector<T>& out) const
    {
        queryarr(name, out);
    }
    bool contains(const char* name) const { return m_pp.find(name) != nullptr; }

private:
    vd::ParmParse m_pp;
};

namespace Gpu {
inline void htod_memcpy(void* dst, const void* src, std::size_t n) { std::memcpy(dst, src, n); }
} // namespace Gpu
// the OpenMP `if` of the reference's host loops over a box
namespace GPU {
constexpr bool notInLaunchRegion = false;
}

namespace literals {
constexpr Real operator""_rt(long double x) { return Real(x); }
constexpr Real operator""_rt(unsigned long long x) { return Real(x); }
} // namespace literals
} // namespace amrex

// the integrated-current arguments of the reference's boundary hooks
#define VD_CURRENT_ARGS                                                        \
    , vd::GpuArray<vd::Real, MAX_CURRENT_LOCS>{}, vd::GpuArray<vd::Real, MAX_CURRENT_LOCS>{}, \
        vd::GpuArray<int, MAX_CURRENT_LOCS>{}
