// B200-native per-timestep species-and-field update of Vidyut3d on one
// uniform level: host driver and C ABI (include/vidyut_b200.h).
//
// One translation unit per case directory (-I <case>): the case's hook
// headers are compiled into every kernel, as the reference compiles one
// executable per case.  All device memory is allocated in vd_create; a
// step allocates nothing.  Work is ordered on one CUDA stream per context.
#include <vidyut_b200.h>

#include "vd_vars.H"
#include "vd_parmparse.H"
#include "PlasmaChem.H"
#include <UserFunctions.H>
#include <UserSources.H>
#include <Prob.H>
#include "vd_probinit.H"

#include "vd_common.cuh"
#include "vd_kernels.cuh"
#include "vd_mg_tma.cuh"
#include "vd_adjoint.cuh"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <sstream>
#include <string>
#include <type_traits>
#include <vector>

namespace vd {
long long g_launches = 0;
}
using namespace vd;

namespace {
using vd::Array4;
using vd::Box;
using vd::GeometryData;
using vd::GpuArray;
using vd::IntVect;
using vd::Real;

constexpr int BS = 256;

dim3 gsz(long long n)
{
    long long b = (n + BS - 1) / BS;
    if (b < 1) b = 1;
    if (b > 148LL * 32) b = 148LL * 32;
    return dim3((unsigned)b);
}

// Every launch is a programmatic dependent launch (launch_pdl below): all
// kernels of the library start with VD_PDL_WAIT().
#define LAUNCH(K, G, B, STREAM, ...) launch_pdl(K, G, B, 0, STREAM, __VA_ARGS__)

// Launch as a programmatic dependent launch: the kernel may be scheduled
// while the previous kernel on the stream drains, hiding the launch latency
// that dominates the small multigrid levels.  Only for kernels that begin
// with VD_PDL_WAIT() (the multigrid kernels of vd_mg.cuh).
template <typename... KArgs, typename... Args>
void launch_pdl(void (*k)(KArgs...), dim3 g, dim3 b, size_t smem, cudaStream_t st,
                Args&&... args)
{
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = g;
    cfg.blockDim = b;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    VD_CUDA_OK(cudaLaunchKernelEx(&cfg, k, std::forward<Args>(args)...));
    ++vd::g_launches;
}
#define LAUNCH_PDL(K, G, B, STREAM, ...) launch_pdl(K, G, B, 0, STREAM, __VA_ARGS__)

// Launch-by-launch event timing of one selected kernel.
struct Prof
{
    int id = VD_PROF_NONE;
    std::vector<cudaEvent_t> a, b;
    std::vector<int> cnt; // launches inside each timed region
    int n = 0;
    double bytes = 0.0;
    void begin(cudaStream_t st)
    {
        if (n >= (int)a.size())
        {
            cudaEvent_t x, y;
            VD_CUDA_OK(cudaEventCreate(&x));
            VD_CUDA_OK(cudaEventCreate(&y));
            a.push_back(x);
            b.push_back(y);
        }
        VD_CUDA_OK(cudaEventRecord(a[n], st));
    }
    void end(cudaStream_t st, int launches = 1)
    {
        VD_CUDA_OK(cudaEventRecord(b[n], st));
        if ((int)cnt.size() <= n) cnt.resize(n + 1);
        cnt[n] = launches;
        ++n;
    }
};
thread_local Prof* t_prof = nullptr;

// Allocations left before a simulated out-of-memory failure (host-side
// fault injection for tests: VD_FAULT_ALLOC_AFTER=n makes the allocation
// after the n-th of a context fail as cudaMalloc does when the device is
// full); -1: off.
static long long fault_alloc_after()
{
    const char* e = std::getenv("VD_FAULT_ALLOC_AFTER");
    return (e && *e) ? std::atoll(e) : -1;
}

struct Alloc
{
    std::vector<void*> ptrs;
    long long fault_after = fault_alloc_after();
    template <class T>
    T* get(size_t n)
    {
        if (n == 0) n = 1;
        void* p = nullptr;
        const size_t bytes = n * sizeof(T);
        if (fault_after >= 0 && (long long)ptrs.size() >= fault_after)
            throw OomError("cudaMalloc of " + std::to_string(bytes) +
                           " bytes failed: out of memory (injected by VD_FAULT_ALLOC_AFTER)");
        const cudaError_t r = cudaMalloc(&p, bytes);
        if (r == cudaErrorMemoryAllocation)
        {
            cudaGetLastError(); // not sticky: clear it for the calls that follow
            throw OomError("cudaMalloc of " + std::to_string(bytes) + " bytes failed: out of memory");
        }
        if (r != cudaSuccess)
            throw CudaError("cudaMalloc of " + std::to_string(bytes) + " bytes failed: " +
                            cudaGetErrorString(r));
        ptrs.push_back(p);
        return static_cast<T*>(p);
    }
    void release()
    {
        for (void* p : ptrs) cudaFree(p);
        ptrs.clear();
    }
};

int mg_type(int code)
{
    switch (code)
    {
    case PERBC: return MG_PER;
    case DIRCBC: return MG_DIR;
    case HNEUBC: return MG_NEU;
    case IHNEUBC: return MG_INNEU;
    case ROBINBC: return MG_ROBIN;
    case AXISBC: return MG_NEU;
    default: return MG_ROBIN;
    }
}

// ------------------------------------------------------------ hierarchy
template <typename T>
struct Hier
{
    int nlev = 0;
    int dim = 3;
    bool varb = false;
    std::vector<GridDev> g;
    std::vector<std::array<double, 3>> dx;
    std::vector<T*> x, f;
    std::vector<std::array<T*, 3>> bf;
    std::vector<std::array<T*, 6>> ra, rb, c0;
    std::array<T*, 6> g0{};
    T* t0x = nullptr; // level-0 correction when there is a single level
    T* t0f = nullptr;
    T* scratch = nullptr;
    int* status = nullptr;
    std::vector<MGOp<T>> op;
    int prof_tag = VD_PROF_NONE; // profiling id of this hierarchy's fine sweeps
    int nu1 = 2, nu2 = 2, nub = 0, nuf = 8, bot_maxiter = 200;
    double bot_rel = 1e-4;
};

template <typename T>
void hier_build(Hier<T>& H, Alloc& A, const GridDev& fine, const double* dx, int maxcoarsen,
                bool varb, bool own0)
{
    H.dim = fine.dim;
    H.varb = varb;
    GridDev f0 = fine;
    f0.rb = (fine.n[0] % 2 == 0) ? 1 : 0;
    H.g.push_back(f0);
    H.dx.push_back({dx[0], dx[1], dx[2]});
    while ((int)H.g.size() - 1 < maxcoarsen)
    {
        const GridDev& c = H.g.back();
        bool ok = true;
        for (int d = 0; d < H.dim; ++d)
            if (c.n[d] % 2 != 0 || c.n[d] / 2 < 2) ok = false;
        if (!ok) break;
        GridDev n = c;
        std::array<double, 3> ndx = H.dx.back();
        for (int d = 0; d < H.dim; ++d)
        {
            n.n[d] = c.n[d] / 2;
            ndx[d] = ndx[d] * 2.0;
        }
        n.rb = (n.n[0] % 2 == 0) ? 1 : 0;
        H.g.push_back(n);
        H.dx.push_back(ndx);
    }
    H.nlev = (int)H.g.size();
    H.x.assign(H.nlev, nullptr);
    H.f.assign(H.nlev, nullptr);
    H.bf.assign(H.nlev, {nullptr, nullptr, nullptr});
    H.ra.assign(H.nlev, {});
    H.rb.assign(H.nlev, {});
    H.c0.assign(H.nlev, {});
    for (int l = 0; l < H.nlev; ++l)
    {
        const long long n = H.g[l].ncell();
        if (l > 0 || own0)
        {
            H.x[l] = A.get<T>(n);
            H.f[l] = A.get<T>(n);
        }
        if (varb)
            for (int d = 0; d < H.dim; ++d) H.bf[l][d] = A.get<T>(face_count(H.g[l], d));
        for (int s = 0; s < 6; ++s)
        {
            const int np = plane_count(H.g[l], s % 3);
            H.ra[l][s] = A.get<T>(np);
            H.rb[l][s] = A.get<T>(np);
            H.c0[l][s] = A.get<T>(np);
        }
    }
    for (int s = 0; s < 6; ++s) H.g0[s] = A.get<T>(plane_count(fine, s % 3));
    if (H.nlev == 1)
    {
        H.t0x = A.get<T>(fine.ncell());
        H.t0f = A.get<T>(fine.ncell());
    }
    H.scratch = A.get<T>(6 * H.g.back().ncell());
    H.status = A.get<int>(1);
}

// Level size from which the multigrid sweeps switch to the kernels built for
// levels that live in HBM rather than L2 (two planes per thread).
// The environment variable VD_MG_BIG_LEVEL_CELLS overrides the 8 M default,
// so that tests can drive those kernels on grids the oracle solves quickly.
static long long big_level_cells()
{
    const char* e = std::getenv("VD_MG_BIG_LEVEL_CELLS");
    const long long v = e ? std::atoll(e) : 0;
    return v > 0 ? v : (8LL << 20);
}

// TMA-staged sweeps on the big constant-coefficient levels when the
// environment variable VD_MG_TMA is 1 (the register-staged sweeps are
// faster on B200 and stay the default; the two give the same bits, and
// tests compare them).
static int tma_sweeps()
{
    const char* e = std::getenv("VD_MG_TMA");
    return (e && e[0] == '1') ? 1 : 0;
}

template <typename T>
void hier_set_ops(Hier<T>& H, double aconst, double beta, double bconst, const int* bct,
                  int maxorder)
{
    H.op.assign(H.nlev, MGOp<T>{});
    const long long big = big_level_cells();
    const int tma = tma_sweeps();
    for (int l = 0; l < H.nlev; ++l)
    {
        MGOp<T>& o = H.op[l];
        o.g = H.g[l];
        o.big_cells = big;
        o.tma = tma;
        for (int d = 0; d < 3; ++d)
            o.dh[d] = (d < H.dim) ? T(beta / (H.dx[l][d] * H.dx[l][d])) : T(0);
        o.aconst = T(aconst);
        o.a = nullptr;
        for (int d = 0; d < 3; ++d) o.b[d] = (H.varb && d < H.dim) ? H.bf[l][d] : nullptr;
        o.bconst = T(bconst);
        for (int s = 0; s < 6; ++s)
        {
            const int d = s % 3;
            o.bct[s] = bct[s];
            o.c0s[s] = T(1);
            o.c1s[s] = T(0);
            o.c0[s] = nullptr;
            o.gv[s] = nullptr;
            if (bct[s] == MG_DIR)
            {
                const int NX = std::min(H.g[l].n[d] + 1, maxorder);
                o.c0s[s] = (NX <= 2) ? T(-1) : T(-2);
                o.c1s[s] = (NX <= 2) ? T(0) : T(1.0 / 3.0);
                if (l == 0) o.gv[s] = H.g0[s];
            } else if (bct[s] == MG_ROBIN)
            {
                o.c0[s] = H.c0[l][s];
                if (l == 0) o.gv[s] = H.g0[s];
            }
        }
    }
}

template <typename T>
void hier_coarsen_coeffs(Hier<T>& H, const int* bct, cudaStream_t st)
{
    for (int l = 1; l < H.nlev; ++l)
    {
        if (H.varb)
            for (int d = 0; d < H.dim; ++d)
                LAUNCH(k_mg_avg_faces<T>, gsz(face_count(H.g[l], d)), BS, st, H.g[l - 1],
                       H.g[l], d, H.bf[l - 1][d], H.bf[l][d]);
        for (int s = 0; s < 6; ++s)
            if (bct[s] == MG_ROBIN)
                LAUNCH(k_mg_robin_coarsen<T>, gsz(plane_count(H.g[l], s % 3)), BS, st,
                       H.g[l - 1], H.g[l], s, H.ra[l - 1][s], H.rb[l - 1][s], H.ra[l][s],
                       H.rb[l][s], H.c0[l][s], T(H.dx[l - 1][s % 3]), T(H.dx[l][s % 3]));
    }
}

// 3-D red-black split levels with no periodic direction run the kernels
// that keep several planes per thread in flight (k_mg_sweep3, k_mg_restrict3,
// k_mg_resid3).
template <typename T>
bool mg3_ok(const MGOp<T>& op)
{
    const GridDev& g = op.g;
    return g.rb && g.dim == 3 && g.n[0] >= 4 && g.n[1] >= 4 && g.n[2] >= 4 && !op.a &&
           !g.per[0] && !g.per[1] && !g.per[2] && g.ncell() < (1LL << 31);
}

dim3 mg3_grid(const GridDev& g)
{
    return dim3((g.n[0] / 2 + 31) / 32, (g.n[1] + 7) / 8, (g.n[2] + MG3_U - 1) / MG3_U);
}

// Convergence check fused into the first sweep of a V-cycle (FP64 plain
// solves): the sweep's per-block residual maxima go to part, then one block
// reduces them into dmg->rbits and k_mg_check applies the stopping test.
struct NormFuse
{
    double* part;
    long long npart;
    MGDev* dmg;
    double target;
};

// Whether the first colour-0 sweep of op's level can carry the convergence
// norm (the pair kernel with enough per-block slots).
template <typename T>
bool norm_fusable(const MGOp<T>& op, long long npart)
{
    if (!std::is_same<T, double>::value || !mg3_ok(op) || op.g.n[0] % 4) return false;
    const bool two = op.g.ncell() >= (op.big_cells > 0 ? op.big_cells : (8LL << 20));
    const int uv = two ? 2 : 1;
    const long long nb = (long long)((op.g.n[0] / 2 + 63) / 64) * ((op.g.n[1] + 7) / 8) *
                         ((op.g.n[2] + uv - 1) / uv);
    return nb <= npart;
}

// cuTensorMapEncodeTiled from the driver, through the runtime's entry-point
// query (no link against libcuda); null if the driver does not offer it.
using TmaEncodeFn = decltype(&cuTensorMapEncodeTiled);
static TmaEncodeFn tma_encode_fn()
{
    static const TmaEncodeFn fn = []() -> TmaEncodeFn {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) !=
                cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            return nullptr;
        return reinterpret_cast<TmaEncodeFn>(p);
    }();
    return fn;
}

// Tensor map of one colour half of a 3-D split level: dims (nxh, ny, nz),
// box (bx, by, 1), zero fill outside.  False where TMA cannot address it
// (base or row pitch not a multiple of 16 bytes).
template <typename T>
static bool tma_map_half(CUtensorMap* m, const T* base, const GridDev& g, int bx, int by)
{
    const TmaEncodeFn enc = tma_encode_fn();
    const long long nxh = g.n[0] / 2;
    if (!enc || (reinterpret_cast<uintptr_t>(base) & 15) || (nxh * (long long)sizeof(T)) % 16)
        return false;
    const cuuint64_t dims[3] = {(cuuint64_t)nxh, (cuuint64_t)g.n[1], (cuuint64_t)g.n[2]};
    const cuuint64_t strides[2] = {(cuuint64_t)(nxh * sizeof(T)),
                                   (cuuint64_t)(nxh * g.n[1] * sizeof(T))};
    const cuuint32_t box[3] = {(cuuint32_t)bx, (cuuint32_t)by, 1};
    const cuuint32_t es[3] = {1, 1, 1};
    return enc(m, sizeof(T) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32,
               3, const_cast<T*>(base), dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
               CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

static int sm_count()
{
    static int n[64] = {};
    int dev = 0;
    VD_CUDA_OK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) dev = 0;
    if (!n[dev]) VD_CUDA_OK(cudaDeviceGetAttribute(&n[dev], cudaDevAttrMultiProcessorCount, dev));
    return n[dev];
}

// Launch shape of a TMA-staged sweep: the level's tiles times the z-chunks
// that fill two CTAs per SM (at least one chunk; nzc chunks of a plane each
// at most).  Returns the grid size; *nzc gets the chunk count.
template <typename T>
static int tma_sweep_grid(const GridDev& g, int* nzc = nullptr)
{
    using S = TmaSweepShape<T, false>;
    const int ntiles = ((g.n[0] / 2 + TMA_TX - 1) / TMA_TX) * ((g.n[1] + S::TY - 1) / S::TY);
    const int chunks = std::max(1, std::min(g.n[2], S::MINB * sm_count() / ntiles));
    if (nzc) *nzc = chunks;
    return ntiles * chunks;
}

// One colour sweep of a big constant-coefficient level with TMA-staged
// operands; false (nothing launched) where the level cannot take it.
template <typename T, bool PROL, bool NORM>
static bool sweep_tma(const MGOp<T>& op, T* x, const T* f, int color, bool inh, T ig,
                      const GridDev& gcv, const T* xc, double* part, cudaStream_t st)
{
    using S = TmaSweepShape<T, NORM>;
    const long long half = op.g.ncell() / 2;
    CUtensorMap mx, mf, mv;
    if (!tma_map_half(&mx, x + (1 - color) * half, op.g, TMA_TX + 2 * S::XH, S::TY + 2) ||
        !tma_map_half(&mf, f + color * half, op.g, TMA_TX, S::TY))
        return false;
    if (NORM && !tma_map_half(&mv, x + color * half, op.g, TMA_TX, S::TY)) return false;
    if (!NORM) mv = mf;
    static bool attr = false;
    if (!attr)
    {
        VD_CUDA_OK(cudaFuncSetAttribute(k_mg_sweep3t<T, PROL, NORM>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, S::SMEM));
        attr = true;
    }
    int nzc = 1;
    const int grid = tma_sweep_grid<T>(op.g, &nzc);
    launch_pdl(k_mg_sweep3t<T, PROL, NORM>, dim3(grid), dim3(S::THREADS), (size_t)S::SMEM, st, op,
               mx, mf, mv, x, color, inh ? 1 : 0, ig, gcv, xc, part, op.err, nzc);
    return true;
}

// n Gauss-Seidel iterations (colour 0, colour 1).  With xc given (only for
// mg3_ok levels) the first colour-0 sweep also adds the prolongated coarse
// correction xc of level gc; with nf given (norm_fusable levels) it also
// takes the convergence norm of the current x (NormFuse).
template <typename T>
void smooth(const MGOp<T>& op, T* x, const T* f, bool inh, int n, cudaStream_t st,
            int prof_tag = VD_PROF_NONE, const GridDev* gc = nullptr, const T* xc = nullptr,
            const NormFuse* nf = nullptr)
{
    const long long half = (long long)((op.g.n[0] + 1) / 2) * op.g.n[1] * op.g.n[2];
    const bool prof = t_prof && prof_tag != VD_PROF_NONE && t_prof->id == prof_tag;
    // one colour: read the other colour of x and this colour of f, write
    // this colour of x (plus the face coefficients when they vary)
    if (prof)
        t_prof->bytes = double(3 * sizeof(T)) / 2.0 * (double)op.g.ncell() +
                        (op.b[0] ? double(op.g.dim * sizeof(T)) * (double)op.g.ncell() : 0.0);
    bool open = false;
    int timed = 0;
    for (int s = 0; s < n; ++s)
        for (int color = 0; color < 2; ++color)
        {
            const bool fuse = nf && s == 0 && color == 0;
            const bool pf = prof && !fuse; // the timed sweeps are the plain ones
            // consecutive plain sweeps of one call form one timed region, so
            // the events do not break the launches' programmatic overlap
            if (pf && !open)
            {
                t_prof->begin(st);
                open = true;
            }
            T gamma = op.aconst; // interior diagonal of the constant-coefficient operator
            for (int d = 0; d < op.g.dim; ++d) gamma += op.dh[d] * (op.bconst + op.bconst);
            if (mg3_ok(op))
            {
                const dim3 grid = mg3_grid(op.g);
                const bool pro = xc && s == 0 && color == 0;
                const GridDev gcv = gc ? *gc : op.g;
                if (op.g.n[0] % 4 == 0)
                {
                    // pairs of half-cells per thread, 16-byte accesses
                    const bool two = op.g.ncell() >= (op.big_cells > 0 ? op.big_cells
                                                                       : (8LL << 20));
                    const int uv = two ? 2 : 1;
                    const dim3 gv((op.g.n[0] / 2 + 63) / 64, grid.y, (op.g.n[2] + uv - 1) / uv);
                    const T ig = op.b[0] ? T(0) : T(1) / gamma;
#define VD_SWEEP3V(VB, PR, UV)                                                                \
    LAUNCH_PDL((k_mg_sweep3v<T, VB, PR, UV>), gv, 256, st, op, x, f, color, inh ? 1 : 0, ig, gcv, \
               xc, (double*)nullptr)
#define VD_SWEEP3N(VB, UV)                                                                    \
    LAUNCH_PDL((k_mg_sweep3v<T, VB, false, UV, true>), gv, 256, st, op, x, f, color,          \
               inh ? 1 : 0, ig, gcv, xc, nf->part)
                    // big constant-coefficient levels: TMA-staged sweeps
                    const bool tma = two && op.tma && op.err && !op.b[0];
                    if (fuse)
                    {
                        long long nbv = (long long)gv.x * gv.y * gv.z;
                        if (tma && sweep_tma<T, false, true>(op, x, f, color, inh, ig, gcv, xc,
                                                             nf->part, st))
                            nbv = tma_sweep_grid<T>(op.g);
                        else if (op.b[0])
                            { if (two) VD_SWEEP3N(true, 2); else VD_SWEEP3N(true, 1); }
                        else
                            { if (two) VD_SWEEP3N(false, 2); else VD_SWEEP3N(false, 1); }
                        LAUNCH_PDL(k_mg_max_partials<T>, 1, 1024, st, op, nf->part, nbv, 0,
                                   &nf->dmg->rbits);
                        LAUNCH_PDL(k_mg_check, 1, 1, st, nf->dmg, nf->target);
                    } else if (tma && (pro ? sweep_tma<T, true, false>(op, x, f, color, inh, ig, gcv,
                                                                       xc, nullptr, st)
                                           : sweep_tma<T, false, false>(op, x, f, color, inh, ig,
                                                                        gcv, xc, nullptr, st)))
                    {
                        // launched
                    } else if (op.b[0] && pro)
                        { if (two) VD_SWEEP3V(true, true, 2); else VD_SWEEP3V(true, true, 1); }
                    else if (op.b[0])
                        { if (two) VD_SWEEP3V(true, false, 2); else VD_SWEEP3V(true, false, 1); }
                    else if (pro)
                        { if (two) VD_SWEEP3V(false, true, 2); else VD_SWEEP3V(false, true, 1); }
                    else
                        { if (two) VD_SWEEP3V(false, false, 2); else VD_SWEEP3V(false, false, 1); }
#undef VD_SWEEP3V
#undef VD_SWEEP3N
                } else if (op.b[0])
                {
                    if (pro)
                        LAUNCH_PDL((k_mg_sweep3<T, true, true>), grid, 256, st, op, x, f, color,
                               inh ? 1 : 0, T(0), gcv, xc);
                    else
                        LAUNCH_PDL((k_mg_sweep3<T, true, false>), grid, 256, st, op, x, f, color,
                               inh ? 1 : 0, T(0), gcv, xc);
                } else
                {
                    if (pro)
                        LAUNCH_PDL((k_mg_sweep3<T, false, true>), grid, 256, st, op, x, f, color,
                               inh ? 1 : 0, T(1) / gamma, gcv, xc);
                    else
                        LAUNCH_PDL((k_mg_sweep3<T, false, false>), grid, 256, st, op, x, f, color,
                               inh ? 1 : 0, T(1) / gamma, gcv, xc);
                }
            } else if (op.g.rb && op.g.dim == 3 && op.g.n[0] >= 4 && op.g.n[1] >= 4 &&
                       op.g.n[2] >= 4 && !op.a)
            {
                const int nxh = op.g.n[0] / 2;
                const int bx = nxh >= 128 ? 128 : (nxh >= 64 ? 64 : (nxh >= 32 ? 32 : 16));
                const int by = 256 / bx;
                const dim3 grid((nxh + bx - 1) / bx, (op.g.n[1] + by - 1) / by, op.g.n[2]);
                if (op.b[0])
                    LAUNCH_PDL((k_mg_smooth_rb3<T, true>), grid, dim3(bx, by), st, op, x, f, color,
                           inh ? 1 : 0, T(0));
                else
                    LAUNCH_PDL((k_mg_smooth_rb3<T, false>), grid, dim3(bx, by), st, op, x, f,
                           color, inh ? 1 : 0, T(1) / gamma);
            } else if (op.g.rb)
            {
                const int nxh = op.g.n[0] / 2;
                const int bx = nxh >= 128 ? 128 : (nxh >= 64 ? 64 : 32);
                const dim3 grid((nxh + bx - 1) / bx, op.g.n[1], op.g.n[2]);
                if (op.b[0])
                    LAUNCH_PDL((k_mg_smooth_rb<T, true>), grid, bx, st, op, x, f, color,
                           inh ? 1 : 0, T(0));
                else
                    LAUNCH_PDL((k_mg_smooth_rb<T, false>), grid, bx, st, op, x, f, color,
                           inh ? 1 : 0, T(1) / gamma);
            } else
                LAUNCH_PDL(k_mg_smooth_color<T>, gsz(half), BS, st, op, x, f, color, inh ? 1 : 0);
            if (pf) ++timed;
        }
    if (open) t_prof->end(st, timed);
}

// Launch shape over the cells of a grid: x-blocks along rows, y = j, z = k.
struct Grid3
{
    dim3 g, b;
};
Grid3 rows3(const GridDev& g, int ydiv = 1)
{
    const int nx = g.n[0];
    const int bx = nx >= 128 ? 128 : (nx >= 64 ? 64 : 32);
    return {dim3((nx + bx - 1) / bx, (g.n[1] + ydiv - 1) / ydiv, g.n[2]), dim3(bx)};
}

template <typename T>
void bottom(Hier<T>& H, const MGOp<T>& op, T* x, const T* f, cudaStream_t st)
{
    LAUNCH_PDL(k_mg_bottom<T>, 1, 256, st, op, x, f, H.scratch, T(H.bot_rel), H.bot_maxiter,
           H.nub, H.nuf, H.status);
}

// Levels of at most this many cells run inside the one-CTA coarse cycle;
// larger ones use the grid-wide kernels (a CTA sweeps ~2K cells per
// microsecond, a kernel launch costs a few microseconds).
#ifndef VD_MG_ONCHIP_CELLS
#define VD_MG_ONCHIP_CELLS 4096
#endif

// One V-cycle on level-0 unknown x0 with right-hand side f0; the level-0
// boundary data is inhomogeneous when `inh0` (the solution itself is
// smoothed), homogeneous otherwise (a correction is smoothed).
// Restriction of the colour-0 residuals only (k_mg_restrict3 C0ONLY); 0: all.
#ifndef VD_RESTRICT_C0
#define VD_RESTRICT_C0 1
#endif

// One V-cycle on x0.  With nf given, its first level-0 sweep also takes the
// convergence norm of x0 as it was on entry (NormFuse).
// First level small enough for the one-CTA coarse cycle (never level 0).
template <typename T>
int vcycle_lc(const Hier<T>& H)
{
    const int L = H.nlev;
    int lc = L - 1;
    while (lc > 1 && H.g[lc - 1].ncell() <= VD_MG_ONCHIP_CELLS) --lc;
    return lc;
}

// Whether the coarse levels from lc run as k_mg_coarse3 (3-D, non-periodic,
// on chip).
template <typename T>
bool coarse3_ok(const Hier<T>& H, int lc, size_t* smem = nullptr)
{
    MGCoarse<T> C{};
    C.lc = lc;
    C.nl = H.nlev;
    bool c3 = true;
    for (int l = lc; l < H.nlev; ++l)
    {
        const GridDev& g = H.g[l];
        C.op[l] = H.op[l];
        c3 = c3 && g.dim == 3 && !g.per[0] && !g.per[1] && !g.per[2] && !H.op[l].a &&
             g.n[0] < 1024 && g.n[1] < 1024 && g.n[2] < 1024;
    }
    const size_t smem3 = mg_coarse3_smem(C);
    if (smem) *smem = smem3;
    return c3 && smem3 <= VD_MG_COARSE_SMEM;
}

// The levels above the coarse cycle, going down: smoothing and restriction.
template <typename T>
void vcycle_down(Hier<T>& H, T* x0, T* f0, bool inh0, cudaStream_t st, const NormFuse* nf,
                 int lc)
{
    for (int l = 0; l < lc; ++l)
    {
        T* xl = l ? H.x[l] : x0;
        T* fl = l ? H.f[l] : f0;
        const bool inh = (l == 0) && inh0;
        smooth(H.op[l], xl, fl, inh, H.nu1, st, l == 0 ? H.prof_tag : VD_PROF_NONE,
               (const GridDev*)nullptr, (const T*)nullptr, l == 0 ? nf : nullptr);
        if (mg3_ok(H.op[l]))
        {
            const GridDev& gc = H.g[l + 1];
            const dim3 grid((gc.n[0] + 31) / 32, (gc.n[1] + 7) / 8, gc.n[2]);
            // after pre-smoothing (last sweep colour 1) only colour 0 has a
            // residual
            const bool c0 = VD_RESTRICT_C0 && H.nu1 >= 1;
#define VD_RESTRICT3(VB, C0)                                                                  \
    LAUNCH_PDL((k_mg_restrict3<T, VB, C0>), grid, 256, st, H.op[l], xl, fl, gc, H.f[l + 1],   \
               H.x[l + 1], inh ? 1 : 0)
            if (H.op[l].b[0])
                { if (c0) VD_RESTRICT3(true, true); else VD_RESTRICT3(true, false); }
            else
                { if (c0) VD_RESTRICT3(false, true); else VD_RESTRICT3(false, false); }
#undef VD_RESTRICT3
            continue;
        }
        const Grid3 gr = rows3(H.g[l + 1]);
        LAUNCH_PDL(k_mg_resid_restrict<T>, gr.g, gr.b, st, H.op[l], xl, fl, H.g[l + 1], H.f[l + 1],
               H.x[l + 1], inh ? 1 : 0);
    }
}

template <typename T>
MGCoarse<T> coarse_of(const Hier<T>& H, int lc)
{
    MGCoarse<T> C{};
    C.lc = lc;
    C.nl = H.nlev;
    for (int l = lc; l < H.nlev; ++l)
    {
        C.op[l] = H.op[l];
        C.x[l] = H.x[l];
        C.f[l] = H.f[l];
    }
    return C;
}

// The coarse levels lc .. nl-1 of one component.
template <typename T>
void vcycle_coarse(Hier<T>& H, cudaStream_t st, int lc)
{
    const int L = H.nlev;
    if (lc == L - 1)
    {
        bottom(H, H.op[L - 1], H.x[L - 1], H.f[L - 1], st);
        return;
    }
    const MGCoarse<T> C = coarse_of(H, lc);
    size_t smem3 = 0;
    if (coarse3_ok(H, lc, &smem3))
    {
        if (H.varb)
            launch_pdl(k_mg_coarse3<T, true>, dim3(1), dim3(MGC_THREADS), smem3, st, C,
                       T(H.bot_rel), H.bot_maxiter, H.nu1, H.nu2, H.nub, H.nuf);
        else
            launch_pdl(k_mg_coarse3<T, false>, dim3(1), dim3(MGC_THREADS), smem3, st, C,
                       T(H.bot_rel), H.bot_maxiter, H.nu1, H.nu2, H.nub, H.nuf);
    } else
    {
        const size_t smem = mg_coarse_smem(C);
        const int on_chip = smem <= VD_MG_COARSE_SMEM ? 1 : 0;
        k_mg_coarse_vcycle<T><<<1, 512, on_chip ? smem : 0, st>>>(
            C, H.scratch, T(H.bot_rel), H.bot_maxiter, H.nu1, H.nu2, H.nub, H.nuf, on_chip);
        ++vd::g_launches;
        VD_CUDA_OK(cudaGetLastError());
    }
}

// The levels above the coarse cycle, going up: prolongation and smoothing.
template <typename T>
void vcycle_up(Hier<T>& H, T* x0, T* f0, bool inh0, cudaStream_t st, int lc)
{
    for (int l = lc - 1; l >= 0; --l)
    {
        T* xl = l ? H.x[l] : x0;
        T* fl = l ? H.f[l] : f0;
        const bool inh = (l == 0) && inh0;
        if (mg3_ok(H.op[l]) && H.nu2 >= 1)
        {
            if (H.g[l].n[0] % 4 == 0)
            {
                // correction on colour 1 only; the first sweep (colour 0)
                // rewrites colour 0 without reading it
                const dim3 grid = mg3_grid(H.g[l]);
                const dim3 gv((H.g[l].n[0] / 2 + 63) / 64, grid.y, grid.z);
                LAUNCH_PDL(k_mg_prolong_c1<T>, gv, 256, st, H.g[l], H.g[l + 1], xl,
                       (const T*)H.x[l + 1], H.op[l].stop);
                smooth(H.op[l], xl, fl, inh, H.nu2, st, l == 0 ? H.prof_tag : VD_PROF_NONE);
            } else
                smooth(H.op[l], xl, fl, inh, H.nu2, st, l == 0 ? H.prof_tag : VD_PROF_NONE,
                       &H.g[l + 1], (const T*)H.x[l + 1]);
            continue;
        }
        const Grid3 gp = rows3(H.g[l]);
        LAUNCH_PDL(k_mg_prolong_add<T>, gp.g, gp.b, st, H.g[l], H.g[l + 1], xl, H.x[l + 1],
               H.op[l].stop);
        smooth(H.op[l], xl, fl, inh, H.nu2, st, l == 0 ? H.prof_tag : VD_PROF_NONE);
    }
}

template <typename T>
void vcycle(Hier<T>& H, T* x0, T* f0, bool inh0, unsigned long long* dscr, cudaStream_t st,
            const NormFuse* nf = nullptr)
{
    const int L = H.nlev;
    if (L == 1)
    {
        const Grid3 gn = rows3(H.g[0], 8);
        LAUNCH(k_mg_resid_norm<T>, gn.g, gn.b, st, H.op[0], x0, f0, H.t0f, dscr, inh0 ? 1 : 0,
               0, 8, (double*)nullptr);
        bottom(H, H.op[0], H.t0x, H.t0f, st);
        LAUNCH(k_add_same<T>, gsz(H.g[0].ncell()), BS, st, x0, H.t0x, H.g[0].ncell(),
               H.op[0].stop);
        return;
    }
    const int lc = vcycle_lc(H);
    vcycle_down(H, x0, f0, inh0, st, nf, lc);
    vcycle_coarse(H, st, lc);
    vcycle_up(H, x0, f0, inh0, st, lc);
}

// ------------------------------------------------------------ context
struct Ctx
{
    vd_config cfg{};
    int dev = 0;
    cudaStream_t st = nullptr;
    Geo G{};
    GridDev g{};
    long long N = 0;
    Alloc A;
    double* S = nullptr;
    double* Sold = nullptr; // separate copy only with >1 corrector or the coupling
    double* rxn_e = nullptr; // electron reaction source (electron-Poisson coupling)
    double* ephi = nullptr;  // coupling source of the potential equation
    double* expl = nullptr;
    double* rxn_een = nullptr;
    double* ejh = nullptr;
    double* jface[3] = {};   // Joule term of every face, per direction (energy equation)
    double* u[VD_NT] = {};   // solve outputs, indexed by component
    double* phi_sol = nullptr;
    double* phi_rhs = nullptr;
    double* spec_rhs = nullptr;
    double* r64 = nullptr;  // FP64 residual of the refinement form
    double* zero64 = nullptr; // all-zero level-0 array (warm-started potential)
    SideArrays pside[6]{}, sside[6]{};
    Hier<double> HP, HS;
    Hier<float> HP32, HS32;
    ProbParm hpp{};
    ProbParm* dpp = nullptr;
    unsigned long long* dscal = nullptr;
    unsigned long long* hscal = nullptr;
    double* dpart = nullptr; // per-block partial maxima of the residual norm
    long long npart = 0;
    MGDev* dmg = nullptr;   // device-side solve state (asynchronous V-cycles)
    MGDev* hmg = nullptr;   // pinned host mirror
    int hint[VD_NT + 1] = {}; // last V-cycle count per solve (index VD_NT: Poisson)
    double time = 0.0;
    int step = 0;
    double fixed_dt = 0.0;   // the configured step; cfg.dt is the current one
    double* dts = nullptr;   // electron time-scale maxima (device)
    double* hts = nullptr;   // pinned host mirror
    double tscale[3] = {};   // time scales of the last adaptive step
    int eidx = E_ID;
    int bg[NUM_SPECIES] = {};
    int pbct[6] = {}, ebct[6] = {}, eebct[6] = {}, ibct[6] = {}, nbct[6] = {};
    std::string err;
    Prof prof;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // last-solve bookkeeping
    long long poisson_iters = 0, species_iters = 0, poisson_refs = 0;
    int not_converged = 0;
    double max_poisson_res = 0.0;
    struct AdjState* adjs = nullptr; // discrete-adjoint buffers, made on first use
    // multicomponent species solves: effective chunk sizes and, per chunk
    // slot, a species hierarchy, boundary arrays and a right-hand side
    int ion_chunk = 1, neutral_chunk = 1;
    std::vector<Hier<double>> HJ;
    std::vector<std::array<SideArrays, 6>> JS;
    std::vector<double*> JR;
    MGCoarse<double>* dcoarse = nullptr; // per-slot coarse-cycle descriptors
    MGCoarse<double>* hcoarse = nullptr; // pinned staging copy
    double* rxn_bg = nullptr;            // background species' reaction sources
    int bgslot[NUM_SPECIES] = {};
};

// Effective multicomponent chunk sizes (Source/Vidyut.cpp:146-186): a Robin
// species wall forces chunks of one.  The reference tests lo[0], hi[0], then
// lo[1] twice and lo[2] twice (never hi[1], hi[2]); restated as it reads.
void multicomp_chunks(const vd_config& cfg, int& ion_chunk, int& neutral_chunk)
{
    ion_chunk = cfg.comp_ion_chunks;
    neutral_chunk = cfg.comp_neutral_chunks;
    auto robin = [&](const int* lo, const int* hi) {
        bool r = lo[0] == ROBINBC || hi[0] == ROBINBC;
        if (cfg.dim > 1) r = r || lo[1] == ROBINBC || lo[1] == ROBINBC;
        if (cfg.dim > 2) r = r || lo[2] == ROBINBC || lo[2] == ROBINBC;
        return r;
    };
    if (robin(cfg.ion_bc_lo, cfg.ion_bc_hi)) ion_chunk = 1;
    if (robin(cfg.neutral_bc_lo, cfg.neutral_bc_hi)) neutral_chunk = 1;
}

// [first, first + num) in chunks of `chunk`, then the remainder
// (Source/Evolve.cpp:462-495).
std::vector<std::pair<int, int>> chunk_list(int first, int num, int chunk)
{
    std::vector<std::pair<int, int>> out;
    if (num <= 0 || chunk <= 0) return out;
    int comp = first;
    for (; comp <= first + num - chunk; comp += chunk) out.push_back({comp, chunk});
    if (comp != first + num) out.push_back({comp, first + num - comp});
    return out;
}

bool in_neutral_range(int sp) { return sp >= FIRST_NEUTRAL && sp < FIRST_NEUTRAL + NUM_NEUTRALS; }

std::string g_create_err;

void set_err(Ctx* c, const std::string& m)
{
    if (c)
        c->err = m;
    else
        g_create_err = m;
}

void make_bct(const Ctx& c, const int* lo, const int* hi, int* out)
{
    for (int d = 0; d < 3; ++d)
    {
        if (d >= c.cfg.dim || c.cfg.is_periodic[d])
        {
            out[d] = MG_PER;
            out[d + 3] = MG_PER;
        } else
        {
            out[d] = mg_type(lo[d]);
            out[d + 3] = mg_type(hi[d]);
        }
    }
}

const int* bct_for(const Ctx& c, int comp)
{
    if (comp == c.eidx) return c.ebct;
    if (comp == EEN_ID) return c.eebct;
    return plasmachem::get_charge(comp) != 0 ? c.ibct : c.nbct;
}
const int* bclo_for(const Ctx& c, int comp)
{
    if (comp == c.eidx) return c.cfg.eden_bc_lo;
    if (comp == EEN_ID) return c.cfg.eenrg_bc_lo;
    return plasmachem::get_charge(comp) != 0 ? c.cfg.ion_bc_lo : c.cfg.neutral_bc_lo;
}
const int* bchi_for(const Ctx& c, int comp)
{
    if (comp == c.eidx) return c.cfg.eden_bc_hi;
    if (comp == EEN_ID) return c.cfg.eenrg_bc_hi;
    return plasmachem::get_charge(comp) != 0 ? c.cfg.ion_bc_hi : c.cfg.neutral_bc_hi;
}

double applied_potential(const vd_config& cfg, double t, int domend, int d)
{
    // Source/HelperFuncs.H:125-161
    const double amp = (domend == -1) ? cfg.voltage_amp_lo[d] : cfg.voltage_amp_hi[d];
    if (cfg.voltage_profile == 1) return std::sin(2.0 * PI * cfg.voltage_freq * t) * amp;
    if (cfg.voltage_profile == 2)
    {
        const double vc = cfg.voltage_center, vd_ = cfg.voltage_dur;
        if (t <= vc) return (vc - t < vd_ / 2.0) ? (1.0 - (vc - t) / (vd_ / 2.0)) * amp : 0.0;
        return (t - vc < vd_ / 2.0) ? (1.0 - (t - vc) / (vd_ / 2.0)) * amp : 0.0;
    }
    return amp;
}

double read_norm(Ctx& c)
{
    VD_CUDA_OK(cudaMemcpyAsync(c.hscal, c.dscal, sizeof(unsigned long long),
                               cudaMemcpyDeviceToHost, c.st));
    VD_CUDA_OK(cudaStreamSynchronize(c.st));
    double v;
    std::memcpy(&v, c.hscal, sizeof(double));
    return v;
}

// Residual max-norm in two stages (per-block maxima, then one block), into
// the bit patterns at mx[0] (|r|) and mx[1] (|f| when `fnorm`).
template <typename T>
void launch_norm(Ctx& c, const MGOp<T>& op, const T* x, const T* f, T* rout, bool inh,
                 bool fnorm, unsigned long long* mx, bool both = true, float* r32 = nullptr,
                 float* x32 = nullptr, const double* rscale = nullptr)
{
    if (mg3_ok(op))
    {
        const dim3 grid = mg3_grid(op.g);
        const long long nb = (long long)grid.x * grid.y * grid.z;
        const dim3 gv((op.g.n[0] / 2 + 63) / 64, grid.y, grid.z);
        const long long nbv = (long long)gv.x * gv.y * gv.z;
        if (op.g.n[0] % 4 == 0 && nbv <= c.npart)
        {
            // pairs of half-cells per thread, 16-byte accesses
            if (op.b[0])
                LAUNCH_PDL((k_mg_resid3v<T, true>), gv, 256, c.st, op, x, f, rout, inh ? 1 : 0,
                       both ? 1 : 0, fnorm ? 1 : 0, c.dpart, r32, x32, rscale);
            else
                LAUNCH_PDL((k_mg_resid3v<T, false>), gv, 256, c.st, op, x, f, rout, inh ? 1 : 0,
                       both ? 1 : 0, fnorm ? 1 : 0, c.dpart, r32, x32, rscale);
            LAUNCH_PDL(k_mg_max_partials<T>, 1, 1024, c.st, op, c.dpart, nbv, fnorm ? 1 : 0, mx);
            return;
        }
        if (nb <= c.npart)
        {
            if (op.b[0])
                LAUNCH_PDL((k_mg_resid3<T, true>), grid, 256, c.st, op, x, f, rout, inh ? 1 : 0,
                       both ? 1 : 0, fnorm ? 1 : 0, c.dpart, r32, x32, rscale);
            else
                LAUNCH_PDL((k_mg_resid3<T, false>), grid, 256, c.st, op, x, f, rout, inh ? 1 : 0,
                       both ? 1 : 0, fnorm ? 1 : 0, c.dpart, r32, x32, rscale);
            LAUNCH_PDL(k_mg_max_partials<T>, 1, 1024, c.st, op, c.dpart, nb, fnorm ? 1 : 0, mx);
            return;
        }
    }
    if (op.g.rb)
    {
        const long long half = op.g.ncell() >> 1;
        const long long nb = std::min<long long>((half + 255) / 256, c.npart);
        LAUNCH_PDL(k_mg_resid_norm_rb<T>, dim3((unsigned)nb), 256, c.st, op, x, f, rout,
               inh ? 1 : 0, fnorm ? 1 : 0, c.dpart);
        LAUNCH_PDL(k_mg_max_partials<T>, 1, 1024, c.st, op, c.dpart, nb, fnorm ? 1 : 0, mx);
        return;
    }
    int rows = 8;
    Grid3 gn = rows3(op.g, rows);
    while ((long long)gn.g.x * gn.g.y * gn.g.z > c.npart)
    {
        rows *= 2;
        gn = rows3(op.g, rows);
    }
    const long long nb = (long long)gn.g.x * gn.g.y * gn.g.z;
    LAUNCH_PDL(k_mg_resid_norm<T>, gn.g, gn.b, c.st, op, x, f, rout, mx, inh ? 1 : 0,
           fnorm ? 1 : 0, rows, c.dpart);
    LAUNCH_PDL(k_mg_max_partials<T>, 1, 1024, c.st, op, c.dpart, nb, fnorm ? 1 : 0, mx);
}

template <typename T>
double resid_norm(Ctx& c, const MGOp<T>& op, const T* x, const T* f, T* rout, bool inh,
                  double* fnorm = nullptr)
{
    launch_norm(c, op, x, f, rout, inh, fnorm != nullptr, c.dscal);
    if (fnorm)
    {
        VD_CUDA_OK(cudaMemcpyAsync(c.hscal + 1, c.dscal + 1, sizeof(unsigned long long),
                                   cudaMemcpyDeviceToHost, c.st));
    }
    const double r = read_norm(c);
    if (fnorm) std::memcpy(fnorm, c.hscal + 1, sizeof(double));
    return r;
}

// Boundary data of one solve: hook kernel + conversion to ghost form.
void fill_bc(Ctx& c, int kind, int comp, const int* bct, int maxorder, double scale,
             double time, SideArrays* sides)
{
    for (int s = 0; s < 6; ++s)
    {
        const int d = s % 3;
        if (bct[s] == MG_PER) continue;
        const int np = plane_count(c.g, d);
        const int sgn = (s / 3) ? 1 : -1;
        const double app = (kind == 0) ? applied_potential(c.cfg, time, sgn, d) : 0.0;
        const int udef = (kind == 0) ? c.cfg.user_defined_potential : c.cfg.user_defined_species;
        LAUNCH(k_bc_hook, gsz(np), BS, c.st, c.G, s, kind, comp, c.S, sides[s], time, app, udef,
               c.cfg.gas_temperature, c.cfg.gas_pressure, c.dpp);
        LAUNCH(k_bc_finalize, gsz(np), BS, c.st, np, bct[s], c.g.n[d], maxorder, c.G.dx[d],
               scale, sides[s]);
    }
}

// Level-0 boundary arrays of an FP64 hierarchy point at the side arrays;
// an FP32 hierarchy gets converted copies.
void bind_sides64(Hier<double>& H, SideArrays* sides)
{
    for (int s = 0; s < 6; ++s)
    {
        H.g0[s] = sides[s].g;
        H.c0[0][s] = sides[s].c0;
        H.ra[0][s] = sides[s].ra;
        H.rb[0][s] = sides[s].rb;
    }
}

void bind_sides32(Ctx& c, Hier<float>& H, SideArrays* sides, const int* bct)
{
    for (int s = 0; s < 6; ++s)
    {
        if (bct[s] != MG_ROBIN) continue;
        const int np = plane_count(c.g, s % 3);
        LAUNCH((k_convert<float, double>), gsz(np), BS, c.st, H.c0[0][s], sides[s].c0, 1.0, np);
        LAUNCH((k_convert<float, double>), gsz(np), BS, c.st, H.ra[0][s], sides[s].ra, 1.0, np);
        LAUNCH((k_convert<float, double>), gsz(np), BS, c.st, H.rb[0][s], sides[s].rb, 1.0, np);
    }
}

// Solve L(sol) = rhs on the fine level.  Plain: FP64 V-cycles smoothing the
// solution.  Refined: FP64 residual, FP32 V-cycles on the normalised
// correction, FP64 update; both stop on |r|_inf <= max(abs, rel |r0|_inf).
// `r0_ref` >= 0 replaces the initial residual in the stopping target: a
// solve started from an earlier solution stops where the same solve started
// from the reference's initial guess would (its residual norm is r0_ref).
int mg_solve(Ctx& c, Hier<double>& H64, Hier<float>& H32, double* sol, double* rhs,
             vd_solve_stats* stats, int hint = 1, bool allow32 = true, double r0_ref = -1.0)
{
    const vd_config& cfg = c.cfg;
    double b0 = 0.0;
    const double r0 = resid_norm(c, H64.op[0], sol, rhs, (double*)nullptr, true, &b0);
    // relative to the larger of |rhs| and |r0| (MLMG's "bnorm"/"resid0")
    const double target = std::max(cfg.linsolve_abstol, std::max(cfg.linsolve_reltol, 1e-16) *
                                                            std::max(b0, r0_ref >= 0.0 ? r0_ref : r0));
    vd_solve_stats st{};
    st.initial_residual = r0;
    st.final_residual = r0;
    st.converged = 1;
    if (!(r0 <= target)) // a NaN residual is not converged
    {
        st.converged = 0;
        const bool refined = cfg.mg_precision == VD_MG_FP32_REFINED && allow32;
        if (refined && mg3_ok(H64.op[0]))
        {
            // device-side refinement: each pass is the FP64 residual written
            // as the scaled FP32 right-hand side (with the FP32 unknown
            // zeroed), a device convergence check, `inner` FP32 V-cycles and
            // the FP64 update; passes are enqueued in batches and every
            // kernel returns at once when the stop flag is up
            const long long n = c.N;
            const int inner = std::max(1, cfg.mg_inner_cycles);
            MGDev init{};
            init.sc_cur = 1.0 / r0;
            VD_CUDA_OK(cudaMemcpyAsync(c.dmg, &init, sizeof(MGDev), cudaMemcpyHostToDevice, c.st));
            MGOp<double> op0 = H64.op[0];
            op0.stop = &c.dmg->done;
            for (auto& o : H32.op)
            {
                o.stop = &c.dmg->done;
                o.err = &c.dmg->wait_err;
            }
            int issued = 0;
            int batch = std::max(1, (hint + inner - 1) / inner - 1);
            while (issued * inner < cfg.linsolve_maxiter)
            {
                const int nb = std::min(batch, (cfg.linsolve_maxiter - issued * inner + inner - 1) / inner);
                for (int b = 0; b < nb; ++b)
                {
                    launch_norm(c, op0, (const double*)sol, (const double*)rhs, (double*)nullptr,
                                true, false, &c.dmg->rbits, true, H32.f[0], H32.x[0],
                                &c.dmg->sc_cur);
                    LAUNCH_PDL(k_ref_check, 1, 1, c.st, c.dmg, target);
                    for (int q = 0; q < inner; ++q) vcycle(H32, H32.x[0], H32.f[0], false, c.dscal, c.st);
                    LAUNCH_PDL(k_ref_add, gsz(n), BS, c.st, sol, (const float*)H32.x[0],
                           (const MGDev*)c.dmg, n);
                    LAUNCH_PDL(k_ref_rotate, 1, 1, c.st, c.dmg, inner);
                    ++issued;
                }
                VD_CUDA_OK(cudaMemcpyAsync(c.hmg, c.dmg, sizeof(MGDev), cudaMemcpyDeviceToHost, c.st));
                VD_CUDA_OK(cudaStreamSynchronize(c.st));
                if (c.hmg->done) break;
                batch = 2;
            }
            if (!c.hmg->done)
            {
                // the last pass's update has no residual check yet: take it
                launch_norm(c, op0, (const double*)sol, (const double*)rhs, (double*)nullptr,
                            true, false, &c.dmg->rbits, true, H32.f[0], H32.x[0], &c.dmg->sc_cur);
                LAUNCH_PDL(k_ref_check, 1, 1, c.st, c.dmg, target);
                VD_CUDA_OK(cudaMemcpyAsync(c.hmg, c.dmg, sizeof(MGDev), cudaMemcpyDeviceToHost, c.st));
                VD_CUDA_OK(cudaStreamSynchronize(c.st));
            }
            for (auto& o : H32.op) o.stop = nullptr, o.err = nullptr;
            if (c.hmg->wait_err) throw CudaError("a multigrid kernel's bounded wait gave up");
            st.iterations = c.hmg->iters;
            st.refinements = c.hmg->refs;
            std::memcpy(&st.final_residual, &c.hmg->final_bits, sizeof(double));
            st.converged = c.hmg->done;
        } else if (refined)
        {
            const long long n = c.N;
            double rn = r0;
            // r64 holds f - L(sol)
            resid_norm(c, H64.op[0], sol, rhs, c.r64, true);
            const int inner = std::max(1, cfg.mg_inner_cycles);
            while (st.iterations < cfg.linsolve_maxiter)
            {
                const double s = 1.0 / rn;
                LAUNCH_PDL((k_convert<float, double>), gsz(n), BS, c.st, H32.f[0], c.r64, s, n);
                LAUNCH_PDL(k_fill<float>, gsz(n), BS, c.st, H32.x[0], 0.0f, n);
                for (int q = 0; q < inner; ++q)
                {
                    vcycle(H32, H32.x[0], H32.f[0], false, c.dscal, c.st);
                    ++st.iterations;
                }
                LAUNCH(k_add_scaled<float>, gsz(n), BS, c.st, sol, H32.x[0], rn, n);
                ++st.refinements;
                rn = resid_norm(c, H64.op[0], sol, rhs, c.r64, true);
                st.final_residual = rn;
                if (rn <= target)
                {
                    st.converged = 1;
                    break;
                }
            }
        } else
        {
            // V-cycles are enqueued in batches; each kernel returns at once
            // when the device-side stop flag is up, so the iteration count
            // and result equal those of a cycle-by-cycle host loop
            VD_CUDA_OK(cudaMemsetAsync(c.dmg, 0, sizeof(MGDev), c.st));
            for (auto& o : H64.op)
            {
                o.stop = &c.dmg->done;
                o.err = &c.dmg->wait_err;
            }
            MGOp<double> op0 = H64.op[0];
            // the norm of cycle v's result is taken by the first sweep of
            // cycle v+1 (NormFuse): the check lags one cycle, and a converged
            // solution carries one more colour-0 half-sweep than the cycles
            // counted
            const bool fused = H64.nlev > 1 && H64.nu1 >= 1 && H64.nu2 >= 1 &&
                               norm_fusable(op0, c.npart);
            const NormFuse nf{c.dpart, c.npart, c.dmg, target};
            int issued = 0;
            int batch = fused ? hint + 1 : std::max(1, hint - 1);
            while (issued < cfg.linsolve_maxiter)
            {
                const int nb = std::min(batch, cfg.linsolve_maxiter - issued);
                for (int b = 0; b < nb; ++b)
                {
                    vcycle(H64, sol, rhs, true, c.dscal, c.st, (fused && issued > 0) ? &nf : nullptr);
                    if (!fused)
                    {
                        // the cycle ends with a colour-1 sweep of level 0, whose
                        // cells then have no residual: only colour 0 is scanned
                        launch_norm(c, op0, (const double*)sol, (const double*)rhs,
                                    (double*)nullptr, true, false, &c.dmg->rbits, H64.nu2 < 1);
                        LAUNCH_PDL(k_mg_check, 1, 1, c.st, c.dmg, target);
                    }
                    ++issued;
                }
                VD_CUDA_OK(cudaMemcpyAsync(c.hmg, c.dmg, sizeof(MGDev), cudaMemcpyDeviceToHost, c.st));
                VD_CUDA_OK(cudaStreamSynchronize(c.st));
                if (c.hmg->done) break;
                batch = 2;
            }
            if (fused && !c.hmg->done)
            {
                // the last cycle's result has not been checked yet
                launch_norm(c, op0, (const double*)sol, (const double*)rhs, (double*)nullptr, true,
                            false, &c.dmg->rbits, false);
                LAUNCH_PDL(k_mg_check, 1, 1, c.st, c.dmg, target);
                VD_CUDA_OK(cudaMemcpyAsync(c.hmg, c.dmg, sizeof(MGDev), cudaMemcpyDeviceToHost, c.st));
                VD_CUDA_OK(cudaStreamSynchronize(c.st));
            }
            for (auto& o : H64.op) o.stop = nullptr, o.err = nullptr;
            if (c.hmg->wait_err) throw CudaError("a multigrid kernel's bounded wait gave up");
            st.iterations = c.hmg->iters;
            std::memcpy(&st.final_residual, &c.hmg->final_bits, sizeof(double));
            st.converged = c.hmg->done;
        }
    }
    if (stats) *stats = st;
    if (!st.converged) c.not_converged++;
    return st.iterations;
}

GradCtx grad_ctx(Ctx& c, Hier<double>& H, SideArrays* sides)
{
    GradCtx gc{};
    gc.op = H.op[0];
    for (int d = 0; d < 3; ++d) gc.dxi[d] = 1.0 / c.G.dx[d];
    for (int s = 0; s < 6; ++s) gc.inneu_val[s] = sides[s].val;
    return gc;
}

// ---- solve_potential (Source/PotentialSolve.cpp:19-554)
void poisson(Ctx& c, double time, const double* Sold, vd_solve_stats* stats,
             const double* ephi = nullptr)
{
    const vd_config& cfg = c.cfg;
    const double ps = cfg.potential_scale;
    const bool prof_rhs = t_prof && t_prof->id == VD_PROF_POISSON_RHS;
    if (prof_rhs)
    {
        // reads the charged species (and the coupling source, the last
        // potential when warm), writes the right-hand side and the guess
        int kc[NUM_SPECIES];
        CKCHRG(kc);
        int nq = 0;
        for (int sp = 0; sp < NUM_SPECIES; ++sp) nq += (kc[sp] != 0 && cfg.do_spacechrg) ? 1 : 0;
        const int nin = nq + (ephi ? 1 : 0) + (cfg.poisson_warm_start ? 1 : 0);
        t_prof->bytes = 8.0 * (nin + 2) * (double)c.N;
        t_prof->begin(c.st);
    }
    LAUNCH(k_poisson_rhs, gsz(c.N), BS, c.st, c.G, c.HP.g[0], Sold, c.S, c.phi_rhs, c.phi_sol,
           cfg.do_spacechrg, cfg.poisson_warm_start, ps, time, c.dpp, ephi);
    if (prof_rhs) t_prof->end(c.st);
    fill_bc(c, 0, POT_ID, c.pbct, 2, 1.0 / ps, time, c.pside);
    if (c.HP.varb)
    {
        // electron-Poisson coupling: b = -(1 + dt/tau_diel) on the faces of
        // the coupled solve, b = -1 for a plain one
        for (int d = 0; d < cfg.dim; ++d)
        {
            const long long nf = face_count(c.g, d);
            if (ephi)
                LAUNCH(k_pot_faces, gsz(nf), BS, c.st, c.g, d, (const double*)c.S, c.eidx,
                       cfg.gas_temperature, cfg.dt, c.HP.bf[0][d]);
            else
                LAUNCH(k_fill<double>, gsz(nf), BS, c.st, c.HP.bf[0][d], -1.0, nf);
        }
    }
    hier_set_ops(c.HP, 0.0, 1.0, -1.0, c.pbct, 2);
    hier_coarsen_coeffs(c.HP, c.pbct, c.st);
    if (cfg.mg_precision == VD_MG_FP32_REFINED)
    {
        bind_sides32(c, c.HP32, c.pside, c.pbct);
        hier_set_ops(c.HP32, 0.0, 1.0, -1.0, c.pbct, 2);
        hier_coarsen_coeffs(c.HP32, c.pbct, c.st);
    }
    for (int s = 0; s < 6; ++s)
        if (c.pbct[s] == MG_INNEU)
            LAUNCH(k_inneu_adjust, gsz(plane_count(c.g, s % 3)), BS, c.st, c.HP.g[0], s,
                   (const double*)nullptr, -1.0, 1.0, c.G.dx[s % 3], c.pside[s].val, c.phi_rhs);
    // a warm-started solve keeps the stopping target of the reference's
    // zero-initial-guess solve (Source/PotentialSolve.cpp:479-488): its
    // initial residual |f - L(0)| (inhomogeneous boundaries), one norm pass
    // over an all-zero array
    double r0_zero = -1.0;
    if (cfg.poisson_warm_start && c.zero64)
        r0_zero = resid_norm(c, c.HP.op[0], (const double*)c.zero64, (const double*)c.phi_rhs,
                             (double*)nullptr, true);
    vd_solve_stats st{};
    const int it = mg_solve(c, c.HP, c.HP32, c.phi_sol, c.phi_rhs, &st, c.hint[VD_NT],
                            !c.HP.varb, r0_zero);
    if (st.converged && it > 0) c.hint[VD_NT] = it;
    c.poisson_iters += it;
    c.poisson_refs += st.refinements;
    c.max_poisson_res = std::max(c.max_poisson_res, st.final_residual);
    if (stats) *stats = st;
    const bool prof_ef = t_prof && t_prof->id == VD_PROF_EFIELD;
    if (prof_ef)
    {
        // reads the potential and every species, writes E (dim), E/N and
        // the potential
        t_prof->bytes = 8.0 * (1 + NUM_SPECIES + cfg.dim + 2) * (double)c.N;
        t_prof->begin(c.st);
    }
    if (c.g.n[0] % 2 == 0)
    {
        // two cells per thread, 16-byte state accesses
        const dim3 grid((c.g.n[0] / 2 + 127) / 128, c.g.n[1], c.g.n[2]);
        LAUNCH(k_efield2, grid, 128, c.st, grad_ctx(c, c.HP, c.pside), c.phi_sol, c.S, ps);
        if (prof_ef) t_prof->end(c.st);
    } else
    {
        const Grid3 ge = rows3(c.g);
        LAUNCH(k_efield, ge.g, ge.b, c.st, grad_ctx(c, c.HP, c.pside), c.phi_sol, c.S, ps);
    }
}

// ---- explicit sources of every transported component
// Planes per CTA of k_explicit_stream in z.  A CTA's time grows with its
// planes plus the six halo planes of the z stencil, and the grid runs in
// waves of the CTAs resident on the device, so the chunk count minimises
// waves x (planes + 6): at 256^3 three chunks (2 waves of 32x7-column tiles)
// against eight of 32 planes (5.3 waves), 4.73 -> 4.36 ms of explicit work
// per step.  EX_ZC > 0 fixes the chunk height instead.
int explicit_zchunk(const GridDev& g)
{
    if (EX_ZC > 0) return std::min(EX_ZC, g.n[2]);
    static int resident = 0;
    if (!resident)
    {
        int dev = 0, nsm = 0, per_sm = 0;
        VD_CUDA_OK(cudaGetDevice(&dev));
        VD_CUDA_OK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
        VD_CUDA_OK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_explicit_stream,
                                                                 EX_THREADS, 0));
        resident = std::max(1, per_sm) * nsm;
    }
    const long long tiles =
        (long long)((g.n[0] + EX_TX - 1) / EX_TX) * ((g.n[1] + EX_TY - 1) / EX_TY);
    const int nz = g.n[2];
    int best = nz;
    long long best_cost = -1;
    for (int nch = 1; nch <= nz; ++nch)
    {
        const int zc = (nz + nch - 1) / nch;
        if ((nz + zc - 1) / zc != nch) continue; // same chunking as a smaller count
        const long long waves = (tiles * nch + resident - 1) / resident;
        const long long cost = waves * (zc + 6);
        if (best_cost < 0 || cost < best_cost)
        {
            best_cost = cost;
            best = zc;
        }
    }
    return best;
}

// Launches [qlo, qhi) of the component groups (default: all).  The first
// launch also evaluates the chemistry of every component.
void explicit_rhs(Ctx& c, double time, int qlo = 0, int qhi = 1 << 30)
{
    const vd_config& cfg = c.cfg;
    ExplParams P{};
    P.G = c.G;
    P.S = c.S;
    P.expl = c.expl;
    P.rxn_een = cfg.elecenergy_solve ? c.rxn_een : nullptr;
    P.rxn_e = c.rxn_e;
    P.eidx = c.eidx;
    P.Tg = cfg.gas_temperature;
    P.Pg = cfg.gas_pressure;
    P.time = time;
    P.dt = cfg.dt;
    P.dxmin = c.G.dx[0];
    for (int d = 1; d < cfg.dim; ++d) P.dxmin = std::min(P.dxmin, c.G.dx[d]);
    P.hyp_order = cfg.hyp_order;
    P.weno_scheme = cfg.weno_scheme;
    P.user_vel = cfg.user_defined_vel;
    P.do_transport = cfg.do_transport;
    P.do_reactions = cfg.do_reactions;
    P.do_bg_rxn = cfg.do_bg_reactions;
    P.pp = c.dpp;
    P.rxn_bg = c.rxn_bg;
    int n = 0;
    for (int sp = 0; sp < NUM_SPECIES; ++sp)
    {
        P.bg[sp] = c.bg[sp];
        P.bgslot[sp] = c.bgslot[sp];
        // multicomponent solves take the background species of the neutral
        // range into their chunk (Source/Evolve.cpp:496-533): they need
        // their explicit source like any transported species
        if (c.bg[sp] && !(cfg.multicompsolves && in_neutral_range(sp))) continue;
        P.comp[n] = sp;
        for (int d = 0; d < 3; ++d)
        {
            P.bclo[n][d] = bclo_for(c, sp)[d];
            P.bchi[n][d] = bchi_for(c, sp)[d];
        }
        ++n;
    }
    if (cfg.elecenergy_solve)
    {
        P.comp[n] = EEN_ID;
        for (int d = 0; d < 3; ++d)
        {
            P.bclo[n][d] = cfg.eenrg_bc_lo[d];
            P.bchi[n][d] = cfg.eenrg_bc_hi[d];
        }
        ++n;
    }
    P.ntr = n;
    const bool prof = t_prof && t_prof->id == VD_PROF_EXPLICIT;
    if (prof)
    {
        // inputs: every species, E (3), Te, reduced field (EEN too when it is
        // transported); outputs: one source per non-background component
        // (+ the energy-exchange term)
        const int nin = NUM_SPECIES + 5 + (cfg.elecenergy_solve ? 1 : 0);
        const int nout = NUM_SPECIES + (cfg.elecenergy_solve ? 2 : 0);
        t_prof->bytes = 8.0 * (nin + nout) * (double)c.N;
        t_prof->begin(c.st);
    }
    // streaming kernel: one launch per group of EX_QB components
    const int zc = (cfg.dim == 3) ? explicit_zchunk(c.g) : 1;
    const dim3 grid((c.g.n[0] + EX_TX - 1) / EX_TX, (c.g.n[1] + EX_TY - 1) / EX_TY,
                    (c.g.n[2] + zc - 1) / zc);
    for (int q0 = qlo * EX_QB; q0 < std::min(std::max(n, 1), qhi * EX_QB); q0 += EX_QB)
        LAUNCH(k_explicit_stream, grid, EX_THREADS, c.st, P, q0, zc);
    if (prof) t_prof->end(c.st);
}

// ---- implicit_solve_scalar (Source/ScalarSolve.cpp:380-858)
// FP64 set-up of one species' (or the electron energy's) system into a
// hierarchy H with boundary arrays `sides` and right-hand side `rhs`: face
// diffusivities, scaled right-hand side and initial guess (the current
// state), boundary data from the species_bc hook, operators, coarse
// coefficients, inhomogeneous-Neumann adjustment.
void species_setup64(Ctx& c, int comp, double time, const double* Sold, Hier<double>& H,
                     SideArrays* sides, double* rhs)
{
    const vd_config& cfg = c.cfg;
    const double ts = cfg.time_scale;
    const double scale = (comp == EEN_ID) ? cfg.elecenergy_scale : cfg.species_scale[comp];
    const int* bct = bct_for(c, comp);
    const bool faces3 = [] {
        // VD_SPECIES_FACES3=0: one k_species_faces launch per direction (the
        // same bits; tests compare the two)
        const char* e = std::getenv("VD_SPECIES_FACES3");
        return !(e && e[0] == '0');
    }();
    if (!faces3)
        for (int d = 0; d < cfg.dim; ++d)
            LAUNCH(k_species_faces, gsz(face_count(c.g, d)), BS, c.st, c.g, d, c.S, comp,
                   cfg.gas_temperature, H.bf[0][d]);
    else
    {
        // face coefficients of every direction in one pass (k_species_faces3):
        // 32 x 8 cells a block, z in chunks for about 32 blocks per SM (short
        // marches: 4, 8, 16, 32 blocks per SM measured 31.0, 30.3, 30.2,
        // 30.1 ms per 192^3 LMEA step against 32.3 ms for one launch per
        // direction; the 256^3 Townsend step, whose ion diffusivity is a
        // constant, within 0.05 ms either way)
        const int gx = (c.g.n[0] + 31) / 32, gy = (c.g.n[1] + 7) / 8, nz = c.g.n[2];
        const int chunks =
            std::max(1, std::min(nz, (32 * sm_count() + gx * gy - 1) / (gx * gy)));
        const int kchunk = (nz + chunks - 1) / chunks;
        LAUNCH(k_species_faces3, dim3(gx, gy, (nz + kchunk - 1) / kchunk), 256, c.st, c.g, c.S,
               comp, cfg.gas_temperature, kchunk, H.bf[0][0],
               cfg.dim > 1 ? H.bf[0][1] : (double*)nullptr,
               cfg.dim > 2 ? H.bf[0][2] : (double*)nullptr);
    }
    const bool prof_srhs = t_prof && t_prof->id == VD_PROF_SPECIES_RHS;
    if (prof_srhs)
    {
        // reads the old and current density and the explicit source, writes
        // the right-hand side and the initial guess
        t_prof->bytes = 8.0 * 5 * (double)c.N;
        t_prof->begin(c.st);
    }
    LAUNCH(k_species_rhs, gsz(c.N), BS, c.st, c.g, H.g[0], c.S, Sold, c.expl, comp, cfg.dt,
           ts, scale, rhs, c.u[comp]);
    if (prof_srhs) t_prof->end(c.st);
    fill_bc(c, 1, comp, bct, 3, 1.0 / scale, time, sides);
    hier_set_ops(H, (1.0 / cfg.dt) * ts * 1.0, ts, 1.0, bct, 3);
    hier_coarsen_coeffs(H, bct, c.st);
    for (int s = 0; s < 6; ++s)
        if (bct[s] == MG_INNEU)
            LAUNCH(k_inneu_adjust, gsz(plane_count(c.g, s % 3)), BS, c.st, H.g[0], s,
                   (const double*)H.bf[0][s % 3], 1.0, ts, c.G.dx[s % 3], sides[s].val, rhs);
}

void species_solve(Ctx& c, int comp, double time, const double* Sold, vd_solve_stats* stats)
{
    const vd_config& cfg = c.cfg;
    const double ts = cfg.time_scale;
    const int* bct = bct_for(c, comp);
    species_setup64(c, comp, time, Sold, c.HS, c.sside, c.spec_rhs);
    if (cfg.mg_precision == VD_MG_FP32_REFINED)
    {
        for (int d = 0; d < cfg.dim; ++d)
        {
            const long long nf = face_count(c.g, d);
            LAUNCH((k_convert<float, double>), gsz(nf), BS, c.st, c.HS32.bf[0][d], c.HS.bf[0][d],
                   1.0, nf);
        }
        bind_sides32(c, c.HS32, c.sside, bct);
        hier_set_ops(c.HS32, (1.0 / cfg.dt) * ts * 1.0, ts, 1.0, bct, 3);
        hier_coarsen_coeffs(c.HS32, bct, c.st);
    }
    vd_solve_stats st{};
    // species solves run in FP64 unless the last one needed more than two
    // V-cycles: the implicit-diffusion operator is strongly diagonal (one
    // cycle from the current state in every benchmark configuration), and a
    // refinement pass of mg_inner_cycles FP32 cycles would cost more than the
    // one FP64 cycle it replaces; a refined solve records its inner-cycle
    // count, which keeps a genuinely hard species solve in the refined form
    const bool allow32 = c.hint[comp] > 2;
    const int it = mg_solve(c, c.HS, c.HS32, c.u[comp], c.spec_rhs, &st, c.hint[comp], allow32);
    if (st.converged && it > 0) c.hint[comp] = it;
    c.species_iters += it;
    if (stats) *stats = st;
}

// One multicomponent solve of species [first, first + nc) (MLMG with
// ncomp = nc, Source/ScalarSolve.cpp:540-875): each component is set up in
// its own chunk slot and smoothed, restricted and prolonged on its own; the
// stopping test takes the max-norm over all components and the bottom
// BiCGStab runs jointly in a thread-block cluster of nc CTAs
// (k_mg_coarse3_joint).  FP64 in both precision forms.  Cycles are enqueued
// one at a time with the joint norm read back after each.
void joint_solve(Ctx& c, int first, int nc, double time, const double* Sold,
                 vd_solve_stats* stats)
{
    const vd_config& cfg = c.cfg;
    if (nc > (int)c.HJ.size())
        throw CudaError("multicomponent chunk larger than the slots made at vd_create");
    for (int q = 0; q < nc; ++q)
    {
        species_setup64(c, first + q, time, Sold, c.HJ[q], c.JS[q].data(), c.JR[q]);
        for (auto& o : c.HJ[q].op) o.stop = nullptr;
    }
    Hier<double>& H0 = c.HJ[0];
    const int lc = vcycle_lc(H0);
    size_t smem3 = 0;
    if (H0.nlev < 2 || lc == H0.nlev - 1 || !coarse3_ok(H0, lc, &smem3) ||
        H0.g[H0.nlev - 1].ncell() > 32)
        throw UnsupportedError("multicomponent solves of more than one component need a 3-D, "
                               "non-periodic grid whose coarsest multigrid level holds at most "
                               "32 cells");
    auto norms = [&](double* bmax) {
        double r = 0.0, b = 0.0;
        for (int q = 0; q < nc; ++q)
        {
            double bq = 0.0;
            const double rq = resid_norm(c, c.HJ[q].op[0], (const double*)c.u[first + q],
                                         (const double*)c.JR[q], (double*)nullptr, true,
                                         bmax ? &bq : nullptr);
            r = nanmax(r, rq);
            b = nanmax(b, bq);
        }
        if (bmax) *bmax = b;
        return r;
    };
    double b0 = 0.0;
    const double r0 = norms(&b0);
    const double target =
        std::max(cfg.linsolve_abstol, std::max(cfg.linsolve_reltol, 1e-16) * std::max(b0, r0));
    vd_solve_stats st{};
    st.initial_residual = st.final_residual = r0;
    st.converged = r0 <= target;
    if (!st.converged)
    {
        for (int q = 0; q < nc; ++q) c.hcoarse[q] = coarse_of(c.HJ[q], lc);
        VD_CUDA_OK(cudaMemcpyAsync(c.dcoarse, c.hcoarse, nc * sizeof(MGCoarse<double>),
                                   cudaMemcpyHostToDevice, c.st));
        for (int it = 1; it <= cfg.linsolve_maxiter; ++it)
        {
            for (int q = 0; q < nc; ++q)
                vcycle_down(c.HJ[q], c.u[first + q], c.JR[q], true, c.st, nullptr, lc);
            cudaLaunchConfig_t lcfg{};
            lcfg.gridDim = dim3(nc);
            lcfg.blockDim = dim3(MGC_THREADS);
            lcfg.dynamicSmemBytes = smem3;
            lcfg.stream = c.st;
            cudaLaunchAttribute at[1];
            at[0].id = cudaLaunchAttributeClusterDimension;
            at[0].val.clusterDim.x = nc;
            at[0].val.clusterDim.y = 1;
            at[0].val.clusterDim.z = 1;
            lcfg.attrs = at;
            lcfg.numAttrs = 1;
            VD_CUDA_OK(cudaLaunchKernelEx(&lcfg, k_mg_coarse3_joint<double, true>,
                                          (const MGCoarse<double>*)c.dcoarse, H0.bot_rel,
                                          H0.bot_maxiter, H0.nu1, H0.nu2, H0.nub, H0.nuf));
            ++vd::g_launches;
            for (int q = 0; q < nc; ++q)
                vcycle_up(c.HJ[q], c.u[first + q], c.JR[q], true, c.st, lc);
            st.iterations = it;
            st.final_residual = norms(nullptr);
            if (st.final_residual <= target)
            {
                st.converged = 1;
                break;
            }
        }
    }
    c.species_iters += st.iterations;
    if (!st.converged) c.not_converged++;
    if (stats) *stats = st;
}

void joule(Ctx& c)
{
    JouleParams P{};
    P.pot = grad_ctx(c, c.HP, c.pside);
    P.phi_sol = c.phi_sol;
    P.ps = c.cfg.potential_scale;
    P.ue = c.u[c.eidx];
    P.gm = c.HS.g[0];
    P.escale = c.cfg.species_scale[c.eidx];
    P.S = c.S;
    P.expl = c.expl;
    P.ejh = c.ejh;
    for (int d = 0; d < 3; ++d) P.dx[d] = c.G.dx[d];
    P.Tg = c.cfg.gas_temperature;
    P.floor_jh = c.cfg.floor_jh;
    P.eidx = c.eidx;
    for (int d = 0; d < c.cfg.dim; ++d)
        LAUNCH(k_joule_faces, gsz(face_count(c.g, d)), BS, c.st, P, d, c.jface[d]);
    LAUNCH(k_joule_sum, gsz(c.N), BS, c.st, P, c.jface[0], c.jface[1], c.jface[2]);
}

FinalParams final_params(Ctx& c)
{
    FinalParams P{};
    P.g = c.g;
    P.S = c.S;
    P.bound_specden = c.cfg.bound_specden;
    P.min_e = c.cfg.min_electron_density;
    P.min_s = c.cfg.min_species_density;
    P.min_te = c.cfg.min_electron_temp;
    P.eidx = c.eidx;
    P.Tg = c.cfg.gas_temperature;
    P.ejh = c.ejh;
    P.rxn_een = c.rxn_een;
    P.expl = c.expl;
    P.dt = c.cfg.dt;
    P.gm = c.HS.g[0];
    for (int sp = 0; sp < NUM_SPECIES; ++sp) P.bg[sp] = c.bg[sp];
    return P;
}

void add_solved(Ctx& c, FinalParams& P, int comp)
{
    P.comp[P.nsol] = comp;
    P.u[P.nsol] = c.u[comp];
    P.scale[P.nsol] = (comp == EEN_ID) ? c.cfg.elecenergy_scale : c.cfg.species_scale[comp];
    P.nsol++;
}

// The species solves of one corrector iteration with multicompsolves: ions
// then neutrals in chunks (Source/Evolve.cpp:458-533); background species
// take part and their solutions are dropped (k_finalize resets them).
void multicomp_species(Ctx& c, FinalParams& P, double t, const double* Sold)
{
    auto run = [&](int first, int num, int chunk) {
        for (const auto& ch : chunk_list(first, num, chunk))
        {
            if (ch.second == 1)
                species_solve(c, ch.first, t, Sold, nullptr);
            else
                joint_solve(c, ch.first, ch.second, t, Sold, nullptr);
            for (int q = 0; q < ch.second; ++q)
                if (!c.bg[ch.first + q]) add_solved(c, P, ch.first + q);
        }
    };
    if (NUM_IONS > 0) run(FIRST_ION, NUM_IONS, c.ion_chunk);
    if (NUM_NEUTRALS > 0) run(FIRST_NEUTRAL, NUM_NEUTRALS, c.neutral_chunk);
    P.Sold = Sold;
    P.rxn_bg = c.rxn_bg;
    for (int sp = 0; sp < NUM_SPECIES; ++sp) P.bgslot[sp] = c.bgslot[sp];
}


// ---- one coarse step (Source/Evolve.cpp:136-617)
// ---- find_time_scales + ComputeDt (Source/TimeStep.cpp:14-134): the
// electron drift, diffusion and dielectric-relaxation time scales of the
// current state, and the step size they give.  Sets c.cfg.dt.
void compute_dt(Ctx& c)
{
    const vd_config& cfg = c.cfg;
    const double big = std::numeric_limits<double>::max();
    const int nb = (int)std::min<long long>((c.N + 255) / 256, 4 * 148);
    LAUNCH(k_time_scales, nb, 256, c.st, c.g, (const double*)c.S, c.eidx, cfg.gas_temperature,
           c.dpart);
    LAUNCH(k_time_scales_final, 1, 256, c.st, (const double*)c.dpart, nb, c.dts);
    VD_CUDA_OK(cudaMemcpyAsync(c.hts, c.dts, 3 * sizeof(double), cudaMemcpyDeviceToHost, c.st));
    VD_CUDA_OK(cudaStreamSynchronize(c.st));
    const double max_edriftvel = c.hts[0], max_ediff = c.hts[1], max_muene = c.hts[2];
    double dt_edrift = big, dt_ediff = big, dt_diel_relax = big;
    if (max_edriftvel > 0)
        for (int d = 0; d < cfg.dim; ++d) dt_edrift = std::min(dt_edrift, c.G.dx[d] / max_edriftvel);
    if (max_ediff > 0)
        for (int d = 0; d < cfg.dim; ++d)
            dt_ediff = std::min(dt_ediff, 0.5 * c.G.dx[d] * c.G.dx[d] / max_ediff / cfg.dim);
    if (max_muene > 0) dt_diel_relax = EPS0 / ECHARGE / max_muene;
    c.tscale[0] = dt_edrift;
    c.tscale[1] = dt_ediff;
    c.tscale[2] = dt_diel_relax;
    if (cfg.adaptive_dt && c.time > cfg.adaptive_dt_delay)
    {
        const double old_dt = cfg.dt;
        double trans_min_dt = big;
        if (cfg.do_transport)
            trans_min_dt = std::min(dt_edrift * cfg.advective_cfl, dt_ediff * cfg.diffusive_cfl);
        double adp_dt = std::min(trans_min_dt, dt_diel_relax * cfg.dielectric_cfl);
        if (adp_dt > cfg.dt_max) adp_dt = cfg.dt_max;
        if (adp_dt < cfg.dt_min) adp_dt = cfg.dt_min;
        c.cfg.dt = std::min(old_dt * cfg.dt_stretch, adp_dt);
    } else
        c.cfg.dt = c.fixed_dt;
}

void step_once(Ctx& c)
{
    if (c.cfg.adaptive_dt)
        compute_dt(c);
    else
        c.cfg.dt = c.fixed_dt;
    const vd_config& cfg = c.cfg;
    const double dt = cfg.dt;
    const int ncorr = std::max(1, cfg.num_timestep_correctors);
    const size_t bytes = sizeof(double) * (size_t)NVAR * c.N;
    const bool own_old = ncorr > 1 || cfg.electron_poisson_coupling;
    if (own_old) VD_CUDA_OK(cudaMemcpyAsync(c.Sold, c.S, bytes, cudaMemcpyDeviceToDevice, c.st));
    const double* Sold = own_old ? c.Sold : c.S;
    for (int niter = 0; niter < ncorr; ++niter)
    {
        const double t = c.time + ((niter > 0) ? 0.5 * dt : 0.0);
        FinalParams P = final_params(c);
        if (!cfg.electron_poisson_coupling)
        {
            poisson(c, t, Sold, nullptr);
            explicit_rhs(c, t);
            species_solve(c, c.eidx, t, Sold, nullptr);
        } else
        {
            // electron solve first, then the potential with the electron
            // density change (Source/Evolve.cpp:281-352); the electron
            // component is the first group launch, which also evaluates the
            // chemistry that the later launches read back
            for (int it = 0; it < std::max(1, cfg.electron_poisson_maxiters); ++it)
            {
                explicit_rhs(c, t, 0, 1);
                species_solve(c, c.eidx, t, Sold, nullptr);
                LAUNCH(k_ephi, gsz(c.N), BS, c.st, c.g, c.HS.g[0], c.S, Sold,
                       (const double*)c.u[c.eidx], cfg.species_scale[c.eidx],
                       (const double*)c.expl, (const double*)c.rxn_e, c.eidx,
                       cfg.bound_specden, cfg.min_electron_density, dt, c.ephi);
                poisson(c, t, Sold, nullptr, c.ephi);
            }
            explicit_rhs(c, t, 1);
        }
        add_solved(c, P, c.eidx);
        if (cfg.elecenergy_solve)
        {
            joule(c);
            species_solve(c, EEN_ID, t, Sold, nullptr);
            add_solved(c, P, EEN_ID);
            P.een_solved = 1;
            P.heat_diag = 1;
        }
        P.lfa = cfg.using_LFA;
        if (cfg.multicompsolves)
            multicomp_species(c, P, t, Sold);
        else
            for (int sp = 0; sp < NUM_SPECIES; ++sp)
            {
                if (c.bg[sp] || sp == c.eidx) continue;
                species_solve(c, sp, t, Sold, nullptr);
                add_solved(c, P, sp);
            }
        P.do_bg_rxn = cfg.do_bg_reactions;
        LAUNCH(k_finalize, gsz(c.N), BS, c.st, P);
        if (niter < ncorr - 1)
            LAUNCH(k_midpoint, gsz((long long)NVAR * c.N), BS, c.st, c.S, c.Sold,
                   (long long)NVAR * c.N);
    }
    c.time += dt;
    c.step += 1;
}

__global__ void k_initdomain(Geo G, double* S, const ProbParm* pp)
{
    VD_PDL_WAIT();
    const long long N = G.g.ncell();
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < N;
         t += (long long)gridDim.x * blockDim.x)
    {
        int i, j, k;
        cell_of(G.g, t, i, j, k);
        vd::Array4 v = state_view(S, G.g);
        v.clamp = 0;
        vd::GeometryData gd;
        for (int d = 0; d < 3; ++d)
        {
            gd.prob_lo[d] = G.plo[d];
            gd.prob_hi[d] = G.phi[d];
            gd.dx[d] = G.dx[d];
            gd.n_cell[d] = G.g.n[d];
        }
        vd::Box bx{{i, j, k}, {i, j, k}};
        // a reference Prob.H takes a non-const ProbParm* (it only reads it)
        initdomaindata(bx, v, gd, const_cast<ProbParm*>(pp));
    }
}

// ---------------------------------------------------------- config I/O
struct Key
{
    const char* name;
    int kind; // 0 int, 1 double, 2 int[3], 3 double[3]
    size_t off;
};

#define KI(n, f) {n, 0, offsetof(vd_config, f)}
#define KD(n, f) {n, 1, offsetof(vd_config, f)}
#define KI3(n, f) {n, 2, offsetof(vd_config, f)}
#define KD3(n, f) {n, 3, offsetof(vd_config, f)}

const Key g_keys[] = {
    KI3("amr.n_cell", n_cell), KD3("geometry.prob_lo", prob_lo), KD3("geometry.prob_hi", prob_hi),
    KI3("geometry.is_periodic", is_periodic), KD("vidyut.dt", dt),
    KI("vidyut.num_timestep_correctors", num_timestep_correctors),
    KI("vidyut.electron_poisson_coupling", electron_poisson_coupling),
    KI("vidyut.electron_poisson_maxiters", electron_poisson_maxiters),
    KI("vidyut.adaptive_dt", adaptive_dt), KD("vidyut.advective_cfl", advective_cfl),
    KD("vidyut.diffusive_cfl", diffusive_cfl), KD("vidyut.dielectric_cfl", dielectric_cfl),
    KD("vidyut.dt_min", dt_min), KD("vidyut.dt_max", dt_max),
    KD("vidyut.adaptive_dt_delay", adaptive_dt_delay), KD("vidyut.dt_stretch", dt_stretch),
    KI("vidyut.hyp_order", hyp_order), KI("vidyut.weno_scheme", weno_scheme),
    KI("vidyut.do_reactions", do_reactions), KI("vidyut.do_transport", do_transport),
    KI("vidyut.do_spacechrg", do_spacechrg), KI("vidyut.elecenergy_solve", elecenergy_solve),
    KI("vidyut.using_LFA", using_LFA), KI("vidyut.floor_jh", floor_jh),
    KI("vidyut.bound_specden", bound_specden), KI("vidyut.do_bg_reactions", do_bg_reactions),
    KI("vidyut.user_defined_potential", user_defined_potential),
    KI("vidyut.user_defined_species", user_defined_species),
    KI("vidyut.user_defined_vel", user_defined_vel),
    KD("vidyut.min_species_density", min_species_density),
    KD("vidyut.min_electron_density", min_electron_density),
    KD("vidyut.min_electron_temp", min_electron_temp),
    KD("vidyut.gas_temperature", gas_temperature), KD("vidyut.gas_pressure", gas_pressure),
    KI3("vidyut.pot_bc_lo", pot_bc_lo), KI3("vidyut.pot_bc_hi", pot_bc_hi),
    KI3("vidyut.eden_bc_lo", eden_bc_lo), KI3("vidyut.eden_bc_hi", eden_bc_hi),
    KI3("vidyut.eenrg_bc_lo", eenrg_bc_lo), KI3("vidyut.eenrg_bc_hi", eenrg_bc_hi),
    KI3("vidyut.ion_bc_lo", ion_bc_lo), KI3("vidyut.ion_bc_hi", ion_bc_hi),
    KI3("vidyut.neutral_bc_lo", neutral_bc_lo), KI3("vidyut.neutral_bc_hi", neutral_bc_hi),
    KI("vidyut.voltage_profile", voltage_profile),
    KD3("vidyut.voltage_amp_lo", voltage_amp_lo), KD3("vidyut.voltage_amp_hi", voltage_amp_hi),
    KD("vidyut.voltage_freq", voltage_freq), KD("vidyut.voltage_dur", voltage_dur),
    KD("vidyut.voltage_center", voltage_center),
    KD("vidyut.linsolve_reltol", linsolve_reltol), KD("vidyut.linsolve_abstol", linsolve_abstol),
    KD("vidyut.linsolve_bot_reltol", linsolve_bot_reltol),
    KD("vidyut.linsolve_bot_abstol", linsolve_bot_abstol),
    KI("vidyut.linsolve_num_pre_smooth", linsolve_num_pre_smooth),
    KI("vidyut.linsolve_num_post_smooth", linsolve_num_post_smooth),
    KI("vidyut.linsolve_num_final_smooth", linsolve_num_final_smooth),
    KI("vidyut.linsolve_num_bottom_smooth", linsolve_num_bottom_smooth),
    KI("vidyut.linsolve_maxiter", linsolve_maxiter),
    KI("vidyut.linsolve_max_coarsening_level", linsolve_max_coarsening_level),
    KD("vidyut.potential_scale", potential_scale), KD("vidyut.elecenergy_scale", elecenergy_scale),
    KD("vidyut.time_scale", time_scale), KI("vidyut.mg_precision", mg_precision),
    KI("vidyut.mg_inner_cycles", mg_inner_cycles),
    KI("vidyut.poisson_warm_start", poisson_warm_start), KI("vidyut.device", device),
    KI("vidyut.multicompsolves", multicompsolves), KI("vidyut.comp_ion_chunks", comp_ion_chunks),
    KI("vidyut.comp_neutral_chunks", comp_neutral_chunks),
};


// ---- discrete adjoint of N explicit flux + source steps (vd_adjoint.cuh)
struct AdjState
{
    Alloc A;
    int nt = 0;                 // transported species
    int spec[NUM_SPECIES] = {}; // their components, ascending
    int eslot = -1;
    std::vector<double*> slot;  // state slots, nt x N each
    double* mu = nullptr;
    double* dmu = nullptr;
    double* lam = nullptr;
    double* adj = nullptr;
    double* adjnd = nullptr;
    double* theta = nullptr; // device log pre-factor shifts
    double* acc = nullptr;   // [0] J, [1..R] dJ/dtheta_r, [R+1] dJ/dscale
    double* opart = nullptr; // per-block double-double partials of the objective
    double* hacc = nullptr;  // pinned mirror of acc
    std::vector<double> params; // theta_0 .. theta_{R-1}, electron mobility scale
    ~AdjState()
    {
        A.release();
        if (hacc) cudaFreeHost(hacc);
    }
};

#ifdef VD_HAS_MECH_ADJOINT
constexpr int ADJ_NR = NUM_REACTIONS;

dim3 gsz128(long long n)
{
    long long b = (n + 127) / 128;
    if (b < 1) b = 1;
    if (b > 148LL * 64) b = 148LL * 64;
    return dim3((unsigned)b);
}

// Segments a line for the line-march kernels (128-thread blocks, one thread
// per segment of a line and species): whole lines leave the launch's last
// wave part-empty (128^3, 7 species: 3.03 waves of the face adjoint at 2
// blocks per SM), shorter segments fill it at the cost of the faces a
// segment forms twice or the window it loads first.  Model: waves x (faces
// a segment + 1) at the occupancy the kernel reaches; VD_ADJ_LINE_SEGMENTS
// fixes the count (tests).
template <typename K>
int line_segments(K kernel, long long lines, int nf)
{
    if (const char* e = std::getenv("VD_ADJ_LINE_SEGMENTS"))
        return std::max(1, std::atoi(e));
    int occ = 0;
    VD_CUDA_OK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kernel, 128, 0));
    const double slots = (double)std::max(occ, 1) * sm_count() * 128;
    int best = 1;
    double bc = 1e300;
    for (int S = 1; S <= 8; ++S)
    {
        const double cost = std::ceil((double)lines * S / slots) * ((double)nf / S + 1.0);
        if (cost < bc * (1.0 - 1e-9))
        {
            bc = cost;
            best = S;
        }
    }
    return best;
}

AdjState& adj_state(Ctx& c, int slots)
{
    const long long N = c.N;
    if (!c.adjs)
    {
        AdjState* a = new AdjState();
        c.adjs = a;
        for (int sp = 0; sp < NUM_SPECIES; ++sp)
            if (!c.bg[sp])
            {
                if (sp == c.eidx) a->eslot = a->nt;
                a->spec[a->nt++] = sp;
            }
        if (a->eslot < 0) throw CudaError("the electrons are a background species");
        a->mu = a->A.get<double>((size_t)a->nt * N);
        a->dmu = a->A.get<double>((size_t)a->nt * N);
        a->lam = a->A.get<double>((size_t)a->nt * N);
        a->adj = a->A.get<double>((size_t)a->nt * N);
        a->adjnd = a->A.get<double>(N);
        a->theta = a->A.get<double>(ADJ_NR);
        a->acc = a->A.get<double>(ADJ_NR + 2);
        a->opart = a->A.get<double>(2 * (size_t)gsz(N).x);
        VD_CUDA_OK(cudaMallocHost(&a->hacc, sizeof(double) * (ADJ_NR + 2)));
        a->params.assign(ADJ_NR + 1, 0.0);
        a->params[ADJ_NR] = 1.0;
    }
    AdjState& a = *c.adjs;
    while ((int)a.slot.size() < slots) a.slot.push_back(a.A.get<double>((size_t)a.nt * N));
    return a;
}

AdjParams adj_params(Ctx& c, AdjState& a)
{
    AdjParams P{};
    P.g = c.g;
    P.g.rb = 0;
    for (int d = 0; d < 3; ++d) P.dx[d] = c.G.dx[d];
    P.dt = c.cfg.dt;
    P.dxmin = c.G.dx[0];
    for (int d = 1; d < c.cfg.dim; ++d) P.dxmin = std::min(P.dxmin, c.G.dx[d]);
    P.Tg = c.cfg.gas_temperature;
    P.mob_scale = a.params[ADJ_NR];
    P.hyp_order = c.cfg.hyp_order;
    P.weno_scheme = c.cfg.weno_scheme;
    P.nt = a.nt;
    P.eslot = a.eslot;
    for (int s = 0; s < a.nt; ++s)
    {
        P.spec[s] = a.spec[s];
        for (int d = 0; d < 3; ++d)
        {
            P.bclo[s][d] = bclo_for(c, a.spec[s])[d];
            P.bchi[s][d] = bchi_for(c, a.spec[s])[d];
        }
    }
    P.S = c.S;
    P.theta = a.theta;
    P.mu = a.mu;
    P.dmu = a.dmu;
    return P;
}

void adj_step(Ctx& c, const AdjParams& P, const double* from, double* to)
{
    LAUNCH(k_adj_props, gsz(c.N), BS, c.st, P, from);
    // chemistry, then one line march per direction with each face flux
    // formed once; VD_ADJ_STEP_LINE=0 keeps one thread per cell forming
    // both of its faces (k_adj_step; tests compare the two)
    const char* e = std::getenv("VD_ADJ_STEP_LINE");
    if (e && e[0] == '0')
    {
        LAUNCH(k_adj_step, gsz(c.N), BS, c.st, P, from, to);
        return;
    }
    LAUNCH(k_adj_chem_step, gsz(c.N), BS, c.st, P, from, to);
    for (int d = 0; d < c.cfg.dim; ++d)
    {
        const long long lines = c.N / c.g.n[d] * P.nt;
        const int nseg = line_segments(k_adj_flux_line, lines, c.g.n[d] + 1);
        LAUNCH(k_adj_flux_line, gsz128(lines * nseg), 128, c.st, P, d, nseg, from, to);
    }
}

double adj_cell_volume(const Ctx& c)
{
    double dv = 1.0;
    for (int d = 0; d < c.cfg.dim; ++d) dv *= c.G.dx[d];
    return dv;
}

// Forward sweep from the state's transported species.  With K > 0 the state
// at every step k = bK is kept in slot b; the objective is added into acc[0].
// Returns the slot holding the final state.
double* adj_forward(Ctx& c, AdjState& a, const AdjParams& P, int nsteps, int K)
{
    const long long N = c.N;
    const int nck = (K > 0) ? (nsteps + K - 1) / K : 1;
    double* w[2] = {a.slot[nck], a.slot[nck + 1]};
    double* cur = a.slot[0];
    for (int s = 0; s < a.nt; ++s)
        VD_CUDA_OK(cudaMemcpyAsync(cur + (size_t)s * N, c.S + (size_t)a.spec[s] * N,
                                   sizeof(double) * N, cudaMemcpyDeviceToDevice, c.st));
    for (int k = 0; k < nsteps; ++k)
    {
        double* nxt;
        if (K > 0 && (k + 1) % K == 0 && k + 1 < nsteps)
            nxt = a.slot[(k + 1) / K];
        else
            nxt = (cur == w[0]) ? w[1] : w[0];
        adj_step(c, P, cur, nxt);
        cur = nxt;
    }
    const dim3 gob = gsz(N);
    LAUNCH(k_adj_objective, gob, BS, c.st, N, cur + (size_t)a.eslot * N, a.opart);
    LAUNCH(k_adj_objective_final, 1, 1024, c.st, (int)gob.x, (const double*)a.opart,
           adj_cell_volume(c), a.acc);
    return cur;
}

void adj_read_acc(Ctx& c, AdjState& a)
{
    VD_CUDA_OK(cudaMemcpyAsync(a.hacc, a.acc, sizeof(double) * (ADJ_NR + 2),
                               cudaMemcpyDeviceToHost, c.st));
    VD_CUDA_OK(cudaStreamSynchronize(c.st));
}

void adj_upload(Ctx& c, AdjState& a)
{
    VD_CUDA_OK(cudaMemcpyAsync(a.theta, a.params.data(), sizeof(double) * ADJ_NR,
                               cudaMemcpyHostToDevice, c.st));
    VD_CUDA_OK(cudaMemsetAsync(a.acc, 0, sizeof(double) * (ADJ_NR + 2), c.st));
}

// Gradient of the objective by the backward sweep: checkpoints every K steps,
// the states of each K-block recomputed from its checkpoint.
void adj_run(Ctx& c, int nsteps, int K)
{
    const long long N = c.N;
    const int nck = (nsteps + K - 1) / K;
    const int ntraj = std::max(K, 2);
    AdjState& a = adj_state(c, nck + ntraj);
    const AdjParams P = adj_params(c, a);
    adj_upload(c, a);
    adj_forward(c, a, P, nsteps, K);
    // lambda = dJ/du at the last step: dV on the electrons
    VD_CUDA_OK(cudaMemsetAsync(a.lam, 0, sizeof(double) * (size_t)a.nt * N, c.st));
    LAUNCH(k_fill<double>, gsz(N), BS, c.st, a.lam + (size_t)a.eslot * N, adj_cell_volume(c), N);
    // WENO faces by line march (k_adj_faces_line); VD_ADJ_FACES_LINE=0 keeps
    // one thread per face (k_adj_faces; tests compare the two)
    const char* le = std::getenv("VD_ADJ_FACES_LINE");
    const bool line_faces = P.hyp_order > 2 && !(le && le[0] == '0');
    std::vector<double*> t(ntraj);
    for (int b = nck - 1; b >= 0; --b)
    {
        const int k0 = b * K, k1 = std::min(nsteps, k0 + K);
        t[0] = a.slot[b];
        for (int i = 1; i < k1 - k0; ++i)
        {
            t[i] = a.slot[nck + i];
            adj_step(c, P, t[i - 1], t[i]);
        }
        for (int k = k1 - 1; k >= k0; --k)
        {
            const double* uk = t[k - k0];
            LAUNCH(k_adj_props, gsz(N), BS, c.st, P, uk);
            VD_CUDA_OK(cudaMemsetAsync(a.adj, 0, sizeof(double) * (size_t)a.nt * N, c.st));
            VD_CUDA_OK(cudaMemsetAsync(a.adjnd, 0, sizeof(double) * N, c.st));
            for (int d = 0; d < c.cfg.dim; ++d)
            {
                if (line_faces)
                {
                    const long long lines = N / c.g.n[d] * a.nt;
                    const int nseg = line_segments(k_adj_faces_line, lines, c.g.n[d] + 1);
                    LAUNCH(k_adj_faces_line, gsz128(lines * nseg), 128, c.st, P, d, nseg, uk,
                           a.lam, a.adj, a.adjnd, a.acc + 1 + ADJ_NR);
                    continue;
                }
                const long long nf = N / c.g.n[d] * (c.g.n[d] + 1);
                LAUNCH(k_adj_faces, gsz128(nf), 128, c.st, P, d, uk, a.lam, a.adj, a.adjnd,
                       a.acc + 1 + ADJ_NR);
            }
            LAUNCH(k_adj_chem_update, gsz128(N), 128, c.st, P, uk, a.lam, a.adj, a.adjnd,
                   a.acc + 1);
        }
    }
    adj_read_acc(c, a);
}
#endif // VD_HAS_MECH_ADJOINT

} // namespace

// ================================================================ C ABI
extern "C" {

vd_status vd_config_init(vd_config* c)
{
    if (!c) return VD_ERR_INVALID_ARG;
    std::memset(c, 0, sizeof(*c));
    c->dim = 3;
    for (int d = 0; d < 3; ++d)
    {
        c->n_cell[d] = 32;
        c->prob_hi[d] = 1.0;
        c->pot_bc_lo[d] = c->pot_bc_hi[d] = HNEUBC;
        c->eden_bc_lo[d] = c->eden_bc_hi[d] = HNEUBC;
        c->eenrg_bc_lo[d] = c->eenrg_bc_hi[d] = HNEUBC;
        c->ion_bc_lo[d] = c->ion_bc_hi[d] = HNEUBC;
        c->neutral_bc_lo[d] = c->neutral_bc_hi[d] = HNEUBC;
    }
    c->dt = 1e-12;
    c->num_timestep_correctors = 1;
    // Source/Vidyut.H:251-262
    c->electron_poisson_coupling = 0;
    c->electron_poisson_maxiters = 1;
    c->adaptive_dt = 0;
    c->advective_cfl = 0.7;
    c->diffusive_cfl = 1.0;
    c->dielectric_cfl = 1.0;
    c->dt_min = 1e-14;
    c->dt_max = 1e-9;
    c->adaptive_dt_delay = 0.0;
    c->dt_stretch = std::numeric_limits<double>::max();
    c->hyp_order = 1;
    c->weno_scheme = 3;
    c->do_reactions = 1;
    c->do_transport = 1;
    c->do_spacechrg = 1;
    c->min_species_density = 1e-20;
    c->min_electron_density = 1e12;
    c->min_electron_temp = 300.0;
    c->gas_temperature = T_NTP;
    c->gas_pressure = P_NTP;
    c->voltage_freq = 1.0;
    c->linsolve_reltol = 1e-10;
    c->linsolve_abstol = 1e-10;
    c->linsolve_bot_reltol = 1e-10;
    c->linsolve_bot_abstol = -1.0;
    c->linsolve_num_pre_smooth = 2;
    c->linsolve_num_post_smooth = 2;
    c->linsolve_num_final_smooth = 8;
    c->linsolve_num_bottom_smooth = 0;
    c->linsolve_maxiter = 100;
    c->linsolve_max_coarsening_level = 10;
    c->potential_scale = 1.0;
    c->elecenergy_scale = 1.0;
    c->time_scale = 1.0;
    for (int i = 0; i < VD_MAX_SPECIES; ++i) c->species_scale[i] = 1.0;
    c->mg_precision = VD_MG_FP64;
    c->mg_inner_cycles = 2;
    c->multicompsolves = 0;
    c->comp_ion_chunks = NUM_IONS;
    c->comp_neutral_chunks = NUM_NEUTRALS;
    return VD_OK;
}

vd_status vd_config_set(vd_config* c, const char* key, const char* value)
{
    if (!c || !key || !value) return VD_ERR_INVALID_ARG;
    const std::string k(key);
    std::istringstream vs(value);
    if (k == "dim")
    {
        vs >> c->dim;
        return (c->dim == 2 || c->dim == 3) ? VD_OK : VD_ERR_INVALID_ARG;
    }
    if (k == "vidyut.bg_species_ids")
    {
        int v, n = 0;
        while (vs >> v && n < VD_MAX_SPECIES) c->bg_species_ids[n++] = v;
        c->num_bg_species = n;
        return VD_OK;
    }
    if (k == "vidyut.scaling_species_ids" || k == "vidyut.scale_values")
        return VD_ERR_UNSUPPORTED; // use vd_config.species_scale directly
    for (const Key& e : g_keys)
    {
        if (k != e.name) continue;
        char* base = reinterpret_cast<char*>(c) + e.off;
        switch (e.kind)
        {
        case 0: vs >> *reinterpret_cast<int*>(base); break;
        case 1: vs >> *reinterpret_cast<double*>(base); break;
        case 2:
            for (int d = 0; d < 3 && (vs >> reinterpret_cast<int*>(base)[d]); ++d) {}
            break;
        case 3:
            for (int d = 0; d < 3 && (vs >> reinterpret_cast<double*>(base)[d]); ++d) {}
            break;
        }
        return vs.fail() && !vs.eof() ? VD_ERR_INVALID_ARG : VD_OK;
    }
    return VD_ERR_INVALID_ARG;
}

vd_status vd_case_info(vd_case_info_t* info)
{
    if (!info) return VD_ERR_INVALID_ARG;
    std::memset(info, 0, sizeof(*info));
    info->num_species = NUM_SPECIES;
    info->nvar = NVAR;
    info->e_id = E_ID;
    info->een_id = EEN_ID;
    info->etemp_id = ETEMP_ID;
    info->pot_id = POT_ID;
    info->efx_id = EFX_ID;
    info->ref_id = REF_ID;
    info->ejh_id = EJH_ID;
    info->eih_id = EIH_ID;
    info->cmask_id = CMASK_ID;
    int q[NUM_SPECIES];
    CKCHRG(q);
    std::vector<std::string> names;
    CKSYMS_STR(names);
    for (int s = 0; s < NUM_SPECIES && s < VD_MAX_SPECIES; ++s)
    {
        info->charge[s] = q[s];
        if (s < (int)names.size()) std::strncpy(info->names[s], names[s].c_str(), 15);
    }
#ifdef VD_CASE_NAME
    std::strncpy(info->case_name, VD_CASE_NAME, 63);
#endif
    return VD_OK;
}

vd_status vd_create(const vd_config* cfg, void** out)
{
    if (!cfg || !out) return VD_ERR_INVALID_ARG;
    *out = nullptr;
    if (cfg->dim != 2 && cfg->dim != 3)
    {
        g_create_err = "dim must be 2 or 3";
        return VD_ERR_INVALID_ARG;
    }
    if (cfg->hyp_order != 1 && cfg->hyp_order != 2 && cfg->hyp_order != 5)
    {
        g_create_err = "hyp_order must be 1, 2 or 5 (Source/Vidyut.cpp:448-461)";
        return VD_ERR_INVALID_ARG;
    }
    if (cfg->weno_scheme < 1 || cfg->weno_scheme > 3)
    {
        g_create_err = "weno_scheme must be 1, 2 or 3";
        return VD_ERR_INVALID_ARG;
    }
#ifndef VD_HAS_USER_TRANSPORT
    if (cfg->user_defined_potential || cfg->user_defined_species || cfg->user_defined_vel)
    {
        g_create_err = "this case defines no user_transport hooks";
        return VD_ERR_UNSUPPORTED;
    }
#endif
    for (int d = 0; d < cfg->dim; ++d)
        if (cfg->n_cell[d] < 1 || !(cfg->prob_hi[d] > cfg->prob_lo[d]))
        {
            g_create_err = "bad grid";
            return VD_ERR_INVALID_ARG;
        }
    if (cfg->electron_poisson_coupling)
    {
        // the coupled step runs the electrons as the first explicit group
        // launch (E_ID is the first transported species) and forms the
        // potential operator from face coefficients, for which the
        // inhomogeneous-Neumann right-hand-side adjustment is not built
        bool first = true;
        for (int sp = 0; sp < E_ID; ++sp)
        {
            bool bg = false;
            for (int i = 0; i < cfg->num_bg_species; ++i) bg = bg || cfg->bg_species_ids[i] == sp;
            first = first && bg;
        }
        for (int s = 0; s < 6; ++s)
        {
            const int code = (s < 3) ? cfg->pot_bc_lo[s] : cfg->pot_bc_hi[s - 3];
            if (s % 3 < cfg->dim && code == IHNEUBC) first = false;
        }
        if (!first || cfg->mg_precision != VD_MG_FP64)
        {
            g_create_err = "electron_poisson_coupling needs the electrons as the first transported "
                           "species, no inhomogeneous-Neumann potential boundary, and the FP64 "
                           "multigrid form";
            return VD_ERR_UNSUPPORTED;
        }
    }
    Ctx* c = new Ctx();
    try
    {
        c->cfg = *cfg;
        c->dev = cfg->device;
        VD_CUDA_OK(cudaSetDevice(c->dev));
        VD_CUDA_OK(cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking));
        GridDev& g = c->g;
        g.dim = cfg->dim;
        for (int d = 0; d < 3; ++d)
        {
            const bool act = d < cfg->dim;
            g.n[d] = act ? cfg->n_cell[d] : 1;
            g.per[d] = act ? cfg->is_periodic[d] : 0;
            c->G.plo[d] = act ? cfg->prob_lo[d] : 0.0;
            c->G.phi[d] = act ? cfg->prob_hi[d] : 1.0;
            c->G.dx[d] = act ? (cfg->prob_hi[d] - cfg->prob_lo[d]) / cfg->n_cell[d] : 1.0;
        }
        c->G.g = g;
        c->N = g.ncell();
        for (int i = 0; i < cfg->num_bg_species; ++i)
        {
            const int b = cfg->bg_species_ids[i];
            if (b < 0 || b >= NUM_SPECIES) throw CudaError("bg_species_ids out of range");
            c->bg[b] = 1;
        }
        make_bct(*c, cfg->pot_bc_lo, cfg->pot_bc_hi, c->pbct);
        make_bct(*c, cfg->eden_bc_lo, cfg->eden_bc_hi, c->ebct);
        make_bct(*c, cfg->eenrg_bc_lo, cfg->eenrg_bc_hi, c->eebct);
        make_bct(*c, cfg->ion_bc_lo, cfg->ion_bc_hi, c->ibct);
        make_bct(*c, cfg->neutral_bc_lo, cfg->neutral_bc_hi, c->nbct);

        const long long N = c->N;
        c->S = c->A.get<double>((size_t)NVAR * N);
        VD_CUDA_OK(cudaMemset(c->S, 0, sizeof(double) * (size_t)NVAR * N));
        const bool coupled = cfg->electron_poisson_coupling != 0;
        c->Sold = (cfg->num_timestep_correctors > 1 || coupled)
                      ? c->A.get<double>((size_t)NVAR * N)
                      : c->S;
        if (coupled)
        {
            c->rxn_e = c->A.get<double>(N);
            c->ephi = c->A.get<double>(N);
        }
        c->expl = c->A.get<double>((size_t)VD_NT * N);
        VD_CUDA_OK(cudaMemset(c->expl, 0, sizeof(double) * (size_t)VD_NT * N));
        c->rxn_een = c->A.get<double>(N);
        c->ejh = c->A.get<double>(N);
        if (cfg->elecenergy_solve)
            for (int d = 0; d < c->cfg.dim; ++d) c->jface[d] = c->A.get<double>(face_count(c->g, d));
        // a solution array per species (background ones too: a
        // multicomponent chunk or vd_implicit_diffusion_chunk may solve them)
        for (int sp = 0; sp < NUM_SPECIES; ++sp) c->u[sp] = c->A.get<double>(N);
        c->u[EEN_ID] = c->A.get<double>(N);
        c->phi_sol = c->A.get<double>(N);
        c->phi_rhs = c->A.get<double>(N);
        c->spec_rhs = c->A.get<double>(N);
        for (int s = 0; s < 6; ++s)
        {
            const int np = plane_count(g, s % 3);
            for (SideArrays* sa : {&c->pside[s], &c->sside[s]})
            {
                sa->val = c->A.get<double>(np);
                sa->ra = c->A.get<double>(np);
                sa->rb = c->A.get<double>(np);
                sa->rf = c->A.get<double>(np);
                sa->g = c->A.get<double>(np);
                sa->c0 = c->A.get<double>(np);
            }
        }
        const double dx[3] = {c->G.dx[0], c->G.dx[1], c->G.dx[2]};
        const int mcl = cfg->linsolve_max_coarsening_level;
        // the coupled potential operator has face coefficients
        hier_build(c->HP, c->A, g, dx, mcl, coupled, false);
        hier_build(c->HS, c->A, g, dx, mcl, true, false);
        // the FP64 species hierarchy's level-0 faces are written by the set-up
        // kernels; boundary arrays of both FP64 hierarchies alias the side arrays
        bind_sides64(c->HP, c->pside);
        bind_sides64(c->HS, c->sside);
        if (cfg->mg_precision == VD_MG_FP32_REFINED)
        {
            hier_build(c->HP32, c->A, g, dx, mcl, false, true);
            hier_build(c->HS32, c->A, g, dx, mcl, true, true);
            c->r64 = c->A.get<double>(N);
        }
        // multicomponent species solves: one slot per component of the
        // largest chunk, and the background species' reaction sources
        multicomp_chunks(*cfg, c->ion_chunk, c->neutral_chunk);
        if (cfg->multicompsolves && (c->ion_chunk < 1 || c->neutral_chunk < 1))
            throw UnsupportedError("comp_ion_chunks and comp_neutral_chunks must be at least 1");
        {
            int maxk = 1;
            if (cfg->multicompsolves)
            {
                for (const auto& ch : chunk_list(FIRST_ION, NUM_IONS, c->ion_chunk))
                    maxk = std::max(maxk, ch.second);
                for (const auto& ch : chunk_list(FIRST_NEUTRAL, NUM_NEUTRALS, c->neutral_chunk))
                    maxk = std::max(maxk, ch.second);
            }
            if (maxk > 8)
                throw UnsupportedError("multicomponent chunks hold at most 8 components (one "
                                       "thread-block cluster of the joint bottom solve)");
            // vd_implicit_diffusion_chunk can ask for chunks in any mode
            maxk = std::max(maxk, std::min(8, std::max(NUM_IONS, NUM_NEUTRALS)));
            if (maxk > 1)
            {
                c->HJ.resize(maxk);
                c->JS.resize(maxk);
                c->JR.resize(maxk);
                for (int q = 0; q < maxk; ++q)
                {
                    for (int s = 0; s < 6; ++s)
                    {
                        const int np = plane_count(g, s % 3);
                        SideArrays* sa = &c->JS[q][s];
                        sa->val = c->A.get<double>(np);
                        sa->ra = c->A.get<double>(np);
                        sa->rb = c->A.get<double>(np);
                        sa->rf = c->A.get<double>(np);
                        sa->g = c->A.get<double>(np);
                        sa->c0 = c->A.get<double>(np);
                    }
                    c->JR[q] = c->A.get<double>(N);
                }
                c->dcoarse = c->A.get<MGCoarse<double>>(maxk);
                VD_CUDA_OK(cudaMallocHost(&c->hcoarse, maxk * sizeof(MGCoarse<double>)));
            }
        }
        if (cfg->multicompsolves)
        {
            int nbg = 0;
            for (int sp = 0; sp < NUM_SPECIES; ++sp)
                if (c->bg[sp]) c->bgslot[sp] = nbg++;
            if (nbg) c->rxn_bg = c->A.get<double>((size_t)nbg * N);
        }
        if (cfg->poisson_warm_start)
        {
            c->zero64 = c->A.get<double>(N);
            VD_CUDA_OK(cudaMemset(c->zero64, 0, sizeof(double) * (size_t)N));
        }
        for (size_t q = 0; q < c->HJ.size(); ++q)
        {
            hier_build(c->HJ[q], c->A, g, dx, mcl, true, false);
            bind_sides64(c->HJ[q], c->JS[q].data());
            c->HJ[q].nu1 = cfg->linsolve_num_pre_smooth;
            c->HJ[q].nu2 = cfg->linsolve_num_post_smooth;
        }
        for (Hier<double>* h : {&c->HP, &c->HS})
        {
            h->nu1 = cfg->linsolve_num_pre_smooth;
            h->nu2 = cfg->linsolve_num_post_smooth;
        }
        for (Hier<float>* h : {&c->HP32, &c->HS32})
        {
            h->nu1 = cfg->linsolve_num_pre_smooth;
            h->nu2 = cfg->linsolve_num_post_smooth;
        }
        for (const void* kf : {(const void*)k_mg_coarse3<double, false>,
                               (const void*)k_mg_coarse3<double, true>,
                               (const void*)k_mg_coarse3_joint<double, true>,
                               (const void*)k_mg_coarse3<float, false>,
                               (const void*)k_mg_coarse3<float, true>})
            VD_CUDA_OK(cudaFuncSetAttribute(kf, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            VD_MG_COARSE_SMEM));
        VD_CUDA_OK(cudaFuncSetAttribute(k_mg_coarse_vcycle<double>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        VD_MG_COARSE_SMEM));
        VD_CUDA_OK(cudaFuncSetAttribute(k_mg_coarse_vcycle<float>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        VD_MG_COARSE_SMEM));
        c->HP.prof_tag = VD_PROF_POISSON_SMOOTH;
        c->HP32.prof_tag = VD_PROF_POISSON_SMOOTH32;
        VD_CUDA_OK(cudaEventCreate(&c->ev0));
        VD_CUDA_OK(cudaEventCreate(&c->ev1));
        c->dpp = c->A.get<ProbParm>(1);
        VD_CUDA_OK(cudaMemcpy(c->dpp, &c->hpp, sizeof(ProbParm), cudaMemcpyHostToDevice));
        c->dscal = c->A.get<unsigned long long>(2);
        VD_CUDA_OK(cudaMallocHost(&c->hscal, 2 * sizeof(unsigned long long)));
        c->dmg = c->A.get<MGDev>(1);
        c->npart = 65536;
        c->dpart = c->A.get<double>(2 * c->npart);
        VD_CUDA_OK(cudaMallocHost(&c->hmg, sizeof(MGDev)));
        c->fixed_dt = cfg->dt;
        c->dts = c->A.get<double>(3);
        VD_CUDA_OK(cudaMallocHost(&c->hts, 3 * sizeof(double)));
        for (int q = 0; q < 3; ++q) c->tscale[q] = std::numeric_limits<double>::max();
        // electron index (Source/Vidyut.cpp:132-144)
        c->eidx = E_ID;
        VD_CUDA_OK(cudaDeviceSynchronize());
    } catch (const CudaError& e)
    {
        const bool unsup = dynamic_cast<const UnsupportedError*>(&e) != nullptr;
        const bool oom = dynamic_cast<const OomError*>(&e) != nullptr;
        g_create_err = e.msg;
        vd_destroy(c); // everything made so far: device and pinned memory, stream, events
        return unsup ? VD_ERR_UNSUPPORTED : (oom ? VD_ERR_OOM : VD_ERR_CUDA);
    }
    *out = c;
    return VD_OK;
}

vd_status vd_destroy(void* ctx)
{
    if (!ctx) return VD_ERR_INVALID_ARG;
    Ctx* c = static_cast<Ctx*>(ctx);
    cudaSetDevice(c->dev);
    cudaStreamSynchronize(c->st);
    c->A.release();
    for (auto e : c->prof.a) cudaEventDestroy(e);
    for (auto e : c->prof.b) cudaEventDestroy(e);
    if (c->ev0) cudaEventDestroy(c->ev0);
    if (c->ev1) cudaEventDestroy(c->ev1);
    if (c->hscal) cudaFreeHost(c->hscal);
    if (c->hmg) cudaFreeHost(c->hmg);
    if (c->hts) cudaFreeHost(c->hts);
    if (c->hcoarse) cudaFreeHost(c->hcoarse);
    delete c->adjs;
    if (c->st) cudaStreamDestroy(c->st);
    delete c;
    return VD_OK;
}

#define VD_TRY(body)                                                             \
    if (!ctx) return VD_ERR_INVALID_ARG;                                         \
    Ctx* c = static_cast<Ctx*>(ctx);                                             \
    t_prof = &c->prof;                                                           \
    try                                                                          \
    {                                                                            \
        VD_CUDA_OK(cudaSetDevice(c->dev));                                       \
        body;                                                                    \
        VD_CUDA_OK(cudaStreamSynchronize(c->st));                                \
    } catch (const UnsupportedError& e)                                          \
    {                                                                            \
        c->err = e.msg;                                                          \
        return VD_ERR_UNSUPPORTED;                                               \
    } catch (const OomError& e)                                                  \
    {                                                                            \
        c->err = e.msg;                                                          \
        return VD_ERR_OOM;                                                       \
    } catch (const CudaError& e)                                                 \
    {                                                                            \
        c->err = e.msg;                                                          \
        return VD_ERR_CUDA;                                                      \
    }

vd_status vd_init_domain(void* ctx, const char* prob_inputs)
{
    VD_TRY({
        c->hpp = ProbParm{};
        vd_probinit(c->hpp, prob_inputs);
        VD_CUDA_OK(cudaMemcpyAsync(c->dpp, &c->hpp, sizeof(ProbParm), cudaMemcpyHostToDevice, c->st));
        LAUNCH(k_initdomain, gsz(c->N), BS, c->st, c->G, c->S, c->dpp);
        c->time = 0.0;
        c->step = 0;
    });
    return VD_OK;
}

vd_status vd_set_state(void* ctx, int comp, int ncomp, const double* src, int on_device)
{
    if (!ctx || !src || comp < 0 || ncomp < 1 || comp + ncomp > NVAR) return VD_ERR_INVALID_ARG;
    VD_TRY({
        VD_CUDA_OK(cudaMemcpyAsync(c->S + (size_t)comp * c->N, src,
                                   sizeof(double) * (size_t)ncomp * c->N,
                                   on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                                   c->st));
    });
    return VD_OK;
}

vd_status vd_get_state(void* ctx, int comp, int ncomp, double* dst, int on_device)
{
    if (!ctx || !dst || comp < 0 || ncomp < 1 || comp + ncomp > NVAR) return VD_ERR_INVALID_ARG;
    VD_TRY({
        VD_CUDA_OK(cudaMemcpyAsync(dst, c->S + (size_t)comp * c->N,
                                   sizeof(double) * (size_t)ncomp * c->N,
                                   on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                                   c->st));
    });
    return VD_OK;
}

vd_status vd_set_time(void* ctx, double time, int step)
{
    if (!ctx) return VD_ERR_INVALID_ARG;
    Ctx* c = static_cast<Ctx*>(ctx);
    c->time = time;
    c->step = step;
    return VD_OK;
}

vd_status vd_set_dt(void* ctx, double dt)
{
    if (!ctx || !(dt > 0.0)) return VD_ERR_INVALID_ARG;
    static_cast<Ctx*>(ctx)->cfg.dt = dt;
    return VD_OK;
}

vd_status vd_get_dt(void* ctx, double* dt)
{
    if (!ctx || !dt) return VD_ERR_INVALID_ARG;
    *dt = static_cast<Ctx*>(ctx)->cfg.dt;
    return VD_OK;
}

vd_status vd_get_time(void* ctx, double* time, int* step)
{
    if (!ctx) return VD_ERR_INVALID_ARG;
    Ctx* c = static_cast<Ctx*>(ctx);
    if (time) *time = c->time;
    if (step) *step = c->step;
    return VD_OK;
}

vd_status vd_step(void* ctx, int nsteps, vd_step_stats* stats)
{
    if (nsteps < 0) return VD_ERR_INVALID_ARG;
    VD_TRY({
        c->poisson_iters = 0;
        c->species_iters = 0;
        c->poisson_refs = 0;
        c->not_converged = 0;
        c->max_poisson_res = 0.0;
        VD_CUDA_OK(cudaEventRecord(c->ev0, c->st));
        for (int s = 0; s < nsteps; ++s) step_once(*c);
        VD_CUDA_OK(cudaEventRecord(c->ev1, c->st));
        VD_CUDA_OK(cudaEventSynchronize(c->ev1));
        float ms = 0.f;
        VD_CUDA_OK(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
        if (stats)
        {
            std::memset(stats, 0, sizeof(*stats));
            stats->steps = nsteps;
            stats->poisson_iterations = (int)c->poisson_iters;
            stats->species_iterations = (int)c->species_iters;
            stats->poisson_refinements = (int)c->poisson_refs;
            stats->not_converged = c->not_converged;
            stats->max_poisson_final_residual = c->max_poisson_res;
            stats->time = c->time;
            stats->gpu_ms = ms;
            stats->dt = c->cfg.dt;
            stats->dt_edrift = c->tscale[0];
            stats->dt_ediff = c->tscale[1];
            stats->dt_diel_relax = c->tscale[2];
        }
    });
    return c->not_converged ? VD_ERR_NOT_CONVERGED : VD_OK;
}

vd_status vd_profile_kernel(void* ctx, int kernel_id)
{
    VD_TRY({
        c->prof.id = kernel_id;
        c->prof.n = 0;
        c->prof.bytes = 0.0;
    });
    return VD_OK;
}

vd_status vd_profile_read(void* ctx, long long* launches, double* total_ms,
                          double* bytes_per_launch)
{
    double tot = 0.0;
    long long used = 0;
    VD_TRY({
        std::vector<float> t(c->prof.n);
        std::vector<float> per(c->prof.n);
        for (int i = 0; i < c->prof.n; ++i)
        {
            VD_CUDA_OK(cudaEventSynchronize(c->prof.b[i]));
            VD_CUDA_OK(cudaEventElapsedTime(&t[i], c->prof.a[i], c->prof.b[i]));
            per[i] = t[i] / (c->prof.cnt[i] > 0 ? c->prof.cnt[i] : 1);
        }
        // V-cycles are enqueued in batches, and the launches of a cycle
        // enqueued past convergence return at once on the stop flag (a few
        // µs against tens for a working sweep): those did no work and are
        // left out, by their per-launch duration, below a quarter of the
        // median
        std::vector<float> srt = per;
        std::sort(srt.begin(), srt.end());
        const float cut = srt.empty() ? 0.f : 0.25f * srt[srt.size() / 2];
        for (int i = 0; i < c->prof.n; ++i)
            if (per[i] >= cut)
            {
                tot += t[i];
                used += c->prof.cnt[i] > 0 ? c->prof.cnt[i] : 1;
            }
    });
    if (launches) *launches = used;
    if (total_ms) *total_ms = tot;
    if (bytes_per_launch) *bytes_per_launch = c->prof.bytes;
    return VD_OK;
}

vd_status vd_poisson_solve(void* ctx, double time, vd_solve_stats* stats)
{
    VD_TRY({
        c->not_converged = 0;
        poisson(*c, time, c->S, stats);
    });
    return c->not_converged ? VD_ERR_NOT_CONVERGED : VD_OK;
}

vd_status vd_explicit_rhs(void* ctx, double time, double* out, int on_device)
{
    VD_TRY({
        explicit_rhs(*c, time);
        if (out)
            VD_CUDA_OK(cudaMemcpyAsync(out, c->expl, sizeof(double) * (size_t)VD_NT * c->N,
                                       on_device ? cudaMemcpyDeviceToDevice
                                                 : cudaMemcpyDeviceToHost,
                                       c->st));
    });
    return VD_OK;
}

vd_status vd_implicit_diffusion(void* ctx, int spec, double time, const double* expl_in,
                                int on_device, vd_solve_stats* stats)
{
    if (!ctx || !expl_in || spec < 0 || spec > NUM_SPECIES) return VD_ERR_INVALID_ARG;
    VD_TRY({
        c->not_converged = 0;
        VD_CUDA_OK(cudaMemcpyAsync(c->expl, expl_in, sizeof(double) * (size_t)VD_NT * c->N,
                                   on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                                   c->st));
        species_solve(*c, spec, time, c->S, stats);
        FinalParams P = final_params(*c);
        add_solved(*c, P, spec);
        P.een_solved = (spec == EEN_ID) ? 1 : 0;
        LAUNCH(k_finalize, gsz(c->N), BS, c->st, P);
    });
    return c->not_converged ? VD_ERR_NOT_CONVERGED : VD_OK;
}

vd_status vd_implicit_diffusion_chunk(void* ctx, int startspec, int numspec, double time,
                                      const double* expl_in, int on_device,
                                      vd_solve_stats* stats)
{
    if (!ctx || !expl_in || numspec < 1 || startspec < 0) return VD_ERR_INVALID_ARG;
    if (numspec == 1) return vd_implicit_diffusion(ctx, startspec, time, expl_in, on_device, stats);
    if (startspec + numspec > NUM_SPECIES) return VD_ERR_INVALID_ARG;
    VD_TRY({
        c->not_converged = 0;
        VD_CUDA_OK(cudaMemcpyAsync(c->expl, expl_in, sizeof(double) * (size_t)VD_NT * c->N,
                                   on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                                   c->st));
        joint_solve(*c, startspec, numspec, time, c->S, stats);
        FinalParams P = final_params(*c);
        for (int q = 0; q < numspec; ++q) add_solved(*c, P, startspec + q);
        LAUNCH(k_finalize, gsz(c->N), BS, c->st, P);
    });
    return c->not_converged ? VD_ERR_NOT_CONVERGED : VD_OK;
}

vd_status vd_check_state(void* ctx, long long* nonfinite)
{
    if (!nonfinite) return VD_ERR_INVALID_ARG;
    VD_TRY({
        VD_CUDA_OK(cudaMemsetAsync(c->dscal, 0, sizeof(unsigned long long), c->st));
        LAUNCH(k_nonfinite, gsz((long long)(NUM_SPECIES + 3) * c->N), BS, c->st, c->S,
               (long long)(NUM_SPECIES + 3) * c->N, c->dscal);
        VD_CUDA_OK(cudaMemcpyAsync(c->hscal, c->dscal, sizeof(unsigned long long),
                                   cudaMemcpyDeviceToHost, c->st));
    });
    *nonfinite = (long long)*c->hscal;
    return *nonfinite ? VD_ERR_NONFINITE : VD_OK;
}

vd_status vd_adjoint_num_params(void* ctx, int* n_params)
{
    if (!ctx || !n_params) return VD_ERR_INVALID_ARG;
#ifdef VD_HAS_MECH_ADJOINT
    *n_params = ADJ_NR + 1;
#else
    *n_params = 0;
#endif
    return VD_OK;
}

#ifdef VD_HAS_MECH_ADJOINT
#define VD_ADJ_CASE_CHECK
#else
#define VD_ADJ_CASE_CHECK                                                        \
    {                                                                            \
        static_cast<Ctx*>(ctx)->err = "this case's mechanism has no adjoint form"; \
        return VD_ERR_UNSUPPORTED;                                               \
    }
#endif

vd_status vd_adjoint_set_params(void* ctx, const double* params, int n_params)
{
    if (!ctx || !params) return VD_ERR_INVALID_ARG;
    VD_ADJ_CASE_CHECK
#ifdef VD_HAS_MECH_ADJOINT
    if (n_params != ADJ_NR + 1 || !(params[ADJ_NR] > 0.0))
    {
        static_cast<Ctx*>(ctx)->err = "expected NUM_REACTIONS log pre-factor shifts and a "
                                      "positive electron mobility scale";
        return VD_ERR_INVALID_ARG;
    }
    VD_TRY({
        AdjState& a = adj_state(*c, 0);
        a.params.assign(params, params + ADJ_NR + 1);
    });
#endif
    return VD_OK;
}

vd_status vd_adjoint_forward(void* ctx, int nsteps, int objective_id, double* objective,
                             double* species_out)
{
    if (!ctx || nsteps < 0 || objective_id != VD_ADJ_OBJ_ELECTRONS) return VD_ERR_INVALID_ARG;
    VD_ADJ_CASE_CHECK
#ifdef VD_HAS_MECH_ADJOINT
    VD_TRY({
        AdjState& a = adj_state(*c, 3);
        const AdjParams P = adj_params(*c, a);
        adj_upload(*c, a);
        const double* fin = adj_forward(*c, a, P, nsteps, 0);
        if (species_out)
            VD_CUDA_OK(cudaMemcpyAsync(species_out, fin, sizeof(double) * (size_t)a.nt * c->N,
                                       cudaMemcpyDeviceToHost, c->st));
        adj_read_acc(*c, a);
        if (objective) *objective = a.hacc[0];
    });
#endif
    return VD_OK;
}

vd_status vd_adjoint_run(void* ctx, int nsteps, int K, int objective_id, double* objective,
                         double* grad_out, int n_params)
{
    if (!ctx || nsteps < 1 || K < 1 || objective_id != VD_ADJ_OBJ_ELECTRONS || !grad_out)
        return VD_ERR_INVALID_ARG;
    VD_ADJ_CASE_CHECK
#ifdef VD_HAS_MECH_ADJOINT
    if (n_params != ADJ_NR + 1) return VD_ERR_INVALID_ARG;
    VD_TRY({
        adj_run(*c, nsteps, K);
        AdjState& a = *c->adjs;
        if (objective) *objective = a.hacc[0];
        for (int r = 0; r <= ADJ_NR; ++r) grad_out[r] = a.hacc[1 + r];
    });
#endif
    return VD_OK;
}

vd_status vd_launch_count(void* ctx, long long* launches)
{
    if (!launches) return VD_ERR_INVALID_ARG;
    *launches = vd::g_launches;
    return VD_OK;
}

vd_status vd_last_error(void* ctx, char* buf, int len)
{
    if (!buf || len < 1) return VD_ERR_INVALID_ARG;
    const std::string& m = ctx ? static_cast<Ctx*>(ctx)->err : g_create_err;
    std::strncpy(buf, m.c_str(), len - 1);
    buf[len - 1] = 0;
    return VD_OK;
}

} // extern "C"

// ======================================================================
// Allocation-free Poisson solve.
//
// Some callers cannot call cudaMalloc at solve time: a host framework that
// owns all device memory through its own pool and forbids allocation
// inside its step (allocation would break its memory accounting), or code
// running where a device allocation could synchronise the device or fail
// late.  vd_poisson_solve_noalloc serves them: the caller passes the
// right-hand side and the potential as device arrays it already owns, and
// every scratch array the multigrid needs (coarse levels, boundary planes,
// bottom-solver vectors, residual norms) lives in the file-scope device
// array below, which every GPU that loads this library holds until the
// process exits.
// ======================================================================
namespace {
using vd::Array4;
using vd::Box;
using vd::GeometryData;
using vd::GpuArray;
using vd::IntVect;
using vd::Real;

constexpr long long VD_NA_SCRATCH_DOUBLES = 1LL << 20; // 8 MiB per device
constexpr int VD_NA_MAX_LEVELS = 16;

static __device__ __align__(256) double vd_na_scratch[VD_NA_SCRATCH_DOUBLES];

void na_msg(char* err, int errlen, const char* m)
{
    if (err && errlen > 0)
    {
        std::strncpy(err, m, errlen - 1);
        err[errlen - 1] = 0;
    }
}

#define NA_LAUNCH(K, G, B, ...)                                                   \
    do                                                                            \
    {                                                                             \
        K<<<(G), (B), 0, 0>>>(__VA_ARGS__);                                       \
        ++vd::g_launches;                                                         \
        const cudaError_t e_ = cudaGetLastError();                                \
        if (e_ != cudaSuccess)                                                    \
        {                                                                         \
            na_msg(err, errlen, cudaGetErrorString(e_));                          \
            return VD_ERR_CUDA;                                                   \
        }                                                                         \
    } while (0)

long long na_round(long long n) { return (n + 31) & ~31LL; }

struct NAHier
{
    int nlev;
    GridDev g[VD_NA_MAX_LEVELS];
    double dx[VD_NA_MAX_LEVELS][3];
    double* x[VD_NA_MAX_LEVELS];
    double* f[VD_NA_MAX_LEVELS];
    MGOp<double> op[VD_NA_MAX_LEVELS];
    double* g0[6];
    double* scratch;
    double* t0x;
    double* t0f;
    unsigned long long* norm;
};

int na_vcycle(NAHier& H, double* x0, const double* f0, char* err, int errlen)
{
    const int L = H.nlev;
    if (L == 1)
    {
        const Grid3 gn = rows3(H.g[0], 8);
        NA_LAUNCH(k_mg_resid_norm<double>, gn.g, gn.b, H.op[0], x0, f0, H.t0f, H.norm + 2, 1,
                  0, 8);
        NA_LAUNCH(k_mg_bottom<double>, 1, 256, H.op[0], H.t0x, H.t0f, H.scratch, 1e-4, 200, 0,
                  8, (int*)nullptr);
        NA_LAUNCH(k_add_same<double>, gsz(H.g[0].ncell()), BS, x0, H.t0x, H.g[0].ncell(),
                  (const int*)nullptr);
        return VD_OK;
    }
    for (int l = 0; l < L; ++l)
    {
        double* xl = l ? H.x[l] : x0;
        const double* fl = l ? H.f[l] : f0;
        if (l == L - 1)
        {
            NA_LAUNCH(k_mg_bottom<double>, 1, 256, H.op[l], xl, fl, H.scratch, 1e-4, 200, 0, 8,
                      (int*)nullptr);
            break;
        }
        for (int s = 0; s < 2; ++s)
            for (int color = 0; color < 2; ++color)
                NA_LAUNCH(k_mg_smooth_color<double>,
                          gsz((long long)((H.g[l].n[0] + 1) / 2) * H.g[l].n[1] * H.g[l].n[2]), BS,
                          H.op[l], xl, fl, color, l == 0 ? 1 : 0);
        const Grid3 gr = rows3(H.g[l + 1]);
        NA_LAUNCH(k_mg_resid_restrict<double>, gr.g, gr.b, H.op[l], xl, fl, H.g[l + 1],
                  H.f[l + 1], H.x[l + 1], l == 0 ? 1 : 0);
    }
    for (int l = L - 2; l >= 0; --l)
    {
        double* xl = l ? H.x[l] : x0;
        const double* fl = l ? H.f[l] : f0;
        const Grid3 gp = rows3(H.g[l]);
        NA_LAUNCH(k_mg_prolong_add<double>, gp.g, gp.b, H.g[l], H.g[l + 1], xl, H.x[l + 1],
                  (const int*)nullptr);
        for (int s = 0; s < 2; ++s)
            for (int color = 0; color < 2; ++color)
                NA_LAUNCH(k_mg_smooth_color<double>,
                          gsz((long long)((H.g[l].n[0] + 1) / 2) * H.g[l].n[1] * H.g[l].n[2]), BS,
                          H.op[l], xl, fl, color, l == 0 ? 1 : 0);
    }
    return VD_OK;
}

__global__ void k_na_fill_side(double* g, int np, double v)
{
    VD_PDL_WAIT();
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < np; q += gridDim.x * blockDim.x)
        g[q] = v;
}

} // namespace

extern "C" vd_status vd_poisson_solve_noalloc(int dim, const int* n_cell, const double* dx,
                                              const int* bc_lo, const int* bc_hi,
                                              const double* bcval_lo, const double* bcval_hi,
                                              const double* rhs, double* phi, double reltol,
                                              double abstol, int maxiter,
                                              vd_solve_stats* stats, char* err, int errlen)
{
    if ((dim != 2 && dim != 3) || !n_cell || !dx || !bc_lo || !bc_hi || !rhs || !phi)
    {
        na_msg(err, errlen, "vd_poisson_solve_noalloc: bad arguments");
        return VD_ERR_INVALID_ARG;
    }
    // The host-side name vd_na_scratch is not a device address.  Its device
    // address is looked up on every call, with the caller's device current:
    // the lookup allocates nothing, and it stays right after a device reset
    // or a rebuilt primary context (which reload the module and may move the
    // array), where an address cached from an earlier call would dangle.
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess)
    {
        na_msg(err, errlen, "vd_poisson_solve_noalloc: no usable current CUDA device");
        return VD_ERR_CUDA;
    }
    double* base = nullptr;
    {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, vd_na_scratch);
        if (e != cudaSuccess || !p)
        {
            na_msg(err, errlen, cudaGetErrorString(e));
            return VD_ERR_CUDA;
        }
        base = static_cast<double*>(p);
    }

    // level hierarchy (fine level: the caller's arrays, natural layout)
    NAHier H{};
    GridDev fine{};
    fine.dim = dim;
    for (int d = 0; d < 3; ++d)
    {
        fine.n[d] = d < dim ? n_cell[d] : 1;
        fine.per[d] = (d < dim && bc_lo[d] == PERBC) ? 1 : 0;
        if (fine.n[d] < 1 || (d < dim && !(dx[d] > 0.0)))
        {
            na_msg(err, errlen, "vd_poisson_solve_noalloc: bad grid");
            return VD_ERR_INVALID_ARG;
        }
    }
    fine.rb = 0;
    H.g[0] = fine;
    for (int d = 0; d < 3; ++d) H.dx[0][d] = d < dim ? dx[d] : 1.0;
    H.nlev = 1;
    while (H.nlev < VD_NA_MAX_LEVELS)
    {
        const GridDev& c = H.g[H.nlev - 1];
        bool ok = true;
        for (int d = 0; d < dim; ++d)
            if (c.n[d] % 2 != 0 || c.n[d] / 2 < 2) ok = false;
        if (!ok) break;
        GridDev nxt = c;
        for (int d = 0; d < dim; ++d)
        {
            nxt.n[d] = c.n[d] / 2;
            H.dx[H.nlev][d] = H.dx[H.nlev - 1][d] * 2.0;
        }
        for (int d = dim; d < 3; ++d) H.dx[H.nlev][d] = 1.0;
        nxt.rb = (nxt.n[0] % 2 == 0) ? 1 : 0;
        H.g[H.nlev++] = nxt;
    }
    if (H.g[H.nlev - 1].ncell() > 4096)
    {
        na_msg(err, errlen, "vd_poisson_solve_noalloc: grid does not coarsen to 4096 cells");
        return VD_ERR_INVALID_ARG;
    }
    // carve the scratch: norms, boundary planes, coarse levels, bottom vectors
    long long off = 32;
    for (int s = 0; s < 6; ++s)
    {
        H.g0[s] = base + off;
        off += na_round(plane_count(fine, s % 3));
    }
    for (int l = 1; l < H.nlev; ++l)
    {
        H.x[l] = base + off;
        off += na_round(H.g[l].ncell());
        H.f[l] = base + off;
        off += na_round(H.g[l].ncell());
    }
    H.scratch = base + off;
    off += na_round(6 * H.g[H.nlev - 1].ncell());
    if (H.nlev == 1)
    {
        H.t0x = base + off;
        off += na_round(fine.ncell());
        H.t0f = base + off;
        off += na_round(fine.ncell());
    }
    if (off > VD_NA_SCRATCH_DOUBLES)
    {
        char m[256];
        std::snprintf(m, sizeof(m),
                      "vd_poisson_solve_noalloc: this grid needs %lld doubles of scratch, the "
                      "allocation-free solve holds at most %lld (about 128^3 cells)",
                      off, VD_NA_SCRATCH_DOUBLES);
        na_msg(err, errlen, m);
        return VD_ERR_INVALID_ARG;
    }
    H.norm = reinterpret_cast<unsigned long long*>(base);

    // operator: del^2 phi = rhs  (a = 0, b = -1, beta = 1, maxorder 2),
    // the field solve's operator (Source/PotentialSolve.cpp:205-219)
    int bct[6];
    for (int d = 0; d < 3; ++d)
    {
        if (d >= dim || fine.per[d])
        {
            bct[d] = bct[d + 3] = MG_PER;
            continue;
        }
        bct[d] = mg_type(bc_lo[d]);
        bct[d + 3] = mg_type(bc_hi[d]);
        if ((bct[d] != MG_DIR && bct[d] != MG_NEU) || (bct[d + 3] != MG_DIR && bct[d + 3] != MG_NEU))
        {
            na_msg(err, errlen, "vd_poisson_solve_noalloc: boundaries must be periodic, "
                                "Dirichlet or homogeneous Neumann");
            return VD_ERR_UNSUPPORTED;
        }
    }
    for (int l = 0; l < H.nlev; ++l)
    {
        MGOp<double>& o = H.op[l];
        o = MGOp<double>{};
        o.g = H.g[l];
        for (int d = 0; d < 3; ++d) o.dh[d] = d < dim ? 1.0 / (H.dx[l][d] * H.dx[l][d]) : 0.0;
        o.aconst = 0.0;
        o.bconst = -1.0;
        for (int s = 0; s < 6; ++s)
        {
            o.bct[s] = bct[s];
            o.c0s[s] = 1.0;
            o.c1s[s] = 0.0;
            if (bct[s] == MG_DIR)
            {
                o.c0s[s] = -1.0;
                if (l == 0) o.gv[s] = H.g0[s];
            }
        }
    }
    for (int s = 0; s < 6; ++s)
        if (bct[s] == MG_DIR)
        {
            const int np = plane_count(fine, s % 3);
            const double v = (s < 3 ? (bcval_lo ? bcval_lo[s] : 0.0) : (bcval_hi ? bcval_hi[s - 3] : 0.0));
            NA_LAUNCH(k_na_fill_side, gsz(np), BS, H.g0[s], np, 2.0 * v);
        }

    // solve (max-norm test against max(|rhs|, |r0|), as the context path)
    auto norm = [&](double* r, double* fmax) -> int {
        if (cudaMemsetAsync(H.norm, 0, 2 * sizeof(unsigned long long), 0) != cudaSuccess)
            return VD_ERR_CUDA;
        const Grid3 gn = rows3(fine, 8);
        NA_LAUNCH(k_mg_resid_norm<double>, gn.g, gn.b, H.op[0], phi, rhs, (double*)nullptr,
                  H.norm, 1, fmax ? 1 : 0, 8);
        unsigned long long h[2] = {0, 0};
        if (cudaMemcpy(h, H.norm, sizeof(h), cudaMemcpyDeviceToHost) != cudaSuccess)
            return VD_ERR_CUDA;
        std::memcpy(r, &h[0], sizeof(double));
        if (fmax) std::memcpy(fmax, &h[1], sizeof(double));
        return VD_OK;
    };
    vd_solve_stats st{};
    double r0 = 0.0, b0 = 0.0;
    if (norm(&r0, &b0) != VD_OK)
    {
        na_msg(err, errlen, "vd_poisson_solve_noalloc: CUDA error");
        return VD_ERR_CUDA;
    }
    const double target = std::max(abstol, std::max(reltol, 1e-16) * std::max(b0, r0));
    st.initial_residual = st.final_residual = r0;
    st.converged = (r0 <= target) ? 1 : 0;
    for (int it = 1; !st.converged && it <= maxiter; ++it)
    {
        const int rc = na_vcycle(H, phi, rhs, err, errlen);
        if (rc != VD_OK) return (vd_status)rc;
        double rn = 0.0;
        if (norm(&rn, nullptr) != VD_OK)
        {
            na_msg(err, errlen, "vd_poisson_solve_noalloc: CUDA error");
            return VD_ERR_CUDA;
        }
        st.iterations = it;
        st.final_residual = rn;
        if (rn <= target) st.converged = 1;
    }
    if (stats) *stats = st;
    na_msg(err, errlen, "");
    return st.converged ? VD_OK : VD_ERR_NOT_CONVERGED;
}
