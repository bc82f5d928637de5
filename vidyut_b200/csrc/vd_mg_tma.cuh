// Red-black Gauss-Seidel colour sweep of a 3-D split level with its
// operands staged in shared memory by the Tensor Memory Accelerator: an
// alternative to the register-staged k_mg_sweep3v on the levels that live
// in HBM, selected with VD_MG_TMA=1 (off by default; measured below).
//
// The level is cut into tiles of TMA_TX half-cells by TY rows.  A CTA owns
// one tile and one z-chunk of its planes and streams the planes through
// rings in shared memory:
//   X ring: the other colour of x, tile plus a halo of XH half-cells in x
//           (XH * sizeof(T) = 16 bytes, so the box starts on a 16-byte
//           boundary) and one row in y; planes k-1, k, k+1 in use;
//   F ring: this colour of f (and, NORM, this colour of x before the
//           update), the tile; plane k in use.
// A producer warp issues cp.async.bulk.tensor loads ahead into free slots
// (full/empty mbarrier pairs); eight consumer warps read shared memory only
// and write their updated pairs with 16-byte stores.  A load may start at a
// negative or past-the-end coordinate (the first tile, the planes k = -1
// and k = nz): the tensor map fills those boxes with zeros, which the ghost
// closure never reads (an outside neighbour takes the opposite neighbour's
// value, as in k_mg_sweep3v).  The CTAs of one z-chunk stream the same
// planes at the same time, so the halo rows come from L2 (DRAM reads of a
// 256^3 launch: 139.5 MB, against 134.2 MB algorithmic).
//
// The cell arithmetic is mg3_gs_value / mg3_residual on the same neighbour
// values as k_mg_sweep3v, so both kernels give the same bits.  Constant
// coefficients only (the Poisson operator).
//
// Measured at 256^3 (FP64 fine-level sweep): 59.9 us per launch against
// 46.5 us for k_mg_sweep3v.  The consumers are the limit, not the bytes in
// flight: two CTAs per SM (the rings take ~92 KB each, 96 registers a
// thread) leave four consumer warps per scheduler, against eight in the
// register-staged sweep, for the same ~170 instructions per warp and pair
// row, so latency stalls (fixed-latency dependencies, then the x-boundary
// lanes' ghost loads) are not hidden.
//
// Waits are bounded: a wait that gives up (or sees another thread give up)
// sets *err and the thread leaves; the producer first lets its copies in
// flight land (bounded), and the host reports the failure.
#pragma once
#include "vd_mg.cuh"
#include <cuda.h>

namespace vd {

#ifndef VD_TMA_SPIN
#define VD_TMA_SPIN (1 << 22)
#endif

constexpr int TMA_TX = 64; // half-cells of a tile in x

__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(ok)
                 : "r"(bar), "r"(parity)
                 : "memory");
    return ok != 0;
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

// Bounded wait for the phase of the given parity; false if it gave up or
// another thread of the CTA raised *abort (checked every 256 polls).
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, const int* abort)
{
    for (int it = 0; it < VD_TMA_SPIN; ++it)
    {
        if (mbar_try(bar, parity)) return true;
        if (abort && (it & 255) == 255 && *(const volatile int*)abort) return false;
    }
    return false;
}

__device__ __forceinline__ void tma_load_3d(uint32_t dst, const CUtensorMap* map, uint32_t bar,
                                            int c0, int c1, int c2)
{
    asm volatile("cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
                 " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(dst),
                 "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(bar)
                 : "memory");
}

// Ring sizes (slots) and slot bytes of one instantiation.
template <typename T, bool NORM>
struct TmaSweepShape
{
    static constexpr int TY = 16;                  // rows of a tile
    static constexpr int RR = TY / 8;              // rows of a consumer thread
    static constexpr int THREADS = 288;            // 8 consumer warps + 1 producer warp
    static constexpr int MINB = 2;                 // CTAs per SM the rings allow
    static constexpr int XH = 16 / (int)sizeof(T); // x halo: 16 bytes
    static constexpr int XW = TMA_TX + 2 * XH;     // smem row of the X box
    static constexpr int SX = sizeof(T) == 8 ? (NORM ? 5 : 6) : 8;
    static constexpr int SF = sizeof(T) == 8 ? (NORM ? 3 : 4) : (NORM ? 5 : 6);
    static constexpr int XBYTES = (TY + 2) * XW * (int)sizeof(T);
    static constexpr int XSLOT = (XBYTES + 127) / 128 * 128;
    static constexpr int FBYTES = TY * TMA_TX * (int)sizeof(T);
    static constexpr int FSLOT = FBYTES * (NORM ? 2 : 1); // f tile, then (NORM) x tile
    static constexpr int NBAR = 2 * SX + 2 * SF;         // full and empty per slot
    static constexpr int SMEM = SX * XSLOT + SF * FSLOT + NBAR * 8 + 16 + 128;
};

// Gauss-Seidel update of the consumer thread's pairs (rows w and w + 8 of
// the tile, half-cells 2 lane, 2 lane + 1) in plane k from the staged planes
// X0, X1, X2 (k-1, k, k+1), F and V.  EDGE: some row or the plane is on the
// level boundary in y or z (warp-uniform), so outside neighbours take the
// opposite one's value and the ghost closure; x ends are folded in always.
// Every load of both rows is issued before any arithmetic.
template <typename T, bool PROL, bool NORM, bool EDGE>
__device__ __forceinline__ void tma_pairs(const MGOp<T>& L, const T* X0, const T* X1,
                                          const T* X2, const T* F, const T* V, int lane, int w,
                                          int x0, int y0, int k, int color, bool inhomog,
                                          T inv_gamma, const GridDev& gc, const T* xc,
                                          T* __restrict__ xs, double& mres)
{
    using S = TmaSweepShape<T, NORM>;
    using V2 = typename Vec2<T>::type;
    constexpr int RR = S::RR, XW = S::XW;
    const GridDev& g = L.g;
    const int nx = g.n[0], nxh = nx >> 1, ny = g.n[1], nz = g.n[2];
    const int ih = x0 + 2 * lane, c = S::XH + 2 * lane;
    const int q = (y0 + w + k + color) & 1; // rows w and w + 8 share it
    // the pair's outer x neighbour: 2l-1 (q = 0) or 2l+2 (q = 1); at the
    // ends of a row the ghost closure replaces it (the opposite one read)
    const bool xlo = q == 0 && ih == 0, xhi = q == 1 && ih + 2 == nxh;
    const int so = q ? (xhi ? 1 : 2) : (xlo ? 0 : -1);
    const T* PZm = (EDGE && k == 0) ? X2 : X0;
    const T* PZp = (EDGE && k == nz - 1) ? X0 : X2;
    V2 vx[RR], vym[RR], vyp[RR], vzm[RR], vzp[RR], vf[RR], v0[NORM ? RR : 1];
    T sx[RR];
#pragma unroll
    for (int rr = 0; rr < RR; ++rr)
    {
        const int r = w + 8 * rr, j = y0 + r;
        const int rm = (EDGE && j == 0) ? r + 2 : r, rp = (EDGE && j == ny - 1) ? r : r + 2;
        const T* R1 = X1 + (r + 1) * XW + c;
        vx[rr] = *reinterpret_cast<const V2*>(R1);
        sx[rr] = R1[so];
        vym[rr] = *reinterpret_cast<const V2*>(X1 + rm * XW + c);
        vyp[rr] = *reinterpret_cast<const V2*>(X1 + rp * XW + c);
        vzm[rr] = *reinterpret_cast<const V2*>(PZm + (r + 1) * XW + c);
        vzp[rr] = *reinterpret_cast<const V2*>(PZp + (r + 1) * XW + c);
        vf[rr] = *reinterpret_cast<const V2*>(F + r * TMA_TX + 2 * lane);
        if (NORM) v0[rr] = *reinterpret_cast<const V2*>(V + r * TMA_TX + 2 * lane);
    }
#pragma unroll
    for (int rr = 0; rr < RR; ++rr)
    {
        const int j = y0 + w + 8 * rr;
        if (j >= ny || ih >= nxh) continue;
        if (PROL)
        {
            // x + P e: an other-colour neighbour at half-index h' of row j'
            // has coarse column h', row j' >> 1, plane k' >> 1
            const int J = j >> 1, K = k >> 1;
            const int jm = (EDGE && j == 0) ? j + 1 : j - 1;
            const int jp = (EDGE && j == ny - 1) ? j - 1 : j + 1;
            const int km = (EDGE && k == 0) ? k + 1 : k - 1;
            const int kp = (EDGE && k == nz - 1) ? k - 1 : k + 1;
            T cx[3];
#pragma unroll
            for (int e = 0; e < 3; ++e)
                cx[e] = __ldg(xc + gc.idx(min(max(ih - 1 + q + e, 0), nxh - 1), J, K));
            if (q == 0)
            {
                sx[rr] += cx[0];
                vx[rr].x += cx[1];
                vx[rr].y += cx[2];
            } else
            {
                vx[rr].x += cx[0];
                vx[rr].y += cx[1];
                sx[rr] += cx[2];
            }
            vym[rr].x += __ldg(xc + gc.idx(ih, jm >> 1, K));
            vym[rr].y += __ldg(xc + gc.idx(ih + 1, jm >> 1, K));
            vyp[rr].x += __ldg(xc + gc.idx(ih, jp >> 1, K));
            vyp[rr].y += __ldg(xc + gc.idx(ih + 1, jp >> 1, K));
            vzm[rr].x += __ldg(xc + gc.idx(ih, J, km >> 1));
            vzm[rr].y += __ldg(xc + gc.idx(ih + 1, J, km >> 1));
            vzp[rr].x += __ldg(xc + gc.idx(ih, J, kp >> 1));
            vzp[rr].y += __ldg(xc + gc.idx(ih + 1, J, kp >> 1));
        }
        T nA[6], nB[6];
        if (q == 0)
        {
            nA[0] = sx[rr];
            nA[1] = vx[rr].x;
            nB[0] = vx[rr].x;
            nB[1] = vx[rr].y;
        } else
        {
            nA[0] = vx[rr].x;
            nA[1] = vx[rr].y;
            nB[0] = vx[rr].y;
            nB[1] = sx[rr];
        }
        nA[2] = vym[rr].x;
        nB[2] = vym[rr].y;
        nA[3] = vyp[rr].x;
        nB[3] = vyp[rr].y;
        nA[4] = vzm[rr].x;
        nB[4] = vzm[rr].y;
        nA[5] = vzp[rr].x;
        nB[5] = vzp[rr].y;
        const int iA = 2 * ih + q, iB = iA + 2;
        const int oyz = EDGE ? (((j == 0) << 2) | ((j == ny - 1) << 3) | ((k == 0) << 4) |
                                ((k == nz - 1) << 5))
                             : 0;
        const int oA = (iA == 0 ? 1 : 0) | oyz, oB = (iB == nx - 1 ? 2 : 0) | oyz;
        if (NORM)
        {
            T rA[6], rB[6], bb[6];
#pragma unroll
            for (int m = 0; m < 6; ++m)
            {
                rA[m] = nA[m];
                rB[m] = nB[m];
            }
            mg3_faces<T, false>(L, iA, j, k, bb);
            const double ra =
                fabs((double)mg3_residual(L, vf[rr].x, v0[rr].x, rA, bb, oA, iA, j, k, inhomog));
            const double rb =
                fabs((double)mg3_residual(L, vf[rr].y, v0[rr].y, rB, bb, oB, iB, j, k, inhomog));
            mres = nanmax(mres, nanmax(ra, rb));
        }
        V2 o;
        o.x = mg3_gs_value<T, false>(L, iA, j, k, oA, inhomog, inv_gamma, vf[rr].x, nA);
        o.y = mg3_gs_value<T, false>(L, iB, j, k, oB, inhomog, inv_gamma, vf[rr].y, nB);
        *reinterpret_cast<V2*>(xs + ih + (long long)nxh * (j + (long long)ny * k)) = o;
    }
}

// One colour of Gauss-Seidel (PROL and NORM as in k_mg_sweep3v).  CTA b
// owns tile b % ntiles (tiles of TMA_TX half-cells by TY rows) and the
// planes of z-chunk b / ntiles of nzc, so the CTAs sharing a chunk stream
// the same planes at the same time and read each other's halo rows from L2.
// Warp 8 is the producer: its lane 0 issues the loads, X plane p into slot
// ord % SX and F (and V) plane p into slot ord % SF, once the consumers have
// released the slot's previous use (empty barrier, 8 arrivals).  Warps 0-7
// wait for a slot's full barrier, update their pairs and release the slots
// of planes k-1 (X) and k (F) -- no CTA-wide barrier after the setup.
// tmx: the other colour of x, dims (nxh, ny, nz), box (TX + 2 XH, TY + 2, 1);
// tmf: this colour of f, box (TX, TY, 1); tmv (NORM): this colour of x,
// box (TX, TY, 1).  part[blockIdx.x] gets the CTA's residual max-norm (NORM).
template <typename T, bool PROL, bool NORM>
__global__ void __launch_bounds__(288, 2)
    k_mg_sweep3t(const __grid_constant__ MGOp<T> L, const __grid_constant__ CUtensorMap tmx,
                 const __grid_constant__ CUtensorMap tmf, const __grid_constant__ CUtensorMap tmv,
                 T* __restrict__ x, int color, int inhomog, T inv_gamma, GridDev gc,
                 const T* __restrict__ xc, double* __restrict__ part, int* __restrict__ err,
                 int nzc)
{
    using S = TmaSweepShape<T, NORM>;
    constexpr int SX = S::SX, SF = S::SF;
    VD_PDL_WAIT();
    __shared__ unsigned long long s_max;
    __shared__ int s_done;
    // the stop flag only changes between kernels: the whole CTA leaves
    if (L.stop && __ldg(L.stop)) return;
    extern __shared__ unsigned char dsm_raw[];
    unsigned char* base = reinterpret_cast<unsigned char*>(
        (reinterpret_cast<uintptr_t>(dsm_raw) + 127) & ~uintptr_t(127));
    unsigned char* xr = base;
    unsigned char* fr = base + SX * S::XSLOT;
    uint64_t* bars = reinterpret_cast<uint64_t*>(fr + SF * S::FSLOT);
    uint64_t* full_x = bars;
    uint64_t* empty_x = bars + SX;
    uint64_t* full_f = bars + 2 * SX;
    uint64_t* empty_f = bars + 2 * SX + SF;
    int* abort = reinterpret_cast<int*>(bars + S::NBAR);
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const GridDev& g = L.g;
    const int nxh = g.n[0] >> 1, ny = g.n[1], nz = g.n[2];
    const int tiles_x = (nxh + TMA_TX - 1) / TMA_TX, tiles_y = (ny + S::TY - 1) / S::TY;
    const int ntiles = tiles_x * tiles_y;
    const int tile = blockIdx.x % ntiles, chunk = blockIdx.x / ntiles;
    const int kb = (int)((long long)nz * chunk / nzc), ke = (int)((long long)nz * (chunk + 1) / nzc);
    const int x0 = (tile % tiles_x) * TMA_TX, y0 = (tile / tiles_x) * S::TY;
    if (tid == 0)
    {
        for (int b = 0; b < SX; ++b)
        {
            mbar_init(smem_u32(full_x + b), 1);
            mbar_init(smem_u32(empty_x + b), 8);
        }
        for (int b = 0; b < SF; ++b)
        {
            mbar_init(smem_u32(full_f + b), 1);
            mbar_init(smem_u32(empty_f + b), 8);
        }
        *abort = 0;
        s_max = 0ull;
        s_done = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    __syncthreads();
    if (w == 8)
    {
        // producer: X planes kb-1 .. ke, F (V) planes kb .. ke-1, X kept one
        // plane ahead of F in the issue order
        if (lane != 0) return;
        unsigned xo = 0, fo = 0;
        auto issue_x = [&](int p) -> bool {
            const int sl = (int)(xo % SX);
            if (xo >= (unsigned)SX &&
                !mbar_wait(smem_u32(empty_x + sl), ((xo / SX) - 1) & 1, abort))
                return false;
            const uint32_t fb = smem_u32(full_x + sl);
            mbar_expect_tx(fb, S::XBYTES);
            tma_load_3d(smem_u32(xr + sl * S::XSLOT), &tmx, fb, x0 - S::XH, y0 - 1, p);
            ++xo;
            return true;
        };
        auto issue_f = [&](int p) -> bool {
            const int sl = (int)(fo % SF);
            if (fo >= (unsigned)SF &&
                !mbar_wait(smem_u32(empty_f + sl), ((fo / SF) - 1) & 1, abort))
                return false;
            const uint32_t fb = smem_u32(full_f + sl);
            mbar_expect_tx(fb, S::FSLOT);
            tma_load_3d(smem_u32(fr + sl * S::FSLOT), &tmf, fb, x0, y0, p);
            if (NORM) tma_load_3d(smem_u32(fr + sl * S::FSLOT + S::FBYTES), &tmv, fb, x0, y0, p);
            ++fo;
            return true;
        };
        bool ok = issue_x(kb - 1) && issue_x(kb);
        for (int k = kb; ok && k < ke; ++k) ok = issue_x(k + 1) && issue_f(k);
        if (!ok)
        {
            *(volatile int*)abort = 1;
            atomicExch(err, 1);
            // let the copies still in flight land (bounded) before leaving
            for (int s = 0; s < SX; ++s)
                if (xo > (unsigned)s)
                {
                    const unsigned o = (xo - 1) - ((xo - 1 - s) % SX);
                    mbar_wait(smem_u32(full_x + s), (o / SX) & 1, nullptr);
                }
            for (int s = 0; s < SF; ++s)
                if (fo > (unsigned)s)
                {
                    const unsigned o = (fo - 1) - ((fo - 1 - s) % SF);
                    mbar_wait(smem_u32(full_f + s), (o / SF) & 1, nullptr);
                }
        }
        return;
    }
    // consumers
    T* __restrict__ xs = x + color * (g.ncell() >> 1);
    const bool in_h = inhomog != 0;
    double mres = 0.0;
    bool ok = mbar_wait(smem_u32(full_x + 0), 0, abort) && mbar_wait(smem_u32(full_x + 1), 0, abort);
    for (int k = kb; ok && k < ke; ++k)
    {
        const unsigned ox = (unsigned)(k - kb), of = ox; // X ordinal of plane k-1, F of k
        ok = mbar_wait(smem_u32(full_x + (ox + 2) % SX), ((ox + 2) / SX) & 1, abort) &&
             mbar_wait(smem_u32(full_f + of % SF), (of / SF) & 1, abort);
        if (!ok) break;
        const T* X0 = reinterpret_cast<const T*>(xr + (ox % SX) * S::XSLOT);
        const T* X1 = reinterpret_cast<const T*>(xr + ((ox + 1) % SX) * S::XSLOT);
        const T* X2 = reinterpret_cast<const T*>(xr + ((ox + 2) % SX) * S::XSLOT);
        const T* F = reinterpret_cast<const T*>(fr + (of % SF) * S::FSLOT);
        const T* V = reinterpret_cast<const T*>(fr + (of % SF) * S::FSLOT + S::FBYTES);
        const bool edge = k == 0 || k == nz - 1 || (y0 == 0 && w == 0) || y0 + w == ny - 1 ||
                          y0 + w + 8 == ny - 1;
        if (edge)
            tma_pairs<T, PROL, NORM, true>(L, X0, X1, X2, F, V, lane, w, x0, y0, k, color, in_h,
                                           inv_gamma, gc, xc, xs, mres);
        else
            tma_pairs<T, PROL, NORM, false>(L, X0, X1, X2, F, V, lane, w, x0, y0, k, color, in_h,
                                            inv_gamma, gc, xc, xs, mres);
        // this warp is done with plane k-1's X slot and plane k's F slot
        __syncwarp();
        if (lane == 0)
        {
            mbar_arrive(smem_u32(empty_x + ox % SX));
            mbar_arrive(smem_u32(empty_f + of % SF));
        }
    }
    if (!ok && lane == 0)
    {
        *(volatile int*)abort = 1;
        atomicExch(err, 1);
    }
    if (NORM)
    {
        // CTA max without a CTA barrier: warp max, shared atomic max of the
        // bit pattern (IEEE order of non-negative doubles; a NaN stays on
        // top), and the last warp to finish writes the partial
        mres = warp_max(mres);
        if (lane == 0)
        {
            atomicMax(&s_max, (unsigned long long)__double_as_longlong(mres));
            __threadfence_block();
            if (atomicAdd(&s_done, 1) == 7)
                part[blockIdx.x] = __longlong_as_double((long long)atomicMax(&s_max, 0ull));
        }
    }
}

} // namespace vd
