// k_umma.cu -- stage 1 of the m-domain search on the tcgen05 tensor cores.
//
// For one angular frequency m, X[col][rs] = 4 sum_k UA(rs,k) conj(UB(col,k)) is
// computed as a real GEMM with the particles on the UMMA M side and the (ref, shift)
// rows on the N side, for the planes m and P - m of a pair together so that the
// epilogue stores stage 2's packed spectrum Z(m), Z(P - m) (make_z) instead of X:
//   particle row  : [Br(k) | Bi(k) | 0]                       (K = Kp reals)
//   N row 2i      : [Ar(k) | Ai(k) | 0]   -> column 2i   = Re X
//   N row 2i+1    : [Ai(k) | -Ar(k) | 0]  -> column 2i+1 = Im X
// so the accumulator's column pair (2i, 2i+1) is the complex X of rs = i.  Every
// FP32 operand value v is split into bf16 hi = rn(v) and lo = rn(v - hi); the
// product is accumulated in FP32 TMEM as hi*hi + hi*lo + lo*hi (three
// kind::f16 MMAs per 16-wide K step).  Operands are pre-tiled in global memory in
// the canonical no-swizzle K-major layout ([chunk of 8 K][row][8 K]), each tile one
// contiguous block, so that one bulk copy (cp.async.bulk) per tile lands it ready for
// the UMMA descriptors (a tiled tensor copy of this layout would move 16-byte rows).
//
// Kernel roles (320 threads, one persistent CTA per SM):
//   warp 0   producer: both planes' particle tiles once per work item (plane pair,
//            particle tile), one at a time through a single shared-memory tile, then the
//            ring of row tiles (32 (ref, shift) rows of each plane per stage)
//   warp 1   TMEM allocation and the single MMA-issuing thread; accumulators are
//            double buffered, each buffer 2 x 64 TMEM columns (one per plane); each
//            particle tile is copied into TMEM (tcgen05.cp, 8 columns per 16-wide K step)
//            and the MMAs read their A operand from there, so shared memory holds one
//            particle tile in transit and a deeper ring of row tiles; before an item's
//            copies replace the particle tiles the previous item's MMAs are waited for
//   warps 2-9 epilogue, two per TMEM lane quadrant (warp w: quadrant w mod 4, half
//            (w - 2) / 4 of the tile): tcgen05.ld of its 16 (ref, shift) rows of both
//            planes' accumulators, Z(m) and Z(P - m) into two 128B-swizzled staging tiles,
//            written out with one TMA bulk store each to Z[plane][col][rs]
// The factor 4 of X is carried by the packed particle operand (exact in BF16).
// Every mbarrier wait is bounded; on timeout the kernel records an error code,
// drains its own outstanding copies (bounded), frees its TMEM and returns.  The pipeline
// waits take their poll limit from the launch (pftcc_set_wait_limit); the drains keep the
// full limit, so a short limit never leaves a copy or an MMA running after the exit.
#include "pftcc_internal.cuh"

#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cstdio>

namespace pftcc {

constexpr int U_BM = 128;        // particles per tile (UMMA M)
constexpr int U_BN = 64;         // N columns per plane and tile = 32 rs x (re, im)
constexpr int U_RS = 32;         // (ref, shift) rows per tile
constexpr int U_THREADS = 320;
constexpr int ACC_COLS = 2 * 2 * U_BN;        // TMEM: two accumulator buffers x two planes x U_BN columns
constexpr int TMEM_COLS = 512;                // accumulators, then both planes' particle tiles (A operands)
constexpr long long WAIT_LIMIT = 20000000;   // polls of a bounded wait (~seconds)
constexpr int STAGE_TILE = 32 * 128;          // one staged 32-row x 128-byte block
constexpr int STAGE_BYTES = 8 * 2 * STAGE_TILE;   // eight epilogue warps x (Z(m), Z(P-m)) blocks

struct UmmaParams {
    int M;              // m planes of the packed operands (P + 1)
    int Kp;             // padded real K per operand part (multiple of 16)
    int KC;             // 8-element chunks per operand row: 2*Kp/8 (hi then lo)
    int ptiles_m;       // particle tiles per m plane in the packed particle operand
    int rtiles_m;       // rs tiles per m plane in the packed row operand
    int stages;         // N-tile ring depth (each stage holds the row tiles of both planes)
    const __nv_bfloat16 *P16;   // packed particle operand, one contiguous tile per (m, particle tile)
    const __nv_bfloat16 *R16;   // packed row operand, one contiguous tile per (m, rs tile)
    const S1Wave *waves;        // the launch's waves (device), items of wave w from waves[w].item0
    const CUtensorMap *maps;    // each wave's Z as a tensor map (device, 64-byte aligned)
    int nwaves, nitems;
    int *err;           // device error word (0 = ok)
    long long wait_limit;   // polls of a pipeline wait before the kernel gives up (the drains of
                            // copies and MMAs already issued always use WAIT_LIMIT)
};

// ---- PTX wrappers --------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, int count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_try(uint64_t *bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// bounded wait: false after `limit` polls or when another role has aborted
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, volatile int *abort_flag, long long limit)
{
    for (long long i = 0; i < limit; ++i) {
        if (mbar_try(bar, parity)) return true;
        if (*abort_flag) return false;
        if (i > 64) __nanosleep(64);
    }
    return false;
}

// bulk copy of one pre-tiled operand tile (contiguous in global memory, already in the
// UMMA canonical layout) into shared memory, completing on the mbarrier's transaction count;
// both addresses 16-byte aligned, size a multiple of 16
__device__ __forceinline__ void bulk_load(void *dst, const void *src, uint32_t bytes, uint64_t *bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 :
                 : "r"(smem_u32(dst)), "l"((uint64_t)src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

// TMA bulk store of a 2-D box from shared memory (bulk-group completion)
__device__ __forceinline__ void tma_store_2d(const CUtensorMap *map, const void *src, int c0, int c1)
{
    asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.bulk_group [%0, {%2, %3}], [%1];"
                 :
                 : "l"((uint64_t)map), "r"(smem_u32(src)), "r"(c0), "r"(c1)
                 : "memory");
}

__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo)
{
    // canonical K-major layout without swizzle: start >> 4, LBO (K direction) >> 4,
    // SBO (8-row groups) >> 4, descriptor version 1, layout type 0
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFF);
    d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
    d |= (uint64_t)1 << 46;
    return d;
}

__device__ __forceinline__ void umma_bf16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t acc)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
        :
        : "r"(d_tmem), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc));
}

// the same MMA with the A operand read from tensor memory (K-major, one row per lane)
__device__ __forceinline__ void umma_bf16_at(uint32_t d_tmem, uint32_t a_tmem, uint64_t bdesc, uint32_t idesc,
                                             uint32_t acc)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %3, p;\n\t}\n"
        :
        : "r"(d_tmem), "r"(a_tmem), "l"(bdesc), "r"(idesc), "r"(acc));
}

// copy of a 128-row x 256-bit block (16 bf16 per row) from shared memory (matrix descriptor)
// into tensor memory: row i to lane i, 8 columns
__device__ __forceinline__ void tmem_cp_128x256b(uint32_t taddr, uint64_t sdesc)
{
    asm volatile("tcgen05.cp.cta_group::1.128x256b [%0], %1;" ::"r"(taddr), "l"(sdesc));
}

__device__ __forceinline__ void umma_commit(uint64_t *bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&r)[32])
{
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
        "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
}

// completes every tcgen05.ld this thread issued before it
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// ---- the GEMM ------------------------------------------------------------------------
// the wave of work item w: the cursor `wv` only moves forward, as every role walks its items in
// increasing order
__device__ __forceinline__ void wave_of(const UmmaParams &up, int w, int &wv)
{
    while (wv + 1 < up.nwaves && w >= __ldg(&up.waves[wv + 1].item0)) ++wv;
}

__global__ void __launch_bounds__(U_THREADS, 1) k_umma_stage1(const __grid_constant__ UmmaParams up)
{
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    unsigned char *smem = (unsigned char *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    const uint32_t a_bytes = (uint32_t)U_BM * up.KC * 16;     // one plane's particle tile
    const uint32_t b_bytes = (uint32_t)U_BN * up.KC * 16;     // one plane's row tile
    unsigned char *sA = smem;                                  // one plane's particle tile (on its way to TMEM)
    unsigned char *sB = smem + a_bytes;                        // [stages][2 planes] row tiles
    unsigned char *stg = sB + (size_t)up.stages * 2 * b_bytes; // [4 warps][2][32][128 B], 1024-B aligned
    uint64_t *bars = reinterpret_cast<uint64_t *>(stg + STAGE_BYTES);
    uint64_t *full = bars;                    // [stages]
    uint64_t *empty = bars + up.stages;       // [stages]
    uint64_t *a_full = bars + 2 * up.stages;
    uint64_t *a_empty = a_full + 1;
    uint64_t *t_full = a_full + 2;            // [2]
    uint64_t *t_empty = a_full + 4;           // [2]
    uint64_t *mma_done = a_full + 6;
    uint64_t *item_done = a_full + 7;          // an item's MMAs finished (its TMEM A may be replaced)
    volatile int *abort_flag = reinterpret_cast<volatile int *>(a_full + 8);
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(a_full + 9);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        for (int s = 0; s < up.stages; ++s) { mbar_init(full + s, 1); mbar_init(empty + s, 1); }
        mbar_init(a_full, 1);
        mbar_init(a_empty, 1);
        mbar_init(t_full, 1); mbar_init(t_full + 1, 1);
        mbar_init(t_empty, 256); mbar_init(t_empty + 1, 256);
        mbar_init(mma_done, 1);
        mbar_init(item_done, 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem_base = *tmem_slot;
    // work item = (plane pair mp, particle tile): planes mA = mp and mB = P - mp (mp = 0
    // pairs plane 0 with plane P, mp = P/2 of an even P pairs the plane with itself)
    const int P = up.M - 1;
    const int nitems = up.nitems;
    auto fail = [&](int code) {
        if (!*abort_flag) atomicCAS(up.err, 0, code);
        *abort_flag = 1;
    };

    if (warp == 0 && lane == 0) {
        // ------------------------------------------------------------ TMA producer
        long long itb = 0, na = 0;     // row-tile stages and particle tiles loaded
        bool ok = true;
        int wv = 0;
        for (int w = blockIdx.x; w < nitems && ok; w += gridDim.x) {
            wave_of(up, w, wv);
            const S1Wave *W = up.waves + wv;
            const int n_pt = __ldg(&W->n_ptiles), wi = w - __ldg(&W->item0);
            const int mp = wi / n_pt, pt = wi - mp * n_pt;
            const int pt0 = __ldg(&W->ptile0), rt0 = __ldg(&W->rtile0), n_rt = __ldg(&W->n_rtiles);
            const int pm[2] = {mp, mp == 0 ? P : P - mp};
            // both planes' particle tiles, one at a time through sA (the MMA issuer copies each to TMEM)
            for (int h = 0; h < 2; ++h, ++na) {
                if (na > 0 && !mbar_wait(a_empty, (uint32_t)((na - 1) & 1), abort_flag, up.wait_limit)) { fail(1); ok = false; break; }
                mbar_expect_tx(a_full, a_bytes);
                bulk_load(sA, up.P16 + (size_t)(pm[h] * up.ptiles_m + pt0 + pt) * (a_bytes / 2), a_bytes, a_full);
            }
            if (!ok) break;
            for (int j = 0; j < n_rt; ++j, ++itb) {
                const int s = (int)(itb % up.stages);
                if (itb >= up.stages && !mbar_wait(empty + s, (uint32_t)((itb / up.stages - 1) & 1), abort_flag, up.wait_limit)) {
                    fail(2); ok = false; break;
                }
                mbar_expect_tx(full + s, 2 * b_bytes);
                for (int h = 0; h < 2; ++h)
                    bulk_load(sB + ((size_t)s * 2 + h) * b_bytes,
                              up.R16 + (size_t)(pm[h] * up.rtiles_m + rt0 + j) * (b_bytes / 2), b_bytes, full + s);
            }
        }
        // drain: every issued copy must land before the CTA exits
        for (long long t = (itb > up.stages ? itb - up.stages : 0); t < itb; ++t) {
            const int s = (int)(t % up.stages);
            for (long long i = 0; i < WAIT_LIMIT && !mbar_try(full + s, (uint32_t)((t / up.stages) & 1)); ++i)
                __nanosleep(64);
        }
        if (na > 0)
            for (long long i = 0; i < WAIT_LIMIT && !mbar_try(a_full, (uint32_t)((na - 1) & 1)); ++i) __nanosleep(64);
    } else if (warp == 1 && lane == 0) {
        // ------------------------------------------------------------ MMA issuer
        // instruction descriptor: F32 accumulate, BF16 x BF16, both K-major, N=64, M=128
        const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(U_BN >> 3) << 17) |
                               ((uint32_t)(U_BM >> 4) << 24);
        const uint32_t a_base = smem_u32(sA), b_base0 = smem_u32(sB);
        const int ksteps = up.Kp / 16, lo_off = up.Kp / 8;
        const int acol = up.KC * 4;              // TMEM columns of one plane's particle tile (8 per 16-wide K step)
        long long itb = 0, tacc = 0, na = 0;
        int ii = 0, wv = 0;
        bool ok = true;
        for (int w = blockIdx.x; w < nitems && ok; w += gridDim.x, ++ii) {
            wave_of(up, w, wv);
            const int n_rt = __ldg(&up.waves[wv].n_rtiles);
            if (ii > 0) {
                // the previous item's MMAs read the TMEM particle tiles: let them finish first
                umma_commit(item_done);
                if (!mbar_wait(item_done, (uint32_t)((ii - 1) & 1), abort_flag, up.wait_limit)) { fail(7); ok = false; break; }
            }
            for (int h = 0; h < 2; ++h, ++na) {
                if (!mbar_wait(a_full, (uint32_t)(na & 1), abort_flag, up.wait_limit)) { fail(3); ok = false; break; }
                tc_fence_after();
                const uint32_t tcol = tmem_base + ACC_COLS + (uint32_t)(h * acol);
                for (int st = 0; st < up.KC / 2; ++st)
                    tmem_cp_128x256b(tcol + 8 * st, umma_desc(a_base + (uint32_t)(2 * st) * (U_BM * 16), U_BM * 16, 128));
                umma_commit(a_empty);            // sA reusable once the copies have read it
            }
            if (!ok) break;
            for (int j = 0; j < n_rt; ++j, ++itb, ++tacc) {
                const int s = (int)(itb % up.stages);
                if (!mbar_wait(full + s, (uint32_t)((itb / up.stages) & 1), abort_flag, up.wait_limit)) { fail(4); ok = false; break; }
                const int acc = (int)(tacc & 1);
                if (tacc >= 2 && !mbar_wait(t_empty + acc, (uint32_t)((tacc / 2 - 1) & 1), abort_flag, up.wait_limit)) {
                    fail(5); ok = false; break;
                }
                tc_fence_after();
                // accumulator buffer acc: columns [0, 64) plane mA, [64, 128) plane mB
                for (int h = 0; h < 2; ++h) {
                    const uint32_t d_tmem = tmem_base + (uint32_t)(acc * 2 * U_BN + h * U_BN);
                    const uint32_t at = tmem_base + ACC_COLS + (uint32_t)(h * acol);   // this plane's particle tile
                    const uint32_t b_base = b_base0 + ((uint32_t)s * 2 + h) * b_bytes;
                    for (int ks = 0; ks < ksteps; ++ks) {
#pragma unroll
                        for (int prod = 0; prod < 3; ++prod) {
                            const int ac = (prod == 2 ? lo_off : 0) + 2 * ks;   // lo(A) * hi(B)
                            const int bc = (prod == 1 ? lo_off : 0) + 2 * ks;   // hi(A) * lo(B)
                            const uint64_t bd = umma_desc(b_base + (uint32_t)bc * (U_BN * 16), U_BN * 16, 128);
                            umma_bf16_at(d_tmem, at + (uint32_t)(ac * 4), bd, idesc, (ks > 0 || prod > 0) ? 1u : 0u);
                        }
                    }
                }
                umma_commit(empty + s);      // N stage reusable once these MMAs finish
                umma_commit(t_full + acc);   // accumulator ready for the epilogue
            }
        }
        umma_commit(mma_done);
        for (long long i = 0; i < WAIT_LIMIT && !mbar_try(mma_done, 0); ++i) __nanosleep(64);
    } else if (warp >= 2) {
        // ------------------------------------------------------------ epilogue
        const int q = warp & 3;                       // TMEM lane quadrant of this warp
        const int c = (warp - 2) >> 2;                // its half of the tile: complex rs 16c .. 16c + 15
        unsigned char *stg_w = stg + (size_t)(warp - 2) * 2 * STAGE_TILE;   // boxes of Z(mA), Z(mB)
        long long tacc = 0;
        bool ok = true;
        const int N = 2 * P;
        int wv = 0;
        for (int w = blockIdx.x; w < nitems && ok; w += gridDim.x) {
            wave_of(up, w, wv);
            const S1Wave *W = up.waves + wv;
            const CUtensorMap *tmX = up.maps + wv;
            const int n_pt = __ldg(&W->n_ptiles), wi = w - __ldg(&W->item0);
            const int mp = wi / n_pt, pt = wi - mp * n_pt;
            const int n_rt = __ldg(&W->n_rtiles), xcols = __ldg(&W->xcols);
            const int mA = mp, mB = mp == 0 ? P : P - mp;
            const bool two = mp != 0 && mB != mA;      // a second output plane
            const float2 wA = wn_of(mA, N), wB = wn_of(mB, N);
            // rows of this warp: particles 32q .. 32q+31 of the tile = box rows of Z's tensor map
            const int yA = mA * xcols + pt * U_BM + 32 * q, yB = (two ? mB : 0) * xcols + pt * U_BM + 32 * q;
            for (int j = 0; j < n_rt; ++j, ++tacc) {
                const int acc = (int)(tacc & 1);
                // warp-uniform outcome: the .sync.aligned TMEM loads below must run on all 32 lanes
                const bool got = __all_sync(0xffffffffu, mbar_wait(t_full + acc, (uint32_t)((tacc / 2) & 1), abort_flag, up.wait_limit));
                if (!got) { if (lane == 0) fail(6); ok = false; break; }
                tc_fence_after();
                // both planes' 64 columns in flight at once, one wait; the accumulator is handed
                // back to the MMA issuer before Z is formed and stored
                uint32_t ra[32], rb[32];     // this half's 32 columns (16 complex) of each plane
                tmem_ld32(tmem_base + ((uint32_t)(32 * q) << 16) + (uint32_t)(acc * 2 * U_BN + 32 * c), ra);
                tmem_ld32(tmem_base + ((uint32_t)(32 * q) << 16) + (uint32_t)(acc * 2 * U_BN + U_BN + 32 * c), rb);
                tmem_wait_ld();
                tc_fence_before();
                mbar_arrive(t_empty + acc);
                {
                    // the staging boxes of the previous chunk must have been read out
                    if (lane == 0) asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
                    __syncwarp();
                    // row `lane` of each box, 16-byte chunk e at position e ^ (lane & 7) (128B swizzle)
                    float4 *rowA = reinterpret_cast<float4 *>(stg_w + lane * 128);
                    float4 *rowB = reinterpret_cast<float4 *>(stg_w + STAGE_TILE + lane * 128);
#pragma unroll
                    for (int e = 0; e < 8; ++e) {
                        float2 xa0 = make_float2(__uint_as_float(ra[4 * e]), __uint_as_float(ra[4 * e + 1]));
                        float2 xa1 = make_float2(__uint_as_float(ra[4 * e + 2]), __uint_as_float(ra[4 * e + 3]));
                        float2 xb0 = make_float2(__uint_as_float(rb[4 * e]), __uint_as_float(rb[4 * e + 1]));
                        float2 xb1 = make_float2(__uint_as_float(rb[4 * e + 2]), __uint_as_float(rb[4 * e + 3]));
                        if (mp == 0) {                 // X(0) and X(P) are real
                            xa0.y = xa1.y = xb0.y = xb1.y = 0.f;
                        }
                        const float2 za0 = make_z(xa0, xb0, wA), za1 = make_z(xa1, xb1, wA);
                        rowA[e ^ (lane & 7)] = make_float4(za0.x, za0.y, za1.x, za1.y);
                        if (two) {
                            const float2 zb0 = make_z(xb0, xa0, wB), zb1 = make_z(xb1, xa1, wB);
                            rowB[e ^ (lane & 7)] = make_float4(zb0.x, zb0.y, zb1.x, zb1.y);
                        }
                    }
                    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                    __syncwarp();
                    if (lane == 0) {
                        // x in floats: complex rs = j * U_RS + 16 c, two floats each (a multiple of 32)
                        const int x = 2 * (j * U_RS + 16 * c);
                        tma_store_2d(tmX, stg_w, x, yA);
                        if (two) tma_store_2d(tmX, stg_w + STAGE_TILE, x, yB);
                        asm volatile("cp.async.bulk.commit_group;" ::: "memory");
                    }
                }
            }
        }
        // every store has finished reading shared memory and writing X before the CTA exits
        if (lane == 0) asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
        __syncwarp();
    }
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_base), "r"(TMEM_COLS));
    }
}

// ---- operand packing -------------------------------------------------------------------
__device__ __forceinline__ void split_bf16(float v, __nv_bfloat16 &hi, __nv_bfloat16 &lo)
{
    hi = __float2bfloat16_rn(v);
    lo = __float2bfloat16_rn(v - __bfloat162float(hi));
}

__device__ __forceinline__ uint32_t bf16x2_bits(__nv_bfloat16 a, __nv_bfloat16 b)
{
    return (uint32_t)__bfloat16_as_ushort(a) | ((uint32_t)__bfloat16_as_ushort(b) << 16);
}

// one thread per 16-byte chunk pair: the 8 K values kk = 8c .. 8c + 7 (c < Kp / 8) of one
// operand row, given by val(kk), split into the hi chunk c and the lo chunk c + Kp / 8 of the
// tile layout [chunk][rows][8]
template <class Val>
__device__ __forceinline__ void pack_chunk(const Val &val, int c, int half, int nrows, int i, __nv_bfloat16 *tile)
{
    uint32_t hw[4], lw[4];
#pragma unroll
    for (int el = 0; el < 8; el += 2) {
        __nv_bfloat16 h0, l0, h1, l1;
        split_bf16(val(8 * c + el), h0, l0);
        split_bf16(val(8 * c + el + 1), h1, l1);
        hw[el >> 1] = bf16x2_bits(h0, h1);
        lw[el >> 1] = bf16x2_bits(l0, l1);
    }
    uint4 *t4 = reinterpret_cast<uint4 *>(tile);
    t4[(size_t)c * nrows + i] = make_uint4(hw[0], hw[1], hw[2], hw[3]);
    t4[(size_t)(c + half) * nrows + i] = make_uint4(lw[0], lw[1], lw[2], lw[3]);
}

// (ref, shift) rows -> R16[m][rt][chunk][U_BN][8]: U_RS rows = U_BN N-rows per tile, N-row
// 2i + 0 = [Ar | Ai | 0], 2i + 1 = [Ai | -Ar | 0] of row i
__global__ void k_pack_rows(int M, int Ks, int Kp, int KC, int rtiles, int rows_pad, const float2 *__restrict__ UA,
                            __nv_bfloat16 *__restrict__ R16)
{
    const int half = Kp / 8;
    const size_t per_tile = (size_t)KC * U_BN * 8;
    const size_t total = (size_t)M * rtiles * half * U_BN;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(e % U_BN);
        const size_t q = e / U_BN;
        const int c = (int)(q % half);
        const size_t tile = q / half;
        const int m = (int)(tile / rtiles), rt = (int)(tile - (size_t)m * rtiles);
        const int rs = rt * U_RS + (i >> 1), kind = i & 1;
        const float2 *src = UA + ((size_t)m * rows_pad + rs) * Ks;
        auto val = [&](int kk) {
            if (kk >= 2 * Ks || rs >= rows_pad) return 0.f;
            const float2 a = src[kk < Ks ? kk : kk - Ks];
            return kind == 0 ? (kk < Ks ? a.x : a.y) : (kk < Ks ? a.y : -a.x);
        };
        pack_chunk(val, c, half, U_BN, i, R16 + tile * per_tile);
    }
}

// particle columns [c0, c0 + ptiles*128) -> P16[m][pt][chunk][128][8], row = [4 Br | 4 Bi | 0]
__global__ void k_pack_cols(int M, int Ks, int Kp, int KC, int ptiles, int cols_pad, int c0,
                            const float2 *__restrict__ UB, __nv_bfloat16 *__restrict__ P16)
{
    const int half = Kp / 8;
    const size_t per_tile = (size_t)KC * U_BM * 8;
    const size_t total = (size_t)M * ptiles * half * U_BM;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(e % U_BM);
        const size_t q = e / U_BM;
        const int c = (int)(q % half);
        const size_t tile = q / half;
        const int m = (int)(tile / ptiles), pt = (int)(tile - (size_t)m * ptiles);
        const int col = c0 + pt * U_BM + i;
        const float2 *src = UB + ((size_t)m * cols_pad + col) * Ks;
        auto val = [&](int kk) {
            if (kk >= 2 * Ks || col >= cols_pad) return 0.f;
            const float2 b = src[kk < Ks ? kk : kk - Ks];
            return 4.f * (kk < Ks ? b.x : b.y);      // X = 4 sum_k ...: the power of two splits exactly
        };
        pack_chunk(val, c, half, U_BM, i, P16 + tile * per_tile);
    }
}

// ---- host side --------------------------------------------------------------------------
static PFN_cuTensorMapEncodeTiled_v12000 get_encode()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        cudaDriverEntryPointQueryResult q;
        void *p = nullptr;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
    }
    return fn;
}

// X[M][xcols][xrows] float2 as a 2-D FP32 tensor: x = 2 * rs + (re, im), y = m * xcols + col;
// boxes of 32 floats (128 B) x 32 rows, 128-byte swizzle (the staging layout of the epilogue)
static int make_xmap(pftcc_handle *h, CUtensorMap *map, void *X, int xrows, int xcols, int nplanes)
{
    auto enc = get_encode();
    if (!enc) return set_err(h, PFTCC_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
    if (((uintptr_t)X & 15) != 0) return set_err(h, PFTCC_ERR_ARG, "X base not 16-byte aligned");
    if (xrows % 64 != 0 || (long long)xcols * nplanes >= (1LL << 31))
        return set_err(h, PFTCC_ERR_ARG, "umma stage 1: X extents outside the tensor-map limits");
    cuuint64_t dims[2] = {(cuuint64_t)2 * xrows, (cuuint64_t)xcols * nplanes};
    cuuint64_t strides[1] = {(cuuint64_t)xrows * sizeof(float2)};
    cuuint32_t box[2] = {32, 32};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, X, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                     CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_NONE, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return set_err(h, PFTCC_ERR_CUDA, "cuTensorMapEncodeTiled (X) failed: " + std::to_string((int)r));
    return PFTCC_OK;
}

static UmmaState &ustate(pftcc_handle *h) { return h->ws.umma; }

int umma_stage1(pftcc_handle *h, int M, int Ks, const float2 *UA, int rs0, int nrs_w, int rows_pad, const float2 *UB,
                int c0, int ncols_w, int cols_pad, float2 *X, int prepare, int parity_group)
{
    (void)parity_group;
    SearchWS &ws = h->ws;
    UmmaState &us = ustate(h);
    const int Kp = (2 * Ks + 15) / 16 * 16;
    const int KC = 2 * Kp / 8;
    cudaError_t e;
    if (prepare) {
        const int rtiles = rows_pad / U_RS;
        const int ptiles = (ncols_w + U_BM - 1) / U_BM;
        const size_t r16 = (size_t)M * rtiles * KC * U_BN * 8, p16 = (size_t)M * ptiles * KC * U_BM * 8;
        int st = ensure(h, (void **)&ws.A16, &ws.A16_elems, r16 * sizeof(__nv_bfloat16), "packed rows");
        if (st) return st;
        st = ensure(h, (void **)&ws.B16, &ws.B16_elems, p16 * sizeof(__nv_bfloat16), "packed particles");
        if (st) return st;
        us.Kp = Kp; us.KC = KC; us.rtiles = rtiles; us.ptiles = ptiles; us.group_c0 = c0;
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&us.sms, cudaDevAttrMultiProcessorCount, dev);
        PFTCC_LAUNCH(h);
        KTimer kt(h, PFTCC_K_PACK);
        k_pack_rows<<<us.sms * 8, 256, 0, h->stream>>>(M, Ks, Kp, KC, rtiles, rows_pad, UA, ws.A16);
        if ((e = cudaGetLastError()) != cudaSuccess) return cuda_err(h, e, "pack rows");
        PFTCC_LAUNCH(h);
        k_pack_cols<<<us.sms * 8, 256, 0, h->stream>>>(M, Ks, Kp, KC, ptiles, cols_pad, c0, UB, ws.B16);
        if ((e = cudaGetLastError()) != cudaSuccess) return cuda_err(h, e, "pack cols");
        return PFTCC_OK;
    }
    if (rs0 % U_RS || nrs_w % U_RS || (c0 - us.group_c0) % U_BM || ncols_w % U_BM)
        return set_err(h, PFTCC_ERR_ARG, "umma stage 1: wave not tile aligned");
    std::vector<S1Wave> w(1);
    w[0] = S1Wave{X, rs0 / U_RS, nrs_w / U_RS, (c0 - us.group_c0) / U_BM, ncols_w / U_BM, 0, 0, 0, 0};
    return umma_stage1_waves(h, M, w);
}

int umma_stage1_waves(pftcc_handle *h, int M, std::vector<S1Wave> &waves)
{
    SearchWS &ws = h->ws;
    UmmaState &us = ustate(h);
    const int Kp = us.Kp, KC = us.KC;
    cudaError_t e;
    const int nw = (int)waves.size();
    if (nw == 0) return PFTCC_OK;
    const int npairs = (M - 1) / 2 + 1;        // plane pairs (m, P - m)
    long long nitems = 0;
    for (S1Wave &w : waves) {
        if (w.n_rtiles <= 0 || w.n_ptiles <= 0 || w.rtile0 < 0 || w.ptile0 < 0 || w.rtile0 + w.n_rtiles > us.rtiles ||
            w.ptile0 + w.n_ptiles > us.ptiles)
            return set_err(h, PFTCC_ERR_ARG, "umma stage 1: wave outside the packed operands");
        w.item0 = (int)nitems;
        w.xrows = w.n_rtiles * U_RS;
        w.xcols = w.n_ptiles * U_BM;
        nitems += (long long)npairs * w.n_ptiles;
    }
    if (nitems >= (1LL << 31)) return set_err(h, PFTCC_ERR_ARG, "umma stage 1: too many work items");
    if (((uintptr_t)ws.A16 & 15) != 0 || ((uintptr_t)ws.B16 & 15) != 0)
        return set_err(h, PFTCC_ERR_ARG, "umma stage 1: packed operands not 16-byte aligned");
    // the waves' Z tensor maps, and both tables on the device (stream-ordered after any launch that
    // still reads the previous contents)
    std::vector<CUtensorMap> maps(nw);
    for (int i = 0; i < nw; ++i) {
        int st = make_xmap(h, &maps[i], waves[i].X, waves[i].xrows, waves[i].xcols, M - 1);   // Z has P = M - 1 planes
        if (st) return st;
    }
    if (us.waves_cap < nw) {
        dev_free(h, us.d_waves);
        dev_free(h, us.d_maps);
        us.d_waves = nullptr;
        us.d_maps = nullptr;
        us.waves_cap = 0;
        const int cap = std::max(nw, 16);
        int st = dev_alloc(h, (void **)&us.d_waves, (size_t)cap * sizeof(S1Wave), "stage-1 waves");
        if (st) return st;
        st = dev_alloc(h, &us.d_maps, (size_t)cap * sizeof(CUtensorMap), "stage-1 tensor maps");
        if (st) return st;
        if (((uintptr_t)us.d_maps & 63) != 0) return set_err(h, PFTCC_ERR_CUDA, "stage-1 tensor maps not 64-byte aligned");
        us.waves_cap = cap;
    }
    {
        int st = stage_upload(h, us.d_waves, waves.data(), (size_t)nw * sizeof(S1Wave), "stage-1 waves");
        if (st) return st;
        st = stage_upload(h, us.d_maps, maps.data(), (size_t)nw * sizeof(CUtensorMap), "stage-1 tensor maps");
        if (st) return st;
    }
    UmmaParams up{};
    up.M = M; up.Kp = Kp; up.KC = KC;
    up.ptiles_m = us.ptiles; up.rtiles_m = us.rtiles;
    const size_t a_bytes = (size_t)U_BM * KC * 16, b_bytes = (size_t)U_BN * KC * 16;
    // 1 KiB alignment slack, one particle tile on its way to TMEM, the N ring (per stage both
    // planes' row tiles), 512 B of barriers and the epilogue's staging tiles; both planes'
    // particle tiles sit in TMEM beside the accumulators
    const size_t tail = 512 + STAGE_BYTES;
    if (ACC_COLS + 2 * 4 * KC > TMEM_COLS)
        return set_err(h, PFTCC_ERR_UNSUPPORTED, "umma stage 1: particle tiles too large for tensor memory");
    int stages = h->tune.s1_stages >= 2 && h->tune.s1_stages <= 4 ? h->tune.s1_stages : 4;
    while (stages > 1 && 1024 + a_bytes + stages * 2 * b_bytes + tail > 227 * 1024) --stages;
    if (1024 + a_bytes + stages * 2 * b_bytes + tail > 227 * 1024)
        return set_err(h, PFTCC_ERR_UNSUPPORTED, "umma stage 1: operands too large for shared memory");
    up.stages = stages;
    up.P16 = ws.B16; up.R16 = ws.A16;
    up.waves = us.d_waves;
    up.maps = reinterpret_cast<const CUtensorMap *>(us.d_maps);
    up.nwaves = nw;
    up.nitems = (int)nitems;
    up.err = us.err;
    up.wait_limit = h->wait_limit > 0 ? h->wait_limit : WAIT_LIMIT;
    const size_t smem = 1024 + a_bytes + stages * 2 * b_bytes + tail;
    if ((e = smem_limit((const void *)k_umma_stage1, smem)) != cudaSuccess)
        return cuda_err(h, e, "umma attr");
    const int grid = (int)std::min<long long>(nitems, us.sms);
    PFTCC_LAUNCH(h);
    KTimer kt(h, PFTCC_K_STAGE1);
    k_umma_stage1<<<grid, U_THREADS, smem, h->stream>>>(up);
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_err(h, e, "umma stage 1 launch");
    return PFTCC_OK;
}

// the device error word of the bounded waits, zeroed once when it is allocated: it then holds the
// first expiry of any search since the last umma_check, graph replays included
int umma_reset(pftcc_handle *h)
{
    UmmaState &us = ustate(h);
    if (us.err) return PFTCC_OK;
    const int st = dev_alloc(h, (void **)&us.err, sizeof(int), "umma error word");
    if (st) return st;
    const cudaError_t e = cudaMemsetAsync(us.err, 0, sizeof(int), h->stream);
    return e == cudaSuccess ? PFTCC_OK : cuda_err(h, e, "umma error word reset");
}

// reads the error word after the stream has drained and clears it when a wait had expired
int umma_check(pftcc_handle *h)
{
    UmmaState &us = ustate(h);
    if (!us.err) return PFTCC_OK;
    int v = 0;
    cudaError_t e = cudaMemcpyAsync(&v, us.err, sizeof(int), cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e == cudaSuccess && v != 0) e = cudaMemsetAsync(us.err, 0, sizeof(int), h->stream);
    if (e != cudaSuccess) return cuda_err(h, e, "umma error word");
    if (v != 0) return set_err(h, PFTCC_ERR_TIMEOUT, "tcgen05 stage 1: bounded wait expired (code " + std::to_string(v) + ")");
    return PFTCC_OK;
}

void umma_free(pftcc_handle *h)
{
    UmmaState &us = ustate(h);
    dev_free(h, us.err);
    dev_free(h, us.d_waves);
    dev_free(h, us.d_maps);
    us.err = nullptr;
    us.d_waves = nullptr;
    us.d_maps = nullptr;
    us.waves_cap = 0;
}

}  // namespace pftcc
