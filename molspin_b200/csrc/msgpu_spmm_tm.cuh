// msgpu_spmm_tm.cuh -- quartet SpMM of the complex64 Lanczos form with its
// inputs staged in tensor memory (TMEM) and the block arithmetic on the FP32
// pipes.
//
// U = s_j H w_j over a trajectory group (the H v product of
// SpinSpace::LanczosProcess / ArnoldiProcess, SpinSpace_operators.cpp:1362,
// applied per column by HSPropagator::Step, HSPropagator.cpp:64-78).
//
// Why TMEM.  The SIMT quartet SpMM (k_lanczos_apply_np) gathers 1 + P input
// quartets per output quartet through the L1 data path, and the LSU
// wavefronts of those gathers are its limit, whether they hit L1 or not.
// Here no input passes through the LSU: 2D tensor-map boxes bring the inputs
// into shared memory, tcgen05.cp moves them into TMEM, and tcgen05.ld hands
// each thread its trajectory pair's values.  The 4x4 blocks are applied with
// the packed FP32x2 arithmetic of the SIMT kernels (quartet_block), their
// values read from shared memory.
//
// Structure used (checked on the host by build_tc, as for the tensor-core
// SpMM): for radical pairs whose other spins are all spin-1/2, the quartet
// index q is a P-bit number, H couples quartet q only to itself and to
// q ^ 2^p, and the block of flip p depends only on p and on bit p of the
// output quartet.
//
// Work split.  Persistent CTAs, one per SM (a CTA holds all 512 TMEM columns),
// loop over items: a cube of NQ = 2^CB output quartets (the low CB bits free)
// times a tile of 256 trajectories (128 trajectory pairs, one per TMEM lane).
// An item reads the P - CB translated cubes q ^ 2^p, p >= CB (every input
// feeds one output), then its own cube (every input feeds its own output and
// CB in-cube flips); the own cube comes last, so that it is still in TMEM for
// the alpha partial.  Each input cube is a chunk: four tensor-map boxes (one
// per electron row a: NQ consecutive quartet rows x 256 trajectories, 16 KB)
// into a shared-memory stage, then 2 NQ tcgen05.cp.128x256b into a 16 NQ
// column TMEM slot.  Lane i of the slot holds pair i; columns 16 l + 4 a + c
// hold {re t, re t+1, im t, im t+1}[c] of row a of quartet l, the pair-planar
// 16 bytes as they lie in memory.  A copy reads the stage as a K-major
// operand without swizzle: core matrices of 8 pairs x 16 B, SBO = 128 B to
// the next 8 pairs, LBO = one box to the next electron row, so one copy moves
// rows a and a + 1 of a quartet (8 columns).  The own cube's stage also
// carries the cube's diagonal blocks (1 KB, full 4x4 form, bulk copy); copy
// warp 0 moves them into a buffer of the item's parity before it releases the
// stage, and signals them with a plain arrival on the slot's cfull.  Item
// n + 2 reuses that buffer only after the copy warps' tempty wait for a chunk
// after item n's own cube (an item has P - CB + 1 >= 3 chunks, NS = 4), so
// the compute warps are done with it.
//
// Block values.  The compute warps stage every flip block (2P entries,
// compact form) in shared memory once per CTA; the diagonal blocks come with
// the own cube.  No compute-warp load waits on global memory inside the
// chunk loop (a timing copy of an earlier form that read the values with
// __ldg between TMEM loads measured 2.2k cycles per translated chunk against
// 0.5k without the arithmetic).
//
// Roles: one TMA warp (lanes 0..3 each issue one electron row's box), NCP
// copy warps (lane 0 of each issues its share of a chunk's copies: four
// issuing threads measured about 64 B/cycle of copies, one about 40; three
// keep the CTA at 12 warps, whose register file allows 168 registers a
// thread), and 4 G compute warps (warp w reads TMEM lanes 32 (w % 4) .. + 31;
// warpgroup w / 4 owns NQ / G consecutive outputs of the cube).
// Rings: NSTG shared-memory stages (sfull: the TMA bytes landed; sfree: the
// copies that read the stage completed) and NS TMEM slots (cfull: the copies
// into the slot completed, and copy warp 0's arrival; tempty: every compute
// warp has read the slot).
// Chunk k of a CTA uses stage k % NSTG and slot k % NS; every role counts
// the same chunks, so the n-th use of a barrier completes its phase n.
//
// Every mbarrier wait is bounded; after the limit the kernel records status
// bit 4, skips the remaining work (the compute warps still take their one
// named barrier per item, so none of them waits on a warp that left), lets
// its own copies drain (bounded), frees TMEM and returns.
#pragma once

#include <cuda.h>

#include <cstdint>

#include "msgpu_kernels.cuh"
#include "msgpu_spmm_tc.cuh"

namespace msgpu {

constexpr int kTmMaxFlips = 2 * kTcMaxBits;  // flip entries (2 per quartet bit)

template <int CB, int G, int NCP>
struct TmCfg {
    static constexpr int NQ = 1 << CB;               // output quartets per item
    static constexpr int Pairs = 128;                // TMEM lanes
    static constexpr int Traj = 2 * Pairs;           // trajectories per item
    static constexpr int SlotCols = 16 * NQ;         // TMEM columns of one chunk
    static constexpr int NS = 512 / SlotCols;        // TMEM slots
    static constexpr int RowBytes = Traj * 8;        // one quartet row of the tile (complex64)
    static constexpr int BoxBytes = NQ * RowBytes;   // one electron row of a chunk
    static constexpr int ChunkBytes = 4 * BoxBytes;  // one chunk's boxes
    static constexpr int DiagBytes = NQ * 128;       // the own cube's diagonal blocks (8 float4 each)
    static constexpr int StageBytes = ChunkBytes + DiagBytes;
    static constexpr int NSTG = 3;                   // shared-memory stages
    static constexpr int NO = NQ / G;                // outputs per compute warp
    static constexpr int Compute = 4 * G;            // compute warps
    static constexpr int TmaWarp = Compute, CpWarp0 = Compute + 1;
    static constexpr int Threads = 32 * (Compute + 1 + NCP);
    static constexpr int NCopies = 2 * NQ;           // tcgen05.cp.128x256b per chunk
    static constexpr int NBar = 2 * NSTG + 2 * NS + 1;
    static constexpr int OffDiag = NSTG * StageBytes;             // float4 [2][NQ][8]: diagonal blocks by item parity
    static constexpr int OffFlip = OffDiag + 2 * DiagBytes;       // float4 [kTmMaxFlips][8]
    static constexpr int OffFType = OffFlip + kTmMaxFlips * 128;  // int [kTmMaxFlips]
    static constexpr int OffBar = OffFType + kTmMaxFlips * 4;
    static constexpr int OffFlag = OffBar + NBar * 8;     // abort flag, TMEM address
    static constexpr int OffAlpha = OffFlag + 16;         // double [2][G][Traj]
    static constexpr int Smem = OffAlpha + 2 * G * Traj * 8;
    // the own cube's four inputs per output (CB = 3, two loads of 32 columns) and a
    // translated chunk's four outputs (two loads)
    static_assert(CB == 3 && NCP >= 1 && NO == 4 && NS >= 2, "TMEM-staged SpMM shape");
    static_assert(StageBytes % 128 == 0 && OffBar % 8 == 0 && OffAlpha % 8 == 0 && Smem <= 227 * 1024,
                  "shared memory");
};

// tcgen05.cp source descriptor: K-major, no swizzle, LBO = one box (the next
// electron row), SBO = 128 B (the next 8 trajectory pairs), version 1.
template <int BoxBytes>
__device__ __forceinline__ uint64_t tm_desc(uint32_t addr)
{
    return static_cast<uint64_t>((addr >> 4) & 0x3FFF) | (static_cast<uint64_t>((BoxBytes >> 4) & 0x3FFF) << 16) |
           (static_cast<uint64_t>(128 >> 4) << 32) | (static_cast<uint64_t>(1) << 46);
}

__device__ __forceinline__ void tm_cp(uint32_t taddr, uint64_t desc)
{
    asm volatile("tcgen05.cp.cta_group::1.128x256b [%0], %1;" ::"r"(taddr), "l"(desc) : "memory");
}

__device__ __forceinline__ void tm_ld32(uint32_t taddr, uint32_t (&v)[32])
{
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
                 : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
                 : "r"(taddr));
}

// 16 columns into registers v[16 r .. 16 r + 15]
template <int r>
__device__ __forceinline__ void tm_ld16_at(uint32_t taddr, uint32_t (&v)[32])
{
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(v[16 * r]), "=r"(v[16 * r + 1]), "=r"(v[16 * r + 2]), "=r"(v[16 * r + 3]), "=r"(v[16 * r + 4]),
          "=r"(v[16 * r + 5]), "=r"(v[16 * r + 6]), "=r"(v[16 * r + 7]), "=r"(v[16 * r + 8]), "=r"(v[16 * r + 9]),
          "=r"(v[16 * r + 10]), "=r"(v[16 * r + 11]), "=r"(v[16 * r + 12]), "=r"(v[16 * r + 13]),
          "=r"(v[16 * r + 14]), "=r"(v[16 * r + 15])
        : "r"(taddr));
}

// tcgen05.wait::ld naming the 32 loaded registers, so that no use of them is
// scheduled before it.
__device__ __forceinline__ void tm_wait32(uint32_t (&v)[32])
{
    asm volatile("tcgen05.wait::ld.sync.aligned;"
                 : "+r"(v[0]), "+r"(v[1]), "+r"(v[2]), "+r"(v[3]), "+r"(v[4]), "+r"(v[5]), "+r"(v[6]), "+r"(v[7]), "+r"(v[8]), "+r"(v[9]), "+r"(v[10]), "+r"(v[11]), "+r"(v[12]), "+r"(v[13]), "+r"(v[14]), "+r"(v[15]), "+r"(v[16]), "+r"(v[17]), "+r"(v[18]), "+r"(v[19]), "+r"(v[20]), "+r"(v[21]), "+r"(v[22]), "+r"(v[23]), "+r"(v[24]), "+r"(v[25]), "+r"(v[26]), "+r"(v[27]), "+r"(v[28]), "+r"(v[29]), "+r"(v[30]), "+r"(v[31])
                 :
                 : "memory");
}

// Rows a of quartet r of the 32 loaded registers (16 columns a quartet).
template <int r>
__device__ __forceinline__ void tm_rows(const uint32_t (&v)[32], float4 (&x)[4])
{
#pragma unroll
    for (int a = 0; a < 4; ++a)
        x[a] = make_float4(__uint_as_float(v[16 * r + 4 * a]), __uint_as_float(v[16 * r + 4 * a + 1]),
                           __uint_as_float(v[16 * r + 4 * a + 2]), __uint_as_float(v[16 * r + 4 * a + 3]));
}

__device__ __forceinline__ void tm_named_sync(int id, int threads)
{
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(threads) : "memory");
}

// Block table of the TMEM-staged SpMM, [2P + Q][8] float4: entry e < 2P is
// flip entry e of src in its compact form (the float4s its type uses, then
// zeros), entry 2P + q the diagonal block of quartet q in the full 4x4 form
// (type 0; zeros when the quartet has none).  Rebuilt whenever the quartet
// values change.  One thread per (entry, float4).
__global__ void __launch_bounds__(256) k_tm_tables(const int2 *__restrict__ src, int nflip, int nent,
                                                   const float4 *__restrict__ qval, float4 *__restrict__ out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nent * 8) return;
    const int e = i >> 3, f = i & 7;
    const int2 s = src[e];
    float4 r = make_float4(0.f, 0.f, 0.f, 0.f);
    if (s.x >= 0) {
        if (e < nflip) {
            const int used = s.y == 0 ? 8 : (s.y <= 2 ? 4 : 2);
            if (f < used) r = qval[s.x + f];
        } else {
            float2 h[4][4];
            tc_expand(s.y, reinterpret_cast<const float2 *>(qval + s.x), h);
            const int a = f >> 1, b = 2 * (f & 1);
            r = make_float4(h[a][b].x, h[a][b].y, h[a][b + 1].x, h[a][b + 1].y);
        }
    }
    out[i] = r;
}

// U = s_j H w_j for one trajectory group: grid = min(items, SMs) persistent
// CTAs, TmCfg::Threads threads, TmCfg::Smem bytes of dynamic shared memory.
//   map: 2D tensor map over the Krylov basis (8-byte elements, rows of ldm
//   trajectories, boxes of 256 x NQ); w_j's rows start at map row y0 and the
//   group's first trajectory at column x0;
//   src: the block entries {value offset (< 0: no block), type} of build_tc:
//   2P flip entries (2 p + bit p of the output quartet), then one diagonal
//   entry per quartet; tab: the k_tm_tables table of the same entries;
//   quartet_base(q, s1, s2) + {0, s2, s1, s1 + s2}: the rows of quartet q (a
//   cube's quartets have consecutive rows: the host checks s2 % NQ == 0);
//   sj, U, part start at the group's first trajectory; width = its
//   trajectories (a multiple of 64); part gets one row per cube.
template <int CB, int G, int NCP>
__global__ void __launch_bounds__(TmCfg<CB, G, NCP>::Threads, 1)
k_lanczos_apply_tm(const __grid_constant__ CUtensorMap map, int x0, int y0, const int2 *__restrict__ src,
                   const float4 *__restrict__ tab, int P, int s1, int s2, const double *__restrict__ sj,
                   float2 *__restrict__ U, double *__restrict__ part, int ldm, int width, int *__restrict__ status)
{
    using Cfg = TmCfg<CB, G, NCP>;
    constexpr int NS = Cfg::NS, NSTG = Cfg::NSTG, NO = Cfg::NO;
    extern __shared__ __align__(1024) unsigned char tm_raw[];
    unsigned char *sm = tm_raw;
    const uint32_t sbase = tc_smem(sm);
    const uint32_t bar0 = sbase + Cfg::OffBar;
    auto bar_sfull = [&](int s) { return bar0 + 8 * s; };
    auto bar_sfree = [&](int s) { return bar0 + 8 * (NSTG + s); };
    auto bar_cfull = [&](int s) { return bar0 + 8 * (2 * NSTG + s); };
    auto bar_tempty = [&](int s) { return bar0 + 8 * (2 * NSTG + NS + s); };
    const uint32_t bar_cpdone = bar0 + 8 * (2 * NSTG + 2 * NS);
    volatile int *abort = reinterpret_cast<volatile int *>(sm + Cfg::OffFlag);
    uint32_t *tslot = reinterpret_cast<uint32_t *>(sm + Cfg::OffFlag + 8);
    double *s_alpha = reinterpret_cast<double *>(sm + Cfg::OffAlpha);
    float4 *s_fval = reinterpret_cast<float4 *>(sm + Cfg::OffFlip);
    float4 *s_diag = reinterpret_cast<float4 *>(sm + Cfg::OffDiag);
    int *s_ftype = reinterpret_cast<int *>(sm + Cfg::OffFType);

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int ntiles = (width + Cfg::Traj - 1) / Cfg::Traj;
    const int nitems = (1 << (P - CB)) * ntiles;
    const int NCH = P - CB + 1;  // chunks per item: P - CB translated cubes, then the own cube
    // first quartet of chunk c of the item whose cube starts at quartet q0
    auto chunk_q = [&](int q0, int c) { return c < NCH - 1 ? q0 ^ (1 << (CB + c)) : q0; };

    if (tid == 0) {
        *abort = 0;
        for (int s = 0; s < NSTG; ++s) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar_sfull(s)));
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar_sfree(s)), "r"(NCP));
        }
        for (int s = 0; s < NS; ++s) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar_cfull(s)), "r"(NCP + 1));
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar_tempty(s)), "r"(Cfg::Compute));
        }
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar_cpdone), "r"(NCP));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(tc_smem(tslot)),
                     "r"(512));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tslot;

    if (warp == Cfg::TmaWarp) {
        // ------------------------------------------------------------ TMA warp
        // lane 0 waits and posts the byte count; lanes 0..3 load electron row a = lane,
        // lane 0 also the own cube's diagonal blocks
        const int lane_off = (lane & 1 ? s2 : 0) + (lane & 2 ? s1 : 0);
        int k = 0;  // chunks issued
        bool ok = true;
        for (int it = blockIdx.x; it < nitems && ok; it += gridDim.x) {
            const int q0 = (it / ntiles) << CB;
            const int x = x0 + (it % ntiles) * Cfg::Traj;
            for (int c = 0; c < NCH; ++c) {
                const int s = k % NSTG;
                const bool own = c == NCH - 1;
                int got = 1;
                if (lane == 0) {
                    if (k >= NSTG) got = tc_wait(bar_sfree(s), ((k / NSTG) & 1) ^ 1, abort);
                    if (got)
                        tc_expect(bar_sfull(s), static_cast<uint32_t>(Cfg::ChunkBytes + (own ? Cfg::DiagBytes : 0)));
                }
                got = __shfl_sync(0xffffffffu, got, 0);
                if (!got) {
                    ok = false;
                    break;
                }
                const uint32_t st = sbase + s * Cfg::StageBytes;
                if (lane < 4)
                    tc_box(st + lane * Cfg::BoxBytes, &map, x, y0 + quartet_base(chunk_q(q0, c), s1, s2) + lane_off,
                           bar_sfull(s));
                if (own && lane == 0)
                    tc_bulk(st + Cfg::ChunkBytes, tab + static_cast<size_t>(2 * P + q0) * 8,
                            static_cast<uint32_t>(Cfg::DiagBytes), bar_sfull(s));
                ++k;
            }
        }
        // every copy this CTA started lands before the CTA can exit: only the
        // last NSTG stages can be in flight (a stage is reloaded after its copies read it)
        if (lane == 0)
            for (int kk = max(0, k - NSTG); kk < k; ++kk)
                for (uint32_t i = 0; i < kTcWait && !tc_try(bar_sfull(kk % NSTG), (kk / NSTG) & 1); ++i) {
                }
    } else if (warp >= Cfg::CpWarp0) {
        // ------------------------------------------------------------ copy warps
        // lane 0 waits, issues this warp's copies and commits; warp 0's lanes move
        // the own cube's diagonal blocks out of the stage before it is released
        const int cw = warp - Cfg::CpWarp0;
        int k = 0, n = 0;
        bool ok = true;
        for (int it = blockIdx.x; it < nitems && ok; it += gridDim.x, ++n)
            for (int c = 0; c < NCH; ++c, ++k) {
                const int s = k % NSTG, slot = k % NS;
                int got = 1;
                if (lane == 0)
                    got = tc_wait(bar_sfull(s), (k / NSTG) & 1, abort) &&
                          (k < NS || tc_wait(bar_tempty(slot), ((k / NS) & 1) ^ 1, abort));
                got = __shfl_sync(0xffffffffu, got, 0);
                if (!got) {
                    ok = false;
                    break;
                }
                if (cw == 0 && c == NCH - 1) {
                    const float4 *sd = reinterpret_cast<const float4 *>(sm + s * Cfg::StageBytes + Cfg::ChunkBytes);
                    float4 *dd = s_diag + (n & 1) * (Cfg::DiagBytes / 16);
                    for (int i = lane; i < Cfg::DiagBytes / 16; i += 32) dd[i] = sd[i];
                }
                __syncwarp();
                if (lane == 0) {
                    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                    const uint32_t st = sbase + s * Cfg::StageBytes, dst = tmem + slot * Cfg::SlotCols;
                    for (int i = cw; i < Cfg::NCopies; i += NCP) {
                        const int l = i >> 1, a = (i & 1) * 2;  // quartet, first of the two electron rows
                        tm_cp(dst + 16 * l + 4 * a, tm_desc<Cfg::BoxBytes>(st + a * Cfg::BoxBytes + l * Cfg::RowBytes));
                    }
                    tc_commit(bar_cfull(slot));  // both arrive once these copies complete
                    tc_commit(bar_sfree(s));
                    if (cw == 0) tc_arrive(bar_cfull(slot));  // releases the diagonal blocks' stores
                }
            }
        // every copy this warp issued completes before TMEM is freed
        if (lane == 0) {
            tc_commit(bar_cpdone);
            for (uint32_t i = 0; i < kTcWait && !tc_try(bar_cpdone, 0); ++i) {
            }
        }
    } else {
        // ------------------------------------------------------------ compute warps
        const int wq = warp & 3, grp = warp >> 2;
        const int pair = 32 * wq + lane;
        const uint32_t lane_addr = tmem + (static_cast<uint32_t>(32 * wq) << 16);
        const int o0 = grp * NO;  // this warp's first output of the cube
        const int off[4] = {0, s2, s1, s1 + s2};
        // flip blocks into shared memory, once per CTA
        for (int i = tid; i < 2 * P * 8; i += 32 * Cfg::Compute) s_fval[i] = tab[i];
        for (int i = tid; i < 2 * P; i += 32 * Cfg::Compute) {
            const int2 b = src[i];
            s_ftype[i] = b.x >= 0 ? b.y : -1;
        }
        tm_named_sync(1, 32 * Cfg::Compute);
        int k = 0, n = 0;  // chunks consumed, items
        bool ok = true;
        for (int it = blockIdx.x; it < nitems; it += gridDim.x, ++n) {
            const int cube = it / ntiles, q0 = cube << CB;
            const int t = (it % ntiles) * Cfg::Traj + 2 * pair;  // the pair's first trajectory in the group
            const bool live = t < width;                          // width is even: t + 1 < width too
            double al0 = 0.0, al1 = 0.0;
            if (ok) {
                // issued here, first used at the end of the item
                const float sc0 = live ? static_cast<float>(sj[t]) : 0.f, sc1 = live ? static_cast<float>(sj[t + 1]) : 0.f;
                const int brow0 = quartet_base(q0, s1, s2);  // the cube's quartets have consecutive rows
                float2 o[NO][4][2];
#pragma unroll
                for (int i = 0; i < NO; ++i)
#pragma unroll
                    for (int a = 0; a < 4; ++a) o[i][a][0] = o[i][a][1] = make_float2(0.f, 0.f);
                for (int c = 0; c < NCH; ++c, ++k) {
                    const int slot = k % NS;
                    if (!__all_sync(0xffffffffu, tc_wait(bar_cfull(slot), (k / NS) & 1, abort))) {
                        ok = false;
                        break;
                    }
                    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                    const uint32_t sa = lane_addr + slot * Cfg::SlotCols;
                    uint32_t v[32];
                    if (c < NCH - 1) {
                        // translated cube of nucleus p: output l reads quartet l; one block for all four,
                        // two outputs per TMEM load
                        const int p = CB + c;
                        const int e = 2 * p + ((q0 >> p) & 1);
                        const int type = s_ftype[e];
                        if (type >= 0) {
                            const float4 *bv = s_fval + 8 * e;
#pragma unroll
                            for (int h = 0; h < NO / 2; ++h) {
                                tm_ld32(sa + 16 * (o0 + 2 * h), v);
                                tm_wait32(v);
                                float4 x[4];
                                tm_rows<0>(v, x);
                                quartet_block<false>(o[2 * h], type, bv, x);
                                tm_rows<1>(v, x);
                                quartet_block<false>(o[2 * h + 1], type, bv, x);
                            }
                        }
                    } else {
                        // own cube: output l reads quartet l (diagonal block) and l ^ 2^p, p < CB;
                        // quartets l and l ^ 1 in one load, l ^ 2 and l ^ 4 in the next
                        const float4 *dv = s_diag + (n & 1) * (Cfg::DiagBytes / 16);
#pragma unroll
                        for (int i = 0; i < NO; ++i) {
                            const int l = o0 + i;
                            float4 xo[4], x[4];
                            tm_ld16_at<0>(sa + 16 * l, v);
                            tm_ld16_at<1>(sa + 16 * (l ^ 1), v);
                            tm_wait32(v);
                            tm_rows<0>(v, xo);
                            quartet_block<false>(o[i], 0, dv + 8 * l, xo);
                            tm_rows<1>(v, x);
                            int e = (l & 1);
                            if (s_ftype[e] >= 0) quartet_block<false>(o[i], s_ftype[e], s_fval + 8 * e, x);
                            tm_ld16_at<0>(sa + 16 * (l ^ 2), v);
                            tm_ld16_at<1>(sa + 16 * (l ^ 4), v);
                            tm_wait32(v);
                            tm_rows<0>(v, x);
                            e = 2 + ((l >> 1) & 1);
                            if (s_ftype[e] >= 0) quartet_block<false>(o[i], s_ftype[e], s_fval + 8 * e, x);
                            tm_rows<1>(v, x);
                            e = 4 + ((l >> 2) & 1);
                            if (s_ftype[e] >= 0) quartet_block<false>(o[i], s_ftype[e], s_fval + 8 * e, x);
                            // output quartet q0 + l is complete: U rows and the alpha partial
#pragma unroll
                            for (int a = 0; a < 4; ++a) {
                                const float2 ure = make_float2(o[i][a][0].x * sc0, o[i][a][0].y * sc1);
                                const float2 uim = make_float2(o[i][a][1].x * sc0, o[i][a][1].y * sc1);
                                if (live)
                                    *reinterpret_cast<float4 *>(U + static_cast<size_t>(brow0 + l + off[a]) * ldm + t) =
                                        make_float4(ure.x, ure.y, uim.x, uim.y);
                                al0 += (static_cast<double>(xo[a].x) * ure.x + static_cast<double>(xo[a].z) * uim.x) * sc0;
                                al1 += (static_cast<double>(xo[a].y) * ure.y + static_cast<double>(xo[a].w) * uim.y) * sc1;
                            }
                        }
                    }
                    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
                    __syncwarp();
                    if (lane == 0) tc_arrive(bar_tempty(slot));
                }
            }
            // alpha partial of the cube: the G warpgroups' sums in group order
            double *sa_n = s_alpha + static_cast<size_t>(n & 1) * G * Cfg::Traj;
            sa_n[grp * Cfg::Traj + 2 * pair] = al0;
            sa_n[grp * Cfg::Traj + 2 * pair + 1] = al1;
            tm_named_sync(1, 32 * Cfg::Compute);
            if (ok && grp == 0 && live) {
                double a0 = 0.0, a1 = 0.0;
#pragma unroll
                for (int g = 0; g < G; ++g) {
                    a0 += sa_n[g * Cfg::Traj + 2 * pair];
                    a1 += sa_n[g * Cfg::Traj + 2 * pair + 1];
                }
                part[static_cast<size_t>(cube) * ldm + t] = a0;
                part[static_cast<size_t>(cube) * ldm + t + 1] = a1;
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (*abort && tid == 0) atomicOr(status, 4);
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512));
    }
}

}  // namespace msgpu
