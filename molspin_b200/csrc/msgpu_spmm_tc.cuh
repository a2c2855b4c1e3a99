// msgpu_spmm_tc.cuh -- quartet SpMM of the complex64 Lanczos form on the
// 5th-generation tensor cores (tcgen05, TMEM, TMA bulk copies).
//
// U = s_j H w_j over a trajectory block (the H v product of
// SpinSpace::LanczosProcess / ArnoldiProcess, SpinSpace_operators.cpp:1362,
// applied per column by HSPropagator::Step, HSPropagator.cpp:64-78).
//
// Structure used.  For radical pairs whose other spins are all spin-1/2, the
// quartet index q (the row index with the two electron digits removed) is a
// P-bit number, one bit per nucleus, and H couples quartet q only to itself
// (a 4x4 diagonal block that depends on q) and to q ^ 2^p (one block per
// nucleus p that depends only on p and on bit p of the output quartet).  The
// host checks this on the quartet form before it enables the kernel.
//
// Work split.  A CTA owns a cube of 2^CB output quartets (the low CB bits
// free, the high bits fixed) for 128 trajectories.  Its inputs are the cube
// itself (each input feeds its own output and CB in-cube flips) and, for
// every nucleus p >= CB, the translated cube q ^ 2^p (each input feeds one
// output).  Every input quartet is loaded once per CTA and feeds all of the
// CTA's outputs that need it through the tensor cores: 1 + P - CB loads per
// output quartet against 1 + P in the SIMT kernels, whose limit is the L1
// data path.
//
// Data path per input quartet (4 rows x 128 trajectories, complex64,
// pair-planar): 2D tensor-map boxes of 8 consecutive quartet rows x 128
// trajectories (one box per electron row; the cube's quartets have
// consecutive rows when the second electron stride is a multiple of 2^CB,
// which the host checks) into shared memory; producer threads (thread = trajectory = TMEM lane; several warpgroups take
// alternate inputs) read their 8 real values (Re/Im of the 4 rows), split
// each into a TF32 head and an FP32 tail, x = hi + lo with hi = x with its 13
// low mantissa bits cleared (exact in TF32) and lo = x - hi (exact in FP32),
// and store [hi | lo] (16 TMEM columns) into a TMEM slot.  Each output
// quartet owns 16 accumulator columns, [main (8) | correction (8)], and the
// MMA warp of output o (o % 4) issues, per (output, input) pair, two tcgen05.mma kind::tf32
// (M = 128 trajectories, N = 16, K = 8, A from TMEM, B from shared memory):
//     [main | corr] += hi . [H_hi | H_lo]   (hi H_hi | hi H_lo)
//     [main | corr] += lo . [  0  | H_hi]   (   0    | lo H_hi)
// with H = H_hi + H_lo the same split of the block's real form (8 x 8:
// [[Re H, -Im H], [Im H, Re H]] acting on [Re x ; Im x]).  The dropped lo H_lo
// and the tensor core's TF32 reading of lo and H_lo are 2^-22 of the result.
// The correction products accumulate apart from the main one: the FP32
// accumulation of tcgen05.mma rounds towards zero, and keeping the
// 2^-11-sized corrections out of the main accumulator limits that bias to the
// main products' own.  An output's first MMA overwrites its 16 columns; the
// epilogue adds the two halves (round to nearest), scales by s_j, stores U and
// the per-trajectory FP64 partial of alpha_j = Re <v_j, U>.  The pace is set
// by the cycle producer store -> MMA -> commit -> TMEM slot release, not by
// the tensor pipe: every instruction is small (N = 16, K = 8).
//
// TMEM columns (CB = 4, 512 allocated): accumulators [0, 256), then 16 input
// slots of 16 columns.  CB = 3 allocates 256 columns.
//
// Every mbarrier wait is bounded; after the limit the kernel records status
// bit 4, lets its own copies and MMAs drain (bounded), frees TMEM and
// returns.
#pragma once

#include <cuda.h>

#include <cstdint>
#include <cstring>

#include "msgpu_device.cuh"

namespace msgpu {

constexpr int kTcTraj = 128;            // trajectories per CTA (TMEM lanes, MMA M)
constexpr int kTcB = 512;               // bytes of one B operand (16 N rows x 8 K TF32)
constexpr int kTcMaxBits = 14;          // quartet bits P (D <= 65536)
constexpr uint32_t kTcWait = 1u << 23;  // iterations of a bounded mbarrier wait

template <int CB>
struct TcCfg {
    static constexpr int NQ = 1 << CB;             // output quartets per CTA
    // producer warpgroups (each of 4 warps covers the 128 TMEM lanes; they take
    // alternate input pairs and alternate outputs), then one TMA warp and four
    // MMA-issuing warps (output o is issued by MMA warp o % 4: one thread issues
    // a tcgen05.mma about every 50 cycles whatever its N up to 64, and four
    // issuing warps measured four times that rate)
    static constexpr int G = CB == 4 ? 4 : 2;
    static constexpr int NMMA = 4;
    static constexpr int Threads = 32 * (4 * G + 1 + NMMA);
    static constexpr int Cols = CB == 4 ? 512 : 256;
    static constexpr int Slot0 = 16 * NQ;            // accumulators [0, Slot0): 16 columns per output
    static constexpr int NS = (Cols - Slot0) / 16;   // TMEM input slots
    // Inputs arrive as 2D tensor-map boxes of HB consecutive quartet rows x 128
    // trajectories (8 KB, one electron row a): a 1 KB bulk copy costs the TMA
    // unit about 60 cycles, an 8 KB box about 130 (62 B/cycle with four issuing
    // lanes).  A stage holds one box per row a, i.e. HB input quartets.
    static constexpr int HB = 8;
    static constexpr int BoxBytes = HB * kTcTraj * 8;  // 8 KB
    static constexpr int StageBytes = 4 * BoxBytes;    // HB inputs, 32 KB
    static constexpr int NSTG = CB == 4 ? 3 : 2;       // stages for translated inputs
    // shared memory: own cube | stage ring | diagonal B operands | flip B operands (P bits) | barriers
    static constexpr int OffOwn = 0;
    static constexpr int OffStage = OffOwn + (NQ / HB) * StageBytes;
    static constexpr int OffDiag = OffStage + NSTG * StageBytes;
    static constexpr int OffFlip = OffDiag + NQ * 2 * kTcB;
    // own, tables, stage full/empty, slot-quad empty (one commit per issuer frees 4 slots), slot full, done
    static constexpr int NBar = 2 + 2 * NSTG + NS / 4 + NS + 1;
    __host__ __device__ static constexpr int off_bar(int P) { return OffFlip + P * 2 * 2 * kTcB; }
    // then the abort flag and TMEM slot (16 B) and the first row of every input quartet (int)
    __host__ __device__ static constexpr int off_rows(int P) { return off_bar(P) + NBar * 8 + 16; }
    __host__ __device__ static constexpr int smem(int P) { return off_rows(P) + 4 * NQ * (1 + P - CB); }
    static_assert(NS >= 4 && NS % 4 == 0 && NQ % HB == 0, "TMEM slots, boxes");
};

__device__ __forceinline__ uint32_t tc_smem(const void *p) { return static_cast<uint32_t>(__cvta_generic_to_shared(p)); }

__device__ __forceinline__ bool tc_try(uint32_t bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait: false after the limit (the abort flag is then set) or when
// another role aborted.
__device__ __forceinline__ bool tc_wait(uint32_t bar, uint32_t parity, volatile int *abort)
{
    for (uint32_t it = 0; it < kTcWait; ++it) {
        if (tc_try(bar, parity)) return true;
        if (*abort) return false;
    }
    *abort = 1;
    return false;
}

__device__ __forceinline__ void tc_bulk(uint32_t dst, const void *src, uint32_t bytes, uint32_t bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
}

__device__ __forceinline__ void tc_expect(uint32_t bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ void tc_arrive(uint32_t bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

// B operand descriptor: K-major, no swizzle, core matrices of 8 rows x 16 B;
// LBO = 128 B (the next 16 bytes of K), SBO = 256 B (the next 8 N rows), version 1.
__device__ __forceinline__ uint64_t tc_bdesc(uint32_t addr)
{
    return static_cast<uint64_t>((addr >> 4) & 0x3FFF) | (static_cast<uint64_t>(128 >> 4) << 16) |
           (static_cast<uint64_t>(256 >> 4) << 32) | (static_cast<uint64_t>(1) << 46);
}

// kind::tf32 instruction descriptor: D = F32, A = B = TF32, both K-major, M = 128, N = 16.
constexpr uint32_t kTcIdesc = (1u << 4) | (2u << 7) | (2u << 10) | (static_cast<uint32_t>(16 >> 3) << 17) |
                              (static_cast<uint32_t>(128 >> 4) << 24);

__device__ __forceinline__ void tc_mma(uint32_t d, uint32_t a, uint64_t b, uint32_t acc)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], [%1], %2, %3, p;\n\t}"
        :
        : "r"(d), "r"(a), "l"(b), "r"(kTcIdesc), "r"(acc)
        : "memory");
}

// The same two instructions issued by one lane elected in a warp that runs the
// issuing loop together, so that the operands are warp-uniform values (from a
// single active lane they are moved to uniform registers for every MMA; this
// form measured 6 % faster over the whole kernel).
__device__ __forceinline__ void tc_mma_elect(uint32_t d, uint32_t a, uint64_t b, uint32_t acc)
{
    asm volatile(
        "{\n\t.reg .pred e, p;\n\telect.sync _|e, 0xffffffff;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "@e tcgen05.mma.cta_group::1.kind::tf32 [%0], [%1], %2, %3, p;\n\t}"
        :
        : "r"(d), "r"(a), "l"(b), "r"(kTcIdesc), "r"(acc)
        : "memory");
}

__device__ __forceinline__ void tc_commit_elect(uint32_t bar)
{
    asm volatile(
        "{\n\t.reg .pred e;\n\telect.sync _|e, 0xffffffff;\n\t"
        "@e tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n\t}" ::"r"(bar)
        : "memory");
}

__device__ __forceinline__ void tc_commit(uint32_t bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void tc_st16(uint32_t taddr, const uint32_t (&v)[16])
{
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16};" ::"r"(
            taddr),
        "r"(v[0]), "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]), "r"(v[7]), "r"(v[8]), "r"(v[9]),
        "r"(v[10]), "r"(v[11]), "r"(v[12]), "r"(v[13]), "r"(v[14]), "r"(v[15])
        : "memory");
}

__device__ __forceinline__ void tc_ld16(uint32_t taddr, uint32_t (&v)[16])
{
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]), "=r"(v[8]),
          "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
        : "r"(taddr));
}

// Byte offset of element (n, k) in a 16 (N) x 8 (K) TF32 B operand (see tc_bdesc).
__host__ __device__ constexpr int tc_boff(int n, int k) { return (n >> 3) * 256 + (k >> 2) * 128 + (n & 7) * 16 + (k & 3) * 4; }

// TF32 head of x: its 13 low mantissa bits cleared (exact as TF32); x - head is exact in FP32.
__host__ __device__ inline float tc_head(float x)
{
#ifdef __CUDA_ARCH__
    return __uint_as_float(__float_as_uint(x) & 0xFFFFE000u);
#else
    uint32_t u;
    std::memcpy(&u, &x, 4);
    u &= 0xFFFFE000u;
    std::memcpy(&x, &u, 4);
    return x;
#endif
}

// Full 4x4 complex block from the compact quartet form (the types of QuartetC).
__device__ __forceinline__ void tc_expand(int type, const float2 *__restrict__ v, float2 (&h)[4][4])
{
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) h[a][b] = make_float2(0.f, 0.f);
    switch (type) {
    case 0:
        for (int a = 0; a < 4; ++a)
            for (int b = 0; b < 4; ++b) h[a][b] = v[4 * a + b];
        break;
    case 1:  // digit 1, a2 == b2: [a2][a1][b1]
        for (int a2 = 0; a2 < 2; ++a2)
            for (int a1 = 0; a1 < 2; ++a1)
                for (int b1 = 0; b1 < 2; ++b1) h[2 * a1 + a2][2 * b1 + a2] = v[(2 * a2 + a1) * 2 + b1];
        break;
    case 2:  // digit 2, a1 == b1: [a1][a2][b2]
        for (int a1 = 0; a1 < 2; ++a1)
            for (int a2 = 0; a2 < 2; ++a2)
                for (int b2 = 0; b2 < 2; ++b2) h[2 * a1 + a2][2 * a1 + b2] = v[(2 * a1 + a2) * 2 + b2];
        break;
    case 3:
        for (int a = 0; a < 4; ++a) h[a][a] = v[a];
        break;
    case 4:  // A (x) I on digit 1: [a1][b1]
        for (int a1 = 0; a1 < 2; ++a1)
            for (int b1 = 0; b1 < 2; ++b1)
                for (int a2 = 0; a2 < 2; ++a2) h[2 * a1 + a2][2 * b1 + a2] = v[2 * a1 + b1];
        break;
    default:  // I (x) A on digit 2: [a2][b2]
        for (int a2 = 0; a2 < 2; ++a2)
            for (int b2 = 0; b2 < 2; ++b2)
                for (int a1 = 0; a1 < 2; ++a1) h[2 * a1 + a2][2 * a1 + b2] = v[2 * a2 + b2];
        break;
    }
}

// B-operand tables.  Entry e (src[e] = {value offset in float4 units, type} of
// a block of the quartet form; offset < 0: no block, a zero operand) becomes
// two 16 (N) x 8 (K) TF32 B operands of the block's real form R[k][n] (k < 4
// Re x_k, 4 <= k < 8 Im x_{k-4}; n < 4 Re y_n, 4 <= n < 8 Im y_{n-4}):
//   BA: columns 0..7 R_hi (main), columns 8..15 R_lo (correction)
//   BB: columns 0..7 zero,        columns 8..15 R_hi (correction)
// One block of 128 threads per entry, thread (n, k).
__global__ void __launch_bounds__(128) k_tc_tables(const int2 *__restrict__ src, int nentries,
                                                   const float4 *__restrict__ qval, unsigned char *__restrict__ out)
{
    const int e = blockIdx.x;
    if (e >= nentries) return;
    const int n = threadIdx.x >> 3, k = threadIdx.x & 7;
    const int nn = n & 7;  // the real output component of column n
    float r = 0.f;
    const int2 s = src[e];  // s.x < 0: no such block (zero operand)
    if (s.x >= 0) {
        float2 h[4][4];
        tc_expand(s.y, reinterpret_cast<const float2 *>(qval + s.x), h);
        const int b = k & 3, a = nn & 3;
        const float2 hab = h[a][b];
        if (k < 4) r = nn < 4 ? hab.x : hab.y;  // Re x_b -> Re y_a: Re H; -> Im y_a: Im H
        else r = nn < 4 ? -hab.y : hab.x;       // Im x_b -> Re y_a: -Im H; -> Im y_a: Re H
    }
    const float hi = tc_head(r), lo = r - hi;
    const bool main_col = n < 8;
    unsigned char *o = out + static_cast<size_t>(e) * 2 * kTcB + tc_boff(n, k);
    *reinterpret_cast<float *>(o) = main_col ? hi : lo;            // BA
    *reinterpret_cast<float *>(o + kTcB) = main_col ? 0.f : hi;    // BB
}

__device__ __forceinline__ void tc_box(uint32_t dst, const CUtensorMap *map, int x, int y, uint32_t bar)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(dst),
        "l"(map), "r"(x), "r"(y), "r"(bar)
        : "memory");
}

// U = s_j H w_j for one trajectory group: grid (Q >> CB cubes, ceil(width / 128)),
// TcCfg<CB>::Threads threads, TcCfg<CB>::smem(P) bytes of dynamic shared memory.
//   map: 2D tensor map over the Krylov basis (8-byte elements, rows of ldm
//   trajectories, boxes of 128 x HB); w_j's rows start at map row y0 and its
//   group's first trajectory at column x0;
//   tflip: [P][2 (output bit)][2] B operands; tdiag: [Q][2] B operands;
//   quartet_base(q, s1, s2) + {0, s2, s1, s1 + s2}: the rows of quartet q (tabled in
//   shared memory for the CTA's inputs before the roles split); HB consecutive
//   quartets of a cube have consecutive rows (the host checks s2 % NQ == 0);
//   each MMA warp frees TMEM input slots four at a time (one tcgen05.commit per
//   quad), so NI and NS are multiples of 4;
//   sj, U, part start at the group's first trajectory; width = its trajectories
//   (a multiple of 64); ldm = the row stride.
template <int CB>
__global__ void __launch_bounds__(TcCfg<CB>::Threads, 1)
k_lanczos_apply_tc(const __grid_constant__ CUtensorMap map, int x0, int y0, const unsigned char *__restrict__ tflip,
                   const unsigned char *__restrict__ tdiag, int P, int s1, int s2, const double *__restrict__ sj,
                   float2 *__restrict__ U, double *__restrict__ part, int ldm, int width, int *__restrict__ status)
{
    using Cfg = TcCfg<CB>;
    constexpr int NQ = Cfg::NQ, NS = Cfg::NS, NSTG = Cfg::NSTG, G = Cfg::G, HB = Cfg::HB, NMMA = Cfg::NMMA;
    constexpr int kTmaWarp = 4 * G, kMmaWarp0 = 4 * G + 1;
    __shared__ double s_alpha[G][kTcTraj];  // per-group alpha partials, summed in group order
    extern __shared__ __align__(1024) unsigned char tc_raw[];
    unsigned char *sm = tc_raw;
    const uint32_t sbase = tc_smem(sm);
    const uint32_t bar0 = sbase + Cfg::off_bar(P);
    const uint32_t bar_own = bar0, bar_tab = bar0 + 8;
    auto bar_sfull = [&](int s) { return bar0 + 16 + 8 * s; };
    auto bar_sempty = [&](int s) { return bar0 + 16 + 8 * (NSTG + s); };
    auto bar_tfull = [&](int s) { return bar0 + 16 + 8 * (2 * NSTG + s); };
    auto bar_tempty = [&](int s) { return bar0 + 16 + 8 * (2 * NSTG + NS + s / 4); };  // slot s's quad
    const uint32_t bar_done = bar0 + 16 + 8 * (2 * NSTG + NS + NS / 4);
    volatile int *abort = reinterpret_cast<volatile int *>(sm + Cfg::off_bar(P) + Cfg::NBar * 8);
    uint32_t *tslot = reinterpret_cast<uint32_t *>(sm + Cfg::off_bar(P) + Cfg::NBar * 8 + 8);

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int cube = blockIdx.x, q0 = cube << CB;
    const int t0 = blockIdx.y * kTcTraj;          // first trajectory of the tile (in the group)
    const int nvalid = min(kTcTraj, width - t0);  // a multiple of 64 (width is)
    const int NI = NQ * (1 + P - CB);             // input quartets
    const int NC = (NI - NQ) / HB;                // stages of translated inputs
    const int off[4] = {0, s2, s1, s1 + s2};
    int *rows = reinterpret_cast<int *>(sm + Cfg::off_rows(P));  // first row of input quartet j

    // input j -> quartet (global index): the own cube, then one translated cube per nucleus p >= CB
    auto input_quartet = [&](int j) {
        const int g = j >> CB, l = j & (NQ - 1);
        return g == 0 ? q0 + l : (q0 + l) ^ (1 << (CB + g - 1));
    };
    // byte offset of row a of input j in shared memory: boxes of HB inputs, [a][input]
    auto input_row = [&](int j, int a) {
        if (j < NQ) return Cfg::OffOwn + (j / HB) * Cfg::StageBytes + a * Cfg::BoxBytes + (j % HB) * kTcTraj * 8;
        const int k = j - NQ;
        return Cfg::OffStage + ((k / HB) % NSTG) * Cfg::StageBytes + a * Cfg::BoxBytes + (k % HB) * kTcTraj * 8;
    };
    // the row arithmetic (integer divisions) of every input, spread over the CTA
    for (int j = tid; j < NI; j += Cfg::Threads) rows[j] = quartet_base(input_quartet(j), s1, s2);

    if (tid == 0) {
        *abort = 0;
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar_own));
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar_tab));
        for (int s = 0; s < NSTG; ++s) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar_sfull(s)));
            // every producer warp arrives once per input pair it read: HB / 2 pairs x 4 warps
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar_sempty(s)), "r"(2 * HB));
        }
        for (int s = 0; s < NS; ++s) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar_tfull(s)), "r"(4));
            if (s % 4 == 0) asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar_tempty(s)), "r"(NMMA));
        }
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar_done), "r"(NMMA));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(tc_smem(tslot)),
                     "r"(Cfg::Cols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tslot;

    if (warp == kTmaWarp) {
        // ------------------------------------------------------------ TMA warp
        // lane 0 waits and posts the byte counts; lanes 0..3 load row a = lane
        const int x = x0 + t0;
        const int lane_off = (lane & 1 ? s2 : 0) + (lane & 2 ? s1 : 0);  // row offset of electron row a = lane
        if (lane == 0) {
            // B operands: every flip entry and this cube's diagonal blocks
            tc_expect(bar_tab, static_cast<uint32_t>((P * 2 + NQ) * 2 * kTcB));
            tc_bulk(sbase + Cfg::OffFlip, tflip, static_cast<uint32_t>(P * 2 * 2 * kTcB), bar_tab);
            tc_bulk(sbase + Cfg::OffDiag, tdiag + static_cast<size_t>(q0) * 2 * kTcB,
                    static_cast<uint32_t>(NQ * 2 * kTcB), bar_tab);
            tc_expect(bar_own, static_cast<uint32_t>((NQ / HB) * Cfg::StageBytes));  // the own cube
        }
        __syncwarp();
        if (lane < 4)
            for (int h = 0; h < NQ / HB; ++h)
                tc_box(sbase + Cfg::OffOwn + h * Cfg::StageBytes + lane * Cfg::BoxBytes, &map, x,
                       y0 + rows[h * HB] + lane_off, bar_own);
        // translated inputs through the stage ring, HB quartets per stage
        int issued = 0;
        for (int c = 0; c < NC; ++c) {
            const int s = c % NSTG, r = c / NSTG;
            int got = 1;
            if (lane == 0) {
                got = tc_wait(bar_sempty(s), (r & 1) ^ 1, abort);
                if (got) tc_expect(bar_sfull(s), static_cast<uint32_t>(Cfg::StageBytes));
            }
            got = __shfl_sync(0xffffffffu, got, 0);
            if (!got) break;
            if (lane < 4)
                tc_box(sbase + Cfg::OffStage + s * Cfg::StageBytes + lane * Cfg::BoxBytes, &map, x,
                       y0 + rows[NQ + c * HB] + lane_off, bar_sfull(s));
            issued = c + 1;
        }
        // every copy this CTA started lands before the CTA can exit
        if (lane == 0) {
            for (int c = max(0, issued - NSTG); c < issued; ++c)
                for (uint32_t it = 0; it < kTcWait && !tc_try(bar_sfull(c % NSTG), (c / NSTG) & 1); ++it) {
                }
            for (uint32_t it = 0; it < kTcWait && !tc_try(bar_own, 0); ++it) {
            }
            for (uint32_t it = 0; it < kTcWait && !tc_try(bar_tab, 0); ++it) {
            }
        }
    } else if (warp >= kMmaWarp0) {
        // ------------------------------------------------------------ MMA warps
        const int mw = warp - kMmaWarp0;  // issues the MMAs of outputs o with o % NMMA == mw
        {
            // the whole warp runs the loop (uniform operands); one elected lane issues
            bool ok = __all_sync(0xffffffffu, tc_wait(bar_tab, 0, abort));
            const uint32_t flip_s = sbase + Cfg::OffFlip, diag_s = sbase + Cfg::OffDiag;
            uint32_t written = 0;  // bit o: output o's accumulator columns hold a value
            for (int j = 0; j < NI && ok; ++j) {
                const int s = j % NS, r = j / NS;
                const int g = j >> CB, l = j & (NQ - 1);
                bool mine = (l % NMMA) == mw;  // the own block, or the one output of a translated input
                if (g == 0)
#pragma unroll
                    for (int p = 0; p < CB; ++p) mine = mine || ((l ^ (1 << p)) % NMMA) == mw;
                if (mine) {
                    if (!__all_sync(0xffffffffu, tc_wait(bar_tfull(s), r & 1, abort))) break;
                    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                    const uint32_t a_hi = tmem + Cfg::Slot0 + 16 * s, a_lo = a_hi + 8;
                    auto issue = [&](int o, uint32_t bt) {
                        if (o % NMMA != mw) return;
                        const uint32_t d = tmem + 16 * o;
                        tc_mma_elect(d, a_hi, tc_bdesc(bt), (written >> o) & 1u);  // the first one overwrites
                        tc_mma_elect(d, a_lo, tc_bdesc(bt + kTcB), 1u);
                        written |= 1u << o;
                    };
                    if (g == 0) {
                        issue(l, diag_s + l * 2 * kTcB);  // own block
#pragma unroll
                        for (int p = 0; p < CB; ++p) {
                            const int o = l ^ (1 << p);
                            issue(o, flip_s + ((p * 2 + ((o >> p) & 1)) * 2) * kTcB);
                        }
                    } else {
                        const int p = CB + g - 1;
                        issue(l, flip_s + ((p * 2 + ((q0 >> p) & 1)) * 2) * kTcB);
                    }
                }
                if (s % 4 == 3) tc_commit_elect(bar_tempty(s));  // this warp's share of the quad's release
            }
            tc_commit_elect(bar_done);  // completes once every MMA this warp issued has
        }
    } else {
        // ------------------------------------------------------------ producers
        const int grp = warp >> 2, wq = warp & 3;       // warpgroup, and its warp's TMEM lane quarter
        const int lane_traj = 32 * wq + lane;           // TMEM lane = trajectory in the tile
        const int pair_off = (lane_traj & ~1) * 8;      // byte offset of the trajectory pair in a row
        const bool odd = lane_traj & 1;
        const uint32_t lane_addr = tmem + (static_cast<uint32_t>(32 * wq) << 16);
        // every wait's outcome is made uniform over the warp: the tcgen05.st/ld
        // and the shuffles below are warp-collective
        bool ok = __all_sync(0xffffffffu, tc_wait(bar_own, 0, abort));
        // Inputs go in pairs (NI and HB are even, pairs never straddle a stage):
        // both are split and stored before one tcgen05.wait::st.
        for (int j0 = 2 * grp; j0 < NI && ok; j0 += 2 * G) {
            uint32_t pk[2][16];
            if (j0 >= NQ) {
                const int c = (j0 - NQ) / HB;
                if (!__all_sync(0xffffffffu, tc_wait(bar_sfull(c % NSTG), (c / NSTG) & 1, abort))) break;
            }
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                float x[8];  // Re rows 0..3, Im rows 0..3
#pragma unroll
                for (int a = 0; a < 4; ++a) {
                    const float4 v = *reinterpret_cast<const float4 *>(sm + input_row(j0 + h, a) + pair_off);
                    x[a] = odd ? v.y : v.x;
                    x[4 + a] = odd ? v.w : v.z;
                }
#pragma unroll
                for (int cc = 0; cc < 8; ++cc) {
                    const float hi = tc_head(x[cc]);
                    pk[h][cc] = __float_as_uint(hi);
                    pk[h][8 + cc] = __float_as_uint(x[cc] - hi);
                }
            }
            if (j0 >= NQ) {
                __syncwarp();
                if (lane == 0) tc_arrive(bar_sempty(((j0 - NQ) / HB) % NSTG));
            }
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int j = j0 + h, s = j % NS, r = j / NS;
                if (!__all_sync(0xffffffffu, tc_wait(bar_tempty(s), (r & 1) ^ 1, abort))) {
                    ok = false;
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                tc_st16(lane_addr + Cfg::Slot0 + 16 * s, pk[h]);
            }
            if (!ok) break;
            asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncwarp();
            if (lane == 0) {
                tc_arrive(bar_tfull(j0 % NS));
                tc_arrive(bar_tfull((j0 + 1) % NS));
            }
        }
        // ------------------------------------------------------------ epilogue
        bool done = tc_wait(bar_done, 0, abort);
        if (!done)  // every MMA warp commits this barrier whatever happened: let their MMAs drain
            for (uint32_t it = 0; it < kTcWait && !tc_try(bar_done, 0); ++it) {
            }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        double acc = 0.0;
        const bool live = lane_traj < nvalid;
        const int t = t0 + lane_traj;
        const float sc = live ? static_cast<float>(sj[t]) : 0.f;
        if (__all_sync(0xffffffffu, done && ok && !*abort)) {
            for (int o = grp; o < NQ; o += G) {
                uint32_t dv[16];  // [main (8) | correction (8)]
                tc_ld16(lane_addr + 16 * o, dv);
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                float y[8];
#pragma unroll
                for (int i = 0; i < 8; ++i) y[i] = (__uint_as_float(dv[8 + i]) + __uint_as_float(dv[i])) * sc;
                const int b = rows[o];
#pragma unroll
                for (int a = 0; a < 4; ++a) {
                    // own input rows of this output (for alpha), pair-planar
                    const float4 v = *reinterpret_cast<const float4 *>(sm + input_row(o, a) + pair_off);
                    const float vr = odd ? v.y : v.x, vi = odd ? v.w : v.z;
                    acc += static_cast<double>(vr) * y[a] + static_cast<double>(vi) * y[4 + a];
                    // the pair's float4 {re t, re t+1, im t, im t+1}: lanes t, t^1 exchange
                    const float pr = __shfl_xor_sync(0xffffffffu, y[a], 1);
                    const float pi = __shfl_xor_sync(0xffffffffu, y[4 + a], 1);
                    if (live && ((a & 1) == static_cast<int>(odd))) {
                        // even lanes store rows 0 and 2, odd lanes rows 1 and 3
                        const float4 st = odd ? make_float4(pr, y[a], pi, y[4 + a]) : make_float4(y[a], pr, y[4 + a], pi);
                        *reinterpret_cast<float4 *>(U + static_cast<size_t>(b + off[a]) * ldm + t0 + (lane_traj & ~1)) = st;
                    }
                }
            }
        }
        s_alpha[grp][lane_traj] = acc;
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (*abort) {
        if (tid == 0) atomicOr(status, 4);
    } else if (tid < kTcTraj && tid < nvalid) {
        // alpha partial of trajectory t0 + tid over this cube, groups in order
        double a = 0.0;
#pragma unroll
        for (int g = 0; g < G; ++g) a += s_alpha[g][tid];
        part[static_cast<size_t>(cube) * ldm + t0 + tid] = a * static_cast<double>(static_cast<float>(sj[t0 + tid]));
    }
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(Cfg::Cols));
    }
}

}  // namespace msgpu
