// msgpu_fused.cuh -- the complex64 Lanczos recurrence of one time step as
// one cluster-resident kernel (sm_90+ thread-block clusters, distributed
// shared memory).
//
// The streamed complex64 step runs, for every Krylov iteration j, the quartet
// SpMM U = H v_j (13 neighbour quartets gathered through L1/L2 per output
// quartet), a reduction for alpha_j, the three-term update into w_{j+1} and a
// reduction for beta_{j+1}: four launches and about 48 bytes of HBM traffic
// per vector element and iteration, with the SpMM held by its L2 gathers.
//
// Here one thread-block cluster of C CTAs owns two trajectory pairs (four
// trajectories) for the whole recurrence.  CTA r holds quartets
// [r Qc, (r+1) Qc) of those trajectories' current and previous Krylov vectors
// in shared memory, together with its quartets' block descriptors and row
// pointers (staged once per launch); thread l holds quartet r Qc + l for both
// pairs, so a block's descriptor, gather address and values serve four
// trajectories.  The SpMM gathers come from the CTA's own shared memory or,
// for a quartet owned by another CTA, from that CTA's shared memory through
// the cluster window.  alpha_j and
// |w_{j+1}|^2 are summed per CTA, exchanged through distributed shared memory
// and closed by a cluster barrier; every CTA then holds the same scalars.
// HBM sees the state once and each new basis vector once (the combine reads
// them back): 8 bytes per element and iteration.
//
// The arithmetic is that of k_lanczos_apply_* (the same quartet blocks, FP32
// pair-planar FMAs), k_lanczos_reduce and k_lanczos_update.  The blocks of a
// quartet are taken in stride order (diagonal first, one flip block per
// nucleus), the same on every lane of a warp, rather than in neighbour-row
// order, so U agrees with the four-kernel iteration to FP32 rounding, and
// alpha and |w|^2 differ from it in the order of their FP64 sums.
//
// Control flow is uniform: every thread of every CTA runs the same m
// iterations and reaches the same cluster barriers (inactive quartets are
// skipped with a branch, never with a return), and no CTA touches another
// CTA's shared memory after the last barrier it takes part in.
#pragma once

#include <cooperative_groups.h>

#include "msgpu_kernels.cuh"

namespace msgpu {

constexpr int kFusedThreads = 512;
constexpr int kFusedPairs = 2;                  // trajectory pairs per cluster, both held by every thread
constexpr int kFusedMaxQc = kFusedThreads;      // quartets per CTA: one per thread
constexpr int kFusedWarps = kFusedThreads / 32;

// Quartet form for the fused kernel.  Each quartet's own (diagonal) block is
// kept apart as a full 4x4 (diag, row-major in the pair index, 8 float4 per
// quartet, staged in shared memory); the other blocks are listed per quartet
// in stride order with blk.x = local quartet << 7 | owner rank << 3 | type
// (owner and local index of the neighbour quartet for the cluster size the
// descriptors were built for) and blk.y = value offset into val (float4 units,
// two complex values each, in the storage order of the type).
struct QuartetF {
    const int *rowptr;    // Q + 1, over the off-diagonal blocks
    const int2 *blk;
    const float4 *val;
    const float4 *diag;   // Q x 8
    const int *base;      // Q
};

// Dynamic shared memory of one CTA: the vector buffer [4 rows][2 pairs][Qc],
// the diagonal blocks [8][Qc], the CTA's descriptors and row pointers, and
// the reduction scratch.
__host__ __device__ inline size_t fused_smem_bytes(int Qc, int nblk, int C)
{
    return static_cast<size_t>(4 * kFusedPairs + 8) * Qc * sizeof(float4) + static_cast<size_t>(nblk) * sizeof(int2) +
           (2 * static_cast<size_t>(C) * 4 + kFusedWarps * 4 + 2 * 4) * sizeof(double) + 2 * 4 * sizeof(float) +
           (4 + static_cast<size_t>(Qc) + 1) * sizeof(int) + 16;
}

// diag[q] = the full 4x4 of quartet q's own block from the quartet values
// (qv: complex64 pairs; src[q] = {type, value offset in float4 units}, type
// -1 for a quartet without one).  The element (a, b) of each type sits where
// quartet_block reads it.  One thread per (quartet, float4 of the output).
__global__ void k_fused_diag(const int2 *__restrict__ src, const float2 *__restrict__ qv, float4 *__restrict__ diag,
                             int Q)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 8 * Q) return;
    const int q = i >> 3, s = i & 7;
    const int2 d = src[q];
    float v[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        const int f = 2 * s + h, a = f >> 2, b = f & 3;
        const int a1 = a >> 1, a2 = a & 1, b1 = b >> 1, b2 = b & 1;
        int ci = -1;
        switch (d.x) {
        case 0: ci = f; break;
        case 1: ci = a2 == b2 ? (2 * a2 + a1) * 2 + b1 : -1; break;
        case 2: ci = a1 == b1 ? (2 * a1 + a2) * 2 + b2 : -1; break;
        case 3: ci = a == b ? a : -1; break;
        case 4: ci = a2 == b2 ? 2 * a1 + b1 : -1; break;
        case 5: ci = a1 == b1 ? 2 * a2 + b2 : -1; break;
        default: break;
        }
        if (ci >= 0) {
            const float2 c = qv[2 * static_cast<size_t>(d.y) + ci];
            v[2 * h] = c.x;
            v[2 * h + 1] = c.y;
        }
    }
    diag[i] = make_float4(v[0], v[1], v[2], v[3]);
}

// Sum of v over the 32 lanes of a warp (every lane receives it).
__device__ __forceinline__ double fused_warp_sum(double v)
{
#pragma unroll
    for (int s = 16; s > 0; s >>= 1) v += __shfl_xor_sync(0xffffffffu, v, s);
    return v;
}

// Per-CTA sums of the four trajectories' partials v[0..3] (every thread
// contributes), written into slot `rank` of `dst` in every CTA of the cluster.
template <int C>
__device__ __forceinline__ void fused_cluster_partials(cooperative_groups::cluster_group &cl, int rank, double *dst,
                                                       double *wred, const double (&v)[4])
{
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const double s = fused_warp_sum(v[i]);
        if (lane == 0) wred[warp * 4 + i] = s;
    }
    __syncthreads();
    if (tid < 4) {
        double s = 0.0;
        for (int w = 0; w < kFusedWarps; ++w) s += wred[w * 4 + tid];
#pragma unroll
        for (int r = 0; r < C; ++r) cl.map_shared_rank(dst, r)[rank * 4 + tid] = s;
    }
}

// Wb: basis slots [m][D][ldm] (slot 0 = the state); sc: scales [m][ldm] (slot
// 0 set by the caller); td/to: per trajectory T diagonal / off-diagonal (stride
// m); mdim: per trajectory Krylov dimension, 0 on entry.  Outputs are those
// of the streamed loop: slots 1..m-1 of Wb and sc, td, to and mdim.  Grid:
// C x (ldm / 4) CTAs in clusters of C; thread l of CTA r holds quartet
// r Qc + l for both pairs; nblk_max: descriptors of the largest CTA range.
//
// One vector buffer suffices: the gathers of iteration j read v_j before the
// first cluster barrier, and only after it does each thread overwrite its own
// elements with w_{j+1}; v_{j-1} for the update comes back from basis slot
// j-1, which the same thread wrote.
template <int C>
__global__ void __launch_bounds__(kFusedThreads, 1)
k_lanczos_fused(QuartetF H, float2 *__restrict__ Wb, size_t n, double *__restrict__ sc, double *__restrict__ td,
                double *__restrict__ to, int *__restrict__ mdim, int Q, int Qc, int nblk_max, int ldm, int m, int s1,
                int s2)
{
    namespace cg = cooperative_groups;
    cg::cluster_group cl = cg::this_cluster();
    const int rank = static_cast<int>(cl.block_rank());
    const int ql = threadIdx.x;
    const int t0 = static_cast<int>(blockIdx.x / C) * (2 * kFusedPairs);  // first trajectory of the cluster

    extern __shared__ __align__(16) unsigned char fsm[];
    float4 *buf = reinterpret_cast<float4 *>(fsm);                        // [4 rows][2 pairs][Qc]
    float4 *sdiag = buf + 4 * kFusedPairs * static_cast<size_t>(Qc);     // [8][Qc]
    int2 *sblk = reinterpret_cast<int2 *>(sdiag + 8 * static_cast<size_t>(Qc));
    double *apart = reinterpret_cast<double *>(sblk + nblk_max);  // [C][4] alpha partials, by source rank
    double *npart = apart + C * 4;                                // [C][4] |w|^2 partials
    double *wred = npart + C * 4;                                 // [warps][4]
    double *tsc = wred + kFusedWarps * 4;                         // s_j per trajectory
    double *tsp = tsc + 4;                                        // s_{j-1}
    float *tca = reinterpret_cast<float *>(tsp + 4);              // alpha_j s_j
    float *tcb = tca + 4;                                         // s_{j-1} / s_j
    int *tmd = reinterpret_cast<int *>(tcb + 4);                  // Krylov dimension (0: open)
    int *srow = tmd + 4;                                          // local row pointers (Qc + 1)
    const int off[4] = {0, s2, s1, s1 + s2};

    // ---- stage this CTA's quartet structure and the state
    const int qbeg = min(Q, rank * Qc), qend = min(Q, qbeg + Qc);
    const int kb0 = __ldg(H.rowptr + qbeg), nloc = qend - qbeg;
    const bool live = ql < nloc;
    for (int i = ql; i <= Qc; i += kFusedThreads) srow[i] = __ldg(H.rowptr + min(qbeg + i, qend)) - kb0;
    for (int i = ql; i < __ldg(H.rowptr + qend) - kb0; i += kFusedThreads) sblk[i] = __ldg(H.blk + kb0 + i);
    const int b0 = live ? __ldg(H.base + qbeg + ql) : 0;
    if (live) {
#pragma unroll
        for (int k = 0; k < 8; ++k) sdiag[k * Qc + ql] = __ldg(H.diag + 8 * static_cast<size_t>(qbeg + ql) + k);
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int p = 0; p < kFusedPairs; ++p)
                buf[(a * kFusedPairs + p) * Qc + ql] =
                    *reinterpret_cast<const float4 *>(Wb + static_cast<size_t>(b0 + off[a]) * ldm + t0 + 2 * p);
    }
    if (ql < 4) {
        tsc[ql] = sc[t0 + ql];
        tsp[ql] = 0.0;
        tmd[ql] = mdim[t0 + ql];
    }
    cl.sync();

    for (int j = 0; j < m; ++j) {
        float s[kFusedPairs][2];
#pragma unroll
        for (int p = 0; p < kFusedPairs; ++p) {
            s[p][0] = static_cast<float>(tsc[2 * p]);
            s[p][1] = static_cast<float>(tsc[2 * p + 1]);
        }

        // ---- U = H v_j on this thread's quartet; partial alpha_j = Re <v_j, U>
        float2 U[kFusedPairs][4][2];
#pragma unroll
        for (int p = 0; p < kFusedPairs; ++p)
#pragma unroll
            for (int a = 0; a < 4; ++a) U[p][a][0] = U[p][a][1] = make_float2(0.f, 0.f);
        if (live) {
            {
                // own block, values from shared memory (the full type-0 arithmetic)
                float4 x[kFusedPairs][4];
#pragma unroll
                for (int b = 0; b < 4; ++b)
#pragma unroll
                    for (int p = 0; p < kFusedPairs; ++p) x[p][b] = buf[(b * kFusedPairs + p) * Qc + ql];
#pragma unroll
                for (int a = 0; a < 4; ++a) {
                    const float4 pv = sdiag[(2 * a) * Qc + ql], qv = sdiag[(2 * a + 1) * Qc + ql];
#pragma unroll
                    for (int p = 0; p < kFusedPairs; ++p) {
                        mac_pp(U[p][a], pv.x, pv.y, x[p][0]);
                        mac_pp(U[p][a], pv.z, pv.w, x[p][1]);
                        mac_pp(U[p][a], qv.x, qv.y, x[p][2]);
                        mac_pp(U[p][a], qv.z, qv.w, x[p][3]);
                    }
                }
            }
            const int ke = srow[ql + 1];
            for (int kk = srow[ql]; kk < ke; ++kk) {
                const int2 bd = sblk[kk];
                const int r = (bd.x >> 3) & 15;
                float4 x[kFusedPairs][4];
                if (r == rank) {
                    const float4 *src = buf + (bd.x >> 7);
#pragma unroll
                    for (int b = 0; b < 4; ++b)
#pragma unroll
                        for (int p = 0; p < kFusedPairs; ++p) x[p][b] = src[(b * kFusedPairs + p) * Qc];
                } else {
                    const float4 *src = cl.map_shared_rank(buf + (bd.x >> 7), r);
#pragma unroll
                    for (int b = 0; b < 4; ++b)
#pragma unroll
                        for (int p = 0; p < kFusedPairs; ++p) x[p][b] = src[(b * kFusedPairs + p) * Qc];
                }
                quartet_block_np<kFusedPairs>(U, bd.x & 7, H.val + bd.y, x);
            }
        }
        double part[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
        for (int p = 0; p < kFusedPairs; ++p)
#pragma unroll
            for (int a = 0; a < 4; ++a) {
                U[p][a][0] = make_float2(U[p][a][0].x * s[p][0], U[p][a][0].y * s[p][1]);
                U[p][a][1] = make_float2(U[p][a][1].x * s[p][0], U[p][a][1].y * s[p][1]);
                if (live) {
                    const float4 v = buf[(a * kFusedPairs + p) * Qc + ql];  // {re t, re t+1, im t, im t+1}
                    part[2 * p] += (static_cast<double>(v.x) * U[p][a][0].x + static_cast<double>(v.z) * U[p][a][1].x) *
                                   s[p][0];
                    part[2 * p + 1] +=
                        (static_cast<double>(v.y) * U[p][a][0].y + static_cast<double>(v.w) * U[p][a][1].y) * s[p][1];
                }
            }
        fused_cluster_partials<C>(cl, rank, apart, wred, part);
        cl.sync();

        // ---- alpha_j (k_lanczos_reduce mode 0) and the update coefficients
        if (ql < 4) {
            double al = 0.0;
#pragma unroll
            for (int r = 0; r < C; ++r) al += apart[r * 4 + ql];
            if (tmd[ql] == 0) {
                if (rank == 0) td[static_cast<size_t>(t0 + ql) * m + j] = al;
                if (j == m - 1) {
                    tmd[ql] = m;
                    if (rank == 0) mdim[t0 + ql] = m;
                }
            }
            tca[ql] = static_cast<float>(al * tsc[ql]);
            tcb[ql] = (j > 0 && tsc[ql] > 0.0) ? static_cast<float>(tsp[ql] / tsc[ql]) : 0.f;
        }
        if (j == m - 1) break;  // T_m is complete; w_m is never used
        __syncthreads();

        // ---- w_{j+1} = U - alpha_j v_j - beta_j v_{j-1} (k_lanczos_update), in
        // place of v_j; partial |w_{j+1}|^2
        double nrm[4] = {0.0, 0.0, 0.0, 0.0};
        if (live) {
            float2 *wn = Wb + static_cast<size_t>(j + 1) * n;
            const float2 *wp = Wb + static_cast<size_t>(j > 0 ? j - 1 : 0) * n;
            float4 pv[kFusedPairs][4];
#pragma unroll
            for (int p = 0; p < kFusedPairs; ++p)
#pragma unroll
                for (int a = 0; a < 4; ++a)
                    pv[p][a] = j > 0 ? *reinterpret_cast<const float4 *>(wp + static_cast<size_t>(b0 + off[a]) * ldm +
                                                                          t0 + 2 * p)
                                     : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
            for (int p = 0; p < kFusedPairs; ++p) {
                const float ca0 = tca[2 * p], ca1 = tca[2 * p + 1], cb0 = tcb[2 * p], cb1 = tcb[2 * p + 1];
#pragma unroll
                for (int a = 0; a < 4; ++a) {
                    const size_t e = static_cast<size_t>(a * kFusedPairs + p) * Qc + ql;
                    const float4 v = buf[e];
                    float4 w;
                    w.x = fmaf(-ca0, v.x, U[p][a][0].x);
                    w.y = fmaf(-ca1, v.y, U[p][a][0].y);
                    w.z = fmaf(-ca0, v.z, U[p][a][1].x);
                    w.w = fmaf(-ca1, v.w, U[p][a][1].y);
                    if (j > 0) {
                        w.x = fmaf(-cb0, pv[p][a].x, w.x);
                        w.y = fmaf(-cb1, pv[p][a].y, w.y);
                        w.z = fmaf(-cb0, pv[p][a].z, w.z);
                        w.w = fmaf(-cb1, pv[p][a].w, w.w);
                    }
                    buf[e] = w;
                    *reinterpret_cast<float4 *>(wn + static_cast<size_t>(b0 + off[a]) * ldm + t0 + 2 * p) = w;
                    nrm[2 * p] += static_cast<double>(w.x) * w.x + static_cast<double>(w.z) * w.z;
                    nrm[2 * p + 1] += static_cast<double>(w.y) * w.y + static_cast<double>(w.w) * w.w;
                }
            }
        }
        fused_cluster_partials<C>(cl, rank, npart, wred, nrm);
        cl.sync();

        // ---- beta_{j+1} (k_lanczos_reduce mode 1): scale of w_{j+1}, breakdown
        if (ql < 4) {
            double ss = 0.0;
#pragma unroll
            for (int r = 0; r < C; ++r) ss += npart[r * 4 + ql];
            const double beta = sqrt(ss);
            double scn = 0.0;
            if (tmd[ql] == 0) {
                if (rank == 0) to[static_cast<size_t>(t0 + ql) * m + j] = beta;
                if (beta < 1e-14) {
                    tmd[ql] = j + 1;
                    if (rank == 0) mdim[t0 + ql] = j + 1;
                } else {
                    scn = 1.0 / beta;
                }
            }
            if (rank == 0) sc[static_cast<size_t>(j + 1) * ldm + t0 + ql] = scn;
            tsp[ql] = tsc[ql];
            tsc[ql] = scn;
        }
        __syncthreads();
    }
}

}  // namespace msgpu
