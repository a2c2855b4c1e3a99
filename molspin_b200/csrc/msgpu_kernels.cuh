// msgpu_kernels.cuh -- kernels of the streamed Krylov propagation.
//
// One propagation step of a block of trajectories is a fixed sequence of
// kernels on one stream (captured into a CUDA graph by the host):
//
//   for j in 0..m-1:    apply   : W = A V_j          (CSR SpMM over the block)
//                       reduce  : per-trajectory dot products / norms
//                       orth    : Gram-Schmidt / three-term update
//   expm                : per-trajectory exp(dt H_m) e1 (one warp each)
//   combine             : psi = sum_j c_j V_j, singlet-triplet flips,
//                         electron-pair observables (quartet threads)
//   yield               : trapezoid accumulation per trajectory
//
// Reductions over the Hilbert dimension are two-phase and deterministic:
// every CTA writes one partial per trajectory, and a separate kernel sums the
// partials of all row tiles in a fixed order, so a trajectory's result does
// not depend on how many other trajectories share the launch.
#pragma once

#include <utility>

#include "msgpu_device.cuh"

namespace msgpu {
// Kernels defined in these headers have internal linkage: every translation
// unit that includes them gets its own copies.
namespace {

constexpr int kWarps = 8;           // warps per CTA in the row-tiled kernels
constexpr int kThreads = 32 * kWarps;
constexpr int kMaxKrylov = 32;

struct CsrD {
    const int *rowptr;
    const int *col;
    const double2 *val;
};
struct CsrF {
    const int *rowptr;
    const int *col;
    const float2 *hi;
    const float2 *lo;  // may be null: single-word values
};

// ===================================================================== c128
// Arnoldi on G = -iH - K with classical Gram-Schmidt applied twice (CGS2),
// trajectory tile of 32 (one trajectory per lane, 16-byte loads).

// The Krylov index j is a template parameter (J) of k_arnoldi_dots and
// k_arnoldi_orth, so that the per-trajectory arrays over i <= j (dot
// accumulators, a row of every V_i) have static indices and live in
// registers: with a runtime j they sat in local memory, whose traffic spilled
// to DRAM (more bytes written by the Gram-Schmidt pass than the vector it
// updates).  The host picks the instantiation from a table
// (arnoldi_orth_fn); the arithmetic and its order are those of one generic
// loop over i.

// W = G * v_j where v_j = src * scale[t]; also stores v_j into Vj.  The
// first-pass dots <V_i, W> are k_arnoldi_dots: fused here they held
// this kernel (whose CSR gathers want occupancy) to two CTAs per SM.
__global__ void __launch_bounds__(kThreads)
k_arnoldi_apply(CsrD H, CsrD K, double kappa, const double2 *__restrict__ src, const double *__restrict__ scale,
                double2 *__restrict__ Vj, double2 *__restrict__ W, int D, int ldm, int R)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int t = blockIdx.y * 32 + lane;
    const int r0 = blockIdx.x * R;
    const double sc = scale[t];
    // a row's column indices and values, 32 at a time, staged by the warp with
    // one coalesced load each, so the gathers below wait on no dependent load
    __shared__ int scol[kWarps][32];
    __shared__ double2 sval[kWarps][32];
    for (int r = r0 + warp; r < min(r0 + R, D); r += kWarps) {
        double2 acc = make_double2(0.0, 0.0);
        const int kb = __ldg(H.rowptr + r), ke = __ldg(H.rowptr + r + 1);
        for (int k0 = kb; k0 < ke; k0 += 32) {
            const int nk = min(32, ke - k0);
            __syncwarp();
            if (lane < nk) {
                scol[warp][lane] = __ldg(H.col + k0 + lane);
                sval[warp][lane] = __ldg(H.val + k0 + lane);
            }
            __syncwarp();
#pragma unroll 4
            for (int u = 0; u < nk; ++u)
                acc = cfma(sval[warp][u], src[static_cast<size_t>(scol[warp][u]) * ldm + t], acc);
        }
        acc = cscale(acc, sc);
        const double2 vr = cscale(src[static_cast<size_t>(r) * ldm + t], sc);
        double2 g = make_double2(acc.y, -acc.x);  // -i * acc
        if (K.rowptr) {
            double2 ka = make_double2(0.0, 0.0);
            const int qb = __ldg(K.rowptr + r), qe = __ldg(K.rowptr + r + 1);
            for (int k = qb; k < qe; ++k)
                ka = cfma(__ldg(K.val + k), src[static_cast<size_t>(__ldg(K.col + k)) * ldm + t], ka);
            g = csub(g, cscale(ka, sc));
        } else {
            g = csub(g, cscale(vr, kappa));
        }
        const size_t e = static_cast<size_t>(r) * ldm + t;
        Vj[e] = vr;
        W[e] = g;
    }
}

// The complex128 quartet form: the compact blocks of QuartetC with FP64
// values (double2 per complex value, in the same order; a block's value
// offset counts float4 units, two complex values each).
struct QuartetD {
    const int *rowptr;   // Q + 1
    const int2 *blk;     // nblocks
    const double2 *val;  // complex values
    const int *base;     // Q
};

// o[a] += sum_b B[a][b] x[b] for one compact block of type `type` (the
// layouts of QuartetC), complex128.
__device__ __forceinline__ void quartet_block_d(double2 o[4], int type, const double2 *__restrict__ v,
                                                const double2 x[4])
{
    switch (type) {
    case 0:
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < 4; ++b) o[a] = cfma(__ldg(v + 4 * a + b), x[b], o[a]);
        break;
    case 1:  // [a2][a1][b1]
#pragma unroll
        for (int a2 = 0; a2 < 2; ++a2)
#pragma unroll
            for (int a1 = 0; a1 < 2; ++a1)
#pragma unroll
                for (int b1 = 0; b1 < 2; ++b1)
                    o[2 * a1 + a2] = cfma(__ldg(v + (2 * a2 + a1) * 2 + b1), x[2 * b1 + a2], o[2 * a1 + a2]);
        break;
    case 2:  // [a1][a2][b2]
#pragma unroll
        for (int a1 = 0; a1 < 2; ++a1)
#pragma unroll
            for (int a2 = 0; a2 < 2; ++a2)
#pragma unroll
                for (int b2 = 0; b2 < 2; ++b2)
                    o[2 * a1 + a2] = cfma(__ldg(v + (2 * a1 + a2) * 2 + b2), x[2 * a1 + b2], o[2 * a1 + a2]);
        break;
    case 3:
#pragma unroll
        for (int a = 0; a < 4; ++a) o[a] = cfma(__ldg(v + a), x[a], o[a]);
        break;
    case 4: {  // A (x) I on digit 1: [a1][b1]
        const double2 A00 = __ldg(v), A01 = __ldg(v + 1), A10 = __ldg(v + 2), A11 = __ldg(v + 3);
#pragma unroll
        for (int a2 = 0; a2 < 2; ++a2) {
            const double2 x0 = x[a2], x1 = x[2 + a2];
            o[a2] = cfma(A01, x1, cfma(A00, x0, o[a2]));
            o[2 + a2] = cfma(A11, x1, cfma(A10, x0, o[2 + a2]));
        }
        break;
    }
    default: {  // I (x) A on digit 2: [a2][b2]
        const double2 A00 = __ldg(v), A01 = __ldg(v + 1), A10 = __ldg(v + 2), A11 = __ldg(v + 3);
#pragma unroll
        for (int a1 = 0; a1 < 2; ++a1) {
            const double2 x0 = x[2 * a1], x1 = x[2 * a1 + 1];
            o[2 * a1] = cfma(A01, x1, cfma(A00, x0, o[2 * a1]));
            o[2 * a1 + 1] = cfma(A11, x1, cfma(A10, x0, o[2 * a1 + 1]));
        }
        break;
    }
    }
}

// k_arnoldi_apply over quartet blocks for K = kappa I: a warp per output
// quartet, a lane per trajectory.  A row and trajectory gathers 13 quartet
// rows of 16 B at D = 16384 (radical pair, 12 nuclear spins) against 27 CSR
// entries, and the block descriptors and values are loaded once per quartet
// for its four rows.  Summation runs in block order, not CSR order.
__global__ void __launch_bounds__(kThreads)
k_arnoldi_apply_q(QuartetD H, double kappa, const double2 *__restrict__ src, const double *__restrict__ scale,
                  double2 *__restrict__ Vj, double2 *__restrict__ W, int Q, int s1, int s2, int ldm)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int t = blockIdx.y * 32 + lane;
    const int q = blockIdx.x * kWarps + warp;
    if (q >= Q) return;
    const double sc = scale[t];
    const int off[4] = {0, s2, s1, s1 + s2};
    double2 o[4];
#pragma unroll
    for (int a = 0; a < 4; ++a) o[a] = make_double2(0.0, 0.0);
    double2 x[4];
    int last = -1;
    const int kb = __ldg(H.rowptr + q), ke = __ldg(H.rowptr + q + 1);
    for (int kk = kb; kk < ke; ++kk) {
        const int2 cur = __ldg(H.blk + kk);
        last = cur.x >> 3;
#pragma unroll
        for (int b = 0; b < 4; ++b) x[b] = src[static_cast<size_t>(last + off[b]) * ldm + t];
        quartet_block_d(o, cur.x & 7, H.val + 2 * static_cast<size_t>(cur.y), x);
    }
    // the quartet's own block comes last: its gathered rows are v_j here
    const int base = __ldg(H.base + q);
    const bool own = last == base;
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        const size_t e = static_cast<size_t>(base + off[a]) * ldm + t;
        const double2 vr = cscale(own ? x[a] : src[e], sc);
        const double2 acc = cscale(o[a], sc);
        Vj[e] = vr;
        W[e] = csub(make_double2(acc.y, -acc.x), cscale(vr, kappa));  // -i H v - kappa v
    }
}

// Partial dots <V_i, W>, i <= j (the first Gram-Schmidt pass; W unchanged,
// h unused).  Each V_i is used once and the compiler keeps every load of a
// row in flight; two CTAs per SM bound its registers.
template <int J>
__global__ void __launch_bounds__(kThreads, 2)
k_arnoldi_dots(double2 *__restrict__ W, const double2 *__restrict__ V, size_t vstride,
               const double2 *__restrict__ h, double2 *__restrict__ part, int D, int ldm, int R)
{
    (void)h;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int t = blockIdx.y * 32 + lane;
    const int r0 = blockIdx.x * R;
    double2 dacc[J + 1];
#pragma unroll
    for (int i = 0; i <= J; ++i) dacc[i] = make_double2(0.0, 0.0);
    for (int r = r0 + warp; r < min(r0 + R, D); r += kWarps) {
        const size_t e = static_cast<size_t>(r) * ldm + t;
        const double2 w = W[e];
#pragma unroll
        for (int i = 0; i <= J; ++i) dacc[i] = cadd(dacc[i], cconjmul(__ldg(V + i * vstride + e), w));
    }
    __shared__ double2 sm[kWarps][32];
#pragma unroll  // static indices keep dacc in registers
    for (int i = 0; i <= J; ++i) {
        sm[warp][lane] = dacc[i];
        __syncthreads();
        if (warp == 0) {
            double2 s = sm[0][lane];
            for (int w = 1; w < kWarps; ++w) s = cadd(s, sm[w][lane]);
            part[(static_cast<size_t>(blockIdx.x) * (J + 1) + i) * ldm + t] = s;
        }
        __syncthreads();
    }
}

// W -= sum_{i<=j} h[i][t] V_i; then partial dots <V_i, W> (MODE 1) or the
// partial squared norm |W|^2 (MODE 2, stored in .x).  The coefficients sit in
// shared memory; a row's V_i are all loaded before the first is used.
template <int J, int MODE>
__global__ void __launch_bounds__(kThreads)
k_arnoldi_orth(double2 *__restrict__ W, const double2 *__restrict__ V, size_t vstride,
               const double2 *__restrict__ h, double2 *__restrict__ part, int D, int ldm, int R)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int t = blockIdx.y * 32 + lane;
    const int r0 = blockIdx.x * R;
    __shared__ double2 hc[J + 1][32];
    for (int k = threadIdx.x; k < (J + 1) * 32; k += kThreads)
        hc[k >> 5][k & 31] = h[static_cast<size_t>(k >> 5) * ldm + blockIdx.y * 32 + (k & 31)];
    __syncthreads();
    constexpr int ND = MODE == 1 ? J + 1 : 1;
    double2 dacc[ND];
#pragma unroll
    for (int i = 0; i < ND; ++i) dacc[i] = make_double2(0.0, 0.0);
    for (int r = r0 + warp; r < min(r0 + R, D); r += kWarps) {
        const size_t e = static_cast<size_t>(r) * ldm + t;
        double2 w = W[e];
        double2 vi[J + 1];  // every load of the row in flight before the first use
#pragma unroll
        for (int i = 0; i <= J; ++i) vi[i] = __ldg(V + i * vstride + e);
#pragma unroll
        for (int i = 0; i <= J; ++i) w = csub(w, cmul(hc[i][lane], vi[i]));
        W[e] = w;
        if (MODE == 1) {
#pragma unroll
            for (int i = 0; i <= J; ++i) dacc[i] = cadd(dacc[i], cconjmul(vi[i], w));
        } else {
            dacc[0].x += cabs2(w);
        }
    }
    __shared__ double2 sm[kWarps][32];
#pragma unroll  // static indices keep dacc in registers
    for (int i = 0; i < ND; ++i) {
        sm[warp][lane] = dacc[i];
        __syncthreads();
        if (warp == 0) {
            double2 s = sm[0][lane];
            for (int w = 1; w < kWarps; ++w) s = cadd(s, sm[w][lane]);
            part[(static_cast<size_t>(blockIdx.x) * ND + i) * ldm + t] = s;
        }
        __syncthreads();
    }
}

// ------------------------------------------------ complex64 Arnoldi (general K on the pair)
// The complex64 form for a reaction operator K = I (x) K4 that acts on the
// electron pair only (unequal sinks: K = sum_c k_c/2 P_c).  Basis slot j holds
// w_j unnormalised in the pair-planar layout, with the per-trajectory scale
// s_j = 1 / |w_j| (v_j = s_j w_j), as in the Lanczos form; the quartet SpMM
// gives U = H v_j.  Arithmetic in FP64 (FP32 storage), one trajectory per lane:
// a lane reads its trajectory's re and im words of the pair's 16 bytes.

struct PairK {
    double2 k[16];  // K4, row-major in the pair index a = 2 a1 + a2
};

// W = -i U - K4 v_j per quartet, stored as w_{j+1} (before orthogonalisation).
// Grid (ceil(Q / 8), ldm / 64), 256 threads: a warp per quartet, a lane per
// trajectory pair.
__global__ void __launch_bounds__(kThreads)
k_arn64_apply(PairK K, const float2 *__restrict__ U, const float2 *__restrict__ wj, const double *__restrict__ sj,
              float2 *__restrict__ W, int Q, int s1, int s2, int ldm)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int t = blockIdx.y * 64 + 2 * lane;
    const int q = blockIdx.x * kWarps + warp;
    if (q >= Q) return;
    const int base = quartet_base(q, s1, s2);
    const int off[4] = {0, s2, s1, s1 + s2};
    const double sc0 = sj[t], sc1 = sj[t + 1];
    double2 v[2][4], u[2][4];
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        const size_t e = static_cast<size_t>(base + off[a]) * ldm + t;
        const float4 x = *reinterpret_cast<const float4 *>(wj + e);
        const float4 h = *reinterpret_cast<const float4 *>(U + e);
        v[0][a] = make_double2(x.x * sc0, x.z * sc0);
        v[1][a] = make_double2(x.y * sc1, x.w * sc1);
        u[0][a] = make_double2(h.x, h.z);
        u[1][a] = make_double2(h.y, h.w);
    }
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        double2 g[2];
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            double2 kv = make_double2(0.0, 0.0);
#pragma unroll
            for (int b = 0; b < 4; ++b) kv = cfma(K.k[4 * a + b], v[k][b], kv);
            g[k] = csub(make_double2(u[k][a].y, -u[k][a].x), kv);  // -i U - K v
        }
        *reinterpret_cast<float4 *>(W + static_cast<size_t>(base + off[a]) * ldm + t) =
            make_float4(static_cast<float>(g[0].x), static_cast<float>(g[1].x), static_cast<float>(g[0].y),
                        static_cast<float>(g[1].y));
    }
}

// MODE 0: partial dots <v_i, W>, i <= J; MODE 1: W -= sum_i h_i v_i, then the
// dots again; MODE 2: W -= sum_i h_i v_i, then |W|^2 (in .x).  v_i = s_i w_i
// from the basis slots: the update uses h_i s_i and the dots scale by s_i once
// at the end, so the per-element work is that of the complex128 kernels.
// Grid (ntiles, ldm / 32), a lane per trajectory (its re and im words of the
// pair's 16 bytes).  Partials go to part[tile][i][t] (the layout of the
// complex128 kernels).
template <int J, int MODE>
__global__ void __launch_bounds__(kThreads)
k_arn64_orth(float2 *__restrict__ W, const float2 *__restrict__ V, size_t vstride, const double *__restrict__ sc,
             const double2 *__restrict__ h, double2 *__restrict__ part, int D, int ldm, int R)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int t = blockIdx.y * 32 + lane;
    const int r0 = blockIdx.x * R;
    // per-trajectory h_i s_i and s_i, once per CTA
    __shared__ double2 hs[J + 1][32];
    __shared__ double si[J + 1][32];
    for (int k = threadIdx.x; k < (J + 1) * 32; k += kThreads) {
        const size_t e = static_cast<size_t>(k >> 5) * ldm + blockIdx.y * 32 + (k & 31);
        si[k >> 5][k & 31] = sc[e];
        hs[k >> 5][k & 31] = MODE == 0 ? make_double2(0.0, 0.0) : cscale(h[e], sc[e]);
    }
    __syncthreads();
    constexpr int ND = MODE == 2 ? 1 : J + 1;
    double2 dacc[ND];
#pragma unroll
    for (int i = 0; i < ND; ++i) dacc[i] = make_double2(0.0, 0.0);
    auto ld = [&](const float2 *x, int r) {
        const float *f = reinterpret_cast<const float *>(x + static_cast<size_t>(r) * ldm + (t & ~1)) + (t & 1);
        return make_double2(f[0], f[2]);
    };
    for (int r = r0 + warp; r < min(r0 + R, D); r += kWarps) {
        double2 w = ld(W, r);
        if (MODE != 0) {
#pragma unroll
            for (int i = 0; i <= J; ++i) w = csub(w, cmul(hs[i][lane], ld(V + i * vstride, r)));
            float *f = reinterpret_cast<float *>(W + static_cast<size_t>(r) * ldm + (t & ~1)) + (t & 1);
            f[0] = static_cast<float>(w.x);
            f[2] = static_cast<float>(w.y);
            w = make_double2(f[0], f[2]);  // the stored (rounded) vector is the one the next pass sees
        }
        if (MODE != 2) {
#pragma unroll
            for (int i = 0; i <= J; ++i) dacc[i] = cadd(dacc[i], cconjmul(ld(V + i * vstride, r), w));
        } else {
            dacc[0].x += cabs2(w);
        }
    }
    __shared__ double2 sm[kWarps][32];
#pragma unroll  // static indices keep dacc in registers
    for (int i = 0; i < ND; ++i) {
        sm[warp][lane] = MODE == 2 ? dacc[i] : cscale(dacc[i], si[i][lane]);
        __syncthreads();
        if (warp == 0) {
            double2 s = sm[0][lane];
            for (int w2 = 1; w2 < kWarps; ++w2) s = cadd(s, sm[w2][lane]);
            part[(static_cast<size_t>(blockIdx.x) * ND + i) * ldm + t] = s;
        }
        __syncthreads();
    }
}

using Arn64Fn = void (*)(float2 *, const float2 *, size_t, const double *, const double2 *, double2 *, int, int, int);
template <int J, int MODE>
constexpr Arn64Fn arn64_kernel() { return &k_arn64_orth<J, MODE>; }
template <int MODE, int... J>
Arn64Fn arn64_pick(int j, std::integer_sequence<int, J...>)
{
    static constexpr Arn64Fn table[] = {arn64_kernel<J, MODE>()...};
    return table[j];
}
// The complex64 Gram-Schmidt kernel of iteration j (0 <= j < kMaxKrylov), mode 0, 1 or 2.
inline Arn64Fn arn64_orth_fn(int j, int mode)
{
    constexpr auto js = std::make_integer_sequence<int, kMaxKrylov>{};
    return mode == 0 ? arn64_pick<0>(j, js) : mode == 1 ? arn64_pick<1>(j, js) : arn64_pick<2>(j, js);
}

using ArnoldiOrthFn = void (*)(double2 *, const double2 *, size_t, const double2 *, double2 *, int, int, int);

template <int J, int MODE>
constexpr ArnoldiOrthFn arnoldi_kernel()
{
    if constexpr (MODE == 0) return &k_arnoldi_dots<J>;
    else return &k_arnoldi_orth<J, MODE>;
}
template <int MODE, int... J>
ArnoldiOrthFn arnoldi_orth_pick(int j, std::integer_sequence<int, J...>)
{
    static constexpr ArnoldiOrthFn table[] = {arnoldi_kernel<J, MODE>()...};
    return table[j];
}
// The kernel of iteration j, 0 <= j < kMaxKrylov: mode 0 k_arnoldi_dots,
// modes 1 and 2 k_arnoldi_orth.
inline ArnoldiOrthFn arnoldi_orth_fn(int j, int mode)
{
    constexpr auto js = std::make_integer_sequence<int, kMaxKrylov>{};
    return mode == 0 ? arnoldi_orth_pick<0>(j, js) : mode == 1 ? arnoldi_orth_pick<1>(j, js) : arnoldi_orth_pick<2>(j, js);
}

// out[i][t] = sum over tiles of part[tile][i][t] (fixed order).
// Launch with blockDim (32, 8) and (ldm/32, ni) blocks; fixed summation order.
__global__ void k_reduce_partials(const double2 *__restrict__ part, int ntiles, int ni, int ldm,
                                  double2 *__restrict__ out)
{
    __shared__ double2 red[8][33];
    const int t = blockIdx.x * 32 + threadIdx.x, i = blockIdx.y;
    double2 ps = make_double2(0.0, 0.0);
    for (int tile = threadIdx.y; tile < ntiles; tile += 8)
        ps = cadd(ps, part[(static_cast<size_t>(tile) * ni + i) * ldm + t]);
    red[threadIdx.y][threadIdx.x] = ps;
    __syncthreads();
    if (threadIdx.y != 0) return;
    double2 s = make_double2(0.0, 0.0);
#pragma unroll
    for (int y = 0; y < 8; ++y) s = cadd(s, red[y][threadIdx.x]);
    out[static_cast<size_t>(i) * ldm + t] = s;
}

// Per-trajectory Arnoldi bookkeeping after CGS2 of iteration j:
// H_m[i][j] = h1[i] + h2[i]; beta = |W|; H_m[j+1][j] = beta; scale = 1/beta;
// a trajectory whose beta falls below 1e-14 (breakdown, as the reference) or
// that reached the last iteration keeps dimension j+1.
__global__ void k_arnoldi_finalize(const double2 *__restrict__ h1, const double2 *__restrict__ h2,
                                   const double2 *__restrict__ nrm, int j, int m, int ldm,
                                   double2 *__restrict__ hess, int *__restrict__ mdim, double *__restrict__ scale)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ldm) return;
    const bool active = mdim[t] == 0;
    double2 *Ht = hess + static_cast<size_t>(t) * m * m;  // column-major m x m
    for (int i = 0; i <= j; ++i) {
        const double2 v = cadd(h1[static_cast<size_t>(i) * ldm + t], h2[static_cast<size_t>(i) * ldm + t]);
        if (active) Ht[i + j * m] = v;
    }
    const double beta = sqrt(nrm[t].x);
    if (!active) { scale[t] = 0.0; return; }
    if (j == m - 1) { mdim[t] = m; scale[t] = 0.0; return; }
    Ht[(j + 1) + j * m] = make_double2(beta, 0.0);
    if (beta < 1e-14) { mdim[t] = j + 1; scale[t] = 0.0; return; }
    scale[t] = 1.0 / beta;
}

// ===================================================================== c64
// Lanczos on H (Hermitian) with complex64 vectors, complex64 H (optionally a
// hi+lo split), FP64 dot products / norms.  Trajectory tile of 64: each lane
// carries two trajectories in one 16-byte load.  Vectors are stored
// unnormalised (w_j) with a per-trajectory scale s_j = 1/|w_j|.

// ---------------------------------------------------------------- quartet SpMM
// H in quartet-block form: the rows of an electron-pair quartet (the four
// states of the two electron digits at one configuration of all other
// spins) form a block row; H[quartet q, quartet q'] is a 4x4 complex block.
// For radical pairs a block row has 1 + (number of nuclear flips) blocks
// (13 at D=16384 instead of 27 scalars per row), and each gathered quartet
// feeds all four output rows from registers.  Blocks are typed by their
// sparsity so the inner product only touches structural nonzeros.
//
// Compact quartet form: per block an int2 {base row << 3 | type, value
// offset}; values are complex64, two per float4 (offset counted in float4),
// and hold only what the type needs:
//   0 full 4x4 (16, row-major in the pair index a = 2*a1 + a2)
//   1 acts on digit 1 with a2 == b2: 8 values [a2][a1][b1]
//   2 acts on digit 2 with a1 == b1: 8 values [a1][a2][b2]
//   3 diagonal: 4 values [a]
//   4 A (x) I on digit 1: 4 values [a1][b1]
//   5 I (x) A on digit 2: 4 values [a2][b2]
// A hyperfine flip block S_e.A.I_n is type 4 or 5: 4 values instead of 16.
struct QuartetC {
    const int *rowptr;  // Q + 1
    const int2 *blk;    // nblocks
    const float4 *val;  // value pairs
    const int *base;    // Q
};

// Complex64 vectors are stored "pair-planar": the 16 bytes of trajectories
// (t, t+1), t even, hold {re(t), re(t+1), im(t), im(t+1)}.  One complex
// multiply-accumulate of a scalar b into both trajectories is then four
// packed FP32x2 FMAs (Blackwell FFMA2) on the re and im pairs.  Matrix values
// stay compact (two complex values per 16-byte load); they are broadcast into
// pairs in registers.
__device__ __forceinline__ void mac_pp(float2 o[2], float br_, float bi_, float4 x)
{
    const float2 br = make_float2(br_, br_), bi = make_float2(bi_, bi_), nbi = make_float2(-bi_, -bi_);
    const float2 re = make_float2(x.x, x.y), im = make_float2(x.z, x.w);
    o[0] = __ffma2_rn(br, re, o[0]);
    o[0] = __ffma2_rn(nbi, im, o[0]);
    o[1] = __ffma2_rn(br, im, o[1]);
    o[1] = __ffma2_rn(bi, re, o[1]);
}

// Load of a block value: read-only global path, or a plain load (values
// staged in shared memory).
template <bool kGlobal>
__device__ __forceinline__ float4 qb_ld(const float4 *v)
{
    if constexpr (kGlobal) return __ldg(v);
    else return *v;
}

// o[a] = {re pair, im pair} of output row a; v = the block's values, two
// complex values per float4 in the storage order of the type (in global
// memory, or with kGlobal = false anywhere a plain load reaches).
template <bool kGlobal = true>
__device__ __forceinline__ void quartet_block(float2 o[4][2], int type, const float4 *__restrict__ v,
                                              const float4 x[4])
{
    switch (type) {
    case 0:
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            const float4 p = qb_ld<kGlobal>(v + 2 * a), q = qb_ld<kGlobal>(v + 2 * a + 1);
            mac_pp(o[a], p.x, p.y, x[0]);
            mac_pp(o[a], p.z, p.w, x[1]);
            mac_pp(o[a], q.x, q.y, x[2]);
            mac_pp(o[a], q.z, q.w, x[3]);
        }
        break;
    case 1:
#pragma unroll
        for (int a2 = 0; a2 < 2; ++a2)
#pragma unroll
            for (int a1 = 0; a1 < 2; ++a1) {
                const float4 p = qb_ld<kGlobal>(v + 2 * a2 + a1);
                mac_pp(o[2 * a1 + a2], p.x, p.y, x[a2]);
                mac_pp(o[2 * a1 + a2], p.z, p.w, x[2 + a2]);
            }
        break;
    case 2:
#pragma unroll
        for (int a1 = 0; a1 < 2; ++a1)
#pragma unroll
            for (int a2 = 0; a2 < 2; ++a2) {
                const float4 p = qb_ld<kGlobal>(v + 2 * a1 + a2);
                mac_pp(o[2 * a1 + a2], p.x, p.y, x[2 * a1]);
                mac_pp(o[2 * a1 + a2], p.z, p.w, x[2 * a1 + 1]);
            }
        break;
    case 3: {
        const float4 p = qb_ld<kGlobal>(v), q = qb_ld<kGlobal>(v + 1);
        mac_pp(o[0], p.x, p.y, x[0]);
        mac_pp(o[1], p.z, p.w, x[1]);
        mac_pp(o[2], q.x, q.y, x[2]);
        mac_pp(o[3], q.z, q.w, x[3]);
        break;
    }
    case 4: {
        const float4 p = qb_ld<kGlobal>(v), q = qb_ld<kGlobal>(v + 1);  // A00 A01 | A10 A11
#pragma unroll
        for (int a2 = 0; a2 < 2; ++a2) {
            mac_pp(o[a2], p.x, p.y, x[a2]);
            mac_pp(o[a2], p.z, p.w, x[2 + a2]);
            mac_pp(o[2 + a2], q.x, q.y, x[a2]);
            mac_pp(o[2 + a2], q.z, q.w, x[2 + a2]);
        }
        break;
    }
    default: {
        const float4 p = qb_ld<kGlobal>(v), q = qb_ld<kGlobal>(v + 1);
#pragma unroll
        for (int a1 = 0; a1 < 2; ++a1) {
            mac_pp(o[2 * a1], p.x, p.y, x[2 * a1]);
            mac_pp(o[2 * a1], p.z, p.w, x[2 * a1 + 1]);
            mac_pp(o[2 * a1 + 1], q.x, q.y, x[2 * a1]);
            mac_pp(o[2 * a1 + 1], q.z, q.w, x[2 * a1 + 1]);
        }
        break;
    }
    }
}

// U = H v_j over quartet tiles (QT quartets x 64 trajectories per CTA) with
// the compact block form; the gathers of block k+1 are issued before the
// arithmetic of block k.  Partial alpha_j = Re <v_j, U> in FP64.
// kPrefetch: issue block k+1's gathers before block k's arithmetic (more
// loads in flight, more registers); kMinBlocks: CTAs per SM the register
// allocation must allow.  The autotuner picks the variant per shape.
template <bool kPrefetch, int kMinBlocks>
__global__ void __launch_bounds__(kThreads, kMinBlocks)
k_lanczos_apply_compact(QuartetC H, const float2 *__restrict__ wj, const double *__restrict__ sj,
                        float2 *__restrict__ U, double *__restrict__ part, int Q, int s1, int s2, int ldm, int QT)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int t = blockIdx.y * 64 + 2 * lane;
    const int q0 = blockIdx.x * QT;
    const float sc0 = static_cast<float>(sj[t]), sc1 = static_cast<float>(sj[t + 1]);
    const int off[4] = {0, s2, s1, s1 + s2};
    double a0 = 0.0, a1 = 0.0;
    for (int q = q0 + warp; q < min(q0 + QT, Q); q += kWarps) {
        float2 o[4][2];
#pragma unroll
        for (int a = 0; a < 4; ++a) o[a][0] = o[a][1] = make_float2(0.f, 0.f);
        const int kb = __ldg(H.rowptr + q), ke = __ldg(H.rowptr + q + 1);
        int2 cur = __ldg(H.blk + kb);
        float4 x[4];
#pragma unroll
        for (int b = 0; b < 4; ++b)
            x[b] = *reinterpret_cast<const float4 *>(wj + static_cast<size_t>((cur.x >> 3) + off[b]) * ldm + t);
        for (int k = kb; k < ke; ++k) {
            if (kPrefetch) {
                int2 nxt = cur;
                float4 xn[4];
                if (k + 1 < ke) {
                    nxt = __ldg(H.blk + k + 1);
#pragma unroll
                    for (int b = 0; b < 4; ++b)
                        xn[b] = *reinterpret_cast<const float4 *>(wj + static_cast<size_t>((nxt.x >> 3) + off[b]) * ldm + t);
                }
                quartet_block(o, cur.x & 7, H.val + cur.y, x);
                cur = nxt;
#pragma unroll
                for (int b = 0; b < 4; ++b) x[b] = xn[b];
            } else {
                quartet_block(o, cur.x & 7, H.val + cur.y, x);
                if (k + 1 < ke) {
                    cur = __ldg(H.blk + k + 1);
#pragma unroll
                    for (int b = 0; b < 4; ++b)
                        x[b] = *reinterpret_cast<const float4 *>(wj + static_cast<size_t>((cur.x >> 3) + off[b]) * ldm + t);
                }
            }
        }
        const int base = __ldg(H.base + q);
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            const size_t e = static_cast<size_t>(base + off[a]) * ldm + t;
            const float2 ure = make_float2(o[a][0].x * sc0, o[a][0].y * sc1);
            const float2 uim = make_float2(o[a][1].x * sc0, o[a][1].y * sc1);
            *reinterpret_cast<float4 *>(U + e) = make_float4(ure.x, ure.y, uim.x, uim.y);
            const float4 v = *reinterpret_cast<const float4 *>(wj + e);  // {re t, re t+1, im t, im t+1}
            a0 += (static_cast<double>(v.x) * ure.x + static_cast<double>(v.z) * uim.x) * sc0;
            a1 += (static_cast<double>(v.y) * ure.y + static_cast<double>(v.w) * uim.y) * sc1;
        }
    }
    __shared__ double sm[kWarps][64];
    sm[warp][2 * lane] = a0;
    sm[warp][2 * lane + 1] = a1;
    __syncthreads();
    if (threadIdx.x < 64) {
        double s = 0.0;
        for (int w = 0; w < kWarps; ++w) s += sm[w][threadIdx.x];
        part[static_cast<size_t>(blockIdx.x) * ldm + blockIdx.y * 64 + threadIdx.x] = s;
    }
}

// quartet_block for NP trajectory pairs per thread: the block's values are
// loaded and broadcast once and applied to every pair.
template <int NP>
__device__ __forceinline__ void quartet_block_np(float2 (&o)[NP][4][2], int type, const float4 *__restrict__ v,
                                                 const float4 (&x)[NP][4])
{
    switch (type) {
    case 0:
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            const float4 p = __ldg(v + 2 * a), q = __ldg(v + 2 * a + 1);
#pragma unroll
            for (int k = 0; k < NP; ++k) {
                mac_pp(o[k][a], p.x, p.y, x[k][0]);
                mac_pp(o[k][a], p.z, p.w, x[k][1]);
                mac_pp(o[k][a], q.x, q.y, x[k][2]);
                mac_pp(o[k][a], q.z, q.w, x[k][3]);
            }
        }
        break;
    case 1:
#pragma unroll
        for (int a2 = 0; a2 < 2; ++a2)
#pragma unroll
            for (int a1 = 0; a1 < 2; ++a1) {
                const float4 p = __ldg(v + 2 * a2 + a1);
#pragma unroll
                for (int k = 0; k < NP; ++k) {
                    mac_pp(o[k][2 * a1 + a2], p.x, p.y, x[k][a2]);
                    mac_pp(o[k][2 * a1 + a2], p.z, p.w, x[k][2 + a2]);
                }
            }
        break;
    case 2:
#pragma unroll
        for (int a1 = 0; a1 < 2; ++a1)
#pragma unroll
            for (int a2 = 0; a2 < 2; ++a2) {
                const float4 p = __ldg(v + 2 * a1 + a2);
#pragma unroll
                for (int k = 0; k < NP; ++k) {
                    mac_pp(o[k][2 * a1 + a2], p.x, p.y, x[k][2 * a1]);
                    mac_pp(o[k][2 * a1 + a2], p.z, p.w, x[k][2 * a1 + 1]);
                }
            }
        break;
    case 3: {
        const float4 p = __ldg(v), q = __ldg(v + 1);
#pragma unroll
        for (int k = 0; k < NP; ++k) {
            mac_pp(o[k][0], p.x, p.y, x[k][0]);
            mac_pp(o[k][1], p.z, p.w, x[k][1]);
            mac_pp(o[k][2], q.x, q.y, x[k][2]);
            mac_pp(o[k][3], q.z, q.w, x[k][3]);
        }
        break;
    }
    case 4: {
        const float4 p = __ldg(v), q = __ldg(v + 1);  // A00 A01 | A10 A11
#pragma unroll
        for (int k = 0; k < NP; ++k)
#pragma unroll
            for (int a2 = 0; a2 < 2; ++a2) {
                mac_pp(o[k][a2], p.x, p.y, x[k][a2]);
                mac_pp(o[k][a2], p.z, p.w, x[k][2 + a2]);
                mac_pp(o[k][2 + a2], q.x, q.y, x[k][a2]);
                mac_pp(o[k][2 + a2], q.z, q.w, x[k][2 + a2]);
            }
        break;
    }
    default: {
        const float4 p = __ldg(v), q = __ldg(v + 1);
#pragma unroll
        for (int k = 0; k < NP; ++k)
#pragma unroll
            for (int a1 = 0; a1 < 2; ++a1) {
                mac_pp(o[k][2 * a1], p.x, p.y, x[k][2 * a1]);
                mac_pp(o[k][2 * a1], p.z, p.w, x[k][2 * a1 + 1]);
                mac_pp(o[k][2 * a1 + 1], q.x, q.y, x[k][2 * a1]);
                mac_pp(o[k][2 * a1 + 1], q.z, q.w, x[k][2 * a1 + 1]);
            }
        break;
    }
    }
}

// Variant of k_lanczos_apply_compact with NP trajectory pairs per thread:
// lane l holds pairs (t0 + 2 l + 64 k, +1), k < NP, so a CTA covers 64 NP
// trajectories (ldm must be a multiple of 64 NP) and the block descriptors,
// values and addresses serve NP pairs.  Same arithmetic per trajectory.
template <int NP, int kMinBlocks>
__global__ void __launch_bounds__(kThreads, kMinBlocks)
k_lanczos_apply_np(QuartetC H, const float2 *__restrict__ wj, const double *__restrict__ sj, float2 *__restrict__ U,
                   double *__restrict__ part, int Q, int s1, int s2, int ldm, int QT)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int tb = blockIdx.y * 64 * NP + 2 * lane;
    const int q0 = blockIdx.x * QT;
    float sc[NP][2];
#pragma unroll
    for (int k = 0; k < NP; ++k) {
        sc[k][0] = static_cast<float>(sj[tb + 64 * k]);
        sc[k][1] = static_cast<float>(sj[tb + 64 * k + 1]);
    }
    const int off[4] = {0, s2, s1, s1 + s2};
    double acc[NP][2];
#pragma unroll
    for (int k = 0; k < NP; ++k) acc[k][0] = acc[k][1] = 0.0;
    for (int q = q0 + warp; q < min(q0 + QT, Q); q += kWarps) {
        float2 o[NP][4][2];
#pragma unroll
        for (int k = 0; k < NP; ++k)
#pragma unroll
            for (int a = 0; a < 4; ++a) o[k][a][0] = o[k][a][1] = make_float2(0.f, 0.f);
        const int kb = __ldg(H.rowptr + q), ke = __ldg(H.rowptr + q + 1);
        // The host stores each quartet's own (diagonal) block last, so the
        // gathered rows of the final block are v_j at this quartet's rows and
        // serve the alpha partial below without a second read.
        float4 x[NP][4];
        int last = -1;
        for (int kk = kb; kk < ke; ++kk) {
            const int2 cur = __ldg(H.blk + kk);
            last = cur.x >> 3;
#pragma unroll
            for (int b = 0; b < 4; ++b) {
                const float2 *row = wj + static_cast<size_t>(last + off[b]) * ldm + tb;
#pragma unroll
                for (int k = 0; k < NP; ++k) x[k][b] = *reinterpret_cast<const float4 *>(row + 64 * k);
            }
            quartet_block_np<NP>(o, cur.x & 7, H.val + cur.y, x);
        }
        const int base = __ldg(H.base + q);
        const bool own = last == base;
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            const size_t e = static_cast<size_t>(base + off[a]) * ldm + tb;
#pragma unroll
            for (int k = 0; k < NP; ++k) {
                const float2 ure = make_float2(o[k][a][0].x * sc[k][0], o[k][a][0].y * sc[k][1]);
                const float2 uim = make_float2(o[k][a][1].x * sc[k][0], o[k][a][1].y * sc[k][1]);
                *reinterpret_cast<float4 *>(U + e + 64 * k) = make_float4(ure.x, ure.y, uim.x, uim.y);
                const float4 v = own ? x[k][a] : *reinterpret_cast<const float4 *>(wj + e + 64 * k);
                acc[k][0] += (static_cast<double>(v.x) * ure.x + static_cast<double>(v.z) * uim.x) * sc[k][0];
                acc[k][1] += (static_cast<double>(v.y) * ure.y + static_cast<double>(v.w) * uim.y) * sc[k][1];
            }
        }
    }
    __shared__ double sm[kWarps][64 * NP];
#pragma unroll
    for (int k = 0; k < NP; ++k) {
        sm[warp][64 * k + 2 * lane] = acc[k][0];
        sm[warp][64 * k + 2 * lane + 1] = acc[k][1];
    }
    __syncthreads();
    for (int i = threadIdx.x; i < 64 * NP; i += kThreads) {
        double s = 0.0;
        for (int w = 0; w < kWarps; ++w) s += sm[w][i];
        part[static_cast<size_t>(blockIdx.x) * ldm + blockIdx.y * 64 * NP + i] = s;
    }
}

// Variant of k_lanczos_apply_compact that first stages the CTA's own input
// quartets (its QT output quartets x 64 trajectories, 4 rows each, 16 bytes
// a lane) in shared memory with cp.async: the diagonal block and every
// nucleus flip that stays inside the tile (the low quartet-index bits) then
// read shared memory instead of gathering from L2; the rest gathers as
// before.  Needs the tile's quartet bases to be contiguous (QT divides s2),
// which the host checks; dynamic shared memory QT x 4 x 512 bytes.
template <int kMinBlocks>
__global__ void __launch_bounds__(kThreads, kMinBlocks)
k_lanczos_apply_cube(QuartetC H, const float2 *__restrict__ wj, const double *__restrict__ sj, float2 *__restrict__ U,
                     double *__restrict__ part, int Q, int s1, int s2, int ldm, int QT)
{
    extern __shared__ float4 cube[];  // [QT * 4 rows][32 lanes]
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int t = blockIdx.y * 64 + 2 * lane;
    const int q0 = blockIdx.x * QT;
    const int nq = min(QT, Q - q0);
    const int base0 = __ldg(H.base + q0);
    const int off[4] = {0, s2, s1, s1 + s2};
    // stage: row slot i = 4 j + a holds quartet q0 + j, offset a
    for (int i = warp; i < 4 * nq; i += kWarps) {
        const int j = i >> 2, a = i & 3;
        const float4 *src = reinterpret_cast<const float4 *>(wj + static_cast<size_t>(base0 + j + off[a]) * ldm + t);
        const uint32_t dst = static_cast<uint32_t>(__cvta_generic_to_shared(cube + i * 32 + lane));
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    __syncthreads();
    const float sc0 = static_cast<float>(sj[t]), sc1 = static_cast<float>(sj[t + 1]);
    double a0 = 0.0, a1 = 0.0;
    for (int q = q0 + warp; q < q0 + nq; q += kWarps) {
        float2 o[4][2];
#pragma unroll
        for (int a = 0; a < 4; ++a) o[a][0] = o[a][1] = make_float2(0.f, 0.f);
        const int kb = __ldg(H.rowptr + q), ke = __ldg(H.rowptr + q + 1);
        for (int k = kb; k < ke; ++k) {
            const int2 cur = __ldg(H.blk + k);
            const int cb = cur.x >> 3;
            const unsigned rel = static_cast<unsigned>(cb - base0);
            float4 x[4];
            if (rel < static_cast<unsigned>(nq)) {
#pragma unroll
                for (int b = 0; b < 4; ++b) x[b] = cube[(4 * rel + b) * 32 + lane];
            } else {
#pragma unroll
                for (int b = 0; b < 4; ++b)
                    x[b] = *reinterpret_cast<const float4 *>(wj + static_cast<size_t>(cb + off[b]) * ldm + t);
            }
            quartet_block(o, cur.x & 7, H.val + cur.y, x);
        }
        const int jq = q - q0;
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            const size_t e = static_cast<size_t>(base0 + jq + off[a]) * ldm + t;
            const float2 ure = make_float2(o[a][0].x * sc0, o[a][0].y * sc1);
            const float2 uim = make_float2(o[a][1].x * sc0, o[a][1].y * sc1);
            *reinterpret_cast<float4 *>(U + e) = make_float4(ure.x, ure.y, uim.x, uim.y);
            const float4 v = cube[(4 * jq + a) * 32 + lane];  // {re t, re t+1, im t, im t+1}
            a0 += (static_cast<double>(v.x) * ure.x + static_cast<double>(v.z) * uim.x) * sc0;
            a1 += (static_cast<double>(v.y) * ure.y + static_cast<double>(v.w) * uim.y) * sc1;
        }
    }
    __shared__ double sm[kWarps][64];
    sm[warp][2 * lane] = a0;
    sm[warp][2 * lane + 1] = a1;
    __syncthreads();
    if (threadIdx.x < 64) {
        double s = 0.0;
        for (int w = 0; w < kWarps; ++w) s += sm[w][threadIdx.x];
        part[static_cast<size_t>(blockIdx.x) * ldm + blockIdx.y * 64 + threadIdx.x] = s;
    }
}

// w_{j+1} = U - alpha_j v_j - beta_j v_{j-1}; partial |w_{j+1}|^2 (FP64).
__global__ void __launch_bounds__(kThreads)
k_lanczos_update(const float2 *__restrict__ U, const float2 *__restrict__ wj, const float2 *__restrict__ wjm1,
                 const double *__restrict__ sj, const double *__restrict__ sjm1, const double *__restrict__ alpha,
                 float2 *__restrict__ wn, double *__restrict__ part, int D, int ldm, int R)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int t = blockIdx.y * 64 + 2 * lane;
    const int r0 = blockIdx.x * R;
    // coefficients: alpha*s_j and beta_j*s_{j-1} where beta_j = 1/s_j
    const float ca0 = static_cast<float>(alpha[t] * sj[t]), ca1 = static_cast<float>(alpha[t + 1] * sj[t + 1]);
    float cb0 = 0.f, cb1 = 0.f;
    if (wjm1) {
        cb0 = sj[t] > 0.0 ? static_cast<float>(sjm1[t] / sj[t]) : 0.f;
        cb1 = sj[t + 1] > 0.0 ? static_cast<float>(sjm1[t + 1] / sj[t + 1]) : 0.f;
    }
    double n0 = 0.0, n1 = 0.0;
    for (int r = r0 + warp; r < min(r0 + R, D); r += kWarps) {
        const size_t e = static_cast<size_t>(r) * ldm + t;
        const float4 u = *reinterpret_cast<const float4 *>(U + e);
        const float4 v = *reinterpret_cast<const float4 *>(wj + e);
        // pair-planar {re t, re t+1, im t, im t+1}
        float4 o;
        o.x = fmaf(-ca0, v.x, u.x); o.y = fmaf(-ca1, v.y, u.y);
        o.z = fmaf(-ca0, v.z, u.z); o.w = fmaf(-ca1, v.w, u.w);
        if (wjm1) {
            const float4 p = *reinterpret_cast<const float4 *>(wjm1 + e);
            o.x = fmaf(-cb0, p.x, o.x); o.y = fmaf(-cb1, p.y, o.y);
            o.z = fmaf(-cb0, p.z, o.z); o.w = fmaf(-cb1, p.w, o.w);
        }
        *reinterpret_cast<float4 *>(wn + e) = o;
        n0 += static_cast<double>(o.x) * o.x + static_cast<double>(o.z) * o.z;
        n1 += static_cast<double>(o.y) * o.y + static_cast<double>(o.w) * o.w;
    }
    __shared__ double sm[kWarps][64];
    sm[warp][2 * lane] = n0;
    sm[warp][2 * lane + 1] = n1;
    __syncthreads();
    if (threadIdx.x < 64) {
        double s = 0.0;
        for (int w = 0; w < kWarps; ++w) s += sm[w][threadIdx.x];
        part[static_cast<size_t>(blockIdx.x) * ldm + blockIdx.y * 64 + threadIdx.x] = s;
    }
}

// out[t] = sum over tiles of part[tile][t] (fixed order), optional sqrt and
// Lanczos bookkeeping: mode 0 -> alpha_j (stored to T diag), mode 1 -> beta_{j+1}
// (stored to T offdiag, scale = 1/beta, breakdown marks the dimension).
// Launch with blockDim (32, kRedRows) and ldm/32 blocks: thread (x, y) sums
// tiles y, y + kRedRows, ... of trajectory t, then the kRedRows column sums
// are added in order.  A group of 512 trajectories gives only 16 CTAs, so each
// thread's chain of dependent L2 loads sets the time: 32 rows keep it at
// 8 loads for the 256 tile partials of the SpMM.
constexpr int kRedRows = 32;
__global__ void __launch_bounds__(32 * kRedRows)
k_lanczos_reduce(const double *__restrict__ part, int ntiles, int ldm, int mode, int j, int m, double *__restrict__ out,
                 double *__restrict__ tdiag, double *__restrict__ toff, int *__restrict__ mdim)
{
    __shared__ double red[kRedRows][33];
    const int t = blockIdx.x * 32 + threadIdx.x;
    double ps = 0.0;
    for (int tile = threadIdx.y; tile < ntiles; tile += kRedRows) ps += part[static_cast<size_t>(tile) * ldm + t];
    red[threadIdx.y][threadIdx.x] = ps;
    __syncthreads();
    if (threadIdx.y != 0) return;
    double s = 0.0;
#pragma unroll
    for (int y = 0; y < kRedRows; ++y) s += red[y][threadIdx.x];
    const bool active = mdim[t] == 0;
    if (mode == 0) {
        out[t] = s;
        if (active) {
            tdiag[static_cast<size_t>(t) * m + j] = s;
            if (j == m - 1) mdim[t] = m;
        }
        return;
    }
    const double beta = sqrt(s);
    if (!active) { out[t] = 0.0; return; }
    if (j == m - 1) { mdim[t] = m; out[t] = 0.0; return; }
    toff[static_cast<size_t>(t) * m + j] = beta;
    if (beta < 1e-14) { mdim[t] = j + 1; out[t] = 0.0; return; }
    out[t] = 1.0 / beta;
}

// ===================================================================== shared
// Per-trajectory small exponential: y = beta0 * exp(dt*A_m) e1 where A_m is
// the Arnoldi Hessenberg matrix of G (hess != null) or -iT - kappa I from the
// Lanczos tridiagonal (tdiag/toff).  One warp per trajectory.  coef[t][j]
// receives y_j times the storage scale of basis vector j (vscale, may be null).
__global__ void k_krylov_expm(const double2 *__restrict__ hess, const double *__restrict__ tdiag,
                              const double *__restrict__ toff, double kappa, const int *__restrict__ mdim,
                              const double *__restrict__ beta0, const double *__restrict__ vscale, int m,
                              int ldm, int M, double dt, double2 *__restrict__ coef, int *__restrict__ status)
{
    extern __shared__ double2 smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int t = blockIdx.x * (blockDim.x >> 5) + warp;
    if (t >= ldm) return;
    double2 *A = smem + static_cast<size_t>(warp) * (4 * m * m + m);
    double2 *X = A + m * m, *N = X + m * m, *Dm = N + m * m, *y = Dm + m * m;
    const int n = max(1, mdim[t]);
    const double b0 = beta0[t];
    if (lane < n) {
        for (int i = 0; i < n; ++i) {
            double2 v;
            if (hess) {
                // upper Hessenberg part only; entries below the subdiagonal are never written
                v = i <= lane + 1 ? hess[static_cast<size_t>(t) * m * m + i + lane * m] : make_double2(0.0, 0.0);
            } else {
                v = make_double2(0.0, 0.0);
                if (i == lane) v = make_double2(-kappa, -tdiag[static_cast<size_t>(t) * m + i]);
                else if (i == lane + 1) v = make_double2(0.0, -toff[static_cast<size_t>(t) * m + lane]);
                else if (i + 1 == lane) v = make_double2(0.0, -toff[static_cast<size_t>(t) * m + i]);
            }
            A[i + lane * n] = cscale(v, dt);
        }
    }
    __syncwarp();
    bool ok = true;
    if (b0 > 0.0) ok = warp_expm_col0(n, A, X, N, Dm, y);
    if (lane < m) {
        double2 c = make_double2(0.0, 0.0);
        if (b0 > 0.0 && ok && lane < n) {
            c = cscale(y[lane], b0);
            if (vscale) c = cscale(c, vscale[static_cast<size_t>(lane) * ldm + t]);
        }
        coef[static_cast<size_t>(lane) * ldm + t] = c;
    }
    if (!ok && lane == 0 && t < M) atomicOr(status, 1);
}

// ---------------------------------------------------------------- Taylor propagator
// One term of the truncated Taylor series of exp(tau (G - mu I)) applied to
// the trajectory block (HSPropagator's autoexpm, SpinSpace::HighamProp,
// SpinSpace_operators.cpp:1028-1134): out = scale (G - mu I) in with
// G = -iH - K, scale = tau / (s k), and F += out.  Thread (row, trajectory);
// a warp covers 32 trajectories of one row (coalesced 16-byte accesses).
__global__ void __launch_bounds__(256)
k_taylor_term(CsrD H, CsrD K, double kappa, double2 mu, const double2 *__restrict__ in, double2 *__restrict__ out,
              double2 *__restrict__ F, double scale, int D, int ldm)
{
    const int t = blockIdx.y * 32 + threadIdx.x;
    const int r = blockIdx.x * 8 + threadIdx.y;
    if (r >= D) return;
    double2 h = make_double2(0.0, 0.0);
    for (int k = __ldg(H.rowptr + r); k < __ldg(H.rowptr + r + 1); ++k)
        h = cfma(H.val[k], in[static_cast<size_t>(__ldg(H.col + k)) * ldm + t], h);
    const size_t e = static_cast<size_t>(r) * ldm + t;
    const double2 x = in[e];
    double2 g = make_double2(h.y, -h.x);  // -i (H x)_r
    if (K.rowptr) {
        double2 kk = make_double2(0.0, 0.0);
        for (int k = __ldg(K.rowptr + r); k < __ldg(K.rowptr + r + 1); ++k)
            kk = cfma(K.val[k], in[static_cast<size_t>(__ldg(K.col + k)) * ldm + t], kk);
        g = csub(g, kk);
    } else {
        g = csub(g, cscale(x, kappa));
    }
    g = csub(g, cmul(mu, x));
    const double2 o = cscale(g, scale);
    out[e] = o;
    const double2 f = F[e];
    F[e] = make_double2(f.x + o.x, f.y + o.y);
}

// One stage of the classical RK4 step for dB/dt = G B (propagationmethod=rk4,
// HSPropagator::Step, HSPropagator.cpp:80-90): k = G y_in at (row, trajectory),
// then stage 1: acc = psi + w k, y_out = psi + c k; stages 2, 3: acc += w k,
// y_out = psi + c k; stage 4: psi = acc + w k.  No stage writes a buffer it
// gathers from (stage 1 reads psi, stage 4 writes it and reads y_in).
__global__ void __launch_bounds__(256)
k_rk4_stage(CsrD H, CsrD K, double kappa, const double2 *__restrict__ y_in, double2 *psi, double2 *__restrict__ y_out,
            double2 *__restrict__ acc, double c, double w, int stage, int D, int ldm)
{
    const int t = blockIdx.y * 32 + threadIdx.x;
    const int r = blockIdx.x * 8 + threadIdx.y;
    if (r >= D) return;
    double2 h = make_double2(0.0, 0.0);
    for (int k = __ldg(H.rowptr + r); k < __ldg(H.rowptr + r + 1); ++k)
        h = cfma(H.val[k], y_in[static_cast<size_t>(__ldg(H.col + k)) * ldm + t], h);
    const size_t e = static_cast<size_t>(r) * ldm + t;
    double2 g = make_double2(h.y, -h.x);  // -i (H y)_r
    if (K.rowptr) {
        double2 kk = make_double2(0.0, 0.0);
        for (int k = __ldg(K.rowptr + r); k < __ldg(K.rowptr + r + 1); ++k)
            kk = cfma(K.val[k], y_in[static_cast<size_t>(__ldg(K.col + k)) * ldm + t], kk);
        g = csub(g, kk);
    } else {
        g = csub(g, cscale(y_in[e], kappa));
    }
    if (stage == 4) {
        const double2 a = acc[e];
        psi[e] = make_double2(a.x + w * g.x, a.y + w * g.y);
        return;
    }
    const double2 p = psi[e];
    y_out[e] = make_double2(p.x + c * g.x, p.y + c * g.y);
    const double2 a = stage == 1 ? p : acc[e];
    acc[e] = make_double2(a.x + w * g.x, a.y + w * g.y);
}

// End of a Taylor sub-step: F <- eta F (the shift e^{tau mu / s}), B <- F.
__global__ void k_taylor_rescale(double2 *__restrict__ F, double2 *__restrict__ B, double2 eta, size_t n)
{
    const size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double2 f = cmul(eta, F[i]);
    F[i] = f;
    B[i] = f;
}

// trace(H) and max_r sum_k |H_rk| (= the 1-norm of a Hermitian H) in a fixed
// order: one block; out = {tr.re, tr.im, max row sum}.
__global__ void __launch_bounds__(256) k_g_stats(CsrD H, int D, double *__restrict__ out)
{
    __shared__ double sre[256], sim[256], smx[256];
    double tr = 0.0, ti = 0.0, mx = 0.0;
    for (int r = threadIdx.x; r < D; r += blockDim.x) {
        double rs = 0.0;
        for (int k = H.rowptr[r]; k < H.rowptr[r + 1]; ++k) {
            const double2 v = H.val[k];
            rs += sqrt(v.x * v.x + v.y * v.y);
            if (H.col[k] == r) {
                tr += v.x;
                ti += v.y;
            }
        }
        mx = fmax(mx, rs);
    }
    sre[threadIdx.x] = tr;
    sim[threadIdx.x] = ti;
    smx[threadIdx.x] = mx;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (static_cast<int>(threadIdx.x) < w) {
            sre[threadIdx.x] += sre[threadIdx.x + w];
            sim[threadIdx.x] += sim[threadIdx.x + w];
            smx[threadIdx.x] = fmax(smx[threadIdx.x], smx[threadIdx.x + w]);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        out[0] = sre[0];
        out[1] = sim[0];
        out[2] = smx[0];
    }
}

// Krylov exponential of the Lanczos form (tridiagonal, see
// warp_tridiag_expm_e1): one warp per trajectory.  Coefficients as in
// k_krylov_expm: coef[j][t] = beta0 * vscale_j * y_j.
__global__ void __launch_bounds__(256)
k_lanczos_expm(const double *__restrict__ tdiag, const double *__restrict__ toff, double kappa,
               const int *__restrict__ mdim, const double *__restrict__ beta0, const double *__restrict__ vscale,
               int m, int ldm, int M, double dt, double2 *__restrict__ coef, int *__restrict__ status)
{
    const int lane = threadIdx.x & 31;
    const int t = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (t >= ldm) return;  // whole warps leave together
    const int n = max(1, mdim[t]);
    const double b0 = beta0[t];
    const bool live = lane < n;
    const double d = live ? tdiag[static_cast<size_t>(t) * m + lane] : 0.0;
    const double lo = (live && lane > 0) ? toff[static_cast<size_t>(t) * m + lane - 1] : 0.0;
    const double hi = (lane + 1 < n) ? toff[static_cast<size_t>(t) * m + lane] : 0.0;
    double2 y;
    const bool ok = warp_tridiag_expm_e1(n, d, lo, hi, kappa, dt, y) && b0 > 0.0;
    if (lane < m) {
        double2 c = make_double2(0.0, 0.0);
        if (ok && live) {
            c = cscale(y, b0);
            if (vscale) c = cscale(c, vscale[static_cast<size_t>(lane) * ldm + t]);
        }
        coef[static_cast<size_t>(lane) * ldm + t] = c;
    }
    if (!ok && b0 > 0.0 && lane == 0 && t < M) atomicOr(status, 1);
}

// Flip bit for trajectory t at (global step, half): replay bits (layout
// ((step*2+half)*M + t)) or Philox.
struct Noise {
    int mode;                // 0 none, 1 replay bits, 2 philox
    const uint8_t *bits;     // replay
    long long bits_steps;    // number of steps covered by bits
    int M;                   // trajectories in the bit layout
    uint64_t seed;           // philox
    uint32_t traj_offset;    // added to the launch's trajectory index (a trajectory group's first)
    double p_full;           // flip probability for a half step of the current step
};

__device__ __forceinline__ int noise_bit(const Noise &nz, int t, long long step, int half, double p)
{
    if (step < 0) return 0;
    if (nz.mode == 1) {
        const int ta = t + static_cast<int>(nz.traj_offset);  // trajectory in the bit layout
        if (ta >= nz.M || step < 0 || step >= nz.bits_steps) return 0;
        const long long bit = (step * 2 + half) * nz.M + ta;
        return (nz.bits[bit >> 3] >> (bit & 7)) & 1;
    }
    if (nz.mode == 2)
        return philox_flip(nz.seed, nz.traj_offset + static_cast<uint32_t>(t), static_cast<uint32_t>(step),
                           static_cast<uint32_t>(half), p) ? 1 : 0;
    return 0;
}

struct PairObs {
    int nobs;
    double2 op[8][16];  // 4x4 row-major in the pair basis
};

// Quartet epilogue shared by both precisions: apply the singlet-triplet flip
// U = PS - PT (x4 -> -(swap middle), negate ends) when flip is set, and add
// <x|O_o|x> to obs[o] and |x|^2 to nrm.
__device__ __forceinline__ void quartet_epilogue(double2 x[4], int flip, const PairObs &po, double *obs, double &nrm)
{
    if (flip) {
        const double2 a = x[1];
        x[0] = make_double2(-x[0].x, -x[0].y);
        x[1] = make_double2(-x[2].x, -x[2].y);
        x[2] = make_double2(-a.x, -a.y);
        x[3] = make_double2(-x[3].x, -x[3].y);
    }
    nrm += cabs2(x[0]) + cabs2(x[1]) + cabs2(x[2]) + cabs2(x[3]);
    for (int o = 0; o < po.nobs; ++o) {
        double s = 0.0;
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            double2 ox = make_double2(0.0, 0.0);
#pragma unroll
            for (int b = 0; b < 4; ++b) ox = cfma(po.op[o][a * 4 + b], x[b], ox);
            s += x[a].x * ox.x + x[a].y * ox.y;  // Re(conj(x_a) (O x)_a)
        }
        obs[o] += s;
    }
}

// psi = sum_{j<n_t} coef[t][j] V_j at the four rows of each quartet, then the
// combined flip of this half step pair, observables and norm partials.
// kBasis=false evaluates psi itself (start of a run: flip of the first half
// step only, no Krylov combination).
template <typename T, bool kBasis>
__global__ void __launch_bounds__(256)
k_combine(T *__restrict__ psi, const T *__restrict__ V, size_t vstride, const double2 *__restrict__ coef,
          const int *__restrict__ mdim, int m, int s1, int s2, int Q, int ldm, int QR, Noise nz, long long stepA,
          int halfA, double pA, long long stepB, int halfB, double pB, PairObs po, double *__restrict__ part_obs,
          double *__restrict__ part_nrm)
{
    // blockDim = (32, 8): x over trajectories, y over quartets of the tile
    const int t = blockIdx.y * 32 + threadIdx.x;
    const int q0 = blockIdx.x * QR;
    double obs[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    double nrm = 0.0;
    const int n = kBasis ? max(1, mdim[t]) : 0;
    int flip = noise_bit(nz, t, stepA, halfA, pA);
    if (stepB >= 0) flip ^= noise_bit(nz, t, stepB, halfB, pB);
    for (int q = q0 + threadIdx.y; q < min(q0 + QR, Q); q += blockDim.y) {
        const int base = quartet_base(q, s1, s2);
        size_t e[4];
        e[0] = static_cast<size_t>(base) * ldm + t;
        e[1] = static_cast<size_t>(base + s2) * ldm + t;
        e[2] = static_cast<size_t>(base + s1) * ldm + t;
        e[3] = static_cast<size_t>(base + s1 + s2) * ldm + t;
        double2 x[4];
        if (kBasis) {
#pragma unroll
            for (int a = 0; a < 4; ++a) x[a] = make_double2(0.0, 0.0);
            for (int jj = 0; jj < n; ++jj) {
                const double2 c = coef[static_cast<size_t>(jj) * ldm + t];
#pragma unroll
                for (int a = 0; a < 4; ++a) {
                    const T v = V[jj * vstride + e[a]];
                    x[a] = cfma(c, make_double2(v.x, v.y), x[a]);
                }
            }
        } else {
#pragma unroll
            for (int a = 0; a < 4; ++a) { const T v = psi[e[a]]; x[a] = make_double2(v.x, v.y); }
        }
        quartet_epilogue(x, flip, po, obs, nrm);
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            T o;
            o.x = x[a].x;
            o.y = x[a].y;
            psi[e[a]] = o;
        }
    }
    __shared__ double sm[9][8][33];
    for (int o = 0; o < po.nobs; ++o) sm[o][threadIdx.y][threadIdx.x] = obs[o];
    sm[8][threadIdx.y][threadIdx.x] = nrm;
    __syncthreads();
    if (threadIdx.y == 0) {
        for (int o = 0; o < po.nobs; ++o) {
            double s = 0.0;
            for (int w = 0; w < blockDim.y; ++w) s += sm[o][w][threadIdx.x];
            part_obs[(static_cast<size_t>(blockIdx.x) * po.nobs + o) * ldm + t] = s;
        }
        double s = 0.0;
        for (int w = 0; w < blockDim.y; ++w) s += sm[8][w][threadIdx.x];
        part_nrm[static_cast<size_t>(blockIdx.x) * ldm + t] = s;
    }
}

// Pair-planar complex64 form of k_combine: each thread owns a trajectory pair
// (t, t+1) of a quartet (16-byte loads).  blockDim = (32, 8): x over 32
// pairs (64 trajectories), y over quartets of the tile.
template <bool kBasis>
__global__ void __launch_bounds__(256)
k_combine_pp(float2 *__restrict__ psi, const float2 *__restrict__ V, size_t vstride, const double2 *__restrict__ coef,
             const int *__restrict__ mdim, int s1, int s2, int Q, int ldm, int QR, Noise nz, long long stepA, int halfA,
             double pA, long long stepB, int halfB, double pB, PairObs po, double *__restrict__ part_obs,
             double *__restrict__ part_nrm)
{
    const int t = blockIdx.y * 64 + 2 * threadIdx.x;
    const int q0 = blockIdx.x * QR;
    double obs[2][8] = {{0, 0, 0, 0, 0, 0, 0, 0}, {0, 0, 0, 0, 0, 0, 0, 0}};
    double nrm[2] = {0.0, 0.0};
    int n = 0;
    if (kBasis) n = max(max(1, mdim[t]), max(1, mdim[t + 1]));
    int flip[2];
    for (int k = 0; k < 2; ++k) {
        flip[k] = noise_bit(nz, t + k, stepA, halfA, pA);
        if (stepB >= 0) flip[k] ^= noise_bit(nz, t + k, stepB, halfB, pB);
    }
    for (int q = q0 + threadIdx.y; q < min(q0 + QR, Q); q += blockDim.y) {
        const int base = quartet_base(q, s1, s2);
        size_t e[4];
        e[0] = static_cast<size_t>(base) * ldm + t;
        e[1] = static_cast<size_t>(base + s2) * ldm + t;
        e[2] = static_cast<size_t>(base + s1) * ldm + t;
        e[3] = static_cast<size_t>(base + s1 + s2) * ldm + t;
        double2 x[2][4];
        if (kBasis) {
#pragma unroll
            for (int a = 0; a < 4; ++a) x[0][a] = x[1][a] = make_double2(0.0, 0.0);
#pragma unroll 4
            for (int jj = 0; jj < n; ++jj) {
                // coefficients are zero beyond a trajectory's own Krylov dimension
                const double2 c0 = coef[static_cast<size_t>(jj) * ldm + t];
                const double2 c1 = coef[static_cast<size_t>(jj) * ldm + t + 1];
#pragma unroll
                for (int a = 0; a < 4; ++a) {
                    const float4 v = *reinterpret_cast<const float4 *>(V + jj * vstride + e[a]);
                    x[0][a] = cfma(c0, make_double2(v.x, v.z), x[0][a]);
                    x[1][a] = cfma(c1, make_double2(v.y, v.w), x[1][a]);
                }
            }
        } else {
#pragma unroll
            for (int a = 0; a < 4; ++a) {
                const float4 v = *reinterpret_cast<const float4 *>(psi + e[a]);
                x[0][a] = make_double2(v.x, v.z);
                x[1][a] = make_double2(v.y, v.w);
            }
        }
        quartet_epilogue(x[0], flip[0], po, obs[0], nrm[0]);
        quartet_epilogue(x[1], flip[1], po, obs[1], nrm[1]);
#pragma unroll
        for (int a = 0; a < 4; ++a)
            *reinterpret_cast<float4 *>(psi + e[a]) =
                make_float4(static_cast<float>(x[0][a].x), static_cast<float>(x[1][a].x),
                            static_cast<float>(x[0][a].y), static_cast<float>(x[1][a].y));
    }
    __shared__ double sm[9][8][65];
    for (int o = 0; o < po.nobs; ++o) {
        sm[o][threadIdx.y][2 * threadIdx.x] = obs[0][o];
        sm[o][threadIdx.y][2 * threadIdx.x + 1] = obs[1][o];
    }
    sm[8][threadIdx.y][2 * threadIdx.x] = nrm[0];
    sm[8][threadIdx.y][2 * threadIdx.x + 1] = nrm[1];
    __syncthreads();
    const int tid = threadIdx.y * 32 + threadIdx.x;
    if (tid < 64) {
        const int tt = blockIdx.y * 64 + tid;
        for (int o = 0; o < po.nobs; ++o) {
            double s = 0.0;
            for (int w = 0; w < blockDim.y; ++w) s += sm[o][w][tid];
            part_obs[(static_cast<size_t>(blockIdx.x) * po.nobs + o) * ldm + tt] = s;
        }
        double s = 0.0;
        for (int w = 0; w < blockDim.y; ++w) s += sm[8][w][tid];
        part_nrm[static_cast<size_t>(blockIdx.x) * ldm + tt] = s;
    }
}

// complex128 interleaved <-> complex64 pair-planar (n = D * ldm elements)
__global__ void k_c128_to_pp(float4 *__restrict__ out, const double2 *__restrict__ in, size_t npairs)
{
    const size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= npairs) return;
    const double2 a = in[2 * i], b = in[2 * i + 1];
    out[i] = make_float4(static_cast<float>(a.x), static_cast<float>(b.x), static_cast<float>(a.y),
                         static_cast<float>(b.y));
}

__global__ void k_pp_to_c128(double2 *__restrict__ out, const float4 *__restrict__ in, size_t npairs)
{
    const size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= npairs) return;
    const float4 v = in[i];
    out[2 * i] = make_double2(v.x, v.z);
    out[2 * i + 1] = make_double2(v.y, v.w);
}

// Per-trajectory trapezoid accumulation (compensated) of the observable
// values of this time point; init=1 only records the first value.
// Also refreshes beta0 = |psi| and the inverse scale of the next step, and
// optionally writes the ensemble value (sum over trajectories < M) of this
// time point to values_out[o].  Launch with one CTA of 1024 threads.
__global__ void k_yield_update(const double *__restrict__ part_obs, const double *__restrict__ part_nrm,
                               int ntiles, int nobs, int ldm, int M, const double *__restrict__ rates, double dt,
                               int init, double *__restrict__ prev, double *__restrict__ acc,
                               double *__restrict__ comp, double *__restrict__ beta0, double *__restrict__ inv0,
                               double *__restrict__ values_out, int *__restrict__ status)
{
    __shared__ double red[8][32];
    double ens[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    bool bad = false;
    for (int t = threadIdx.x; t < ldm; t += blockDim.x) {
        for (int o = 0; o < nobs; ++o) {
            double v = 0.0;
            for (int tile = 0; tile < ntiles; ++tile) v += part_obs[(static_cast<size_t>(tile) * nobs + o) * ldm + t];
            v *= rates[o];
            const size_t k = static_cast<size_t>(o) * ldm + t;
            if (!init) {
                // Kahan-compensated acc += 0.5*dt*(prev+v)
                const double term = 0.5 * dt * (prev[k] + v) - comp[k];
                const double s = acc[k] + term;
                comp[k] = (s - acc[k]) - term;
                acc[k] = s;
            }
            prev[k] = v;
            if (t < M) ens[o] += v;
            if (!isfinite(v)) bad = true;
        }
        double nn = 0.0;
        for (int tile = 0; tile < ntiles; ++tile) nn += part_nrm[static_cast<size_t>(tile) * ldm + t];
        const double b = sqrt(nn);
        beta0[t] = b;
        inv0[t] = b > 0.0 ? 1.0 / b : 0.0;
        if (!isfinite(b)) bad = true;
    }
    if (bad) atomicOr(status, 2);
    if (!values_out) return;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int o = 0; o < nobs; ++o) {
        double v = warp_sum(ens[o]);
        if (lane == 0) red[o][warp] = v;
    }
    __syncthreads();
    if (threadIdx.x < nobs) {
        double s = 0.0;
        for (int w = 0; w < (blockDim.x >> 5); ++w) s += red[threadIdx.x][w];
        values_out[threadIdx.x] = s;
    }
}

// The per-trajectory part of k_yield_update spread over the GPU: thread t of
// grid row o sums the tile partials of observable o (o == nobs: the squared
// norm) in tile order, exactly as k_yield_update does, so the results are the
// same bits.  One 1024-thread CTA reads 5 x 64 partials per thread serially
// and took about 120 us per time step at 1024 trajectories; this form takes a
// few microseconds.  Grid (ceil(ldm / 128), nobs + 1), 128 threads.
__global__ void __launch_bounds__(128)
k_yield_traj(const double *__restrict__ part_obs, const double *__restrict__ part_nrm, int ntiles, int nobs, int ldm,
             const double *__restrict__ rates, double dt, int init, double *__restrict__ prev,
             double *__restrict__ acc, double *__restrict__ comp, double *__restrict__ beta0,
             double *__restrict__ inv0, int *__restrict__ status)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int o = blockIdx.y;
    if (t >= ldm) return;
    bool bad = false;
    if (o < nobs) {
        double v = 0.0;
#pragma unroll 8
        for (int tile = 0; tile < ntiles; ++tile) v += part_obs[(static_cast<size_t>(tile) * nobs + o) * ldm + t];
        v *= rates[o];
        const size_t k = static_cast<size_t>(o) * ldm + t;
        if (!init) {
            const double term = 0.5 * dt * (prev[k] + v) - comp[k];
            const double s = acc[k] + term;
            comp[k] = (s - acc[k]) - term;
            acc[k] = s;
        }
        prev[k] = v;
        if (!isfinite(v)) bad = true;
    } else {
        double nn = 0.0;
#pragma unroll 8
        for (int tile = 0; tile < ntiles; ++tile) nn += part_nrm[static_cast<size_t>(tile) * ldm + t];
        const double b = sqrt(nn);
        beta0[t] = b;
        inv0[t] = b > 0.0 ? 1.0 / b : 0.0;
        if (!isfinite(b)) bad = true;
    }
    if (bad) atomicOr(status, 2);
}

// Ensemble value of this time point, values_out[o] = sum over trajectories
// t < M of prev[o][t], summed in k_yield_update's order (thread-strided, then
// warps, then the warp totals).  One CTA of 1024 threads.
__global__ void __launch_bounds__(1024)
k_yield_values(const double *__restrict__ prev, int nobs, int ldm, int M, double *__restrict__ values_out)
{
    __shared__ double red[8][32];
    double ens[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int t = threadIdx.x; t < ldm; t += blockDim.x)
        for (int o = 0; o < nobs; ++o)
            if (t < M) ens[o] += prev[static_cast<size_t>(o) * ldm + t];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int o = 0; o < nobs; ++o) {
        double v = warp_sum(ens[o]);
        if (lane == 0) red[o][warp] = v;
    }
    __syncthreads();
    if (threadIdx.x < nobs) {
        double s = 0.0;
        for (int w = 0; w < (blockDim.x >> 5); ++w) s += red[threadIdx.x][w];
        values_out[threadIdx.x] = s;
    }
}

template <typename Dst, typename Src>
__global__ void k_convert(Dst *__restrict__ out, const Src *__restrict__ in, size_t n)
{
    const size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    Dst o;
    o.x = in[i].x;
    o.y = in[i].y;
    out[i] = o;
}


// Column-major D x M (one trajectory per column, as HSPreparedState factors)
// <-> trajectory-interleaved (row r, trajectory t at r*ldm + t), through 32x32
// shared-memory tiles so both sides stay coalesced.  Padding trajectories
// M <= t < ldm are written as zero.
template <typename Dst>
__global__ void k_cols_to_interleaved(Dst *__restrict__ out, const double2 *__restrict__ in, int D, int M, int ldm)
{
    __shared__ double2 tile[32][33];
    const int r0 = blockIdx.x * 32, t0 = blockIdx.y * 32;
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const int t = t0 + k, r = r0 + threadIdx.x;
        tile[k][threadIdx.x] = (t < M && r < D) ? in[static_cast<size_t>(t) * D + r] : make_double2(0.0, 0.0);
    }
    __syncthreads();
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const int r = r0 + k, t = t0 + threadIdx.x;
        if (r < D && t < ldm) {
            Dst o;
            o.x = tile[threadIdx.x][k].x;
            o.y = tile[threadIdx.x][k].y;
            out[static_cast<size_t>(r) * ldm + t] = o;
        }
    }
}

template <typename Src>
__global__ void k_interleaved_to_cols(double2 *__restrict__ out, const Src *__restrict__ in, int D, int M, int ldm)
{
    __shared__ double2 tile[32][33];
    const int r0 = blockIdx.x * 32, t0 = blockIdx.y * 32;
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const int r = r0 + k, t = t0 + threadIdx.x;
        if (r < D && t < ldm) {
            const Src v = in[static_cast<size_t>(r) * ldm + t];
            tile[k][threadIdx.x] = make_double2(v.x, v.y);
        }
    }
    __syncthreads();
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const int t = t0 + k, r = r0 + threadIdx.x;
        if (t < M && r < D) out[static_cast<size_t>(t) * D + r] = tile[threadIdx.x][k];
    }
}

}  // namespace
}  // namespace msgpu
