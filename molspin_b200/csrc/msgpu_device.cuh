// msgpu_device.cuh -- device-side building blocks shared by the msgpu kernels.
//
// Data layout in HBM (all kernels): a block of M trajectories of a D-dimensional
// Hilbert space is stored "trajectory-interleaved": element (row r, trajectory t)
// lives at r * ldm + t, with ldm = M rounded up to the trajectory tile.  A warp
// that walks one Hamiltonian row therefore reads a contiguous run of
// trajectories for every gathered column (128-bit loads per lane).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <map>
#include <mutex>
#include <utility>

#include "msgpu_philox.h"

namespace msgpu {

// Raises a kernel's dynamic shared-memory limit on the current device to at
// least `bytes` and never lowers it.  The limit is one attribute per kernel,
// shared by every context of the process; contexts driven from several host
// threads (the batching form's large systems) would otherwise race: a smaller
// value set by one thread between another thread's set and launch fails that
// launch with an invalid argument.
inline cudaError_t raise_smem_limit(const void *fn, int bytes)
{
    static std::mutex mu;
    static std::map<std::pair<int, const void *>, int> limit;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lock(mu);
    int &cur = limit[{dev, fn}];
    if (bytes <= cur) return cudaSuccess;
    e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess) cur = bytes;
    return e;
}

// ------------------------------------------------------------ complex helpers
__device__ __forceinline__ double2 cmul(double2 a, double2 b)
{
    return make_double2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ double2 cfma(double2 a, double2 b, double2 c)  // a*b + c
{
    return make_double2(fma(a.x, b.x, fma(-a.y, b.y, c.x)), fma(a.x, b.y, fma(a.y, b.x, c.y)));
}
__device__ __forceinline__ double2 cconjmul(double2 a, double2 b)  // conj(a)*b
{
    return make_double2(fma(a.x, b.x, a.y * b.y), fma(a.x, b.y, -a.y * b.x));
}
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 cscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
__device__ __forceinline__ double cabs2(double2 a) { return fma(a.x, a.x, a.y * a.y); }

__device__ __forceinline__ float2 cfmaf(float2 a, float2 b, float2 c)
{
    return make_float2(fmaf(a.x, b.x, fmaf(-a.y, b.y, c.x)), fmaf(a.x, b.y, fmaf(a.y, b.x, c.y)));
}

// ------------------------------------------------------------ warp reductions
__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ double warp_max(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// ------------------------------------------------------------ pair quartets
// The singlet-triplet structure lives on two spin-1/2 digits of the product
// basis with strides s1 > s2.  Quartet q enumerates all basis indices whose
// two electron digits are zero; its four members are base + a*s1 + b*s2 with
// pair index 2a+b: 0=|up up>, 1=|up down>, 2=|down up>, 3=|down down>.
__device__ __forceinline__ int quartet_base(int q, int s1, int s2)
{
    const int lo = q % s2;
    const int mid = (q / s2) % (s1 / (2 * s2));
    const int hi = q / (s1 / 2);
    return hi * (2 * s1) + mid * (2 * s2) + lo;
}

// Lanczos form (K = kappa I, H Hermitian): the Krylov matrix is
// dt (-kappa I - i T) with T real symmetric tridiagonal, so its exponential
// applied to e1 is e^{-kappa dt} exp(-i dt T) e1.  Lane i < n supplies T_ii
// (diag), T_i,i-1 (lo; 0 on lane 0) and T_i,i+1 (hi; 0 on lane n-1); every
// lane of the warp must call.  exp(B) e1 with B = -i dt T is taken as r equal
// sub-steps exp(B / r), r = ceil(||B||_inf / 4), each a Taylor series whose
// degree K is the smallest with theta^(K+1) / (K+1)! < 1e-17,
// theta = ||B||_inf / r (terms never exceed 4^4/4!, so the cancellation costs
// about one digit); the tridiagonal matvec is two warp shuffles.  Lane i
// returns y_i (0 for i >= n); false on a non-finite result or a norm beyond
// 4 x kTridiagMaxSubsteps.
constexpr int kTridiagMaxSubsteps = 1 << 14;

__device__ inline bool warp_tridiag_expm_e1(int n, double diag, double lo, double hi, double kappa, double dt,
                                            double2 &y)
{
    const int lane = threadIdx.x & 31;
    const bool live = lane < n;
    const double d = live ? -dt * diag : 0.0;
    const double l = (live && lane > 0) ? -dt * lo : 0.0;
    const double h = (lane + 1 < n) ? -dt * hi : 0.0;
    const double nrm = warp_max(fabs(d) + fabs(l) + fabs(h));
    y = make_double2(lane == 0 ? 1.0 : 0.0, 0.0);
    if (!(isfinite(nrm) && nrm <= 4.0 * kTridiagMaxSubsteps)) return false;
    const int r = max(1, static_cast<int>(ceil(nrm / 4.0)));
    const double theta = nrm / r, inv_r = 1.0 / r;
    int K = 1;
    for (double rem = theta * theta / 2.0; rem >= 1e-17 && K < 64; ++K) rem *= theta / (K + 2);
    const double ds = d * inv_r, ls = l * inv_r, hs = h * inv_r;
    for (int rep = 0; rep < r; ++rep) {
        double2 term = y, acc = y;
        for (int k = 1; k <= K; ++k) {
            // (B term)_i = i (l term_{i-1} + d term_i + h term_{i+1})
            const double pr = __shfl_up_sync(0xffffffffu, term.x, 1), pi = __shfl_up_sync(0xffffffffu, term.y, 1);
            const double nr = __shfl_down_sync(0xffffffffu, term.x, 1), ni = __shfl_down_sync(0xffffffffu, term.y, 1);
            const double re = ls * pr + ds * term.x + hs * nr;
            const double im = ls * pi + ds * term.y + hs * ni;
            const double inv = 1.0 / k;
            term = live ? make_double2(-im * inv, re * inv) : make_double2(0.0, 0.0);  // times i / k
            acc.x += term.x;
            acc.y += term.y;
        }
        y = acc;
    }
    const double sk = exp(-kappa * dt);
    y = make_double2(y.x * sk, y.y * sk);
    return __all_sync(0xffffffffu, isfinite(y.x) && isfinite(y.y));
}

// ------------------------------------------------------------ small expm
// Per-warp matrix exponential of an n x n complex matrix (n <= 32) held in
// shared memory, column-major, by scaling and squaring with the diagonal (6,6)
// Pade approximant (Golub & Van Loan, Matrix Computations, Alg. 11.3.1) and an
// LU solve with partial pivoting.  Lane j owns column j.  A is overwritten.
// Only column 0 of exp(A) is returned (in y[0..n)), which is all a Krylov
// step needs: exp(dt H_m) e1.  Scratch: X, N, Dm (n*n each).
__device__ inline bool warp_expm_col0(int n, double2 *A, double2 *X, double2 *N, double2 *Dm, double2 *y)
{
    const int lane = threadIdx.x & 31;
    // infinity norm: row sums, lane i owns row i
    double rs = 0.0;
    if (lane < n)
        for (int j = 0; j < n; ++j) rs += sqrt(cabs2(A[lane + j * n]));
    double norm = warp_max(lane < n ? rs : 0.0);
    if (!isfinite(norm)) return false;
    int sc = 0;
    if (norm > 0.0) sc = max(0, 1 + static_cast<int>(floor(log2(norm))));
    const double scale = ldexp(1.0, -sc);
    __syncwarp();
    if (lane < n)
        for (int i = 0; i < n; ++i) A[i + lane * n] = cscale(A[i + lane * n], scale);
    if (lane < n)
        for (int i = 0; i < n; ++i) {
            const double2 e = make_double2(i == lane ? 1.0 : 0.0, 0.0);
            N[i + lane * n] = e;
            Dm[i + lane * n] = e;
            X[i + lane * n] = e;
        }
    __syncwarp();
    double c = 1.0;
    const int q = 6;
    double2 col[32];
    for (int k = 1; k <= q; ++k) {
        c = c * (q - k + 1) / static_cast<double>((2 * q - k + 1) * k);
        // X = A * X ; lane j computes column j
        if (lane < n) {
            for (int i = 0; i < n; ++i) {
                double2 s = make_double2(0.0, 0.0);
                for (int kk = 0; kk < n; ++kk) s = cfma(A[i + kk * n], X[kk + lane * n], s);
                col[i] = s;
            }
        }
        __syncwarp();
        const double sgn = (k % 2 == 0) ? 1.0 : -1.0;
        if (lane < n)
            for (int i = 0; i < n; ++i) {
                X[i + lane * n] = col[i];
                N[i + lane * n] = cadd(N[i + lane * n], cscale(col[i], c));
                Dm[i + lane * n] = cadd(Dm[i + lane * n], cscale(col[i], sgn * c));
            }
        __syncwarp();
    }
    // LU with partial pivoting on Dm, applied to N (lane j: column j of both)
    for (int k = 0; k < n; ++k) {
        double v = (lane >= k && lane < n) ? cabs2(Dm[lane + k * n]) : -1.0;
        int p = lane;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const double v2 = __shfl_xor_sync(0xffffffffu, v, o);
            const int p2 = __shfl_xor_sync(0xffffffffu, p, o);
            if (v2 > v || (v2 == v && p2 < p)) { v = v2; p = p2; }
        }
        if (!(v > 0.0)) return false;
        if (p != k && lane < n) {
            double2 t = Dm[k + lane * n]; Dm[k + lane * n] = Dm[p + lane * n]; Dm[p + lane * n] = t;
            t = N[k + lane * n]; N[k + lane * n] = N[p + lane * n]; N[p + lane * n] = t;
        }
        __syncwarp();
        const double2 piv = Dm[k + k * n];
        const double pinv = 1.0 / cabs2(piv);
        // multipliers f_i = Dm[i,k]/piv for i > k (computed by every lane identically)
        if (lane < n && lane > k) {
            for (int i = k + 1; i < n; ++i) {
                const double2 a = Dm[i + k * n];
                const double2 f = make_double2((a.x * piv.x + a.y * piv.y) * pinv, (a.y * piv.x - a.x * piv.y) * pinv);
                Dm[i + lane * n] = csub(Dm[i + lane * n], cmul(f, Dm[k + lane * n]));
            }
        }
        if (lane < n) {
            for (int i = k + 1; i < n; ++i) {
                const double2 a = Dm[i + k * n];
                const double2 f = make_double2((a.x * piv.x + a.y * piv.y) * pinv, (a.y * piv.x - a.x * piv.y) * pinv);
                N[i + lane * n] = csub(N[i + lane * n], cmul(f, N[k + lane * n]));
            }
        }
        __syncwarp();
    }
    // back substitution: lane j solves column j of N in place
    if (lane < n) {
        for (int i = n - 1; i >= 0; --i) {
            double2 s = N[i + lane * n];
            for (int kk = i + 1; kk < n; ++kk) s = csub(s, cmul(Dm[i + kk * n], N[kk + lane * n]));
            const double2 d = Dm[i + i * n];
            const double dinv = 1.0 / cabs2(d);
            N[i + lane * n] = make_double2((s.x * d.x + s.y * d.y) * dinv, (s.y * d.x - s.x * d.y) * dinv);
        }
    }
    __syncwarp();
    // exp(A) e1 = F^(2^sc) e1: repeated squaring of F, then take column 0.
    for (int s = 0; s < sc; ++s) {
        if (lane < n) {
            for (int i = 0; i < n; ++i) {
                double2 t = make_double2(0.0, 0.0);
                for (int kk = 0; kk < n; ++kk) t = cfma(N[i + kk * n], N[kk + lane * n], t);
                col[i] = t;
            }
        }
        __syncwarp();
        if (lane < n)
            for (int i = 0; i < n; ++i) X[i + lane * n] = col[i];
        __syncwarp();
        if (lane < n)
            for (int i = 0; i < n; ++i) N[i + lane * n] = X[i + lane * n];
        __syncwarp();
    }
    if (lane < n) y[lane] = N[lane];
    __syncwarp();
    return true;
}

}  // namespace msgpu
