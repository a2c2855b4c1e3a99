// msgpu_resident.cuh -- "resident" form for small Hilbert dimensions.
//
// One warp owns one trajectory for the whole time loop: its Krylov basis,
// Hessenberg matrix and expm scratch live in shared memory, the trajectory is
// read from and written back to its column of the reference's column-major
// D x M factor block once per launch, and every time step (evaluation, ST
// flips, Krylov step, trapezoid) runs inside one kernel launch.  For small D
// (the radical pair with a handful of nuclei) this removes the per-step
// launches of the streamed path; the arithmetic is FP64-latency bound.
//
// Recurrences:
//   complex128: Arnoldi with modified Gram-Schmidt in the order of
//     SpinSpace::ArnoldiProcess (SpinSpace_operators.cpp:1352-1408), on
//     G = -iH - K, breakdown below 1e-14;
//   complex64: Lanczos on H (K = kappa I) with FP32 vectors and SpMV, FP64
//     dot products, norms, tridiagonal and expm.
//
// Work items are (system, trajectory) pairs so that one launch can serve
// several systems of different dimension (the batching form).
#pragma once

#include "msgpu_kernels.cuh"

namespace msgpu {
namespace {  // internal linkage (see msgpu_kernels.cuh)

struct ResidentSystem {
    // H (rad/ns) as CSR; values complex128 and complex64 copies
    const int *rowptr;
    const int *col;
    const double2 *val;
    const float2 *valf;
    // K: CSR (krow != null) or kappa * I
    const int *krow;
    const int *kcol;
    const double2 *kval;
    double kappa;
    int D, M, m;       // dimension, trajectories, Krylov dimension
    int acc_ld;        // stride of acc/comp/prev (>= M)
    int s1, s2;        // electron-pair strides (s1 > s2)
    int nobs;
    const double2 *obs;   // nobs x 16 (row-major 4x4, kernel pair basis)
    const double *rates;  // nobs
    Noise nz;             // flip stream (replay bits indexed by this system's M)
    void *psi;            // D x M column-major, double2 or float2
    double *acc, *comp, *prev;  // nobs x M (observable-major)
    double *traj_values;        // (ntimes) x M x nobs, or null
    const double *times;        // ntimes
    const double *pflip;        // per step flip probability of a half step
    int ntimes;
    long long step_offset;
    int accumulate;
};

struct ResidentWork {
    int sys;
    int traj;
};

template <typename T>
struct ResidentSmem;

__device__ __forceinline__ double2 ld2(const double2 *p) { return *p; }
__device__ __forceinline__ double2 ld2(const float2 *p) { const float2 v = *p; return make_double2(v.x, v.y); }
__device__ __forceinline__ void st2(double2 *p, double2 v) { *p = v; }
__device__ __forceinline__ void st2(float2 *p, double2 v) { *p = make_float2(static_cast<float>(v.x), static_cast<float>(v.y)); }

// Bytes of shared memory one warp needs.
__host__ __device__ inline size_t resident_warp_bytes(int D, int m, int elem)
{
    // basis m*D + work vector D (elements), then FP64 Hessenberg/tridiagonal
    // (m*m complex) and expm scratch (4 m*m + m complex)
    size_t b = static_cast<size_t>(elem) * D * (m + 1);
    b = (b + 15) / 16 * 16;
    b += sizeof(double2) * (static_cast<size_t>(m) * m + 4 * static_cast<size_t>(m) * m + m);
    return b;
}

// Evaluate the pair observables of the trajectory held in x (shared), apply
// the flip first; returns per-lane partials summed over the warp.
template <typename T>
__device__ void resident_epilogue(T *x, const ResidentSystem &S, int flip, double *vals, double &nrm)
{
    const int lane = threadIdx.x & 31;
    const int Q = S.D / 4;
    double obs[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    double nn = 0.0;
    for (int q = lane; q < Q; q += 32) {
        const int base = quartet_base(q, S.s1, S.s2);
        const int r[4] = {base, base + S.s2, base + S.s1, base + S.s1 + S.s2};
        double2 v[4];
#pragma unroll
        for (int a = 0; a < 4; ++a) v[a] = ld2(x + r[a]);
        if (flip) {  // U = PS - PT on the pair
            const double2 b = v[1];
            v[0] = make_double2(-v[0].x, -v[0].y);
            v[1] = make_double2(-v[2].x, -v[2].y);
            v[2] = make_double2(-b.x, -b.y);
            v[3] = make_double2(-v[3].x, -v[3].y);
        }
        nn += cabs2(v[0]) + cabs2(v[1]) + cabs2(v[2]) + cabs2(v[3]);
        for (int o = 0; o < S.nobs; ++o) {
            const double2 *op = S.obs + o * 16;
            double sum = 0.0;
#pragma unroll
            for (int a = 0; a < 4; ++a) {
                double2 ox = make_double2(0.0, 0.0);
#pragma unroll
                for (int b = 0; b < 4; ++b) ox = cfma(__ldg(op + a * 4 + b), v[b], ox);
                sum += v[a].x * ox.x + v[a].y * ox.y;
            }
            obs[o] += sum;
        }
#pragma unroll
        for (int a = 0; a < 4; ++a) st2(x + r[a], v[a]);
    }
    for (int o = 0; o < S.nobs; ++o) vals[o] = warp_sum(obs[o]) * S.rates[o];
    nrm = warp_sum(nn);
    __syncwarp();
}

// y = G v (complex128, G = -iH - K) or y = H v (complex64 Lanczos) for the
// rows owned by this lane; v, y in shared memory.
template <typename T>
__device__ __forceinline__ void resident_apply(const ResidentSystem &S, const T *v, T *y, bool lanczos)
{
    const int lane = threadIdx.x & 31;
    for (int r = lane; r < S.D; r += 32) {
        const int kb = __ldg(S.rowptr + r), ke = __ldg(S.rowptr + r + 1);
        double2 acc = make_double2(0.0, 0.0);
        if (sizeof(T) == sizeof(double2)) {
            for (int k = kb; k < ke; ++k) acc = cfma(__ldg(S.val + k), ld2(v + __ldg(S.col + k)), acc);
        } else {
            float2 a = make_float2(0.f, 0.f);
            for (int k = kb; k < ke; ++k) {
                const float2 h = __ldg(S.valf + k);
                const double2 xv = ld2(v + __ldg(S.col + k));
                a = cfmaf(h, make_float2(static_cast<float>(xv.x), static_cast<float>(xv.y)), a);
            }
            acc = make_double2(a.x, a.y);
        }
        if (lanczos) {
            st2(y + r, acc);
        } else {
            double2 g = make_double2(acc.y, -acc.x);  // -i * (H v)
            if (S.krow) {
                double2 ka = make_double2(0.0, 0.0);
                for (int k = __ldg(S.krow + r); k < __ldg(S.krow + r + 1); ++k)
                    ka = cfma(__ldg(S.kval + k), ld2(v + __ldg(S.kcol + k)), ka);
                g = csub(g, ka);
            } else {
                g = csub(g, cscale(ld2(v + r), S.kappa));
            }
            st2(y + r, g);
        }
    }
    __syncwarp();
}

template <typename T>
__device__ double resident_dot_re(const T *a, const T *b, int D, double2 *cplx)
{
    const int lane = threadIdx.x & 31;
    double2 s = make_double2(0.0, 0.0);
    for (int r = lane; r < D; r += 32) s = cadd(s, cconjmul(ld2(a + r), ld2(b + r)));
    s.x = warp_sum(s.x);
    s.y = warp_sum(s.y);
    if (cplx) *cplx = s;
    return s.x;
}

// One launch = the whole time loop for every work item (one warp each).
template <typename T, bool kLanczos>
__global__ void k_resident(const ResidentSystem *__restrict__ systems, const ResidentWork *__restrict__ work,
                           int nwork, size_t warp_bytes, int *__restrict__ status)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int wi = blockIdx.x * (blockDim.x >> 5) + warp;
    if (wi >= nwork) return;
    const ResidentWork w = work[wi];
    const ResidentSystem &S = systems[w.sys];
    const int D = S.D, m = S.m, t = w.traj;
    unsigned char *base = smem_raw + static_cast<size_t>(warp) * warp_bytes;
    T *V = reinterpret_cast<T *>(base);               // m x D basis
    T *z = V + static_cast<size_t>(m) * D;            // work vector / state
    size_t off = (sizeof(T) * static_cast<size_t>(D) * (m + 1) + 15) / 16 * 16;
    double2 *Hm = reinterpret_cast<double2 *>(base + off);  // m x m, column-major
    double2 *A = Hm + static_cast<size_t>(m) * m;
    double2 *X = A + static_cast<size_t>(m) * m, *N = X + static_cast<size_t>(m) * m;
    double2 *Dm = N + static_cast<size_t>(m) * m, *y = Dm + static_cast<size_t>(m) * m;

    T *col = reinterpret_cast<T *>(S.psi) + static_cast<size_t>(t) * D;
    for (int r = lane; r < D; r += 32) z[r] = col[r];
    __syncwarp();

    double accv[8], compv[8], prevv[8], vals[8];
    for (int o = 0; o < S.nobs; ++o) {
        accv[o] = S.accumulate ? S.acc[static_cast<size_t>(o) * S.acc_ld + t] : 0.0;
        compv[o] = S.accumulate ? S.comp[static_cast<size_t>(o) * S.acc_ld + t] : 0.0;
    }
    const int steps = S.ntimes - 1;
    const long long g0 = S.step_offset;
    double nrm2 = 0.0;
    bool bad = false;
    // first time point: evaluate, then the first half-step flip of step 0
    {
        const int f = steps > 0 ? noise_bit(S.nz, t, g0, 0, S.pflip[0]) : 0;
        resident_epilogue(z, S, f, vals, nrm2);
        for (int o = 0; o < S.nobs; ++o) prevv[o] = vals[o];
        if (S.traj_values && lane == 0)
            for (int o = 0; o < S.nobs; ++o) S.traj_values[static_cast<size_t>(t) * S.nobs + o] = vals[o];
    }
    for (int s = 0; s < steps; ++s) {
        const double dt = S.times[s + 1] - S.times[s];
        const double beta0 = sqrt(nrm2);
        int n = m;
        if (beta0 > 0.0) {
            const double inv = 1.0 / beta0;
            for (int r = lane; r < D; r += 32) st2(V + r, cscale(ld2(z + r), inv));
            __syncwarp();
            if (!kLanczos) {
                // Arnoldi with modified Gram-Schmidt (reference order)
                for (int j = 0; j < m; ++j) {
                    resident_apply(S, V + static_cast<size_t>(j) * D, z, false);
                    for (int i = 0; i <= j; ++i) {
                        double2 h;
                        resident_dot_re(V + static_cast<size_t>(i) * D, z, D, &h);
                        for (int r = lane; r < D; r += 32)
                            st2(z + r, csub(ld2(z + r), cmul(h, ld2(V + static_cast<size_t>(i) * D + r))));
                        if (lane == 0) Hm[i + j * m] = h;
                        __syncwarp();
                    }
                    const double zn = sqrt(resident_dot_re(z, z, D, nullptr));
                    if (j == m - 1) break;
                    if (lane == 0) Hm[(j + 1) + j * m] = make_double2(zn, 0.0);
                    if (zn < 1e-14) { n = j + 1; break; }
                    const double zi = 1.0 / zn;
                    for (int r = lane; r < D; r += 32)
                        st2(V + static_cast<size_t>(j + 1) * D + r, cscale(ld2(z + r), zi));
                    __syncwarp();
                }
                __syncwarp();
                // upper Hessenberg part only; entries below the subdiagonal are never written
                if (lane < n)
                    for (int i = 0; i < n; ++i)
                        A[i + lane * n] = i <= lane + 1 ? cscale(Hm[i + lane * m], dt) : make_double2(0.0, 0.0);
            } else {
                // Lanczos on H: alpha on Hm[j] .x, beta_{j+1} on Hm[j] .y
                double bprev = 0.0;
                for (int j = 0; j < m; ++j) {
                    T *vj = V + static_cast<size_t>(j) * D;
                    resident_apply(S, vj, z, true);
                    const double alpha = resident_dot_re(vj, z, D, nullptr);
                    for (int r = lane; r < D; r += 32) {
                        double2 u = csub(ld2(z + r), cscale(ld2(vj + r), alpha));
                        if (j > 0) u = csub(u, cscale(ld2(vj - D + r), bprev));
                        st2(z + r, u);
                    }
                    __syncwarp();
                    const double bn = sqrt(resident_dot_re(z, z, D, nullptr));
                    if (lane == 0) Hm[j] = make_double2(alpha, bn);
                    if (j == m - 1) break;
                    if (bn < 1e-14) { n = j + 1; break; }
                    const double bi = 1.0 / bn;
                    for (int r = lane; r < D; r += 32) st2(vj + D + r, cscale(ld2(z + r), bi));
                    bprev = bn;
                    __syncwarp();
                }
                __syncwarp();
            }
            __syncwarp();
            bool ok;
            if (kLanczos) {
                // tridiagonal: alpha on Hm[i].x, beta_{i+1} on Hm[i].y
                const double d = lane < n ? Hm[lane].x : 0.0;
                const double lo = (lane < n && lane > 0) ? Hm[lane - 1].y : 0.0;
                const double hi = lane + 1 < n ? Hm[lane].y : 0.0;
                double2 yl;
                ok = warp_tridiag_expm_e1(n, d, lo, hi, S.kappa, dt, yl);
                if (lane < n) y[lane] = yl;
                __syncwarp();
            } else {
                ok = warp_expm_col0(n, A, X, N, Dm, y);
            }
            if (!ok) {
                if (lane == 0) atomicOr(status, 1);
                n = 0;
            }
            for (int r = lane; r < D; r += 32) {
                double2 sacc = make_double2(0.0, 0.0);
                for (int j = 0; j < n; ++j) sacc = cfma(y[j], ld2(V + static_cast<size_t>(j) * D + r), sacc);
                st2(z + r, cscale(sacc, beta0));
            }
            __syncwarp();
        }
        // second half flip of step s, first half flip of step s+1, evaluation
        const long long g = g0 + s;
        int f = noise_bit(S.nz, t, g, 1, S.pflip[s]);
        if (s + 1 < steps) f ^= noise_bit(S.nz, t, g + 1, 0, S.pflip[s + 1]);
        resident_epilogue(z, S, f, vals, nrm2);
        for (int o = 0; o < S.nobs; ++o) {
            const double term = 0.5 * dt * (prevv[o] + vals[o]) - compv[o];
            const double sum = accv[o] + term;
            compv[o] = (sum - accv[o]) - term;
            accv[o] = sum;
            prevv[o] = vals[o];
            if (!isfinite(vals[o])) bad = true;
        }
        if (S.traj_values && lane == 0)
            for (int o = 0; o < S.nobs; ++o)
                S.traj_values[(static_cast<size_t>(s + 1) * S.M + t) * S.nobs + o] = vals[o];
    }
    for (int r = lane; r < D; r += 32) col[r] = z[r];
    if (lane == 0) {
        for (int o = 0; o < S.nobs; ++o) {
            S.acc[static_cast<size_t>(o) * S.acc_ld + t] = accv[o];
            S.comp[static_cast<size_t>(o) * S.acc_ld + t] = compv[o];
            S.prev[static_cast<size_t>(o) * S.acc_ld + t] = prevv[o];
        }
        if (bad) atomicOr(status, 2);
    }
}

// values[s][o] = sum over trajectories of traj_values[s][t][o] (fixed order);
// one block per time point.
__global__ void k_resident_values(const double *__restrict__ traj_values, int M, int nobs, double *__restrict__ values)
{
    __shared__ double red[8][32];
    const int s = blockIdx.x, lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int t = threadIdx.x; t < M; t += blockDim.x)
        for (int o = 0; o < nobs; ++o) acc[o] += traj_values[(static_cast<size_t>(s) * M + t) * nobs + o];
    for (int o = 0; o < nobs; ++o) {
        const double v = warp_sum(acc[o]);
        if (lane == 0) red[o][warp] = v;
    }
    __syncthreads();
    if (threadIdx.x < nobs) {
        double v = 0.0;
        for (int w = 0; w < (blockDim.x >> 5); ++w) v += red[threadIdx.x][w];
        values[static_cast<size_t>(s) * nobs + threadIdx.x] = v;
    }
}

}  // namespace
}  // namespace msgpu
