// msgpu_batch.cuh -- batching form: many spin systems of uneven dimension
// and uneven trajectory counts in ONE persistent launch.
//
// The launch covers every time step of every (system, trajectory) item of
// the batch.  CTAs are persistent (a few per SM) and pull work from two
// queues:
//   * large items (dimension >= team threshold): the whole CTA (8 warps)
//     propagates one trajectory, block-level reductions;
//   * small items: each warp of the CTA propagates its own trajectory.
// The Krylov vectors of a team live in its slice of a global scratch buffer
// (L2-resident for all but the largest systems); shared memory holds the
// per-warp small-matrix exponential scratch and the reduction buffers.
// The recurrence is Lanczos on H (K = kappa I) with complex64 vectors and
// FP32 SpMV, FP64 dot products, norms, tridiagonal and expm -- the precision
// form.  Results are independent of batch composition: a trajectory's
// arithmetic, its noise (counter-based) and its reductions do not depend on
// which team or CTA processes it.
#pragma once

#include "msgpu_resident.cuh"

namespace msgpu {
namespace {  // internal linkage (see msgpu_kernels.cuh)

constexpr int kBatchWarps = 8;
constexpr int kBatchThreads = 32 * kBatchWarps;

// complex words of per-warp shared scratch for Krylov dimension m
__host__ __device__ inline size_t batch_expm_words(int m) { return 4 * static_cast<size_t>(m) * m + 2 * m; }

struct WarpTeam {
    __device__ int rank() const { return threadIdx.x & 31; }
    __device__ int size() const { return 32; }
    __device__ void sync() const { __syncwarp(); }
    __device__ bool leader() const { return (threadIdx.x & 31) == 0; }
    __device__ bool expm_warp() const { return true; }
    __device__ double sum(double v) const { return warp_sum(v); }
};

struct CtaTeam {
    double *red;  // kBatchWarps doubles of shared memory
    __device__ int rank() const { return threadIdx.x; }
    __device__ int size() const { return kBatchThreads; }
    __device__ void sync() const { __syncthreads(); }
    __device__ bool leader() const { return threadIdx.x == 0; }
    __device__ bool expm_warp() const { return threadIdx.x < 32; }
    __device__ double sum(double v) const
    {
        v = warp_sum(v);
        __syncthreads();
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
        __syncthreads();
        double s = 0.0;
#pragma unroll
        for (int w = 0; w < kBatchWarps; ++w) s += red[w];
        return s;
    }
};

// team-strided H v (FP32) into y
template <class Team>
__device__ __forceinline__ void team_apply(const Team &tm, const ResidentSystem &S, const float2 *v, float2 *y)
{
    for (int r = tm.rank(); r < S.D; r += tm.size()) {
        const int kb = __ldg(S.rowptr + r), ke = __ldg(S.rowptr + r + 1);
        float2 a = make_float2(0.f, 0.f);
        for (int k = kb; k < ke; ++k) a = cfmaf(__ldg(S.valf + k), v[__ldg(S.col + k)], a);
        y[r] = a;
    }
    tm.sync();
}

template <class Team>
__device__ void team_epilogue(const Team &tm, const ResidentSystem &S, float2 *x, int flip, double *vals,
                              double &nrm)
{
    const int Q = S.D / 4;
    double obs[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    double nn = 0.0;
    for (int q = tm.rank(); q < Q; q += tm.size()) {
        const int base = quartet_base(q, S.s1, S.s2);
        const int r[4] = {base, base + S.s2, base + S.s1, base + S.s1 + S.s2};
        double2 v[4];
#pragma unroll
        for (int a = 0; a < 4; ++a) v[a] = ld2(x + r[a]);
        if (flip) {
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
    for (int o = 0; o < S.nobs; ++o) vals[o] = tm.sum(obs[o]) * S.rates[o];
    nrm = tm.sum(nn);
    tm.sync();
}

// Whole time loop of one trajectory by one team.  V: (m+1) x D scratch
// (slot m is the work vector / state); ex: batch_expm_words(m) complex of
// shared memory: alpha/beta (m), the expm matrices A, X, N, Dm (4 m^2), y (m).
template <class Team>
__device__ void team_propagate(const Team &tm, const ResidentSystem &S, int t, float2 *V, double2 *ex, int *status)
{
    const int D = S.D, m = S.m;
    float2 *z = V + static_cast<size_t>(m) * D;
    double2 *Hm = ex;  // alpha in .x, beta in .y (m entries)
    double2 *A = Hm + m, *X = A + static_cast<size_t>(m) * m, *N = X + static_cast<size_t>(m) * m;
    double2 *Dm = N + static_cast<size_t>(m) * m, *y = Dm + static_cast<size_t>(m) * m;
    float2 *col = reinterpret_cast<float2 *>(S.psi) + static_cast<size_t>(t) * D;
    for (int r = tm.rank(); r < D; r += tm.size()) z[r] = col[r];
    tm.sync();
    double accv[8], compv[8], prevv[8], vals[8];
    for (int o = 0; o < S.nobs; ++o) {
        accv[o] = S.accumulate ? S.acc[static_cast<size_t>(o) * S.acc_ld + t] : 0.0;
        compv[o] = S.accumulate ? S.comp[static_cast<size_t>(o) * S.acc_ld + t] : 0.0;
    }
    const int steps = S.ntimes - 1;
    const long long g0 = S.step_offset;
    double nrm2 = 0.0;
    bool bad = false;
    {
        const int f = steps > 0 ? noise_bit(S.nz, t, g0, 0, S.pflip[0]) : 0;
        team_epilogue(tm, S, z, f, vals, nrm2);
        for (int o = 0; o < S.nobs; ++o) prevv[o] = vals[o];
        if (S.traj_values && tm.leader())
            for (int o = 0; o < S.nobs; ++o) S.traj_values[static_cast<size_t>(t) * S.nobs + o] = vals[o];
    }
    for (int s = 0; s < steps; ++s) {
        const double dt = S.times[s + 1] - S.times[s];
        const double beta0 = sqrt(nrm2);
        int n = m;
        if (beta0 > 0.0) {
            const float inv = static_cast<float>(1.0 / beta0);
            for (int r = tm.rank(); r < D; r += tm.size()) V[r] = make_float2(z[r].x * inv, z[r].y * inv);
            tm.sync();
            double bprev = 0.0;
            for (int j = 0; j < m; ++j) {
                float2 *vj = V + static_cast<size_t>(j) * D;
                team_apply(tm, S, vj, z);
                double ps = 0.0;
                for (int r = tm.rank(); r < D; r += tm.size())
                    ps += static_cast<double>(vj[r].x) * z[r].x + static_cast<double>(vj[r].y) * z[r].y;
                const double alpha = tm.sum(ps);
                double pn = 0.0;
                const float fa = static_cast<float>(alpha), fb = static_cast<float>(bprev);
                for (int r = tm.rank(); r < D; r += tm.size()) {
                    float2 u = z[r];
                    u.x = fmaf(-fa, vj[r].x, u.x);
                    u.y = fmaf(-fa, vj[r].y, u.y);
                    if (j > 0) {
                        u.x = fmaf(-fb, vj[r - D].x, u.x);
                        u.y = fmaf(-fb, vj[r - D].y, u.y);
                    }
                    z[r] = u;
                    pn += static_cast<double>(u.x) * u.x + static_cast<double>(u.y) * u.y;
                }
                const double bn = sqrt(tm.sum(pn));
                if (tm.leader()) Hm[j] = make_double2(alpha, bn);
                if (j == m - 1) break;
                if (bn < 1e-14) { n = j + 1; break; }
                const float bi = static_cast<float>(1.0 / bn);
                for (int r = tm.rank(); r < D; r += tm.size()) vj[D + r] = make_float2(z[r].x * bi, z[r].y * bi);
                bprev = bn;
                tm.sync();
            }
            tm.sync();
            bool ok = true;
            if (tm.expm_warp()) {
                const int lane = threadIdx.x & 31;
                // tridiagonal Lanczos matrix: alpha on Hm[i].x, beta_{i+1} on Hm[i].y
                const double d = lane < n ? Hm[lane].x : 0.0;
                const double lo = (lane < n && lane > 0) ? Hm[lane - 1].y : 0.0;
                const double hi = lane + 1 < n ? Hm[lane].y : 0.0;
                double2 yl;
                ok = warp_tridiag_expm_e1(n, d, lo, hi, S.kappa, dt, yl);
                if (lane < n) y[lane] = yl;
                if (!ok && lane == 0) atomicOr(status, 1);
                if (!ok && lane < n) y[lane] = make_double2(0.0, 0.0);
                __syncwarp();
            }
            tm.sync();
            for (int r = tm.rank(); r < D; r += tm.size()) {
                double2 sacc = make_double2(0.0, 0.0);
                for (int j = 0; j < n; ++j) {
                    const float2 v = V[static_cast<size_t>(j) * D + r];
                    sacc = cfma(y[j], make_double2(v.x, v.y), sacc);
                }
                z[r] = make_float2(static_cast<float>(sacc.x * beta0), static_cast<float>(sacc.y * beta0));
            }
            tm.sync();
        }
        const long long g = g0 + s;
        int f = noise_bit(S.nz, t, g, 1, S.pflip[s]);
        if (s + 1 < steps) f ^= noise_bit(S.nz, t, g + 1, 0, S.pflip[s + 1]);
        team_epilogue(tm, S, z, f, vals, nrm2);
        for (int o = 0; o < S.nobs; ++o) {
            const double term = 0.5 * dt * (prevv[o] + vals[o]) - compv[o];
            const double sum = accv[o] + term;
            compv[o] = (sum - accv[o]) - term;
            accv[o] = sum;
            prevv[o] = vals[o];
            if (!isfinite(vals[o])) bad = true;
        }
        if (S.traj_values && tm.leader())
            for (int o = 0; o < S.nobs; ++o)
                S.traj_values[(static_cast<size_t>(s + 1) * S.M + t) * S.nobs + o] = vals[o];
    }
    for (int r = tm.rank(); r < D; r += tm.size()) col[r] = z[r];
    if (tm.leader()) {
        for (int o = 0; o < S.nobs; ++o) {
            S.acc[static_cast<size_t>(o) * S.acc_ld + t] = accv[o];
            S.comp[static_cast<size_t>(o) * S.acc_ld + t] = compv[o];
            S.prev[static_cast<size_t>(o) * S.acc_ld + t] = prevv[o];
        }
        if (bad) atomicOr(status, 2);
    }
    tm.sync();
}

// Persistent batch launch.  items[0, nlarge) are CTA-team items, the rest
// are warp-team items.  queue[0] / queue[1] are the two work counters
// (zeroed before the launch).  scratch: per CTA `slice` float2 elements
// (large items use all of it; warp w of a small item uses its eighth).
// Dynamic shared memory: kBatchWarps x batch_expm_words(m) complex.
__global__ void __launch_bounds__(kBatchThreads)
k_batch(const ResidentSystem *__restrict__ systems, const ResidentWork *__restrict__ items, int nlarge, int nitems,
        int *__restrict__ queue, float2 *__restrict__ scratch, size_t slice, int mmax, int *__restrict__ status)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ int s_item;
    __shared__ double red[kBatchWarps];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const size_t ex_per_warp = batch_expm_words(mmax);
    double2 *ex_base = reinterpret_cast<double2 *>(smem_raw);
    float2 *my = scratch + static_cast<size_t>(blockIdx.x) * slice;
    // large items: whole CTA per trajectory
    CtaTeam cta{red};
    for (;;) {
        if (threadIdx.x == 0) s_item = atomicAdd(queue, 1);
        __syncthreads();
        const int it = s_item;
        __syncthreads();
        if (it >= nlarge) break;
        const ResidentWork w = items[it];
        team_propagate(cta, systems[w.sys], w.traj, my, ex_base, status);
    }
    // small items: one trajectory per warp
    WarpTeam wt;
    float2 *mine = my + static_cast<size_t>(warp) * (slice / kBatchWarps);
    double2 *ex = ex_base + static_cast<size_t>(warp) * ex_per_warp;
    const int nsmall = nitems - nlarge;
    for (;;) {
        int it = 0;
        if (lane == 0) it = atomicAdd(queue + 1, 1);
        it = __shfl_sync(0xffffffffu, it, 0);
        if (it >= nsmall) break;
        const ResidentWork w = items[nlarge + it];
        team_propagate(wt, systems[w.sys], w.traj, mine, ex, status);
    }
}

}  // namespace
}  // namespace msgpu
