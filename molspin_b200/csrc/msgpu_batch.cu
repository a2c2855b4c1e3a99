// msgpu_batch.cu -- C ABI of the batching form (include/msgpu.h,
// msgpu_batch_*): many radical-pair systems of uneven dimension and
// trajectory count propagated together.  Systems below kStreamDim run in
// one persistent launch (k_batch), replayed from a CUDA graph, with the team
// threshold and the persistent grid size picked by an autotuner on the batch
// itself.  A large system is better served by the streamed single-system
// path, which advances all its trajectories in lockstep through the
// quartet-block SpMM (one read of H per 64 trajectories instead of one per
// trajectory): those systems get their own context and stream and run
// concurrently with the persistent launch and with each other.

#include "msgpu.h"

#include <algorithm>
#include <array>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "msgpu_batch.cuh"

using namespace msgpu;

namespace {

struct Buf {
    void *p = nullptr;
    size_t bytes = 0;
};

// Systems of at least this dimension take the streamed single-system path
// (measured on the 64-system benchmark batch: the persistent teams win below
// it, the lockstep SpMM above it).
constexpr int kStreamDim = 2048;
constexpr int kStreamWorkers = 8;  // host threads driving streamed systems

struct BatchSystem {
    int D = 0, M = 0, nobs = 0, s1 = 0, s2 = 0;
    double kappa = 0.0, st_rate = 0.0;
    unsigned long long seed = 0;
    Buf rowptr, col, valf, obs, rates, psi, acc, comp, prev, pflip;
    msgpu_ctx *ctx = nullptr;  // streamed single-system path (D >= kStreamDim)
};

}  // namespace

struct msgpu_batch {
    int device = 0;
    size_t budget = 0, used = 0;
    cudaStream_t stream = nullptr;
    std::string err;
    std::vector<BatchSystem> sys;
    // systems of the persistent route dropped by msgpu_batch_clear: their device
    // buffers serve the next msgpu_batch_add_system (no cudaMalloc / cudaFree per reuse)
    std::vector<BatchSystem> spare;
    Buf sys_d, items_d, queue_d, status_d, scratch, times_d, backup;
    int threshold = 512, ctas_per_sm = 2, tuned = 0;
    int sm_count = 0;
    cudaGraphExec_t graph = nullptr;
    size_t graph_key = 0;
    float last_ms = 0.f;
    int m = 0;
    long long launches = 0;  // persistent launches (tuning probes included)
};

namespace {

int bfail(msgpu_batch *b, int code, const std::string &msg)
{
    if (b) b->err = msg;
    return code;
}

void brelease(msgpu_batch *b, Buf &x)
{
    if (x.p) {
        cudaFree(x.p);
        b->used -= x.bytes;
    }
    x.p = nullptr;
    x.bytes = 0;
}

int bensure(msgpu_batch *b, Buf &x, size_t bytes, const char *what)
{
    if (bytes == 0) bytes = 16;
    if (x.p && x.bytes >= bytes) return MSGPU_OK;
    brelease(b, x);
    if (b->budget && b->used + bytes > b->budget)
        return bfail(b, MSGPU_ERR_BUDGET, std::string("batch: device memory budget exceeded allocating ") + what);
    cudaError_t e = cudaMalloc(&x.p, bytes);
    if (e != cudaSuccess) {
        x.p = nullptr;
        return bfail(b, MSGPU_ERR_CUDA, std::string("batch: ") + what + ": " + cudaGetErrorString(e));
    }
    x.bytes = bytes;
    b->used += bytes;
    return MSGPU_OK;
}

int upload(msgpu_batch *b, Buf &x, const void *src, size_t bytes, const char *what)
{
    if (int rc = bensure(b, x, bytes, what)) return rc;
    cudaError_t e = cudaMemcpyAsync(x.p, src, bytes, cudaMemcpyHostToDevice, b->stream);
    if (e) return bfail(b, MSGPU_ERR_CUDA, std::string("batch: upload ") + what + ": " + cudaGetErrorString(e));
    return MSGPU_OK;
}

void drop_graph(msgpu_batch *b)
{
    if (b->graph) cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
    b->graph_key = 0;
}

double flip_prob(double st_rate, double h) { return -0.5 * std::expm1(-2.0 * (0.5 * st_rate) * h); }

// Descriptors, work items and scratch for the given schedule; returns the
// grid size through *grid.
int prepare(msgpu_batch *b, int ntimes, int m, int accumulate, long long step_offset, int threshold,
            int ctas_per_sm, int *grid, size_t *slice, size_t *smem, int *nlarge, int *nitems)
{
    std::vector<ResidentSystem> desc(b->sys.size());
    std::vector<ResidentWork> large, small;
    int dmax_large = 0, dmax_small = 0;
    for (size_t i = 0; i < b->sys.size(); ++i) {
        BatchSystem &s = b->sys[i];
        ResidentSystem S;
        std::memset(&S, 0, sizeof(S));
        S.rowptr = static_cast<const int *>(s.rowptr.p);
        S.col = static_cast<const int *>(s.col.p);
        S.valf = static_cast<const float2 *>(s.valf.p);
        S.kappa = s.kappa;
        S.D = s.D;
        S.M = s.M;
        S.acc_ld = s.M;
        S.m = std::min(m, s.D);
        S.s1 = s.s1;
        S.s2 = s.s2;
        S.nobs = s.nobs;
        S.obs = static_cast<const double2 *>(s.obs.p);
        S.rates = static_cast<const double *>(s.rates.p);
        S.nz.mode = s.st_rate > 0.0 ? MSGPU_NOISE_PHILOX : MSGPU_NOISE_NONE;
        S.nz.M = s.M;
        S.nz.seed = s.seed;
        S.psi = s.psi.p;
        S.acc = static_cast<double *>(s.acc.p);
        S.comp = static_cast<double *>(s.comp.p);
        S.prev = static_cast<double *>(s.prev.p);
        S.traj_values = nullptr;
        S.times = static_cast<const double *>(b->times_d.p);
        S.pflip = static_cast<const double *>(s.pflip.p);
        S.ntimes = ntimes;
        S.step_offset = step_offset;
        S.accumulate = accumulate;
        desc[i] = S;
        if (s.ctx) continue;  // streamed path: no work items here
        auto &dst = s.D >= threshold ? large : small;
        for (int t = 0; t < s.M; ++t) dst.push_back(ResidentWork{static_cast<int>(i), t});
        if (s.D >= threshold) dmax_large = std::max(dmax_large, s.D);
        else dmax_small = std::max(dmax_small, s.D);
    }
    // largest systems first so that the long items start early
    auto byD = [&](const ResidentWork &x, const ResidentWork &y) {
        return b->sys[x.sys].D > b->sys[y.sys].D || (b->sys[x.sys].D == b->sys[y.sys].D && x.sys < y.sys);
    };
    std::stable_sort(large.begin(), large.end(), byD);
    std::stable_sort(small.begin(), small.end(), byD);
    std::vector<ResidentWork> items = large;
    items.insert(items.end(), small.begin(), small.end());
    *nlarge = static_cast<int>(large.size());
    *nitems = static_cast<int>(items.size());
    const size_t per_large = static_cast<size_t>(m + 1) * dmax_large;
    const size_t per_small = static_cast<size_t>(m + 1) * dmax_small * kBatchWarps;
    *slice = (std::max(per_large, per_small) + 63) / 64 * 64;
    *grid = std::max(1, b->sm_count * ctas_per_sm);
    *smem = sizeof(double2) * kBatchWarps * batch_expm_words(m);
    int rc;
    if ((rc = upload(b, b->sys_d, desc.data(), sizeof(ResidentSystem) * desc.size(), "descriptors")) ||
        (rc = upload(b, b->items_d, items.data(), sizeof(ResidentWork) * std::max<size_t>(1, items.size()), "items")) ||
        (rc = bensure(b, b->queue_d, 2 * sizeof(int), "queue")) ||
        (rc = bensure(b, b->status_d, sizeof(int), "status")) ||
        (rc = bensure(b, b->scratch, sizeof(float2) * *slice * *grid, "scratch")))
        return rc;
    return MSGPU_OK;
}

int launch(msgpu_batch *b, int grid, size_t slice, size_t smem, int nlarge, int nitems, int m, bool use_graph)
{
    cudaError_t e;
    if ((e = raise_smem_limit(reinterpret_cast<const void *>(k_batch), static_cast<int>(smem))))
        return bfail(b, MSGPU_ERR_CUDA, std::string("batch: shared memory: ") + cudaGetErrorString(e));
    const size_t key = (static_cast<size_t>(grid) << 40) ^ (slice << 8) ^ (static_cast<size_t>(nlarge) << 20) ^
                       static_cast<size_t>(nitems) ^ (static_cast<size_t>(m) << 56) ^ reinterpret_cast<size_t>(b->scratch.p) ^
                       (reinterpret_cast<size_t>(b->sys_d.p) << 1) ^ (reinterpret_cast<size_t>(b->items_d.p) << 2) ^
                       (reinterpret_cast<size_t>(b->queue_d.p) << 3) ^ (reinterpret_cast<size_t>(b->status_d.p) << 4);
    auto enqueue = [&]() {
        cudaMemsetAsync(b->queue_d.p, 0, 2 * sizeof(int), b->stream);
        cudaMemsetAsync(b->status_d.p, 0, sizeof(int), b->stream);
        k_batch<<<grid, kBatchThreads, smem, b->stream>>>(
            static_cast<const ResidentSystem *>(b->sys_d.p), static_cast<const ResidentWork *>(b->items_d.p), nlarge,
            nitems, static_cast<int *>(b->queue_d.p), static_cast<float2 *>(b->scratch.p), slice, m,
            static_cast<int *>(b->status_d.p));
    };
    if (!use_graph) {
        enqueue();
    } else {
        if (!b->graph || b->graph_key != key) {
            drop_graph(b);
            cudaGraph_t g;
            if ((e = cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal)))
                return bfail(b, MSGPU_ERR_CUDA, std::string("batch: capture: ") + cudaGetErrorString(e));
            enqueue();
            if ((e = cudaStreamEndCapture(b->stream, &g)))
                return bfail(b, MSGPU_ERR_CUDA, std::string("batch: capture: ") + cudaGetErrorString(e));
            e = cudaGraphInstantiate(&b->graph, g, 0);
            cudaGraphDestroy(g);
            if (e) return bfail(b, MSGPU_ERR_CUDA, std::string("batch: instantiate: ") + cudaGetErrorString(e));
            b->graph_key = key;
        }
        if ((e = cudaGraphLaunch(b->graph, b->stream)))
            return bfail(b, MSGPU_ERR_CUDA, std::string("batch: graph launch: ") + cudaGetErrorString(e));
    }
    if ((e = cudaGetLastError())) return bfail(b, MSGPU_ERR_CUDA, std::string("batch: launch: ") + cudaGetErrorString(e));
    return MSGPU_OK;
}

int set_times(msgpu_batch *b, const double *times, int ntimes)
{
    for (int s = 0; s < ntimes; ++s)
        if (!std::isfinite(times[s]) || (s > 0 && !(times[s] > times[s - 1])))
            return bfail(b, MSGPU_ERR_INVALID, "batch: times must be finite and strictly increasing");
    if (int rc = upload(b, b->times_d, times, sizeof(double) * ntimes, "times")) return rc;
    std::vector<double> pf(ntimes, 0.0);
    for (auto &s : b->sys) {
        if (s.ctx) continue;
        for (int k = 0; k + 1 < ntimes; ++k) pf[k] = flip_prob(s.st_rate, 0.5 * (times[k + 1] - times[k]));
        if (int rc = upload(b, s.pflip, pf.data(), sizeof(double) * ntimes, "flip probabilities")) return rc;
    }
    return MSGPU_OK;
}

int run_once(msgpu_batch *b, int ntimes, int m, int accumulate, long long step_offset, int threshold, int cps,
             bool graph, float *ms, const double *times = nullptr)
{
    int grid, nlarge, nitems;
    size_t slice, smem;
    if (int rc = prepare(b, ntimes, m, accumulate, step_offset, threshold, cps, &grid, &slice, &smem, &nlarge, &nitems))
        return rc;
    const auto w0 = std::chrono::steady_clock::now();
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, b->stream);
    int rc = nitems > 0 ? launch(b, grid, slice, smem, nlarge, nitems, m, graph) : MSGPU_OK;
    if (nitems > 0) b->launches += graph ? 1 : 3;  // a replay of the captured graph, or memsets + kernel
    cudaEventRecord(e1, b->stream);
    // streamed systems (times given: a real run, not a tuning probe), each on
    // its own context and stream, while the persistent launch runs
    std::vector<int> routed;
    if (times)
        for (size_t i = 0; i < b->sys.size(); ++i)
            if (b->sys[i].ctx) routed.push_back(static_cast<int>(i));
    std::vector<int> rcs(routed.size(), MSGPU_OK);
    if (!routed.empty() && rc == MSGPU_OK) {
        msgpu_run_params p;
        std::memset(&p, 0, sizeof(p));
        p.times = times;
        p.ntimes = ntimes;
        p.krylov_dim = m;
        p.precision = MSGPU_PREC_C64;
        p.recurrence = MSGPU_REC_AUTO;
        p.propagator = MSGPU_PROP_KRYLOV;
        p.step_offset = step_offset;
        p.accumulate = accumulate;
        std::atomic<size_t> next{0};
        auto worker = [&]() {
            for (size_t k; (k = next.fetch_add(1)) < routed.size();) rcs[k] = msgpu_run(b->sys[routed[k]].ctx, &p);
        };
        std::vector<std::thread> pool;
        const int nw = std::min<int>(kStreamWorkers, static_cast<int>(routed.size()));
        for (int i = 0; i < nw; ++i) pool.emplace_back(worker);
        for (auto &th : pool) th.join();
        cudaSetDevice(b->device);
    }
    cudaError_t e = cudaEventSynchronize(e1);
    float t = 0.f;
    cudaEventElapsedTime(&t, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) return rc;
    if (e) return bfail(b, MSGPU_ERR_CUDA, std::string("batch: run: ") + cudaGetErrorString(e));
    for (size_t k = 0; k < routed.size(); ++k)
        if (rcs[k])
            return bfail(b, rcs[k], "batch: system " + std::to_string(routed[k]) + ": " +
                                        msgpu_last_error(b->sys[routed[k]].ctx));
    int status = 0;
    if (nitems > 0 && (e = cudaMemcpy(&status, b->status_d.p, sizeof(int), cudaMemcpyDeviceToHost)))
        return bfail(b, MSGPU_ERR_CUDA, std::string("batch: status: ") + cudaGetErrorString(e));
    if (status & 2) return bfail(b, MSGPU_ERR_NONFINITE, "batch: non-finite observable on the device");
    if (status & 1) return bfail(b, MSGPU_ERR_EXPM, "batch: small matrix exponential failed");
    // persistent launch alone: its device time; with streamed systems: the
    // wall time of the whole run (host threads, several streams)
    if (ms)
        *ms = routed.empty() ? t
                             : std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - w0).count();
    return MSGPU_OK;
}

}  // namespace

extern "C" {

msgpu_batch *msgpu_batch_create(int device, size_t hbm_budget_bytes)
{
    if (cudaSetDevice(device) != cudaSuccess) return nullptr;
    auto *b = new msgpu_batch();
    b->device = device;
    b->budget = hbm_budget_bytes;
    cudaDeviceGetAttribute(&b->sm_count, cudaDevAttrMultiProcessorCount, device);
    if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete b;
        return nullptr;
    }
    return b;
}

void msgpu_batch_destroy(msgpu_batch *b)
{
    if (!b) return;
    cudaSetDevice(b->device);
    cudaStreamSynchronize(b->stream);
    drop_graph(b);
    for (auto *list : {&b->sys, &b->spare})
        for (auto &s : *list) {
            Buf *all[] = {&s.rowptr, &s.col, &s.valf, &s.obs, &s.rates, &s.psi, &s.acc, &s.comp, &s.prev, &s.pflip};
            for (Buf *x : all) brelease(b, *x);
            if (s.ctx) msgpu_destroy(s.ctx);
        }
    Buf *all[] = {&b->sys_d, &b->items_d, &b->queue_d, &b->status_d, &b->scratch, &b->times_d, &b->backup};
    for (Buf *x : all) brelease(b, *x);
    cudaStreamDestroy(b->stream);
    delete b;
}

const char *msgpu_batch_last_error(const msgpu_batch *b) { return b ? b->err.c_str() : "null batch"; }

int msgpu_batch_clear(msgpu_batch *b)
{
    if (!b) return MSGPU_ERR_INVALID;
    cudaSetDevice(b->device);
    if (cudaStreamSynchronize(b->stream) != cudaSuccess) return bfail(b, MSGPU_ERR_CUDA, "batch: clear: stream failed");
    drop_graph(b);
    for (auto &s : b->sys) {
        if (s.ctx) {
            msgpu_destroy(s.ctx);  // a streamed system's context goes with it
            s.ctx = nullptr;
        } else {
            b->spare.push_back(s);
        }
    }
    b->sys.clear();
    b->tuned = 0;
    return MSGPU_OK;
}

int msgpu_batch_add_system(msgpu_batch *b, int dim, const int *rowptr, const int *col, const double *val,
                           double kappa, int stride1, int stride2, int nobs, const double *ops, const double *rates,
                           double st_rate, unsigned long long seed, int ntraj, const double *factors)
{
    if (!b) return -MSGPU_ERR_INVALID;
    if (dim < 4 || dim % 4 || !rowptr || !col || !val || ntraj <= 0 || !factors || nobs < 1 || nobs > 8 || !ops ||
        !rates || !std::isfinite(kappa) || !(st_rate >= 0.0))
        return -bfail(b, MSGPU_ERR_INVALID, "batch: invalid system arguments");
    const int hi = std::max(stride1, stride2), lo = std::min(stride1, stride2);
    if (lo <= 0 || hi == lo || hi % (2 * lo) || dim % (2 * hi))
        return -bfail(b, MSGPU_ERR_INVALID, "batch: electron strides do not belong to two spin-1/2 digits");
    cudaSetDevice(b->device);
    for (int k = 0; k < rowptr[dim]; ++k)
        if (col[k] < 0 || col[k] >= dim || !std::isfinite(val[2 * k]) || !std::isfinite(val[2 * k + 1]))
            return -bfail(b, MSGPU_ERR_INVALID, "batch: malformed Hamiltonian");
    if (dim >= kStreamDim) {
        // streamed single-system path: own context (charged to the batch budget)
        const size_t room = b->budget ? (b->budget > b->used ? b->budget - b->used : 1) : 0;
        msgpu_ctx *c = msgpu_create(b->device, room);
        if (!c) return -bfail(b, MSGPU_ERR_CUDA, "batch: cannot create a context for a large system");
        int rc = msgpu_upload_hamiltonian_csr(c, dim, rowptr, col, val);
        if (!rc) rc = msgpu_set_reaction_scalar(c, kappa);
        if (!rc) rc = msgpu_set_electron_pair(c, stride1, stride2);
        for (int o = 0; o < nobs && !rc; ++o) rc = msgpu_add_pair_observable(c, ops + 32 * static_cast<size_t>(o), rates[o]);
        if (!rc && st_rate > 0.0) rc = msgpu_set_st_noise(c, st_rate, MSGPU_NOISE_PHILOX, seed, nullptr, 0, 0);
        if (!rc) rc = msgpu_upload_factors(c, dim, ntraj, factors);
        if (rc) {
            const std::string why = msgpu_last_error(c);
            msgpu_destroy(c);
            return -bfail(b, rc, "batch: " + why);
        }
        BatchSystem s;
        s.D = dim;
        s.M = ntraj;
        s.nobs = nobs;
        s.s1 = std::max(stride1, stride2);
        s.s2 = std::min(stride1, stride2);
        s.kappa = kappa;
        s.st_rate = st_rate;
        s.seed = seed;
        s.ctx = c;
        b->sys.push_back(s);
        drop_graph(b);
        b->tuned = 0;
        return static_cast<int>(b->sys.size()) - 1;
    }
    BatchSystem s;
    if (!b->spare.empty()) {  // reuse a cleared system's buffers (upload keeps those large enough)
        s = b->spare.back();
        b->spare.pop_back();
    }
    s.D = dim;
    s.M = ntraj;
    s.nobs = nobs;
    s.s1 = hi;
    s.s2 = lo;
    s.kappa = kappa;
    s.st_rate = st_rate;
    s.seed = seed;
    const int nnz = rowptr[dim];
    std::vector<float> vf(2 * static_cast<size_t>(nnz));
    for (int k = 0; k < nnz; ++k) {
        if (col[k] < 0 || col[k] >= dim || !std::isfinite(val[2 * k]) || !std::isfinite(val[2 * k + 1]))
            return -bfail(b, MSGPU_ERR_INVALID, "batch: malformed Hamiltonian");
        vf[2 * k] = static_cast<float>(val[2 * k]);
        vf[2 * k + 1] = static_cast<float>(val[2 * k + 1]);
    }
    // observables in the kernel pair basis (first digit = larger stride)
    const bool swapped = stride1 < stride2;
    const int perm[4] = {0, 2, 1, 3};
    std::vector<double> op(static_cast<size_t>(nobs) * 32);
    for (int o = 0; o < nobs; ++o)
        for (int a = 0; a < 4; ++a)
            for (int c = 0; c < 4; ++c) {
                const int ua = swapped ? perm[a] : a, uc = swapped ? perm[c] : c;
                op[o * 32 + 2 * (a * 4 + c)] = ops[o * 32 + 2 * (ua * 4 + uc)];
                op[o * 32 + 2 * (a * 4 + c) + 1] = ops[o * 32 + 2 * (ua * 4 + uc) + 1];
            }
    std::vector<float> psi(2 * static_cast<size_t>(dim) * ntraj);
    for (size_t i = 0; i < psi.size(); ++i) psi[i] = static_cast<float>(factors[i]);
    std::vector<double> zeros(static_cast<size_t>(nobs) * ntraj, 0.0);
    int rc;
    if ((rc = upload(b, s.rowptr, rowptr, sizeof(int) * (dim + 1), "rowptr")) ||
        (rc = upload(b, s.col, col, sizeof(int) * std::max(1, nnz), "col")) ||
        (rc = upload(b, s.valf, vf.data(), sizeof(float) * std::max<size_t>(2, vf.size()), "values")) ||
        (rc = upload(b, s.obs, op.data(), sizeof(double) * op.size(), "observables")) ||
        (rc = upload(b, s.rates, rates, sizeof(double) * nobs, "rates")) ||
        (rc = upload(b, s.psi, psi.data(), sizeof(float) * psi.size(), "factors")) ||
        (rc = upload(b, s.acc, zeros.data(), sizeof(double) * zeros.size(), "acc")) ||
        (rc = upload(b, s.comp, zeros.data(), sizeof(double) * zeros.size(), "comp")) ||
        (rc = upload(b, s.prev, zeros.data(), sizeof(double) * zeros.size(), "prev"))) {
        b->spare.push_back(s);  // its buffers are freed with the batch
        return -rc;
    }
    if (cudaStreamSynchronize(b->stream) != cudaSuccess) {
        b->spare.push_back(s);
        return -bfail(b, MSGPU_ERR_CUDA, "batch: upload failed");
    }
    b->sys.push_back(s);
    drop_graph(b);
    b->tuned = 0;
    return static_cast<int>(b->sys.size()) - 1;
}

int msgpu_batch_tune(msgpu_batch *b, const double *times, int ntimes, int krylov_dim)
{
    if (!b) return MSGPU_ERR_INVALID;
    if (b->sys.empty() || !times || ntimes < 2 || krylov_dim < 1 || krylov_dim > kMaxKrylov)
        return bfail(b, MSGPU_ERR_INVALID, "batch: tune needs systems, >= 2 time points and krylov_dim in 1..32");
    cudaSetDevice(b->device);
    // back up every state, time a short run per candidate, restore
    size_t total = 0;
    for (auto &s : b->sys) total += s.psi.bytes;  // streamed systems hold no state here
    if (int rc = bensure(b, b->backup, total, "tuning backup")) return rc;
    size_t off = 0;
    for (auto &s : b->sys) {
        if (!s.psi.bytes) continue;
        cudaMemcpyAsync(static_cast<char *>(b->backup.p) + off, s.psi.p, s.psi.bytes, cudaMemcpyDeviceToDevice, b->stream);
        off += s.psi.bytes;
    }
    if (int rc = set_times(b, times, ntimes)) return rc;
    const int thresholds[] = {256, 512, 1024, 2048};
    const int cps[] = {1, 2, 3, 4};
    float best = 1e30f;
    for (int th : thresholds)
        for (int c : cps) {
            float ms = 0.f;
            if (int rc = run_once(b, ntimes, krylov_dim, 0, 0, th, c, false, &ms)) return rc;
            if (ms < best) {
                best = ms;
                b->threshold = th;
                b->ctas_per_sm = c;
            }
        }
    off = 0;
    for (auto &s : b->sys) {
        if (!s.psi.bytes) continue;
        cudaMemcpyAsync(s.psi.p, static_cast<char *>(b->backup.p) + off, s.psi.bytes, cudaMemcpyDeviceToDevice, b->stream);
        off += s.psi.bytes;
    }
    brelease(b, b->backup);
    if (cudaStreamSynchronize(b->stream) != cudaSuccess) return bfail(b, MSGPU_ERR_CUDA, "batch: restore failed");
    b->tuned = 1;
    drop_graph(b);
    return MSGPU_OK;
}

int msgpu_batch_run(msgpu_batch *b, const double *times, int ntimes, int krylov_dim, long long step_offset,
                    int accumulate)
{
    if (!b) return MSGPU_ERR_INVALID;
    if (b->sys.empty() || !times || ntimes < 1 || krylov_dim < 1 || krylov_dim > kMaxKrylov)
        return bfail(b, MSGPU_ERR_INVALID, "batch: run needs systems, time points and krylov_dim in 1..32");
    cudaSetDevice(b->device);
    if (int rc = set_times(b, times, ntimes)) return rc;
    b->m = krylov_dim;
    return run_once(b, ntimes, krylov_dim, accumulate, step_offset, b->threshold, b->ctas_per_sm, true, &b->last_ms,
                    times);
}

int msgpu_batch_fetch_yields(msgpu_batch *b, int system, double *per_traj, double *ensemble)
{
    if (!b) return MSGPU_ERR_INVALID;
    if (system < 0 || system >= static_cast<int>(b->sys.size())) return bfail(b, MSGPU_ERR_INVALID, "batch: no such system");
    BatchSystem &s = b->sys[system];
    if (s.ctx) {
        const int rc = msgpu_fetch_yields(s.ctx, per_traj, ensemble);
        return rc ? bfail(b, rc, std::string("batch: ") + msgpu_last_error(s.ctx)) : MSGPU_OK;
    }
    std::vector<double> acc(static_cast<size_t>(s.nobs) * s.M);
    if (cudaMemcpy(acc.data(), s.acc.p, sizeof(double) * acc.size(), cudaMemcpyDeviceToHost) != cudaSuccess)
        return bfail(b, MSGPU_ERR_CUDA, "batch: fetch failed");
    for (int o = 0; o < s.nobs; ++o) {
        double sum = 0.0;
        for (int t = 0; t < s.M; ++t) {
            const double v = acc[static_cast<size_t>(o) * s.M + t];
            if (per_traj) per_traj[static_cast<size_t>(t) * s.nobs + o] = v;
            sum += v;
        }
        if (ensemble) ensemble[o] = sum;
    }
    return MSGPU_OK;
}

long long msgpu_batch_launch_count(const msgpu_batch *b)
{
    if (!b) return 0;
    long long n = b->launches;
    for (const auto &s : b->sys)
        if (s.ctx) n += msgpu_launch_count(s.ctx);
    return n;
}

int msgpu_batch_system_info(const msgpu_batch *b, int i, int *streamed, int *variant, int *tile, int *groups)
{
    if (!b || i < 0 || i >= static_cast<int>(b->sys.size())) return MSGPU_ERR_INVALID;
    const BatchSystem &s = b->sys[i];
    if (streamed) *streamed = s.ctx ? 1 : 0;
    if (s.ctx) return msgpu_spmm_choice(s.ctx, variant, tile, groups);
    if (variant) *variant = -1;
    if (tile) *tile = -1;
    if (groups) *groups = -1;
    return MSGPU_OK;
}

int msgpu_batch_stats(const msgpu_batch *b, double *last_run_ms, int *team_threshold, int *ctas_per_sm)
{
    if (!b) return MSGPU_ERR_INVALID;
    if (last_run_ms) *last_run_ms = b->last_ms;
    if (team_threshold) *team_threshold = b->threshold;
    if (ctas_per_sm) *ctas_per_sm = b->ctas_per_sm;
    return MSGPU_OK;
}

}  // extern "C"
