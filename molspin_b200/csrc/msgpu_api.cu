// msgpu_api.cu -- C ABI of msgpu (include/msgpu.h): context, uploads and the
// host-side orchestration of the per-step kernel sequence.

#include "msgpu.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "msgpu_dense.h"
#include "msgpu_fused.cuh"
#include "msgpu_kernels.cuh"
#include "msgpu_resident.cuh"
#include "msgpu_spmm_tc.cuh"
#include "msgpu_spmm_tm.cuh"

using namespace msgpu;

namespace {

enum KClass {
    KC_APPLY = 0, KC_ORTH = 1, KC_REDUCE = 2, KC_EXPM = 3, KC_COMBINE = 4, KC_YIELD = 5, KC_GEMM = 6, KC_LANCZOS = 7,
    KC_N = 8
};
constexpr int kNumSimtVariants = 8;  // entries of kApplyVariants (checked there)
constexpr int kNumSpmmVariants = kNumSimtVariants + 3;  // + the tensor-core SpMM (cube bits 4, 3), the TMEM-staged one
constexpr int kTmVariant = kNumSimtVariants + 2;

struct DevBuf {
    void *p = nullptr;
    size_t bytes = 0;
};

}  // namespace

struct msgpu_ctx {
    int device = 0;
    size_t budget = 0;
    size_t used = 0;
    cudaStream_t own = nullptr, stream = nullptr;
    std::string err;
    long long launches = 0;

    // Hamiltonian
    int D = 0, nnz = 0;
    DevBuf hrow, hcol, hval, hhi, hlo;
    std::vector<int> h_rowptr, h_col;  // host copy for the quartet-block form
    std::vector<double> h_val;
    // quartet-block form of H for the current electron strides
    DevBuf qrow, qcolt, qval, qbase;
    DevBuf qval64;  // the quartet values in FP64 (complex128 Arnoldi apply)
    int q_s1 = 0, q_s2 = 0, q_D = 0, q_nblocks = 0;
    long long q_build = 0;            // counts quartet-form builds
    std::vector<int> q_hrow;          // host copies of the quartet form
    std::vector<int2> q_hblk;
    std::vector<float> q_hval;
    // cluster-resident complex64 Lanczos (k_lanczos_fused): descriptors for
    // cluster size f_C, built from quartet build f_build
    DevBuf fblk, fval, frow, fdsrc, fdiag;
    int f_C = 0, f_nblk_max = 0, f_opt = 0;  // f_opt: MSGPU_OPT_LANCZOS_CLUSTER
    bool f_dedup = false;
    long long f_build = -1;
    int f_probe_D = 0, f_probe_ldm = 0, f_probe_C = 0;  // cached cluster choice for (D, ldm, build)
    long long f_probe_build = -1;
    // complex64 streamed step in trajectory groups (MSGPU_OPT_TRAJ_GROUPS): one
    // group's SpMM overlaps the other's update and combine on a second stream
    int tgroups_opt = 0;  // 0 auto, else the number of groups asked for
    int combine_tile_opt = 0;  // MSGPU_OPT_COMBINE_TILE: quartets per evaluation tile (0: by dimension)
    cudaStream_t gside[3] = {nullptr, nullptr, nullptr};  // trajectory groups 1..3 (group 0: the context stream)
    cudaEvent_t gfork = nullptr, gjoin[3] = {nullptr, nullptr, nullptr};
    // H as a fixed-pattern linear combination of terms (msgpu_upload_hamiltonian_terms):
    // the host copy h_val then holds a generic combination (structure only)
    bool terms = false;
    int nterms = 0;
    DevBuf hterms, qsrc;   // nterms x nnz complex128; CSR index of every quartet value slot (-1: zero)
    size_t q_nslots = 0;
    std::array<double, 16> hcoef{};  // current coefficients
    // time-dependent H: coefficients per global step, evaluated by the caller
    // at each step's midpoint (sched_rows = 1: sched_steps x nterms) or at its
    // start and midpoint plus the last step's end (sched_rows = 2, the
    // dynamic RK4 layout: (2 sched_steps + 1) x nterms)
    std::vector<double> sched;
    long long sched_first = 0, sched_steps = 0;
    int sched_rows = 1;
    // tensor-core SpMM (k_lanczos_apply_tc): B-operand tables of the quartet
    // form, built when the quartet form has the nuclear-bit structure
    DevBuf tc_src, tc_tab;
    DevBuf tm_tab;             // block table of the TMEM-staged SpMM (k_tm_tables)
    int tc_P = 0, tc_entries = 0;
    CUtensorMap tc_map{};      // 2D map over the Krylov basis (boxes of 128 trajectories x TcCfg::HB rows)
    const void *tc_map_base = nullptr;
    long long tc_map_rows = 0;
    int tc_map_ldm = 0;
    CUtensorMap tm_map{};      // the same basis in boxes of 256 trajectories x 8 rows (k_lanczos_apply_tm)
    bool tm_map_ok = false;
    int sm_count = 0;          // SMs of the device (persistent SpMM grid)
    long long tc_build = -1;   // quartet build the tables were validated for
    bool tc_ok = false;        // structure present (tables valid)
    int q_tile = 0, q_tile_ldm = 0;  // autotuned quartets per CTA (and the ldm it was tuned for)
    int q_variant = 0;               // autotuned kernel variant (kApplyVariants)
    // resident (one warp per trajectory, whole time loop per launch) form
    int form = MSGPU_FORM_AUTO;
    DevBuf colbuf, trajval, times_d, pflip_d, sys_d, work_d, obs_d, dense_part;
    // dense tensor-core form
    msgpu::DenseState dense;
    std::vector<std::pair<void *, size_t>> dense_allocs;
    int dense_renorm = 1;
    // reaction
    bool k_scalar = true;
    // host copy of a CSR K (interleaved complex values): the complex64 Arnoldi form
    // checks on it that K acts on the electron pair only
    std::vector<int> k_hrow, k_hcol;
    std::vector<double> k_hval;
    double kappa = 0.0;
    double2 k_trace = {0.0, 0.0};  // trace of a CSR K
    double k_norm1 = 0.0;          // its 1-norm (max column sum)
    double taylor_tol = 0x1p-53;   // MSGPU_OPT_TAYLOR_TOL
    int spmm_variant = -1;         // MSGPU_OPT_SPMM_VARIANT (-1: autotuned)
    DevBuf krow, kcol, kval;
    // electron pair
    int s1 = 0, s2 = 0;
    bool pair_swapped = false;
    std::vector<std::array<double, 32>> obs;  // user basis, row-major 4x4 complex
    std::vector<double> rates;
    // noise
    int noise_mode = MSGPU_NOISE_NONE;
    double st_rate = 0.0;
    unsigned long long seed = 0;
    DevBuf bits;
    long long bits_steps = 0;
    int bits_ntraj = 0;
    // state
    int M = 0, ldm = 0;
    DevBuf psi128;       // ldm x D interleaved complex128 (plain form state)
    int state_prec = -1;  // precision holding the current state
    // workspace
    int ws_prec = -1, ws_m = 0;
    DevBuf basis, wbuf, zbuf, ubuf, part, part2, hess, tdiag, toff, coef, mdim, scale, alpha, beta0;
    DevBuf qpart_obs, qpart_nrm, prev, acc, comp, rates_d, status, values_d;
    int ntiles = 0, rows_per_tile = 0, qtiles = 0, quartets_per_tile = 0;
    // yields
    bool have_integrals = false;
    std::vector<double> last_values;
    int last_ntimes = 0;
    // profiling
    int prof = 0;                   // 0 off, 1 every launch, 2 sampled (see msgpu_profile_enable)
    long long prof_tick = -1;       // time step being issued (-1 outside the step loop)
    std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> ev;
    std::vector<cudaEvent_t> evpool;  // recycled timing events (creating two per timed launch stalls the host)
    double prof_ms[KC_N] = {0};
    long long prof_n[KC_N] = {0};
};

namespace {

int fail(msgpu_ctx *c, int code, const std::string &msg)
{
    if (c) c->err = msg;
    return code;
}

int cuda_fail(msgpu_ctx *c, cudaError_t e, const char *what)
{
    return fail(c, MSGPU_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

void release(msgpu_ctx *c, DevBuf &b)
{
    if (b.p) {
        cudaFree(b.p);
        c->used -= b.bytes;
    }
    b.p = nullptr;
    b.bytes = 0;
}

int ensure(msgpu_ctx *c, DevBuf &b, size_t bytes, const char *what)
{
    if (bytes == 0) bytes = 16;
    if (b.p && b.bytes >= bytes) return MSGPU_OK;
    release(c, b);
    if (c->budget && c->used + bytes > c->budget)
        return fail(c, MSGPU_ERR_BUDGET, std::string("device memory budget exceeded allocating ") + what + " (" +
                                             std::to_string(bytes) + " bytes, " + std::to_string(c->used) +
                                             " in use, budget " + std::to_string(c->budget) + ")");
    cudaError_t e = cudaMalloc(&b.p, bytes);
    if (e != cudaSuccess) {
        b.p = nullptr;
        return cuda_fail(c, e, what);
    }
    b.bytes = bytes;
    c->used += bytes;
    return MSGPU_OK;
}

int device_guard(msgpu_ctx *c)
{
    cudaError_t e = cudaSetDevice(c->device);
    if (e != cudaSuccess) return cuda_fail(c, e, "cudaSetDevice");
    return MSGPU_OK;
}

// Sampled profiling times every launch of every kProfileEvery-th time step
// of the streamed loop: an event between two kernels costs them their
// overlap, and a timed step also runs its trajectory groups back to back, so
// timing every launch slows the step by 10 % or more; one step in 32 costs
// about 1 %.  (The first launch of a class in a step is not representative:
// the first SpMM after the combine runs slower.)  The dense form times every
// kProfileEveryDense-th GEMM.
constexpr int kProfileEvery = 32;
constexpr int kProfileEveryDense = 8;

struct Timed {
    msgpu_ctx *c;
    int cls;
    cudaStream_t s;
    bool on = false;
    cudaEvent_t a = nullptr, b = nullptr;
    Timed(msgpu_ctx *c_, int cls_, cudaStream_t s_ = nullptr) : c(c_), cls(cls_), s(s_ ? s_ : c_->stream)
    {
        ++c->launches;
        if (c->prof == 1) {
            on = true;
        } else if (c->prof == 2 && c->prof_tick >= 0 && c->prof_tick % kProfileEvery == 0) {
            on = true;
        }
        if (!on) return;
        a = take();
        b = take();
        cudaEventRecord(a, s);
    }
    cudaEvent_t take()
    {
        cudaEvent_t e = nullptr;
        if (!c->evpool.empty()) {
            e = c->evpool.back();
            c->evpool.pop_back();
        } else {
            cudaEventCreate(&e);
        }
        return e;
    }
    ~Timed()
    {
        if (!on) return;
        cudaEventRecord(b, s);
        c->ev.push_back({cls, {a, b}});
    }
};

void collect_profile(msgpu_ctx *c)
{
    for (auto &e : c->ev) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e.second.first, e.second.second);
        c->prof_ms[e.first] += ms;
        c->prof_n[e.first] += 1;
        c->evpool.push_back(e.second.first);
        c->evpool.push_back(e.second.second);
    }
    c->ev.clear();
}

inline int ceil_div(long long a, long long b) { return static_cast<int>((a + b - 1) / b); }

// Trajectory groups of the complex64 streamed step (MSGPU_OPT_TRAJ_GROUPS).
// Each group is a multiple of 128 trajectories, the width of the widest SpMM
// variant's CTA; auto takes two groups from 512 trajectories up.
int traj_groups(const msgpu_ctx *c)
{
    const int want = c->tgroups_opt > 0 ? c->tgroups_opt : (c->ldm >= 512 ? 2 : 1);
    for (int g = want; g > 1; g /= 2)
        if (c->ldm % (128 * g) == 0) return g;
    return 1;
}

// Rows per tile: keep about 64-128 row tiles per trajectory tile so that the
// partial-sum buffers stay small and every SM has several CTAs.
int pick_rows_per_tile(int D)
{
    int R = D / 64;
    R = std::max(8, std::min(512, R));
    R = (R + 7) / 8 * 8;
    return R;
}

PairObs make_pair_obs(const msgpu_ctx *c)
{
    PairObs po;
    std::memset(&po, 0, sizeof(po));
    po.nobs = static_cast<int>(c->obs.size());
    // kernel pair basis index = 2*digit(stride s1) + digit(stride s2); when the
    // user's first electron has the smaller stride the roles swap (1 <-> 2).
    const int perm[4] = {0, 2, 1, 3};
    for (int o = 0; o < po.nobs; ++o)
        for (int a = 0; a < 4; ++a)
            for (int b = 0; b < 4; ++b) {
                const int ua = c->pair_swapped ? perm[a] : a, ub = c->pair_swapped ? perm[b] : b;
                po.op[o][a * 4 + b] = make_double2(c->obs[o][2 * (ua * 4 + ub)], c->obs[o][2 * (ua * 4 + ub) + 1]);
            }
    return po;
}

void dense_release_cb(void *ctx, void *p);  // defined with the dense form below
}  // namespace

extern "C" {

msgpu_ctx *msgpu_create(int device, size_t hbm_budget_bytes)
{
    auto *c = new msgpu_ctx();
    c->device = device;
    c->budget = hbm_budget_bytes;
    if (cudaSetDevice(device) != cudaSuccess) {
        delete c;
        return nullptr;
    }
    if (cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) c->sm_count = 0;
    if (cudaStreamCreateWithFlags(&c->own, cudaStreamNonBlocking) != cudaSuccess) {
        delete c;
        return nullptr;
    }
    c->stream = c->own;
    return c;
}

void msgpu_destroy(msgpu_ctx *c)
{
    if (!c) return;
    cudaSetDevice(c->device);
    cudaStreamSynchronize(c->stream);
    collect_profile(c);
    DevBuf *all[] = {&c->hrow, &c->hcol, &c->hval, &c->hhi, &c->hlo, &c->qrow, &c->qcolt, &c->qval, &c->qbase, &c->qval64,
                     &c->fblk, &c->fval, &c->frow, &c->fdsrc, &c->fdiag, &c->krow, &c->kcol, &c->kval, &c->bits,
                     &c->psi128, &c->basis, &c->wbuf, &c->zbuf, &c->ubuf, &c->part, &c->part2, &c->hess,
                     &c->tdiag, &c->toff, &c->coef, &c->mdim, &c->scale, &c->alpha, &c->beta0, &c->qpart_obs,
                     &c->qpart_nrm, &c->prev, &c->acc, &c->comp, &c->rates_d, &c->status, &c->values_d,
                     &c->colbuf, &c->trajval, &c->times_d, &c->pflip_d, &c->sys_d, &c->work_d, &c->obs_d,
                     &c->dense_part, &c->hterms, &c->qsrc, &c->tc_src, &c->tc_tab, &c->tm_tab};
    for (DevBuf *b : all) release(c, *b);
    msgpu::dense_release(c->dense, dense_release_cb, c);  // its stream and events, then its buffers
    for (cudaEvent_t e : c->evpool) cudaEventDestroy(e);
    if (c->gfork) cudaEventDestroy(c->gfork);
    for (int k = 0; k < 3; ++k) {
        if (c->gjoin[k]) cudaEventDestroy(c->gjoin[k]);
        if (c->gside[k]) cudaStreamDestroy(c->gside[k]);
    }
    for (auto &a : c->dense_allocs) cudaFree(a.first);
    if (c->own) cudaStreamDestroy(c->own);
    delete c;
}

const char *msgpu_last_error(const msgpu_ctx *c) { return c ? c->err.c_str() : "null context"; }

size_t msgpu_device_bytes(const msgpu_ctx *c) { return c ? c->used : 0; }

long long msgpu_launch_count(const msgpu_ctx *c) { return c ? c->launches : 0; }

int msgpu_set_option(msgpu_ctx *c, int key, double value)
{
    if (!c) return MSGPU_ERR_INVALID;
    if (key == MSGPU_OPT_DENSE_RENORMALIZE) {
        c->dense_renorm = value != 0.0;
        return MSGPU_OK;
    }
    if (key == MSGPU_OPT_SPMM_VARIANT) {
        const int v = static_cast<int>(value);
        if (v < -1 || v >= kNumSpmmVariants || v != value) return fail(c, MSGPU_ERR_INVALID, "SpMM variant out of range");
        c->spmm_variant = v;
        c->q_tile = 0;  // tune again among the allowed variants
        return MSGPU_OK;
    }
    if (key == MSGPU_OPT_TRAJ_GROUPS) {
        const int v = static_cast<int>(value);
        if (v != value || !(v == 0 || v == 1 || v == 2 || v == 4))
            return fail(c, MSGPU_ERR_INVALID, "trajectory groups must be 0 (auto), 1, 2 or 4");
        c->tgroups_opt = v;
        c->q_tile = 0;  // the variants that fit depend on a group's width
        return MSGPU_OK;
    }
    if (key == MSGPU_OPT_COMBINE_TILE) {
        const int v = static_cast<int>(value);
        if (v != value || v < 0 || v > 4096) return fail(c, MSGPU_ERR_INVALID, "combine tile must be 0..4096 quartets");
        c->combine_tile_opt = v;
        return MSGPU_OK;
    }
    if (key == MSGPU_OPT_LANCZOS_CLUSTER) {
        const int v = static_cast<int>(value);
        if (v != value || !(v == -1 || v == 0 || v == 1 || v == 2 || v == 4 || v == 8 || v == 16))
            return fail(c, MSGPU_ERR_INVALID, "Lanczos cluster size must be -1, 0, 1, 2, 4, 8 or 16");
        c->f_opt = v;
        c->f_probe_D = 0;  // choose again
        return MSGPU_OK;
    }
    if (key == MSGPU_OPT_TAYLOR_TOL) {
        if (!(value > 0.0 && value < 1.0)) return fail(c, MSGPU_ERR_INVALID, "Taylor tolerance must be in (0, 1)");
        c->taylor_tol = value;
        return MSGPU_OK;
    }
    return fail(c, MSGPU_ERR_INVALID, "unknown option");
}

int msgpu_get_option(msgpu_ctx *c, int key, double *value)
{
    if (!c || !value) return MSGPU_ERR_INVALID;
    switch (key) {
    case MSGPU_OPT_DENSE_RENORMALIZE: *value = c->dense_renorm; return MSGPU_OK;
    case MSGPU_OPT_TAYLOR_TOL: *value = c->taylor_tol; return MSGPU_OK;
    case MSGPU_OPT_SPMM_VARIANT: *value = c->spmm_variant; return MSGPU_OK;
    case MSGPU_OPT_LANCZOS_CLUSTER: *value = c->f_opt; return MSGPU_OK;
    case MSGPU_OPT_TRAJ_GROUPS: *value = c->ldm ? traj_groups(c) : c->tgroups_opt; return MSGPU_OK;
    case MSGPU_OPT_COMBINE_TILE: *value = c->combine_tile_opt; return MSGPU_OK;
    default: return fail(c, MSGPU_ERR_INVALID, "unknown option");
    }
}

int msgpu_set_form(msgpu_ctx *c, int form)
{
    if (!c) return MSGPU_ERR_INVALID;
    if (form < MSGPU_FORM_AUTO || form > MSGPU_FORM_RESIDENT) return fail(c, MSGPU_ERR_INVALID, "unknown form");
    c->form = form;
    return MSGPU_OK;
}

int msgpu_set_stream(msgpu_ctx *c, void *s)
{
    if (!c) return MSGPU_ERR_INVALID;
    c->stream = s ? static_cast<cudaStream_t>(s) : c->own;
    return MSGPU_OK;
}

int msgpu_upload_hamiltonian_csr(msgpu_ctx *c, int dim, const int *rowptr, const int *col, const double *val)
{
    if (!c) return MSGPU_ERR_INVALID;
    if (dim < 4 || !rowptr || !col || !val) return fail(c, MSGPU_ERR_INVALID, "Hamiltonian: dimension >= 4 and CSR arrays required");
    if (int rc = device_guard(c)) return rc;
    const int nnz = rowptr[dim];
    if (rowptr[0] != 0 || nnz < 0) return fail(c, MSGPU_ERR_INVALID, "Hamiltonian: malformed row pointer");
    for (int r = 0; r < dim; ++r)
        if (rowptr[r + 1] < rowptr[r]) return fail(c, MSGPU_ERR_INVALID, "Hamiltonian: row pointer not monotone");
    std::vector<float> hi(2 * static_cast<size_t>(nnz)), lo(2 * static_cast<size_t>(nnz));
    for (int k = 0; k < nnz; ++k) {
        if (col[k] < 0 || col[k] >= dim) return fail(c, MSGPU_ERR_INVALID, "Hamiltonian: column index out of range");
        for (int p = 0; p < 2; ++p) {
            const double v = val[2 * k + p];
            if (!std::isfinite(v)) return fail(c, MSGPU_ERR_NONFINITE, "Hamiltonian: non-finite value");
            const float h = static_cast<float>(v);
            hi[2 * k + p] = h;
            lo[2 * k + p] = static_cast<float>(v - static_cast<double>(h));
        }
    }
    if (c->D != 0 && c->D != dim) {
        // dimension change invalidates state and reaction operator
        c->state_prec = -1;
        c->M = 0;
        c->k_scalar = true;
    }
    int rc;
    if ((rc = ensure(c, c->hrow, sizeof(int) * (dim + 1), "H rowptr")) ||
        (rc = ensure(c, c->hcol, sizeof(int) * std::max(1, nnz), "H col")) ||
        (rc = ensure(c, c->hval, sizeof(double2) * std::max(1, nnz), "H val")) ||
        (rc = ensure(c, c->hhi, sizeof(float2) * std::max(1, nnz), "H hi")) ||
        (rc = ensure(c, c->hlo, sizeof(float2) * std::max(1, nnz), "H lo")))
        return rc;
    cudaError_t e;
    if ((e = cudaMemcpyAsync(c->hrow.p, rowptr, sizeof(int) * (dim + 1), cudaMemcpyHostToDevice, c->stream)) ||
        (e = cudaMemcpyAsync(c->hcol.p, col, sizeof(int) * nnz, cudaMemcpyHostToDevice, c->stream)) ||
        (e = cudaMemcpyAsync(c->hval.p, val, sizeof(double2) * nnz, cudaMemcpyHostToDevice, c->stream)) ||
        (e = cudaMemcpyAsync(c->hhi.p, hi.data(), sizeof(float2) * nnz, cudaMemcpyHostToDevice, c->stream)) ||
        (e = cudaMemcpyAsync(c->hlo.p, lo.data(), sizeof(float2) * nnz, cudaMemcpyHostToDevice, c->stream)))
        return cuda_fail(c, e, "Hamiltonian upload");
    if ((e = cudaStreamSynchronize(c->stream))) return cuda_fail(c, e, "Hamiltonian upload");
    c->D = dim;
    c->nnz = nnz;
    c->h_rowptr.assign(rowptr, rowptr + dim + 1);
    c->h_col.assign(col, col + nnz);
    c->h_val.assign(val, val + 2 * static_cast<size_t>(nnz));
    c->q_D = 0;  // quartet form must be rebuilt
    c->terms = false;
    c->dense.have_u = false;  // a cached dense propagator belongs to the old H
    return MSGPU_OK;
}

int msgpu_set_reaction_scalar(msgpu_ctx *c, double kappa)
{
    if (!c) return MSGPU_ERR_INVALID;
    if (!std::isfinite(kappa)) return fail(c, MSGPU_ERR_NONFINITE, "reaction: non-finite kappa");
    c->k_scalar = true;
    c->kappa = kappa;
    return MSGPU_OK;
}

int msgpu_upload_reaction_csr(msgpu_ctx *c, const int *rowptr, const int *col, const double *val)
{
    if (!c) return MSGPU_ERR_INVALID;
    if (c->D == 0) return fail(c, MSGPU_ERR_STATE, "reaction: upload the Hamiltonian first");
    if (!rowptr || !col || !val) return fail(c, MSGPU_ERR_INVALID, "reaction: CSR arrays required");
    if (int rc = device_guard(c)) return rc;
    const int D = c->D, nnz = rowptr[D];
    if (rowptr[0] != 0 || nnz < 0) return fail(c, MSGPU_ERR_INVALID, "reaction: malformed row pointer");
    for (int r = 0; r < D; ++r)
        if (rowptr[r + 1] < rowptr[r]) return fail(c, MSGPU_ERR_INVALID, "reaction: row pointer not monotone");
    for (int k = 0; k < nnz; ++k) {
        if (col[k] < 0 || col[k] >= D) return fail(c, MSGPU_ERR_INVALID, "reaction: column index out of range");
        if (!std::isfinite(val[2 * k]) || !std::isfinite(val[2 * k + 1]))
            return fail(c, MSGPU_ERR_NONFINITE, "reaction: non-finite value");
    }
    int rc;
    if ((rc = ensure(c, c->krow, sizeof(int) * (D + 1), "K rowptr")) ||
        (rc = ensure(c, c->kcol, sizeof(int) * std::max(1, nnz), "K col")) ||
        (rc = ensure(c, c->kval, sizeof(double2) * std::max(1, nnz), "K val")))
        return rc;
    cudaError_t e;
    if ((e = cudaMemcpyAsync(c->krow.p, rowptr, sizeof(int) * (D + 1), cudaMemcpyHostToDevice, c->stream)) ||
        (e = cudaMemcpyAsync(c->kcol.p, col, sizeof(int) * nnz, cudaMemcpyHostToDevice, c->stream)) ||
        (e = cudaMemcpyAsync(c->kval.p, val, sizeof(double2) * nnz, cudaMemcpyHostToDevice, c->stream)) ||
        (e = cudaStreamSynchronize(c->stream)))
        return cuda_fail(c, e, "reaction upload");
    c->k_scalar = false;
    c->k_hrow.assign(rowptr, rowptr + D + 1);
    c->k_hcol.assign(col, col + nnz);
    c->k_hval.assign(val, val + 2 * static_cast<size_t>(nnz));
    // trace and 1-norm (max column sum) for the Taylor propagator's shift and sub-steps
    std::vector<double> colsum(D, 0.0);
    c->k_trace = make_double2(0.0, 0.0);
    for (int r = 0; r < D; ++r)
        for (int k = rowptr[r]; k < rowptr[r + 1]; ++k) {
            colsum[col[k]] += std::hypot(val[2 * k], val[2 * k + 1]);
            if (col[k] == r) {
                c->k_trace.x += val[2 * k];
                c->k_trace.y += val[2 * k + 1];
            }
        }
    c->k_norm1 = colsum.empty() ? 0.0 : *std::max_element(colsum.begin(), colsum.end());
    return MSGPU_OK;
}

int msgpu_set_electron_pair(msgpu_ctx *c, int stride1, int stride2)
{
    if (!c) return MSGPU_ERR_INVALID;
    if (stride1 <= 0 || stride2 <= 0 || stride1 == stride2)
        return fail(c, MSGPU_ERR_INVALID, "electron pair: two distinct positive strides required");
    const int hi = std::max(stride1, stride2), lo = std::min(stride1, stride2);
    if (hi % (2 * lo) != 0)
        return fail(c, MSGPU_ERR_INVALID, "electron pair: strides must belong to two spin-1/2 digits of the product basis");
    if (c->D && (c->D % (2 * hi) != 0))
        return fail(c, MSGPU_ERR_INVALID, "electron pair: strides inconsistent with the Hilbert dimension");
    c->s1 = hi;
    c->s2 = lo;
    c->pair_swapped = stride1 < stride2;
    return MSGPU_OK;
}

int msgpu_clear_observables(msgpu_ctx *c)
{
    if (!c) return MSGPU_ERR_INVALID;
    c->obs.clear();
    c->rates.clear();
    c->have_integrals = false;
    return MSGPU_OK;
}

int msgpu_add_pair_observable(msgpu_ctx *c, const double *op, double rate)
{
    if (!c) return MSGPU_ERR_INVALID;
    if (!op || !std::isfinite(rate)) return fail(c, MSGPU_ERR_INVALID, "observable: operator and finite rate required");
    if (c->obs.size() >= 8) return fail(c, MSGPU_ERR_INVALID, "observable: at most 8 pair observables");
    std::array<double, 32> a;
    for (int i = 0; i < 32; ++i) {
        if (!std::isfinite(op[i])) return fail(c, MSGPU_ERR_NONFINITE, "observable: non-finite entry");
        a[i] = op[i];
    }
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) {
            const double dr = a[2 * (i * 4 + j)] - a[2 * (j * 4 + i)];
            const double di = a[2 * (i * 4 + j) + 1] + a[2 * (j * 4 + i) + 1];
            if (std::abs(dr) > 1e-12 || std::abs(di) > 1e-12)
                return fail(c, MSGPU_ERR_INVALID, "observable: operator must be Hermitian");
        }
    c->obs.push_back(a);
    c->rates.push_back(rate);
    c->have_integrals = false;
    return MSGPU_OK;
}

int msgpu_set_st_noise(msgpu_ctx *c, double st_rate, int mode, unsigned long long seed, const unsigned char *bits,
                       long long nsteps, int ntraj)
{
    if (!c) return MSGPU_ERR_INVALID;
    if (!std::isfinite(st_rate) || st_rate < 0.0) return fail(c, MSGPU_ERR_INVALID, "noise: rate must be finite and >= 0");
    if (mode < MSGPU_NOISE_NONE || mode > MSGPU_NOISE_PHILOX) return fail(c, MSGPU_ERR_INVALID, "noise: unknown mode");
    if (int rc = device_guard(c)) return rc;
    c->noise_mode = (st_rate > 0.0) ? mode : MSGPU_NOISE_NONE;
    c->st_rate = st_rate;
    c->seed = seed;
    if (c->noise_mode == MSGPU_NOISE_REPLAY) {
        if (!bits || nsteps <= 0 || ntraj <= 0) return fail(c, MSGPU_ERR_INVALID, "noise: replay bits required");
        const size_t bytes = static_cast<size_t>((nsteps * 2 * ntraj + 7) / 8);
        if (int rc = ensure(c, c->bits, bytes, "noise bits")) return rc;
        cudaError_t e;
        if ((e = cudaMemcpyAsync(c->bits.p, bits, bytes, cudaMemcpyHostToDevice, c->stream)) ||
            (e = cudaStreamSynchronize(c->stream)))
            return cuda_fail(c, e, "noise bits upload");
        c->bits_steps = nsteps;
        c->bits_ntraj = ntraj;
    }
    return MSGPU_OK;
}

}  // extern "C"

namespace msgpu {
namespace {  // internal linkage, beside the other kernels

// H = sum_k coef_k H_k on the common CSR pattern: complex128 values and
// their FP32 hi/lo split; bit 2 of status on a non-finite value.
struct TermCoef {
    double c[16];
};

__global__ void k_combine_terms(const double2 *__restrict__ terms, int nterms, TermCoef cf, int nnz,
                                double2 *__restrict__ val, float2 *__restrict__ hi, float2 *__restrict__ lo,
                                int *__restrict__ status)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nnz) return;
    double2 v = make_double2(0.0, 0.0);
    for (int t = 0; t < nterms; ++t) {
        const double2 x = terms[static_cast<size_t>(t) * nnz + k];
        v.x += cf.c[t] * x.x;
        v.y += cf.c[t] * x.y;
    }
    if (!isfinite(v.x) || !isfinite(v.y)) atomicOr(status, 2);
    val[k] = v;
    const float2 h = make_float2(static_cast<float>(v.x), static_cast<float>(v.y));
    hi[k] = h;
    lo[k] = make_float2(static_cast<float>(v.x - static_cast<double>(h.x)),
                        static_cast<float>(v.y - static_cast<double>(h.y)));
}

// quartet value slot s (two FP32 per complex value, and its FP64 copy) <- the
// CSR value it came from
__global__ void k_quartet_refresh(const int *__restrict__ src, size_t nslots, const double2 *__restrict__ val,
                                  float2 *__restrict__ qval, double2 *__restrict__ qval64)
{
    const size_t s = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (s >= nslots) return;
    const int k = src[s];
    const double2 v = k >= 0 ? val[k] : make_double2(0.0, 0.0);
    qval[s] = make_float2(static_cast<float>(v.x), static_cast<float>(v.y));
    qval64[s] = v;
}

}  // namespace
}  // namespace msgpu

namespace {

int upload_factors_impl(msgpu_ctx *c, int dim, int ntraj, const void *src, cudaMemcpyKind kind)
{
    if (!c) return MSGPU_ERR_INVALID;
    if (c->D == 0) return fail(c, MSGPU_ERR_STATE, "factors: upload the Hamiltonian first");
    if (dim != c->D) return fail(c, MSGPU_ERR_INVALID, "factors: dimension differs from the Hamiltonian");
    if (ntraj <= 0 || !src) return fail(c, MSGPU_ERR_INVALID, "factors: at least one trajectory required");
    if (int rc = device_guard(c)) return rc;
    const int ldm = (ntraj + 63) / 64 * 64;
    const size_t n = static_cast<size_t>(dim) * ldm;
    if (int rc = ensure(c, c->psi128, n * sizeof(double2), "state")) return rc;
    // staging copy in column-major order, then a tiled transpose on the device;
    // the staging area is the Krylov workspace when it is large enough.
    const size_t sbytes = static_cast<size_t>(dim) * ntraj * sizeof(double2);
    if (int rc = ensure(c, c->zbuf, sbytes, "upload staging")) return rc;
    cudaError_t e = cudaMemcpyAsync(c->zbuf.p, src, sbytes, kind, c->stream);
    if (e) return cuda_fail(c, e, "factors upload");
    dim3 grid(ceil_div(dim, 32), ldm / 32), block(32, 8);
    {
        Timed tm(c, KC_COMBINE);
        k_cols_to_interleaved<double2><<<grid, block, 0, c->stream>>>(static_cast<double2 *>(c->psi128.p),
                                                                      static_cast<const double2 *>(c->zbuf.p), dim,
                                                                      ntraj, ldm);
    }
    if ((e = cudaGetLastError())) return cuda_fail(c, e, "factors transpose");
    if ((e = cudaStreamSynchronize(c->stream))) return cuda_fail(c, e, "factors upload");
    if (c->M != ntraj) c->ws_prec = -1;
    c->M = ntraj;
    c->ldm = ldm;
    c->state_prec = MSGPU_PREC_C128;
    c->have_integrals = false;
    return MSGPU_OK;
}

// Workspace for (precision, Krylov dimension m) at the current (D, ldm).
int ensure_workspace(msgpu_ctx *c, int prec, int m)
{
    const int D = c->D, ldm = c->ldm, nobs = std::max<int>(1, static_cast<int>(c->obs.size()));
    const size_t n = static_cast<size_t>(D) * ldm;
    c->rows_per_tile = pick_rows_per_tile(D);
    c->ntiles = ceil_div(D, c->rows_per_tile);
    const int Q = D / 4;
    c->quartets_per_tile = c->combine_tile_opt > 0 ? std::min(c->combine_tile_opt, Q)
                                                   : std::max(8, std::min(256, Q / 64));
    c->qtiles = ceil_div(Q, c->quartets_per_tile);
    int rc;
    if (prec == MSGPU_PREC_C128) {
        // basis V_0..V_{m-1}; W/Z ping-pong
        if ((rc = ensure(c, c->basis, n * m * sizeof(double2), "Krylov basis")) ||
            (rc = ensure(c, c->wbuf, n * sizeof(double2), "Krylov W")) ||
            (rc = ensure(c, c->zbuf, n * sizeof(double2), "Krylov Z")) ||
            (rc = ensure(c, c->part, static_cast<size_t>(c->ntiles) * (m + 1) * ldm * sizeof(double2), "partials")) ||
            (rc = ensure(c, c->part2, static_cast<size_t>(3) * (m + 1) * ldm * sizeof(double2), "dots")) ||
            (rc = ensure(c, c->hess, static_cast<size_t>(ldm) * m * m * sizeof(double2), "Hessenberg")))
            return rc;
    } else {
        // w_0 (= state) .. w_m, and U
        if ((rc = ensure(c, c->basis, n * (m + 1) * sizeof(float2), "Lanczos basis")) ||
            (rc = ensure(c, c->ubuf, n * sizeof(float2), "Lanczos U")) ||
            (rc = ensure(c, c->part, static_cast<size_t>(std::max(c->ntiles, ceil_div(Q, 8))) * ldm * sizeof(double),
                         "partials")) ||
            (rc = ensure(c, c->tdiag, static_cast<size_t>(ldm) * m * sizeof(double), "T diagonal")) ||
            (rc = ensure(c, c->toff, static_cast<size_t>(ldm) * m * sizeof(double), "T offdiagonal")) ||
            (rc = ensure(c, c->alpha, static_cast<size_t>(ldm) * sizeof(double), "alpha")))
            return rc;
    }
    if ((rc = ensure(c, c->coef, static_cast<size_t>(ldm) * m * sizeof(double2), "coefficients")) ||
        (rc = ensure(c, c->mdim, static_cast<size_t>(ldm) * sizeof(int), "Krylov dims")) ||
        (rc = ensure(c, c->scale, static_cast<size_t>(ldm) * (m + 1) * sizeof(double), "scales")) ||
        (rc = ensure(c, c->beta0, static_cast<size_t>(ldm) * sizeof(double), "beta0")) ||
        (rc = ensure(c, c->qpart_obs, static_cast<size_t>(c->qtiles) * nobs * ldm * sizeof(double), "obs partials")) ||
        (rc = ensure(c, c->qpart_nrm, static_cast<size_t>(c->qtiles) * ldm * sizeof(double), "norm partials")) ||
        (rc = ensure(c, c->prev, static_cast<size_t>(nobs) * ldm * sizeof(double), "yield prev")) ||
        (rc = ensure(c, c->acc, static_cast<size_t>(nobs) * ldm * sizeof(double), "yield acc")) ||
        (rc = ensure(c, c->comp, static_cast<size_t>(nobs) * ldm * sizeof(double), "yield comp")) ||
        (rc = ensure(c, c->rates_d, 8 * sizeof(double), "rates")) ||
        (rc = ensure(c, c->status, sizeof(int), "status")))
        return rc;
    c->ws_prec = prec;
    c->ws_m = m;
    return MSGPU_OK;
}

// Bring the state into the precision of the run.  The complex64 state lives
// in slot 0 of the Lanczos basis.
int ensure_state(msgpu_ctx *c, int prec)
{
    if (c->state_prec == prec) return MSGPU_OK;
    const size_t npairs = static_cast<size_t>(c->D) * c->ldm / 2;
    const int threads = 256;
    const int blocks = ceil_div(static_cast<long long>(npairs), threads);
    if (prec == MSGPU_PREC_C64 && c->state_prec == MSGPU_PREC_C128) {
        Timed tm(c, KC_COMBINE);
        k_c128_to_pp<<<blocks, threads, 0, c->stream>>>(static_cast<float4 *>(c->basis.p),
                                                         static_cast<const double2 *>(c->psi128.p), npairs);
    } else if (prec == MSGPU_PREC_C128 && c->state_prec == MSGPU_PREC_C64) {
        // msgpu_run parks the complex64 state here before the basis buffer is
        // reused or reallocated
        Timed tm(c, KC_COMBINE);
        k_pp_to_c128<<<blocks, threads, 0, c->stream>>>(static_cast<double2 *>(c->psi128.p),
                                                         static_cast<const float4 *>(c->basis.p), npairs);
    } else {
        return fail(c, MSGPU_ERR_STATE, "no trajectory state uploaded");
    }
    cudaError_t e = cudaGetLastError();
    if (e) return cuda_fail(c, e, "state conversion");
    c->state_prec = prec;
    return MSGPU_OK;
}

double flip_p(double st_rate, double h) { return -0.5 * std::expm1(-2.0 * (0.5 * st_rate) * h); }

// Device allocations of the dense form, charged to the context's budget.
int dense_alloc_cb(void *ctx, void **p, size_t bytes, const char *what)
{
    auto *c = static_cast<msgpu_ctx *>(ctx);
    if (c->budget && c->used + bytes > c->budget)
        return fail(c, MSGPU_ERR_BUDGET, std::string("device memory budget exceeded allocating ") + what);
    cudaError_t e = cudaMalloc(p, bytes);
    if (e != cudaSuccess) {
        *p = nullptr;
        return cuda_fail(c, e, what);
    }
    c->used += bytes;
    c->dense_allocs.push_back({*p, bytes});
    return MSGPU_OK;
}

void dense_release_cb(void *ctx, void *p)
{
    auto *c = static_cast<msgpu_ctx *>(ctx);
    if (!p) return;
    for (size_t i = 0; i < c->dense_allocs.size(); ++i)
        if (c->dense_allocs[i].first == p) {
            cudaFree(p);
            c->used -= c->dense_allocs[i].second;
            c->dense_allocs.erase(c->dense_allocs.begin() + i);
            return;
        }
}

int run_dense(msgpu_ctx *c, const msgpu_run_params *p)
{
    const int D = c->D, ldm = c->ldm, M = c->M;
    const int nobs = static_cast<int>(c->obs.size());
    cudaStream_t st = c->stream;
    int rc;
    if ((rc = ensure_state(c, MSGPU_PREC_C128)) ||
        (rc = ensure(c, c->acc, static_cast<size_t>(nobs) * ldm * sizeof(double), "yield acc")) ||
        (rc = ensure(c, c->comp, static_cast<size_t>(nobs) * ldm * sizeof(double), "yield comp")) ||
        (rc = ensure(c, c->prev, static_cast<size_t>(nobs) * ldm * sizeof(double), "yield prev")) ||
        (rc = ensure(c, c->rates_d, 8 * sizeof(double), "rates")) ||
        (rc = ensure(c, c->status, sizeof(int), "status")) ||
        (rc = ensure(c, c->values_d, static_cast<size_t>(p->ntimes) * nobs * sizeof(double), "values")) ||
        (rc = ensure(c, c->obs_d, 8 * 16 * sizeof(double2), "observables")) ||
        (rc = ensure(c, c->dense_part, 2 * static_cast<size_t>(p->ntimes) * nobs * sizeof(double), "dense values")))
        return rc;
    const PairObs po = make_pair_obs(c);
    cudaError_t e;
    if ((e = cudaMemcpyAsync(c->rates_d.p, c->rates.data(), nobs * sizeof(double), cudaMemcpyHostToDevice, st)) ||
        (e = cudaMemcpyAsync(c->obs_d.p, po.op, sizeof(double2) * 16 * nobs, cudaMemcpyHostToDevice, st)) ||
        (e = cudaMemsetAsync(c->status.p, 0, sizeof(int), st)))
        return cuda_fail(c, e, "dense setup");
    if (!p->accumulate) {
        if ((e = cudaMemsetAsync(c->acc.p, 0, static_cast<size_t>(nobs) * ldm * sizeof(double), st)) ||
            (e = cudaMemsetAsync(c->comp.p, 0, static_cast<size_t>(nobs) * ldm * sizeof(double), st)))
            return cuda_fail(c, e, "dense setup");
    }
    msgpu::DenseRun run;
    std::memset(&run, 0, sizeof(run));
    run.rowptr = static_cast<const int *>(c->hrow.p);
    run.col = static_cast<const int *>(c->hcol.p);
    run.val = static_cast<const double *>(c->hval.p);
    if (!c->k_scalar) {
        run.krow = static_cast<const int *>(c->krow.p);
        run.kcol = static_cast<const int *>(c->kcol.p);
        run.kval = static_cast<const double *>(c->kval.p);
    }
    run.kappa = c->k_scalar ? c->kappa : 0.0;
    run.s1 = c->s1;
    run.s2 = c->s2;
    run.nobs = nobs;
    run.obs = static_cast<const double *>(c->obs_d.p);
    run.obs_host = reinterpret_cast<const double *>(po.op);
    run.rates = static_cast<const double *>(c->rates_d.p);
    run.noise_mode = c->noise_mode;
    run.bits = static_cast<const unsigned char *>(c->bits.p);
    run.bits_steps = c->bits_steps;
    run.bits_ntraj = c->bits_ntraj;
    run.seed = c->seed;
    run.acc = static_cast<double *>(c->acc.p);
    run.comp = static_cast<double *>(c->comp.p);
    run.prev = static_cast<double *>(c->prev.p);
    run.acc_ld = ldm;
    run.values = static_cast<double *>(c->values_d.p);
    run.times = p->times;
    run.ntimes = p->ntimes;
    run.step_offset = p->step_offset;
    run.accumulate = p->accumulate;
    run.st_rate = c->st_rate;
    run.renormalize = c->dense_renorm;
    run.status = static_cast<int *>(c->status.p);
    run.part = static_cast<double *>(c->dense_part.p);
    const int parts = p->precision == MSGPU_PREC_INT8X4 ? 4 : p->precision == MSGPU_PREC_BF16X6 ? 3 : 2;
    const double dt = p->ntimes > 1 ? p->times[1] - p->times[0] : 1.0;
    for (int s = 1; s + 1 < p->ntimes; ++s)
        if (std::abs((p->times[s + 1] - p->times[s]) - dt) > 1e-12 * std::abs(dt))
            return fail(c, MSGPU_ERR_INVALID, "run: the dense propagator needs a uniform time step");
    std::string err;
    if (c->dense.psi && (c->dense.D != D || c->dense.M != M || c->dense.parts != parts))
        msgpu::dense_release(c->dense, dense_release_cb, c);  // shape changed: rebuild
    if ((rc = msgpu::dense_prepare(c->dense, D, M, ldm, parts, dt, run, c->psi128.p, st, err, dense_alloc_cb, c)))
        return err.empty() ? rc : fail(c, rc, err);
    float gemm_ms = 0.f;
    long long gemm_n = 0;
    c->launches += 2LL * (p->ntimes - 1) + 4;  // GEMM + epilogue per step; first epilogue, last values, two layout copies
    if ((rc = msgpu::dense_run(c->dense, run, c->psi128.p, ldm, st, err, c->prof ? &gemm_ms : nullptr, &gemm_n,
                               c->prof == 2 ? kProfileEveryDense : 1)))
        return fail(c, rc, err);
    if (c->prof) {
        c->prof_ms[KC_GEMM] += gemm_ms;
        c->prof_n[KC_GEMM] += gemm_n;
    }
    int status = 0;
    c->last_values.assign(static_cast<size_t>(p->ntimes) * nobs, 0.0);
    if ((e = cudaMemcpyAsync(&status, c->status.p, sizeof(int), cudaMemcpyDeviceToHost, st)) ||
        (e = cudaMemcpyAsync(c->last_values.data(), c->values_d.p, c->last_values.size() * sizeof(double),
                             cudaMemcpyDeviceToHost, st)) ||
        (e = cudaStreamSynchronize(st)))
        return cuda_fail(c, e, "dense run");
    c->state_prec = MSGPU_PREC_C128;
    c->last_ntimes = p->ntimes;
    c->have_integrals = true;
    if (status & 4) return fail(c, MSGPU_ERR_CUDA, "run: dense GEMM pipeline timed out (bounded wait expired)");
    if (status & 2) return fail(c, MSGPU_ERR_NONFINITE, "run: non-finite observable or norm on the device");
    return MSGPU_OK;
}

// Warps per CTA of the resident form for this problem, 0 if it does not
// apply (streamed form forced, dimension too large for the shared-memory
// basis, Lanczos asked for with a non-scalar K).
constexpr size_t kResidentSmemBudget = 200 * 1024;
constexpr int kResidentMaxDim = 1024;

int resident_warps(const msgpu_ctx *c, int prec, int m)
{
    if (c->form == MSGPU_FORM_STREAMED || c->sched_steps) return 0;  // a schedule changes H between launches
    if (prec == MSGPU_PREC_C64 && !c->k_scalar) return 0;
    if (c->form == MSGPU_FORM_AUTO && c->D > kResidentMaxDim) return 0;
    const size_t wb = resident_warp_bytes(c->D, m, prec == MSGPU_PREC_C128 ? 16 : 8);
    // Warps never wait on one another, so a CTA's warp count only places them:
    // while the block has fewer trajectories than 4 per SM, fewer warps per
    // CTA spread them over more SMs (cfg1, 256 trajectories: 1.26M -> 1.41M
    // traj-steps/s in complex128 with one warp per CTA instead of four).
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device) != cudaSuccess || sms < 1) sms = 1;
    const int spread = std::max(1, c->M / sms);
    const int w = static_cast<int>(std::min<size_t>(std::min(4, spread), kResidentSmemBudget / wb));
    return w;
}

// K as I (x) K4 on the electron pair (the 4 x 4 block in the pair index
// a = 2 a1 + a2, a1 the digit of stride s1): true when every quartet's rows
// couple only to the same quartet, with the same block (to 1e-12 of the
// largest entry).  A scalar K is kappa I.
bool pair_reaction(const msgpu_ctx *c, PairK *out)
{
    for (int i = 0; i < 16; ++i) out->k[i] = make_double2(0.0, 0.0);
    if (c->k_scalar) {
        for (int a = 0; a < 4; ++a) out->k[5 * a] = make_double2(c->kappa, 0.0);
        return true;
    }
    const int D = c->D, s1 = c->s1, s2 = c->s2;
    if (static_cast<int>(c->k_hrow.size()) != D + 1 || s1 <= 0 || s2 <= 0) return false;
    double kmax = 0.0;
    for (size_t k = 0; k < c->k_hcol.size(); ++k) kmax = std::max(kmax, std::hypot(c->k_hval[2 * k], c->k_hval[2 * k + 1]));
    const double tol = 1e-12 * kmax;
    bool have[4] = {false, false, false, false};
    for (int r = 0; r < D; ++r) {
        const int a1 = (r / s1) & 1, a2 = (r / s2) & 1, a = 2 * a1 + a2;
        const int base = r - a1 * s1 - a2 * s2;
        double row[4][2] = {{0, 0}, {0, 0}, {0, 0}, {0, 0}};
        for (int k = c->k_hrow[r]; k < c->k_hrow[r + 1]; ++k) {
            const int col = c->k_hcol[k];
            const int b1 = (col / s1) & 1, b2 = (col / s2) & 1;
            if (col - b1 * s1 - b2 * s2 != base) return false;  // leaves the quartet
            row[2 * b1 + b2][0] += c->k_hval[2 * static_cast<size_t>(k)];
            row[2 * b1 + b2][1] += c->k_hval[2 * static_cast<size_t>(k) + 1];
        }
        for (int b = 0; b < 4; ++b) {
            double2 &kk = out->k[4 * a + b];
            if (!have[a]) kk = make_double2(row[b][0], row[b][1]);
            else if (std::abs(kk.x - row[b][0]) > tol || std::abs(kk.y - row[b][1]) > tol) return false;
        }
        have[a] = true;
    }
    return true;
}

int run_resident(msgpu_ctx *c, const msgpu_run_params *p, int prec, int m)
{
    const int D = c->D, ldm = c->ldm, M = c->M;
    const int nobs = static_cast<int>(c->obs.size());
    const int warps = resident_warps(c, prec, m);
    const size_t wb = resident_warp_bytes(D, m, prec == MSGPU_PREC_C128 ? 16 : 8);
    cudaStream_t st = c->stream;
    int rc;
    if ((rc = ensure_state(c, MSGPU_PREC_C128)) ||
        (rc = ensure(c, c->colbuf, static_cast<size_t>(D) * M * sizeof(double2), "resident state")) ||
        (rc = ensure(c, c->acc, static_cast<size_t>(nobs) * ldm * sizeof(double), "yield acc")) ||
        (rc = ensure(c, c->comp, static_cast<size_t>(nobs) * ldm * sizeof(double), "yield comp")) ||
        (rc = ensure(c, c->prev, static_cast<size_t>(nobs) * ldm * sizeof(double), "yield prev")) ||
        (rc = ensure(c, c->rates_d, 8 * sizeof(double), "rates")) ||
        (rc = ensure(c, c->status, sizeof(int), "status")) ||
        (rc = ensure(c, c->values_d, static_cast<size_t>(p->ntimes) * nobs * sizeof(double), "values")) ||
        (rc = ensure(c, c->trajval, static_cast<size_t>(p->ntimes) * M * nobs * sizeof(double), "values per trajectory")) ||
        (rc = ensure(c, c->times_d, static_cast<size_t>(p->ntimes) * sizeof(double), "times")) ||
        (rc = ensure(c, c->pflip_d, static_cast<size_t>(p->ntimes) * sizeof(double), "flip probabilities")) ||
        (rc = ensure(c, c->sys_d, sizeof(ResidentSystem), "system")) ||
        (rc = ensure(c, c->work_d, static_cast<size_t>(M) * sizeof(ResidentWork), "work list")) ||
        (rc = ensure(c, c->obs_d, 8 * 16 * sizeof(double2), "observables")))
        return rc;
    // flip probabilities and observables in the kernel's pair basis
    std::vector<double> pf(p->ntimes, 0.0);
    for (int s = 0; s + 1 < p->ntimes; ++s) pf[s] = flip_p(c->st_rate, 0.5 * (p->times[s + 1] - p->times[s]));
    const PairObs po = make_pair_obs(c);
    std::vector<ResidentWork> work(M);
    for (int t = 0; t < M; ++t) work[t] = ResidentWork{0, t};
    ResidentSystem S;
    std::memset(&S, 0, sizeof(S));
    S.rowptr = static_cast<const int *>(c->hrow.p);
    S.col = static_cast<const int *>(c->hcol.p);
    S.val = static_cast<const double2 *>(c->hval.p);
    S.valf = static_cast<const float2 *>(c->hhi.p);
    if (!c->k_scalar) {
        S.krow = static_cast<const int *>(c->krow.p);
        S.kcol = static_cast<const int *>(c->kcol.p);
        S.kval = static_cast<const double2 *>(c->kval.p);
    }
    S.kappa = c->k_scalar ? c->kappa : 0.0;
    S.D = D;
    S.M = M;
    S.acc_ld = ldm;  // acc/comp/prev share the streamed layout [nobs][ldm]
    S.m = m;
    S.s1 = c->s1;
    S.s2 = c->s2;
    S.nobs = nobs;
    S.obs = static_cast<const double2 *>(c->obs_d.p);
    S.rates = static_cast<const double *>(c->rates_d.p);
    S.nz.mode = c->noise_mode;
    S.nz.bits = static_cast<const uint8_t *>(c->bits.p);
    S.nz.bits_steps = c->bits_steps;
    S.nz.M = c->noise_mode == MSGPU_NOISE_REPLAY ? c->bits_ntraj : M;
    S.nz.seed = c->seed;
    S.psi = c->colbuf.p;
    S.acc = static_cast<double *>(c->acc.p);
    S.comp = static_cast<double *>(c->comp.p);
    S.prev = static_cast<double *>(c->prev.p);
    S.traj_values = static_cast<double *>(c->trajval.p);
    S.times = static_cast<const double *>(c->times_d.p);
    S.pflip = static_cast<const double *>(c->pflip_d.p);
    S.ntimes = p->ntimes;
    S.step_offset = p->step_offset;
    S.accumulate = p->accumulate;
    cudaError_t e;
    if ((e = cudaMemcpyAsync(c->rates_d.p, c->rates.data(), nobs * sizeof(double), cudaMemcpyHostToDevice, st)) ||
        (e = cudaMemcpyAsync(c->obs_d.p, po.op, sizeof(double2) * 16 * nobs, cudaMemcpyHostToDevice, st)) ||
        (e = cudaMemcpyAsync(c->times_d.p, p->times, sizeof(double) * p->ntimes, cudaMemcpyHostToDevice, st)) ||
        (e = cudaMemcpyAsync(c->pflip_d.p, pf.data(), sizeof(double) * p->ntimes, cudaMemcpyHostToDevice, st)) ||
        (e = cudaMemcpyAsync(c->sys_d.p, &S, sizeof(S), cudaMemcpyHostToDevice, st)) ||
        (e = cudaMemcpyAsync(c->work_d.p, work.data(), sizeof(ResidentWork) * M, cudaMemcpyHostToDevice, st)) ||
        (e = cudaMemsetAsync(c->status.p, 0, sizeof(int), st)))
        return cuda_fail(c, e, "resident setup");
    // column-major state for the warps (complex64: narrowed through zbuf)
    const size_t ne = static_cast<size_t>(D) * M;
    double2 *col128 = static_cast<double2 *>(c->colbuf.p);
    if (prec == MSGPU_PREC_C64)
        if (int rc2 = ensure(c, c->zbuf, ne * sizeof(double2), "resident staging")) return rc2;
    double2 *stage = prec == MSGPU_PREC_C64 ? static_cast<double2 *>(c->zbuf.p) : col128;
    {
        Timed tm(c, KC_COMBINE);
        dim3 grid(ceil_div(D, 32), ldm / 32), block(32, 8);
        k_interleaved_to_cols<double2><<<grid, block, 0, st>>>(stage, static_cast<const double2 *>(c->psi128.p), D, M, ldm);
        if (prec == MSGPU_PREC_C64)
            k_convert<float2, double2><<<ceil_div(ne, 256), 256, 0, st>>>(reinterpret_cast<float2 *>(col128), stage, ne);
    }
    const size_t smem = static_cast<size_t>(warps) * wb;
    const int blocks = ceil_div(M, warps);
    {
        Timed tm(c, KC_APPLY);
        if (prec == MSGPU_PREC_C128) {
            if ((e = raise_smem_limit(reinterpret_cast<const void *>(k_resident<double2, false>), static_cast<int>(smem))))
                return cuda_fail(c, e, "resident shared memory");
            k_resident<double2, false><<<blocks, 32 * warps, smem, st>>>(
                static_cast<const ResidentSystem *>(c->sys_d.p), static_cast<const ResidentWork *>(c->work_d.p), M, wb,
                static_cast<int *>(c->status.p));
        } else {
            if ((e = raise_smem_limit(reinterpret_cast<const void *>(k_resident<float2, true>), static_cast<int>(smem))))
                return cuda_fail(c, e, "resident shared memory");
            k_resident<float2, true><<<blocks, 32 * warps, smem, st>>>(
                static_cast<const ResidentSystem *>(c->sys_d.p), static_cast<const ResidentWork *>(c->work_d.p), M, wb,
                static_cast<int *>(c->status.p));
        }
    }
    {
        Timed tm(c, KC_YIELD);
        k_resident_values<<<p->ntimes, 256, 0, st>>>(static_cast<const double *>(c->trajval.p), M, nobs,
                                                      static_cast<double *>(c->values_d.p));
    }
    {
        Timed tm(c, KC_COMBINE);
        if (prec == MSGPU_PREC_C64)
            k_convert<double2, float2><<<ceil_div(ne, 256), 256, 0, st>>>(stage, reinterpret_cast<const float2 *>(col128), ne);
        dim3 grid(ceil_div(D, 32), ldm / 32), block(32, 8);
        k_cols_to_interleaved<double2><<<grid, block, 0, st>>>(static_cast<double2 *>(c->psi128.p), stage, D, M, ldm);
    }
    int status = 0;
    c->last_values.assign(static_cast<size_t>(p->ntimes) * nobs, 0.0);
    if ((e = cudaGetLastError()) ||
        (e = cudaMemcpyAsync(&status, c->status.p, sizeof(int), cudaMemcpyDeviceToHost, st)) ||
        (e = cudaMemcpyAsync(c->last_values.data(), c->values_d.p, c->last_values.size() * sizeof(double),
                             cudaMemcpyDeviceToHost, st)) ||
        (e = cudaStreamSynchronize(st)))
        return cuda_fail(c, e, "resident run");
    collect_profile(c);
    c->state_prec = MSGPU_PREC_C128;
    c->last_ntimes = p->ntimes;
    c->have_integrals = true;
    if (status & 2) return fail(c, MSGPU_ERR_NONFINITE, "run: non-finite observable or norm on the device");
    if (status & 1) return fail(c, MSGPU_ERR_EXPM, "run: small matrix exponential failed");
    return MSGPU_OK;
}

// Quartet-block form of H for the current electron strides (see QuartetC).
// B-operand tables of the tensor-core SpMM from the current quartet values.
int tc_tables(msgpu_ctx *c)
{
    if (!c->tc_ok) return MSGPU_OK;
    k_tc_tables<<<c->tc_entries, 128, 0, c->stream>>>(static_cast<const int2 *>(c->tc_src.p), c->tc_entries,
                                                      static_cast<const float4 *>(c->qval.p),
                                                      static_cast<unsigned char *>(c->tc_tab.p));
    k_tm_tables<<<ceil_div(8 * c->tc_entries, 256), 256, 0, c->stream>>>(
        static_cast<const int2 *>(c->tc_src.p), 2 * c->tc_P, c->tc_entries, static_cast<const float4 *>(c->qval.p),
        static_cast<float4 *>(c->tm_tab.p));
    const cudaError_t e = cudaGetLastError();
    return e ? cuda_fail(c, e, "tensor-core SpMM tables") : MSGPU_OK;
}

int refresh_quartet_values(msgpu_ctx *c)
{
    if (!c->q_nslots) return MSGPU_OK;
    k_quartet_refresh<<<static_cast<unsigned>((c->q_nslots + 255) / 256), 256, 0, c->stream>>>(
        static_cast<const int *>(c->qsrc.p), c->q_nslots, static_cast<const double2 *>(c->hval.p),
        static_cast<float2 *>(c->qval.p), static_cast<double2 *>(c->qval64.p));
    const cudaError_t e = cudaGetLastError();
    if (e) return cuda_fail(c, e, "quartet value refresh");
    return c->tc_build == c->q_build ? tc_tables(c) : MSGPU_OK;
}

int build_quartet(msgpu_ctx *c)
{
    if (c->q_D == c->D && c->q_s1 == c->s1 && c->q_s2 == c->s2) return MSGPU_OK;
    const int D = c->D, s1 = c->s1, s2 = c->s2, Q = D / 4;
    const int off[4] = {0, s2, s1, s1 + s2};
    std::vector<int> rowptr(Q + 1, 0), base(Q);
    std::vector<int2> blks;
    std::vector<float> vals;
    std::vector<double> vals64;  // the same values in FP64
    std::vector<std::pair<int, std::array<double, 32>>> blocks;  // (neighbour base, 16 complex)
    std::vector<std::array<int, 16>> bsrc;                        // CSR index of each block entry
    std::vector<int> src;                                         // CSR index per stored value slot
    for (int q = 0; q < Q; ++q) {
        const int lo = q % s2, mid = (q / s2) % (s1 / (2 * s2)), hi = q / (s1 / 2);
        const int b = hi * (2 * s1) + mid * (2 * s2) + lo;
        base[q] = b;
        blocks.clear();
        bsrc.clear();
        for (int a = 0; a < 4; ++a) {
            const int r = b + off[a];
            for (int k = c->h_rowptr[r]; k < c->h_rowptr[r + 1]; ++k) {
                const int col = c->h_col[k];
                const int a1 = (col / s1) & 1, a2 = (col / s2) & 1;
                const int cb = col - a1 * s1 - a2 * s2, bi = 2 * a1 + a2;
                size_t slot = 0;
                while (slot < blocks.size() && blocks[slot].first != cb) ++slot;
                if (slot == blocks.size()) {
                    std::array<double, 32> z;
                    z.fill(0.0);
                    blocks.push_back({cb, z});
                    std::array<int, 16> none;
                    none.fill(-1);
                    bsrc.push_back(none);
                }
                bsrc[slot][a * 4 + bi] = k;
                blocks[slot].second[2 * (a * 4 + bi)] += c->h_val[2 * static_cast<size_t>(k)];
                blocks[slot].second[2 * (a * 4 + bi) + 1] += c->h_val[2 * static_cast<size_t>(k) + 1];
            }
        }
        std::vector<size_t> ord(blocks.size());
        for (size_t i = 0; i < ord.size(); ++i) ord[i] = i;
        // by neighbour base, the quartet's own block last (the SpMM reuses its
        // gathered rows for the alpha partial)
        std::sort(ord.begin(), ord.end(), [&](size_t x, size_t y) {
            const bool ox = blocks[x].first == b, oy = blocks[y].first == b;
            return ox != oy ? oy : blocks[x].first < blocks[y].first;
        });
        for (size_t oi : ord) {
            const auto &blk = blocks[oi];
            const auto &B = blk.second;  // 16 complex, row-major in the pair index
            auto re = [&](int a, int b) { return B[2 * (a * 4 + b)]; };
            auto im = [&](int a, int b) { return B[2 * (a * 4 + b) + 1]; };
            double bmax = 0.0;
            bool e1only = true, e2only = true;
            for (int a = 0; a < 4; ++a)
                for (int bb = 0; bb < 4; ++bb) {
                    bmax = std::max(bmax, std::abs(re(a, bb)) + std::abs(im(a, bb)));
                    const bool nz = re(a, bb) != 0.0 || im(a, bb) != 0.0;
                    if (!nz) continue;
                    if ((a & 1) != (bb & 1)) e1only = false;  // couples different second digits
                    if ((a & 2) != (bb & 2)) e2only = false;  // couples different first digits
                }
            auto same = [&](int a, int b, int a2, int b2) {
                return std::abs(re(a, b) - re(a2, b2)) + std::abs(im(a, b) - im(a2, b2)) <= 1e-13 * bmax;
            };
            // emit (a, b) pairs of the block in the storage order of its type
            std::vector<std::pair<int, int>> order;
            int type;
            if (e1only && e2only) {
                type = 3;
                for (int a = 0; a < 4; ++a) order.push_back({a, a});
            } else if (e1only) {
                // acts on the first digit; A (x) I when both second-digit halves agree
                const bool kron = same(0, 0, 1, 1) && same(0, 2, 1, 3) && same(2, 0, 3, 1) && same(2, 2, 3, 3);
                type = kron ? 4 : 1;
                for (int a2 = 0; a2 < (kron ? 1 : 2); ++a2)
                    for (int a1 = 0; a1 < 2; ++a1)
                        for (int b1 = 0; b1 < 2; ++b1) order.push_back({2 * a1 + a2, 2 * b1 + a2});
            } else if (e2only) {
                const bool kron = same(0, 0, 2, 2) && same(0, 1, 2, 3) && same(1, 0, 3, 2) && same(1, 1, 3, 3);
                type = kron ? 5 : 2;
                for (int a1 = 0; a1 < (kron ? 1 : 2); ++a1)
                    for (int a2 = 0; a2 < 2; ++a2)
                        for (int b2 = 0; b2 < 2; ++b2) order.push_back({2 * a1 + a2, 2 * a1 + b2});
            } else {
                type = 0;
                for (int a = 0; a < 4; ++a)
                    for (int bb = 0; bb < 4; ++bb) order.push_back({a, bb});
            }
            blks.push_back({(blk.first << 3) | type, static_cast<int>(vals.size() / 4)});
            for (auto &ab : order) {
                vals.push_back(static_cast<float>(re(ab.first, ab.second)));
                vals.push_back(static_cast<float>(im(ab.first, ab.second)));
                vals64.push_back(re(ab.first, ab.second));
                vals64.push_back(im(ab.first, ab.second));
                src.push_back(bsrc[oi][ab.first * 4 + ab.second]);
            }
        }
        rowptr[q + 1] = static_cast<int>(blks.size());
    }
    const int nb = static_cast<int>(blks.size());
    int rc;
    if ((rc = ensure(c, c->qrow, sizeof(int) * (Q + 1), "quartet rowptr")) ||
        (rc = ensure(c, c->qcolt, sizeof(int2) * std::max(1, nb), "quartet blocks")) ||
        (rc = ensure(c, c->qval, sizeof(float) * std::max<size_t>(4, vals.size()), "quartet values")) ||
        (rc = ensure(c, c->qval64, sizeof(double) * std::max<size_t>(4, vals64.size()), "quartet values (FP64)")) ||
        (rc = ensure(c, c->qbase, sizeof(int) * Q, "quartet bases")))
        return rc;
    cudaError_t e;
    if ((e = cudaMemcpyAsync(c->qrow.p, rowptr.data(), sizeof(int) * (Q + 1), cudaMemcpyHostToDevice, c->stream)) ||
        (e = cudaMemcpyAsync(c->qcolt.p, blks.data(), sizeof(int2) * nb, cudaMemcpyHostToDevice, c->stream)) ||
        (e = cudaMemcpyAsync(c->qval.p, vals.data(), sizeof(float) * vals.size(), cudaMemcpyHostToDevice, c->stream)) ||
        (e = cudaMemcpyAsync(c->qval64.p, vals64.data(), sizeof(double) * vals64.size(), cudaMemcpyHostToDevice,
                             c->stream)) ||
        (e = cudaMemcpyAsync(c->qbase.p, base.data(), sizeof(int) * Q, cudaMemcpyHostToDevice, c->stream)) ||
        (e = cudaStreamSynchronize(c->stream)))
        return cuda_fail(c, e, "quartet upload");
    c->q_D = D;
    c->q_s1 = s1;
    c->q_s2 = s2;
    c->q_nblocks = nb;
    ++c->q_build;
    c->q_hrow = std::move(rowptr);
    c->q_hblk = std::move(blks);
    c->q_hval = std::move(vals);
    c->q_tile = 0;
    c->q_nslots = src.size();
    if (c->terms) {
        // the structure came from a generic combination of the terms; the
        // values of the current coefficients come from the device CSR
        if ((rc = ensure(c, c->qsrc, sizeof(int) * std::max<size_t>(1, src.size()), "quartet value map")))
            return rc;
        if ((e = cudaMemcpyAsync(c->qsrc.p, src.data(), sizeof(int) * src.size(), cudaMemcpyHostToDevice, c->stream)))
            return cuda_fail(c, e, "quartet value map");
        if ((rc = refresh_quartet_values(c))) return rc;
    }
    return MSGPU_OK;
}

QuartetC quartet_view(const msgpu_ctx *c)
{
    return QuartetC{static_cast<const int *>(c->qrow.p), static_cast<const int2 *>(c->qcolt.p),
                    static_cast<const float4 *>(c->qval.p), static_cast<const int *>(c->qbase.p)};
}

// Validates the nuclear-bit structure the tensor-core SpMM relies on, on the
// host copy of the quartet form: Q = 2^P quartets, every block couples q to
// itself or to q ^ 2^p, every quartet has the same set of flip bits, and the
// flip block of (p, bit p of the output quartet) is the same in every quartet.
// Then builds the table entries (2P flip entries, then Q diagonal entries) and
// the B-operand tables.  tc_ok stays false when the structure is absent.
int build_tc(msgpu_ctx *c)
{
    if (c->tc_build == c->q_build) return MSGPU_OK;
    c->tc_build = c->q_build;
    c->tc_ok = false;
    const int Q = c->D / 4, s1 = c->s1, s2 = c->s2;
    int P = 0;
    while ((1 << P) < Q) ++P;
    if ((1 << P) != Q || P < 5 || P > kTcMaxBits) return MSGPU_OK;
    // quartet index of a base row (inverse of the base map of build_quartet)
    auto qindex = [&](int b) {
        const int lo = b % s2, mid = (b / (2 * s2)) % (s1 / (2 * s2)), hi = b / (2 * s1);
        return hi * (s1 / 2) + mid * s2 + lo;
    };
    // full 4 x 4 complex block of a compact entry (host twin of tc_expand)
    auto expand = [&](int type, int off, std::array<float, 32> &h) {
        h.fill(0.f);
        const float *v = c->q_hval.data() + 4 * static_cast<size_t>(off);
        auto set = [&](int a, int b, int i) {
            h[2 * (4 * a + b)] = v[2 * i];
            h[2 * (4 * a + b) + 1] = v[2 * i + 1];
        };
        switch (type) {
        case 0:
            for (int a = 0; a < 4; ++a)
                for (int b = 0; b < 4; ++b) set(a, b, 4 * a + b);
            break;
        case 1:
            for (int a2 = 0; a2 < 2; ++a2)
                for (int a1 = 0; a1 < 2; ++a1)
                    for (int b1 = 0; b1 < 2; ++b1) set(2 * a1 + a2, 2 * b1 + a2, (2 * a2 + a1) * 2 + b1);
            break;
        case 2:
            for (int a1 = 0; a1 < 2; ++a1)
                for (int a2 = 0; a2 < 2; ++a2)
                    for (int b2 = 0; b2 < 2; ++b2) set(2 * a1 + a2, 2 * a1 + b2, (2 * a1 + a2) * 2 + b2);
            break;
        case 3:
            for (int a = 0; a < 4; ++a) set(a, a, a);
            break;
        case 4:
            for (int a1 = 0; a1 < 2; ++a1)
                for (int b1 = 0; b1 < 2; ++b1)
                    for (int a2 = 0; a2 < 2; ++a2) set(2 * a1 + a2, 2 * b1 + a2, 2 * a1 + b1);
            break;
        default:
            for (int a2 = 0; a2 < 2; ++a2)
                for (int b2 = 0; b2 < 2; ++b2)
                    for (int a1 = 0; a1 < 2; ++a1) set(2 * a1 + a2, 2 * a1 + b2, 2 * a2 + b2);
            break;
        }
    };
    const int nent = 2 * P + Q;
    std::vector<int2> src(nent, make_int2(-1, 0));
    std::vector<std::array<float, 32>> rep(2 * P);
    std::vector<unsigned> mask(Q, 0u);
    std::array<float, 32> h;
    for (int q = 0; q < Q; ++q)
        for (int k = c->q_hrow[q]; k < c->q_hrow[q + 1]; ++k) {
            const int2 blk = c->q_hblk[k];
            const int d = q ^ qindex(blk.x >> 3), type = blk.x & 7;
            if (d == 0) {
                src[2 * P + q] = make_int2(blk.y, type);
                continue;
            }
            if (d & (d - 1)) return MSGPU_OK;  // not a single nuclear flip
            int p = 0;
            while ((1 << p) != d) ++p;
            mask[q] |= 1u << p;
            const int e = 2 * p + ((q >> p) & 1);
            expand(type, blk.y, h);
            if (src[e].x < 0) {
                src[e] = make_int2(blk.y, type);
                rep[e] = h;
                continue;
            }
            float amax = 0.f, dmax = 0.f;
            for (int i = 0; i < 32; ++i) {
                amax = std::max(amax, std::abs(rep[e][i]));
                dmax = std::max(dmax, std::abs(rep[e][i] - h[i]));
            }
            if (dmax > 0x1p-22f * amax) return MSGPU_OK;  // the flip block depends on more than (p, bit)
        }
    for (int q = 1; q < Q; ++q)
        if (mask[q] != mask[0]) return MSGPU_OK;
    int rc;
    if ((rc = ensure(c, c->tc_src, sizeof(int2) * nent, "tensor-core SpMM table entries")) ||
        (rc = ensure(c, c->tc_tab, static_cast<size_t>(nent) * 2 * kTcB, "tensor-core SpMM tables")) ||
        (rc = ensure(c, c->tm_tab, static_cast<size_t>(nent) * 8 * sizeof(float4), "TMEM-staged SpMM tables")))
        return rc;
    cudaError_t e;
    if ((e = cudaMemcpyAsync(c->tc_src.p, src.data(), sizeof(int2) * nent, cudaMemcpyHostToDevice, c->stream)) ||
        (e = cudaStreamSynchronize(c->stream)))
        return cuda_fail(c, e, "tensor-core SpMM table entries");
    c->tc_P = P;
    c->tc_entries = nent;
    c->tc_ok = true;
    return tc_tables(c);
}


// ------------------------------------------------- cluster-resident Lanczos
// Bound on the off-diagonal blocks one CTA of k_lanczos_fused<C> stages (the
// quartets' own blocks are counted too).
int fused_blocks_max(const msgpu_ctx *c, int C)
{
    const int Q = c->D / 4, Qc = ceil_div(Q, C);
    int mx = 0;
    for (int r = 0; r < C; ++r) {
        const int qb = std::min(Q, r * Qc), qe = std::min(Q, qb + Qc);
        mx = std::max(mx, c->q_hrow[qe] - c->q_hrow[qb]);
    }
    return mx;
}

// Descriptors of k_lanczos_fused for cluster size C (Qc = ceil(Q / C)
// quartets per CTA).  Each quartet's own block is set apart (its type and
// value offset, expanded to a full 4x4 on the device by k_fused_diag before
// every launch, so values refreshed in place are followed); the other blocks
// keep their values and get (owner rank, local quartet) for their neighbour.
// For a static H, off-diagonal value blocks with equal bits share one copy --
// the flip blocks of a nucleus repeat over all quartets -- so the values the
// CTAs read stay in L1.  With Hamiltonian terms the values are refreshed in
// place every step, so the blocks keep their own slots.
int build_fused(msgpu_ctx *c, int C)
{
    if (c->f_build == c->q_build && c->f_C == C) return MSGPU_OK;
    const int Q = c->D / 4, Qc = ceil_div(Q, C), s1 = c->s1, s2 = c->s2;
    const bool dedup = !c->terms;
    const std::vector<int2> &hb = c->q_hblk;
    const std::vector<float> &hv = c->q_hval;
    std::vector<int> frow(Q + 1, 0);
    std::vector<int2> fb, dsrc(Q, make_int2(-1, 0));
    fb.reserve(hb.size());
    std::vector<float> fv;
    std::map<std::vector<uint32_t>, int> seen;  // value bits -> offset in fv (float4 units)
    std::vector<int> ord;
    for (int q = 0; q < Q; ++q) {
        const int own = (q / (s1 / 2)) * (2 * s1) + ((q / s2) % (s1 / (2 * s2))) * (2 * s2) + q % s2;
        const int kb = c->q_hrow[q], ke = c->q_hrow[q + 1];
        // Off-diagonal blocks by |neighbour base - own base|, one flip block per
        // nucleus in stride order: the lanes of a warp hold neighbouring
        // quartets, so block k is the same nucleus, type and owner CTA on every
        // lane (no divergent block types, no split between local and remote
        // gathers).
        ord.clear();
        for (int k = kb; k < ke; ++k) {
            if ((hb[k].x >> 3) == own)
                dsrc[q] = make_int2(hb[k].x & 7, hb[k].y);
            else
                ord.push_back(k);
        }
        std::stable_sort(ord.begin(), ord.end(), [&](int x, int y) {
            const long long dx = (hb[x].x >> 3) - own, dy = (hb[y].x >> 3) - own;
            return std::llabs(dx) != std::llabs(dy) ? std::llabs(dx) < std::llabs(dy) : dx < dy;
        });
        for (int k : ord) {
            const int b = hb[k].x >> 3, type = hb[k].x & 7;
            // inverse of quartet_base: drop the two electron digits of the base row
            const int qn = (b / (2 * s1)) * (s1 / 2) + ((b / (2 * s2)) % (s1 / (2 * s2))) * s2 + b % s2;
            const int r = qn / Qc, lq = qn - r * Qc;
            int voff = hb[k].y;
            if (dedup) {
                const size_t nf = 4 * static_cast<size_t>(type == 0 ? 8 : type <= 2 ? 4 : 2);
                const size_t at = 4 * static_cast<size_t>(voff);
                std::vector<uint32_t> key(nf);
                std::memcpy(key.data(), hv.data() + at, nf * sizeof(float));
                auto it = seen.find(key);
                if (it == seen.end()) {
                    const int fo = static_cast<int>(fv.size() / 4);
                    fv.insert(fv.end(), hv.begin() + at, hv.begin() + at + nf);
                    it = seen.emplace(std::move(key), fo).first;
                }
                voff = it->second;
            }
            fb.push_back(make_int2((lq << 7) | (r << 3) | type, voff));
        }
        frow[q + 1] = static_cast<int>(fb.size());
    }
    int rc;
    cudaError_t e;
    if ((rc = ensure(c, c->fblk, sizeof(int2) * std::max<size_t>(1, fb.size()), "fused Lanczos blocks")) ||
        (rc = ensure(c, c->frow, sizeof(int) * (Q + 1), "fused Lanczos row pointers")) ||
        (rc = ensure(c, c->fdsrc, sizeof(int2) * Q, "fused Lanczos diagonal map")) ||
        (rc = ensure(c, c->fdiag, sizeof(float4) * 8 * static_cast<size_t>(Q), "fused Lanczos diagonal blocks")))
        return rc;
    if ((e = cudaMemcpyAsync(c->fblk.p, fb.data(), sizeof(int2) * fb.size(), cudaMemcpyHostToDevice, c->stream)) ||
        (e = cudaMemcpyAsync(c->frow.p, frow.data(), sizeof(int) * (Q + 1), cudaMemcpyHostToDevice, c->stream)) ||
        (e = cudaMemcpyAsync(c->fdsrc.p, dsrc.data(), sizeof(int2) * Q, cudaMemcpyHostToDevice, c->stream)))
        return cuda_fail(c, e, "fused Lanczos blocks");
    if (dedup) {
        if ((rc = ensure(c, c->fval, sizeof(float) * std::max<size_t>(4, fv.size()), "fused Lanczos values")))
            return rc;
        if ((e = cudaMemcpyAsync(c->fval.p, fv.data(), sizeof(float) * fv.size(), cudaMemcpyHostToDevice, c->stream)))
            return cuda_fail(c, e, "fused Lanczos values");
    }
    if ((e = cudaStreamSynchronize(c->stream))) return cuda_fail(c, e, "fused Lanczos blocks");
    c->f_C = C;
    c->f_build = c->q_build;
    c->f_dedup = dedup;
    c->f_nblk_max = fused_blocks_max(c, C);
    return MSGPU_OK;
}

using FusedFn = void (*)(QuartetF, float2 *, size_t, double *, double *, double *, int *, int, int, int, int, int, int,
                         int);

FusedFn fused_kernel(int C)
{
    switch (C) {
    case 1: return k_lanczos_fused<1>;
    case 2: return k_lanczos_fused<2>;
    case 4: return k_lanczos_fused<4>;
    case 8: return k_lanczos_fused<8>;
    case 16: return k_lanczos_fused<16>;
    default: return nullptr;
    }
}

// Allow the kernel the device's opt-in shared memory (each launch still asks
// for its own size) and, for 16-CTA clusters, the non-portable cluster size.
cudaError_t fused_prepare(const msgpu_ctx *c, FusedFn fn, int C)
{
    int optin = 0;
    cudaError_t e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->device);
    if (!e) e = raise_smem_limit(reinterpret_cast<const void *>(fn), optin);
    if (!e && C > 8)
        e = cudaFuncSetAttribute(reinterpret_cast<const void *>(fn), cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    return e;
}

cudaLaunchConfig_t fused_config(int C, int ldm, size_t smem, cudaStream_t st, cudaLaunchAttribute *attr)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(static_cast<unsigned>(C * (ldm / (2 * kFusedPairs))));
    cfg.blockDim = dim3(kFusedThreads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = C;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cfg;
}

// Whether k_lanczos_fused<C> runs this shape: a CTA's share of the vectors and
// of the quartet structure fits its shared memory, and at least one cluster of
// C such CTAs can be resident on the device.
bool fused_fits(msgpu_ctx *c, int C)
{
    const int Q = c->D / 4, Qc = ceil_div(Q, C);
    if (Qc > kFusedMaxQc) return false;
    const FusedFn fn = fused_kernel(C);
    const size_t smem = fused_smem_bytes(Qc, fused_blocks_max(c, C), C);
    int optin = 0, nclusters = 0;
    cudaLaunchAttribute attr[1];
    const cudaLaunchConfig_t cfg = fused_config(C, c->ldm, smem, c->stream, attr);
    const bool ok = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->device) == cudaSuccess &&
                    smem <= static_cast<size_t>(optin) && fused_prepare(c, fn, C) == cudaSuccess &&
                    cudaOccupancyMaxActiveClusters(&nclusters, reinterpret_cast<const void *>(fn), &cfg) == cudaSuccess &&
                    nclusters > 0;
    cudaGetLastError();  // a refused query is an answer, not an error of the run
    return ok;
}

// Cluster size of k_lanczos_fused for the current shape, or 0 for the
// four-kernel iteration (MSGPU_OPT_LANCZOS_CLUSTER 0, the default, or nothing
// fits): with -1 the smallest power of two whose CTAs hold their share (unless
// MSGPU_OPT_SPMM_VARIANT forces an SpMM variant), else the size asked for.
// Needs the quartet form.
int fused_cluster(msgpu_ctx *c)
{
    if (c->f_opt == 0 || (c->f_opt < 0 && c->spmm_variant >= 0)) return 0;  // a forced SpMM variant keeps its loop
    if (c->f_probe_D == c->D && c->f_probe_ldm == c->ldm && c->f_probe_build == c->q_build) return c->f_probe_C;
    int pick = 0;
    for (int C : {1, 2, 4, 8, 16})
        if ((c->f_opt < 0 || c->f_opt == C) && fused_fits(c, C)) {
            pick = C;
            break;
        }
    c->f_probe_D = c->D;
    c->f_probe_ldm = c->ldm;
    c->f_probe_build = c->q_build;
    c->f_probe_C = pick;
    return pick;
}

int launch_fused(msgpu_ctx *c, int C, float2 *Wb, size_t n, double *sc, double *td, double *to, int *mdim, int m)
{
    if (int rc = build_fused(c, C)) return rc;
    const int Q = c->D / 4, Qc = ceil_div(Q, C);
    const size_t smem = fused_smem_bytes(Qc, c->f_nblk_max, C);
    const QuartetF H{static_cast<const int *>(c->frow.p), static_cast<const int2 *>(c->fblk.p),
                     static_cast<const float4 *>(c->f_dedup ? c->fval.p : c->qval.p),
                     static_cast<const float4 *>(c->fdiag.p), static_cast<const int *>(c->qbase.p)};
    k_fused_diag<<<ceil_div(8 * Q, 256), 256, 0, c->stream>>>(static_cast<const int2 *>(c->fdsrc.p),
                                                               static_cast<const float2 *>(c->qval.p),
                                                               static_cast<float4 *>(c->fdiag.p), Q);
    const FusedFn fn = fused_kernel(C);
    cudaError_t e = cudaGetLastError();
    if (!e) e = fused_prepare(c, fn, C);
    cudaLaunchAttribute attr[1];
    const cudaLaunchConfig_t cfg = fused_config(C, c->ldm, smem, c->stream, attr);
    if (!e)
        e = cudaLaunchKernelEx(&cfg, fn, H, Wb, n, sc, td, to, mdim, Q, Qc, c->f_nblk_max, c->ldm, m, c->s1, c->s2);
    return e ? cuda_fail(c, e, "fused Lanczos launch") : MSGPU_OK;
}

// Autotuner for the quartet SpMM: times each candidate tile (quartets per
// CTA) on the context's own data with CUDA events and keeps the fastest for
// this (D, trajectory block).  Runs once per context and shape.
using ApplyFn = void (*)(QuartetC, const float2 *, const double *, float2 *, double *, int, int, int, int, int);
struct ApplyVariant {
    ApplyFn fn;
    bool cube;  // stages the tile's own input quartets in shared memory (QT x 2 KB)
    int np;     // trajectory pairs per thread (a CTA covers 64 np trajectories)
};
const ApplyVariant kApplyVariants[] = {
    {k_lanczos_apply_compact<true, 2>, false, 1},
    {k_lanczos_apply_compact<true, 3>, false, 1},
    {k_lanczos_apply_compact<false, 3>, false, 1},
    {k_lanczos_apply_compact<false, 4>, false, 1},
    {k_lanczos_apply_cube<2>, true, 1},
    {k_lanczos_apply_cube<3>, true, 1},
    {k_lanczos_apply_np<2, 2>, false, 2},
    {k_lanczos_apply_np<2, 3>, false, 2},
};
constexpr int kNumApplyVariants = sizeof(kApplyVariants) / sizeof(kApplyVariants[0]);
static_assert(kNumApplyVariants == kNumSimtVariants, "SpMM variant count");
constexpr int kCubeMaxQT = 64;  // 128 KB of shared memory
// Whether the tensor-core SpMM (variants kNumSimtVariants + 0 / + 1: cube bits
// 4 / 3) takes part in the tuner's choice; it can always be forced with
// MSGPU_OPT_SPMM_VARIANT.
constexpr bool kTcInTuner = false;
// The TMEM-staged SpMM (variant kTmVariant): cubes of 8 quartets, two compute
// warpgroups, three copy warps.
using TmK = TmCfg<3, 2, 3>;
constexpr bool kTmInTuner = false;

int tc_cube_bits(int v) { return v == kNumSimtVariants ? 4 : 3; }

bool in_tuner(int v) { return v < kNumSimtVariants || (v == kTmVariant ? kTmInTuner : kTcInTuner); }

// U = s H w over `width` trajectories with the tensor-core SpMM.
using TcEncodeTiled = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                   const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

// The tensor-core SpMM's 2D tensor map over the complex64 Krylov basis:
// 8-byte elements, rows of ldm trajectories, boxes of 128 trajectories x HB
// rows; re-encoded when the basis buffer or its shape changes.  On failure the
// tensor-core variants are switched off for this context (tc_ok = false).
int tc_prepare_map(msgpu_ctx *c)
{
    if (!c->tc_ok || !c->basis.p) return MSGPU_OK;
    const long long rows = static_cast<long long>(c->basis.bytes / (8 * static_cast<size_t>(c->ldm)));
    if (c->tc_map_base == c->basis.p && c->tc_map_rows == rows && c->tc_map_ldm == c->ldm) return MSGPU_OK;
    // looked up once (thread-safe static initialisation: batch contexts prepare from several host threads)
    static const TcEncodeTiled enc = []() -> TcEncodeTiled {
        void *fp = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fp, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            return reinterpret_cast<TcEncodeTiled>(fp);
        return nullptr;
    }();
    const cuuint64_t dims[2] = {static_cast<cuuint64_t>(c->ldm), static_cast<cuuint64_t>(rows)};
    const cuuint64_t strides[1] = {static_cast<cuuint64_t>(c->ldm) * 8};
    const cuuint32_t box[2] = {static_cast<cuuint32_t>(kTcTraj), static_cast<cuuint32_t>(TcCfg<4>::HB)};
    const cuuint32_t estr[2] = {1, 1};
    static_assert(TcCfg<4>::HB == TcCfg<3>::HB, "one box shape");
    if (!enc || enc(&c->tc_map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, c->basis.p, dims, strides, box, estr,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS) {
        c->tc_ok = false;
        c->tc_map_base = nullptr;
        return MSGPU_OK;
    }
    // the TMEM-staged SpMM's boxes: 256 trajectories x one cube of 8 quartet rows
    const cuuint32_t tbox[2] = {static_cast<cuuint32_t>(TmK::Traj), static_cast<cuuint32_t>(TmK::NQ)};
    c->tm_map_ok = enc(&c->tm_map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, c->basis.p, dims, strides, tbox, estr,
                       CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                       CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
    c->tc_map_base = c->basis.p;
    c->tc_map_rows = rows;
    c->tc_map_ldm = c->ldm;
    return MSGPU_OK;
}

void launch_tc(const msgpu_ctx *c, int cb, cudaStream_t st, const float2 *w, const double *s, float2 *U, double *part,
               int width)
{
    const int Q = c->D / 4, P = c->tc_P;
    const unsigned char *tflip = static_cast<const unsigned char *>(c->tc_tab.p);
    const unsigned char *tdiag = tflip + static_cast<size_t>(2 * P) * 2 * kTcB;
    const dim3 grid(Q >> cb, ceil_div(width, kTcTraj));
    int *status = static_cast<int *>(c->status.p);
    // w lies in the basis the map covers (apply_fits checks the map): its first row and column
    const long long offs = w - static_cast<const float2 *>(c->tc_map_base);
    const int y0 = static_cast<int>(offs / c->ldm), x0 = static_cast<int>(offs % c->ldm);
    if (cb == 4) {
        const int smem = TcCfg<4>::smem(P);
        raise_smem_limit(reinterpret_cast<const void *>(k_lanczos_apply_tc<4>), smem);
        k_lanczos_apply_tc<4><<<grid, TcCfg<4>::Threads, smem, st>>>(c->tc_map, x0, y0, tflip, tdiag, P, c->s1, c->s2, s, U,
                                                                     part, c->ldm, width, status);
    } else {
        const int smem = TcCfg<3>::smem(P);
        raise_smem_limit(reinterpret_cast<const void *>(k_lanczos_apply_tc<3>), smem);
        k_lanczos_apply_tc<3><<<grid, TcCfg<3>::Threads, smem, st>>>(c->tc_map, x0, y0, tflip, tdiag, P, c->s1, c->s2, s, U,
                                                                     part, c->ldm, width, status);
    }
}

// U = s H w over `width` trajectories with the TMEM-staged SpMM: one
// persistent CTA per SM (at most one per item).
void launch_tm(const msgpu_ctx *c, cudaStream_t st, const float2 *w, const double *s, float2 *U, double *part,
               int width)
{
    const int Q = c->D / 4, P = c->tc_P;
    const int items = (Q / TmK::NQ) * ceil_div(width, TmK::Traj);
    const int grid = std::max(1, std::min(items, c->sm_count));
    const long long offs = w - static_cast<const float2 *>(c->tc_map_base);
    const int y0 = static_cast<int>(offs / c->ldm), x0 = static_cast<int>(offs % c->ldm);
    auto fn = k_lanczos_apply_tm<3, 2, 3>;
    raise_smem_limit(reinterpret_cast<const void *>(fn), TmK::Smem);
    fn<<<grid, TmK::Threads, TmK::Smem, st>>>(c->tm_map, x0, y0, static_cast<const int2 *>(c->tc_src.p),
                                              static_cast<const float4 *>(c->tm_tab.p), P, c->s1, c->s2, s, U, part,
                                              c->ldm, width, static_cast<int *>(c->status.p));
}

// Whether variant v can run with tile QT on this system, and its shared memory.
bool apply_fits(const msgpu_ctx *c, int v, int qt, size_t *smem)
{
    *smem = 0;
    if (v == kTmVariant) {
        // the maps cover this basis, a cube's 8 quartets have consecutive rows, and a
        // group's width is a multiple of 64 trajectories
        if (!c->tc_ok || !c->tm_map_ok || qt != TmK::NQ || c->tc_P < 4 || c->s2 % TmK::NQ != 0 ||
            !c->tc_map_base || c->tc_map_base != c->basis.p || c->tc_map_ldm != c->ldm || c->sm_count < 1 ||
            (c->ldm / traj_groups(c)) % 64 != 0)
            return false;
        *smem = static_cast<size_t>(TmK::Smem);
        return true;
    }
    if (v >= kNumSimtVariants) {
        const int cb = tc_cube_bits(v);
        // the map covers this basis, and the cube's quartets have consecutive rows (boxes of HB rows)
        if (!c->tc_ok || qt != (1 << cb) || c->tc_P < cb + 1 || c->s2 % (1 << cb) != 0 || !c->tc_map_base ||
            c->tc_map_base != c->basis.p || c->tc_map_ldm != c->ldm)
            return false;
        *smem = static_cast<size_t>(cb == 4 ? TcCfg<4>::smem(c->tc_P) : TcCfg<3>::smem(c->tc_P));
        return true;
    }
    // the step launches it over one trajectory group, the tuner over the whole block
    if ((c->ldm / traj_groups(c)) % (64 * kApplyVariants[v].np) != 0 || c->ldm % (64 * kApplyVariants[v].np) != 0)
        return false;
    if (!kApplyVariants[v].cube) return true;
    // the tile's quartet bases must be contiguous: QT divides the second stride
    if (qt > kCubeMaxQT || c->s2 % qt != 0) return false;
    *smem = static_cast<size_t>(qt) * 4 * 32 * sizeof(float4);
    return true;
}

// width: trajectories of the launch (the pointers start at its first one)
void launch_apply(const msgpu_ctx *c, int v, int qt, dim3 grid, cudaStream_t st, const float2 *w, const double *s,
                  float2 *U, double *part, int width)
{
    if (v == kTmVariant) {
        launch_tm(c, st, w, s, U, part, width);
        return;
    }
    if (v >= kNumSimtVariants) {
        launch_tc(c, tc_cube_bits(v), st, w, s, U, part, width);
        return;
    }
    size_t smem = 0;
    apply_fits(c, v, qt, &smem);
    grid.y = width / (64 * kApplyVariants[v].np);
    if (smem) raise_smem_limit(reinterpret_cast<const void *>(kApplyVariants[v].fn), static_cast<int>(smem));
    kApplyVariants[v].fn<<<grid, kThreads, smem, st>>>(quartet_view(c), w, s, U, part, c->D / 4, c->s1, c->s2, c->ldm,
                                                       qt);
}

int tune_quartet_tile(msgpu_ctx *c, const float2 *w, const double *s, float2 *U, double *part)
{
    if (c->q_tile && c->q_tile_ldm == c->ldm) return MSGPU_OK;
    const int Q = c->D / 4;
    const int cand[] = {8, 16, 32, 64, 128};
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    // three interleaved rounds over all candidates, each candidate scored by
    // its best round: a one-off delay (another stream, a profiler) then cannot
    // pick the shape
    std::vector<std::pair<int, int>> cands;
    size_t smem;
    for (int v = 0; v < kNumSpmmVariants; ++v) {
        if (c->spmm_variant >= 0 && v != c->spmm_variant) continue;
        if (c->spmm_variant < 0 && !in_tuner(v)) continue;
        for (int qt : cand)
            if ((qt <= Q || qt == cand[0]) && apply_fits(c, v, qt, &smem)) cands.push_back({v, qt});
    }
    if (cands.empty()) return fail(c, MSGPU_ERR_INVALID, "SpMM variant does not fit this system");
    std::vector<float> score(cands.size(), 1e30f);
    for (int round = 0; round < 3; ++round)
        for (size_t k = 0; k < cands.size(); ++k) {
            const int v = cands[k].first, qt = cands[k].second;
            dim3 grid(ceil_div(Q, qt), c->ldm / 64);
            // timed over the whole block, not one group: the step overlaps the
            // groups, and the tile chosen this way measured faster there (179k
            // against 175k traj-steps/s at D=16384, 2 x 512 trajectories) although
            // alone it is the slower one at a group's width (90 against 86 us)
            launch_apply(c, v, qt, grid, c->stream, w, s, U, part, c->ldm);
            cudaEventRecord(a, c->stream);
            for (int rep = 0; rep < 2; ++rep) launch_apply(c, v, qt, grid, c->stream, w, s, U, part, c->ldm);
            cudaEventRecord(b, c->stream);
            cudaEventSynchronize(b);
            float ms = 0.f;
            cudaEventElapsedTime(&ms, a, b);
            score[k] = std::min(score[k], ms);
        }
    size_t pick = 0;
    for (size_t k = 1; k < cands.size(); ++k)
        if (score[k] < score[pick]) pick = k;
    const int best_v = cands[pick].first, best_qt = cands[pick].second;
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaError_t e = cudaGetLastError();
    if (e) return cuda_fail(c, e, "quartet tile tuning");
    c->q_tile = best_qt;
    c->q_variant = best_v;
    c->q_tile_ldm = c->ldm;
    return MSGPU_OK;
}

}  // namespace

extern "C" {

int msgpu_upload_hamiltonian_terms(msgpu_ctx *c, int dim, const int *rowptr, const int *col, int nterms,
                                   const double *vals, const double *coef)
{
    if (!c) return MSGPU_ERR_INVALID;
    if (nterms < 1 || nterms > 16 || !vals || !coef || dim < 4 || !rowptr)
        return fail(c, MSGPU_ERR_INVALID, "Hamiltonian terms: 1..16 terms, values and coefficients required");
    const int nnz = rowptr[dim];
    if (nnz < 0) return fail(c, MSGPU_ERR_INVALID, "Hamiltonian terms: malformed row pointer");
    for (size_t i = 0; i < 2 * static_cast<size_t>(nnz) * nterms; ++i)
        if (!std::isfinite(vals[i])) return fail(c, MSGPU_ERR_NONFINITE, "Hamiltonian terms: non-finite value");
    // a generic combination (fixed irrational-looking weights) fixes the
    // sparsity and block structure for every combination of the terms
    std::vector<double> gen(2 * static_cast<size_t>(nnz), 0.0);
    for (int t = 0; t < nterms; ++t) {
        const double w = 1.0 + 0.7548776662466927 * (t + 1) - std::floor(0.7548776662466927 * (t + 1));
        for (size_t i = 0; i < gen.size(); ++i) gen[i] += w * vals[static_cast<size_t>(t) * gen.size() + i];
    }
    if (int rc = msgpu_upload_hamiltonian_csr(c, dim, rowptr, col, gen.data())) return rc;
    int rc;
    if ((rc = ensure(c, c->hterms, sizeof(double2) * std::max<size_t>(1, static_cast<size_t>(nnz) * nterms),
                     "Hamiltonian terms")))
        return rc;
    cudaError_t e;
    if ((e = cudaMemcpyAsync(c->hterms.p, vals, sizeof(double2) * static_cast<size_t>(nnz) * nterms,
                             cudaMemcpyHostToDevice, c->stream)))
        return cuda_fail(c, e, "Hamiltonian terms upload");
    c->terms = true;
    c->nterms = nterms;
    return msgpu_set_hamiltonian_coefficients(c, coef);
}

int msgpu_set_hamiltonian_coefficients(msgpu_ctx *c, const double *coef)
{
    if (!c) return MSGPU_ERR_INVALID;
    if (!c->terms) return fail(c, MSGPU_ERR_STATE, "Hamiltonian coefficients: no terms uploaded");
    if (!coef) return fail(c, MSGPU_ERR_INVALID, "Hamiltonian coefficients: null array");
    if (int rc = device_guard(c)) return rc;
    TermCoef cf;
    std::memset(&cf, 0, sizeof(cf));
    for (int t = 0; t < c->nterms; ++t) {
        if (!std::isfinite(coef[t])) return fail(c, MSGPU_ERR_NONFINITE, "Hamiltonian coefficients: non-finite value");
        cf.c[t] = coef[t];
        c->hcoef[t] = coef[t];
    }
    if (int rc = ensure(c, c->status, sizeof(int), "status")) return rc;
    cudaError_t e;
    if ((e = cudaMemsetAsync(c->status.p, 0, sizeof(int), c->stream))) return cuda_fail(c, e, "Hamiltonian update");
    k_combine_terms<<<ceil_div(std::max(1, c->nnz), 256), 256, 0, c->stream>>>(
        static_cast<const double2 *>(c->hterms.p), c->nterms, cf, c->nnz, static_cast<double2 *>(c->hval.p),
        static_cast<float2 *>(c->hhi.p), static_cast<float2 *>(c->hlo.p), static_cast<int *>(c->status.p));
    if ((e = cudaGetLastError())) return cuda_fail(c, e, "Hamiltonian update");
    // the quartet form keeps its structure; only its values follow H
    if (c->q_D == c->D)
        if (int rc = refresh_quartet_values(c)) return rc;
    c->dense.have_u = false;
    int status = 0;
    if ((e = cudaMemcpyAsync(&status, c->status.p, sizeof(int), cudaMemcpyDeviceToHost, c->stream)) ||
        (e = cudaStreamSynchronize(c->stream)))
        return cuda_fail(c, e, "Hamiltonian update");
    if (status & 2) return fail(c, MSGPU_ERR_NONFINITE, "Hamiltonian coefficients: non-finite combined value");
    return MSGPU_OK;
}

namespace {

// rows_per_step 1: one midpoint row per step; 2: start and midpoint rows per
// step plus one final end row (row 2j + 2 is step j's end and step j+1's start)
int set_schedule(msgpu_ctx *c, const double *coef, long long first_step, long long nsteps, int rows_per_step)
{
    if (!c) return MSGPU_ERR_INVALID;
    if (nsteps == 0) {
        c->sched.clear();
        c->sched_steps = 0;
        c->sched_rows = 1;
        return MSGPU_OK;
    }
    if (!c->terms) return fail(c, MSGPU_ERR_STATE, "Hamiltonian schedule: no terms uploaded");
    if (!coef || nsteps < 0 || first_step < 0) return fail(c, MSGPU_ERR_INVALID, "Hamiltonian schedule: invalid arguments");
    const size_t rows = rows_per_step == 1 ? static_cast<size_t>(nsteps) : 2 * static_cast<size_t>(nsteps) + 1;
    const size_t n = rows * c->nterms;
    for (size_t i = 0; i < n; ++i)
        if (!std::isfinite(coef[i])) return fail(c, MSGPU_ERR_NONFINITE, "Hamiltonian schedule: non-finite coefficient");
    c->sched.assign(coef, coef + n);
    c->sched_first = first_step;
    c->sched_steps = nsteps;
    c->sched_rows = rows_per_step;
    return MSGPU_OK;
}

// Coefficient row of global step g at point which (0 start, 1 midpoint, 2 end);
// a midpoint-only schedule has only which = 1.
const double *sched_row(const msgpu_ctx *c, long long g, int which)
{
    const size_t k = static_cast<size_t>(g - c->sched_first);
    const size_t row = c->sched_rows == 1 ? k : 2 * k + static_cast<size_t>(which);
    return c->sched.data() + row * c->nterms;
}

}  // namespace

int msgpu_set_hamiltonian_schedule(msgpu_ctx *c, const double *coef, long long first_step, long long nsteps)
{
    return set_schedule(c, coef, first_step, nsteps, 1);
}

int msgpu_set_hamiltonian_schedule_rk4(msgpu_ctx *c, const double *coef, long long first_step, long long nsteps)
{
    return set_schedule(c, coef, first_step, nsteps, 2);
}

int msgpu_upload_factors(msgpu_ctx *c, int dim, int ntraj, const double *factors)
{
    return upload_factors_impl(c, dim, ntraj, factors, cudaMemcpyHostToDevice);
}

int msgpu_upload_factors_device(msgpu_ctx *c, int dim, int ntraj, const void *factors)
{
    return upload_factors_impl(c, dim, ntraj, factors, cudaMemcpyDeviceToDevice);
}

int msgpu_download_factors(msgpu_ctx *c, double *factors)
{
    if (!c) return MSGPU_ERR_INVALID;
    if (c->state_prec < 0 || !factors) return fail(c, MSGPU_ERR_STATE, "no trajectory state to download");
    if (int rc = device_guard(c)) return rc;
    const size_t sbytes = static_cast<size_t>(c->D) * c->M * sizeof(double2);
    // a complex64 state is widened into the complex128 state first (exact)
    if (c->state_prec == MSGPU_PREC_C64)
        if (int rc = ensure_state(c, MSGPU_PREC_C128)) return rc;
    if (int rc = ensure(c, c->zbuf, sbytes, "download staging")) return rc;
    dim3 grid(ceil_div(c->D, 32), c->ldm / 32), block(32, 8);
    {
        Timed tm(c, KC_COMBINE);
        k_interleaved_to_cols<double2><<<grid, block, 0, c->stream>>>(
            static_cast<double2 *>(c->zbuf.p), static_cast<const double2 *>(c->psi128.p), c->D, c->M, c->ldm);
    }
    cudaError_t e;
    if ((e = cudaGetLastError()) || (e = cudaMemcpyAsync(factors, c->zbuf.p, sbytes, cudaMemcpyDeviceToHost, c->stream)) ||
        (e = cudaStreamSynchronize(c->stream)))
        return cuda_fail(c, e, "factors download");
    return MSGPU_OK;
}

int msgpu_run(msgpu_ctx *c, const msgpu_run_params *p)
{
    if (!c) return MSGPU_ERR_INVALID;
    c->prof_tick = -1;
    if (!p || !p->times || p->ntimes < 1) return fail(c, MSGPU_ERR_INVALID, "run: a time grid with at least one point is required");
    if (c->D == 0) return fail(c, MSGPU_ERR_STATE, "run: no Hamiltonian uploaded");
    if (c->state_prec < 0) return fail(c, MSGPU_ERR_STATE, "run: no trajectory factors uploaded");
    if (c->s1 == 0) return fail(c, MSGPU_ERR_STATE, "run: electron pair strides not set");
    if (c->D % (2 * c->s1) != 0) return fail(c, MSGPU_ERR_INVALID, "run: electron strides inconsistent with the Hilbert dimension");
    if (c->obs.empty()) return fail(c, MSGPU_ERR_STATE, "run: no observables");
    for (int s = 0; s < p->ntimes; ++s)
        if (!std::isfinite(p->times[s]) || (s > 0 && !(p->times[s] > p->times[s - 1])))
            return fail(c, MSGPU_ERR_INVALID, "run: times must be finite and strictly increasing");
    if (c->sched_steps && (p->step_offset < c->sched_first ||
                           p->step_offset + (p->ntimes - 1) > c->sched_first + c->sched_steps))
        return fail(c, MSGPU_ERR_INVALID, "run: the Hamiltonian schedule does not cover the requested steps");
    if (p->propagator == MSGPU_PROP_DENSE) {
        if (c->sched_steps) return fail(c, MSGPU_ERR_INVALID, "run: the dense propagator needs a time-independent H");
        if (p->precision != MSGPU_PREC_BF16X3 && p->precision != MSGPU_PREC_BF16X6 &&
            p->precision != MSGPU_PREC_INT8X4)
            return fail(c, MSGPU_ERR_INVALID,
                        "run: the dense propagator takes MSGPU_PREC_BF16X3, MSGPU_PREC_BF16X6 or MSGPU_PREC_INT8X4");
        if (c->D > 4096) return fail(c, MSGPU_ERR_INVALID, "run: the dense propagator is limited to dimension 4096");
        if (c->noise_mode == MSGPU_NOISE_REPLAY &&
            (c->bits_ntraj != c->M || p->step_offset < 0 || p->step_offset + (p->ntimes - 1) > c->bits_steps))
            return fail(c, MSGPU_ERR_INVALID, "run: replay bits do not cover the requested steps");
        if (p->accumulate && !c->have_integrals) return fail(c, MSGPU_ERR_STATE, "run: nothing to continue (accumulate=1)");
        if (int rc = device_guard(c)) return rc;
        return run_dense(c, p);
    }
    if (p->precision != MSGPU_PREC_C128 && p->precision != MSGPU_PREC_C64)
        return fail(c, MSGPU_ERR_INVALID, "run: unknown precision");
    const bool rk4 = p->propagator == MSGPU_PROP_RK4;
    const bool taylor = p->propagator == MSGPU_PROP_TAYLOR;
    if (p->propagator != MSGPU_PROP_KRYLOV && !taylor && !rk4) return fail(c, MSGPU_ERR_INVALID, "run: unknown propagator");
    if ((taylor || rk4) && p->precision != MSGPU_PREC_C128)
        return fail(c, MSGPU_ERR_INVALID, "run: the Taylor and RK4 propagators are complex128 only");
    if (rk4 && c->sched_steps && c->sched_rows != 2)
        return fail(c, MSGPU_ERR_INVALID,
                    "run: RK4 with a time-dependent H needs the start, midpoint and end coefficients of every step "
                    "(msgpu_set_hamiltonian_schedule_rk4)");
    if (!taylor && !rk4 && (p->krylov_dim < 1 || p->krylov_dim > kMaxKrylov))
        return fail(c, MSGPU_ERR_INVALID, "run: krylov_dim must be in 1..32");
    int rec = p->recurrence;
    if (rec == MSGPU_REC_AUTO || taylor || rk4)
        rec = (p->precision == MSGPU_PREC_C64 && c->k_scalar) ? MSGPU_REC_LANCZOS : MSGPU_REC_ARNOLDI;
    if (rec == MSGPU_REC_LANCZOS && !c->k_scalar)
        return fail(c, MSGPU_ERR_INVALID, "run: Lanczos requires a scalar reaction operator K");
    PairK pair_k{};  // K on the electron pair, for the complex64 Arnoldi form
    if (p->precision == MSGPU_PREC_C64 && rec == MSGPU_REC_ARNOLDI && !pair_reaction(c, &pair_k))
        return fail(c, MSGPU_ERR_INVALID,
                    "run: the complex64 Arnoldi form needs K acting on the electron pair only (K = I x K4, e.g. "
                    "unequal sinks on the pair's states); use complex128 for a general K");
    if (p->precision == MSGPU_PREC_C128 && rec != MSGPU_REC_ARNOLDI)
        return fail(c, MSGPU_ERR_INVALID, "run: the complex128 form implements the Arnoldi recurrence only");
    if (c->noise_mode == MSGPU_NOISE_REPLAY) {
        if (c->bits_ntraj != c->M) return fail(c, MSGPU_ERR_INVALID, "run: replay bits cover a different trajectory count");
        if (p->step_offset < 0 || p->step_offset + (p->ntimes - 1) > c->bits_steps)
            return fail(c, MSGPU_ERR_INVALID, "run: replay bits do not cover the requested steps");
    }
    if (p->accumulate && !c->have_integrals) return fail(c, MSGPU_ERR_STATE, "run: nothing to continue (accumulate=1)");
    if (int rc = device_guard(c)) return rc;

    const int D = c->D, ldm = c->ldm, M = c->M;
    const int m = (taylor || rk4) ? 1 : std::min(p->krylov_dim, D);  // no Krylov basis (RK4 uses slot 0 as its sum)
    const int prec = p->precision;
    if (!taylor && !rk4 && resident_warps(c, prec, m) > 0) return run_resident(c, p, prec, m);
    if (c->form == MSGPU_FORM_RESIDENT)
        return fail(c, MSGPU_ERR_INVALID, "run: the resident form does not fit this dimension / recurrence / propagator");
    const int nobs = static_cast<int>(c->obs.size());
    const size_t n = static_cast<size_t>(D) * ldm;
    // The complex64 state lives in slot 0 of the Lanczos basis: park it in the
    // complex128 state before that buffer is reused or reallocated.
    if (c->state_prec == MSGPU_PREC_C64) {
        const size_t need = n * (m + 1) * sizeof(float2);
        if (prec != MSGPU_PREC_C64 || c->basis.bytes < need)
            if (int rc = ensure_state(c, MSGPU_PREC_C128)) return rc;
    }
    if (int rc = ensure_workspace(c, prec, m)) return rc;
    if (prec == MSGPU_PREC_C64 && rec == MSGPU_REC_ARNOLDI) {
        // the complex64 Arnoldi form's Hessenberg matrices, dots and Gram-Schmidt partials
        int rc;
        if ((rc = ensure(c, c->hess, static_cast<size_t>(ldm) * m * m * sizeof(double2), "Hessenberg")) ||
            (rc = ensure(c, c->part2, static_cast<size_t>(3) * (m + 1) * ldm * sizeof(double2), "dots")) ||
            (rc = ensure(c, c->wbuf, static_cast<size_t>(c->ntiles) * (m + 1) * ldm * sizeof(double2), "partials")))
            return rc;
    }
    if (int rc = ensure_state(c, prec)) return rc;
    const int mws = m;  // layout stride of the per-trajectory Krylov arrays
    cudaError_t e;
    cudaStream_t st = c->stream;
    if ((e = cudaMemcpyAsync(c->rates_d.p, c->rates.data(), nobs * sizeof(double), cudaMemcpyHostToDevice, st)) ||
        (e = cudaMemsetAsync(c->status.p, 0, sizeof(int), st)))
        return cuda_fail(c, e, "run setup");
    if (!p->accumulate) {
        if ((e = cudaMemsetAsync(c->acc.p, 0, static_cast<size_t>(nobs) * ldm * sizeof(double), st)) ||
            (e = cudaMemsetAsync(c->comp.p, 0, static_cast<size_t>(nobs) * ldm * sizeof(double), st)))
            return cuda_fail(c, e, "run setup");
    }
    if (int rc = ensure(c, c->values_d, static_cast<size_t>(p->ntimes) * nobs * sizeof(double), "values")) return rc;

    const PairObs po = make_pair_obs(c);
    Noise nz;
    nz.mode = c->noise_mode;
    nz.bits = static_cast<const uint8_t *>(c->bits.p);
    nz.bits_steps = c->bits_steps;
    nz.M = c->noise_mode == MSGPU_NOISE_REPLAY ? c->bits_ntraj : M;
    nz.seed = c->seed;
    nz.traj_offset = 0;
    nz.p_full = 0.0;
    const int steps = p->ntimes - 1;
    const long long g0 = p->step_offset;
    auto pstep = [&](int s) { return s < steps ? flip_p(c->st_rate, 0.5 * (p->times[s + 1] - p->times[s])) : 0.0; };

    const int Q = D / 4, QR = c->quartets_per_tile, qt = c->qtiles;
    dim3 qgrid(qt, ldm / 32), qblock(32, 8);
    double *values = static_cast<double *>(c->values_d.p);
    double *sc = static_cast<double *>(c->scale.p);  // [m+1][ldm]; slot 0 = 1/|psi|
    double *beta0 = static_cast<double *>(c->beta0.p);
    auto yield_update = [&](double dt, int init, int row) {
        Timed tm(c, KC_YIELD);
        ++c->launches;  // two kernels: per trajectory, then the ensemble value
        k_yield_traj<<<dim3(ceil_div(ldm, 128), nobs + 1), 128, 0, st>>>(
            static_cast<double *>(c->qpart_obs.p), static_cast<double *>(c->qpart_nrm.p), qt, nobs, ldm,
            static_cast<double *>(c->rates_d.p), dt, init, static_cast<double *>(c->prev.p),
            static_cast<double *>(c->acc.p), static_cast<double *>(c->comp.p), beta0, sc,
            static_cast<int *>(c->status.p));
        k_yield_values<<<1, 1024, 0, st>>>(static_cast<double *>(c->prev.p), nobs, ldm, M,
                                           values + static_cast<size_t>(row) * nobs);
    };

    // Evaluate the first time point and apply the first half-step flip.
    {
        Timed tm(c, KC_COMBINE);
        const long long sB = -1;
        if (prec == MSGPU_PREC_C128)
            k_combine<double2, false><<<qgrid, qblock, 0, st>>>(
                static_cast<double2 *>(c->psi128.p), nullptr, 0, nullptr, nullptr, mws, c->s1, c->s2, Q, ldm, QR, nz,
                steps > 0 ? g0 : -1, 0, pstep(0), sB, 0, 0.0, po, static_cast<double *>(c->qpart_obs.p),
                static_cast<double *>(c->qpart_nrm.p));
        else
            k_combine_pp<false><<<dim3(qt, ldm / 64), qblock, 0, st>>>(
                static_cast<float2 *>(c->basis.p), nullptr, 0, nullptr, nullptr, c->s1, c->s2, Q, ldm, QR, nz,
                steps > 0 ? g0 : -1, 0, pstep(0), sB, 0, 0.0, po, static_cast<double *>(c->qpart_obs.p),
                static_cast<double *>(c->qpart_nrm.p));
    }
    yield_update(0.0, 1, 0);
    int fused_c = 0;  // cluster size of k_lanczos_fused, 0: the four-kernel iteration
    const bool arn64 = prec == MSGPU_PREC_C64 && rec == MSGPU_REC_ARNOLDI;
    // the complex128 Arnoldi apply runs over quartet blocks when K = kappa I
    const bool quartet128 = prec == MSGPU_PREC_C128 && !taylor && !rk4 && c->k_scalar;
    if (quartet128)
        if (int rc = build_quartet(c)) return rc;
    if (prec == MSGPU_PREC_C64) {
        if (int rc = build_quartet(c)) return rc;
        if (int rc = build_tc(c)) return rc;
        if (int rc = tc_prepare_map(c)) return rc;
        fused_c = arn64 ? 0 : fused_cluster(c);
        if (!fused_c)
            if (int rc = tune_quartet_tile(c, static_cast<const float2 *>(c->basis.p), sc,
                                           static_cast<float2 *>(c->ubuf.p), static_cast<double *>(c->part.p)))
                return rc;
    }

    const int R = c->rows_per_tile, nt = c->ntiles;
    CsrD Hd{static_cast<const int *>(c->hrow.p), static_cast<const int *>(c->hcol.p), static_cast<const double2 *>(c->hval.p)};
    CsrD Kd{c->k_scalar ? nullptr : static_cast<const int *>(c->krow.p), static_cast<const int *>(c->kcol.p),
            static_cast<const double2 *>(c->kval.p)};
    const double kappa = c->k_scalar ? c->kappa : 0.0;
    const size_t expm_smem_warp = (4 * static_cast<size_t>(m) * m + m) * sizeof(double2);
    const int expm_warps = std::max(1, std::min(8, static_cast<int>(160 * 1024 / expm_smem_warp)));
    if ((e = raise_smem_limit(reinterpret_cast<const void *>(k_krylov_expm), static_cast<int>(expm_warps * expm_smem_warp))))
        return cuda_fail(c, e, "expm shared memory");

    // Taylor propagator: the shift mu = trace(G)/D and a bound on ||G - mu I||_1
    double2 tmu = make_double2(0.0, 0.0);
    double tnorm = 0.0;
    std::vector<double> term_stats;  // per term {tr.re, tr.im, max row sum} when a schedule drives H
    if (taylor && c->sched_steps) {
        if (int rc = ensure(c, c->work_d, 4 * sizeof(double), "Taylor statistics")) return rc;
        term_stats.resize(3 * static_cast<size_t>(c->nterms));
        for (int k = 0; k < c->nterms; ++k) {
            CsrD Tk{Hd.rowptr, Hd.col, static_cast<const double2 *>(c->hterms.p) + static_cast<size_t>(k) * c->nnz};
            k_g_stats<<<1, 256, 0, st>>>(Tk, D, static_cast<double *>(c->work_d.p));
            if ((e = cudaMemcpyAsync(&term_stats[3 * k], c->work_d.p, 3 * sizeof(double), cudaMemcpyDeviceToHost, st)) ||
                (e = cudaStreamSynchronize(st)))
                return cuda_fail(c, e, "Taylor statistics");
        }
    }
    // shift and norm bound of G - mu I from the H statistics {tr.re, tr.im, max row sum}
    auto taylor_shift = [&](const double *hs) {
        const double2 ktr = c->k_scalar ? make_double2(c->kappa * D, 0.0) : c->k_trace;
        const double kn = c->k_scalar ? std::abs(c->kappa) : c->k_norm1;
        // trace(G) = -i trace(H) - trace(K)
        tmu = make_double2((hs[1] - ktr.x) / D, (-hs[0] - ktr.y) / D);
        tnorm = hs[2] + kn + std::hypot(tmu.x, tmu.y);
    };
    if (taylor && !c->sched_steps) {
        if (int rc = ensure(c, c->work_d, 4 * sizeof(double), "Taylor statistics")) return rc;
        k_g_stats<<<1, 256, 0, st>>>(Hd, D, static_cast<double *>(c->work_d.p));
        double hs[3] = {0.0, 0.0, 0.0};
        if ((e = cudaMemcpyAsync(hs, c->work_d.p, sizeof(hs), cudaMemcpyDeviceToHost, st)) ||
            (e = cudaStreamSynchronize(st)))
            return cuda_fail(c, e, "Taylor statistics");
        taylor_shift(hs);
        if (!std::isfinite(tnorm)) return fail(c, MSGPU_ERR_NONFINITE, "run: non-finite Hamiltonian norm");
    }
    for (int s = 0; s < steps; ++s) {
        c->prof_tick = s;
        const double dt = p->times[s + 1] - p->times[s];
        const long long g = g0 + s;
        if (c->sched_steps && !rk4) {
            // H at this step's midpoint from the schedule: combine the terms
            // on the device, refresh the quartet values of the complex64 form
            const double *row = sched_row(c, g, 1);
            TermCoef cf;
            std::memset(&cf, 0, sizeof(cf));
            double hs[3] = {0.0, 0.0, 0.0};
            for (int k = 0; k < c->nterms; ++k) {
                cf.c[k] = row[k];
                if (taylor) {
                    hs[0] += row[k] * term_stats[3 * k];
                    hs[1] += row[k] * term_stats[3 * k + 1];
                    hs[2] += std::abs(row[k]) * term_stats[3 * k + 2];  // norm bound of the combination
                }
            }
            k_combine_terms<<<ceil_div(std::max(1, c->nnz), 256), 256, 0, st>>>(
                static_cast<const double2 *>(c->hterms.p), c->nterms, cf, c->nnz, static_cast<double2 *>(c->hval.p),
                static_cast<float2 *>(c->hhi.p), static_cast<float2 *>(c->hlo.p), static_cast<int *>(c->status.p));
            if (prec == MSGPU_PREC_C64 || quartet128)
                if (int rc = refresh_quartet_values(c)) return rc;
            if (taylor) taylor_shift(hs);
        }
        if ((e = cudaMemsetAsync(c->mdim.p, 0, ldm * sizeof(int), st))) return cuda_fail(c, e, "mdim reset");
        if (taylor) {
            // exp(dt (G - mu I)) by s sub-steps of a degree-mt Taylor series
            // (theta^(mt+1)/(mt+1)! e^theta <= tol with theta = |dt| ||G - mu I||_1 / s <= 4),
            // each ending with F <- e^{dt mu / s} F (SpinSpace::HighamProp's loop)
            double2 *F = static_cast<double2 *>(c->psi128.p);
            double2 *cur = static_cast<double2 *>(c->wbuf.p), *nxt = static_cast<double2 *>(c->zbuf.p);
            const int nsub = std::max(1, static_cast<int>(std::ceil(std::abs(dt) * tnorm / 4.0)));
            const double theta = std::abs(dt) * tnorm / nsub;
            int mt = 1;
            for (double rem = theta * theta / 2.0; rem * std::exp(theta) > c->taylor_tol && mt < 55; ++mt)
                rem *= theta / (mt + 2);
            const double er = std::exp(dt * tmu.x / nsub), ea = dt * tmu.y / nsub;
            const double2 eta = make_double2(er * std::cos(ea), er * std::sin(ea));
            if ((e = cudaMemcpyAsync(cur, F, n * sizeof(double2), cudaMemcpyDeviceToDevice, st)))
                return cuda_fail(c, e, "Taylor step");
            dim3 tgrid(ceil_div(D, 8), ldm / 32), tblock(32, 8);
            for (int sub = 0; sub < nsub; ++sub) {
                for (int k = 1; k <= mt; ++k) {
                    Timed tm(c, KC_APPLY);
                    k_taylor_term<<<tgrid, tblock, 0, st>>>(Hd, Kd, kappa, tmu, cur, nxt, F, dt / (nsub * k), D, ldm);
                    std::swap(cur, nxt);
                }
                Timed tm(c, KC_ORTH);
                k_taylor_rescale<<<static_cast<unsigned>((n + 255) / 256), 256, 0, st>>>(F, cur, eta, n);
            }
            {
                Timed tm(c, KC_COMBINE);
                k_combine<double2, false><<<qgrid, qblock, 0, st>>>(
                    F, nullptr, 0, nullptr, nullptr, mws, c->s1, c->s2, Q, ldm, QR, nz, g, 1, pstep(s),
                    s + 1 < steps ? g + 1 : -1, 0, pstep(s + 1), po, static_cast<double *>(c->qpart_obs.p),
                    static_cast<double *>(c->qpart_nrm.p));
            }
        } else if (rk4) {
            double2 *psi = static_cast<double2 *>(c->psi128.p);
            double2 *ya = static_cast<double2 *>(c->wbuf.p), *yb = static_cast<double2 *>(c->zbuf.p);
            double2 *acc = static_cast<double2 *>(c->basis.p);
            dim3 tgrid(ceil_div(D, 8), ldm / 32), tblock(32, 8);
            const double cs[4] = {0.5 * dt, 0.5 * dt, dt, 0.0}, ws[4] = {dt / 6.0, dt / 3.0, dt / 3.0, dt / 6.0};
            const double2 *in[4] = {psi, ya, yb, ya};
            double2 *out[4] = {ya, yb, ya, nullptr};
            for (int stage = 0; stage < 4; ++stage) {
                if (c->sched_steps && stage != 2) {
                    // dynamic RK4 (HSPropagator.cpp:104-128): G at the step's start
                    // (stage 1), midpoint (stages 2, 3) and end (stage 4); the
                    // stages are stream-ordered, so H is recombined in place
                    const double *row = sched_row(c, g, stage == 0 ? 0 : stage == 1 ? 1 : 2);
                    TermCoef cf;
                    std::memset(&cf, 0, sizeof(cf));
                    for (int k = 0; k < c->nterms; ++k) cf.c[k] = row[k];
                    k_combine_terms<<<ceil_div(std::max(1, c->nnz), 256), 256, 0, st>>>(
                        static_cast<const double2 *>(c->hterms.p), c->nterms, cf, c->nnz,
                        static_cast<double2 *>(c->hval.p), static_cast<float2 *>(c->hhi.p),
                        static_cast<float2 *>(c->hlo.p), static_cast<int *>(c->status.p));
                }
                Timed tm(c, KC_APPLY);
                k_rk4_stage<<<tgrid, tblock, 0, st>>>(Hd, Kd, kappa, in[stage], psi, out[stage], acc, cs[stage],
                                                      ws[stage], stage + 1, D, ldm);
            }
            {
                Timed tm(c, KC_COMBINE);
                k_combine<double2, false><<<qgrid, qblock, 0, st>>>(
                    psi, nullptr, 0, nullptr, nullptr, mws, c->s1, c->s2, Q, ldm, QR, nz, g, 1, pstep(s),
                    s + 1 < steps ? g + 1 : -1, 0, pstep(s + 1), po, static_cast<double *>(c->qpart_obs.p),
                    static_cast<double *>(c->qpart_nrm.p));
            }
        } else if (prec == MSGPU_PREC_C128) {
            double2 *V = static_cast<double2 *>(c->basis.p);
            double2 *bufA = static_cast<double2 *>(c->wbuf.p), *bufB = static_cast<double2 *>(c->zbuf.p);
            double2 *dots = static_cast<double2 *>(c->part2.p);  // [3][m+1][ldm]: h1, h2, norm
            double2 *h1 = dots, *h2 = dots + static_cast<size_t>(m + 1) * ldm, *nr = dots + 2 * static_cast<size_t>(m + 1) * ldm;
            const double2 *src = static_cast<const double2 *>(c->psi128.p);
            double2 *W = bufA;
            dim3 grid(nt, ldm / 32);
            for (int j = 0; j < m; ++j) {
                {
                    Timed tm(c, KC_APPLY);
                    if (quartet128)
                        k_arnoldi_apply_q<<<dim3(ceil_div(Q, kWarps), ldm / 32), kThreads, 0, st>>>(
                            QuartetD{static_cast<const int *>(c->qrow.p), static_cast<const int2 *>(c->qcolt.p),
                                     static_cast<const double2 *>(c->qval64.p), static_cast<const int *>(c->qbase.p)},
                            kappa, src, j == 0 ? sc : sc + ldm, V + j * n, W, Q, c->s1, c->s2, ldm);
                    else
                        k_arnoldi_apply<<<grid, kThreads, 0, st>>>(Hd, Kd, kappa, src, j == 0 ? sc : sc + ldm, V + j * n,
                                                                   W, D, ldm, R);
                    arnoldi_orth_fn(j, 0)<<<grid, kThreads, 0, st>>>(W, V, n, nullptr, static_cast<double2 *>(c->part.p), D,
                                                                     ldm, R);
                }
                {
                    Timed tm(c, KC_REDUCE);
                    k_reduce_partials<<<dim3(ldm / 32, j + 1), dim3(32, 8), 0, st>>>(
                        static_cast<double2 *>(c->part.p), nt, j + 1, ldm, h1);
                }
                {
                    Timed tm(c, KC_ORTH);
                    arnoldi_orth_fn(j, 1)<<<grid, kThreads, 0, st>>>(W, V, n, h1, static_cast<double2 *>(c->part.p), D, ldm, R);
                }
                {
                    Timed tm(c, KC_REDUCE);
                    k_reduce_partials<<<dim3(ldm / 32, j + 1), dim3(32, 8), 0, st>>>(
                        static_cast<double2 *>(c->part.p), nt, j + 1, ldm, h2);
                }
                {
                    Timed tm(c, KC_ORTH);
                    arnoldi_orth_fn(j, 2)<<<grid, kThreads, 0, st>>>(W, V, n, h2, static_cast<double2 *>(c->part.p), D, ldm, R);
                }
                {
                    Timed tm(c, KC_REDUCE);
                    k_reduce_partials<<<dim3(ldm / 32, 1), dim3(32, 8), 0, st>>>(static_cast<double2 *>(c->part.p), nt, 1, ldm, nr);
                    k_arnoldi_finalize<<<ceil_div(ldm, 256), 256, 0, st>>>(h1, h2, nr, j, mws, ldm,
                                                                           static_cast<double2 *>(c->hess.p),
                                                                           static_cast<int *>(c->mdim.p), sc + ldm);
                }
                // next iteration reads W scaled by 1/beta; write into the other buffer
                src = W;
                W = (W == bufA) ? bufB : bufA;
            }
            {
                Timed tm(c, KC_EXPM);
                k_krylov_expm<<<ceil_div(ldm, expm_warps), 32 * expm_warps, expm_warps * expm_smem_warp, st>>>(
                    static_cast<double2 *>(c->hess.p), nullptr, nullptr, 0.0, static_cast<int *>(c->mdim.p), beta0,
                    nullptr, mws, ldm, M, dt, static_cast<double2 *>(c->coef.p), static_cast<int *>(c->status.p));
            }
            {
                Timed tm(c, KC_COMBINE);
                k_combine<double2, true><<<qgrid, qblock, 0, st>>>(
                    static_cast<double2 *>(c->psi128.p), V, n, static_cast<double2 *>(c->coef.p),
                    static_cast<int *>(c->mdim.p), mws, c->s1, c->s2, Q, ldm, QR, nz, g, 1, pstep(s),
                    s + 1 < steps ? g + 1 : -1, 0, pstep(s + 1), po, static_cast<double *>(c->qpart_obs.p),
                    static_cast<double *>(c->qpart_nrm.p));
            }
        } else if (arn64) {
            // complex64 Arnoldi (CGS2) for K = I (x) K4: basis slot j holds w_j with
            // scale sc[j] = 1/|w_j|, as the Lanczos form; one trajectory group
            float2 *Wb = static_cast<float2 *>(c->basis.p);
            float2 *U = static_cast<float2 *>(c->ubuf.p);
            double2 *dots = static_cast<double2 *>(c->part2.p);  // [3][m+1][ldm]: h1, h2, norm
            double2 *h1 = dots, *h2 = dots + static_cast<size_t>(m + 1) * ldm, *nr = dots + 2 * static_cast<size_t>(m + 1) * ldm;
            double2 *apart = static_cast<double2 *>(c->wbuf.p);  // Gram-Schmidt partials [tile][i][t]
            const int QT = c->q_tile;
            const dim3 ogrid(nt, ldm / 32);
            for (int j = 0; j < m; ++j) {
                float2 *Wn = Wb + static_cast<size_t>(j + 1) * n;
                {
                    Timed tm(c, KC_APPLY);
                    launch_apply(c, c->q_variant, QT, dim3(ceil_div(Q, std::max(1, QT))), st, Wb + j * n,
                                 sc + static_cast<size_t>(j) * ldm, U, static_cast<double *>(c->part.p), ldm);
                    k_arn64_apply<<<dim3(ceil_div(Q, kWarps), ldm / 64), kThreads, 0, st>>>(
                        pair_k, U, Wb + j * n, sc + static_cast<size_t>(j) * ldm, Wn, Q, c->s1, c->s2, ldm);
                }
                {
                    Timed tm(c, KC_ORTH);
                    arn64_orth_fn(j, 0)<<<ogrid, kThreads, 0, st>>>(Wn, Wb, n, sc, nullptr, apart, D, ldm, R);
                    k_reduce_partials<<<dim3(ldm / 32, j + 1), dim3(32, 8), 0, st>>>(apart, nt, j + 1, ldm, h1);
                    arn64_orth_fn(j, 1)<<<ogrid, kThreads, 0, st>>>(Wn, Wb, n, sc, h1, apart, D, ldm, R);
                    k_reduce_partials<<<dim3(ldm / 32, j + 1), dim3(32, 8), 0, st>>>(apart, nt, j + 1, ldm, h2);
                    arn64_orth_fn(j, 2)<<<ogrid, kThreads, 0, st>>>(Wn, Wb, n, sc, h2, apart, D, ldm, R);
                    k_reduce_partials<<<dim3(ldm / 32, 1), dim3(32, 8), 0, st>>>(apart, nt, 1, ldm, nr);
                    k_arnoldi_finalize<<<ceil_div(ldm, 256), 256, 0, st>>>(
                        h1, h2, nr, j, mws, ldm, static_cast<double2 *>(c->hess.p), static_cast<int *>(c->mdim.p),
                        sc + static_cast<size_t>(j + 1) * ldm);
                }
            }
            {
                Timed tm(c, KC_EXPM);
                k_krylov_expm<<<ceil_div(ldm, expm_warps), 32 * expm_warps, expm_warps * expm_smem_warp, st>>>(
                    static_cast<double2 *>(c->hess.p), nullptr, nullptr, 0.0, static_cast<int *>(c->mdim.p), beta0, sc,
                    mws, ldm, M, dt, static_cast<double2 *>(c->coef.p), static_cast<int *>(c->status.p));
            }
            {
                Timed tm(c, KC_COMBINE);
                k_combine_pp<true><<<dim3(qt, ldm / 64), qblock, 0, st>>>(
                    Wb, Wb, n, static_cast<double2 *>(c->coef.p), static_cast<int *>(c->mdim.p), c->s1, c->s2, Q, ldm,
                    QR, nz, g, 1, pstep(s), s + 1 < steps ? g + 1 : -1, 0, pstep(s + 1), po,
                    static_cast<double *>(c->qpart_obs.p), static_cast<double *>(c->qpart_nrm.p));
            }
        } else {
            float2 *Wb = static_cast<float2 *>(c->basis.p);  // w_0 = state
            float2 *U = static_cast<float2 *>(c->ubuf.p);
            double *part = static_cast<double *>(c->part.p);
            double *alpha = static_cast<double *>(c->alpha.p);
            double *td = static_cast<double *>(c->tdiag.p), *to = static_cast<double *>(c->toff.p);
            int *mdim = static_cast<int *>(c->mdim.p);
            double2 *coef = static_cast<double2 *>(c->coef.p);
            double *qobs = static_cast<double *>(c->qpart_obs.p), *qnrm = static_cast<double *>(c->qpart_nrm.p);
            const int QT = c->q_tile, nqt = ceil_div(Q, std::max(1, QT));
            if (fused_c) {
                Timed tm(c, KC_LANCZOS);
                if (int rc = launch_fused(c, fused_c, Wb, n, sc, td, to, mdim, m)) return rc;
            }
            // Trajectory groups: every kernel below works on columns [t0, t0 + width)
            // through offset pointers with the row stride ldm, so the groups share
            // the buffers. With overlap, odd groups run on the second stream and
            // one group's SpMM runs beside another's update and combine; profiled
            // steps run the groups back to back so that each launch is timed alone.
            const int G = fused_c ? 1 : traj_groups(c), width = ldm / G;
            const bool timed_step = c->prof == 1 || (c->prof == 2 && c->prof_tick % kProfileEvery == 0);
            const bool overlap = G > 1 && !timed_step;
            // each group on its own stream (group 0 on the context stream)
            const int nside = overlap ? G - 1 : 0;
            if (overlap) {
                if (!c->gfork && (e = cudaEventCreateWithFlags(&c->gfork, cudaEventDisableTiming)))
                    return cuda_fail(c, e, "trajectory group stream");
                for (int k = 0; k < nside; ++k)
                    if (!c->gside[k] && ((e = cudaStreamCreateWithFlags(&c->gside[k], cudaStreamNonBlocking)) ||
                                         (e = cudaEventCreateWithFlags(&c->gjoin[k], cudaEventDisableTiming))))
                        return cuda_fail(c, e, "trajectory group stream");
                if ((e = cudaEventRecord(c->gfork, st))) return cuda_fail(c, e, "trajectory group fork");
                for (int k = 0; k < nside; ++k)
                    if ((e = cudaStreamWaitEvent(c->gside[k], c->gfork, 0))) return cuda_fail(c, e, "trajectory group fork");
            }
            for (int gi = 0; gi < G; ++gi) {
                const int t0 = gi * width;
                const size_t tm0 = static_cast<size_t>(t0) * mws;  // offset into the [t][m] T arrays
                cudaStream_t gs = (overlap && gi > 0) ? c->gside[gi - 1] : st;
                dim3 grid(nt, width / 64);
                for (int j = 0; j < (fused_c ? 0 : m); ++j) {
                    {
                        Timed tm(c, KC_APPLY, gs);
                        launch_apply(c, c->q_variant, QT, dim3(nqt), gs, Wb + j * n + t0,
                                     sc + static_cast<size_t>(j) * ldm + t0, U + t0, part + t0, width);
                    }
                    {
                        Timed tm(c, KC_REDUCE, gs);
                        k_lanczos_reduce<<<width / 32, dim3(32, kRedRows), 0, gs>>>(part + t0, nqt, ldm, 0, j, mws, alpha + t0,
                                                                             td + tm0, to + tm0, mdim + t0);
                    }
                    if (j == m - 1) break;  // T_m is complete; w_m is never used
                    {
                        Timed tm(c, KC_ORTH, gs);
                        k_lanczos_update<<<grid, kThreads, 0, gs>>>(
                            U + t0, Wb + j * n + t0, j > 0 ? Wb + (j - 1) * n + t0 : nullptr,
                            sc + static_cast<size_t>(j) * ldm + t0, j > 0 ? sc + static_cast<size_t>(j - 1) * ldm + t0 : nullptr,
                            alpha + t0, Wb + (j + 1) * n + t0, part + t0, D, ldm, R);
                    }
                    {
                        Timed tm(c, KC_REDUCE, gs);
                        k_lanczos_reduce<<<width / 32, dim3(32, kRedRows), 0, gs>>>(part + t0, nt, ldm, 1, j, mws,
                                                                             sc + static_cast<size_t>(j + 1) * ldm + t0,
                                                                             td + tm0, to + tm0, mdim + t0);
                    }
                }
                {
                    Timed tm(c, KC_EXPM, gs);
                    k_lanczos_expm<<<ceil_div(width, 8), 256, 0, gs>>>(
                        td + tm0, to + tm0, kappa, mdim + t0, beta0 + t0, sc + t0, mws, ldm,
                        std::max(0, std::min(M - t0, width)), dt, coef + t0, static_cast<int *>(c->status.p));
                }
                {
                    Timed tm(c, KC_COMBINE, gs);
                    Noise gnz = nz;
                    gnz.traj_offset = static_cast<uint32_t>(t0);
                    k_combine_pp<true><<<dim3(qt, width / 64), qblock, 0, gs>>>(
                        Wb + t0, Wb + t0, n, coef + t0, mdim + t0, c->s1, c->s2, Q, ldm, QR, gnz, g, 1, pstep(s),
                        s + 1 < steps ? g + 1 : -1, 0, pstep(s + 1), po, qobs + t0, qnrm + t0);
                }
            }
            for (int k = 0; k < nside; ++k)
                if ((e = cudaEventRecord(c->gjoin[k], c->gside[k])) || (e = cudaStreamWaitEvent(st, c->gjoin[k], 0)))
                    return cuda_fail(c, e, "trajectory group join");
        }
        yield_update(dt, 0, s + 1);
        if ((e = cudaGetLastError())) return cuda_fail(c, e, "step launch");
    }
    c->prof_tick = -1;
    int status = 0;
    c->last_values.assign(static_cast<size_t>(p->ntimes) * nobs, 0.0);
    if ((e = cudaMemcpyAsync(&status, c->status.p, sizeof(int), cudaMemcpyDeviceToHost, st)) ||
        (e = cudaMemcpyAsync(c->last_values.data(), values, c->last_values.size() * sizeof(double),
                             cudaMemcpyDeviceToHost, st)) ||
        (e = cudaStreamSynchronize(st)))
        return cuda_fail(c, e, "run");
    collect_profile(c);
    c->last_ntimes = p->ntimes;
    c->have_integrals = true;
    if (status & 4) return fail(c, MSGPU_ERR_CUDA, "run: tensor-core or TMEM-staged SpMM pipeline timed out (bounded wait expired)");
    if (status & 2) return fail(c, MSGPU_ERR_NONFINITE, "run: non-finite observable or norm on the device");
    if (status & 1) return fail(c, MSGPU_ERR_EXPM, "run: small matrix exponential failed");
    return MSGPU_OK;
}

int msgpu_fetch_yields(msgpu_ctx *c, double *per_traj, double *ensemble)
{
    if (!c) return MSGPU_ERR_INVALID;
    if (!c->have_integrals) return fail(c, MSGPU_ERR_STATE, "no yields: run first");
    if (int rc = device_guard(c)) return rc;
    const int nobs = static_cast<int>(c->obs.size()), ldm = c->ldm, M = c->M;
    std::vector<double> acc(static_cast<size_t>(nobs) * ldm);
    cudaError_t e;
    if ((e = cudaMemcpyAsync(acc.data(), c->acc.p, acc.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream)) ||
        (e = cudaStreamSynchronize(c->stream)))
        return cuda_fail(c, e, "fetch yields");
    for (int o = 0; o < nobs; ++o) {
        double s = 0.0;
        for (int t = 0; t < M; ++t) {
            const double v = acc[static_cast<size_t>(o) * ldm + t];
            if (per_traj) per_traj[static_cast<size_t>(t) * nobs + o] = v;
            s += v;
        }
        if (ensemble) ensemble[o] = s;
    }
    return MSGPU_OK;
}

int msgpu_fetch_values(msgpu_ctx *c, double *values)
{
    if (!c) return MSGPU_ERR_INVALID;
    if (!c->have_integrals || !values) return fail(c, MSGPU_ERR_STATE, "no values: run first");
    std::copy(c->last_values.begin(), c->last_values.end(), values);
    return MSGPU_OK;
}

int msgpu_spmm_choice(const msgpu_ctx *c, int *variant, int *tile, int *groups)
{
    if (!c) return MSGPU_ERR_INVALID;
    const bool tuned = c->q_tile > 0;
    if (variant) *variant = tuned ? c->q_variant : -1;
    if (tile) *tile = tuned ? c->q_tile : -1;
    if (groups) *groups = tuned ? traj_groups(c) : -1;
    return MSGPU_OK;
}

int msgpu_profile_enable(msgpu_ctx *c, int enable)
{
    if (!c) return MSGPU_ERR_INVALID;
    if (enable < 0 || enable > 2) return fail(c, MSGPU_ERR_INVALID, "profile: mode must be 0, 1 or 2");
    c->prof = enable;
    for (int k = 0; k < KC_N; ++k) { c->prof_ms[k] = 0.0; c->prof_n[k] = 0; }
    return MSGPU_OK;
}

int msgpu_profile_read(msgpu_ctx *c, int cls, double *total_ms, long long *launches)
{
    if (!c || cls < 0 || cls >= KC_N) return MSGPU_ERR_INVALID;
    collect_profile(c);
    if (total_ms) *total_ms = c->prof_ms[cls];
    if (launches) *launches = c->prof_n[cls];
    return MSGPU_OK;
}

}  // extern "C"

// ============================================================================
// Allocation-free Krylov step (msgpu_krylov_step_noalloc).
//
// Some callers cannot call cudaMalloc: hosts whose memory pool owns every
// device allocation, code that must not take the implicit device
// synchronisation of cudaMalloc / cudaFree, or embedders that must bound
// device memory at load time.  For
// them this entry point runs one complex128 Arnoldi step with all of its
// temporaries in one static device array.  The array lives in this library
// image, so every GPU that loads the library holds MSGPU_NOALLOC_SCRATCH_BYTES
// until the process exits.  Host code may not use the array's name as a
// device address (on the host it names a stand-in object), so the address is
// looked up once per device with cudaGetSymbolAddress and passed to kernels.
// ============================================================================

static __device__ __align__(256) unsigned char g_noalloc_scratch[MSGPU_NOALLOC_SCRATCH_BYTES];

namespace {

constexpr int kNoallocMaxDevices = 64;
std::mutex g_noalloc_mutex;
void *g_noalloc_ptr[kNoallocMaxDevices] = {};

// Device address of the scratch array on the current device.  It is looked
// up on the first call per device; later calls check that the cached address
// still belongs to a live device allocation of that device (a
// cudaDeviceReset unloads the library image and the array moves when the
// context is recreated) and look it up again when it does not.
cudaError_t noalloc_scratch(void **out)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kNoallocMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (g_noalloc_ptr[dev]) {
        cudaPointerAttributes attr;
        const cudaError_t ae = cudaPointerGetAttributes(&attr, g_noalloc_ptr[dev]);
        if (ae != cudaSuccess || attr.type != cudaMemoryTypeDevice || attr.device != dev) {
            if (ae != cudaSuccess) (void)cudaGetLastError();  // this probe's own error only
            g_noalloc_ptr[dev] = nullptr;
        }
    }
    if (!g_noalloc_ptr[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return e;
        g_noalloc_ptr[dev] = p;
    }
    *out = g_noalloc_ptr[dev];
    return cudaSuccess;
}

// Carves 256-byte aligned sub-buffers out of the scratch array.
struct Carve {
    unsigned char *base;
    size_t off = 0;
    template <typename T>
    T *take(size_t n)
    {
        T *p = reinterpret_cast<T *>(base + off);
        off += (n * sizeof(T) + 255) / 256 * 256;
        return p;
    }
};

}  // namespace

extern "C" int msgpu_krylov_step_noalloc(int dim, const int *rowptr, const int *col, const double *val,
                                         double kappa, int ntraj, const double *psi_in, double *psi_out, double dt,
                                         int krylov_dim, void *stream)
{
    if (dim < 4 || dim % 4 != 0 || ntraj <= 0 || !rowptr || !col || !val || !psi_in || !psi_out)
        return MSGPU_ERR_INVALID;
    if (krylov_dim < 1 || krylov_dim > kMaxKrylov || !std::isfinite(dt) || !(dt > 0.0) || !std::isfinite(kappa))
        return MSGPU_ERR_INVALID;
    // The state alone takes 16 bytes per (row, trajectory) and dim >= 4, so a
    // trajectory count above this bound cannot fit; refusing it here keeps the
    // index arithmetic below free of overflow.
    if (static_cast<size_t>(ntraj) > MSGPU_NOALLOC_SCRATCH_BYTES / 64) return MSGPU_ERR_SCRATCH;
    if (static_cast<size_t>(dim) > MSGPU_NOALLOC_SCRATCH_BYTES / 16) return MSGPU_ERR_SCRATCH;
    // An error the caller left pending belongs to the caller: report it
    // without clearing it, before queuing anything.
    if (cudaPeekAtLastError() != cudaSuccess) return MSGPU_ERR_CUDA;
    const int D = dim, m = std::min(krylov_dim, dim);
    const int ldm = (ntraj + 63) / 64 * 64;
    const size_t n = static_cast<size_t>(D) * ldm;
    const int R = pick_rows_per_tile(D), nt = ceil_div(D, R);
    const int Q = D / 4, QR = std::max(8, std::min(256, Q / 64)), qt = ceil_div(Q, QR);
    // Sizes of every temporary, checked against the static capacity before
    // anything is queued.
    Carve probe{nullptr};
    probe.take<double2>(n);                                  // interleaved state
    probe.take<double2>(n * m);                              // Krylov basis
    probe.take<double2>(n);                                  // W
    probe.take<double2>(n);                                  // Z
    probe.take<double2>(static_cast<size_t>(nt) * (m + 1) * ldm);  // partials
    probe.take<double2>(static_cast<size_t>(3) * (m + 1) * ldm);   // dots
    probe.take<double2>(static_cast<size_t>(ldm) * m * m);   // Hessenberg
    probe.take<double2>(static_cast<size_t>(ldm) * m);       // coefficients
    probe.take<int>(ldm);                                    // Krylov dims
    probe.take<double>(static_cast<size_t>(m + 1) * ldm);    // scales
    probe.take<double>(ldm);                                 // beta0
    probe.take<double>(static_cast<size_t>(qt) * ldm);       // norm partials
    probe.take<double>(8);                                   // observable partials (none used)
    probe.take<int>(1);                                      // status
    if (probe.off > MSGPU_NOALLOC_SCRATCH_BYTES) return MSGPU_ERR_SCRATCH;

    void *base = nullptr;
    if (noalloc_scratch(&base) != cudaSuccess) return MSGPU_ERR_CUDA;
    Carve cv{static_cast<unsigned char *>(base)};
    double2 *psi = cv.take<double2>(n);
    double2 *V = cv.take<double2>(n * m);
    double2 *bufA = cv.take<double2>(n);
    double2 *bufB = cv.take<double2>(n);
    double2 *part = cv.take<double2>(static_cast<size_t>(nt) * (m + 1) * ldm);
    double2 *dots = cv.take<double2>(static_cast<size_t>(3) * (m + 1) * ldm);
    double2 *hess = cv.take<double2>(static_cast<size_t>(ldm) * m * m);
    double2 *coef = cv.take<double2>(static_cast<size_t>(ldm) * m);
    int *mdim = cv.take<int>(ldm);
    double *sc = cv.take<double>(static_cast<size_t>(m + 1) * ldm);
    double *beta0 = cv.take<double>(ldm);
    double *qnrm = cv.take<double>(static_cast<size_t>(qt) * ldm);
    double *qobs = cv.take<double>(8);
    int *status = cv.take<int>(1);

    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // Contents left by the previous call are stale: clear what must start at zero.
    if (cudaMemsetAsync(status, 0, sizeof(int), st) != cudaSuccess ||
        cudaMemsetAsync(mdim, 0, ldm * sizeof(int), st) != cudaSuccess)
        return MSGPU_ERR_CUDA;
    {
        dim3 grid(ceil_div(D, 32), ldm / 32), block(32, 8);
        k_cols_to_interleaved<double2><<<grid, block, 0, st>>>(psi, reinterpret_cast<const double2 *>(psi_in), D,
                                                               ntraj, ldm);
    }
    PairObs po;
    std::memset(&po, 0, sizeof(po));
    Noise nz;
    std::memset(&nz, 0, sizeof(nz));
    dim3 qgrid(qt, ldm / 32), qblock(32, 8);
    // any two spin-1/2 digit strides partition the rows into quartets; without
    // observables or flips only the norms are read from the quartet pass
    const int s1 = D / 2, s2 = D / 4;
    k_combine<double2, false><<<qgrid, qblock, 0, st>>>(psi, nullptr, 0, nullptr, nullptr, m, s1, s2, Q, ldm, QR, nz,
                                                        -1, 0, 0.0, -1, 0, 0.0, po, qobs, qnrm);
    k_yield_update<<<1, 1024, 0, st>>>(qobs, qnrm, qt, 0, ldm, ntraj, nullptr, 0.0, 1, nullptr, nullptr, nullptr,
                                       beta0, sc, nullptr, status);
    CsrD Hd{rowptr, col, reinterpret_cast<const double2 *>(val)};
    CsrD Kd{nullptr, nullptr, nullptr};
    double2 *h1 = dots, *h2 = dots + static_cast<size_t>(m + 1) * ldm, *nr = dots + 2 * static_cast<size_t>(m + 1) * ldm;
    const double2 *src = psi;
    double2 *W = bufA;
    dim3 grid(nt, ldm / 32);
    for (int j = 0; j < m; ++j) {
        k_arnoldi_apply<<<grid, kThreads, 0, st>>>(Hd, Kd, kappa, src, j == 0 ? sc : sc + ldm, V + j * n, W, D, ldm, R);
        arnoldi_orth_fn(j, 0)<<<grid, kThreads, 0, st>>>(W, V, n, nullptr, part, D, ldm, R);
        k_reduce_partials<<<dim3(ldm / 32, j + 1), dim3(32, 8), 0, st>>>(part, nt, j + 1, ldm, h1);
        arnoldi_orth_fn(j, 1)<<<grid, kThreads, 0, st>>>(W, V, n, h1, part, D, ldm, R);
        k_reduce_partials<<<dim3(ldm / 32, j + 1), dim3(32, 8), 0, st>>>(part, nt, j + 1, ldm, h2);
        arnoldi_orth_fn(j, 2)<<<grid, kThreads, 0, st>>>(W, V, n, h2, part, D, ldm, R);
        k_reduce_partials<<<dim3(ldm / 32, 1), dim3(32, 8), 0, st>>>(part, nt, 1, ldm, nr);
        k_arnoldi_finalize<<<ceil_div(ldm, 256), 256, 0, st>>>(h1, h2, nr, j, m, ldm, hess, mdim, sc + ldm);
        src = W;
        W = (W == bufA) ? bufB : bufA;
    }
    const size_t smem_warp = (4 * static_cast<size_t>(m) * m + m) * sizeof(double2);
    const int warps = std::max(1, std::min(8, static_cast<int>(160 * 1024 / smem_warp)));
    if (raise_smem_limit(reinterpret_cast<const void *>(k_krylov_expm), static_cast<int>(warps * smem_warp)) != cudaSuccess)
        return MSGPU_ERR_CUDA;
    k_krylov_expm<<<ceil_div(ldm, warps), 32 * warps, warps * smem_warp, st>>>(hess, nullptr, nullptr, 0.0, mdim, beta0,
                                                                              nullptr, m, ldm, ntraj, dt, coef, status);
    k_combine<double2, true><<<qgrid, qblock, 0, st>>>(psi, V, n, coef, mdim, m, s1, s2, Q, ldm, QR, nz, -1, 0, 0.0,
                                                       -1, 0, 0.0, po, qobs, qnrm);
    {
        dim3 g(ceil_div(D, 32), ldm / 32), b(32, 8);
        k_interleaved_to_cols<double2><<<g, b, 0, st>>>(reinterpret_cast<double2 *>(psi_out), psi, D, ntraj, ldm);
    }
    if (cudaGetLastError() != cudaSuccess) return MSGPU_ERR_CUDA;
    int h_status = 0;
    if (cudaMemcpyAsync(&h_status, status, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return MSGPU_ERR_CUDA;
    if (h_status & 2) return MSGPU_ERR_NONFINITE;
    if (h_status & 1) return MSGPU_ERR_EXPM;
    return MSGPU_OK;
}

