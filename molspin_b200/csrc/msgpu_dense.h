// msgpu_dense.h -- internal host interface of the dense tensor-core form
// (msgpu_dense.cu), used by msgpu_api.cu for MSGPU_PROP_DENSE.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include <string>

namespace msgpu {

struct DenseState {
    int D = 0, Dp = 0;        // dimension, padded real-interleaved size 2D rounded up to 128
    int M = 0, Mp = 0;        // trajectories, padded to the GEMM N tile
    int parts = 0;            // BF16 split depth (2 or 3), or 4: int8 slices (exact accumulation)
    double dt = 0.0;          // step U was built for
    bool have_u = false;
    void *u_parts = nullptr;  // parts x Dp x Dp bf16 (real interleaved U, K-major rows)
    void *psi = nullptr;      // Mp x Dp fp32 (fp64 for int8), trajectory-major (interleaved complex per trajectory)
    void *b_parts = nullptr;  // parts x Mp x Dp bf16 (split state, K-major rows); int8 slices for parts = 4
    void *u_scale = nullptr;  // int8 form: Dp doubles, the power-of-two scale of each row of U (in u_parts)
    void *b_scale = nullptr;  // int8 form: Mp doubles, the scale of each trajectory's slices (in b_parts)
    void *work = nullptr;     // FP64 scratch for building U (4 x D x D complex)
    void *tmaps = nullptr;    // device copy not needed: tensor maps are kernel parameters
    size_t bytes = 0;
    // second trajectory group: its GEMMs and epilogues run on `side`, so one
    // group's epilogue overlaps the other group's GEMM
    cudaStream_t side = nullptr;
    cudaEvent_t e_main = nullptr, e_side = nullptr;
};

// Arguments of the dense run that come from the context.
struct DenseRun {
    const int *rowptr, *col;  // H CSR on the device
    const double *val;        // interleaved complex128
    const int *krow, *kcol;   // K CSR or null
    const double *kval;
    double kappa;
    int s1, s2;               // electron strides
    int nobs;
    const double *obs;        // device: nobs x 16 complex (kernel pair basis)
    const double *obs_host;   // host copy of the same operators
    const double *rates;      // device: nobs
    int noise_mode;
    const unsigned char *bits;
    long long bits_steps;
    int bits_ntraj;
    unsigned long long seed;
    double *acc, *comp, *prev;  // device: nobs x acc_ld
    int acc_ld;
    double *values;             // device: ntimes x nobs (ensemble per time point)
    const double *times;        // host
    int ntimes;
    long long step_offset;
    int accumulate;
    double st_rate;
    int renormalize;            // restore the exact Haberkorn survival norm each step (scalar K only)
    int *status;                // device status word
    double *part;               // device: 2 x ntimes x nobs per-group ensemble partials
};

// Allocates (budget-checked by the caller through *alloc) and prepares the
// dense state: U = expm(dt(-iH-K)) in FP64, split into BF16 parts; the
// trajectory block is taken from psi128_interleaved (ldm x D complex128).
int dense_prepare(DenseState &st, int D, int M, int ldm, int parts, double dt, const DenseRun &run,
                  const void *psi128_interleaved, cudaStream_t stream, std::string &err,
                  int (*alloc)(void *ctx, void **p, size_t bytes, const char *what), void *alloc_ctx);

// Runs the time loop; returns MSGPU_* status (err filled on failure); the
// final state is written back to psi128_interleaved.
int dense_run(DenseState &st, const DenseRun &run, void *psi128_interleaved, int ldm, cudaStream_t stream,
              std::string &err, float *gemm_ms, long long *gemm_launches, int gemm_every = 1);

void dense_release(DenseState &st, void (*release)(void *ctx, void *p), void *ctx);

}  // namespace msgpu
