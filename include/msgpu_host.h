/* msgpu_host.h -- host-side helpers of the msgpu library (no GPU needed).
 *
 * MolSpin keeps Hamiltonian assembly and trace sampling on the host in C++;
 * these helpers provide the same products for standalone use of msgpu
 * (benchmarks, the serving loop, tests) without Armadillo:
 *
 *  - msgpu_host_build_hamiltonian: H = sum of linear terms w.S_k and bilinear
 *    terms S_i^T C S_j, in rad/ns, as CSR over the Kronecker product basis of
 *    the given spin multiplicities (first spin most significant, digit 0 =
 *    m=+S).  Mirrors SpinSpace::InteractionOperator (Zeeman S.(G.B) and
 *    bilinear S1.A.S2, SpinAPI/SpinSpace/SpinSpace_hamiltonians.cpp:438-535)
 *    summed by SpinSpace::Hamiltonian (:1456-1524) with the single-spin
 *    embedding of SpinSpace::CreateOperator (SpinSpace_operators.cpp:65-106).
 *  - msgpu_host_trace_samples: SU(Z) trace samples of the tensor fast path of
 *    SpinSpace::BuildTraceSamples (SpinSpace_states.cpp:452-486) from a
 *    std::mt19937 seeded as HSStatePreparation::SeedGenerator
 *    (HSStatePreparation.cpp:167-181), scaled by 1/sqrt(M) as
 *    HSStatePreparation::Prepare (:221-226).
 *  - msgpu_host_reference_flip_bits: the reference's singlet-triplet flip
 *    stream (StochasticRelaxationGenerator + std::bernoulli_distribution,
 *    SpinSpace_relaxation.cpp:1201-1254, consumed as StepStochastic does)
 *    packed for MSGPU_NOISE_REPLAY.
 *  - msgpu_host_philox_flip_bits: the device Philox stream as bits, so a
 *    Philox run can be replayed by any other implementation.
 *  - msgpu_host_time_grid: the exact-endpoint grid of TaskHSGeneral.cpp:59-96.
 */
#ifndef MSGPU_HOST_H
#define MSGPU_HOST_H

#ifdef __cplusplus
extern "C" {
#endif

/* Two-call protocol: with rowptr == NULL returns nnz (>= 0) or -1 on error;
 * otherwise fills rowptr[dim+1], col[nnz], val[2*nnz] and returns nnz.
 * lin_w: 3 per linear term; bil_c: 9 per bilinear term (row-major C). */
long long msgpu_host_build_hamiltonian(int nspins, const int *mult, int nlin, const int *lin_spin,
                                       const double *lin_w, int nbil, const int *bil_i, const int *bil_j,
                                       const double *bil_c, int *rowptr, int *col, double *val);

/* out: D x M column-major complex, D = F * Z; fixed is the F-dimensional
 * fixed (leading) state; returns 0 on success. */
int msgpu_host_trace_samples(double seed, const double *fixed, int F, int Z, int M, double *out);


/* The reference flip stream for several dephasing Operators on the same
 * electron pair (st_rates: each Operator's rate; event rate = rate / 2):
 * ApplyStochasticRelaxationHilbert's superposed-Poisson branch
 * (SpinSpace_relaxation.cpp:1239-1252) -- per half step and trajectory one
 * Poisson count of mean (sum of event rates) h and one discrete channel draw
 * per event, from the same generator as msgpu_host_reference_flip_bits.
 * Every channel applies P_S - P_T, so the bit is the parity of the count;
 * replay it with MSGPU_NOISE_REPLAY and st_rate = the sum of the rates.  One
 * rate reduces to msgpu_host_reference_flip_bits.  Returns 0 on success. */
int msgpu_host_reference_flip_bits_multi(double seed, int seed_mode, unsigned long long orientation,
                                         const double *st_rates, int nterms, const double *times, int ntimes, int M,
                                         unsigned char *bits);

/* bits: ((ntimes-1)*2*M + 7)/8 bytes.  seed_mode 0: stream of orientation
 * `orientation` derived from the task seed; 1: std::mt19937(seed) directly. */
int msgpu_host_reference_flip_bits(double seed, int seed_mode, unsigned long long orientation, double st_rate,
                                   const double *times, int ntimes, int M, unsigned char *bits);

int msgpu_host_philox_flip_bits(unsigned long long seed, unsigned int traj_offset, long long step_offset,
                                double st_rate, const double *times, int ntimes, int M, unsigned char *bits);

/* Returns the number of points (<= cap written) or -1. */
long msgpu_host_time_grid(double total, double dt, double *times, long cap);

#ifdef __cplusplus
}
#endif

#endif /* MSGPU_HOST_H */
