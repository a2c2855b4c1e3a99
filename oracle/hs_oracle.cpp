// hs_oracle.cpp -- CPU oracle for the HSGeneral stochastic Hilbert-space path.
//
// TEST INFRASTRUCTURE ONLY.  This file is a plain C++17 restatement of the
// reference algorithm (MolSpin HSGeneral, sampling=stochastic) used to check
// the CUDA implementation.  Only tests/, __graft_entry__.smoke() and the
// cpu_baseline / reference legs of bench.py load it.  The product path never
// links, loads or calls anything from oracle/.
//
// Parity pins: the reference (C++17 + Armadillo 12.8.4) cannot be built here
// because Armadillo is absent, so this restatement is pinned against the
// reference's own known-answer tests (Haberkorn survival law, singlet-triplet
// analytic coherence law, per-column norm, Monte-Carlo RMS law, seeded
// reproducibility and zero-rate no-op, yield-correction closed form, split
// order, stochastic-vs-density agreement); see tests/test_oracle_pins.py.
//
// What follows which reference function (paths relative to the MolSpin tree):
//   time grid ............ RunSection/General/HS/TaskHSGeneral.cpp:59-96
//   loop order ........... TaskHSGeneral.cpp:471-560 (Evaluate, then step)
//   seeding .............. HSStatePreparation.cpp:167-181, TaskHSGeneral.cpp:292-295
//   trace samples ........ SpinAPI/SpinSpace/SpinSpace_states.cpp:452-486
//                          (+ 1/sqrt(M) scaling HSStatePreparation.cpp:221-226)
//   generator G=-iH-K .... RunSection/General/HS/HSPropagator.cpp:56
//   Krylov branch ........ HSPropagator.cpp:64-78
//   dense branch ......... HSPropagator.cpp:92-100
//   split step ........... HSPropagator.cpp:131-140
//   KrylovExpmGeneral .... SpinAPI/SpinSpace/SpinSpace_operators.cpp:1257-1304
//   ArnoldiProcess ....... SpinSpace_operators.cpp:1352-1408 (MGS, breakdown 1e-14)
//   ST projectors ........ SpinAPI/SpinSpace/SpinSpace_relaxation.cpp:1144-1169
//   ST cache ............. SpinSpace_relaxation.cpp:1171-1199 (U=PS-PT, rate/2)
//   noise RNG stream ..... SpinSpace_relaxation.cpp:1201-1209
//   flip application ..... SpinSpace_relaxation.cpp:1211-1254
//   Evaluate ............. RunSection/General/HS/HSObservableCollector.cpp:276-288
//   trapezoid ............ HSObservableCollector.cpp:304-326
//   yield correction ..... HSObservableCollector.cpp:361-392
//
// Third-party arithmetic restated: Armadillo 12.8.4 (Dockerfile pin) expmat()
// is documented as a Pade approximation with scaling and squaring; here the
// published Golub & Van Loan (Matrix Computations, Alg. 11.3.1) form with
// diagonal Pade degree q=6 is used, solved by LU with partial pivoting.
// libstdc++ <random> (std::mt19937, std::seed_seq, std::normal_distribution,
// std::bernoulli_distribution) is used directly, so the random streams are the
// reference's own when built with the same standard library (GCC 13.3 here).

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <limits>
#include <random>
#include <string>
#include <thread>
#include <vector>

namespace {

using cd = std::complex<double>;

struct Csr {
    int n = 0;
    std::vector<int> rowptr, col;
    std::vector<cd> val;
};

Csr make_csr(int n, const int *rowptr, const int *col, const double *val)
{
    Csr a;
    a.n = n;
    if (!rowptr) return a;
    const int nnz = rowptr[n];
    a.rowptr.assign(rowptr, rowptr + n + 1);
    a.col.assign(col, col + nnz);
    a.val.resize(nnz);
    for (int k = 0; k < nnz; ++k) a.val[k] = cd(val[2 * k], val[2 * k + 1]);
    return a;
}

void csr_matvec(const Csr &a, const cd *x, cd *y)
{
    for (int r = 0; r < a.n; ++r) {
        cd s = 0.0;
        for (int k = a.rowptr[r]; k < a.rowptr[r + 1]; ++k) s += a.val[k] * x[a.col[k]];
        y[r] = s;
    }
}

// Sparse sum alpha*A + beta*B (both n x n CSR, columns sorted or not).
Csr csr_axpby(cd alpha, const Csr &a, cd beta, const Csr &b)
{
    Csr c;
    c.n = a.n;
    c.rowptr.assign(a.n + 1, 0);
    std::vector<cd> acc(a.n, cd(0.0));
    std::vector<int> mark(a.n, -1), cols;
    for (int r = 0; r < a.n; ++r) {
        cols.clear();
        auto add = [&](const Csr &m, cd s) {
            if (m.rowptr.empty()) return;
            for (int k = m.rowptr[r]; k < m.rowptr[r + 1]; ++k) {
                int j = m.col[k];
                if (mark[j] != r) { mark[j] = r; acc[j] = 0.0; cols.push_back(j); }
                acc[j] += s * m.val[k];
            }
        };
        add(a, alpha);
        add(b, beta);
        std::sort(cols.begin(), cols.end());
        for (int j : cols) { c.col.push_back(j); c.val.push_back(acc[j]); }
        c.rowptr[r + 1] = static_cast<int>(c.col.size());
    }
    return c;
}

Csr csr_identity(int n, cd s)
{
    Csr c;
    c.n = n;
    c.rowptr.resize(n + 1);
    c.col.resize(n);
    c.val.assign(n, s);
    for (int i = 0; i <= n; ++i) c.rowptr[i] = i;
    for (int i = 0; i < n; ++i) c.col[i] = i;
    return c;
}

// ---------------------------------------------------------------- dense helpers
// Column-major n x n complex matrices.
void matmul(int n, const cd *a, const cd *b, cd *c)
{
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) {
            cd s = 0.0;
            for (int k = 0; k < n; ++k) s += a[i + k * n] * b[k + j * n];
            c[i + j * n] = s;
        }
}

// Solve A X = B (A n x n, B n x nrhs), LU with partial pivoting; A, B overwritten.
bool lu_solve(int n, cd *a, cd *b, int nrhs)
{
    for (int k = 0; k < n; ++k) {
        int p = k;
        double best = std::abs(a[k + k * n]);
        for (int i = k + 1; i < n; ++i) {
            double v = std::abs(a[i + k * n]);
            if (v > best) { best = v; p = i; }
        }
        if (best == 0.0) return false;
        if (p != k) {
            for (int j = 0; j < n; ++j) std::swap(a[k + j * n], a[p + j * n]);
            for (int j = 0; j < nrhs; ++j) std::swap(b[k + j * n], b[p + j * n]);
        }
        const cd piv = a[k + k * n];
        for (int i = k + 1; i < n; ++i) {
            const cd f = a[i + k * n] / piv;
            a[i + k * n] = f;
            for (int j = k + 1; j < n; ++j) a[i + j * n] -= f * a[k + j * n];
            for (int j = 0; j < nrhs; ++j) b[i + j * n] -= f * b[k + j * n];
        }
    }
    for (int j = 0; j < nrhs; ++j)
        for (int i = n - 1; i >= 0; --i) {
            cd s = b[i + j * n];
            for (int k = i + 1; k < n; ++k) s -= a[i + k * n] * b[k + j * n];
            b[i + j * n] = s / a[i + i * n];
        }
    return true;
}

// Matrix exponential: scaling and squaring with the diagonal (6,6) Pade
// approximant, Golub & Van Loan Alg. 11.3.1 (the algorithm family documented
// for Armadillo expmat).  out = exp(a); a is n x n column-major.
bool expm_pade6(int n, const cd *a_in, cd *out)
{
    const int q = 6;
    std::vector<cd> a(a_in, a_in + n * n);
    double norm = 0.0;  // infinity norm
    for (int i = 0; i < n; ++i) {
        double s = 0.0;
        for (int j = 0; j < n; ++j) s += std::abs(a[i + j * n]);
        norm = std::max(norm, s);
    }
    if (!std::isfinite(norm)) return false;
    int sc = 0;
    if (norm > 0.0) sc = std::max(0, 1 + static_cast<int>(std::floor(std::log2(norm))));
    const double scale = std::ldexp(1.0, -sc);
    for (auto &v : a) v *= scale;
    std::vector<cd> N(n * n, 0.0), D(n * n, 0.0), X(n * n, 0.0), T(n * n);
    for (int i = 0; i < n; ++i) N[i + i * n] = D[i + i * n] = X[i + i * n] = 1.0;
    double c = 1.0;
    for (int k = 1; k <= q; ++k) {
        c = c * (q - k + 1) / static_cast<double>((2 * q - k + 1) * k);
        matmul(n, a.data(), X.data(), T.data());
        X.swap(T);
        const double sgn = (k % 2 == 0) ? 1.0 : -1.0;
        for (int i = 0; i < n * n; ++i) { N[i] += c * X[i]; D[i] += sgn * c * X[i]; }
    }
    if (!lu_solve(n, D.data(), N.data(), n)) return false;
    for (int s = 0; s < sc; ++s) {
        matmul(n, N.data(), N.data(), T.data());
        N.swap(T);
    }
    std::copy(N.begin(), N.end(), out);
    return true;
}

double vnorm(int n, const cd *x)
{
    double s = 0.0;
    for (int i = 0; i < n; ++i) s += std::norm(x[i]);
    return std::sqrt(s);
}

// KrylovExpmGeneral + ArnoldiProcess (fixed dimension, MGS, breakdown 1e-14).
// out = exp(dt*G) b.  Workspace is per call, as in the reference.
void krylov_expm_general(const Csr &G, const cd *b, double dt, int kry, cd *out)
{
    const int D = G.n;
    kry = std::max(1, std::min(kry, D));
    const double beta = vnorm(D, b);
    if (beta == 0.0) { std::fill(out, out + D, cd(0.0)); return; }
    std::vector<cd> V(static_cast<size_t>(D) * kry, 0.0), Hm(kry * kry, 0.0), z(D);
    for (int i = 0; i < D; ++i) V[i] = b[i] / beta;
    int actual = 0;
    for (int j = 0; j < kry; ++j) {
        csr_matvec(G, &V[static_cast<size_t>(j) * D], z.data());
        for (int i = 0; i <= j; ++i) {
            const cd *vi = &V[static_cast<size_t>(i) * D];
            cd h = 0.0;
            for (int r = 0; r < D; ++r) h += std::conj(vi[r]) * z[r];
            Hm[i + j * kry] = h;
            for (int r = 0; r < D; ++r) z[r] -= h * vi[r];
        }
        const double zn = vnorm(D, z.data());
        if (j == kry - 1) { actual = j + 1; break; }
        Hm[(j + 1) + j * kry] = zn;
        if (zn < 1e-14) { actual = j + 1; break; }
        cd *vn = &V[static_cast<size_t>(j + 1) * D];
        for (int r = 0; r < D; ++r) vn[r] = z[r] / zn;
        actual = j + 1;
    }
    const int m = actual;
    std::vector<cd> Hs(m * m), E(m * m);
    for (int j = 0; j < m; ++j)
        for (int i = 0; i < m; ++i) Hs[i + j * m] = Hm[i + j * kry] * dt;
    expm_pade6(m, Hs.data(), E.data());
    for (int r = 0; r < D; ++r) {
        cd s = 0.0;
        for (int j = 0; j < m; ++j) s += V[static_cast<size_t>(j) * D + r] * E[j];
        out[r] = beta * s;
    }
}

// ------------------------------------------------------------ spin operators
// Single-spin matrices in the reference basis order m = +s ... -s
// (SpinAPI/Spin.cpp SzFromCollection: diag[i] = s/2 - i with s = 2S).
void spin_matrices(int mult, std::vector<cd> &sx, std::vector<cd> &sy, std::vector<cd> &sz)
{
    const int n = mult;
    const double S = 0.5 * (mult - 1);
    sx.assign(n * n, 0.0); sy.assign(n * n, 0.0); sz.assign(n * n, 0.0);
    for (int i = 0; i < n; ++i) {
        const double m = S - i;
        sz[i + i * n] = m;
        if (i + 1 < n) {
            // <m|S+|m-1> = sqrt(S(S+1) - m(m-1)); row i (m), col i+1 (m-1)
            const double c = std::sqrt(S * (S + 1) - m * (m - 1));
            sx[i + (i + 1) * n] += 0.5 * c;
            sx[(i + 1) + i * n] += 0.5 * c;
            sy[i + (i + 1) * n] += cd(0.0, -0.5 * c);
            sy[(i + 1) + i * n] += cd(0.0, 0.5 * c);
        }
    }
}

// Embed a product of single-spin operators (dense, per spin) into the full
// space as CSR: op = coef * prod_k ops[k] acting on spin k (identity if null).
void add_product(const std::vector<int> &dims, const std::vector<const std::vector<cd> *> &ops, cd coef,
                 std::vector<std::vector<std::pair<int, cd>>> &rows)
{
    const int ns = static_cast<int>(dims.size());
    int D = 1;
    for (int d : dims) D *= d;
    std::vector<int> stride(ns);
    int s = 1;
    for (int k = ns - 1; k >= 0; --k) { stride[k] = s; s *= dims[k]; }
    std::vector<int> digit(ns);
    for (int r = 0; r < D; ++r) {
        int rem = r;
        for (int k = 0; k < ns; ++k) { digit[k] = rem / stride[k]; rem %= stride[k]; }
        // enumerate product of row entries
        std::vector<std::pair<int, cd>> cur{{0, coef}};
        for (int k = 0; k < ns; ++k) {
            std::vector<std::pair<int, cd>> nxt;
            if (!ops[k]) {
                for (auto &e : cur) nxt.push_back({e.first + digit[k] * stride[k], e.second});
            } else {
                const auto &m = *ops[k];
                for (int c = 0; c < dims[k]; ++c) {
                    const cd v = m[digit[k] + c * dims[k]];
                    if (v == cd(0.0)) continue;
                    for (auto &e : cur) nxt.push_back({e.first + c * stride[k], e.second * v});
                }
            }
            cur.swap(nxt);
        }
        for (auto &e : cur) rows[r].push_back(e);
    }
}

Csr rows_to_csr(int D, std::vector<std::vector<std::pair<int, cd>>> &rows)
{
    Csr a;
    a.n = D;
    a.rowptr.assign(D + 1, 0);
    for (int r = 0; r < D; ++r) {
        auto &row = rows[r];
        std::sort(row.begin(), row.end(), [](auto &x, auto &y) { return x.first < y.first; });
        int last = -1;
        for (auto &e : row) {
            if (e.first == last) { a.val.back() += e.second; continue; }
            a.col.push_back(e.first); a.val.push_back(e.second); last = e.first;
        }
        a.rowptr[r + 1] = static_cast<int>(a.col.size());
    }
    return a;
}

// SingletTripletProjectors + PrepareStochasticRelaxationHilbert:
// PS = 1/4 I - S1.S2, PT = I - PS, U = PS - PT.
Csr st_unitary(const std::vector<int> &dims, int e1, int e2)
{
    int D = 1;
    for (int d : dims) D *= d;
    std::vector<std::vector<std::pair<int, cd>>> rows(D);
    std::vector<cd> ax, ay, az, bx, by, bz;
    spin_matrices(dims[e1], ax, ay, az);
    spin_matrices(dims[e2], bx, by, bz);
    const int ns = static_cast<int>(dims.size());
    std::vector<const std::vector<cd> *> ops(ns, nullptr);
    // U = 2 PS - I = -1/2 I - 2 S1.S2
    std::vector<const std::vector<cd> *> id(ns, nullptr);
    add_product(dims, id, cd(-0.5), rows);
    const std::vector<cd> *A[3] = {&ax, &ay, &az}, *B[3] = {&bx, &by, &bz};
    for (int a = 0; a < 3; ++a) {
        std::fill(ops.begin(), ops.end(), nullptr);
        ops[e1] = A[a]; ops[e2] = B[a];
        add_product(dims, ops, cd(-2.0), rows);
    }
    Csr u = rows_to_csr(D, rows);
    // drop exact zeros produced by cancellation
    Csr c; c.n = D; c.rowptr.assign(D + 1, 0);
    for (int r = 0; r < D; ++r) {
        for (int k = u.rowptr[r]; k < u.rowptr[r + 1]; ++k)
            if (std::abs(u.val[k]) > 1e-15) { c.col.push_back(u.col[k]); c.val.push_back(u.val[k]); }
        c.rowptr[r + 1] = static_cast<int>(c.col.size());
    }
    return c;
}

// StochasticRelaxationGenerator: per-orientation stream derived from a copy
// of the seeded trace generator.
std::mt19937 relaxation_generator(std::mt19937 source, unsigned long long stream)
{
    std::vector<std::mt19937::result_type> seed{0x5354524cU, 0x554e4954U,
        static_cast<std::mt19937::result_type>(stream & 0xffffffffULL),
        static_cast<std::mt19937::result_type>(stream >> 32)};
    for (unsigned i = 0; i < 8; ++i) seed.push_back(source());
    std::seed_seq seq(seed.begin(), seed.end());
    return std::mt19937(seq);
}

std::mt19937 seeded(double seed)
{
    // HSStatePreparation::SeedGenerator: seed 0 maps to 1, cast to result_type.
    const double s = seed == 0.0 ? 1.0 : seed;
    std::mt19937 g;
    g.seed(static_cast<std::mt19937::result_type>(s));
    return g;
}

double flip_probability(double eventRate, double h)
{
    return -0.5 * std::expm1(-2.0 * eventRate * h);
}

struct Problem {
    int D = 0, M = 0;
    Csr G;          // -iH - K
    Csr U;          // ST unitary (may be empty)
    double eventRate = 0.0;
    std::vector<Csr> obs;
    std::vector<double> rates;
};

// One stochastic relaxation half step applied with a draw per column in
// column order (ApplyStochasticRelaxationHilbert, single involutory term).
void draw_flips(std::mt19937 &g, double p, int M, std::vector<unsigned char> &flip)
{
    flip.resize(M);
    std::bernoulli_distribution dist(p);
    for (int c = 0; c < M; ++c) flip[c] = dist(g) ? 1 : 0;
}

}  // namespace

extern "C" {

// Number of points of the exact-endpoint free-evolution grid, filling times
// (capacity cap) -- TaskHSGeneral.cpp:59-96.  Returns -1 on error.
long oracle_time_grid(double total, double dt, double *times, long cap)
{
    std::vector<double> t{0.0};
    if (total != 0.0) {
        const double ratio = total / dt;
        if (!std::isfinite(ratio)) return -1;
        const double nearest = std::round(ratio);
        const double tol = 64.0 * std::numeric_limits<double>::epsilon() * std::max(1.0, std::abs(ratio));
        const size_t intervals = static_cast<size_t>(
            nearest >= 1.0 && std::abs(ratio - nearest) <= tol ? nearest : std::ceil(ratio));
        for (size_t s = 1; s <= intervals; ++s) {
            const double target = s == intervals ? total : std::min(total, static_cast<double>(s) * dt);
            if (!(target > t.back())) return -1;
            t.push_back(target);
        }
    }
    if (times)
        for (long i = 0; i < static_cast<long>(t.size()) && i < cap; ++i) times[i] = t[i];
    return static_cast<long>(t.size());
}

// Dense matrix exponential (n x n, column-major, interleaved re/im).
int oracle_expm(int n, const double *a, double *out)
{
    std::vector<cd> A(n * n), E(n * n);
    for (int i = 0; i < n * n; ++i) A[i] = cd(a[2 * i], a[2 * i + 1]);
    if (!expm_pade6(n, A.data(), E.data())) return 1;
    for (int i = 0; i < n * n; ++i) { out[2 * i] = E[i].real(); out[2 * i + 1] = E[i].imag(); }
    return 0;
}

// Single-vector KrylovExpmGeneral with G = -iH - kappa I (H CSR).
int oracle_krylov_expm(int D, const int *rowptr, const int *col, const double *val, double kappa,
                       const double *b, double dt, int kry, double *out)
{
    Csr H = make_csr(D, rowptr, col, val);
    Csr G = csr_axpby(cd(0.0, -1.0), H, cd(-kappa), csr_identity(D, 1.0));
    std::vector<cd> x(D), y(D);
    for (int i = 0; i < D; ++i) x[i] = cd(b[2 * i], b[2 * i + 1]);
    krylov_expm_general(G, x.data(), dt, kry, y.data());
    for (int i = 0; i < D; ++i) { out[2 * i] = y[i].real(); out[2 * i + 1] = y[i].imag(); }
    return 0;
}

// ST unitary U = PS - PT for spins e1, e2 of a product space with the given
// multiplicities, as CSR.  Call with rowptr==NULL to get nnz (returned).
long oracle_st_unitary(int nspins, const int *dims, int e1, int e2, int *rowptr, int *col, double *val)
{
    std::vector<int> d(dims, dims + nspins);
    Csr u = st_unitary(d, e1, e2);
    if (rowptr) {
        std::copy(u.rowptr.begin(), u.rowptr.end(), rowptr);
        std::copy(u.col.begin(), u.col.end(), col);
        for (size_t k = 0; k < u.val.size(); ++k) { val[2 * k] = u.val[k].real(); val[2 * k + 1] = u.val[k].imag(); }
    }
    return static_cast<long>(u.col.size());
}

// SU(Z) trace samples, tensor fast path (SpinSpace_states.cpp:452-486), scaled
// by 1/sqrt(M) as HSStatePreparation::Prepare does.  Output D x M column-major.
// The generator is seeded as SeedGenerator does (autoseed=false).
int oracle_trace_samples(double seed, const double *fixed, int F, int Z, int M, double *out)
{
    std::mt19937 generator = seeded(seed);
    const double sqrtM = std::sqrt(static_cast<double>(M));
    std::vector<cd> fx(F);
    for (int i = 0; i < F; ++i) fx[i] = cd(fixed[2 * i], fixed[2 * i + 1]);
    std::vector<cd> chi(Z);
    for (int s = 0; s < M; ++s) {
        std::normal_distribution<double> distribution(0.0, 1.0);
        for (int i = 0; i < Z; ++i)
            chi[i] = std::complex<double>(distribution(generator), distribution(generator));
        const double nrm = vnorm(Z, chi.data());
        for (int i = 0; i < Z; ++i) chi[i] /= nrm;
        double *col = out + 2 * static_cast<size_t>(s) * F * Z;
        for (int a = 0; a < F; ++a)
            for (int i = 0; i < Z; ++i) {
                const cd v = (fx[a] * chi[i]) / sqrtM;  // normalise, kron, then factors /= sqrt(M)
                col[2 * (a * Z + i)] = v.real();
                col[2 * (a * Z + i) + 1] = v.imag();
            }
    }
    return 0;
}

// Reference flip stream as bits: bit ((s*2+half)*M + c) is the Bernoulli draw
// of column c in half step `half` of step s, consumed exactly as
// StepStochastic consumes the per-orientation generator.  seed_mode 0 derives
// the stream with StochasticRelaxationGenerator(seeded(seed), orientation);
// seed_mode 1 uses std::mt19937(seed) directly (as the reference unit tests).
int oracle_st_flip_bits(double seed, int seed_mode, unsigned long long orientation, double eventRate,
                        const double *times, int ntimes, int M, unsigned char *bits)
{
    std::mt19937 g = seed_mode == 0 ? relaxation_generator(seeded(seed), orientation)
                                    : std::mt19937(static_cast<std::mt19937::result_type>(seed));
    const int steps = ntimes - 1;
    std::memset(bits, 0, (static_cast<size_t>(steps) * 2 * M + 7) / 8);
    std::vector<unsigned char> f;
    for (int s = 0; s < steps; ++s) {
        const double h = 0.5 * (times[s + 1] - times[s]);
        if (eventRate <= 0.0 || h == 0.0) continue;  // no RNG consumption
        const double p = flip_probability(eventRate, h);
        for (int half = 0; half < 2; ++half) {
            draw_flips(g, p, M, f);
            for (int c = 0; c < M; ++c)
                if (f[c]) {
                    const size_t bit = (static_cast<size_t>(s) * 2 + half) * M + c;
                    bits[bit >> 3] |= static_cast<unsigned char>(1u << (bit & 7));
                }
        }
    }
    return 0;
}

// Several stochastic relaxation terms on the same electron pair (all with
// U = P_S - P_T): the reference's superposed-Poisson branch
// (ApplyStochasticRelaxationHilbert, SpinSpace_relaxation.cpp:1239-1252):
// per half step and column one Poisson count of mean (sum of event rates) h,
// then one discrete channel draw per event, in that order.  With every
// channel applying the same involution the column is flipped when the count
// is odd; bit layout as oracle_st_flip_bits.  One term reduces to
// oracle_st_flip_bits (the Bernoulli branch).
int oracle_st_flip_bits_multi(double seed, int seed_mode, unsigned long long orientation, const double *eventRates,
                              int nterms, const double *times, int ntimes, int M, unsigned char *bits)
{
    if (nterms < 1 || !eventRates) return 1;
    if (nterms == 1) return oracle_st_flip_bits(seed, seed_mode, orientation, eventRates[0], times, ntimes, M, bits);
    std::mt19937 g = seed_mode == 0 ? relaxation_generator(seeded(seed), orientation)
                                    : std::mt19937(static_cast<std::mt19937::result_type>(seed));
    double total = 0.0;
    for (int k = 0; k < nterms; ++k) {
        if (!(eventRates[k] > 0.0) || !std::isfinite(eventRates[k])) return 1;
        total += eventRates[k];
    }
    const int steps = ntimes - 1;
    std::memset(bits, 0, (static_cast<size_t>(steps) * 2 * M + 7) / 8);
    for (int s = 0; s < steps; ++s) {
        const double h = 0.5 * (times[s + 1] - times[s]);
        if (h == 0.0) continue;  // no RNG consumption
        for (int half = 0; half < 2; ++half) {
            std::poisson_distribution<unsigned long long> count(total * h);
            std::discrete_distribution<size_t> channel(eventRates, eventRates + nterms);
            for (int c = 0; c < M; ++c) {
                const unsigned long long events = count(g);
                for (unsigned long long e = 0; e < events; ++e) (void)channel(g);
                if (events & 1ULL) {
                    const size_t bit = (static_cast<size_t>(s) * 2 + half) * M + c;
                    bits[bit >> 3] |= static_cast<unsigned char>(1u << (bit & 7));
                }
            }
        }
    }
    return 0;
}

// One ApplyStochasticRelaxationHilbert call on D x M factors (in place), with
// a std::mt19937(seed) generator; U given as CSR.  Used by the analytic-law pins.
int oracle_apply_st(int D, const int *urow, const int *ucol, const double *uval, double eventRate,
                    double dt, unsigned int seed, int M, double *factors)
{
    if (!(dt >= 0.0)) return 1;
    if (eventRate <= 0.0 || dt == 0.0) return 0;
    Csr U = make_csr(D, urow, ucol, uval);
    std::mt19937 g(seed);
    std::bernoulli_distribution flip(flip_probability(eventRate, dt));
    std::vector<cd> x(D), y(D);
    for (int c = 0; c < M; ++c) {
        if (!flip(g)) continue;
        double *col = factors + 2 * static_cast<size_t>(c) * D;
        for (int i = 0; i < D; ++i) x[i] = cd(col[2 * i], col[2 * i + 1]);
        csr_matvec(U, x.data(), y.data());
        for (int i = 0; i < D; ++i) { col[2 * i] = y[i].real(); col[2 * i + 1] = y[i].imag(); }
    }
    return 0;
}

// Full stochastic finite-time loop for one orientation.
//   H: CSR (rad/ns); K: CSR or NULL with K = kappa I; G = -iH - K.
//   factors: D x M column-major (re,im), overwritten with the final state.
//   method: 0 = krylov (krylovsize kry), 1 = dense exponential of dt*G,
//     2 = classical RK4 on dB/dt = G B.
//   noise: U CSR (NULL for none) with event rate lambda (= k_ST/2);
//     noise_mode 0 = reference stream (seed, seed_mode, orientation as in
//     oracle_st_flip_bits), 1 = explicit flip bits (same layout).
//   observables: nobs CSR operators concatenated (obs_rowptr has nobs*(D+1)
//     entries; obs_nnz_off gives each operator's offset into col/val), rates
//     multiply each value (pass 1.0 for state populations).
//   outputs (nullable): values[(ntimes) x nobs] ensemble per time point,
//     traj_yield[M x nobs] per-column trapezoid integrals, yield[nobs].
int oracle_hs_stochastic(int D, int M,
                         const int *h_row, const int *h_col, const double *h_val,
                         const int *k_row, const int *k_col, const double *k_val, double kappa,
                         double *factors, const double *times, int ntimes, int method, int kry,
                         const int *u_row, const int *u_col, const double *u_val, double eventRate,
                         int noise_mode, double seed, int seed_mode, unsigned long long orientation,
                         const unsigned char *flip_bits,
                         int nobs, const int *obs_rowptr, const long *obs_nnz_off, const int *obs_col,
                         const double *obs_val, const double *rates,
                         double *values, double *traj_yield, double *yield, int nthreads)
{
    Csr H = make_csr(D, h_row, h_col, h_val);
    Csr K = k_row ? make_csr(D, k_row, k_col, k_val) : csr_identity(D, cd(kappa));
    Csr G = csr_axpby(cd(0.0, -1.0), H, cd(-1.0), K);
    Csr U;
    const bool noisy = u_row != nullptr && eventRate > 0.0;
    if (noisy) U = make_csr(D, u_row, u_col, u_val);
    std::vector<Csr> O(nobs);
    for (int o = 0; o < nobs; ++o) {
        O[o].n = D;
        const int *rp = obs_rowptr + static_cast<size_t>(o) * (D + 1);
        O[o].rowptr.assign(rp, rp + D + 1);
        const long off = obs_nnz_off[o];
        const int nnz = rp[D];
        O[o].col.assign(obs_col + off, obs_col + off + nnz);
        O[o].val.resize(nnz);
        for (int k = 0; k < nnz; ++k) O[o].val[k] = cd(obs_val[2 * (off + k)], obs_val[2 * (off + k) + 1]);
    }
    std::vector<cd> B(static_cast<size_t>(D) * M);
    for (size_t i = 0; i < B.size(); ++i) B[i] = cd(factors[2 * i], factors[2 * i + 1]);

    std::mt19937 g;
    if (noisy && noise_mode == 0)
        g = seed_mode == 0 ? relaxation_generator(seeded(seed), orientation)
                           : std::mt19937(static_cast<std::mt19937::result_type>(seed));

    // Dense propagator for method 1, rebuilt each step as the reference does
    // (identical values for a static H; computed once per distinct interval).
    std::vector<cd> Uprop;
    double UpropDt = -1.0;

    const int steps = ntimes - 1;
    std::vector<double> prev(static_cast<size_t>(M) * nobs, 0.0), cur(static_cast<size_t>(M) * nobs);
    std::vector<double> integ(static_cast<size_t>(M) * nobs, 0.0);
    std::vector<double> ens_integ(nobs, 0.0);
    nthreads = std::max(1, nthreads);

    auto parallel_cols = [&](auto fn) {
        if (nthreads == 1 || M < 2) { for (int c = 0; c < M; ++c) fn(c); return; }
        std::vector<std::thread> th;
        const int T = std::min(nthreads, M);
        for (int t = 0; t < T; ++t)
            th.emplace_back([&, t]() { for (int c = t; c < M; c += T) fn(c); });
        for (auto &x : th) x.join();
    };

    auto evaluate = [&](std::vector<double> &out) {
        parallel_cols([&](int c) {
            std::vector<cd> y(D);
            const cd *x = &B[static_cast<size_t>(c) * D];
            for (int o = 0; o < nobs; ++o) {
                csr_matvec(O[o], x, y.data());
                cd s = 0.0;
                for (int i = 0; i < D; ++i) s += std::conj(x[i]) * y[i];
                out[static_cast<size_t>(c) * nobs + o] = s.real() * rates[o];
            }
        });
    };

    auto apply_flips = [&](int s, int half, double h) {
        if (!noisy || h == 0.0) return;
        std::vector<unsigned char> f(M, 0);
        if (noise_mode == 0) {
            draw_flips(g, flip_probability(eventRate, h), M, f);
        } else {
            for (int c = 0; c < M; ++c) {
                const size_t bit = (static_cast<size_t>(s) * 2 + half) * M + c;
                f[c] = (flip_bits[bit >> 3] >> (bit & 7)) & 1;
            }
        }
        parallel_cols([&](int c) {
            if (!f[c]) return;
            std::vector<cd> y(D);
            cd *x = &B[static_cast<size_t>(c) * D];
            csr_matvec(U, x, y.data());
            std::copy(y.begin(), y.end(), x);
        });
    };

    for (int s = 0; s <= steps; ++s) {
        evaluate(cur);
        if (values)
            for (int o = 0; o < nobs; ++o) {
                double v = 0.0;
                for (int c = 0; c < M; ++c) v += cur[static_cast<size_t>(c) * nobs + o];
                values[static_cast<size_t>(s) * nobs + o] = v;
            }
        if (s > 0) {
            const double dt = times[s] - times[s - 1];
            for (size_t i = 0; i < integ.size(); ++i) integ[i] += 0.5 * dt * (prev[i] + cur[i]);
            for (int o = 0; o < nobs; ++o) {
                double a = 0.0, b = 0.0;
                for (int c = 0; c < M; ++c) { a += prev[static_cast<size_t>(c) * nobs + o]; b += cur[static_cast<size_t>(c) * nobs + o]; }
                ens_integ[o] += 0.5 * dt * (a + b);
            }
        }
        prev.swap(cur);
        if (s == steps) break;
        const double dt = times[s + 1] - times[s];
        apply_flips(s, 0, 0.5 * dt);
        if (method == 0) {
            parallel_cols([&](int c) {
                std::vector<cd> y(D);
                cd *x = &B[static_cast<size_t>(c) * D];
                krylov_expm_general(G, x, dt, kry, y.data());
                std::copy(y.begin(), y.end(), x);
            });
        } else if (method == 2) {
            // classical RK4 for dB/dt = G B (HSPropagator.cpp:80-90)
            parallel_cols([&](int c) {
                cd *x = &B[static_cast<size_t>(c) * D];
                std::vector<cd> k1(D), k2(D), k3(D), k4(D), y(D);
                csr_matvec(G, x, k1.data());
                for (int i = 0; i < D; ++i) y[i] = x[i] + 0.5 * dt * k1[i];
                csr_matvec(G, y.data(), k2.data());
                for (int i = 0; i < D; ++i) y[i] = x[i] + 0.5 * dt * k2[i];
                csr_matvec(G, y.data(), k3.data());
                for (int i = 0; i < D; ++i) y[i] = x[i] + dt * k3[i];
                csr_matvec(G, y.data(), k4.data());
                for (int i = 0; i < D; ++i) x[i] += (dt / 6.0) * (k1[i] + 2.0 * k2[i] + 2.0 * k3[i] + k4[i]);
            });
        } else {
            if (UpropDt != dt) {
                std::vector<cd> Gd(static_cast<size_t>(D) * D, 0.0);
                for (int r = 0; r < D; ++r)
                    for (int k = G.rowptr[r]; k < G.rowptr[r + 1]; ++k) Gd[r + static_cast<size_t>(G.col[k]) * D] += dt * G.val[k];
                Uprop.assign(static_cast<size_t>(D) * D, 0.0);
                if (!expm_pade6(D, Gd.data(), Uprop.data())) return 2;
                UpropDt = dt;
            }
            parallel_cols([&](int c) {
                std::vector<cd> y(D, 0.0);
                cd *x = &B[static_cast<size_t>(c) * D];
                for (int k = 0; k < D; ++k) {
                    const cd xk = x[k];
                    const cd *uc = &Uprop[static_cast<size_t>(k) * D];
                    for (int r = 0; r < D; ++r) y[r] += uc[r] * xk;
                }
                std::copy(y.begin(), y.end(), x);
            });
        }
        apply_flips(s, 1, 0.5 * dt);
    }
    for (size_t i = 0; i < B.size(); ++i) { factors[2 * i] = B[i].real(); factors[2 * i + 1] = B[i].imag(); }
    if (traj_yield) std::copy(integ.begin(), integ.end(), traj_yield);
    if (yield) std::copy(ens_integ.begin(), ens_integ.end(), yield);
    return 0;
}

// Finite-time yield correction 1/(1-exp(-T kmax)) (HSObservableCollector.cpp:361-392).
double oracle_yield_correction(double totalTime, double kmax)
{
    const double d = 1.0 - std::exp(-totalTime * kmax);
    return (d > 0.0 && std::isfinite(d)) ? 1.0 / d : std::numeric_limits<double>::quiet_NaN();
}

}  // extern "C"
