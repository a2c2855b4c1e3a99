// msgpu_host.cpp -- host helpers of msgpu (see include/msgpu_host.h).
//
// Plain C++17; no CUDA calls.  Hamiltonian assembly and trace sampling stay on
// the host as in MolSpin; these are standalone equivalents used when msgpu is
// driven without MolSpin's SpinAPI (benchmarks, serving, tests).

#include "msgpu_host.h"

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <limits>
#include <random>
#include <vector>

#include "msgpu_philox.h"

namespace {

using cd = std::complex<double>;

// Single-spin operators in the basis m = +S..-S (Spin.cpp SzFromCollection).
struct SpinOps {
    int n;
    std::vector<cd> s[3];  // x, y, z; column-major n x n
};

SpinOps spin_ops(int mult)
{
    SpinOps o;
    o.n = mult;
    const double S = 0.5 * (mult - 1);
    for (auto &m : o.s) m.assign(mult * mult, cd(0.0));
    for (int i = 0; i < mult; ++i) {
        const double m = S - i;
        o.s[2][i + i * mult] = m;
        if (i + 1 < mult) {
            const double c = std::sqrt(S * (S + 1) - m * (m - 1));
            o.s[0][i + (i + 1) * mult] += 0.5 * c;
            o.s[0][(i + 1) + i * mult] += 0.5 * c;
            o.s[1][i + (i + 1) * mult] += cd(0.0, -0.5 * c);
            o.s[1][(i + 1) + i * mult] += cd(0.0, 0.5 * c);
        }
    }
    return o;
}

// A local operator acting on spins (a, b) (b = -1 for a single spin), given
// as a dense (na*nb) x (na*nb) matrix over the digits of those spins.
struct LocalTerm {
    int a, b;
    std::vector<cd> m;  // row-major over local index la*nb + lb
};

}  // namespace

extern "C" {

long long msgpu_host_build_hamiltonian(int nspins, const int *mult, int nlin, const int *lin_spin,
                                       const double *lin_w, int nbil, const int *bil_i, const int *bil_j,
                                       const double *bil_c, int *rowptr, int *col, double *val)
{
    if (nspins <= 0 || !mult) return -1;
    std::vector<int> stride(nspins);
    long long D = 1;
    for (int k = nspins - 1; k >= 0; --k) {
        if (mult[k] < 1) return -1;
        stride[k] = static_cast<int>(D);
        D *= mult[k];
        if (D > (1LL << 30)) return -1;
    }
    std::vector<SpinOps> ops;
    for (int k = 0; k < nspins; ++k) ops.push_back(spin_ops(mult[k]));

    // Collapse all terms into local operators per spin and per spin pair.
    std::vector<LocalTerm> terms;
    auto local_index = [&](int a, int b) -> LocalTerm & {
        for (auto &t : terms)
            if (t.a == a && t.b == b) return t;
        const int n = mult[a] * (b >= 0 ? mult[b] : 1);
        terms.push_back(LocalTerm{a, b, std::vector<cd>(static_cast<size_t>(n) * n, cd(0.0))});
        return terms.back();
    };
    for (int l = 0; l < nlin; ++l) {
        const int k = lin_spin[l];
        if (k < 0 || k >= nspins) return -1;
        auto &t = local_index(k, -1);
        const int n = mult[k];
        for (int ax = 0; ax < 3; ++ax) {
            const double w = lin_w[3 * l + ax];
            if (w == 0.0) continue;
            for (int r = 0; r < n; ++r)
                for (int c = 0; c < n; ++c) t.m[r * n + c] += w * ops[k].s[ax][r + c * n];
        }
    }
    for (int q = 0; q < nbil; ++q) {
        int i = bil_i[q], j = bil_j[q];
        if (i < 0 || j < 0 || i >= nspins || j >= nspins || i == j) return -1;
        const double *C = bil_c + 9 * q;
        bool swapped = false;
        if (i > j) { std::swap(i, j); swapped = true; }
        auto &t = local_index(i, j);
        const int ni = mult[i], nj = mult[j];
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) {
                // S_i^T C S_j with the original (i, j) roles; when swapped the
                // coupling is S_j^T C S_i = sum C[a][b] S_j,a S_i,b.
                const double c = swapped ? C[3 * b + a] : C[3 * a + b];
                if (c == 0.0) continue;
                const auto &A = ops[i].s[a];
                const auto &B = ops[j].s[b];
                for (int ri = 0; ri < ni; ++ri)
                    for (int ci = 0; ci < ni; ++ci) {
                        const cd av = A[ri + ci * ni];
                        if (av == cd(0.0)) continue;
                        for (int rj = 0; rj < nj; ++rj)
                            for (int cj = 0; cj < nj; ++cj) {
                                const cd bv = B[rj + cj * nj];
                                if (bv == cd(0.0)) continue;
                                t.m[(ri * nj + rj) * (ni * nj) + (ci * nj + cj)] += c * av * bv;
                            }
                    }
            }
    }

    // Assemble rows.
    long long nnz = 0;
    std::vector<int> cols;
    std::vector<cd> vals;
    std::vector<int> mark(static_cast<size_t>(D), -1), slot(static_cast<size_t>(D), 0);
    std::vector<int> digit(nspins);
    if (rowptr) rowptr[0] = 0;
    for (long long r = 0; r < D; ++r) {
        long long rem = r;
        for (int k = 0; k < nspins; ++k) { digit[k] = static_cast<int>(rem / stride[k]); rem %= stride[k]; }
        cols.clear();
        vals.clear();
        auto add = [&](long long c, cd v) {
            if (mark[c] != static_cast<int>(r)) {
                mark[c] = static_cast<int>(r);
                slot[c] = static_cast<int>(cols.size());
                cols.push_back(static_cast<int>(c));
                vals.push_back(v);
            } else {
                vals[slot[c]] += v;
            }
        };
        for (const auto &t : terms) {
            if (t.b < 0) {
                const int n = mult[t.a], la = digit[t.a];
                for (int c = 0; c < n; ++c) {
                    const cd v = t.m[la * n + c];
                    if (v == cd(0.0)) continue;
                    add(r + static_cast<long long>(c - la) * stride[t.a], v);
                }
            } else {
                const int na = mult[t.a], nb = mult[t.b], n = na * nb;
                const int li = digit[t.a] * nb + digit[t.b];
                for (int lc = 0; lc < n; ++lc) {
                    const cd v = t.m[static_cast<size_t>(li) * n + lc];
                    if (v == cd(0.0)) continue;
                    const int ca = lc / nb, cb = lc % nb;
                    add(r + static_cast<long long>(ca - digit[t.a]) * stride[t.a] +
                            static_cast<long long>(cb - digit[t.b]) * stride[t.b],
                        v);
                }
            }
        }
        // sorted columns, exact zeros dropped
        std::vector<int> order(cols.size());
        for (size_t k = 0; k < order.size(); ++k) order[k] = static_cast<int>(k);
        std::sort(order.begin(), order.end(), [&](int x, int y) { return cols[x] < cols[y]; });
        for (int k : order) {
            if (vals[k] == cd(0.0)) continue;
            if (col) {
                col[nnz] = cols[k];
                val[2 * nnz] = vals[k].real();
                val[2 * nnz + 1] = vals[k].imag();
            }
            ++nnz;
        }
        if (nnz > std::numeric_limits<int>::max()) return -1;
        if (rowptr) rowptr[r + 1] = static_cast<int>(nnz);
    }
    return nnz;
}

int msgpu_host_trace_samples(double seed, const double *fixed, int F, int Z, int M, double *out)
{
    if (F <= 0 || Z <= 0 || M <= 0 || !fixed || !out) return 1;
    const double s = seed == 0.0 ? 1.0 : seed;
    std::mt19937 generator;
    generator.seed(static_cast<std::mt19937::result_type>(s));
    const double sqrtM = std::sqrt(static_cast<double>(M));
    std::vector<cd> chi(Z);
    for (int sample = 0; sample < M; ++sample) {
        // One distribution object per sample, two draws per complex entry in
        // the argument order of the reference expression.
        std::normal_distribution<double> distribution(0.0, 1.0);
        for (int i = 0; i < Z; ++i) chi[i] = std::complex<double>(distribution(generator), distribution(generator));
        // normalise (divide by the 2-norm), Kronecker product with the fixed
        // state, then the 1/sqrt(M) factor scaling of HSStatePreparation::Prepare
        double nn = 0.0;
        for (int i = 0; i < Z; ++i) nn += std::norm(chi[i]);
        const double nrm = std::sqrt(nn);
        for (int i = 0; i < Z; ++i) chi[i] /= nrm;
        double *colp = out + 2 * static_cast<size_t>(sample) * F * Z;
        for (int a = 0; a < F; ++a) {
            const cd f(fixed[2 * a], fixed[2 * a + 1]);
            for (int i = 0; i < Z; ++i) {
                const cd v = (f * chi[i]) / sqrtM;
                colp[2 * (static_cast<size_t>(a) * Z + i)] = v.real();
                colp[2 * (static_cast<size_t>(a) * Z + i) + 1] = v.imag();
            }
        }
    }
    return 0;
}

int msgpu_host_reference_flip_bits(double seed, int seed_mode, unsigned long long orientation, double st_rate,
                                   const double *times, int ntimes, int M, unsigned char *bits)
{
    if (ntimes < 1 || M <= 0 || !bits) return 1;
    std::mt19937 g;
    if (seed_mode == 0) {
        const double s = seed == 0.0 ? 1.0 : seed;
        std::mt19937 source;
        source.seed(static_cast<std::mt19937::result_type>(s));
        std::vector<std::mt19937::result_type> sd{0x5354524cU, 0x554e4954U,
            static_cast<std::mt19937::result_type>(orientation & 0xffffffffULL),
            static_cast<std::mt19937::result_type>(orientation >> 32)};
        for (unsigned i = 0; i < 8; ++i) sd.push_back(source());
        std::seed_seq seq(sd.begin(), sd.end());
        g = std::mt19937(seq);
    } else {
        g = std::mt19937(static_cast<std::mt19937::result_type>(seed));
    }
    const double eventRate = 0.5 * st_rate;
    const long long steps = ntimes - 1;
    std::memset(bits, 0, static_cast<size_t>((steps * 2 * M + 7) / 8));
    for (long long s = 0; s < steps; ++s) {
        const double h = 0.5 * (times[s + 1] - times[s]);
        if (!(eventRate > 0.0) || h == 0.0) continue;
        const double p = -0.5 * std::expm1(-2.0 * eventRate * h);
        for (int half = 0; half < 2; ++half) {
            std::bernoulli_distribution flip(p);
            for (int c = 0; c < M; ++c)
                if (flip(g)) {
                    const long long bit = (s * 2 + half) * M + c;
                    bits[bit >> 3] |= static_cast<unsigned char>(1u << (bit & 7));
                }
        }
    }
    return 0;
}

int msgpu_host_reference_flip_bits_multi(double seed, int seed_mode, unsigned long long orientation,
                                         const double *st_rates, int nterms, const double *times, int ntimes, int M,
                                         unsigned char *bits)
{
    if (nterms < 1 || !st_rates || ntimes < 1 || M <= 0 || !bits) return 1;
    if (nterms == 1) return msgpu_host_reference_flip_bits(seed, seed_mode, orientation, st_rates[0], times, ntimes, M, bits);
    std::vector<double> rates(nterms);
    double total = 0.0;
    for (int k = 0; k < nterms; ++k) {
        if (!(st_rates[k] > 0.0) || !std::isfinite(st_rates[k])) return 1;
        rates[k] = 0.5 * st_rates[k];  // event rate of a dephasing Operator: rate / 2
        total += rates[k];
    }
    std::mt19937 g;
    if (seed_mode == 0) {
        const double s = seed == 0.0 ? 1.0 : seed;
        std::mt19937 source;
        source.seed(static_cast<std::mt19937::result_type>(s));
        std::vector<std::mt19937::result_type> sd{0x5354524cU, 0x554e4954U,
            static_cast<std::mt19937::result_type>(orientation & 0xffffffffULL),
            static_cast<std::mt19937::result_type>(orientation >> 32)};
        for (unsigned i = 0; i < 8; ++i) sd.push_back(source());
        std::seed_seq seq(sd.begin(), sd.end());
        g = std::mt19937(seq);
    } else {
        g = std::mt19937(static_cast<std::mt19937::result_type>(seed));
    }
    const long long steps = ntimes - 1;
    std::memset(bits, 0, static_cast<size_t>((steps * 2 * M + 7) / 8));
    for (long long s = 0; s < steps; ++s) {
        const double h = 0.5 * (times[s + 1] - times[s]);
        if (h == 0.0) continue;
        for (int half = 0; half < 2; ++half) {
            std::poisson_distribution<unsigned long long> count(total * h);
            std::discrete_distribution<size_t> channel(rates.begin(), rates.end());
            for (int c = 0; c < M; ++c) {
                const unsigned long long events = count(g);
                for (unsigned long long e = 0; e < events; ++e) (void)channel(g);
                if (events & 1ULL) {
                    const long long bit = (s * 2 + half) * M + c;
                    bits[bit >> 3] |= static_cast<unsigned char>(1u << (bit & 7));
                }
            }
        }
    }
    return 0;
}

int msgpu_host_philox_flip_bits(unsigned long long seed, unsigned int traj_offset, long long step_offset,
                                double st_rate, const double *times, int ntimes, int M, unsigned char *bits)
{
    if (ntimes < 1 || M <= 0 || !bits) return 1;
    const long long steps = ntimes - 1;
    std::memset(bits, 0, static_cast<size_t>((steps * 2 * M + 7) / 8));
    const double eventRate = 0.5 * st_rate;
    for (long long s = 0; s < steps; ++s) {
        const double h = 0.5 * (times[s + 1] - times[s]);
        if (!(eventRate > 0.0) || h == 0.0) continue;
        const double p = -0.5 * std::expm1(-2.0 * eventRate * h);
        for (int half = 0; half < 2; ++half)
            for (int c = 0; c < M; ++c)
                if (msgpu::philox_flip(seed, traj_offset + static_cast<unsigned>(c),
                                       static_cast<uint32_t>(step_offset + s), static_cast<uint32_t>(half), p)) {
                    const long long bit = (s * 2 + half) * M + c;
                    bits[bit >> 3] |= static_cast<unsigned char>(1u << (bit & 7));
                }
    }
    return 0;
}

long msgpu_host_time_grid(double total, double dt, double *times, long cap)
{
    if (!std::isfinite(total) || total < 0.0 || !std::isfinite(dt) || dt <= 0.0) return -1;
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

}  // extern "C"
