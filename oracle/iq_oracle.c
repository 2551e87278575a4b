/*
 * iq_oracle.c -- TEST INFRASTRUCTURE ONLY (the oracle).
 *
 * A plain-C, single-threaded restatement of InvariantQ's CPU state-vector and
 * density-matrix kernels (core/src/statevector.cpp, core/src/density_matrix.cpp,
 * core/src/api.cpp).  It exists so that the CUDA library can be checked against
 * the reference algorithm on the same inputs.  Only tests/, the smoke check in
 * __graft_entry__.py and bench.py's CPU-baseline leg may load it; the product
 * library never links or calls it.
 *
 * Parity is pinned: tests/test_oracle_golden.py checks every function here
 * against fixtures in tests/golden/ that tests/golden/make_golden.py produced by
 * running the reference's own C++ core (built from its sources by
 * oracle/Makefile) through the reference's own Python ctypes binding.
 *
 * Layout: complex amplitudes are interleaved (re, im) doubles, exactly like the
 * reference's std::vector<std::complex<double>>.  Qubit q is bit q of the index
 * (little-endian).  A density matrix is row-major rho[r * 2^n + c].
 *
 * Error behaviour differs from the reference on purpose: where the reference
 * throws through extern "C" (and so aborts the process), these functions return
 * a negative status instead.  Happy-path arithmetic follows the reference.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef struct { double re, im; } cplx;

static inline cplx cmul(cplx a, cplx b) {
    cplx r = { a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re };
    return r;
}
static inline cplx cadd(cplx a, cplx b) { cplx r = { a.re + b.re, a.im + b.im }; return r; }
static inline cplx cconj(cplx a) { cplx r = { a.re, -a.im }; return r; }
static inline double cnorm(cplx a) { return a.re * a.re + a.im * a.im; }
static inline cplx cscale(cplx a, double s) { cplx r = { a.re * s, a.im * s }; return r; }

static void load_matrix(cplx* U, const double* ur, const double* ui, size_t count) {
    for (size_t i = 0; i < count; ++i) { U[i].re = ur[i]; U[i].im = ui[i]; }
}

/* ---------------------------------------------------------------- state vector */

/* StateVector::StateVector / reset -- statevector.cpp:9-17 */
void or_sv_init(cplx* s, int n) {
    size_t dim = (size_t)1 << n;
    memset(s, 0, dim * sizeof(cplx));
    s[0].re = 1.0;
}

/* StateVector::apply_1q_gate -- statevector.cpp:26-47 (ABI wrapper api.cpp:30-37).
 * Pair (i0, i1) = (index with bit t clear, same with bit t set); [a,b] <- U [a,b]. */
int or_sv_apply_1q(cplx* s, int n, size_t target, const double* ur, const double* ui) {
    if (target >= (size_t)n) return -1;
    cplx U[4]; load_matrix(U, ur, ui, 4);
    const uint64_t m = 1ULL << target, lo = m - 1, hi = ~lo;
    const uint64_t half = ((uint64_t)1 << n) >> 1;
    for (uint64_t i = 0; i < half; ++i) {
        uint64_t i0 = ((i & hi) << 1) | (i & lo), i1 = i0 | m;
        cplx a = s[i0], b = s[i1];
        s[i0] = cadd(cmul(U[0], a), cmul(U[1], b));
        s[i1] = cadd(cmul(U[2], a), cmul(U[3], b));
    }
    return 0;
}

/* StateVector::apply_2q_gate -- statevector.cpp:49-87 (api.cpp:39-46).
 * Local index (r) of the 4x4 matrix: bit 1 = qubit q0, bit 0 = qubit q1
 * (q0 is the most significant bit of the local index). */
int or_sv_apply_2q(cplx* s, int n, size_t q0, size_t q1, const double* ur, const double* ui) {
    if (q0 >= (size_t)n || q1 >= (size_t)n || q0 == q1) return -1;
    cplx U[16]; load_matrix(U, ur, ui, 16);
    size_t ql = q0 < q1 ? q0 : q1, qh = q0 < q1 ? q1 : q0;
    uint64_t quarter = ((uint64_t)1 << n) >> 2;
    for (uint64_t i = 0; i < quarter; ++i) {
        uint64_t low = i & ((1ULL << ql) - 1);
        uint64_t mid = (i >> ql) & ((1ULL << (qh - ql - 1)) - 1);
        uint64_t high = i >> (qh - 1);
        uint64_t i00 = (high << (qh + 1)) | (mid << (ql + 1)) | low;
        uint64_t idx[4] = { i00, i00 | (1ULL << q1), i00 | (1ULL << q0),
                            i00 | (1ULL << q0) | (1ULL << q1) };
        cplx v[4];
        for (int k = 0; k < 4; ++k) v[k] = s[idx[k]];
        for (int r = 0; r < 4; ++r) {
            cplx acc = cmul(U[r * 4 + 0], v[0]);
            acc = cadd(acc, cmul(U[r * 4 + 1], v[1]));
            acc = cadd(acc, cmul(U[r * 4 + 2], v[2]));
            acc = cadd(acc, cmul(U[r * 4 + 3], v[3]));
            s[idx[r]] = acc;
        }
    }
    return 0;
}

/* StateVector::apply_fused_gate -- statevector.cpp:89-152 (api.cpp:48-57).
 * k == 1 and k == 2 delegate to the 1q / 2q kernels (so k == 2 is MSB-first);
 * k in {3,4}: local index bit b <-> qubits[b] (LSB-first); k > 4 is rejected
 * (the reference throws std::invalid_argument). */
int or_sv_apply_fused(cplx* s, int n, const size_t* qubits, size_t k,
                      const double* ur, const double* ui) {
    if (k == 0) return -1;
    if (k == 1) return or_sv_apply_1q(s, n, qubits[0], ur, ui);
    if (k == 2) return or_sv_apply_2q(s, n, qubits[0], qubits[1], ur, ui);
    if (k > 4) return -2;
    for (size_t i = 0; i < k; ++i) {
        if (qubits[i] >= (size_t)n) return -1;
        for (size_t j = 0; j < i; ++j) if (qubits[i] == qubits[j]) return -1;
    }
    size_t kd = (size_t)1 << k;
    cplx* U = (cplx*)malloc(kd * kd * sizeof(cplx));
    load_matrix(U, ur, ui, kd * kd);
    size_t nother = 0;
    size_t other[64];
    for (size_t q = 0; q < (size_t)n; ++q) {
        int used = 0;
        for (size_t j = 0; j < k; ++j) if (qubits[j] == q) used = 1;
        if (!used) other[nother++] = q;
    }
    uint64_t outer = ((uint64_t)1 << n) >> k;
    uint64_t idx[16]; cplx vec[16];
    for (uint64_t i = 0; i < outer; ++i) {
        uint64_t base = 0;
        for (size_t b = 0; b < nother; ++b) if ((i >> b) & 1ULL) base |= 1ULL << other[b];
        for (size_t st = 0; st < kd; ++st) {
            uint64_t id = base;
            for (size_t bit = 0; bit < k; ++bit) if ((st >> bit) & 1ULL) id |= 1ULL << qubits[bit];
            idx[st] = id; vec[st] = s[id];
        }
        for (size_t r = 0; r < kd; ++r) {
            cplx acc = { 0.0, 0.0 };
            for (size_t c = 0; c < kd; ++c) acc = cadd(acc, cmul(U[r * kd + c], vec[c]));
            s[idx[r]] = acc;
        }
    }
    free(U);
    return 0;
}

/* StateVector::measure_probability -- statevector.cpp:154-169 */
double or_sv_measure_prob(const cplx* s, int n, size_t target, int outcome) {
    if (target >= (size_t)n) return -1.0;
    uint64_t m = 1ULL << target, dim = (uint64_t)1 << n;
    double p = 0.0;
    for (uint64_t i = 0; i < dim; ++i) {
        int bit = (i & m) ? 1 : 0;
        if (bit == outcome) p += cnorm(s[i]);
    }
    return p;
}

/* StateVector::collapse -- statevector.cpp:171-188 (p < 1e-15 is an error) */
int or_sv_collapse(cplx* s, int n, size_t target, int outcome) {
    double p = or_sv_measure_prob(s, n, target, outcome);
    if (p < 1e-15) return -1;
    double f = 1.0 / sqrt(p);
    uint64_t m = 1ULL << target, dim = (uint64_t)1 << n;
    for (uint64_t i = 0; i < dim; ++i) {
        int bit = (i & m) ? 1 : 0;
        if (bit == outcome) s[i] = cscale(s[i], f);
        else { s[i].re = 0.0; s[i].im = 0.0; }
    }
    return 0;
}

/* StateVector::measure -- statevector.cpp:190-195: outcome = (rand < p0) ? 0 : 1 */
int or_sv_measure(cplx* s, int n, size_t target, double rand_val) {
    if (target >= (size_t)n) return -1;
    double p0 = or_sv_measure_prob(s, n, target, 0);
    int outcome = (rand_val < p0) ? 0 : 1;
    if (or_sv_collapse(s, n, target, outcome) != 0) return -1;
    return outcome;
}

/* StateVector::reset_qubit -- statevector.cpp:197-204: measure, then X if 1 */
int or_sv_reset_qubit(cplx* s, int n, size_t target, double rand_val) {
    int o = or_sv_measure(s, n, target, rand_val);
    if (o < 0) return o;
    if (o == 1) {
        const double xr[4] = { 0, 1, 1, 0 }, xi[4] = { 0, 0, 0, 0 };
        or_sv_apply_1q(s, n, target, xr, xi);
    }
    return 0;
}

/* StateVector::norm_squared -- statevector.cpp:206-213 */
double or_sv_norm2(const cplx* s, int n) {
    uint64_t dim = (uint64_t)1 << n;
    double sum = 0.0;
    for (uint64_t i = 0; i < dim; ++i) sum += cnorm(s[i]);
    return sum;
}

/* StateVector::probabilities -- statevector.cpp:226-233 */
void or_sv_probabilities(const cplx* s, int n, double* out) {
    uint64_t dim = (uint64_t)1 << n;
    for (uint64_t i = 0; i < dim; ++i) out[i] = cnorm(s[i]);
}

/* ---- std::mt19937_64 and std::uniform_real_distribution<double>(0,1) ----
 * The reference's sampler (statevector.cpp:244-245) draws from std::mt19937_64
 * seeded with `seed` and maps each 64-bit output x to [0,1) the way libstdc++
 * (GCC 13.3, the toolchain that builds the reference here) implements
 * std::generate_canonical<double,53> for a 64-bit engine: one engine call,
 * (double)x / 2^64, clamped below 1.  The generator below is the published
 * 64-bit Mersenne Twister (Matsumoto & Nishimura; parameters as fixed by the
 * C++ standard for mt19937_64). */
typedef struct { uint64_t mt[312]; int idx; } mt64;

static void mt64_seed(mt64* g, uint64_t seed) {
    g->mt[0] = seed;
    for (int i = 1; i < 312; ++i)
        g->mt[i] = 6364136223846793005ULL * (g->mt[i - 1] ^ (g->mt[i - 1] >> 62)) + (uint64_t)i;
    g->idx = 312;
}

static uint64_t mt64_next(mt64* g) {
    const uint64_t upper = 0xFFFFFFFF80000000ULL, lower = 0x7FFFFFFFULL;
    if (g->idx >= 312) {
        for (int i = 0; i < 312; ++i) {
            uint64_t y = (g->mt[i] & upper) | (g->mt[(i + 1) % 312] & lower);
            uint64_t v = g->mt[(i + 156) % 312] ^ (y >> 1);
            if (y & 1ULL) v ^= 0xB5026F5AA96619E9ULL;
            g->mt[i] = v;
        }
        g->idx = 0;
    }
    uint64_t z = g->mt[g->idx++];
    z ^= (z >> 29) & 0x5555555555555555ULL;
    z ^= (z << 17) & 0x71D67FFFEDA60000ULL;
    z ^= (z << 37) & 0xFFF7EEE000000000ULL;
    z ^= (z >> 43);
    return z;
}

static double mt64_uniform01(mt64* g) {
    double r = (double)mt64_next(g) / 18446744073709551616.0;
    if (r >= 1.0) r = nextafter(1.0, 0.0);
    return r;
}

void or_mt64_uniform(uint64_t seed, size_t count, double* out) {
    mt64 g; mt64_seed(&g, seed);
    for (size_t i = 0; i < count; ++i) out[i] = mt64_uniform01(&g);
}

/* StateVector::sample -- statevector.cpp:235-256: serial CDF, lower_bound,
 * clamp to dim-1. */
void or_sv_sample(const cplx* s, int n, size_t shots, uint64_t seed, uint64_t* out) {
    uint64_t dim = (uint64_t)1 << n;
    double* cdf = (double*)malloc(dim * sizeof(double));
    double cum = 0.0;
    for (uint64_t i = 0; i < dim; ++i) { cum += cnorm(s[i]); cdf[i] = cum; }
    mt64 g; mt64_seed(&g, seed);
    for (size_t k = 0; k < shots; ++k) {
        double r = mt64_uniform01(&g);
        uint64_t lo = 0, hi = dim;           /* first i with cdf[i] >= r */
        while (lo < hi) {
            uint64_t mid = lo + ((hi - lo) >> 1);
            if (cdf[mid] < r) lo = mid + 1; else hi = mid;
        }
        if (lo >= dim) lo = dim - 1;
        out[k] = lo;
    }
    free(cdf);
}

/* StateVector::expectation_value_pauli -- statevector.cpp:258-291.
 * Terms with |a_i|^2 < 1e-18 are skipped, as the reference does (:267). */
int or_sv_expval_pauli(const cplx* s, int n, const char* pauli, const size_t* qubits,
                       size_t len, double* out_re, double* out_im) {
    for (size_t p = 0; p < len; ++p) if (qubits[p] >= (size_t)n) return -1;
    uint64_t dim = (uint64_t)1 << n;
    cplx acc = { 0.0, 0.0 };
    for (uint64_t i = 0; i < dim; ++i) {
        cplx a = s[i];
        if (cnorm(a) < 1e-18) continue;
        uint64_t j = i;
        cplx ph = { 1.0, 0.0 };
        for (size_t p = 0; p < len; ++p) {
            char op = pauli[p];
            size_t q = qubits[p];
            uint64_t bit = (i >> q) & 1ULL;
            if (op == 'X') {
                j ^= 1ULL << q;
            } else if (op == 'Y') {
                j ^= 1ULL << q;
                cplx f = { 0.0, bit == 0 ? 1.0 : -1.0 };
                ph = cmul(ph, f);
            } else if (op == 'Z') {
                if (bit == 1) ph = cscale(ph, -1.0);
            }
        }
        acc = cadd(acc, cmul(cmul(cconj(s[j]), ph), a));
    }
    *out_re = acc.re; *out_im = acc.im;
    return 0;
}

/* Jacobi eigenvalues of a Hermitian matrix, following the reference's
 * hermitian_eigenvalues (statevector.cpp:333-393): largest off-diagonal pivot,
 * at most `max_iter` rotations, stop below `tol`. */
static void jacobi_eigs(cplx* A, size_t n, int max_iter, double tol, double* d) {
    for (int it = 0; it < max_iter; ++it) {
        double mx = 0.0; size_t p = 0, q = 1;
        for (size_t i = 0; i < n; ++i)
            for (size_t j = i + 1; j < n; ++j) {
                double v = sqrt(cnorm(A[i * n + j]));
                if (v > mx) { mx = v; p = i; q = j; }
            }
        if (mx < tol) break;
        double app = A[p * n + p].re, aqq = A[q * n + q].re;
        cplx apq = A[p * n + q];
        double aabs = sqrt(cnorm(apq));
        double theta = 0.5 * atan2(2.0 * aabs, app - aqq);
        cplx phase = { apq.re / aabs, apq.im / aabs };
        double c = cos(theta);
        cplx sn = cscale(phase, sin(theta));
        for (size_t i = 0; i < n; ++i) {
            if (i == p || i == q) continue;
            cplx aip = A[i * n + p], aiq = A[i * n + q];
            cplx nip = cadd(cscale(aip, c), cmul(cconj(sn), aiq));
            cplx niq = cadd(cscale(cmul(sn, aip), -1.0), cscale(aiq, c));
            A[i * n + p] = nip; A[p * n + i] = cconj(nip);
            A[i * n + q] = niq; A[q * n + i] = cconj(niq);
        }
        double ns = cnorm(sn);
        double cross = 2.0 * cmul(cscale(cconj(sn), c), apq).re;
        double napp = c * c * app + ns * aqq + cross;
        double naqq = ns * app + c * c * aqq - cross;
        A[p * n + p].re = napp; A[p * n + p].im = 0.0;
        A[q * n + q].re = naqq; A[q * n + q].im = 0.0;
        A[p * n + q].re = A[p * n + q].im = 0.0;
        A[q * n + p].re = A[q * n + p].im = 0.0;
    }
    for (size_t i = 0; i < n; ++i) d[i] = A[i * n + i].re;
}

/* StateVector::partial_trace + von_neumann_entropy -- statevector.cpp:293-330,
 * 395-410.  rho[r][c] = sum_env a[idx(r,env)] conj(a[idx(c,env)]) with local
 * index bit b <-> keep[b]; eigenvalues above 1e-14 contribute -l log2 l. */
double or_sv_entropy(const cplx* s, int n, const size_t* keep, size_t k) {
    if (k == 0 || k == (size_t)n) return 0.0;
    size_t kd = (size_t)1 << k;
    size_t traced[64], nt = 0;
    for (size_t q = 0; q < (size_t)n; ++q) {
        int in = 0;
        for (size_t j = 0; j < k; ++j) if (keep[j] == q) in = 1;
        if (!in) traced[nt++] = q;
    }
    size_t td = (size_t)1 << nt;
    cplx* rho = (cplx*)calloc(kd * kd, sizeof(cplx));
    for (uint64_t r = 0; r < kd; ++r)
        for (uint64_t c = 0; c < kd; ++c) {
            cplx sum = { 0.0, 0.0 };
            for (uint64_t env = 0; env < td; ++env) {
                uint64_t ir = 0, ic = 0;
                for (size_t b = 0; b < k; ++b) {
                    if ((r >> b) & 1ULL) ir |= 1ULL << keep[b];
                    if ((c >> b) & 1ULL) ic |= 1ULL << keep[b];
                }
                for (size_t b = 0; b < nt; ++b)
                    if ((env >> b) & 1ULL) { ir |= 1ULL << traced[b]; ic |= 1ULL << traced[b]; }
                sum = cadd(sum, cmul(s[ir], cconj(s[ic])));
            }
            rho[r * kd + c] = sum;
        }
    double* d = (double*)malloc(kd * sizeof(double));
    jacobi_eigs(rho, kd, 100, 1e-12, d);
    double e = 0.0;
    for (size_t i = 0; i < kd; ++i) if (d[i] > 1e-14) e -= d[i] * log2(d[i]);
    free(d); free(rho);
    return e > 0.0 ? e : 0.0;
}

/* ------------------------------------------------------------- density matrix */

/* DensityMatrix::DensityMatrix / reset -- density_matrix.cpp:8-16 */
void or_dm_init(cplx* rho, int n) {
    size_t dim = (size_t)1 << n;
    memset(rho, 0, dim * dim * sizeof(cplx));
    rho[0].re = 1.0;
}

/* DensityMatrix::apply_1q_unitary -- density_matrix.cpp:18-67: left pass
 * rho' = U rho over columns into a temporary, right pass rho = rho' U^dagger. */
static void dm_1q(cplx* rho, int n, size_t t, const cplx* U) {
    uint64_t dim = (uint64_t)1 << n, m = 1ULL << t, lo = m - 1, hi = ~lo, half = dim >> 1;
    cplx* nx = (cplx*)calloc(dim * dim, sizeof(cplx));
    for (uint64_t c = 0; c < dim; ++c)
        for (uint64_t i = 0; i < half; ++i) {
            uint64_t r0 = ((i & hi) << 1) | (i & lo), r1 = r0 | m;
            cplx a = rho[r0 * dim + c], b = rho[r1 * dim + c];
            nx[r0 * dim + c] = cadd(cmul(U[0], a), cmul(U[1], b));
            nx[r1 * dim + c] = cadd(cmul(U[2], a), cmul(U[3], b));
        }
    cplx Ud[4] = { cconj(U[0]), cconj(U[2]), cconj(U[1]), cconj(U[3]) };
    for (uint64_t r = 0; r < dim; ++r)
        for (uint64_t i = 0; i < half; ++i) {
            uint64_t c0 = ((i & hi) << 1) | (i & lo), c1 = c0 | m;
            cplx a = nx[r * dim + c0], b = nx[r * dim + c1];
            rho[r * dim + c0] = cadd(cmul(a, Ud[0]), cmul(b, Ud[2]));
            rho[r * dim + c1] = cadd(cmul(a, Ud[1]), cmul(b, Ud[3]));
        }
    free(nx);
}

int or_dm_apply_1q_unitary(cplx* rho, int n, size_t t, const double* ur, const double* ui) {
    if (t >= (size_t)n) return -1;
    cplx U[4]; load_matrix(U, ur, ui, 4);
    dm_1q(rho, n, t, U);
    return 0;
}

/* DensityMatrix::apply_2q_unitary -- density_matrix.cpp:69-145 (q0 = MSB). */
int or_dm_apply_2q_unitary(cplx* rho, int n, size_t q0, size_t q1, const double* ur, const double* ui) {
    if (q0 >= (size_t)n || q1 >= (size_t)n || q0 == q1) return -1;
    cplx U[16]; load_matrix(U, ur, ui, 16);
    uint64_t dim = (uint64_t)1 << n, quarter = dim >> 2;
    size_t ql = q0 < q1 ? q0 : q1, qh = q0 < q1 ? q1 : q0;
    cplx* nx = (cplx*)calloc(dim * dim, sizeof(cplx));
    for (uint64_t c = 0; c < dim; ++c)
        for (uint64_t i = 0; i < quarter; ++i) {
            uint64_t low = i & ((1ULL << ql) - 1);
            uint64_t mid = (i >> ql) & ((1ULL << (qh - ql - 1)) - 1);
            uint64_t high = i >> (qh - 1);
            uint64_t i00 = (high << (qh + 1)) | (mid << (ql + 1)) | low;
            uint64_t idx[4] = { i00, i00 | (1ULL << q1), i00 | (1ULL << q0),
                                i00 | (1ULL << q0) | (1ULL << q1) };
            cplx v[4];
            for (int k = 0; k < 4; ++k) v[k] = rho[idx[k] * dim + c];
            for (int r = 0; r < 4; ++r) {
                cplx acc = cmul(U[r * 4], v[0]);
                for (int k = 1; k < 4; ++k) acc = cadd(acc, cmul(U[r * 4 + k], v[k]));
                nx[idx[r] * dim + c] = acc;
            }
        }
    cplx Ud[16];
    for (int r = 0; r < 4; ++r) for (int c = 0; c < 4; ++c) Ud[r * 4 + c] = cconj(U[c * 4 + r]);
    for (uint64_t r = 0; r < dim; ++r)
        for (uint64_t i = 0; i < quarter; ++i) {
            uint64_t low = i & ((1ULL << ql) - 1);
            uint64_t mid = (i >> ql) & ((1ULL << (qh - ql - 1)) - 1);
            uint64_t high = i >> (qh - 1);
            uint64_t i00 = (high << (qh + 1)) | (mid << (ql + 1)) | low;
            uint64_t idx[4] = { i00, i00 | (1ULL << q1), i00 | (1ULL << q0),
                                i00 | (1ULL << q0) | (1ULL << q1) };
            cplx v[4];
            for (int k = 0; k < 4; ++k) v[k] = nx[r * dim + idx[k]];
            for (int col = 0; col < 4; ++col) {
                cplx acc = cmul(v[0], Ud[col]);
                for (int k = 1; k < 4; ++k) acc = cadd(acc, cmul(v[k], Ud[k * 4 + col]));
                rho[r * dim + idx[col]] = acc;
            }
        }
    free(nx);
    return 0;
}

/* DensityMatrix::apply_1q_kraus -- density_matrix.cpp:147-163: for every K,
 * restart from the initial rho, apply K rho K^dagger, accumulate. Kraus array
 * layout as in api.cpp:146-155: K_k element i at [k*4 + i]. */
int or_dm_apply_kraus_1q(cplx* rho, int n, size_t t, size_t nk, const double* kr, const double* ki) {
    if (t >= (size_t)n) return -1;
    uint64_t dim = (uint64_t)1 << n, tot = dim * dim;
    cplx* init = (cplx*)malloc(tot * sizeof(cplx));
    cplx* res = (cplx*)calloc(tot, sizeof(cplx));
    memcpy(init, rho, tot * sizeof(cplx));
    for (size_t k = 0; k < nk; ++k) {
        cplx K[4]; load_matrix(K, kr + 4 * k, ki + 4 * k, 4);
        memcpy(rho, init, tot * sizeof(cplx));
        dm_1q(rho, n, t, K);
        for (uint64_t i = 0; i < tot; ++i) res[i] = cadd(res[i], rho[i]);
    }
    memcpy(rho, res, tot * sizeof(cplx));
    free(init); free(res);
    return 0;
}

/* DensityMatrix::trace -- density_matrix.cpp:193-199 (serial, real part) */
double or_dm_trace(const cplx* rho, int n) {
    uint64_t dim = (uint64_t)1 << n;
    cplx tr = { 0.0, 0.0 };
    for (uint64_t i = 0; i < dim; ++i) tr = cadd(tr, rho[i * dim + i]);
    return tr.re;
}

/* DensityMatrix::purity -- density_matrix.cpp:201-208: sum |rho_ij|^2 */
double or_dm_purity(const cplx* rho, int n) {
    uint64_t dim = (uint64_t)1 << n, tot = dim * dim;
    double p = 0.0;
    for (uint64_t i = 0; i < tot; ++i) p += cnorm(rho[i]);
    return p;
}

/* DensityMatrix::measure_probability -- density_matrix.cpp:218-229 */
double or_dm_measure_prob(const cplx* rho, int n, size_t t, int outcome) {
    uint64_t dim = (uint64_t)1 << n, m = 1ULL << t;
    double p = 0.0;
    for (uint64_t i = 0; i < dim; ++i) {
        int bit = (i & m) ? 1 : 0;
        if (bit == outcome) p += rho[i * dim + i].re;
    }
    return p > 0.0 ? p : 0.0;
}

/* DensityMatrix::collapse / measure -- density_matrix.cpp:231-256 */
int or_dm_measure(cplx* rho, int n, size_t t, double rand_val) {
    if (t >= (size_t)n) return -1;
    double p0 = or_dm_measure_prob(rho, n, t, 0);
    int outcome = (rand_val < p0) ? 0 : 1;
    double p = or_dm_measure_prob(rho, n, t, outcome);
    if (p < 1e-15) return -1;
    double f = 1.0 / p;
    uint64_t dim = (uint64_t)1 << n, m = 1ULL << t;
    for (uint64_t r = 0; r < dim; ++r) {
        int br = (r & m) ? 1 : 0;
        for (uint64_t c = 0; c < dim; ++c) {
            int bc = (c & m) ? 1 : 0;
            if (br == outcome && bc == outcome) rho[r * dim + c] = cscale(rho[r * dim + c], f);
            else { rho[r * dim + c].re = 0.0; rho[r * dim + c].im = 0.0; }
        }
    }
    return outcome;
}

/* DensityMatrix::reset_qubit -- density_matrix.cpp:258-269: Kraus {|0><0|, |0><1|} */
int or_dm_reset_qubit(cplx* rho, int n, size_t t) {
    const double kr[8] = { 1, 0, 0, 0, 0, 1, 0, 0 }, ki[8] = { 0 };
    return or_dm_apply_kraus_1q(rho, n, t, 2, kr, ki);
}

/* DensityMatrix::von_neumann_entropy -- density_matrix.cpp:310-380: diagonal
 * approximation when dim > 64, else Jacobi (120 rotations, tol 1e-13). */
double or_dm_entropy(const cplx* rho, int n) {
    uint64_t dim = (uint64_t)1 << n;
    double e = 0.0;
    if (dim > 64) {
        for (uint64_t i = 0; i < dim; ++i) {
            double p = rho[i * dim + i].re;
            if (p < 0.0) p = 0.0;
            if (p > 1e-14) e -= p * log2(p);
        }
        return e;
    }
    cplx* A = (cplx*)malloc(dim * dim * sizeof(cplx));
    memcpy(A, rho, dim * dim * sizeof(cplx));
    double* d = (double*)malloc(dim * sizeof(double));
    jacobi_eigs(A, dim, 120, 1e-13, d);
    for (uint64_t i = 0; i < dim; ++i) if (d[i] > 1e-14) e -= d[i] * log2(d[i]);
    free(A); free(d);
    return e > 0.0 ? e : 0.0;
}
