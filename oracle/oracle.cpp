// ORACLE — test infrastructure only. Nothing in the product (the pureadsorb.jl_b200 package,
// its CUDA library or its C ABI) links, loads or calls this file. It is the CPU restatement of
// PureAdsorb.jl's batched Widom insertion path that the CUDA kernels are checked against, and
// the timed CPU baseline ("port") of bench.py. Parity pins: the reference's own known-answer
// tests, restated in tests/test_oracle_pins.py (Madelung constant, alpha/erfc, k-vector counts,
// theta_F bounds, mulhi64 vs 128-bit, rejection safety, two-phase == single-phase, ...).
//
// Everything is FP64 except the pose generation and phase-0 hard-core scan, which also run in
// strict FP32 (every operation individually rounded, explicit fused multiply-adds, no
// contraction: built with -ffp-contract=off) so that their results are bit-identical to the
// device kernels that follow the same operation sequence.
//
// Reference files restated here (paths inside PureAdsorb.jl):
//   src/state.jl:225-230 (splitmix64), src/rng.jl:14-141 (mulhi64, ChainRNG, draws, Shoemake),
//   src/cell.jl (geometry and the cell list), src/energy.jl:13-82 (rotate, LJ, insertion_energy),
//   src/ewald.jl:21-203 (alpha, kmax, pk, kvectors, structure factor, Ewald energy),
//   src/reference.jl:10-67 (full k tables, insertion_energy_reference),
//   src/reject.jl (theta_F, find_r0, hardcore_bound, kmin_table, find_rho2),
//   src/forcefield.jl:22-39,103-124 (Lorentz-Berthelot, tail correction),
//   src/batch.jl:173-432 (verify_replication, FrameworkBatch construction),
//   src/widom.jl (sys_of_index, system_counts, widom loop, boltzmann_weight,
//                 hardcore_kernel!, build_rejection_tables).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <map>
#include <string>
#include <tuple>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

constexpr double KB = 1.38064852e-23 / 1.6021766208e-19;  // eV/K   (src/constants.jl:3)
constexpr double KE = 14.399645351950548;                  // eV*A/e^2 (src/constants.jl:4)
constexpr double PI = 3.14159265358979323846;

// ---------------------------------------------------------------------------------------------
// Counter-based RNG (src/state.jl:225-230, src/rng.jl:14-81)
// ---------------------------------------------------------------------------------------------
inline uint64_t splitmix64(uint64_t seed, uint64_t index) {
    uint64_t z = seed + index * 0x9E3779B97F4A7C15ULL;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

// High 64 bits of a*b from four 32-bit partial products (src/rng.jl:14-23).
inline uint64_t mulhi64(uint64_t a, uint64_t b) {
    uint64_t alo = a & 0xffffffffULL, ahi = a >> 32, blo = b & 0xffffffffULL, bhi = b >> 32;
    uint64_t ll = alo * blo, hl = ahi * blo, lh = alo * bhi, hh = ahi * bhi;
    uint64_t cross = (ll >> 32) + (hl & 0xffffffffULL) + (lh & 0xffffffffULL);
    return hh + (hl >> 32) + (lh >> 32) + (cross >> 32);
}

inline uint64_t chain_key(uint64_t chain_seed, uint64_t cycle, uint64_t move) {
    return splitmix64(splitmix64(chain_seed, cycle), move);
}

inline double unit_f64(uint64_t raw) { return double(raw >> 11) * 1.1102230246251565e-16; }
inline float unit_f32(uint64_t raw) { return float(raw >> 40) * 5.9604645e-8f; }

// sin(2*pi*u), cos(2*pi*u) for u in [0, 1): y = 4u, q = rint(y), r = y - q (exact), then the
// Taylor series of sin/cos((pi/2) r) on |r| <= 1/2, Horner in r^2 with fused multiply-adds,
// rotated by the quadrant q mod 4. Coefficients are (-1)^k (pi/2)^n / n! rounded to the type.
const double SIN64[9] = {1.5707963267948966, -0.6459640975062463, 0.07969262624616705,
                         -0.004681754135318688, 0.00016044118478735983, -3.598843235212085e-06,
                         5.692172921967927e-08, -6.688035109811468e-10, 6.0669357311061955e-12};
const double COS64[10] = {1.0, -1.2337005501361697, 0.25366950790104803, -0.02086348076335296,
                          0.0009192602748394266, -2.5202042373060607e-05, 4.710874778818172e-07,
                          -6.386603083791852e-09, 6.565963114979473e-11, -5.294400200734623e-13};
template <typename F> struct Poly;
template <> struct Poly<double> {
    static double s(double z) { double p = SIN64[8]; for (int k = 7; k >= 0; --k) p = std::fma(p, z, SIN64[k]); return p; }
    static double c(double z) { double p = COS64[9]; for (int k = 8; k >= 0; --k) p = std::fma(p, z, COS64[k]); return p; }
};

inline void sincos2pi(double u, double* sn, double* cs) {
    double y = u * 4.0;
    double q = std::nearbyint(y);  // round half to even (default rounding mode)
    double r = y - q;
    double z = r * r;
    double s = r * Poly<double>::s(z);
    double c = Poly<double>::c(z);
    int qi = int(q) & 3;
    switch (qi) {
        case 0: *sn = s; *cs = c; break;
        case 1: *sn = c; *cs = -s; break;
        case 2: *sn = -s; *cs = -c; break;
        default: *sn = -c; *cs = s; break;
    }
}
// FP32 (Float32 sinpi(2u), cospi(2u), src/rng.jl:126-129): the FP64 values rounded once, which is
// the correctly rounded result for every FP32 uniform; zeros as +0
inline void sincos2pi(float u, float* sn, float* cs) {
    double s, c;
    sincos2pi(double(u), &s, &c);
    *sn = float(s) + 0.0f;
    *cs = float(c) + 0.0f;
}

template <typename F> inline F unit(uint64_t raw);
template <> inline double unit<double>(uint64_t raw) { return unit_f64(raw); }
template <> inline float unit<float>(uint64_t raw) { return unit_f32(raw); }

// Pose of the k-th (1-based) insertion into system s (1-based): the stream of
// ChainRNG(splitmix64(seed, s), k, 0) (src/rng.jl:43-61 keyed like src/state.jl:434), draws 0..5
// giving the fractional position (u_x, u_y, u_z) and Shoemake's (u1, u2, u3); the quaternion is
// (x, y, z, w) = (sqrt(1-u1) cos 2pi u2, sqrt(u1) sin 2pi u3, sqrt(u1) cos 2pi u3,
// sqrt(1-u1) sin 2pi u2) (src/rng.jl:126-141, src/widom.jl:55-61).
template <typename F>
inline void pose(uint64_t seed, uint64_t s, uint64_t k, F rpos[3], F quat[4]) {
    uint64_t key = chain_key(splitmix64(seed, s), k, 0);
    F u[6];
    for (int d = 0; d < 6; ++d) u[d] = unit<F>(splitmix64(key, uint64_t(d)));
    rpos[0] = u[0]; rpos[1] = u[1]; rpos[2] = u[2];
    F a = std::sqrt(F(1) - u[3]), b = std::sqrt(u[3]);
    F s2, c2, s3, c3;
    sincos2pi(u[4], &s2, &c2);
    sincos2pi(u[5], &s3, &c3);
    quat[0] = a * c2; quat[1] = b * s3; quat[2] = b * c3; quat[3] = a * s2;
}

// ---------------------------------------------------------------------------------------------
// Strict small linear algebra (fixed operation order, explicit fma) shared by the pose and
// phase-0 code. Matrices are 3x3 column-major (M[r + 3c]).
// ---------------------------------------------------------------------------------------------
template <typename F> inline F sfma(F a, F b, F c) { return std::fma(a, b, c); }
template <typename F> inline F dot3(F a0, F a1, F a2, F b0, F b1, F b2) {
    return sfma(a2, b2, sfma(a1, b1, a0 * b0));
}
template <typename F> inline void matvec(const F* M, const F* v, F* out) {
    for (int r = 0; r < 3; ++r) out[r] = dot3(M[r], M[r + 3], M[r + 6], v[0], v[1], v[2]);
}
template <typename F> inline F crossc(F a, F b, F c, F d) { return sfma(a, b, -(c * d)); }
// v + 2 u x (u x v + w v), q = (u, w) (src/energy.jl:13-16)
template <typename F> inline void rotate_strict(const F* q, const F* v, F* out) {
    F t0 = sfma(q[3], v[0], crossc(q[1], v[2], q[2], v[1]));
    F t1 = sfma(q[3], v[1], crossc(q[2], v[0], q[0], v[2]));
    F t2 = sfma(q[3], v[2], crossc(q[0], v[1], q[1], v[0]));
    F c0 = crossc(q[1], t2, q[2], t1);
    F c1 = crossc(q[2], t0, q[0], t2);
    F c2 = crossc(q[0], t1, q[1], t0);
    out[0] = sfma(F(2), c0, v[0]); out[1] = sfma(F(2), c1, v[1]); out[2] = sfma(F(2), c2, v[2]);
}
// D - A round(invA D) (src/cell.jl:34-37), round half to even
template <typename F> inline void minimum_image_strict(const F* A, const F* invA, F* D) {
    F f[3]; matvec(invA, D, f);
    F r0 = std::nearbyint(f[0]), r1 = std::nearbyint(f[1]), r2 = std::nearbyint(f[2]);
    for (int r = 0; r < 3; ++r) D[r] = D[r] - dot3(A[r], A[r + 3], A[r + 6], r0, r1, r2);
}

// ---------------------------------------------------------------------------------------------
// Geometry (src/cell.jl)
// ---------------------------------------------------------------------------------------------
inline void inv3(const double* A, double* B) {  // general 3x3 inverse, column-major
    double a = A[0], b = A[3], c = A[6], d = A[1], e = A[4], f = A[7], g = A[2], h = A[5], i = A[8];
    double det = a * (e * i - f * h) - b * (d * i - f * g) + c * (d * h - e * g);
    double r[9] = {(e * i - f * h), -(d * i - f * g), (d * h - e * g),
                   -(b * i - c * h), (a * i - c * g), -(a * h - b * g),
                   (b * f - c * e), -(a * f - c * d), (a * e - b * d)};
    // r holds the cofactor matrix row-major as [C00 C01 C02; C10 ...]; inverse = C^T / det
    for (int row = 0; row < 3; ++row)
        for (int col = 0; col < 3; ++col) B[row + 3 * col] = r[3 * col + row] / det;
}
inline double det3(const double* A) {
    return A[0] * (A[4] * A[8] - A[7] * A[5]) - A[3] * (A[1] * A[8] - A[7] * A[2]) + A[6] * (A[1] * A[5] - A[4] * A[2]);
}
inline void cross3(const double* a, const double* b, double* c) {
    c[0] = a[1] * b[2] - a[2] * b[1]; c[1] = a[2] * b[0] - a[0] * b[2]; c[2] = a[0] * b[1] - a[1] * b[0];
}
inline double norm3(const double* a) { return std::sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]); }
inline void perpendicular_lengths(const double* A, double* L) {
    double V = std::fabs(det3(A)), c[3];
    cross3(A + 3, A + 6, c); L[0] = V / norm3(c);
    cross3(A + 0, A + 6, c); L[1] = V / norm3(c);
    cross3(A + 0, A + 3, c); L[2] = V / norm3(c);
}
inline int32_t grid_dim(double L, double w) { return int32_t(std::max(1.0, std::floor(L / w))); }
inline int32_t stencil_reach(double L, int32_t n, double reach) { return int32_t(std::ceil(reach * n / L)); }
inline int32_t home_cell(double f, int32_t n) { return std::min(int32_t(std::floor(f * n)), n - 1); }
template <typename F> inline int32_t home_cell_dev(F f, int32_t n) {
    F x = std::max(f * F(n), F(0));
    return std::min(int32_t(x), n - 1);
}
template <typename F> inline F wrap_frac(F f) { return f - std::floor(f); }
inline int32_t wrap_cell(int32_t x, int32_t n) { return x + n * int32_t(x < 0) - n * int32_t(x >= n); }
inline void stencil_start_count(int32_t h, int32_t m, int32_t n, int32_t* start, int32_t* count) {
    int32_t span = m + m + 1;
    *count = std::min(span, n);
    *start = span >= n ? 0 : h - m;
}

// ---------------------------------------------------------------------------------------------
// Ewald (src/ewald.jl)
// ---------------------------------------------------------------------------------------------
// alpha with erfc(alpha rc) = rc * precision / 2 by bisection (src/ewald.jl:21-32); the
// reference's SpecialFunctions.erfc is replaced by glibc erfc (both accurate to ~1 ulp).
double ewald_alpha(double cutoff, double precision) {
    double target = cutoff * precision / 2, lo = 0.0, hi = 20.0;
    for (int it = 0; it < 200; ++it) {
        double mid = (lo + hi) / 2;
        if (std::erfc(mid) - target > 0) lo = mid; else hi = mid;
        if (hi - lo < 1.0e-12) break;
    }
    return (lo + hi) / 2 / cutoff;
}
inline double ewald_kmax(double alpha, double precision) { return 2 * alpha * std::sqrt(-std::log(precision / 2)); }
inline double pk(double k2, double alpha, double V) { return 2 * PI / V * std::exp(-k2 / (4 * alpha * alpha)) / k2; }

struct KVecs { std::vector<double> k; std::vector<double> w; std::vector<int32_t> n; };
// Half-space enumeration n1 >= 0, weight 2 for n1 > 0 (src/ewald.jl:142-157).
KVecs kvectors(const double* A, double kmax) {
    double invA[9], B[9];
    inv3(A, invA);
    for (int r = 0; r < 3; ++r) for (int c = 0; c < 3; ++c) B[r + 3 * c] = 2 * PI * invA[c + 3 * r];
    int nmax[3];
    for (int i = 0; i < 3; ++i) nmax[i] = int(std::ceil(kmax * norm3(A + 3 * i) / (2 * PI)));
    KVecs out;
    for (int n1 = 0; n1 <= nmax[0]; ++n1)
        for (int n2 = -nmax[1]; n2 <= nmax[1]; ++n2)
            for (int n3 = -nmax[2]; n3 <= nmax[2]; ++n3) {
                if (n1 == 0 && n2 == 0 && n3 == 0) continue;
                double k[3];
                for (int r = 0; r < 3; ++r) k[r] = B[r] * n1 + B[r + 3] * n2 + B[r + 6] * n3;
                if (norm3(k) > kmax) continue;
                out.k.insert(out.k.end(), k, k + 3);
                out.w.push_back(n1 == 0 ? 1.0 : 2.0);
                out.n.push_back(n1); out.n.push_back(n2); out.n.push_back(n3);
            }
    return out;
}
// S(k) = sum_j q_j exp(i k.r_j) (src/ewald.jl:159-170)
void structure_factor(const double* ks, int64_t nk, const double* pos, const double* q, int64_t na, double* S) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < nk; ++i) {
        double re = 0, im = 0;
        for (int64_t j = 0; j < na; ++j) {
            double ph = ks[3 * i] * pos[3 * j] + ks[3 * i + 1] * pos[3 * j + 1] + ks[3 * i + 2] * pos[3 * j + 2];
            re += q[j] * std::cos(ph);
            im += q[j] * std::sin(ph);
        }
        S[2 * i] = re; S[2 * i + 1] = im;
    }
}

// ---------------------------------------------------------------------------------------------
// Force field (src/forcefield.jl:22-39, 103-124)
// ---------------------------------------------------------------------------------------------
struct FF {
    int n; std::vector<double> sigma, epsilon;  // n x n column-major
    double cutoff; bool tail;
};
FF lorentz_berthelot(int n, const double* s, const double* e, double cutoff, bool tail) {
    FF ff; ff.n = n; ff.cutoff = cutoff; ff.tail = tail;
    ff.sigma.resize(n * n); ff.epsilon.resize(n * n);
    for (int a = 0; a < n; ++a)
        for (int b = 0; b < n; ++b) {
            ff.sigma[a + n * b] = (s[a] + s[b]) / 2;
            ff.epsilon[a + n * b] = std::sqrt(e[a] * e[b]);
        }
    return ff;
}
double tail_delta(const FF& ff, const std::vector<int64_t>& counts, const std::vector<int64_t>& gcounts, double V) {
    if (!ff.tail) return 0.0;
    double acc = 0;
    for (int a = 0; a < ff.n; ++a)
        for (int b = 0; b < ff.n; ++b) {
            double eps = ff.epsilon[a + ff.n * b];
            double c = 0;
            if (eps != 0) {
                double s = ff.sigma[a + ff.n * b], x = s / ff.cutoff;
                c = eps * s * s * s * (std::pow(x, 9) / 3 - x * x * x);
            }
            acc += 2 * double(counts[a]) * double(gcounts[b]) * c + double(gcounts[a]) * double(gcounts[b]) * c;
        }
    return 8 * PI / 3 / V * acc;
}

// ---------------------------------------------------------------------------------------------
// Pair terms, rejection bounds (src/energy.jl:20, src/reject.jl)
// ---------------------------------------------------------------------------------------------
inline double lj_pair(double r2, double s, double e) { double x = s * s / r2; x = x * x * x; return 4 * e * (x * x - x); }
inline double pair_energy(double r, double s, double e, double K, double alpha) {
    return lj_pair(r * r, s, e) + K * std::erfc(alpha * r) / r;
}
constexpr int MAX_BISECT = 200;
const double EPS64 = 2.220446049250313e-16;

// first root below the LJ minimum of the attractive pair energy, clamped to r_lj (src/reject.jl:46-69)
double find_r0(double s, double e, double K, double alpha, double r_lj, int* err) {
    *err = 0;
    if (!(e > 0) || !(K < 0)) { *err = 1; return 0; }
    double hi = s * std::pow(2.0, 1.0 / 6);
    if (!(pair_energy(hi, s, e, K, alpha) < 0)) { *err = 2; return 0; }
    double lo = hi; int it = 0;
    while (pair_energy(lo, s, e, K, alpha) <= 0) { lo /= 2; if (++it > MAX_BISECT) { *err = 3; return 0; } }
    it = 0;
    while (hi - lo > 4 * EPS64 * hi) {
        double mid = (lo + hi) / 2;
        if (pair_energy(mid, s, e, K, alpha) > 0) lo = mid; else hi = mid;
        if (++it > MAX_BISECT) { *err = 4; return 0; }
    }
    return std::min((lo + hi) / 2, r_lj);
}
// rho^2: first root of LJ(r) - |kmin|/r = margin, clamped to r_lj (src/reject.jl:168-209)
double find_rho2(double s, double e, double kmin, double margin, double r_lj, int* err) {
    *err = 0;
    if (!(margin > 0)) { *err = 1; return 0; }
    if (std::isinf(margin)) return 0;
    if (e == 0) return 0;
    auto f = [&](double r) { return lj_pair(r * r, s, e) - std::fabs(kmin) / r - margin; };
    double hi = s; int it = 0;
    while (f(hi) >= 0) { hi *= 2; if (++it > MAX_BISECT) { *err = 2; return 0; } }
    double lo = hi; it = 0;
    while (f(lo) < 0) { lo /= 2; if (++it > MAX_BISECT) { *err = 3; return 0; } }
    it = 0;
    while (hi - lo > 4 * EPS64 * hi) {
        double mid = (lo + hi) / 2;
        if (f(mid) > 0) lo = mid; else hi = mid;
        if (++it > MAX_BISECT) { *err = 4; return 0; }
    }
    double r = std::min((lo + hi) / 2, r_lj);
    return r * r;
}

// smallest theta with exp(-theta) == 0 in the type, by bisection on the float grid (src/reject.jl:11-19)
template <typename F> F theta_F() {
    F lo = 0, hi = 2000;
    while (std::nextafter(lo, hi) != hi) {
        F mid = lo + (hi - lo) / 2;
        if (std::exp(-mid) == F(0)) hi = mid; else lo = mid;
    }
    return hi;
}

}  // namespace

// =============================================================================================
// C ABI
// =============================================================================================
extern "C" {

uint64_t or_splitmix64(uint64_t seed, uint64_t index) { return splitmix64(seed, index); }
uint64_t or_mulhi64(uint64_t a, uint64_t b) { return mulhi64(a, b); }
uint64_t or_chain_bits(uint64_t chain_seed, uint64_t cycle, uint64_t move, uint64_t draw) {
    return splitmix64(chain_key(chain_seed, cycle, move), draw);
}
double or_unit_f64(uint64_t raw) { return unit_f64(raw); }
float or_unit_f32(uint64_t raw) { return unit_f32(raw); }
// Lemire multiply-shift ranged draw in 1:n (src/rng.jl:93-97)
int64_t or_rand_range(uint64_t raw, int64_t n) { return int64_t(mulhi64(raw, uint64_t(n))) + 1; }

void or_sincos2pi_f64(const double* u, int64_t n, double* s, double* c) { for (int64_t i = 0; i < n; ++i) sincos2pi(u[i], s + i, c + i); }
void or_sincos2pi_f32(const float* u, int64_t n, float* s, float* c) { for (int64_t i = 0; i < n; ++i) sincos2pi(u[i], s + i, c + i); }

void or_poses_f64(uint64_t seed, int64_t s, int64_t k0, int64_t n, double* rpos, double* quat) {
    for (int64_t i = 0; i < n; ++i) pose<double>(seed, uint64_t(s), uint64_t(k0 + i), rpos + 3 * i, quat + 4 * i);
}
void or_poses_f32(uint64_t seed, int64_t s, int64_t k0, int64_t n, float* rpos, float* quat) {
    for (int64_t i = 0; i < n; ++i) pose<float>(seed, uint64_t(s), uint64_t(k0 + i), rpos + 3 * i, quat + 4 * i);
}

double or_theta_f64(void) { return theta_F<double>(); }
float or_theta_f32(void) { return theta_F<float>(); }
double or_erfc(double x) { return std::erfc(x); }
double or_ewald_alpha(double cutoff, double precision) { return ewald_alpha(cutoff, precision); }
double or_ewald_kmax(double alpha, double precision) { return ewald_kmax(alpha, precision); }
double or_pk(double k2, double alpha, double V) { return pk(k2, alpha, V); }

// k-vectors of cell A (column-major) within kmax; returns the count and fills up to cap entries.
int64_t or_kvectors(const double* A, double kmax, double* ks, double* w, int32_t* coeffs, int64_t cap) {
    KVecs kv = kvectors(A, kmax);
    int64_t n = int64_t(kv.w.size());
    for (int64_t i = 0; i < std::min(n, cap); ++i) {
        for (int r = 0; r < 3; ++r) { ks[3 * i + r] = kv.k[3 * i + r]; coeffs[3 * i + r] = kv.n[3 * i + r]; }
        w[i] = kv.w[i];
    }
    return n;
}
void or_structure_factor(const double* ks, int64_t nk, const double* pos, const double* q, int64_t na, double* S) {
    structure_factor(ks, nk, pos, q, na, S);
}

// Full Ewald energy of one periodic system with intramolecular exclusions (src/ewald.jl:177-203).
double or_ewald_energy(const double* A, const double* pos, const double* q, const int32_t* mol, int64_t n,
                       double alpha, double cutoff, const double* ks, const double* w, int64_t nk) {
    double invA[9]; inv3(A, invA);
    double V = std::fabs(det3(A));
    double Esr = 0, Eexcl = 0;
    for (int64_t i = 0; i < n; ++i)
        for (int64_t j = i + 1; j < n; ++j) {
            double D[3] = {pos[3 * j] - pos[3 * i], pos[3 * j + 1] - pos[3 * i + 1], pos[3 * j + 2] - pos[3 * i + 2]};
            if (mol[i] == mol[j]) {
                double r = norm3(D);
                Eexcl -= q[i] * q[j] * (1 - std::erfc(alpha * r)) / r;
            } else {
                minimum_image_strict<double>(A, invA, D);
                double r = norm3(D);
                if (r < cutoff) Esr += q[i] * q[j] * std::erfc(alpha * r) / r;
            }
        }
    std::vector<double> S(2 * nk);
    structure_factor(ks, nk, pos, q, n, S.data());
    double Elr = 0;
    for (int64_t i = 0; i < nk; ++i) {
        double k2 = ks[3 * i] * ks[3 * i] + ks[3 * i + 1] * ks[3 * i + 1] + ks[3 * i + 2] * ks[3 * i + 2];
        Elr += w[i] * pk(k2, alpha, V) * (S[2 * i] * S[2 * i] + S[2 * i + 1] * S[2 * i + 1]);
    }
    double q2 = 0, Q = 0;
    for (int64_t i = 0; i < n; ++i) { q2 += q[i] * q[i]; Q += q[i]; }
    double Eself = -alpha / std::sqrt(PI) * q2;
    double Enet = -PI / (2 * V * alpha * alpha) * Q * Q;
    return KE * (Esr + Elr + Eself + Eexcl + Enet);
}

double or_find_r0(double s, double e, double K, double alpha, double r_lj, int* err) { return find_r0(s, e, K, alpha, r_lj, err); }
double or_find_rho2(double s, double e, double kmin, double margin, double r_lj, int* err) { return find_rho2(s, e, kmin, margin, r_lj, err); }
double or_pair_energy(double r, double s, double e, double K, double alpha) { return pair_energy(r, s, e, K, alpha); }

}  // extern "C"

// =============================================================================================
// FrameworkBatch construction (src/batch.jl:237-432) and the widom path (src/widom.jl)
// =============================================================================================
namespace {

struct FwIn {
    double cell[9]; int64_t natoms; const double* frac; const int32_t* types; const double* charges; int32_t rep[3];
};

// A batch in the reference's FrameworkBatch layout (0-based offsets, 1-based type and
// framework indices, FP64).
struct Batch {
    std::vector<double> positions; std::vector<int32_t> types; std::vector<double> charges;
    std::vector<int32_t> atom_offsets{0};
    std::vector<double> cells, invcells, volumes, alphas;
    std::vector<double> ks, kprefactor, Shost; std::vector<int32_t> kcoeffs; std::vector<int32_t> k_offsets{0};
    std::vector<double> constant_offset, self_term_halfrange;
    std::vector<int32_t> ncells, cell_offsets, cellgrid_offsets{0};
    std::vector<double> sigma, epsilon; std::vector<int32_t> compact_to_orig, guest_types;
    std::vector<double> bs, kmin;
    std::vector<int32_t> framework_of;
    std::vector<int32_t> perm;  // cell-sort permutation per framework, concatenated (0-based, local)
    int32_t ntypes = 0, nsys = 0, nfw = 0;
    double cutoff = 0, ewald_cutoff = 0;
    std::string error;
};

}  // namespace

extern "C" {

// Builds the batch. Frameworks are given as flat arrays: cells (9 per framework, column-major),
// natoms, frac (3 per atom), orig types (1-based force-field index per atom), charges,
// replication (3 per framework). ff_sigma/ff_epsilon are per force-field type (Lorentz-Berthelot
// mixing is applied here). The self-term orientations are nself poses passed in as quaternions
// (4 per orientation), so caller and oracle agree on them.
void* or_batch_build(int32_t nfw_in, const double* cells, const int64_t* natoms, const double* frac,
                     const int32_t* types, const double* charges, const int32_t* rep,
                     int32_t nff, const double* ff_sigma, const double* ff_epsilon, double ff_cutoff, int32_t tail,
                     int32_t nguest, const double* gsites, const int32_t* gtypes, const double* gcharges,
                     double ew_cutoff, double ew_precision, double cellwidth, int32_t fullk,
                     int32_t nself, const double* self_quats) {
    Batch* B = new Batch();
    FF ff = lorentz_berthelot(nff, ff_sigma, ff_epsilon, ff_cutoff, tail != 0);
    double rg = 0;
    for (int a = 0; a < nguest; ++a) rg = std::max(rg, norm3(gsites + 3 * a));
    double rc = std::max(ff_cutoff, ew_cutoff), rc_guard = rc + rg;
    // dedup by value (src/batch.jl:252-265)
    std::vector<FwIn> in(nfw_in);
    int64_t aoff = 0;
    for (int n = 0; n < nfw_in; ++n) {
        std::memcpy(in[n].cell, cells + 9 * n, 9 * sizeof(double));
        in[n].natoms = natoms[n]; in[n].frac = frac + 3 * aoff; in[n].types = types + aoff; in[n].charges = charges + aoff;
        for (int r = 0; r < 3; ++r) in[n].rep[r] = rep[3 * n + r];
        aoff += natoms[n];
    }
    auto same = [&](const FwIn& a, const FwIn& b) {
        if (a.natoms != b.natoms) return false;
        if (std::memcmp(a.cell, b.cell, 9 * sizeof(double)) != 0) return false;
        for (int r = 0; r < 3; ++r) if (a.rep[r] != b.rep[r]) return false;
        for (int64_t j = 0; j < a.natoms; ++j) {
            if (a.types[j] != b.types[j] || a.charges[j] != b.charges[j]) return false;
            for (int r = 0; r < 3; ++r) if (a.frac[3 * j + r] != b.frac[3 * j + r]) return false;
        }
        return true;
    };
    std::vector<int> uniq;
    for (int n = 0; n < nfw_in; ++n) {
        int idx = -1;
        for (size_t u = 0; u < uniq.size(); ++u) if (same(in[uniq[u]], in[n])) { idx = int(u); break; }
        if (idx < 0) { uniq.push_back(n); idx = int(uniq.size()) - 1; }
        B->framework_of.push_back(idx + 1);
    }
    B->nsys = nfw_in; B->nfw = int32_t(uniq.size());
    // compact types: sorted union of framework and guest types (src/batch.jl:309-317)
    std::vector<int32_t> all;
    for (int u : uniq) for (int64_t j = 0; j < in[u].natoms; ++j) all.push_back(in[u].types[j]);
    for (int a = 0; a < nguest; ++a) all.push_back(gtypes[a]);
    std::sort(all.begin(), all.end()); all.erase(std::unique(all.begin(), all.end()), all.end());
    B->compact_to_orig = all; B->ntypes = int32_t(all.size());
    std::map<int32_t, int32_t> o2c;
    for (size_t i = 0; i < all.size(); ++i) o2c[all[i]] = int32_t(i + 1);
    int nt = B->ntypes;
    B->sigma.resize(nt * nt); B->epsilon.resize(nt * nt);
    for (int a = 0; a < nt; ++a) for (int b = 0; b < nt; ++b) {
        B->sigma[a + nt * b] = ff.sigma[(all[a] - 1) + nff * (all[b] - 1)];
        B->epsilon[a + nt * b] = ff.epsilon[(all[a] - 1) + nff * (all[b] - 1)];
    }
    for (int a = 0; a < nguest; ++a) B->guest_types.push_back(o2c[gtypes[a]]);
    B->cutoff = ff_cutoff; B->ewald_cutoff = ew_cutoff;
    double alpha = ewald_alpha(ew_cutoff, ew_precision);
    if (alpha * ew_cutoff > 4.0) { B->error = "alpha*ewald_cutoff exceeds PAIR_ERFC_XMAX"; return B; }
    double kmax = ewald_kmax(alpha, ew_precision);
    bool neutral = true;
    for (int a = 0; a < nguest; ++a) if (gcharges[a] != 0) neutral = false;
    std::vector<int64_t> gcounts(nff, 0);
    for (int a = 0; a < nguest; ++a) gcounts[gtypes[a] - 1] += 1;

    for (size_t n = 0; n < uniq.size(); ++n) {
        const FwIn& fw = in[uniq[n]];
        double L[3]; perpendicular_lengths(fw.cell, L);
        for (int r = 0; r < 3; ++r)
            if (int(std::ceil(2 * rc_guard / L[r])) != 1) { B->error = "framework " + std::to_string(n + 1) + " is too small; replicate it"; return B; }
        int32_t ng[3]; for (int r = 0; r < 3; ++r) ng[r] = grid_dim(L[r], cellwidth);
        int64_t na = fw.natoms;
        // cell sort (src/cell.jl:96-118): stable counting sort by the wrapped fractional cell
        int64_t ncell = int64_t(ng[0]) * ng[1] * ng[2];
        std::vector<int32_t> cidx(na), counts(ncell, 0);
        for (int64_t a = 0; a < na; ++a) {
            int32_t c3[3];
            for (int r = 0; r < 3; ++r) {
                double f = fw.frac[3 * a + r]; double fwp = f - std::floor(f);
                c3[r] = home_cell(fwp, ng[r]);
            }
            int32_t c = c3[0] + ng[0] * (c3[1] + ng[1] * c3[2]);
            cidx[a] = c; counts[c] += 1;
        }
        std::vector<int32_t> offs(ncell + 1, 0);
        for (int64_t c = 0; c < ncell; ++c) offs[c + 1] = offs[c] + counts[c];
        std::vector<int32_t> cur(offs.begin(), offs.end() - 1), perm(na);
        for (int64_t a = 0; a < na; ++a) perm[cur[cidx[a]]++] = int32_t(a);
        // cartesian positions A*frac
        std::vector<double> pos(3 * na);
        for (int64_t a = 0; a < na; ++a)
            for (int r = 0; r < 3; ++r)
                pos[3 * a + r] = fw.cell[r] * fw.frac[3 * a] + fw.cell[r + 3] * fw.frac[3 * a + 1] + fw.cell[r + 6] * fw.frac[3 * a + 2];
        for (int64_t a = 0; a < na; ++a) {
            int32_t p = perm[a];
            for (int r = 0; r < 3; ++r) B->positions.push_back(pos[3 * p + r]);
            B->types.push_back(o2c[fw.types[p]]);
            B->charges.push_back(fw.charges[p]);
            B->perm.push_back(p);
        }
        B->atom_offsets.push_back(int32_t(B->positions.size() / 3));
        B->cell_offsets.insert(B->cell_offsets.end(), offs.begin(), offs.end());
        B->cellgrid_offsets.push_back(int32_t(B->cell_offsets.size()));
        for (int r = 0; r < 3; ++r) B->ncells.push_back(ng[r]);
        double invA[9]; inv3(fw.cell, invA);
        double V = std::fabs(det3(fw.cell));
        B->cells.insert(B->cells.end(), fw.cell, fw.cell + 9);
        B->invcells.insert(B->invcells.end(), invA, invA + 9);
        B->volumes.push_back(V); B->alphas.push_back(alpha);
        bool replicated = !(fw.rep[0] == 1 && fw.rep[1] == 1 && fw.rep[2] == 1);
        KVecs kv; std::vector<double> kpref, Sh;
        if (!neutral || replicated) {
            kv = kvectors(fw.cell, kmax);
            int64_t nk = int64_t(kv.w.size());
            kpref.resize(nk); Sh.resize(2 * nk);
            for (int64_t i = 0; i < nk; ++i) {
                double k2 = kv.k[3 * i] * kv.k[3 * i] + kv.k[3 * i + 1] * kv.k[3 * i + 1] + kv.k[3 * i + 2] * kv.k[3 * i + 2];
                kpref[i] = kv.w[i] * pk(k2, alpha, V);
            }
            structure_factor(kv.k.data(), nk, pos.data(), fw.charges, na, Sh.data());
            if (replicated) {  // verify_replication (src/batch.jl:173-195)
                std::vector<int64_t> unc;
                for (int64_t i = 0; i < nk; ++i) {
                    bool cpl = true;
                    for (int r = 0; r < 3; ++r) { int m = kv.n[3 * i + r] % fw.rep[r]; if (m != 0) cpl = false; }
                    if (!cpl) unc.push_back(i);
                }
                if (!unc.empty()) {
                    int64_t stride = std::max<int64_t>(1, (int64_t(unc.size()) + 31) / 32);
                    std::vector<int64_t> sample;
                    for (size_t i = 0; i < unc.size() && sample.size() < 32; i += size_t(stride)) sample.push_back(unc[i]);
                    double maxS = 0, sq = 0;
                    for (int64_t j = 0; j < na; ++j) sq += std::fabs(fw.charges[j]);
                    for (int64_t i : sample) maxS = std::max(maxS, std::hypot(Sh[2 * i], Sh[2 * i + 1]));
                    double thr = std::max(1.0e-8, 100 * EPS64) * sq;
                    if (maxS > thr) { B->error = "framework " + std::to_string(n + 1) + " claims replication that does not describe the atoms"; return B; }
                }
            }
        }
        double self_mean = 0;
        if (!neutral) {
            int64_t nk = int64_t(kv.w.size());
            for (int64_t i = 0; i < nk; ++i) {
                bool cpl = true;
                for (int r = 0; r < 3; ++r) if (kv.n[3 * i + r] % fw.rep[r] != 0) cpl = false;
                if (fullk || cpl) {
                    for (int r = 0; r < 3; ++r) { B->ks.push_back(kv.k[3 * i + r]); B->kcoeffs.push_back(kv.n[3 * i + r]); }
                    B->kprefactor.push_back(kpref[i]);
                    B->Shost.push_back(Sh[2 * i]); B->Shost.push_back(Sh[2 * i + 1]);
                }
            }
            // orientation-averaged guest self term over the full k set (src/batch.jl:354-386)
            std::vector<double> samples(nself);
            for (int o = 0; o < nself; ++o) {
                const double* q = self_quats + 4 * o;
                std::vector<double> gs(3 * nguest);
                for (int a = 0; a < nguest; ++a) rotate_strict<double>(q, gsites + 3 * a, gs.data() + 3 * a);
                double acc = 0;
                for (int64_t i = 0; i < nk; ++i) {
                    double re = 0, im = 0;
                    for (int a = 0; a < nguest; ++a) {
                        double ph = kv.k[3 * i] * gs[3 * a] + kv.k[3 * i + 1] * gs[3 * a + 1] + kv.k[3 * i + 2] * gs[3 * a + 2];
                        re += gcharges[a] * std::cos(ph); im += gcharges[a] * std::sin(ph);
                    }
                    acc += kpref[i] * (re * re + im * im);
                }
                samples[o] = KE * acc;
            }
            double sum = 0, mx = -1e300, mn = 1e300;
            for (double v : samples) { sum += v; mx = std::max(mx, v); mn = std::min(mn, v); }
            self_mean = nself > 0 ? sum / nself : 0.0;
            double half = nself > 0 ? (mx - mn) / 2 : 0.0;
            B->self_term_halfrange.push_back(half);
            if (2 * half / (KB * 300) > 1.0e-3) { B->error = "guest self-term half-range exceeds the guard"; return B; }
        } else {
            B->self_term_halfrange.push_back(0.0);
        }
        B->k_offsets.push_back(int32_t(B->kprefactor.size()));
        // kmin table (src/reject.jl:134-145)
        int64_t a0 = B->atom_offsets[B->atom_offsets.size() - 2], a1 = B->atom_offsets.back();
        std::vector<double> km(nguest * nt, 0.0);
        for (int a = 0; a < nguest; ++a)
            for (int64_t h = a0; h < a1; ++h) {
                double K = KE * gcharges[a] * B->charges[h];
                int t = B->types[h] - 1;
                if (K < km[a * nt + t]) km[a * nt + t] = K;
            }
        B->kmin.insert(B->kmin.end(), km.begin(), km.end());
        // constant offset (src/batch.jl:396-407)
        std::vector<int64_t> cnt(nff, 0);
        for (int64_t j = 0; j < na; ++j) cnt[fw.types[j] - 1] += 1;
        double q2 = 0, Qg = 0, Qh = 0;
        for (int a = 0; a < nguest; ++a) { q2 += gcharges[a] * gcharges[a]; Qg += gcharges[a]; }
        for (int64_t j = 0; j < na; ++j) Qh += fw.charges[j];
        double self = -alpha / std::sqrt(PI) * q2, excl = 0;
        for (int a = 0; a < nguest; ++a)
            for (int c = a + 1; c < nguest; ++c) {
                double d[3] = {gsites[3 * a] - gsites[3 * c], gsites[3 * a + 1] - gsites[3 * c + 1], gsites[3 * a + 2] - gsites[3 * c + 2]};
                double r = norm3(d);
                excl -= gcharges[a] * gcharges[c] * (1 - std::erfc(alpha * r)) / r;
            }
        double net = -PI / (2 * V * alpha * alpha) * ((Qh + Qg) * (Qh + Qg) - Qh * Qh);
        B->constant_offset.push_back(tail_delta(ff, cnt, gcounts, V) + KE * (self + excl + net) + self_mean);
    }
    // hardcore bound per framework (src/reject.jl:95-124)
    B->bs.resize(B->nfw);
    for (int n = 0; n < B->nfw; ++n) {
        int64_t a0 = B->atom_offsets[n], a1 = B->atom_offsets[n + 1];
        double acc = 0; bool inf = false;
        for (int a = 0; a < nguest && !inf; ++a) {
            int gt = B->guest_types[a] - 1;
            for (int64_t h = a0; h < a1; ++h) {
                int ht = B->types[h] - 1;
                double s = B->sigma[gt + nt * ht], e = B->epsilon[gt + nt * ht];
                double K = KE * gcharges[a] * B->charges[h];
                if (K >= 0) acc += e;
                else {
                    if (e == 0) { inf = true; break; }
                    int err; double r0 = find_r0(s, e, K, alpha, ff_cutoff, &err);
                    if (err) { B->error = "find_r0 failed"; return B; }
                    acc += e + std::fabs(K) * std::erfc(alpha * r0) / r0;
                }
            }
        }
        if (inf) { B->bs[n] = INFINITY; continue; }
        double Rs = 0;
        for (int32_t i = B->k_offsets[n]; i < B->k_offsets[n + 1]; ++i) Rs += B->kprefactor[i] * std::hypot(B->Shost[2 * i], B->Shost[2 * i + 1]);
        double sq = 0; for (int a = 0; a < nguest; ++a) sq += std::fabs(gcharges[a]);
        B->bs[n] = acc + 2 * KE * sq * Rs;
    }
    return B;
}

const char* or_batch_error(void* h) { Batch* B = (Batch*)h; return B->error.c_str(); }
void or_batch_free(void* h) { delete (Batch*)h; }

// Field access: returns the element count of field `f` and copies it into out (if non-null).
int64_t or_batch_field(void* h, const char* f, void* out) {
    Batch* B = (Batch*)h;
    std::string n(f);
#define OR_FIELD(name)                                                                               \
    if (n == #name) {                                                                                \
        if (out) std::memcpy(out, B->name.data(), B->name.size() * sizeof(B->name[0]));              \
        return int64_t(B->name.size());                                                              \
    }
    OR_FIELD(positions) OR_FIELD(types) OR_FIELD(charges) OR_FIELD(atom_offsets) OR_FIELD(cells)
    OR_FIELD(invcells) OR_FIELD(volumes) OR_FIELD(alphas) OR_FIELD(ks) OR_FIELD(kprefactor) OR_FIELD(Shost)
    OR_FIELD(kcoeffs) OR_FIELD(k_offsets) OR_FIELD(constant_offset) OR_FIELD(self_term_halfrange)
    OR_FIELD(ncells) OR_FIELD(cell_offsets) OR_FIELD(cellgrid_offsets) OR_FIELD(sigma) OR_FIELD(epsilon)
    OR_FIELD(compact_to_orig) OR_FIELD(guest_types) OR_FIELD(bs) OR_FIELD(kmin) OR_FIELD(framework_of) OR_FIELD(perm)
#undef OR_FIELD
    if (n == "ntypes") return B->ntypes;
    if (n == "nsys") return B->nsys;
    if (n == "nfw") return B->nfw;
    return -1;
}

}  // extern "C"

// ---------------------------------------------------------------------------------------------
// The widom path over an existing batch (any builder's tables, in the reference's layout)
// ---------------------------------------------------------------------------------------------
extern "C" {
typedef struct {
    int32_t nsys, nfw, ntypes, nguest;
    const double* positions; const int32_t* types; const double* charges; const int32_t* atom_offsets;
    const double* cells; const double* invcells; const double* volumes; const double* alphas;
    const double* ks; const double* kprefactor; const double* Shost; const int32_t* k_offsets;
    const double* constant_offset;
    const int32_t* ncells; const int32_t* cell_offsets; const int32_t* cellgrid_offsets;
    const double* sigma; const double* epsilon;
    const int32_t* guest_types; const double* guest_sites; const double* guest_charges;
    double cutoff, ewald_cutoff;
    const int32_t* framework_of;
} or_batch_view;
}

namespace {

// insertion_energy (src/energy.jl:42-82): one minimum image per host atom, each guest site's
// rotated offset added on top, LJ and screened Coulomb inside their cutoffs, plus the reciprocal
// cross term over the batch's k table. FP64 throughout. Returns the energy without the
// framework's constant offset. n_lj/n_ew count the pairs inside each cutoff (if non-null).
double insertion_energy(const or_batch_view& b, int fw, const double* pos, const double* q,
                        int64_t* n_lj, int64_t* n_ew) {
    const int N = b.nguest, nt = b.ntypes;
    double gs[3 * 16];
    for (int s = 0; s < N; ++s) rotate_strict<double>(q, b.guest_sites + 3 * s, gs + 3 * s);
    const double* A = b.cells + 9 * fw; const double* invA = b.invcells + 9 * fw;
    const double rl2 = b.cutoff * b.cutoff, re2 = b.ewald_cutoff * b.ewald_cutoff, alpha = b.alphas[fw];
    double Elj = 0, Esr = 0; int64_t cl = 0, ce = 0;
    for (int32_t j = b.atom_offsets[fw]; j < b.atom_offsets[fw + 1]; ++j) {
        double D0[3] = {pos[0] - b.positions[3 * j], pos[1] - b.positions[3 * j + 1], pos[2] - b.positions[3 * j + 2]};
        minimum_image_strict<double>(A, invA, D0);
        int ht = b.types[j] - 1; double hq = b.charges[j];
        for (int s = 0; s < N; ++s) {
            double D[3] = {D0[0] + gs[3 * s], D0[1] + gs[3 * s + 1], D0[2] + gs[3 * s + 2]};
            double r2 = D[0] * D[0] + D[1] * D[1] + D[2] * D[2];
            if (!(r2 < rl2 || r2 < re2)) continue;
            int gt = b.guest_types[s] - 1;
            if (r2 < rl2) { Elj += lj_pair(r2, b.sigma[gt + nt * ht], b.epsilon[gt + nt * ht]); ++cl; }
            if (r2 < re2) { double r = std::sqrt(r2); Esr += b.guest_charges[s] * hq * std::erfc(alpha * r) / r; ++ce; }
        }
    }
    double Elr = 0;
    for (int32_t i = b.k_offsets[fw]; i < b.k_offsets[fw + 1]; ++i) {
        const double* k = b.ks + 3 * i;
        double re = 0, im = 0;
        for (int s = 0; s < N; ++s) {
            double ph = k[0] * (pos[0] + gs[3 * s]) + k[1] * (pos[1] + gs[3 * s + 1]) + k[2] * (pos[2] + gs[3 * s + 2]);
            re += b.guest_charges[s] * std::cos(ph); im += b.guest_charges[s] * std::sin(ph);
        }
        // 2 Re(conj(S) Sg)
        Elr += b.kprefactor[i] * 2 * (b.Shost[2 * i] * re + b.Shost[2 * i + 1] * im);
    }
    if (n_lj) *n_lj = cl;
    if (n_ew) *n_ew = ce;
    return Elj + KE * (Esr + Elr);
}

// Phase-0 flag of one pose (src/widom.jl:99-151), in type F with the strict operation sequence.
template <typename F>
bool hardcore_flag(const or_batch_view& b, int s, const F* A, const F* invA, const F* posF, const F* rho2F,
                   const int32_t* reach0, const F* gsites_body, const F* quat, const F* atomsF) {
    const int N = b.nguest, nt = b.ntypes;
    int fw = b.framework_of[s] - 1;
    int32_t a0 = b.atom_offsets[fw];
    const int32_t* coff = b.cell_offsets + b.cellgrid_offsets[fw];
    int32_t n1 = b.ncells[3 * fw], n2 = b.ncells[3 * fw + 1], n3 = b.ncells[3 * fw + 2];
    int32_t m1 = reach0[3 * s], m2 = reach0[3 * s + 1], m3 = reach0[3 * s + 2];
    F pos[3]; matvec(A, posF, pos);
    int64_t base = int64_t(s) * N * nt;
    for (int a = 0; a < N; ++a) {
        F g[3]; rotate_strict(quat, gsites_body + 3 * a, g);
        F sp[3] = {pos[0] + g[0], pos[1] + g[1], pos[2] + g[2]};
        F f[3]; matvec(invA, sp, f);
        int32_t h1 = home_cell_dev(wrap_frac(f[0]), n1), h2 = home_cell_dev(wrap_frac(f[1]), n2), h3 = home_cell_dev(wrap_frac(f[2]), n3);
        int32_t st1, c1, st2, c2, st3, c3;
        stencil_start_count(h1, m1, n1, &st1, &c1);
        stencil_start_count(h2, m2, n2, &st2, &c2);
        stencil_start_count(h3, m3, n3, &st3, &c3);
        for (int32_t t3 = 0; t3 < c3; ++t3) {
            int32_t z = wrap_cell(st3 + t3, n3);
            for (int32_t t2 = 0; t2 < c2; ++t2) {
                int32_t y = wrap_cell(st2 + t2, n2);
                for (int32_t t1 = 0; t1 < c1; ++t1) {
                    int32_t x = wrap_cell(st1 + t1, n1);
                    int32_t c = x + n1 * (y + n2 * z);
                    for (int32_t j = a0 + coff[c]; j < a0 + coff[c + 1]; ++j) {
                        F D[3] = {sp[0] - atomsF[3 * j], sp[1] - atomsF[3 * j + 1], sp[2] - atomsF[3 * j + 2]};
                        minimum_image_strict(A, invA, D);
                        F r2 = dot3(D[0], D[1], D[2], D[0], D[1], D[2]);
                        if (r2 < rho2F[base + int64_t(a) * nt + (b.types[j] - 1)]) return true;
                    }
                }
            }
        }
    }
    return false;
}

inline int32_t sys_of_index(int64_t g, int64_t run, int64_t nsys) { return int32_t(((g - 1) / run) % nsys) + 1; }

std::vector<int64_t> system_counts(int64_t ninsert, int64_t nsys, int64_t run) {
    int64_t q = ninsert / run, rem = ninsert % run, full = q / nsys, hi = q % nsys;
    std::vector<int64_t> ns(nsys, full * run);
    for (int64_t r = 0; r < hi; ++r) ns[r] += run;
    if (rem > 0) ns[q % nsys] += rem;
    return ns;
}

template <typename F>
int widom_impl(const or_batch_view& b, double kT, int64_t ninsert, uint64_t seed, int32_t nblocks, int64_t run,
               int32_t reject, const double* rho2, const int32_t* reach0, double* sW, double* sUW, int64_t* nout,
               double* dU_out, uint8_t* flags_out, double* poses_out, int64_t* pairs_out) {
    const int N = b.nguest, nsys = b.nsys, nt = b.ntypes;
    std::vector<int64_t> ns = system_counts(ninsert, nsys, run);
    std::vector<int64_t> off(nsys + 1, 0);
    for (int s = 0; s < nsys; ++s) off[s + 1] = off[s] + ns[s];
    // type-F copies of the geometry the phase-0 path reads
    int64_t natot = b.atom_offsets[b.nfw];
    std::vector<F> atomsF(3 * natot), cellsF(9 * b.nfw), invF(9 * b.nfw), gsF(3 * N);
    for (int64_t i = 0; i < 3 * natot; ++i) atomsF[i] = F(b.positions[i]);
    for (int i = 0; i < 9 * b.nfw; ++i) { cellsF[i] = F(b.cells[i]); invF[i] = F(b.invcells[i]); }
    for (int i = 0; i < 3 * N; ++i) gsF[i] = F(b.guest_sites[i]);
    std::vector<F> rho2F(reject ? int64_t(nsys) * N * nt : 0);
    for (size_t i = 0; i < rho2F.size(); ++i) rho2F[i] = F(rho2[i]);
    std::vector<double> dU(ninsert);
    std::vector<uint8_t> flg(ninsert, 0);
    int64_t pl = 0, pe = 0;
#pragma omp parallel for schedule(dynamic, 256) reduction(+ : pl, pe)
    for (int64_t i = 0; i < ninsert; ++i) {
        int s = int(std::upper_bound(off.begin(), off.end(), i) - off.begin()) - 1;
        int64_t k = i - off[s] + 1;
        int fw = b.framework_of[s] - 1;
        F rp[3], qt[4];
        pose<F>(seed, uint64_t(s + 1), uint64_t(k), rp, qt);
        if (poses_out) {
            for (int r = 0; r < 3; ++r) poses_out[7 * i + r] = double(rp[r]);
            for (int r = 0; r < 4; ++r) poses_out[7 * i + 3 + r] = double(qt[r]);
        }
        bool rej = reject && hardcore_flag<F>(b, s, cellsF.data() + 9 * fw, invF.data() + 9 * fw, rp, rho2F.data(),
                                              reach0, gsF.data(), qt, atomsF.data());
        flg[i] = rej ? 1 : 0;
        if (rej) { dU[i] = INFINITY; continue; }
        double rpd[3] = {double(rp[0]), double(rp[1]), double(rp[2])}, qd[4] = {double(qt[0]), double(qt[1]), double(qt[2]), double(qt[3])};
        double pos[3]; matvec(b.cells + 9 * fw, rpd, pos);
        int64_t cl = 0, ce = 0;
        dU[i] = insertion_energy(b, fw, pos, qd, &cl, &ce) + b.constant_offset[fw];
        pl += cl; pe += ce;
    }
    if (pairs_out) { pairs_out[0] = pl; pairs_out[1] = pe; }
    // accumulation in each system's own sample order (src/widom.jl:430-438, 80-84)
    for (int s = 0; s < nsys; ++s) {
        int64_t blen = ns[s] / nblocks;
        for (int bb = 0; bb < nblocks; ++bb) { sW[s * nblocks + bb] = 0; sUW[s * nblocks + bb] = 0; nout[s * nblocks + bb] = 0; }
        for (int64_t k = 1; k <= ns[s]; ++k) {
            int64_t i = off[s] + k - 1;
            int64_t blk = std::min<int64_t>(nblocks, (k - 1) / blen + 1) - 1;
            double w = 0, uw = 0;
            if (!flg[i]) { w = std::exp(-dU[i] / kT); uw = (w == 0) ? 0.0 : dU[i] * w; }
            sW[s * nblocks + blk] += w; sUW[s * nblocks + blk] += uw; nout[s * nblocks + blk] += 1;
        }
    }
    if (dU_out) std::memcpy(dU_out, dU.data(), ninsert * sizeof(double));
    if (flags_out) std::memcpy(flags_out, flg.data(), ninsert);
    return 0;
}

}  // namespace

extern "C" {

int64_t or_system_counts(int64_t ninsert, int64_t nsys, int64_t run, int64_t* out) {
    auto v = system_counts(ninsert, nsys, run);
    for (int64_t s = 0; s < nsys; ++s) out[s] = v[s];
    return nsys;
}
int32_t or_sys_of_index(int64_t g, int64_t run, int64_t nsys) { return sys_of_index(g, run, nsys); }

// Runs the whole widom path. precision 32 draws FP32 poses and runs the phase-0 scan in strict
// FP32 (the FP32 device path's sequence); energies are FP64 at those poses either way. Outputs:
// sW/sUW/n are nsys x nblocks (row-major); dU_out/flags_out/poses_out (optional) are per
// insertion in system-major, per-system sample order. pairs_out (optional) gets the summed
// LJ/Ewald in-cutoff pair counts of the survivors.
int or_widom(const or_batch_view* b, int32_t precision, double kT, int64_t ninsert, uint64_t seed, int32_t nblocks,
             int64_t run, int32_t reject, const double* rho2, const int32_t* reach0, double* sW, double* sUW, int64_t* n,
             double* dU_out, uint8_t* flags_out, double* poses_out, int64_t* pairs_out, int32_t nthreads) {
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
    if (b->nguest > 16) return 1;
    if (precision == 32)
        return widom_impl<float>(*b, kT, ninsert, seed, nblocks, run, reject, rho2, reach0, sW, sUW, n, dU_out, flags_out, poses_out, pairs_out);
    return widom_impl<double>(*b, kT, ninsert, seed, nblocks, run, reject, rho2, reach0, sW, sUW, n, dU_out, flags_out, poses_out, pairs_out);
}

// insertion_energy for explicit poses (pos Cartesian, quat xyzw), without the constant offset.
void or_insertion_energy(const or_batch_view* b, int32_t fw, int64_t n, const double* pos, const double* quat, double* out) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) out[i] = insertion_energy(*b, fw, pos + 3 * i, quat + 4 * i, nullptr, nullptr);
}

// widom_chain_kernel!'s energy (src/nvt.jl:85-124) of explicit poses of one system, without its
// constant term: insertion_energy against the view's k table and structure factor (the caller's
// view carries the system's running S(k), host plus guests, in place of Shost), plus the
// guest-guest real space over the system's live guests (src/guest.jl:51-75: every site pair its
// own minimum image, LJ inside the LJ cutoff, q_a q_b erfc(alpha r)/r inside the Ewald cutoff).
// gsites: 3*N per live guest, guest-major, Cartesian.
void or_chain_energy(const or_batch_view* bp, int32_t fw, int64_t n, const double* pos, const double* quat, int64_t ng,
                     const double* gsites, double* out) {
    const or_batch_view& b = *bp;
    const int N = b.nguest, nt = b.ntypes;
    const double* A = b.cells + 9 * fw; const double* invA = b.invcells + 9 * fw;
    const double rl2 = b.cutoff * b.cutoff, re2 = b.ewald_cutoff * b.ewald_cutoff, alpha = b.alphas[fw];
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        const double* p = pos + 3 * i; const double* q = quat + 4 * i;
        double e = insertion_energy(b, fw, p, q, nullptr, nullptr);
        double gs[3 * 16];
        for (int a = 0; a < N; ++a) rotate_strict<double>(q, b.guest_sites + 3 * a, gs + 3 * a);
        double Elj = 0, Esr = 0;
        for (int64_t j = 0; j < ng; ++j)
            for (int a = 0; a < N; ++a)
                for (int c = 0; c < N; ++c) {
                    const double* o = gsites + 3 * (j * N + c);
                    double D[3] = {p[0] + gs[3 * a] - o[0], p[1] + gs[3 * a + 1] - o[1], p[2] + gs[3 * a + 2] - o[2]};
                    minimum_image_strict<double>(A, invA, D);
                    const double r2 = D[0] * D[0] + D[1] * D[1] + D[2] * D[2];
                    if (!(r2 < rl2 || r2 < re2)) continue;
                    const int ta = b.guest_types[a] - 1, tc = b.guest_types[c] - 1;
                    if (r2 < rl2) Elj += lj_pair(r2, b.sigma[ta + nt * tc], b.epsilon[ta + nt * tc]);
                    if (r2 < re2) { const double r = std::sqrt(r2); Esr += b.guest_charges[a] * b.guest_charges[c] * std::erfc(alpha * r) / r; }
                }
        out[i] = e + Elj + KE * Esr;
    }
}

// insertion_energy_reference (src/reference.jl:31-67): per-site minimum image, erfc, and the full
// k set with both the cross and the guest self term. hpos/htype(1-based)/hq are the host atoms.
double or_insertion_energy_reference(const double* pos, const double* q, int32_t N, const double* gsites,
                                     const int32_t* gtypes, const double* gq, int32_t nt, const double* sigma,
                                     const double* epsilon, double cutoff, double ewald_cutoff, int64_t na,
                                     const double* hpos, const int32_t* htype, const double* hq, const double* A,
                                     double alpha, int64_t nk, const double* ks, const double* kpref, const double* Sh) {
    double invA[9]; inv3(A, invA);
    std::vector<double> gp(3 * N);
    for (int s = 0; s < N; ++s) {
        double g[3]; rotate_strict<double>(q, gsites + 3 * s, g);
        for (int r = 0; r < 3; ++r) gp[3 * s + r] = pos[r] + g[r];
    }
    double rl2 = cutoff * cutoff, re2 = ewald_cutoff * ewald_cutoff, Elj = 0, Esr = 0;
    for (int s = 0; s < N; ++s)
        for (int64_t j = 0; j < na; ++j) {
            double D[3] = {gp[3 * s] - hpos[3 * j], gp[3 * s + 1] - hpos[3 * j + 1], gp[3 * s + 2] - hpos[3 * j + 2]};
            minimum_image_strict<double>(A, invA, D);
            double r2 = D[0] * D[0] + D[1] * D[1] + D[2] * D[2];
            int gt = gtypes[s] - 1, ht = htype[j] - 1;
            if (r2 < rl2) Elj += lj_pair(r2, sigma[gt + nt * ht], epsilon[gt + nt * ht]);
            if (r2 < re2) { double r = std::sqrt(r2); Esr += gq[s] * hq[j] * std::erfc(alpha * r) / r; }
        }
    double Elr = 0;
    for (int64_t i = 0; i < nk; ++i) {
        double re = 0, im = 0;
        for (int s = 0; s < N; ++s) {
            double ph = ks[3 * i] * gp[3 * s] + ks[3 * i + 1] * gp[3 * s + 1] + ks[3 * i + 2] * gp[3 * s + 2];
            re += gq[s] * std::cos(ph); im += gq[s] * std::sin(ph);
        }
        Elr += kpref[i] * (2 * (Sh[2 * i] * re + Sh[2 * i + 1] * im) + re * re + im * im);
    }
    return Elj + KE * (Esr + Elr);
}

// Phase-0 flags for explicit poses (fractional position, quaternion) of system s (0-based), in
// F32 (precision 32) or F64 strict arithmetic: stencil scan (brute = 0) or every atom (brute = 1).
void or_hardcore_flags(const or_batch_view* b, int32_t precision, int32_t s, int64_t n, const double* rpos,
                       const double* quat, const double* rho2, const int32_t* reach0, int32_t brute, uint8_t* out) {
    const int N = b->nguest, nt = b->ntypes;
    int fw = b->framework_of[s] - 1;
    auto run = [&](auto tag) {
        using F = decltype(tag);
        int64_t natot = b->atom_offsets[b->nfw];
        std::vector<F> atomsF(3 * natot), A(9), iA(9), gs(3 * N), r2t(int64_t(b->nsys) * N * nt);
        for (int64_t i = 0; i < 3 * natot; ++i) atomsF[i] = F(b->positions[i]);
        for (int i = 0; i < 9; ++i) { A[i] = F(b->cells[9 * fw + i]); iA[i] = F(b->invcells[9 * fw + i]); }
        for (int i = 0; i < 3 * N; ++i) gs[i] = F(b->guest_sites[i]);
        for (size_t i = 0; i < r2t.size(); ++i) r2t[i] = F(rho2[i]);
        for (int64_t i = 0; i < n; ++i) {
            F rp[3] = {F(rpos[3 * i]), F(rpos[3 * i + 1]), F(rpos[3 * i + 2])};
            F qt[4] = {F(quat[4 * i]), F(quat[4 * i + 1]), F(quat[4 * i + 2]), F(quat[4 * i + 3])};
            if (!brute) { out[i] = hardcore_flag<F>(*b, s, A.data(), iA.data(), rp, r2t.data(), reach0, gs.data(), qt, atomsF.data()); continue; }
            F pos[3]; matvec(A.data(), rp, pos);
            bool hit = false;
            for (int a = 0; a < N && !hit; ++a) {
                F g[3]; rotate_strict(qt, gs.data() + 3 * a, g);
                F sp[3] = {pos[0] + g[0], pos[1] + g[1], pos[2] + g[2]};
                for (int32_t j = b->atom_offsets[fw]; j < b->atom_offsets[fw + 1]; ++j) {
                    F D[3] = {sp[0] - atomsF[3 * j], sp[1] - atomsF[3 * j + 1], sp[2] - atomsF[3 * j + 2]};
                    minimum_image_strict(A.data(), iA.data(), D);
                    F r2 = dot3(D[0], D[1], D[2], D[0], D[1], D[2]);
                    if (r2 < r2t[int64_t(s) * N * nt + int64_t(a) * nt + (b->types[j] - 1)]) { hit = true; break; }
                }
            }
            out[i] = hit;
        }
    };
    if (precision == 32) run(float(0)); else run(double(0));
}

// build_rejection_tables (src/widom.jl:202-253): rho2 (nsys*N*ntypes) and reach0 (3*nsys).
// eps_F is eps of the kernel's float type. Returns 0, or s+1 for a system with margin <= 0.
int32_t or_rejection_tables(const or_batch_view* b, const double* bs, const double* kmin, double kT, double eps_F,
                            double* rho2, int32_t* reach0) {
    const int N = b->nguest, nt = b->ntypes;
    double theta = theta_F<double>();
    for (int s = 0; s < b->nsys; ++s) {
        int fw = b->framework_of[s] - 1;
        double Bs = bs[fw], cs = b->constant_offset[fw];
        int64_t natoms = b->atom_offsets[fw + 1] - b->atom_offsets[fw], nk = b->k_offsets[fw + 1] - b->k_offsets[fw];
        double n = double(N * natoms + nk + 8);
        double safety = 2 * n * eps_F * (Bs + std::fabs(cs)) + 4.0e-6 * Bs;
        double margin = std::isinf(Bs) ? INFINITY : (theta + 2) * kT + safety + Bs - cs;
        if (!(margin > 0)) return s + 1;
        double rmax = 0;
        for (int a = 0; a < N; ++a)
            for (int t = 0; t < nt; ++t) {
                int gt = b->guest_types[a] - 1;
                int err;
                double r2 = find_rho2(b->sigma[gt + nt * t], b->epsilon[gt + nt * t], kmin[int64_t(fw) * N * nt + a * nt + t], margin, b->cutoff, &err);
                if (err) return -(s + 1);
                rho2[int64_t(s) * N * nt + a * nt + t] = r2;
                rmax = std::max(rmax, r2);
            }
        double L[3]; perpendicular_lengths(b->cells + 9 * fw, L);
        for (int r = 0; r < 3; ++r) reach0[3 * s + r] = stencil_reach(L[r], b->ncells[3 * fw + r], std::sqrt(rmax));
    }
    return 0;
}

}  // extern "C"

// ---------------------------------------------------------------------------------------------
// Adjoint sums. PureAdsorb.jl has no gradients; this is the derivative of its insertion_energy
// (src/energy.jl:42-82) with respect to the pair tables and the stored charges, weighted by the
// Boltzmann factors of one widom call (the reweighting identity
// d ln <W> / dθ = -<W ∂ΔU/∂θ> / (kT <W>)), in FP64 over every survivor.
// ---------------------------------------------------------------------------------------------
namespace {

void grad_insertion(const or_batch_view& b, int fw, const double* pos, const double* q, double w, double* d_eps,
                    double* d_sig, double* d_q, double* sg) {
    const int N = b.nguest, nt = b.ntypes;
    double gs[3 * 16];
    for (int s = 0; s < N; ++s) rotate_strict<double>(q, b.guest_sites + 3 * s, gs + 3 * s);
    const double* A = b.cells + 9 * fw; const double* invA = b.invcells + 9 * fw;
    const double rl2 = b.cutoff * b.cutoff, re2 = b.ewald_cutoff * b.ewald_cutoff, alpha = b.alphas[fw];
    const int32_t a0 = b.atom_offsets[fw];
    for (int32_t j = a0; j < b.atom_offsets[fw + 1]; ++j) {
        double D0[3] = {pos[0] - b.positions[3 * j], pos[1] - b.positions[3 * j + 1], pos[2] - b.positions[3 * j + 2]};
        minimum_image_strict<double>(A, invA, D0);
        const int ht = b.types[j] - 1;
        for (int s = 0; s < N; ++s) {
            double D[3] = {D0[0] + gs[3 * s], D0[1] + gs[3 * s + 1], D0[2] + gs[3 * s + 2]};
            double r2 = D[0] * D[0] + D[1] * D[1] + D[2] * D[2];
            const int gt = b.guest_types[s] - 1;
            if (r2 < rl2) {
                const double sig = b.sigma[gt + nt * ht], eps = b.epsilon[gt + nt * ht];
                double x = sig * sig / r2; x = x * x * x;
                d_eps[s * nt + ht] += w * 4 * x * (x - 1);
                if (sig > 0) d_sig[s * nt + ht] += w * 24 * eps / sig * x * (2 * x - 1);
            }
            if (r2 < re2) {
                const double r = std::sqrt(r2);
                d_q[j - a0] += w * KE * b.guest_charges[s] * std::erfc(alpha * r) / r;
            }
        }
    }
    const int32_t k0 = b.k_offsets[fw];
    for (int32_t i = k0; i < b.k_offsets[fw + 1]; ++i) {
        const double* k = b.ks + 3 * i;
        double re = 0, im = 0;
        for (int s = 0; s < N; ++s) {
            double ph = k[0] * (pos[0] + gs[3 * s]) + k[1] * (pos[1] + gs[3 * s + 1]) + k[2] * (pos[2] + gs[3 * s + 2]);
            re += b.guest_charges[s] * std::cos(ph); im += b.guest_charges[s] * std::sin(ph);
        }
        sg[2 * (i - k0)] += w * re;
        sg[2 * (i - k0) + 1] += w * im;
    }
}

}  // namespace

extern "C" {

// Adjoint sums of one or_widom call, from its per-insertion outputs (system-major order; poses
// as fractional position + quaternion). Per system s: xmax = max over survivors of x = -ΔU/kT,
// sum_w = Σ w, w = exp(x - xmax); d_eps/d_sig [s][a][t] = Σ w ∂ΔU/∂(pair table entry of site a's
// type and host type t); d_charge (system-major, natoms of the system's framework) = Σ w ∂ΔU/∂q_j,
// real-space and reciprocal parts; s_guest (optional, 2 per k-vector) = Σ w S_g(k).
int or_grad_sums(const or_batch_view* bp, double kT, int64_t ninsert, int64_t run, const double* poses,
                 const double* dU, const uint8_t* flags, double* xmax, double* sum_w, double* d_eps, double* d_sig,
                 double* d_charge, double* s_guest, int32_t nthreads) {
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
    const or_batch_view& b = *bp;
    const int N = b.nguest, nt = b.ntypes, nsys = b.nsys;
    if (N > 16) return 1;
    std::vector<int64_t> ns = system_counts(ninsert, nsys, run);
    std::vector<int64_t> off(nsys + 1, 0);
    for (int s = 0; s < nsys; ++s) off[s + 1] = off[s] + ns[s];
    int64_t aoff = 0, koff = 0;
    for (int s = 0; s < nsys; ++s) {
        const int fw = b.framework_of[s] - 1;
        const int32_t na = b.atom_offsets[fw + 1] - b.atom_offsets[fw], nk = b.k_offsets[fw + 1] - b.k_offsets[fw];
        double m = -INFINITY;
        for (int64_t i = off[s]; i < off[s + 1]; ++i)
            if (!flags[i]) m = std::max(m, -dU[i] / kT);
        xmax[s] = m;
        const size_t per = size_t(2 * N * nt + na + 2 * nk);
        int nth = 1;
#ifdef _OPENMP
        nth = omp_get_max_threads();
#endif
        std::vector<double> buf(per * nth, 0.0), wsum(nth, 0.0);
#pragma omp parallel
        {
            int th = 0;
#ifdef _OPENMP
            th = omp_get_thread_num();
#endif
            double* my = buf.data() + per * th;
#pragma omp for schedule(static)
            for (int64_t i = off[s]; i < off[s + 1]; ++i) {
                if (flags[i] || m == -INFINITY) continue;
                const double w = std::exp(-dU[i] / kT - m);
                if (w == 0) continue;
                wsum[th] += w;
                const double* p = poses + 7 * i;
                double pos[3];
                matvec(b.cells + 9 * fw, p, pos);
                grad_insertion(b, fw, pos, p + 3, w, my, my + N * nt, my + 2 * N * nt, my + 2 * N * nt + na);
            }
        }
        double W = 0;
        std::vector<double> tot(per, 0.0);
        for (int t = 0; t < nth; ++t) {
            W += wsum[t];
            for (size_t x = 0; x < per; ++x) tot[x] += buf[per * t + x];
        }
        sum_w[s] = W;
        for (int x = 0; x < N * nt; ++x) {
            d_eps[int64_t(s) * N * nt + x] = tot[x];
            d_sig[int64_t(s) * N * nt + x] = tot[N * nt + x];
        }
        const double* G = tot.data() + 2 * N * nt + na;
        const int32_t a0 = b.atom_offsets[fw], k0 = b.k_offsets[fw];
#pragma omp parallel for schedule(static)
        for (int32_t j = 0; j < na; ++j) {
            const double* r = b.positions + 3 * (a0 + j);
            double acc = 0;
            for (int32_t i = 0; i < nk; ++i) {
                const double* k = b.ks + 3 * (k0 + i);
                const double ph = k[0] * r[0] + k[1] * r[1] + k[2] * r[2];
                acc += 2 * b.kprefactor[k0 + i] * (std::cos(ph) * G[2 * i] + std::sin(ph) * G[2 * i + 1]);
            }
            d_charge[aoff + j] = tot[2 * N * nt + j] + KE * acc;
        }
        if (s_guest)
            for (int32_t i = 0; i < 2 * nk; ++i) s_guest[2 * koff + i] = G[i];
        aoff += na;
        koff += nk;
    }
    return 0;
}

}  // extern "C"
