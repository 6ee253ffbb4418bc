// Shared host/device building blocks of the Widom path: strict (individually rounded)
// arithmetic, the counter-based pose stream and the strict geometry used by pose generation and
// the phase-0 hard-core scan. Everything here compiles for both the host and sm_100a so the
// host-side pose function (pa_pose_host) and the kernels produce identical bits.
#pragma once
#include <cstdint>
#include <cmath>
#include "pa_coeffs.h"

#if defined(__CUDACC__)
#define PA_HD __host__ __device__ __forceinline__
#else
#define PA_HD inline
#endif

namespace pa {

constexpr double KB = 1.38064852e-23 / 1.6021766208e-19;  // eV/K     (src/constants.jl:3)
constexpr double KE = 14.399645351950548;                  // eV*A/e^2 (src/constants.jl:4)

// ---------------------------------------------------------------------------------------------
// Strict arithmetic: each operation is rounded once; device code uses the _rn intrinsics, which
// the compiler never contracts into fused multiply-adds, and host code is compiled with
// -ffp-contract=off. fma is always an explicit single-rounding fused multiply-add.
// ---------------------------------------------------------------------------------------------
template <typename F> struct St;
template <> struct St<float> {
    static PA_HD float mul(float a, float b) {
#ifdef __CUDA_ARCH__
        return __fmul_rn(a, b);
#else
        return a * b;
#endif
    }
    static PA_HD float add(float a, float b) {
#ifdef __CUDA_ARCH__
        return __fadd_rn(a, b);
#else
        return a + b;
#endif
    }
    static PA_HD float sub(float a, float b) {
#ifdef __CUDA_ARCH__
        return __fsub_rn(a, b);
#else
        return a - b;
#endif
    }
    static PA_HD float fma(float a, float b, float c) {
#ifdef __CUDA_ARCH__
        return __fmaf_rn(a, b, c);
#else
        return std::fmaf(a, b, c);
#endif
    }
    static PA_HD float sqrt(float a) {
#ifdef __CUDA_ARCH__
        return __fsqrt_rn(a);
#else
        return std::sqrt(a);
#endif
    }
    static PA_HD float rint(float a) {
#ifdef __CUDA_ARCH__
        return rintf(a);
#else
        return std::nearbyint(a);
#endif
    }
    static PA_HD float floor(float a) {
#ifdef __CUDA_ARCH__
        return floorf(a);
#else
        return std::floor(a);
#endif
    }
};
template <> struct St<double> {
    static PA_HD double mul(double a, double b) {
#ifdef __CUDA_ARCH__
        return __dmul_rn(a, b);
#else
        return a * b;
#endif
    }
    static PA_HD double add(double a, double b) {
#ifdef __CUDA_ARCH__
        return __dadd_rn(a, b);
#else
        return a + b;
#endif
    }
    static PA_HD double sub(double a, double b) {
#ifdef __CUDA_ARCH__
        return __dsub_rn(a, b);
#else
        return a - b;
#endif
    }
    static PA_HD double fma(double a, double b, double c) {
#ifdef __CUDA_ARCH__
        return __fma_rn(a, b, c);
#else
        return std::fma(a, b, c);
#endif
    }
    static PA_HD double div(double a, double b) {
#ifdef __CUDA_ARCH__
        return __ddiv_rn(a, b);
#else
        return a / b;
#endif
    }
    static PA_HD double sqrt(double a) {
#ifdef __CUDA_ARCH__
        return __dsqrt_rn(a);
#else
        return std::sqrt(a);
#endif
    }
    static PA_HD double rint(double a) {
#ifdef __CUDA_ARCH__
        return ::rint(a);
#else
        return std::nearbyint(a);
#endif
    }
    static PA_HD double floor(double a) {
#ifdef __CUDA_ARCH__
        return ::floor(a);
#else
        return std::floor(a);
#endif
    }
};

// ---------------------------------------------------------------------------------------------
// Counter-based stream (src/state.jl:225-230, src/rng.jl:43-81)
// ---------------------------------------------------------------------------------------------
PA_HD uint64_t splitmix64(uint64_t seed, uint64_t index) {
    uint64_t z = seed + index * 0x9E3779B97F4A7C15ULL;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}
// key of ChainRNG(chain_seed, cycle, move)
PA_HD uint64_t chain_key(uint64_t chain_seed, uint64_t cycle, uint64_t move) {
    return splitmix64(splitmix64(chain_seed, cycle), move);
}
template <typename F> PA_HD F unit_from_bits(uint64_t raw);
template <> PA_HD float unit_from_bits<float>(uint64_t raw) {
    // top 24 bits scaled by 2^-24: exact in FP32
    return St<float>::mul(float(uint32_t(raw >> 40)), 5.9604645e-8f);
}
template <> PA_HD double unit_from_bits<double>(uint64_t raw) {
    // top 53 bits scaled by 2^-53: exact in FP64
    return St<double>::mul(double(raw >> 11), 1.1102230246251565e-16);
}

// sin(2 pi u) and cos(2 pi u), u in [0, 1): y = 4u, q = rint(y), r = y - q (both exact), then
// Taylor polynomials of sin/cos((pi/2) r), |r| <= 1/2, in Horner form with fused multiply-adds,
// rotated by the quadrant q mod 4.
template <typename F> struct Trig;
template <> struct Trig<double> {
    static PA_HD void sincos2pi(double u, double* sn, double* cs) {
        typedef St<double> S;
        const double sc[PA_NSIN64] = PA_SIN64_INIT;
        const double cc[PA_NCOS64] = PA_COS64_INIT;
        double y = S::mul(u, 4.0), q = S::rint(y), r = S::sub(y, q), z = S::mul(r, r);
        double ps = sc[PA_NSIN64 - 1];
#pragma unroll
        for (int k = PA_NSIN64 - 2; k >= 0; --k) ps = S::fma(ps, z, sc[k]);
        double pc = cc[PA_NCOS64 - 1];
#pragma unroll
        for (int k = PA_NCOS64 - 2; k >= 0; --k) pc = S::fma(pc, z, cc[k]);
        double s = S::mul(r, ps), c = pc;
        int qi = int(q) & 3;
        *sn = qi == 0 ? s : qi == 1 ? c : qi == 2 ? -s : -c;
        *cs = qi == 0 ? c : qi == 1 ? -s : qi == 2 ? -c : s;
    }
};
// FP32: the FP64 evaluation rounded once to FP32, which is the correctly rounded sin/cos(2 pi u)
// for every FP32 uniform u = k 2^-24 (checked exhaustively over all 2^24 of them against an
// extended-precision reference), i.e. what Float32 sinpi(2u) / cospi(2u) return
// (src/rng.jl:126-129); zeros are returned as +0.
template <> struct Trig<float> {
    static PA_HD void sincos2pi(float u, float* sn, float* cs) {
        double s, c;
        Trig<double>::sincos2pi(double(u), &s, &c);
        *sn = St<float>::add(float(s), 0.0f);
        *cs = St<float>::add(float(c), 0.0f);
    }
};

// Pose of insertion k (1-based) of system s (1-based): words 0..5 of
// ChainRNG(splitmix64(seed, s), k, 0) give the fractional position (u_x, u_y, u_z) and Shoemake's
// (u1, u2, u3); quaternion (x, y, z, w) = (a cos 2pi u2, b sin 2pi u3, b cos 2pi u3, a sin 2pi u2)
// with a = sqrt(1-u1), b = sqrt(u1) (src/rng.jl:126-141, src/widom.jl:55-61).
template <typename F>
PA_HD void draw_pose(uint64_t seed, uint64_t s, uint64_t k, F rpos[3], F quat[4]) {
    typedef St<F> S;
    const uint64_t key = chain_key(splitmix64(seed, s), k, 0);
    F u[6];
#pragma unroll
    for (int d = 0; d < 6; ++d) u[d] = unit_from_bits<F>(splitmix64(key, uint64_t(d)));
    rpos[0] = u[0]; rpos[1] = u[1]; rpos[2] = u[2];
    F a = S::sqrt(S::sub(F(1), u[3])), b = S::sqrt(u[3]);
    F s2, c2, s3, c3;
    Trig<F>::sincos2pi(u[4], &s2, &c2);
    Trig<F>::sincos2pi(u[5], &s3, &c3);
    quat[0] = S::mul(a, c2); quat[1] = S::mul(b, s3); quat[2] = S::mul(b, c3); quat[3] = S::mul(a, s2);
}

// ---------------------------------------------------------------------------------------------
// Strict geometry (fixed operation order). Matrices are 3x3 column-major.
// ---------------------------------------------------------------------------------------------
template <typename F> PA_HD F dot3s(F a0, F a1, F a2, F b0, F b1, F b2) {
    typedef St<F> S;
    return S::fma(a2, b2, S::fma(a1, b1, S::mul(a0, b0)));
}
template <typename F> PA_HD void matvec_s(const F* M, const F* v, F* out) {
#pragma unroll
    for (int r = 0; r < 3; ++r) out[r] = dot3s(M[r], M[r + 3], M[r + 6], v[0], v[1], v[2]);
}
template <typename F> PA_HD F crossc_s(F a, F b, F c, F d) {
    typedef St<F> S;
    return S::fma(a, b, -S::mul(c, d));
}
// v + 2 u x (u x v + w v) with q = (u, w) (src/energy.jl:13-16)
template <typename F> PA_HD void rotate_s(const F* q, const F* v, F* out) {
    typedef St<F> S;
    F t0 = S::fma(q[3], v[0], crossc_s(q[1], v[2], q[2], v[1]));
    F t1 = S::fma(q[3], v[1], crossc_s(q[2], v[0], q[0], v[2]));
    F t2 = S::fma(q[3], v[2], crossc_s(q[0], v[1], q[1], v[0]));
    F c0 = crossc_s(q[1], t2, q[2], t1);
    F c1 = crossc_s(q[2], t0, q[0], t2);
    F c2 = crossc_s(q[0], t1, q[1], t0);
    out[0] = S::fma(F(2), c0, v[0]); out[1] = S::fma(F(2), c1, v[1]); out[2] = S::fma(F(2), c2, v[2]);
}
// D - A round(invA D), round half to even (src/cell.jl:34-37)
template <typename F> PA_HD void minimum_image_s(const F* A, const F* invA, F* D) {
    typedef St<F> S;
    F f[3];
    matvec_s(invA, D, f);
    F r0 = S::rint(f[0]), r1 = S::rint(f[1]), r2 = S::rint(f[2]);
#pragma unroll
    for (int r = 0; r < 3; ++r) D[r] = S::sub(D[r], dot3s(A[r], A[r + 3], A[r + 6], r0, r1, r2));
}
// 0-based home cell of a wrapped fractional coordinate (src/cell.jl:137-138)
template <typename F> PA_HD int32_t home_cell_s(F f, int32_t n) {
    typedef St<F> S;
    F x = S::mul(f, F(n));
    x = x > F(0) ? x : F(0);
    int32_t c = int32_t(x);
    return c < n - 1 ? c : n - 1;
}
template <typename F> PA_HD F wrap_frac_s(F f) { return St<F>::sub(f, St<F>::floor(f)); }
PA_HD int32_t wrap_cell(int32_t x, int32_t n) { return x + n * int32_t(x < 0) - n * int32_t(x >= n); }
PA_HD void stencil_start_count(int32_t h, int32_t m, int32_t n, int32_t* start, int32_t* count) {
    int32_t span = m + m + 1;
    *count = span < n ? span : n;
    *start = span >= n ? 0 : h - m;
}

}  // namespace pa
