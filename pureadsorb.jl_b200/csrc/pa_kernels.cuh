// Device kernels of the B200 Widom path.
//
// Pipeline of one widom call (pa_widom in pa_capi.cu):
//   k_pose      one thread per insertion: counter-based pose, phase-0 hard-core scan over the
//               cell list (strict arithmetic, bit-identical to the oracle), and for survivors a
//               spatial bin plus a slot in it (src/widom.jl:99-151, 399-415);
//   k_scan      one CTA: exclusive scans of the bin counts and of the per-bin tile counts;
//   k_scatter   survivors into bin-sorted order;
//   k_energy32  persistent CTAs of independent warps over (bin, 32-insertion tile) work items:
//               each warp streams its bin's imaged neighbour list into its own shared-memory
//               stages by bulk copies (cp.async.bulk + mbarrier, double buffered), one insertion
//               per lane, FP32 pair arithmetic with a compensated sum, reciprocal term against
//               FP64-built per-bin phase factors (src/energy.jl:42-82); in pa_energy32.cuh;
//   k_energy64  the plain FP64 form of the reference algorithm (linear loop over every atom,
//               one minimum image per atom), tiles per framework;
//   k_segsum    per PA_SEGMENT-insertion segment: max, then Σ exp(x - max) and Σ ΔU exp(x - max),
//               x = -ΔU/kT, with a fixed reduction tree (src/widom.jl:80-84, 430-438).
#pragma once
#include <cuda_runtime.h>
#include "pa_common.cuh"

#define PA_SEGMENT_SIZE 2048

namespace pa {

#define PA_NHP 8  // coefficients of the exp-free screened-Coulomb polynomial (degree 7)

template <typename F> struct Vec4;
template <> struct Vec4<float> { typedef float4 T; };
template <> struct Vec4<double> { typedef double4 T; };

// Device view of an uploaded batch. Index conventions are 0-based on the device.
template <typename F>
struct DevBatch {
    int32_t nsys, nfw, ntypes, nguest, has_charge, nbins;
    int32_t nsub;                                 // sub-bins per bin for the survivor ordering
    F rl2, re2;                                   // LJ and Ewald cutoffs squared
    const int32_t* framework_of;                  // nsys
    const F* cells;                               // 9*nfw column-major
    const F* invcells;                            // 9*nfw
    const double* alphas;                         // nfw
    const double* const_offset;                   // nfw
    const int32_t* atom_offsets;                  // nfw+1
    const typename Vec4<F>::T* atoms;             // cell-sorted x, y, z, q
    const int32_t* types;                         // 0-based compact
    const int32_t* ncells;                        // 3*nfw
    const int32_t* cell_offsets;
    const int32_t* cellgrid_offsets;              // nfw+1
    const int32_t* k_offsets;                     // nfw+1
    const double* kvec;                           // 3*nk Cartesian (FP64 path)
    const float4* kcoef4;                         // nk: (n1, n2, n3, 1 if the k-vector continues its
                                                  //  row of equal (n1, n2) by kstep in n3, else 0)
    const float* kstep;                           // nfw: n3 step along a row
    const double* kS2;                            // 2*nk: 2*kpref*S_re, 2*kpref*S_im (FP64)
    const F* sig2;                                // nguest*ntypes: sigma^2 of (site, host type)
    const F* eps4;                                // nguest*ntypes: 4 eps
    F gsite[3 * PA_MAX_SITES_DEV];
    F gq[PA_MAX_SITES_DEV];
    // spatial bins (FP32 path: per-framework fractional grids; FP64 path: one bin per framework)
    const int32_t* bin_dims;                      // 3*nfw
    const int32_t* bin_base;                      // nfw+1
    const int32_t* bin_fw;                        // nbins
    const int32_t* list_offsets;                  // nbins+1, multiples of PA_LIST_PAD
    const float4* list_xyzq;                      // imaged position relative to the bin centre, charge
    const int32_t* list_type;                     // 0-based type (padding entries: type 0, far away)
    const int32_t* list_atom;                     // stored-atom index of each entry
    const int2* list_runs;                        // nbins*runs_per_bin: each bin's type runs (first entry,
                                                  // type), then (end of the list, 0) up to runs_per_bin
    int32_t runs_per_bin;
    // FP32 path, pairs evaluated in FP64: those closer than the near radius and those whose FP32
    // distance lies within a rounding band of a cutoff (the band's edges, rl2/re2 -+ band)
    const double4* list_xyzq64;                   // the list entries in FP64 (position, charge)
    const double* cells64;                        // 9*nfw
    const double* invcells64;                     // 9*nfw
    const double* sig2_64;                        // nguest*ntypes
    const double* eps4_64;                        // nguest*ntypes
    double gsite64[3 * PA_MAX_SITES_DEV];
    double gq64[PA_MAX_SITES_DEV];
    double rl2_64, re2_64;                        // the cutoffs squared, FP64
    F rn2;                                        // near radius squared (0: no near pairs)
    int32_t rmode;                                // reciprocal term: 0 FP32, 1 FP64, 2 split tables (k_recip)
    // the split tables of a charged FP32 batch: per framework the k-vectors of small |k| (FP64 rows)
    // and the rest (FP32 rows), each in enumeration order with its own row-continuation flags
    const float4* ks64_coef;
    const double* ks64_S2;                        // 2*kpref*S (re, im)
    const int32_t* ks64_off;                      // nfw+1
    const float4* ks32_coef;
    const double* ks32_S2;
    const int32_t* ks32_off;                      // nfw+1
    int32_t has_ksplit;
    F rl2_lo, rl2_hi, re2_lo, re2_hi;             // rounding bands around the cutoffs
    // FP32 screened Coulomb beyond the near radius in the exp-free form (hpoly != 0):
    // erfc(alpha r)/r = exp(-alpha^2 r^2) u H(u), u = 1/r^2, H a polynomial of PA_NHP coefficients
    // hc in x = hk1 u + hk0 (fitted per call on the host for the batch's alpha and [1/re^2, 1/rn^2])
    int32_t hpoly;
    float hk1, hk0;
    float hc[PA_NHP];
};

// Per-call arguments shared by the kernels.
struct CallArgs {
    int64_t i_lo, n_act;        // processed insertions: global indices [i_lo, i_lo + n_act)
    const int64_t* sys_off;     // nsys+1 insertion offsets (system-major)
    uint64_t seed;
    int32_t reject;
    double kT;
    // optional device copies of seed and kT: when set the kernels read these instead, so a
    // launch sequence captured in a CUDA graph replays for any seed and temperature
    const uint64_t* seed_dev;
    const double* kT_dev;
    // added to every insertion's per-system index k (the insertions of one cycle along a chain
    // follow the previous cycles'); koff_dev, when set, is read instead (graph replays)
    int64_t k_offset;
    const int64_t* koff_dev;
    // optional (F-typed, nsys*N): each (system, site)'s largest rejection radius squared, for
    // phase 0's relaxed pre-test; NULL: every atom of the stencil takes the strict test (the
    // FP32 warp kernel then runs the per-site stencil scan)
    const void* rho2max;
};

__device__ __forceinline__ int64_t k_shift(const CallArgs& ca) { return ca.koff_dev ? *ca.koff_dev : ca.k_offset; }

// Per-call device workspace.
struct Work {
    float4* pose_a;    // FP32 path: rpos.xyz; FP64 path uses pose64
    float4* pose_b;    // quaternion
    double4* pose64a;  // FP64 path rpos (xyz)
    double4* pose64b;  // FP64 path quaternion
    int32_t* bin_of;   // n_act: sub-bin of a survivor (bin * nsub + octant), -1 if rejected
    int32_t* slot;     // n_act
    int32_t* sorted;   // n_act: local insertion index in bin order
    double* dU;        // n_act: ΔU (+inf if rejected)
    int32_t* bin_count;   // nbins*nsub: survivors per sub-bin
    int32_t* fine_start;  // nbins*nsub+1
    int32_t* bin_start;   // nbins+1
    int32_t* tile_start;  // nbins+1
    int32_t* counters;    // [0] tile cursor, [1] total tiles, [2] error code, [3] survivors
    double* seg_out;      // 3 per segment: max, Σ w, Σ ΔU w
    const int64_t* seg_rng;  // 2 per segment: local [begin, end)
    // FP32 path: one work item per (survivor, guest site), binned by the site's own position
    // (NULL item_bin: the FP64 path, whose items are the insertions themselves)
    int32_t* item_bin;    // n_act*NS: sub-bin of the item's site, -1 if the insertion was rejected
    int32_t* item_slot;   // n_act*NS
    int32_t* item_count;  // nbins*nsub+1: items per sub-bin
    double* dUs;          // n_act*NS: real-space energy of each item's site
    double* dUr;          // n_act: KE times the reciprocal cross term
    double* dUg;          // n_act: guest-guest real-space term (insertion along a chain), else NULL
    // with the adjoint: per sorted item and type run of its bin's list, the LJ sums (Σ x(x-1),
    // Σ x(2x-1)), x = (sigma/r)^6, over the item's pairs inside the LJ cutoff (else NULL)
    float2* item_pq;
};

// ---------------------------------------------------------------------------------------------
// Small helpers
// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ int32_t find_system(const int64_t* sys_off, int32_t nsys, int64_t i) {
    int32_t lo = 0, hi = nsys;  // sys_off[lo] <= i < sys_off[hi]
    while (hi - lo > 1) {
        int32_t mid = (lo + hi) >> 1;
        if (sys_off[mid] <= i) lo = mid; else hi = mid;
    }
    return lo;
}
__device__ __forceinline__ int32_t find_bin(const int32_t* start, int32_t n, int32_t t) {
    int32_t lo = 0, hi = n;  // largest b with start[b] <= t
    while (hi - lo > 1) {
        int32_t mid = (lo + hi) >> 1;
        if (start[mid] <= t) lo = mid; else hi = mid;
    }
    return lo;
}
__device__ __forceinline__ void kahan_add(float& sum, float& c, float x) {
    float y = __fsub_rn(x, c);
    float t = __fadd_rn(sum, y);
    c = __fsub_rn(__fsub_rn(t, sum), y);
    sum = t;
}

// Phase 0 for one pose: any guest site closer than sqrt(rho2[s, a, type]) to a host atom, over
// the per-site cell stencil (src/widom.jl:99-151). Strict arithmetic (bit-identical to the
// oracle's hardcore_flag).
template <typename F, int NS>
__device__ bool hardcore_scan(const DevBatch<F>& b, int32_t s, int32_t fw, const F* rp, const F* qt,
                              const F* rho2, const int32_t* reach0, const F* rho2max) {
    typedef St<F> S;
    const F* A = b.cells + 9 * fw;
    const F* iA = b.invcells + 9 * fw;
    F Ael[9], iAel[9];
#pragma unroll
    for (int r = 0; r < 9; ++r) { Ael[r] = A[r]; iAel[r] = iA[r]; }
    const int32_t a0 = b.atom_offsets[fw];
    const int32_t* coff = b.cell_offsets + b.cellgrid_offsets[fw];
    const int32_t n1 = b.ncells[3 * fw], n2 = b.ncells[3 * fw + 1], n3 = b.ncells[3 * fw + 2];
    const int32_t m1 = reach0[3 * s], m2 = reach0[3 * s + 1], m3 = reach0[3 * s + 2];
    const int32_t nt = b.ntypes;
    F pos[3];
    matvec_s(Ael, rp, pos);
    const F* r2row = rho2 + int64_t(s) * NS * nt;
    // Relaxed pre-test. Inside the stencil every atom is visited at the image of its unwrapped
    // cell, i.e. at its stored position plus A w, w the row's wrap (-1, 0 or 1 per axis). With the
    // stencil narrower than the grid on every axis, that image lies within a few cells of the site,
    // so it is the strict minimum image whenever the atom is within reach (any other image is at
    // least half a cell width away). Its distance in plain FP32/FP64 arithmetic differs from the
    // strict one by rounding only, far below the 1e-3 A^2 margin, so an atom at least the site's
    // largest radius squared plus the margin away cannot set the flag and skips the strict test.
    const bool pre = rho2max != nullptr && 2 * m1 + 1 < n1 && 2 * m2 + 1 < n2 && 2 * m3 + 1 < n3;
#pragma unroll 1
    for (int a = 0; a < NS; ++a) {
        F g[3];
        rotate_s(qt, b.gsite + 3 * a, g);
        F sp[3] = {S::add(pos[0], g[0]), S::add(pos[1], g[1]), S::add(pos[2], g[2])};
        F f[3];
        matvec_s(iAel, sp, f);
        int32_t h1 = home_cell_s(wrap_frac_s(f[0]), n1);
        int32_t h2 = home_cell_s(wrap_frac_s(f[1]), n2);
        int32_t h3 = home_cell_s(wrap_frac_s(f[2]), n3);
        int32_t st1, c1, st2, c2, st3, c3;
        stencil_start_count(h1, m1, n1, &st1, &c1);
        stencil_start_count(h2, m2, n2, &st2, &c2);
        stencil_start_count(h3, m3, n3, &st3, &c3);
        const F* r2a = r2row + a * nt;
        const F lim = pre ? rho2max[int64_t(s) * NS + a] + F(1e-3) : F(0);
        // the site in its home cell's periodic frame, sp - A floor(f)
        const F fl0 = floor(f[0]), fl1 = floor(f[1]), fl2 = floor(f[2]);
        const F bx = sp[0] - (Ael[0] * fl0 + Ael[3] * fl1 + Ael[6] * fl2);
        const F by = sp[1] - (Ael[1] * fl0 + Ael[4] * fl1 + Ael[7] * fl2);
        const F bz = sp[2] - (Ael[2] * fl0 + Ael[5] * fl1 + Ael[8] * fl2);
        // The x-cells of one (y, z) row of the stencil are consecutive in the cell-sorted atom
        // array, so each row is one contiguous atom range, or two where it wraps around the grid.
        // Atoms are visited in the same order as cell by cell (x innermost).
        const int32_t xa0 = st1 < 0 ? st1 + n1 : st1;
        const int32_t xa1 = st1 < 0 ? n1 : min(st1 + c1, n1);
        const int32_t xb1 = st1 < 0 ? st1 + c1 : max(st1 + c1 - n1, 0);
        for (int32_t t3 = 0; t3 < c3; ++t3) {
            const int32_t z = wrap_cell(st3 + t3, n3);
            const F wz = F((st3 + t3 < 0) ? -1 : (st3 + t3 >= n3 ? 1 : 0));
            for (int32_t t2 = 0; t2 < c2; ++t2) {
                const int32_t row = n1 * (wrap_cell(st2 + t2, n2) + n2 * z);
                const F wy = F((st2 + t2 < 0) ? -1 : (st2 + t2 >= n2 ? 1 : 0));
                // part A: cells [xa0, xa1); part B (wrapped, empty unless the stencil crosses the
                // grid's x boundary): cells [0, xb1)
                for (int part = 0; part < (xb1 > 0 ? 2 : 1); ++part) {
                    const int32_t j0 = a0 + coff[row + (part == 0 ? xa0 : 0)];
                    const int32_t j1 = a0 + coff[row + (part == 0 ? xa1 : xb1)];
                    const F wx = F(part == 0 ? (st1 < 0 ? -1 : 0) : (st1 < 0 ? 0 : 1));
                    // the site relative to this row part's atom images: b - A w
                    const F ex = bx - (Ael[0] * wx + Ael[3] * wy + Ael[6] * wz);
                    const F ey = by - (Ael[1] * wx + Ael[4] * wy + Ael[7] * wz);
                    const F ez = bz - (Ael[2] * wx + Ael[5] * wy + Ael[8] * wz);
                    for (int32_t j = j0; j < j1; ++j) {
                        typename Vec4<F>::T at = b.atoms[j];
                        if (pre) {
                            const F dx = ex - at.x, dy = ey - at.y, dz = ez - at.z;
                            if (dx * dx + dy * dy + dz * dz >= lim) continue;
                        }
                        F D[3] = {S::sub(sp[0], at.x), S::sub(sp[1], at.y), S::sub(sp[2], at.z)};
                        minimum_image_s(Ael, iAel, D);
                        F r2 = dot3s(D[0], D[1], D[2], D[0], D[1], D[2]);
                        if (r2 < r2a[b.types[j]]) return true;
                    }
                }
            }
        }
    }
    return false;
}

// Fractional position of a guest site: rp + A^-1 g (g the rotated body-frame offset), wrapped into
// [0, 1); wrap gets the lattice shift -floor(rp + A^-1 g). k_pose bins each site with it and
// k_energy32 places the site against its bin with the same shift, so both see the same image.
__device__ __forceinline__ void site_frac32(const float rp[3], const float g[3], const float* iA, float fs[3],
                                            float wrap[3]) {
#pragma unroll
    for (int r = 0; r < 3; ++r) {
        const float f = rp[r] + fmaf(iA[6 + r], g[2], fmaf(iA[3 + r], g[1], iA[r] * g[0]));
        wrap[r] = -floorf(f);
        float w = f + wrap[r];
        if (!(w < 1.0f)) {  // f just below an integer rounds up: it is the next image's 0
            w = 0.0f;
            wrap[r] -= 1.0f;
        }
        fs[r] = w;
    }
}

// Sub-bin (bin * nsub + octant) of a fractional position in [0, 1) of framework fw.
template <typename F>
__device__ __forceinline__ int32_t sub_bin_of(const DevBatch<F>& b, int32_t fw, float x, float y, float z) {
    const int32_t* nb = b.bin_dims + 3 * fw;
    const float fx = x * float(nb[0]), fy = y * float(nb[1]), fz = z * float(nb[2]);
    const int32_t bx = min(int32_t(fx), nb[0] - 1), by = min(int32_t(fy), nb[1] - 1), bz = min(int32_t(fz), nb[2] - 1);
    const int32_t bin = b.bin_base[fw] + bx + nb[0] * (by + nb[1] * bz);
    int32_t sub = 0;
    if (b.nsub == 8)
        sub = int32_t(fx - float(bx) >= 0.5f) | (int32_t(fy - float(by) >= 0.5f) << 1) | (int32_t(fz - float(bz) >= 0.5f) << 2);
    return bin * b.nsub + sub;
}

// ---------------------------------------------------------------------------------------------
// Outcome of phase 0 for insertion t: a rejected insertion gets bin -1 and ΔU = +inf; a survivor
// a slot in its centre's sub-bin and, on the FP32 path, one (insertion, site) item per guest site
// in the sub-bin of the site's own position.
// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ void mark_rejected(const Work& w, int64_t t, int ns) {
    w.bin_of[t] = -1;
    w.dU[t] = __longlong_as_double(0x7ff0000000000000LL);  // +inf
    if (w.item_bin)
        for (int a = 0; a < ns; ++a) w.item_bin[t * ns + a] = -1;
}

template <typename F, int NS>
__device__ __forceinline__ void bin_survivor(const DevBatch<F>& b, const Work& w, int64_t t, int32_t fw, const F* rp,
                                             const F* qt) {
    // spatial bin of the pose's reference point; with nsub = 8 the octant inside it orders the
    // survivors, so that a warp's 32 insertions lie in two adjacent octants
    const int32_t fine = sub_bin_of(b, fw, float(rp[0]), float(rp[1]), float(rp[2]));
    w.bin_of[t] = fine;
    w.slot[t] = atomicAdd(&w.bin_count[fine], 1);
    if constexpr (sizeof(F) == 4) {
        if (w.item_bin) {  // each site into the sub-bin of its own position
            const float* iAf = b.invcells + 9 * fw;
            const float q[4] = {float(qt[0]), float(qt[1]), float(qt[2]), float(qt[3])};
            const float rpf[3] = {float(rp[0]), float(rp[1]), float(rp[2])};
#pragma unroll
            for (int a = 0; a < NS; ++a) {
                const float gb[3] = {b.gsite[3 * a], b.gsite[3 * a + 1], b.gsite[3 * a + 2]};
                float g[3], fs[3], sh[3];
                rotate_s(q, gb, g);
                site_frac32(rpf, g, iAf, fs, sh);
                const int32_t sf = sub_bin_of(b, fw, fs[0], fs[1], fs[2]);
                w.item_bin[t * NS + a] = sf;
                w.item_slot[t * NS + a] = atomicAdd(&w.item_count[sf], 1);
            }
        }
    }
}

// ---------------------------------------------------------------------------------------------
// k_pose: pose, phase 0, bin slot (one thread per insertion, in insertion order)
// ---------------------------------------------------------------------------------------------
template <typename F, int NS>
__global__ void __launch_bounds__(256, 4) k_pose(DevBatch<F> b, CallArgs ca, Work w, const F* rho2, const int32_t* reach0) {
    const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= ca.n_act) return;
    const int64_t i = ca.i_lo + t;
    const int32_t s = find_system(ca.sys_off, b.nsys, i);
    const int64_t k = i - ca.sys_off[s] + 1;
    const int32_t fw = b.framework_of[s];
    F rp[3], qt[4];
    draw_pose<F>(ca.seed_dev ? *ca.seed_dev : ca.seed, uint64_t(s + 1), uint64_t(k + k_shift(ca)), rp, qt);
    if (sizeof(F) == 4) {
        w.pose_a[t] = make_float4(float(rp[0]), float(rp[1]), float(rp[2]), 0.0f);
        w.pose_b[t] = make_float4(float(qt[0]), float(qt[1]), float(qt[2]), float(qt[3]));
    } else {
        w.pose64a[t] = make_double4(double(rp[0]), double(rp[1]), double(rp[2]), 0.0);
        w.pose64b[t] = make_double4(double(qt[0]), double(qt[1]), double(qt[2]), double(qt[3]));
    }
    if (ca.reject && hardcore_scan<F, NS>(b, s, fw, rp, qt, rho2, reach0, static_cast<const F*>(ca.rho2max))) {
        mark_rejected(w, t, NS);
        return;
    }
    bin_survivor<F, NS>(b, w, t, fw, rp, qt);
}

// ---------------------------------------------------------------------------------------------
// The FP32 path splits k_pose in two so that phase 0 runs in spatial order: k_draw32 draws every
// pose and gives it a slot in its centre's sub-bin (a scan and scatter then order all insertions
// by sub-bin), and k_phase0_32 tests the hard core of the insertions in that order. The 32
// insertions of a warp then share nearly all of their stencil cells, which the warp stages once,
// where insertion order gives every lane an unrelated stencil.
// ---------------------------------------------------------------------------------------------
template <int NS>
__global__ void __launch_bounds__(256) k_draw32(DevBatch<float> b, CallArgs ca, Work w, Work wa) {
    const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= ca.n_act) return;
    const int64_t i = ca.i_lo + t;
    const int32_t s = find_system(ca.sys_off, b.nsys, i);
    const int64_t k = i - ca.sys_off[s] + 1;
    const int32_t fw = b.framework_of[s];
    float rp[3], qt[4];
    draw_pose<float>(ca.seed_dev ? *ca.seed_dev : ca.seed, uint64_t(s + 1), uint64_t(k + k_shift(ca)), rp, qt);
    w.pose_a[t] = make_float4(rp[0], rp[1], rp[2], 0.0f);
    w.pose_b[t] = make_float4(qt[0], qt[1], qt[2], qt[3]);
    const int32_t fine = sub_bin_of(b, fw, rp[0], rp[1], rp[2]);
    wa.bin_of[t] = fine;
    wa.slot[t] = atomicAdd(&wa.bin_count[fine], 1);
}

__device__ __forceinline__ int32_t floor_div(int32_t x, int32_t n) { return x >= 0 ? x / n : -((n - 1 - x) / n); }
// x / d and x % d for 0 <= x < 2^22 and d >= 1, from the FP32 estimate x * rd (rd = 1/d rounded):
// its error is below one unit there, so one correction each way makes it exact.
__device__ __forceinline__ int32_t div_small(int32_t x, int32_t d, float rd, int32_t& rem) {
    int32_t q = int32_t(float(x) * rd);
    int32_t r = x - q * d;
    if (r < 0) { --q; r += d; } else if (r >= d) { ++q; r -= d; }
    rem = r;
    return q;
}
// floor(x / n) for a cell index x of a region around the grid [0, n): -1, 0 or 1 without a
// division when -n <= x < 2n
__device__ __forceinline__ int32_t wrap_of(int32_t x, int32_t n) {
    if (x >= 0 && x < n) return 0;
    if (x < 0 && x >= -n) return -1;
    if (x >= n && x < 2 * n) return 1;
    return floor_div(x, n);
}

// k_phase0_32: one warp scans the hard core of 32 consecutive insertions of `order` together.
// The warp's insertions lie in one or two centre sub-bins, so their per-site stencils (the cells
// within reach0 of each site's home cell, src/widom.jl:99-151) overlap almost entirely. The warp
// takes as one region of cells the union, over its sites, of the stencil cells that an atom within
// the site's largest hard-core radius can occupy (each site's home cell moved by a whole grid
// period next to the first lane's, so that the region stays compact across the periodic
// boundary), and stages the atom images of the region in shared memory, 32 at a time; every lane
// tests its own insertion against each staged atom, so the lanes do the same work, where one
// stencil walk per lane leaves lanes idle at row boundaries and early exits.
//
// Per staged atom a lane first tests the distance to its insertion's centre against the guest's
// radius plus the largest hard-core radius; only then each site, against the site's largest
// radius squared plus 1e-3 A^2 (the relaxed pre-test, plain FP32). An atom of a site's stencil is
// staged at the image of its stencil cell, which is its strict minimum image whenever it is within
// reach (stencils narrower than the grid), and the plain distances differ from the strict one by
// rounding only, so no atom that can set the flag is skipped. The pairs that pass are queued and
// then decided together, one lane per pair: the strict test of hardcore_scan (minimum image, r^2
// against rho2 of the atom's type), counted only if the atom's cell is in that site's own stencil.
// The flags are therefore exactly those of the per-site stencil scan. Lanes of another system,
// stencils as wide as the grid, or a region wider than the grid take hardcore_scan itself.
#define PA_P0_WARPS 8
#define PA_P0_QMAX 64
template <int NS>
__global__ void __launch_bounds__(32 * PA_P0_WARPS, 4) k_phase0_32(DevBatch<float> b, CallArgs ca, Work w,
                                                                  const int32_t* order, const float* rho2,
                                                                  const int32_t* reach0) {
    __shared__ float4 s_img[PA_P0_WARPS][32];          // staged atom images (x, y, z), packed cell
    __shared__ float4 s_org[PA_P0_WARPS][32];          // the same atoms as stored (x, y, z), type
    __shared__ uint32_t s_q[PA_P0_WARPS][PA_P0_QMAX];  // queued pairs: lane | site << 5 | slot << 10
    __shared__ uint32_t s_hit[PA_P0_WARPS];            // lanes whose insertion overlaps
    __shared__ float s_A[PA_P0_WARPS][18];             // the group's cell, then its inverse
    typedef St<float> S;
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
    const int64_t x = (int64_t(blockIdx.x) * PA_P0_WARPS + wp) * 32 + lane;
    if ((x - lane) >= ca.n_act) return;  // warp-uniform
    const bool valid = x < ca.n_act;
    const int64_t t = valid ? order[x] : 0;
    const int32_t s = valid ? find_system(ca.sys_off, b.nsys, ca.i_lo + t) : -1;
    const int32_t fw = valid ? b.framework_of[s] : 0;
    float rp[3] = {0.f, 0.f, 0.f}, qt[4] = {0.f, 0.f, 0.f, 1.f};
    if (valid) {
        const float4 pa = w.pose_a[t], pq = w.pose_b[t];
        rp[0] = pa.x; rp[1] = pa.y; rp[2] = pa.z;
        qt[0] = pq.x; qt[1] = pq.y; qt[2] = pq.z; qt[3] = pq.w;
    }
    bool hit = false;
    const float* rho2max = static_cast<const float*>(ca.rho2max);
    // the guest's radius: the largest body-frame site distance from its reference point
    float rg = 0.f;
#pragma unroll
    for (int a = 0; a < NS; ++a)
        rg = fmaxf(rg, sqrtf(b.gsite[3 * a] * b.gsite[3 * a] + b.gsite[3 * a + 1] * b.gsite[3 * a + 1] +
                             b.gsite[3 * a + 2] * b.gsite[3 * a + 2]));
    unsigned pending = ca.reject ? __ballot_sync(FULL, valid) : 0u;
    while (pending) {
        const int leader = __ffs(pending) - 1;
        const int32_t s0 = __shfl_sync(FULL, s, leader);
        const bool mine = valid && s == s0;
        pending &= ~__ballot_sync(FULL, mine);
        const int32_t f0 = b.framework_of[s0];
        const int32_t n[3] = {b.ncells[3 * f0], b.ncells[3 * f0 + 1], b.ncells[3 * f0 + 2]};
        const int32_t m[3] = {reach0[3 * s0], reach0[3 * s0 + 1], reach0[3 * s0 + 2]};
        bool wide = rho2max == nullptr || 2 * m[0] + 1 >= n[0] || 2 * m[1] + 1 >= n[1] || 2 * m[2] + 1 >= n[2] ||
                    n[0] >= 1024 || n[1] >= 1024 || n[2] >= 1024;
        const float* A = b.cells + 9 * f0;
        const float* iA = b.invcells + 9 * f0;
        if (lane < 18) s_A[wp][lane] = lane < 9 ? A[lane] : iA[lane - 9];
        if (lane == 0) s_hit[wp] = 0u;
        __syncwarp();
        const float* sA = s_A[wp];
        const float* siA = s_A[wp] + 9;
        // the sites in the frame of their home cell moved next to the leader's: e = b + A k with
        // b = sp - A floor(f); the insertion's reference point c in site 0's frame
        float e[NS][3], lim[NS], c[3], rc2;
        int32_t lo[3] = {INT32_MAX, INT32_MAX, INT32_MAX}, hi[3] = {INT32_MIN, INT32_MIN, INT32_MIN};
        bool off = false;  // sites of one insertion in different frames
        {
            int32_t H[3] = {0, 0, 0};
            float pos[3];
            matvec_s(sA, rp, pos);
            float limmax = 0.f;
#pragma unroll
            for (int a = 0; a < NS; ++a) {
                lim[a] = (mine && !wide) ? rho2max[int64_t(s0) * NS + a] + 1e-3f : -1.0f;
                limmax = fmaxf(limmax, lim[a]);
            }
            // the cells an atom within reach of a site can occupy: |df_r| <= d |row r of A^-1|,
            // d the largest pre-test radius, widened far beyond rounding
            const float dreach = sqrtf(limmax) + 1e-2f;
            float dl[3];
#pragma unroll
            for (int r = 0; r < 3; ++r)
                dl[r] = dreach * float(n[r]) * sqrtf(siA[r] * siA[r] + siA[r + 3] * siA[r + 3] + siA[r + 6] * siA[r + 6]) + 1e-3f;
#pragma unroll
            for (int a = 0; a < NS; ++a) {
                float g[3], sp[3], f[3], fl[3];
                int32_t h[3], k[3];
                rotate_s(qt, b.gsite + 3 * a, g);
                sp[0] = S::add(pos[0], g[0]); sp[1] = S::add(pos[1], g[1]); sp[2] = S::add(pos[2], g[2]);
                matvec_s(siA, sp, f);
#pragma unroll
                for (int r = 0; r < 3; ++r) {
                    h[r] = home_cell_s(wrap_frac_s(f[r]), n[r]);
                    fl[r] = floorf(f[r]);
                }
                if (a == 0) {
#pragma unroll
                    for (int r = 0; r < 3; ++r) H[r] = __shfl_sync(FULL, h[r], leader);
                }
#pragma unroll
                for (int r = 0; r < 3; ++r) {
                    const int32_t d = H[r] - h[r];
                    k[r] = 2 * d > n[r] ? 1 : (2 * d < -n[r] ? -1 : 0);
                    if (mine) {
                        // the site's reach in cells of the moved frame, inside its own stencil
                        const float u = (f[r] - fl[r] + float(k[r])) * float(n[r]);
                        const int32_t hm = h[r] + k[r] * n[r];
                        lo[r] = min(lo[r], max(int32_t(floorf(u - dl[r])), hm - m[r]));
                        hi[r] = max(hi[r], min(int32_t(floorf(u + dl[r])), hm + m[r]));
                    }
                }
                const float sx = fl[0] - float(k[0]), sy = fl[1] - float(k[1]), sz = fl[2] - float(k[2]);
                e[a][0] = sp[0] - (sA[0] * sx + sA[3] * sy + sA[6] * sz);
                e[a][1] = sp[1] - (sA[1] * sx + sA[4] * sy + sA[7] * sz);
                e[a][2] = sp[2] - (sA[2] * sx + sA[5] * sy + sA[8] * sz);
                if (a == 0) { c[0] = e[0][0] - g[0]; c[1] = e[0][1] - g[1]; c[2] = e[0][2] - g[2]; }
                const float ox = e[a][0] - g[0] - c[0], oy = e[a][1] - g[1] - c[1], oz = e[a][2] - g[2] - c[2];
                off = off || !(ox * ox + oy * oy + oz * oz < 1e-4f);
            }
            const float rr = rg + sqrtf(limmax) + 1e-2f;
            rc2 = (mine && !wide) ? rr * rr : -1.0f;
        }
        wide = wide || __any_sync(FULL, mine && off);
#pragma unroll
        for (int r = 0; r < 3; ++r) {
            lo[r] = __reduce_min_sync(FULL, lo[r]);
            hi[r] = __reduce_max_sync(FULL, hi[r]);
            wide = wide || hi[r] - lo[r] + 1 > n[r];
        }
        if (wide) {  // warp-uniform: the per-site stencil walk
            if (mine) hit = hardcore_scan<float, NS>(b, s0, f0, rp, qt, rho2, reach0, rho2max);
            __syncwarp();
            continue;
        }
        const int32_t a0 = b.atom_offsets[f0];
        const int32_t* coff = b.cell_offsets + b.cellgrid_offsets[f0];
        const int32_t nt = b.ntypes;
        const int32_t E0 = hi[0] - lo[0] + 1, E1 = hi[1] - lo[1] + 1;
        const int32_t ncell = E0 * E1 * (hi[2] - lo[2] + 1);
        const float rE0 = 1.0f / float(E0), rE1 = 1.0f / float(E1);
        // decide the queued pairs, one lane each
        const auto flush = [&](int32_t qn) {
            __syncwarp();
            for (int32_t q0 = 0; q0 < qn; q0 += 32) {
                const int32_t qi = q0 + lane;
                const uint32_t ent = qi < qn ? s_q[wp][qi] : 0u;
                const int owner = int(ent & 31u), a = int((ent >> 5) & 31u), slot = int((ent >> 10) & 31u);
                float orp[3], oqt[4];
#pragma unroll
                for (int r = 0; r < 3; ++r) orp[r] = __shfl_sync(FULL, rp[r], owner);
#pragma unroll
                for (int r = 0; r < 4; ++r) oqt[r] = __shfl_sync(FULL, qt[r], owner);
                if (qi < qn) {
                    const float4 at = s_org[wp][slot];
                    const uint32_t cp = __float_as_uint(s_img[wp][slot].w);
                    const float r2lim = rho2[(int64_t(s0) * NS + a) * nt + __float_as_int(at.w)];
                    float pos[3], g[3], sp[3], f[3];
                    matvec_s(sA, orp, pos);
                    rotate_s(oqt, b.gsite + 3 * a, g);
                    sp[0] = S::add(pos[0], g[0]); sp[1] = S::add(pos[1], g[1]); sp[2] = S::add(pos[2], g[2]);
                    float D[3] = {S::sub(sp[0], at.x), S::sub(sp[1], at.y), S::sub(sp[2], at.z)};
                    minimum_image_s(sA, siA, D);
                    const float r2 = dot3s(D[0], D[1], D[2], D[0], D[1], D[2]);
                    matvec_s(siA, sp, f);
                    const int32_t cc[3] = {int32_t(cp & 1023u), int32_t((cp >> 10) & 1023u), int32_t(cp >> 20)};
                    bool in = r2 < r2lim;
#pragma unroll
                    for (int r = 0; r < 3; ++r) {
                        const int32_t h = home_cell_s(wrap_frac_s(f[r]), n[r]);
                        int32_t dd = (cc[r] - (h - m[r])) % n[r];
                        if (dd < 0) dd += n[r];
                        in = in && dd <= 2 * m[r];
                    }
                    if (in) atomicOr(&s_hit[wp], 1u << owner);
                }
            }
            __syncwarp();
            if ((s_hit[wp] >> lane) & 1u) {
                hit = true;
                rc2 = -1.0f;
#pragma unroll
                for (int a = 0; a < NS; ++a) lim[a] = -1.0f;
            }
        };
        for (int32_t p0 = 0; p0 < ncell; p0 += 32) {
            // this round's region cells, one per lane: atom range, image shift, packed cell
            const int32_t pi = p0 + lane;
            int32_t j0 = 0, cnt = 0;
            float Wx = 0.f, Wy = 0.f, Wz = 0.f;
            uint32_t cpk = 0u;
            if (pi < ncell) {
                int32_t u[3];
                if (ncell < (1 << 22)) {
                    int32_t r0, r1;
                    const int32_t q0 = div_small(pi, E0, rE0, r0);
                    const int32_t q1 = div_small(q0, E1, rE1, r1);
                    u[0] = lo[0] + r0; u[1] = lo[1] + r1; u[2] = lo[2] + q1;
                } else {
                    u[0] = lo[0] + pi % E0; u[1] = lo[1] + (pi / E0) % E1; u[2] = lo[2] + pi / (E0 * E1);
                }
                int32_t cc[3];
                float wv[3];
#pragma unroll
                for (int r = 0; r < 3; ++r) {
                    const int32_t wr = wrap_of(u[r], n[r]);
                    cc[r] = u[r] - wr * n[r];
                    wv[r] = float(wr);
                }
                const int32_t ci = cc[0] + n[0] * (cc[1] + n[1] * cc[2]);
                j0 = a0 + coff[ci];
                cnt = a0 + coff[ci + 1] - j0;
                Wx = sA[0] * wv[0] + sA[3] * wv[1] + sA[6] * wv[2];
                Wy = sA[1] * wv[0] + sA[4] * wv[1] + sA[7] * wv[2];
                Wz = sA[2] * wv[0] + sA[5] * wv[1] + sA[8] * wv[2];
                cpk = uint32_t(cc[0]) | (uint32_t(cc[1]) << 10) | (uint32_t(cc[2]) << 20);
            }
            int32_t incl = cnt;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int32_t v = __shfl_up_sync(FULL, incl, o);
                if (lane >= o) incl += v;
            }
            const int32_t excl = incl - cnt;
            const int32_t total = __shfl_sync(FULL, incl, 31);
            for (int32_t q = 0; q < total; q += 32) {
                // the cell holding staged atom q + lane: the last one starting at or before it
                const int32_t gi = q + lane;
                int32_t src = 0;
#pragma unroll
                for (int step = 16; step >= 1; step >>= 1) {
                    const int32_t ex = __shfl_sync(FULL, excl, src + step);
                    if (ex <= gi) src += step;
                }
                const int32_t js = __shfl_sync(FULL, j0, src) + gi - __shfl_sync(FULL, excl, src);
                const float sx = __shfl_sync(FULL, Wx, src), sy = __shfl_sync(FULL, Wy, src),
                            sz = __shfl_sync(FULL, Wz, src);
                const uint32_t scp = __shfl_sync(FULL, cpk, src);
                if (gi < total) {
                    const float4 at = b.atoms[js];
                    const int32_t ty = b.types[js];
                    s_img[wp][lane] = make_float4(at.x + sx, at.y + sy, at.z + sz, __uint_as_float(scp));
                    s_org[wp][lane] = make_float4(at.x, at.y, at.z, __int_as_float(ty));
                }
                __syncwarp();
                const int32_t nb = min(32, total - q);
                int32_t qn = 0;  // queued pairs (the same on every lane)
                for (int32_t kk = 0; kk < nb; ++kk) {
                    const float4 v = s_img[wp][kk];
                    const float cx = c[0] - v.x, cy = c[1] - v.y, cz = c[2] - v.z;
                    const bool near = cx * cx + cy * cy + cz * cz < rc2;
                    if (!__any_sync(FULL, near)) continue;
#pragma unroll
                    for (int a = 0; a < NS; ++a) {
                        const float dx = e[a][0] - v.x, dy = e[a][1] - v.y, dz = e[a][2] - v.z;
                        const bool cand = near && dx * dx + dy * dy + dz * dz < lim[a];
                        const uint32_t bal = __ballot_sync(FULL, cand);
                        if (bal == 0u) continue;
                        if (qn + __popc(bal) > PA_P0_QMAX) {
                            flush(qn);
                            qn = 0;
                        }
                        if (cand) s_q[wp][qn + __popc(bal & ((1u << lane) - 1u))] = uint32_t(lane) | (uint32_t(a) << 5) | (uint32_t(kk) << 10);
                        qn += __popc(bal);
                    }
                }
                if (qn > 0) flush(qn);
                __syncwarp();  // the staged batch is no longer read
            }
        }
    }
    if (!valid) return;
    if (hit) {
        mark_rejected(w, t, NS);
        return;
    }
    bin_survivor<float, NS>(b, w, t, fw, rp, qt);
}

// ---------------------------------------------------------------------------------------------
// k_combine (FP32 path): ΔU = Σ_sites (real-space site sums) + KE E_lr (+ the guest-guest term
// along a chain) + constant offset, in a fixed order; rejected insertions keep +inf.
// ---------------------------------------------------------------------------------------------
template <int NS>
__global__ void __launch_bounds__(256) k_combine(DevBatch<float> b, CallArgs ca, Work w) {
    const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= ca.n_act || w.bin_of[t] < 0) return;
    const int32_t s = find_system(ca.sys_off, b.nsys, ca.i_lo + t);
    const int32_t fw = b.framework_of[s];
    double e = w.dUs[t * NS];
#pragma unroll
    for (int a = 1; a < NS; ++a) e += w.dUs[t * NS + a];
    if (b.has_charge) e += w.dUr[t];
    if (w.dUg) e += w.dUg[t];
    w.dU[t] = e + b.const_offset[fw];
}

// ---------------------------------------------------------------------------------------------
// k_scan: one CTA of 1024 threads; exclusive scans of bin counts and of tile counts
// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ int32_t block_excl_scan(int32_t v, int32_t* s_warp, int32_t* total) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    int32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) s_warp[wid] = x;
    __syncthreads();
    if (wid == 0) {
        int32_t z = lane < nw ? s_warp[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int32_t y = __shfl_up_sync(0xffffffffu, z, o);
            if (lane >= o) z += y;
        }
        if (lane < nw) s_warp[lane] = z;  // inclusive warp prefix
    }
    __syncthreads();
    int32_t warp_excl = wid == 0 ? 0 : s_warp[wid - 1];
    *total = s_warp[nw - 1];
    __syncthreads();
    return warp_excl + x - v;
}

// The arrays of one sort, by value (a kernel parameter whose address is taken would be copied
// to local memory).
struct SortView {
    const int32_t* count;
    int32_t* fine_start;
    int32_t* bin_start;
    int32_t* tile_start;
    int32_t* counters;
    const int32_t* bin_of;
    const int32_t* slot;
    int32_t* sorted;
};
__host__ __device__ inline SortView sort_view(const Work& w) {
    return SortView{w.bin_count, w.fine_start, w.bin_start, w.tile_start, w.counters, w.bin_of, w.slot, w.sorted};
}

// Each thread takes PA_SCAN_V consecutive elements per round (a serial prefix in registers), so
// that a round of the block covers 1024 * PA_SCAN_V elements with one block-wide scan.
#define PA_SCAN_V 8
__device__ __forceinline__ void scan_body(SortView w, int32_t nbins, int32_t nsub, int32_t tile) {
    __shared__ int32_t s_warp[32];
    const int32_t nfine = nbins * nsub;
    const int32_t per = int32_t(blockDim.x) * PA_SCAN_V;
    int32_t carry = 0;
    for (int32_t base = 0; base < nfine; base += per) {  // survivors per sub-bin -> starts
        const int32_t f0 = base + int32_t(threadIdx.x) * PA_SCAN_V;
        int32_t v[PA_SCAN_V], sum = 0;
#pragma unroll
        for (int u = 0; u < PA_SCAN_V; ++u) {
            v[u] = f0 + u < nfine ? w.count[f0 + u] : 0;
            sum += v[u];
        }
        int32_t tot;
        int32_t e = carry + block_excl_scan(sum, s_warp, &tot);
#pragma unroll
        for (int u = 0; u < PA_SCAN_V; ++u) {
            if (f0 + u < nfine) w.fine_start[f0 + u] = e;
            e += v[u];
        }
        carry += tot;
    }
    if (threadIdx.x == 0) w.fine_start[nfine] = carry;
    __syncthreads();
    int32_t carry_t = 0;
    for (int32_t base = 0; base < nbins; base += per) {  // tiles per bin
        const int32_t b0 = base + int32_t(threadIdx.x) * PA_SCAN_V;
        int32_t v[PA_SCAN_V], sum = 0;
#pragma unroll
        for (int u = 0; u < PA_SCAN_V; ++u) {
            const int32_t bn = b0 + u;
            v[u] = 0;
            if (bn < nbins) {
                const int32_t s0 = w.fine_start[bn * nsub], s1 = w.fine_start[(bn + 1) * nsub];
                w.bin_start[bn] = s0;
                v[u] = (s1 - s0 + tile - 1) / tile;
            }
            sum += v[u];
        }
        int32_t tt;
        int32_t e = carry_t + block_excl_scan(sum, s_warp, &tt);
#pragma unroll
        for (int u = 0; u < PA_SCAN_V; ++u) {
            if (b0 + u < nbins) w.tile_start[b0 + u] = e;
            e += v[u];
        }
        carry_t += tt;
    }
    if (threadIdx.x == 0) {
        w.bin_start[nbins] = carry;
        w.tile_start[nbins] = carry_t;
        w.counters[1] = carry_t;
        w.counters[3] = carry;
    }
}

__global__ void __launch_bounds__(1024) k_scan(SortView w, int32_t nbins, int32_t nsub, int32_t tile) {
    scan_body(w, nbins, nsub, tile);
}

// Two independent scans in one launch, one CTA each (the survivors' and the items' sort).
__global__ void __launch_bounds__(1024) k_scan2(SortView w0, SortView w1, int32_t nbins, int32_t nsub, int32_t tile) {
    if (blockIdx.x == 0) scan_body(w0, nbins, nsub, tile);
    else scan_body(w1, nbins, nsub, tile);
}

__device__ __forceinline__ void scatter_one(const SortView& w, int64_t t) {
    const int32_t bin = w.bin_of[t];
    if (bin >= 0) w.sorted[w.fine_start[bin] + w.slot[t]] = int32_t(t);
}

__global__ void k_scatter(SortView w, int64_t n_act) {
    const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t < n_act) scatter_one(w, t);
}

// Two scatters in one launch: entries [0, n0) of w0, then [0, n1) of w1.
__global__ void k_scatter2(SortView w0, int64_t n0, SortView w1, int64_t n1) {
    const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t < n0) scatter_one(w0, t);
    else if (t - n0 < n1) scatter_one(w1, t - n0);
}

// ---------------------------------------------------------------------------------------------
// Bulk-copy pipeline primitives (cp.async.bulk, mbarrier), with bounded waits.
// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return uint32_t(__cvta_generic_to_shared(p)); }
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok) : "r"(smem_u32(bar)), "r"(parity) : "memory");
    return ok != 0;
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 ::"r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// Waits for phase `parity` of `bar`; gives up after PA_WAIT_LIMIT polls and returns false.
#define PA_WAIT_LIMIT (1 << 26)
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
    for (uint32_t it = 0; it < PA_WAIT_LIMIT; ++it)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

// ---------------------------------------------------------------------------------------------
// FP32 helpers. rcp_nr: hardware reciprocal estimate refined by one Newton step (about 1 ulp).
// erfc_over_r: erfc(z)/r with z = alpha r, r = sqrt(r2); erfc(z) = exp(-z^2) P(t), t = 2/(2+z),
// P a degree-9 fit (gen_coeffs.py), about 2e-7 relative on [0, 4].
// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ float rcp_nr(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return fmaf(r, fmaf(-x, r, 1.0f), r);
}
__device__ __forceinline__ float erfc_over_r(float r2, float alpha) {
    float ri = rsqrtf(r2);
    ri = ri * fmaf(-0.5f * r2 * ri, ri, 1.5f);  // one Newton step
    const float z = alpha * (r2 * ri);
    const float t = rcp_nr(fmaf(0.5f, z, 1.0f));
    const float c[PA_NERFC32] = PA_ERFC32_INIT;
    float p = c[PA_NERFC32 - 1];
#pragma unroll
    for (int k = PA_NERFC32 - 2; k >= 0; --k) p = fmaf(p, t, c[k]);
    return p * __expf(-z * z) * ri;
}

#include "pa_energy32.cuh"
#include "pa_grad32.cuh"
#include "pa_chain32.cuh"
#include "pa_build.cuh"

// ---------------------------------------------------------------------------------------------
// k_energy64: the plain FP64 form of the reference algorithm (src/energy.jl:42-82): for every
// atom of the framework one minimum image of pos - r_j, then each site's offset added;
// LJ and screened Coulomb (CUDA's double erfc) inside the cutoffs; reciprocal cross term with
// double sincos. Tiles hold survivors of one framework; atoms staged through shared memory.
// ---------------------------------------------------------------------------------------------
#define PA_TILE64 128
#define PA_CHUNK64 128

template <int NS>
__global__ void __launch_bounds__(PA_TILE64) k_energy64(DevBatch<double> b, CallArgs ca, Work w) {
    __shared__ double4 s_at[PA_CHUNK64];
    __shared__ int32_t s_ty[PA_CHUNK64];
    __shared__ int32_t s_item[4];
    const int tid = threadIdx.x;
    const int32_t total_tiles = w.counters[1];
    const int nt = b.ntypes;
    for (;;) {
        if (tid == 0) {
            int32_t t = atomicAdd(&w.counters[0], 1);
            s_item[0] = t;
            if (t < total_tiles) {
                int32_t bin = find_bin(w.tile_start, b.nbins, t);
                int32_t lo = w.bin_start[bin] + (t - w.tile_start[bin]) * PA_TILE64;
                s_item[1] = bin; s_item[2] = lo; s_item[3] = min(lo + PA_TILE64, w.bin_start[bin + 1]);
            }
        }
        __syncthreads();
        const int32_t t = s_item[0];
        if (t >= total_tiles) break;
        const int32_t bin = s_item[1], lo = s_item[2], hi = s_item[3];
        __syncthreads();
        const int32_t fw = b.bin_fw[bin];
        const bool active = lo + tid < hi;
        const int32_t li = active ? w.sorted[lo + tid] : 0;
        const double4 pa = active ? w.pose64a[li] : make_double4(0.5, 0.5, 0.5, 0);
        const double4 pq = active ? w.pose64b[li] : make_double4(0, 0, 0, 1);
        double A[9], iA[9];
#pragma unroll
        for (int r = 0; r < 9; ++r) { A[r] = b.cells[9 * fw + r]; iA[r] = b.invcells[9 * fw + r]; }
        const double rp[3] = {pa.x, pa.y, pa.z}, q[4] = {pq.x, pq.y, pq.z, pq.w};
        double pos[3];
        matvec_s(A, rp, pos);
        double gx[NS], gy[NS], gz[NS];
#pragma unroll
        for (int s = 0; s < NS; ++s) {
            double g[3];
            rotate_s(q, b.gsite + 3 * s, g);
            gx[s] = g[0]; gy[s] = g[1]; gz[s] = g[2];
        }
        const double rl2 = b.rl2, re2 = b.re2, alpha = b.alphas[fw];
        double elj = 0, esr = 0;
        const int32_t a0 = b.atom_offsets[fw], a1 = b.atom_offsets[fw + 1];
        for (int32_t c0 = a0; c0 < a1; c0 += PA_CHUNK64) {
            const int32_t n = min(PA_CHUNK64, a1 - c0);
            for (int32_t x = tid; x < n; x += blockDim.x) { s_at[x] = b.atoms[c0 + x]; s_ty[x] = b.types[c0 + x]; }
            __syncthreads();
            for (int32_t j = 0; j < n; ++j) {
                const double4 at = s_at[j];
                double D[3] = {pos[0] - at.x, pos[1] - at.y, pos[2] - at.z};
                const double f0 = iA[0] * D[0] + iA[3] * D[1] + iA[6] * D[2];
                const double f1 = iA[1] * D[0] + iA[4] * D[1] + iA[7] * D[2];
                const double f2 = iA[2] * D[0] + iA[5] * D[1] + iA[8] * D[2];
                const double r0 = rint(f0), r1 = rint(f1), r2i = rint(f2);
                D[0] -= A[0] * r0 + A[3] * r1 + A[6] * r2i;
                D[1] -= A[1] * r0 + A[4] * r1 + A[7] * r2i;
                D[2] -= A[2] * r0 + A[5] * r1 + A[8] * r2i;
                const int32_t ty = s_ty[j];
#pragma unroll
                for (int s = 0; s < NS; ++s) {
                    const double dx = D[0] + gx[s], dy = D[1] + gy[s], dz = D[2] + gz[s];
                    const double r2 = dx * dx + dy * dy + dz * dz;
                    if (r2 < rl2) {
                        const double sg = b.sig2[s * nt + ty] / r2;
                        const double x3 = sg * sg * sg;
                        elj += b.eps4[s * nt + ty] * (x3 * x3 - x3);
                    }
                    if (r2 < re2 && b.has_charge) {
                        const double r = sqrt(r2);
                        esr += b.gq[s] * at.w * erfc(alpha * r) / r;
                    }
                }
            }
            __syncthreads();
        }
        double elr = 0;
        if (b.has_charge) {
            for (int32_t kk = b.k_offsets[fw]; kk < b.k_offsets[fw + 1]; ++kk) {
                const double kx = b.kvec[3 * kk], ky = b.kvec[3 * kk + 1], kz = b.kvec[3 * kk + 2];
                double gr = 0, gi = 0;
#pragma unroll
                for (int s = 0; s < NS; ++s) {
                    double sn, cs;
                    sincos(kx * (pos[0] + gx[s]) + ky * (pos[1] + gy[s]) + kz * (pos[2] + gz[s]), &sn, &cs);
                    gr += b.gq[s] * cs; gi += b.gq[s] * sn;
                }
                elr += b.kS2[2 * kk] * gr + b.kS2[2 * kk + 1] * gi;
            }
        }
        if (active) w.dU[li] = elj + KE * (esr + elr) + b.const_offset[fw];
    }
}

// ---------------------------------------------------------------------------------------------
// k_segsum: per segment, x_i = -ΔU_i/kT; m = max x; Σ exp(x - m); Σ ΔU exp(x - m) (terms whose
// weight is exactly zero contribute zero, as in boltzmann_weight). 256 threads, 8 consecutive
// insertions per thread summed in order, then a fixed shuffle/shared-memory tree.
// ---------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_segsum(Work w, double kT, const double* kT_dev) {
    if (kT_dev) kT = *kT_dev;
    __shared__ double s_red[3][8];
    const int64_t b0 = w.seg_rng[2 * blockIdx.x], b1 = w.seg_rng[2 * blockIdx.x + 1];
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const int per = PA_SEGMENT_SIZE / 256;
    const double NEG_INF = __longlong_as_double(0xfff0000000000000LL);
    double xs[per], us[per];
    double m = NEG_INF;
#pragma unroll
    for (int q = 0; q < per; ++q) {
        const int64_t i = b0 + int64_t(tid) * per + q;
        double u = i < b1 ? w.dU[i] : __longlong_as_double(0x7ff0000000000000LL);
        double x = -u / kT;
        xs[q] = x; us[q] = u;
        m = fmax(m, x);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if (lane == 0) s_red[0][wid] = m;
    __syncthreads();
    m = s_red[0][0];
#pragma unroll
    for (int q = 1; q < 8; ++q) m = fmax(m, s_red[0][q]);
    __syncthreads();
    double sw = 0, su = 0;
    if (m != NEG_INF && !isnan(m)) {
#pragma unroll
        for (int q = 0; q < per; ++q) {
            const double e = exp(xs[q] - m);
            if (e != 0.0) { sw += e; su += us[q] * e; }
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        sw += __shfl_xor_sync(0xffffffffu, sw, o);
        su += __shfl_xor_sync(0xffffffffu, su, o);
    }
    if (lane == 0) { s_red[1][wid] = sw; s_red[2][wid] = su; }
    __syncthreads();
    if (tid == 0) {
        double a = 0, c = 0;
#pragma unroll
        for (int q = 0; q < 8; ++q) { a += s_red[1][q]; c += s_red[2][q]; }
        w.seg_out[3 * blockIdx.x] = m;
        w.seg_out[3 * blockIdx.x + 1] = a;
        w.seg_out[3 * blockIdx.x + 2] = c;
    }
}

// ---------------------------------------------------------------------------------------------
// Neighbour lists of the FP32 path: for bin centre c (fractional, FP32-defined) and atom j with
// fractional position f_j, every image A (f_j - c - round(f_j - c) + n), n in [-m, m]^3, within
// radius R is one entry, stored relative to the bin centre. Order: atoms by type (then by index),
// then n (x fastest), so the lists (and every energy sum over them) are deterministic and each
// type is one contiguous run. One CTA per bin.
// ---------------------------------------------------------------------------------------------
struct ListGeom {
    const double* frac;        // 3*natoms fractional coordinates (cell-sorted order)
    const double* charges;     // natoms
    const int32_t* types;      // natoms, 0-based
    const double* cells;       // 9*nfw
    const int32_t* atom_offsets;
    const int32_t* order;      // natoms: the framework's atoms ordered by type (stable), global indices
    const float4* fr32;        // natoms: FP32 fractional coordinates of order[rank], by rank
    const int32_t* bin_dims;   // 3*nfw
    const int32_t* bin_base;   // nfw+1
    const int32_t* bin_fw;     // nbins
    const double* radius2;     // nfw
    const int32_t* nimg;       // nfw: m
    const float* reach;        // 3*nfw: R / L_r plus a margin (images beyond it are never kept)
    int32_t* counts;           // nbins (count pass)
    const int32_t* offsets;    // nbins+1 (fill pass)
    float4* xyzq;
    double4* xyzq64;           // the same entries in FP64
    int32_t* type_out;
    int32_t* atom_out;         // stored-atom index of each entry (for the adjoint)
};

// Neighbour lists of the FP32 path: per bin, every atom image within R of the bin centre, in the
// order (atom rank in `order`, image index) with the image index n0 + side (n1 + side n2) running
// fastest. Each thread takes LIST_ATOMS consecutive atom ranks. An image can only lie within R if
// |d_r + n_r| <= R / L_r on each axis (L_r the perpendicular width), so a thread tests only the
// images inside that box (a margin far above FP32 rounding keeps every image the strict test
// would keep); an ordered block scan of the per-thread counts then places its entries. Count and
// fill passes make the same tests, so the fill writes exactly the counted entries.
// The type runs of every bin's list (entries are in type-major order): one warp per bin, the run
// starts found by ballot in entry order; the remaining slots (at least one) hold (end, 0).
__global__ void __launch_bounds__(32) k_runs(const int32_t* offsets, const int32_t* type, int2* runs, int32_t rm) {
    const int32_t bin = blockIdx.x, lane = threadIdx.x;
    const int32_t l0 = offsets[bin], l1 = offsets[bin + 1];
    int2* r = runs + int64_t(bin) * rm;
    int32_t k = 0;
    for (int32_t e0 = l0; e0 < l1; e0 += 32) {
        const int32_t e = e0 + lane;
        bool start = false;
        int32_t t = 0;
        if (e < l1) {
            t = type[e];
            start = e == l0 || type[e - 1] != t;
        }
        const unsigned bal = __ballot_sync(0xffffffffu, start);
        if (start) {
            const int32_t idx = k + __popc(bal & ((1u << lane) - 1u));
            if (idx < rm - 1) r[idx] = make_int2(e, t);
        }
        k += __popc(bal);
    }
    for (int32_t i = min(k, rm - 1) + lane; i < rm; i += 32) r[i] = make_int2(l1, 0);
}

#define LIST_ATOMS 4
template <bool FILL>
__global__ void __launch_bounds__(256) k_lists(ListGeom g) {
    __shared__ int32_t s_warp[8];
    __shared__ int32_t s_base;
    const int32_t bin = blockIdx.x, fw = g.bin_fw[bin];
    const int32_t* nb = g.bin_dims + 3 * fw;
    const int32_t lb = bin - g.bin_base[fw];
    const int32_t bx = lb % nb[0], by = (lb / nb[0]) % nb[1], bz = lb / (nb[0] * nb[1]);
    const double c[3] = {double(__fdiv_rn(float(bx) + 0.5f, float(nb[0]))),
                         double(__fdiv_rn(float(by) + 0.5f, float(nb[1]))),
                         double(__fdiv_rn(float(bz) + 0.5f, float(nb[2])))};
    double A[9];
    float Af[9];
#pragma unroll
    for (int r = 0; r < 9; ++r) { A[r] = g.cells[9 * fw + r]; Af[r] = float(A[r]); }
    const float cf[3] = {float(c[0]), float(c[1]), float(c[2])};
    const float R2f = float(g.radius2[fw]);
    const float reach[3] = {g.reach[3 * fw], g.reach[3 * fw + 1], g.reach[3 * fw + 2]};
    const int32_t m = g.nimg[fw];
    const int32_t a0 = g.atom_offsets[fw], a1 = g.atom_offsets[fw + 1];
    if (threadIdx.x == 0) s_base = FILL ? g.offsets[bin] : 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    typedef St<float> S;
    // strict FP32 membership of image (n0, n1, n2) of an atom at fractional offset d from the centre
    const auto inside = [&](const float* d, int32_t n0, int32_t n1, int32_t n2) {
        const float e0 = S::add(d[0], float(n0)), e1 = S::add(d[1], float(n1)), e2 = S::add(d[2], float(n2));
        const float x = dot3s(Af[0], Af[3], Af[6], e0, e1, e2);
        const float y = dot3s(Af[1], Af[4], Af[7], e0, e1, e2);
        const float z = dot3s(Af[2], Af[5], Af[8], e0, e1, e2);
        return dot3s(x, y, z, x, y, z) <= R2f;
    };
    int32_t cnt_total = 0;  // count pass: this thread's entries
    // LIST_ATOMS consecutive atom ranks per thread, their loads issued together
    for (int32_t r0 = a0; r0 < a1; r0 += LIST_ATOMS * int32_t(blockDim.x)) {
        int32_t j[LIST_ATOMS], lo[LIST_ATOMS][3], hi[LIST_ATOMS][3];
        float d[LIST_ATOMS][3];
        int32_t cnt = 0;
#pragma unroll
        for (int u = 0; u < LIST_ATOMS; ++u) {
            const int32_t rk = r0 + LIST_ATOMS * int32_t(threadIdx.x) + u;
            j[u] = 0;
#pragma unroll
            for (int r = 0; r < 3; ++r) { lo[u][r] = 0; hi[u][r] = -1; d[u][r] = 0.f; }
            if (rk < a1) {
                if constexpr (FILL) j[u] = g.order[rk];  // the count pass runs before `order` is uploaded
                const float4 f = g.fr32[rk];
                const float fv[3] = {f.x, f.y, f.z};
#pragma unroll
                for (int r = 0; r < 3; ++r) {
                    float v = S::sub(fv[r], cf[r]);
                    d[u][r] = S::sub(v, rintf(v));
                    lo[u][r] = max(-m, int32_t(ceilf(-reach[r] - d[u][r])));
                    hi[u][r] = min(m, int32_t(floorf(reach[r] - d[u][r])));
                }
            }
        }
        // the same tests in both passes: first count, then (fill) write in (rank, image) order
#pragma unroll
        for (int u = 0; u < LIST_ATOMS; ++u)
            for (int32_t n2 = lo[u][2]; n2 <= hi[u][2]; ++n2)
                for (int32_t n1 = lo[u][1]; n1 <= hi[u][1]; ++n1)
                    for (int32_t n0 = lo[u][0]; n0 <= hi[u][0]; ++n0) cnt += inside(d[u], n0, n1, n2) ? 1 : 0;
        if constexpr (!FILL) {  // the count pass only needs the bin's total: one reduction at the end
            cnt_total += cnt;
            continue;
        }
        // ordered exclusive scan of the counts over the block
        int32_t incl = cnt;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int32_t v = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += v;
        }
        if (lane == 31) s_warp[wid] = incl;
        __syncthreads();
        int32_t before = 0, tot = 0;
        for (int q = 0; q < 8; ++q) { int32_t v = s_warp[q]; if (q < wid) before += v; tot += v; }
        if (FILL && cnt > 0) {
            int32_t pos = s_base + before + incl - cnt;
            const int32_t pend = g.offsets[bin + 1];
            typedef St<double> D;
#pragma unroll
            for (int u = 0; u < LIST_ATOMS; ++u) {
                if (lo[u][0] > hi[u][0] || lo[u][1] > hi[u][1] || lo[u][2] > hi[u][2]) continue;
                // the atom's FP64 offset from the bin centre, its charge and type: read once
                const int32_t ja = j[u];
                double b0 = D::sub(g.frac[3 * ja], c[0]), b1 = D::sub(g.frac[3 * ja + 1], c[1]),
                       b2 = D::sub(g.frac[3 * ja + 2], c[2]);
                b0 = D::sub(b0, rint(b0)); b1 = D::sub(b1, rint(b1)); b2 = D::sub(b2, rint(b2));
                const float qa = float(g.charges[ja]);
                const int32_t ta = g.types[ja];
                for (int32_t n2 = lo[u][2]; n2 <= hi[u][2]; ++n2)
                    for (int32_t n1 = lo[u][1]; n1 <= hi[u][1]; ++n1)
                        for (int32_t n0 = lo[u][0]; n0 <= hi[u][0]; ++n0) {
                            if (!inside(d[u], n0, n1, n2)) continue;
                            if (pos < pend) {
                                // the stored position relative to the bin centre, in FP64 then rounded once
                                const double d0 = D::add(b0, double(n0)), d1 = D::add(b1, double(n1)),
                                             d2 = D::add(b2, double(n2));
                                const double dx = dot3s(A[0], A[3], A[6], d0, d1, d2);
                                const double dy = dot3s(A[1], A[4], A[7], d0, d1, d2);
                                const double dz = dot3s(A[2], A[5], A[8], d0, d1, d2);
                                g.xyzq[pos] = make_float4(float(dx), float(dy), float(dz), qa);
                                g.xyzq64[pos] = make_double4(dx, dy, dz, g.charges[ja]);
                                g.type_out[pos] = ta;
                                g.atom_out[pos] = ja;
                            }
                            ++pos;
                        }
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) s_base += tot;
        __syncthreads();
    }
    if constexpr (!FILL) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) cnt_total += __shfl_xor_sync(0xffffffffu, cnt_total, o);
        if (lane == 0) s_warp[wid] = cnt_total;
        __syncthreads();
        if (threadIdx.x == 0) {
            int32_t tot = 0;
            for (int q = 0; q < 8; ++q) tot += s_warp[q];
            g.counts[bin] = tot;
        }
    }
    if (FILL) {  // padding entries up to the next offset: far away, no charge
        const int32_t end = g.offsets[bin + 1];
        for (int32_t q = s_base + threadIdx.x; q < end; q += blockDim.x) {
            g.xyzq[q] = make_float4(1.0e15f, 1.0e15f, 1.0e15f, 0.0f);
            g.xyzq64[q] = make_double4(1.0e15, 1.0e15, 1.0e15, 0.0);
            g.type_out[q] = 0;
            g.atom_out[q] = 0;
        }
    }
}

// Guest self term per orientation (src/batch.jl:357-375): one CTA per orientation o, threads over
// the k-vectors, Σ_k kpref_k |Σ_s q_s e^{i k·g_s(o)}|^2 in FP64, per-thread partial sums then a
// fixed tree over the CTA.
__global__ void __launch_bounds__(256) k_self_term(const double* ks, const double* kpref, int64_t nk,
                                                   const double* sites, const double* q, int32_t N, double* out) {
    __shared__ double s_red[256];
    const int32_t o = blockIdx.x;
    const double* g = sites + int64_t(o) * N * 3;
    double acc = 0.0;
    for (int64_t i = threadIdx.x; i < nk; i += blockDim.x) {
        const double kx = ks[3 * i], ky = ks[3 * i + 1], kz = ks[3 * i + 2];
        double re = 0.0, im = 0.0;
        for (int32_t s = 0; s < N; ++s) {
            double sn, cs;
            sincos(kx * g[3 * s] + ky * g[3 * s + 1] + kz * g[3 * s + 2], &sn, &cs);
            re += q[s] * cs;
            im += q[s] * sn;
        }
        acc += kpref[i] * (re * re + im * im);
    }
    s_red[threadIdx.x] = acc;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (int(threadIdx.x) < w) s_red[threadIdx.x] += s_red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[o] = s_red[0];
}

// FP64 structure factor: one thread per k-vector, sequential sum over atoms (src/ewald.jl:159-170).
__global__ void __launch_bounds__(256) k_structure_factor(const double* ks, int64_t nk, const double* pos,
                                                          const double* q, int64_t na, double* S) {
    __shared__ double4 s_a[256];
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    double kx = 0, ky = 0, kz = 0;
    if (i < nk) { kx = ks[3 * i]; ky = ks[3 * i + 1]; kz = ks[3 * i + 2]; }
    double re = 0, im = 0;
    for (int64_t c0 = 0; c0 < na; c0 += 256) {
        const int64_t n = (na - c0) < 256 ? (na - c0) : 256;
        if (threadIdx.x < n) {
            const int64_t j = c0 + threadIdx.x;
            s_a[threadIdx.x] = make_double4(pos[3 * j], pos[3 * j + 1], pos[3 * j + 2], q[j]);
        }
        __syncthreads();
        for (int64_t j = 0; j < n; ++j) {
            const double4 a = s_a[j];
            double sn, cs;
            sincos(kx * a.x + ky * a.y + kz * a.z, &sn, &cs);
            re += a.w * cs; im += a.w * sn;
        }
        __syncthreads();
    }
    if (i < nk) { S[2 * i] = re; S[2 * i + 1] = im; }
}

// ---------------------------------------------------------------------------------------------
// k_hardcore_bound: the hard-core bound B_s of each framework on the device (src/reject.jl:95-124,
// the reference's `hardcore_bound`): Σ over guest sites a and host atoms j of eps_aj for repulsive
// or neutral pairs, and eps_aj + |K| erfc(alpha r0)/r0 for attractive ones (K = KE q_a q_j < 0),
// r0 the zero of LJ + screened Coulomb below the LJ minimum (find_r0, src/reject.jl:46-69,
// bisection to 4 eps relative, clamped to r_lj). FP64. One CTA per framework, a fixed-order
// reduction; err[0] gets 1 when a bracket search fails and B_s is +inf for an attractive pair
// without an LJ wall.
// ---------------------------------------------------------------------------------------------
struct BoundArgs {
    const int32_t* types;    // natoms, 0-based compact
    const double* charges;   // natoms
    const int32_t* atom_offsets;
    const double* alphas;    // nfw
    const double* site_sig;  // N*nt (site, type)
    const double* site_eps;  // N*nt
    const double* gq;        // N guest charges
    int32_t N, nt;
    double r_lj;
    double* out;             // nfw*nchunk: partial sum of each chunk of BOUND_CHUNK (site, atom) pairs
    int32_t nchunk;          // chunks per framework (the largest framework's count)
    int32_t* err;
};
#define BOUND_CHUNK 2048

__device__ __forceinline__ double bound_pair_energy(double r, double s, double e, double K, double alpha) {
    double x = (s * s) / (r * r);
    x = x * x * x;
    return 4.0 * e * (x * x - x) + K * erfc(alpha * r) / r;
}

__device__ double bound_find_r0(double s, double e, double K, double alpha, double r_lj, int32_t* err) {
    double hi = s * 1.122462048309373;  // 2^(1/6)
    if (!(bound_pair_energy(hi, s, e, K, alpha) < 0)) { *err = 1; return r_lj; }
    double lo = hi;
    int it = 0;
    while (bound_pair_energy(lo, s, e, K, alpha) <= 0) {
        lo *= 0.5;
        if (++it > 200) { *err = 1; return r_lj; }
    }
    it = 0;
    const double eps = 2.220446049250313e-16;
    while (hi - lo > 4 * eps * hi) {
        const double mid = (lo + hi) / 2;
        if (bound_pair_energy(mid, s, e, K, alpha) > 0) lo = mid; else hi = mid;
        if (++it > 200) { *err = 1; return r_lj; }
    }
    return fmin((lo + hi) / 2, r_lj);
}

// One CTA per chunk of BOUND_CHUNK (site, atom) pairs of one framework (blockIdx.y), so that a
// large framework's root searches spread over the GPU; the host adds the chunks' partial sums in
// chunk order.
__global__ void __launch_bounds__(256) k_hardcore_bound(BoundArgs g) {
    __shared__ double s_red[256];
    const int32_t fw = blockIdx.y, ch = blockIdx.x;
    const int32_t a0 = g.atom_offsets[fw], a1 = g.atom_offsets[fw + 1];
    const double alpha = g.alphas[fw];
    const int64_t npair = int64_t(a1 - a0) * g.N;
    const int64_t p0 = int64_t(ch) * BOUND_CHUNK, p1 = min(npair, p0 + BOUND_CHUNK);
    if (p0 >= npair) {
        if (threadIdx.x == 0) g.out[int64_t(fw) * g.nchunk + ch] = 0.0;
        return;
    }
    double acc = 0.0;
    int32_t lerr = 0;
    for (int64_t p = p0 + threadIdx.x; p < p1; p += blockDim.x) {
        const int32_t a = int32_t(p / (a1 - a0)), j = a0 + int32_t(p % (a1 - a0));
        const int32_t t = g.types[j];
        const double e = g.site_eps[a * g.nt + t], s = g.site_sig[a * g.nt + t];
        const double K = KE * g.gq[a] * g.charges[j];
        double term = e;
        if (K < 0) {
            if (e == 0) term = __longlong_as_double(0x7ff0000000000000LL);
            else {
                const double r0 = bound_find_r0(s, e, K, alpha, g.r_lj, &lerr);
                term = e + fabs(K) * erfc(alpha * r0) / r0;
            }
        }
        acc += term;
    }
    if (lerr) atomicExch(g.err, 1);
    s_red[threadIdx.x] = acc;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (int(threadIdx.x) < w) s_red[threadIdx.x] += s_red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) g.out[int64_t(fw) * g.nchunk + ch] = s_red[0];
}

}  // namespace pa
