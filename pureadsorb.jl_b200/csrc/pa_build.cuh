// Batch construction on the device: the k-vector enumeration with its prefactors
// (src/ewald.jl:36-39, 142-157), the per-(site, type) most negative charge product kmin
// (src/reject.jl:134-145), the stable cell sort of the phase-0 cell list (src/cell.jl:96-118), and
// the rejection radii of one widom call (find_rho2, src/reject.jl:168-209). Every FP64 operation
// is individually rounded (St<double>) in the order the host builders use, so the device tables
// equal the host's bit for bit (the k prefactor's exp excepted: CUDA's and the host's exp may
// differ in the last bit). Included by pa_kernels.cuh after its helpers.
#pragma once

// The squared rejection radius: the first root of LJ(r) - |kmin|/r = margin scanning up from
// r -> 0 (bracket by doubling from sigma, then halving, then bisection to 4 eps hi), clamped to
// the LJ cutoff; 0 for an infinite margin or a zero epsilon; -1 when a search exceeds its
// iteration cap (200, the reference's MAX_BISECT_ITERS). Host and device run this same sequence.
PA_HD double lj4_s(double r2, double s, double e) {
    typedef St<double> D;
    double x = D::div(D::mul(s, s), r2);
    x = D::mul(D::mul(x, x), x);
    return D::mul(D::mul(4.0, e), D::sub(D::mul(x, x), x));
}
PA_HD double rho2_search(double s, double e, double kmin, double margin, double r_lj) {
    typedef St<double> D;
    if (isinf(margin) || e == 0) return 0;
    const double ak = kmin < 0 ? -kmin : kmin;
    const auto f = [&](double r) { return D::sub(D::sub(lj4_s(D::mul(r, r), s, e), D::div(ak, r)), margin); };
    const int cap = 200;
    const double eps = 2.220446049250313e-16;
    double hi = s;
    int it = 0;
    while (f(hi) >= 0) { hi = D::mul(hi, 2.0); if (++it > cap) return -1; }
    double lo = hi;
    it = 0;
    while (f(lo) < 0) { lo = D::div(lo, 2.0); if (++it > cap) return -1; }
    it = 0;
    while (D::sub(hi, lo) > D::mul(D::mul(4.0, eps), hi)) {
        const double mid = D::div(D::add(lo, hi), 2.0);
        if (f(mid) > 0) lo = mid; else hi = mid;
        if (++it > cap) return -1;
    }
    double r = D::div(D::add(lo, hi), 2.0);
    r = r < r_lj ? r : r_lj;
    return D::mul(r, r);
}

// One thread per (system, guest site, host type): rho2[(s N + a) nt + t] from the system's margin,
// the (site, type) sigma and epsilon and the framework's kmin.
__global__ void __launch_bounds__(256) k_rho2(const double* sig, const double* eps, const double* kmin,
                                              const double* margin, const int32_t* framework_of, int32_t nsys,
                                              int32_t N, int32_t nt, double r_lj, double* rho2) {
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= int64_t(nsys) * N * nt) return;
    const int32_t t = int32_t(i % nt), a = int32_t((i / nt) % N), s = int32_t(i / (int64_t(N) * nt));
    const int32_t fw = framework_of[s];
    rho2[i] = rho2_search(sig[a * nt + t], eps[a * nt + t], kmin[(int64_t(fw) * N + a) * nt + t], margin[s], r_lj);
}

// The half-space k-vectors of one cell within kmax, in the enumeration order n1 = 0..n[0],
// n2 = -n[1]..n[1], n3 = -n[2]..n[2] (n3 fastest), (0, 0, 0) left out: one CTA of 1024 threads
// takes the candidates in that order 1024 at a time and places the kept ones by an exclusive scan.
// k = (n1 B[:,0] + n2 B[:,1]) + n3 B[:,2] (B row-major 3x3), |k| = sqrt((kx^2 + ky^2) + kz^2),
// weight 1 for n1 = 0 and 2 otherwise, kpref = w ((2 pi / V) exp(-k^2 / (4 alpha^2)) / k^2) with
// c2piv = 2 pi / V and four_a2 = 4 alpha^2 as the host forms them.
struct KvecArgs {
    double B[9];
    int32_t n[3];
    double kmax, c2piv, four_a2;
    double* ks;        // 3 per kept k-vector
    double* w;
    double* kpref;
    int32_t* coeffs;   // 3 per kept k-vector
    int32_t* count;
};
__global__ void __launch_bounds__(1024) k_kvectors(KvecArgs g) {
    typedef St<double> D;
    __shared__ int32_t s_warp[32];
    const int64_t n2s = 2 * int64_t(g.n[1]) + 1, n3s = 2 * int64_t(g.n[2]) + 1;
    const int64_t M = (int64_t(g.n[0]) + 1) * n2s * n3s;
    int32_t base = 0;
    for (int64_t m0 = 0; m0 < M; m0 += blockDim.x) {
        const int64_t m = m0 + threadIdx.x;
        int32_t c[3] = {0, 0, 0};
        double k[3] = {0, 0, 0}, k2 = 0;
        bool keep = false;
        if (m < M) {
            c[0] = int32_t(m / (n2s * n3s));
            c[1] = int32_t((m / n3s) % n2s) - g.n[1];
            c[2] = int32_t(m % n3s) - g.n[2];
            if (c[0] != 0 || c[1] != 0 || c[2] != 0) {
                const double f0 = double(c[0]), f1 = double(c[1]), f2 = double(c[2]);
#pragma unroll
                for (int r = 0; r < 3; ++r)
                    k[r] = D::add(D::add(D::mul(f0, g.B[3 * r]), D::mul(f1, g.B[3 * r + 1])), D::mul(f2, g.B[3 * r + 2]));
                k2 = D::add(D::add(D::mul(k[0], k[0]), D::mul(k[1], k[1])), D::mul(k[2], k[2]));
                keep = D::sqrt(k2) <= g.kmax;
            }
        }
        int32_t total = 0;
        const int32_t pos = base + block_excl_scan(keep ? 1 : 0, s_warp, &total);
        if (keep) {
            const double w = c[0] == 0 ? 1.0 : 2.0;
            for (int r = 0; r < 3; ++r) { g.ks[3 * int64_t(pos) + r] = k[r]; g.coeffs[3 * int64_t(pos) + r] = c[r]; }
            g.w[pos] = w;
            g.kpref[pos] = D::mul(w, D::div(D::mul(g.c2piv, exp(D::div(-k2, g.four_a2))), k2));
        }
        base += total;
    }
    if (threadIdx.x == 0) *g.count = base;
}

// kmin of one framework: for every atom h and guest site a, K = (KE q_a) q_h; the most negative K
// per (a, type of h), or 0. Negative doubles order like the reverse of their bit patterns, so the
// minimum is an atomic maximum of the bits of the negative candidates over a zeroed table (exact,
// independent of order).
__global__ void __launch_bounds__(256) k_kmin(const double* gq, int32_t N, const int32_t* types, const double* q,
                                              int64_t natoms, int32_t nt, unsigned long long* kmin_bits) {
    typedef St<double> D;
    for (int64_t h = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; h < natoms; h += int64_t(gridDim.x) * blockDim.x) {
        const int32_t t = types[h] - 1;
        for (int32_t a = 0; a < N; ++a) {
            const double K = D::mul(D::mul(KE, gq[a]), q[h]);
            if (K < 0) atomicMax(&kmin_bits[a * nt + t], static_cast<unsigned long long>(__double_as_longlong(K)));
        }
    }
}

// Cell sort of one framework (stable counting sort by the linear cell index of each atom's wrapped
// fractional coordinates): k_cell_count gives every atom its cell and counts the cells;
// k_cell_offsets (one CTA) scans the counts into the offsets; k_cell_place (one warp) walks the
// atoms in order, 32 at a time, and places each at its cell's cursor plus its rank among the lanes
// of the same cell (__match_any_sync), so atoms of one cell keep their order.
__global__ void __launch_bounds__(256) k_cell_count(const double* frac, int64_t natoms, int32_t n0, int32_t n1,
                                                    int32_t n2, int32_t* cellidx, int32_t* counts) {
    typedef St<double> D;
    const int64_t a = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (a >= natoms) return;
    const int32_t n[3] = {n0, n1, n2};
    int32_t c[3];
#pragma unroll
    for (int r = 0; r < 3; ++r) {
        const double f = frac[3 * a + r];
        const double fw = D::sub(f, D::floor(f));
        int32_t ci = int32_t(D::floor(D::mul(fw, double(n[r]))));
        c[r] = ci < n[r] - 1 ? ci : n[r] - 1;
    }
    const int32_t lin = c[0] + n0 * (c[1] + n1 * c[2]);
    cellidx[a] = lin;
    atomicAdd(&counts[lin], 1);
}
__global__ void __launch_bounds__(1024) k_cell_offsets(const int32_t* counts, int32_t ncell, int32_t* offsets,
                                                       int32_t* cursor) {
    __shared__ int32_t s_warp[32];
    int32_t base = 0;
    for (int32_t c0 = 0; c0 < ncell; c0 += blockDim.x) {
        const int32_t c = c0 + threadIdx.x;
        const int32_t v = c < ncell ? counts[c] : 0;
        int32_t total = 0;
        const int32_t e = base + block_excl_scan(v, s_warp, &total);
        if (c < ncell) { offsets[c] = e; cursor[c] = e; }
        base += total;
    }
    if (threadIdx.x == 0) offsets[ncell] = base;
}
__global__ void __launch_bounds__(32) k_cell_place(const int32_t* cellidx, int64_t natoms, int32_t* cursor,
                                                   int64_t* perm) {
    const int lane = threadIdx.x;
    const unsigned lt = (1u << lane) - 1u;
    for (int64_t a0 = 0; a0 < natoms; a0 += 32) {
        const int64_t a = a0 + lane;
        const unsigned act = __ballot_sync(0xffffffffu, a < natoms);
        if (a < natoms) {
            const int32_t c = cellidx[a];
            const unsigned peers = __match_any_sync(act, c);
            const int32_t base = cursor[c];
            perm[base + __popc(peers & lt)] = a;
            __syncwarp(act);
            if ((peers & lt) == 0) cursor[c] = base + __popc(peers);
        }
        __syncwarp();
    }
}
