// The FP32 insertion energy (src/energy.jl:42-82 restated for spatial bins), in two kernels.
//
// k_energy32: the real-space pair sum. A work item is one (surviving insertion, guest site);
// items are binned and sorted by the position of their own site, so the 32 lanes of a warp tile
// are 32 sites lying within a small region of one spatial bin (with whole insertions per lane,
// the sites of a tile would spread over the bin plus the guest's extent, and the cutoff sphere of
// some lane would cut through nearly every staged list entry). Persistent CTAs of PA_WARPS32
// independent warps; each warp streams its bin's imaged neighbour list (positions relative to the
// bin centre, charge, type) through its own two shared-memory stages with cp.async.bulk copies
// completing on its own mbarriers, so warps never wait for one another. FP32 Lennard-Jones +
// screened Coulomb inside the cutoffs, each pair's term added exactly to an FP64 sum per item;
// pairs closer than the near radius, or at a cutoff's rounding band, are marked during the walk
// and evaluated in FP64 after each chunk.
//
// k_recip: the reciprocal cross term per insertion, over tiles of 32 insertions of one bin:
// per-bin FP64 phase factors, then cos/sin recurrences along k-vector rows per lane.
//
// k_combine (pa_kernels.cuh) adds the site sums, the reciprocal term and the constant offset in a
// fixed order. Included by pa_kernels.cuh after its helpers.
#pragma once

#define PA_WARPS32 4
#define PA_TILE32 32
#define PA_CHUNK32 128
#define PA_KCHUNK32 64
#define PA_CTAS_PER_SM32 8

__device__ __forceinline__ float rsqrt_ftz(float x) {
    float r;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ float ex2_ftz(float x) {
    float r;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// 1/sqrt(x) in FP64, x > 0 and normal: the hardware approximation (rsqrt.approx.ftz.f64, measured
// within 9.3e-7 relative on [1e-2, 1e4] on the B200) refined by one step of Newton's iteration
// y <- y (3/2 - (x/2) y^2), which squares the relative error: within 1.3e-12 (measured), about
// 1e-11 eV on the largest near-pair terms.
__device__ __forceinline__ double rsqrt64(double x) {
    double y;
    asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
    const double h = 0.5 * x;
    return y * fma(-h * y, y, 1.5);
}

// S(u) = erf(sqrt u)/sqrt u on 0 <= u <= PA_ERFS64_UMAX from the PA_ERFS64 polynomial (Horner).
__device__ __forceinline__ double erfs64(double u) {
    const double c[PA_NERFS64] = PA_ERFS64_INIT;
    double p = c[PA_NERFS64 - 1];
#pragma unroll
    for (int k = PA_NERFS64 - 2; k >= 0; --k) p = fma(p, u, c[k]);
    return p;
}

// erfc(alpha r) / r in FP64 from r^2 and 1/r: 1/r - alpha S(alpha^2 r^2) for alpha r <= 2 (S of
// degree 13, |error| below 2.4e-13 there); CUDA's double erfc beyond that.
__device__ __forceinline__ double screened64(double r2, double ri, double alpha) {
    const double u = (alpha * alpha) * r2;
    if (u <= PA_ERFS64_UMAX) return fma(-alpha, erfs64(u), ri);
    return erfc(alpha * (r2 * ri)) * ri;
}

// Fetches the next tile of a persistent warp: its bin and the [lo, hi) range of sorted entries.
__device__ __forceinline__ bool next_tile(const Work& w, int32_t nbins, int32_t lane, int32_t& bin, int32_t& lo,
                                          int32_t& hi) {
    const unsigned FULL = 0xffffffffu;
    const int32_t total_tiles = w.counters[1];
    int32_t t = 0;
    if (lane == 0) {
        t = atomicAdd(&w.counters[0], 1);
        if (t < total_tiles) {
            bin = find_bin(w.tile_start, nbins, t);
            lo = w.bin_start[bin] + (t - w.tile_start[bin]) * PA_TILE32;
            hi = min(lo + PA_TILE32, w.bin_start[bin + 1]);
        }
    }
    t = __shfl_sync(FULL, t, 0);
    if (t >= total_tiles) return false;
    bin = __shfl_sync(FULL, bin, 0); lo = __shfl_sync(FULL, lo, 0); hi = __shfl_sync(FULL, hi, 0);
    return true;
}

// Centre of bin `bin` of framework fw in fractional coordinates.
__device__ __forceinline__ void bin_centre(const DevBatch<float>& b, int32_t fw, int32_t bin, float& cx, float& cy,
                                           float& cz) {
    const int32_t* nb = b.bin_dims + 3 * fw;
    const int32_t lb = bin - b.bin_base[fw];
    const int32_t bx = lb % nb[0], by = (lb / nb[0]) % nb[1], bz = lb / (nb[0] * nb[1]);
    cx = __fdiv_rn(float(bx) + 0.5f, float(nb[0]));
    cy = __fdiv_rn(float(by) + 0.5f, float(nb[1]));
    cz = __fdiv_rn(float(bz) + 0.5f, float(nb[2]));
}

// One pair in FP64 from the FP64 list entry e (xyzq64) and the item's FP64 site (relative to the
// bin centre): the cutoff tests against rl2 and re2, LJ (lj = (sigma^2, 4 eps) of the site and the
// entry's type) and the screened Coulomb term (skq = KE times the site charge), added to enear; PQ
// also adds the pair's x^6(x^6-1) and x^6(2x^6-1) (x = sigma/r) to the run sums.
template <bool PQ>
__device__ __forceinline__ void pair64(const double4* xyzq64, double rl2, double re2, int32_t e, double px, double py,
                                       double pz, double2 lj, double skq, double alpha, bool charged, double& enear,
                                       float& sp, float& sq) {
    const double4 e64 = xyzq64[e];
    const double ex = px - e64.x, ey = py - e64.y, ez = pz - e64.z;
    const double r2d = fma(ez, ez, fma(ey, ey, ex * ex));
    const double rid = rsqrt64(r2d);
    double en = 0.0;
    if (r2d < rl2) {
        const double x = lj.x * (rid * rid);
        const double x3 = x * x * x;
        const double u = x3 * x3 - x3;
        en = lj.y * u;
        if (PQ) { sp += float(u); sq += float(fma(x3, x3, u)); }
    }
    if (charged && r2d < re2) en = fma(skq * e64.w, screened64(r2d, rid, alpha), en);
    enear += en;
}

// EQCUT: the LJ and Ewald cutoffs are equal, so one test selects both terms. PQ: also store each
// item's LJ sums per type run (w.item_pq) for the adjoint. HP: the FP32 screened Coulomb term in
// the exp-free form (b.hpoly; every FP32 pair lies beyond the near radius), otherwise as
// exp(-z^2) P(t), t = 2/(2 + z), z = alpha r.
template <int NS, bool EQCUT, bool PQ, bool HP>
__global__ void __launch_bounds__(32 * PA_WARPS32, PA_CTAS_PER_SM32) k_energy32(DevBatch<float> b, CallArgs ca, Work w) {
    __shared__ __align__(128) float4 s_xyzq[PA_WARPS32][2][PA_CHUNK32];
    __shared__ __align__(8) uint64_t s_bar[PA_WARPS32][2];
    __shared__ float4 s_site[NS];    // body-frame site offsets, and the site charge times KE
    __shared__ double4 s_site64[NS]; // the same in FP64 (the FP64 pairs)
    __shared__ double2 s_p64[PA_WARPS32][32][2];  // each lane's site in FP64 (x, y | z, -), FP64 pairs
    __shared__ uint32_t s_mk[PA_WARPS32][PA_CHUNK32 / 32][32];  // per lane: the chunk's FP64 entries (bits)
    // the (site, type) LJ tables stay in global memory (read at type-run boundaries and per FP64
    // pair, through L1): in shared memory a batch of many host types would cost CTAs per SM
    const int tid = threadIdx.x, lane = tid & 31, wp = tid >> 5;
    const int nt = b.ntypes;
    if (tid < NS) {
        s_site[tid] = make_float4(b.gsite[3 * tid], b.gsite[3 * tid + 1], b.gsite[3 * tid + 2],
                                  float(KE * double(b.gq[tid])));
        s_site64[tid] = make_double4(b.gsite64[3 * tid], b.gsite64[3 * tid + 1], b.gsite64[3 * tid + 2],
                                     KE * b.gq64[tid]);
    }
    if (lane == 0) { mbar_init(&s_bar[wp][0], 1); mbar_init(&s_bar[wp][1], 1); mbar_fence_init(); }
    __syncthreads();  // the only CTA-wide barrier: tables and barriers are ready
    float4(*xyzq)[PA_CHUNK32] = s_xyzq[wp];
    uint64_t* bar = s_bar[wp];
    uint32_t gchunk = 0;  // chunks this warp has consumed (selects stage and parity)
    const bool charged = b.has_charge != 0;
    const unsigned FULL = 0xffffffffu;
    int32_t bin = 0, lo = 0, hi = 0;
    while (next_tile(w, b.nbins, lane, bin, lo, hi)) {
        const int32_t fw = b.bin_fw[bin];
        const int32_t l0 = b.list_offsets[bin], l1 = b.list_offsets[bin + 1];
        const int32_t nch = (l1 - l0 + PA_CHUNK32 - 1) / PA_CHUNK32;
        if (lane == 0) {  // first two chunks in flight (the warp finished reading both stages)
            for (int c = 0; c < 2 && c < nch; ++c) {
                const uint32_t st = (gchunk + c) & 1;
                const int32_t e0 = l0 + c * PA_CHUNK32, n = min(PA_CHUNK32, l1 - e0);
                fence_proxy_async_smem();
                mbar_arrive_expect_tx(&bar[st], uint32_t(n) * 16u);
                bulk_g2s(xyzq[st], b.list_xyzq + e0, uint32_t(n) * 16u, &bar[st]);
            }
        }
        const bool active = lo + lane < hi;
        const int32_t it = active ? w.sorted[lo + lane] : 0;
        const int32_t li = it / NS, as = it - li * NS;  // insertion and site of this lane's item
        float cx, cy, cz;
        bin_centre(b, fw, bin, cx, cy, cz);
        const float4 pa = active ? w.pose_a[li] : make_float4(cx, cy, cz, 0.f);
        const float4 pq = active ? w.pose_b[li] : make_float4(0.f, 0.f, 0.f, 1.f);
        const float* iA = b.invcells + 9 * fw;
        // the site relative to the bin centre, A (rp + shift - c) + g, in FP64 (the near pairs'
        // geometry) and rounded once to FP32 for the rest; the lattice shift is the binning's own
        float px, py, pz;
        {
            const float q[4] = {pq.x, pq.y, pq.z, pq.w};
            const float4 gs = s_site[as];
            const float gb[3] = {gs.x, gs.y, gs.z};
            float g[3], fs[3], sh[3];
            rotate_s(q, gb, g);
            const float rp[3] = {pa.x, pa.y, pa.z};
            site_frac32(rp, g, iA, fs, sh);
            // rp + shift - c is exact in FP64 (all three are FP32 values)
            const double d0 = (double(pa.x) + double(sh[0])) - double(cx);
            const double d1 = (double(pa.y) + double(sh[1])) - double(cy);
            const double d2 = (double(pa.z) + double(sh[2])) - double(cz);
            const double qd[4] = {double(pq.x), double(pq.y), double(pq.z), double(pq.w)};
            const double4 gs64 = s_site64[as];
            const double gb64[3] = {gs64.x, gs64.y, gs64.z};
            double g64[3];
            rotate_s(qd, gb64, g64);
            const double* A64 = b.cells64 + 9 * fw;
            const double p64x = fma(A64[6], d2, fma(A64[3], d1, A64[0] * d0)) + g64[0];
            const double p64y = fma(A64[7], d2, fma(A64[4], d1, A64[1] * d0)) + g64[1];
            const double p64z = fma(A64[8], d2, fma(A64[5], d1, A64[2] * d0)) + g64[2];
            s_p64[wp][lane][0] = make_double2(p64x, p64y);
            s_p64[wp][lane][1] = make_double2(p64z, 0.0);
            px = float(p64x); py = float(p64y); pz = float(p64z);
        }
        const float qk = s_site[as].w;
        const float rl2 = b.rl2, re2 = b.re2, alpha = float(b.alphas[fw]);
        // FP32 distances below rc2 enter the pair block; of those, the near pairs and the ones in a
        // cutoff's rounding band are evaluated in FP64
        const float rc2 = fmaxf(b.rl2_hi, b.re2_hi), rn2 = b.rn2;
        const float rl2lo = b.rl2_lo, rl2hi = b.rl2_hi, re2lo = b.re2_lo, re2hi = b.re2_hi;
        double enear = 0.0;  // the FP64 pairs' sum
        const float NLOG2E = -1.4426950408889634f;
        const float a2n = (alpha * alpha) * NLOG2E;  // exp(-alpha^2 r^2) = 2^(r^2 a2n)
        const float halpha = 0.5f * alpha;
        double eacc = 0.0;  // the FP32 pairs' terms, each added exactly to an FP64 sum
        // LJ parameters of the current host type for this lane's site: list entries come in runs of
        // one type (the bin's run table), the same for every lane, so the loop runs uniformly from
        // one run boundary to the next and reloads them there
        const int2* runs = b.list_runs + int64_t(bin) * b.runs_per_bin;
        int32_t ri = 0, rnext = runs[1].x, ty = runs[0].y;
        float sg = __ldg(b.sig2 + as * nt + ty), ep = __ldg(b.eps4 + as * nt + ty);
        // without the adjoint sums: 4 eps ((sigma/r)^12 - (sigma/r)^6) = r^-6 (ljA r^-6 - ljB),
        // ljA = 4 eps sigma^12, ljB = 4 eps sigma^6, one multiplication fewer per pair
        float ljB = ep * (sg * sg * sg), ljA = ljB * (sg * sg * sg);
        float sp = 0.f, sq = 0.f;  // PQ: the current run's Σ x(x-1) and Σ x(2x-1)
        float2* runsums = PQ ? w.item_pq + int64_t(lo + lane) * b.runs_per_bin : nullptr;
        // tmo_at: chunk whose copy did not arrive in time (-1: none); after it no copies are issued
        // and only the chunk already in flight is still waited for
        int32_t tmo_at = -1;
        for (int32_t c = 0; c < nch; ++c) {
            const uint32_t g = gchunk + c, st = g & 1, par = (g >> 1) & 1;
            if (!(tmo_at < 0 || c == tmo_at + 1)) break;
            const bool late = __any_sync(FULL, !mbar_wait_bounded(&bar[st], par));
            if (late && tmo_at < 0) tmo_at = c;
            const int32_t n = min(PA_CHUNK32, l1 - (l0 + c * PA_CHUNK32));
            if (tmo_at < 0) {
                const int32_t base = l0 + c * PA_CHUNK32;
                // the chunk's entries this lane evaluates in FP64 afterwards (bit j % 32 of word j / 32)
#pragma unroll
                for (int q = 0; q < PA_CHUNK32 / 32; ++q) s_mk[wp][q][lane] = 0u;
                int32_t j = 0;
                for (;;) {
                    const int32_t jend = min(n, rnext - base);
#pragma unroll 4
                    for (; j < jend; ++j) {
                        const float4 at = xyzq[st][j];
                        const float dx = px - at.x, dy = py - at.y, dz = pz - at.z;
                        const float r2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
                        if (r2 < rc2) {
                            // (with equal cutoffs r2 < rc2 = rl2hi already holds)
                            if (r2 < rn2 || r2 > rl2lo && (EQCUT || r2 < rl2hi) || (!EQCUT && r2 > re2lo && r2 < re2hi)) {
                                // a near pair, or one within a cutoff's rounding band: evaluated in
                                // FP64 (the adjoint's form here, every other form after the chunk)
                                if (PQ) {
                                    const double2 pxy = s_p64[wp][lane][0], pzz = s_p64[wp][lane][1];
                                    pair64<true>(b.list_xyzq64, b.rl2_64, b.re2_64, base + j, pxy.x, pxy.y, pzz.x,
                                                 make_double2(b.sig2_64[as * nt + ty], b.eps4_64[as * nt + ty]),
                                                 s_site64[as].w, b.alphas[fw], charged, enear, sp, sq);
                                } else {
                                    s_mk[wp][j >> 5][lane] |= 1u << (j & 31);
                                }
                                continue;
                            }
                            float e = 0.f;
                            if (HP && charged) {
                                // u = 1/r^2 serves both terms: LJ, and exp(-alpha^2 r^2) u H(u); the
                                // hardware reciprocal (about 1 ulp) without a Newton step: every pair
                                // here lies beyond the near radius, where its terms are small
                                float ri2;
                                asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(ri2) : "f"(r2));
                                if (EQCUT || r2 < rl2) {
                                    if (PQ) {
                                        const float x = sg * ri2;
                                        const float x3 = x * x * x;
                                        const float u = x3 * x3 - x3;
                                        e = ep * u;
                                        sp += u;
                                        sq = fmaf(x3, x3, sq + u);
                                    } else {
                                        const float ri6 = ri2 * ri2 * ri2;
                                        e = ri6 * fmaf(ljA, ri6, -ljB);
                                    }
                                }
                                if (EQCUT || r2 < re2) {
                                    const float x = fmaf(ri2, b.hk1, b.hk0);
                                    float p = b.hc[PA_NHP - 1];
#pragma unroll
                                    for (int k = PA_NHP - 2; k >= 0; --k) p = fmaf(p, x, b.hc[k]);
                                    e = fmaf(qk * at.w, p * ex2_ftz(r2 * a2n) * ri2, e);
                                }
                            } else if (charged) {
                                // one reciprocal square root serves both terms: 1/r^2 = (1/r)^2
                                float ri = rsqrt_ftz(r2);
                                ri = ri * fmaf(-0.5f * r2 * ri, ri, 1.5f);
                                if (EQCUT || r2 < rl2) {
                                    if (PQ) {
                                        const float x = sg * (ri * ri);
                                        const float x3 = x * x * x;
                                        const float u = x3 * x3 - x3;
                                        e = ep * u;
                                        sp += u;
                                        sq = fmaf(x3, x3, sq + u);
                                    } else {
                                        const float ri2 = ri * ri;
                                        const float ri6 = ri2 * ri2 * ri2;
                                        e = ri6 * fmaf(ljA, ri6, -ljB);
                                    }
                                }
                                if (EQCUT || r2 < re2) {
                                    // t = 1 / (1 + z/2), z = alpha r, with alpha/2 exact
                                    const float tt = rcp_nr(fmaf(halpha, r2 * ri, 1.0f));
                                    const float cf[PA_NERFC32] = PA_ERFC32_INIT;
                                    float p = cf[PA_NERFC32 - 1];
#pragma unroll
                                    for (int k = PA_NERFC32 - 2; k >= 0; --k) p = fmaf(p, tt, cf[k]);
                                    e = fmaf(qk * at.w, p * ex2_ftz(r2 * a2n) * ri, e);
                                }
                            } else if (EQCUT || r2 < rl2) {
                                if (PQ) {
                                    const float x = sg * rcp_nr(r2);
                                    const float x3 = x * x * x;
                                    const float u = x3 * x3 - x3;
                                    e = ep * u;
                                    sp += u;
                                    sq = fmaf(x3, x3, sq + u);
                                } else {
                                    const float ri2 = rcp_nr(r2);
                                    const float ri6 = ri2 * ri2 * ri2;
                                    e = ri6 * fmaf(ljA, ri6, -ljB);
                                }
                            }
                            eacc += double(e);
                        }
                    }
                    if (j >= n) break;
                    // entry j starts the next type run
                    if (PQ) {
                        if (active) runsums[ri] = make_float2(sp, sq);
                        sp = 0.f; sq = 0.f;
                    }
                    ++ri;
                    ty = runs[ri].y;
                    rnext = runs[ri + 1].x;
                    sg = __ldg(b.sig2 + as * nt + ty);
                    ep = __ldg(b.eps4 + as * nt + ty);
                    ljB = ep * (sg * sg * sg);
                    ljA = ljB * (sg * sg * sg);
                }
                if (!PQ) {
                    // the marked pairs in FP64, lanes in step: each lane takes its next marked entry
                    // of the chunk (in entry order), so the warp takes as many steps as the lane
                    // with the most marks
                    const double2 pxy = s_p64[wp][lane][0], pzz = s_p64[wp][lane][1];
                    const double skq = s_site64[as].w, alpha64 = b.alphas[fw];
                    const double* sig2 = b.sig2_64 + as * nt;
                    const double* eps4 = b.eps4_64 + as * nt;
                    float dsp = 0.f, dsq = 0.f;
                    int32_t left = 0;
#pragma unroll
                    for (int q = 0; q < PA_CHUNK32 / 32; ++q) left += __popc(s_mk[wp][q][lane]);
                    int32_t q = 0;
                    uint32_t mq = s_mk[wp][0][lane];
                    while (__any_sync(FULL, left > 0)) {
                        if (left > 0) {
                            while (mq == 0) mq = s_mk[wp][++q][lane];  // a mark is left: ends by word 3
                            const int32_t e = base + q * 32 + __ffs(mq) - 1;
                            mq &= mq - 1;
                            --left;
                            const int32_t te = b.list_type[e];
                            pair64<false>(b.list_xyzq64, b.rl2_64, b.re2_64, e, pxy.x, pxy.y, pzz.x,
                                          make_double2(sig2[te], eps4[te]), skq, alpha64, charged, enear, dsp, dsq);
                        }
                    }
                }
            }
            __syncwarp();  // the warp is done with stage st
            if (lane == 0 && tmo_at < 0 && c + 2 < nch) {
                const int32_t e0 = l0 + (c + 2) * PA_CHUNK32, nn = min(PA_CHUNK32, l1 - e0);
                fence_proxy_async_smem();
                mbar_arrive_expect_tx(&bar[st], uint32_t(nn) * 16u);
                bulk_g2s(xyzq[st], b.list_xyzq + e0, uint32_t(nn) * 16u, &bar[st]);
            }
        }
        gchunk += uint32_t(nch);
        if (tmo_at >= 0) {
            if (lane == 0) atomicExch(&w.counters[2], 1);
            return;
        }
        if (PQ && active && nch > 0) runsums[ri] = make_float2(sp, sq);  // the last run
        if (active) w.dUs[it] = eacc + enear;
    }
}

// Reciprocal term per insertion: E_lr = Σ_k Re(B_k G_k), B_k = 2 kpref conj(S_k) e^{2 pi i n.c}
// built in FP64 per bin, G_k = Σ_s q_s e^{2 pi i n.d_s} with d_s the site's fractional offset from
// the bin centre. Along a row of equal (n1, n2), n3 advances by the framework's step, so
// e^{2 pi i n.d_s} is carried by one complex multiplication and evaluated directly only at row
// starts. Tiles of 32 insertions of one bin (insertion order, not site order); writes KE E_lr.
//
// Three forms (RMODE): 0 every k-vector in FP32 (row starts from the hardware sine and cosine of the
// phase reduced to half a turn, FP32 recurrences, rows compensated); 1 every k-vector in FP64
// (sincospi row starts, FP64 recurrences and sums); 2 the batch's split tables: the k-vectors of
// small |k| (the large terms) in FP64, the rest in FP32, chosen at upload so that the FP32 part's
// rounding stays below a few 1e-9 eV.

// The FP64 rows of one table [k0, k1): Σ_k Re(B_k G_k) in FP64.
template <int NS>
__device__ __forceinline__ double rows64(const float4* kcoef, const double* kS2, int32_t k0, int32_t k1,
                                         const double* dfr, const double* stc, const double* sts, const double* gq,
                                         float cx, float cy, float cz, int lane, double2* sB, float4* sKc) {
    double cr[NS], ci[NS];
#pragma unroll
    for (int s = 0; s < NS; ++s) { cr[s] = 1.0; ci[s] = 0.0; }
    double acc = 0.0;
    for (int32_t kb = k0; kb < k1; kb += PA_KCHUNK32) {
        const int32_t kn = min(PA_KCHUNK32, k1 - kb);
        for (int32_t x = lane; x < kn; x += 32) {
            const int32_t kk = kb + x;
            const float4 kc = kcoef[kk];
            sKc[x] = kc;
            double ph = double(kc.x) * double(cx) + double(kc.y) * double(cy) + double(kc.z) * double(cz);
            ph -= rint(ph);
            double sn, cs;
            sincospi(2.0 * ph, &sn, &cs);
            const double Sr = kS2[2 * kk], Si = kS2[2 * kk + 1];
            sB[x] = make_double2(Sr * cs + Si * sn, Sr * sn - Si * cs);
        }
        __syncwarp();
        for (int32_t x = 0; x < kn; ++x) {
            const float4 kc = sKc[x];
            if (kc.w == 0.f) {  // row start: direct evaluation
#pragma unroll
                for (int s = 0; s < NS; ++s) {
                    double ph = fma(double(kc.z), dfr[3 * s + 2], fma(double(kc.y), dfr[3 * s + 1], double(kc.x) * dfr[3 * s]));
                    ph -= rint(ph);
                    sincospi(2.0 * ph, &ci[s], &cr[s]);
                }
            } else {  // next k-vector of the row
#pragma unroll
                for (int s = 0; s < NS; ++s) {
                    const double r = fma(cr[s], stc[s], -ci[s] * sts[s]);
                    ci[s] = fma(cr[s], sts[s], ci[s] * stc[s]);
                    cr[s] = r;
                }
            }
            double gr = 0.0, gi = 0.0;
#pragma unroll
            for (int s = 0; s < NS; ++s) { gr = fma(gq[s], cr[s], gr); gi = fma(gq[s], ci[s], gi); }
            const double2 B = sB[x];
            acc = fma(B.x, gr, fma(-B.y, gi, acc));
        }
        __syncwarp();
    }
    return acc;
}

// The FP32 rows of one table [k0, k1): Σ_k Re(B_k G_k) as a compensated sum of row sums (acc, cacc).
template <int NS>
__device__ __forceinline__ void rows32(const float4* kcoef, const double* kS2, int32_t k0, int32_t k1,
                                       const float* dfr, const float* stc, const float* sts, const float* gqs,
                                       float cx, float cy, float cz, int lane, float2* sB, float4* sKc, float& acc,
                                       float& cacc) {
    float cr[NS], ci[NS];
#pragma unroll
    for (int s = 0; s < NS; ++s) { cr[s] = 1.f; ci[s] = 0.f; }
    // the terms of one k-vector row (a few) are summed plainly, rows then compensated
    float row = 0.f;
    for (int32_t kb = k0; kb < k1; kb += PA_KCHUNK32) {
        const int32_t kn = min(PA_KCHUNK32, k1 - kb);
        for (int32_t x = lane; x < kn; x += 32) {
            const int32_t kk = kb + x;
            const float4 kc = kcoef[kk];
            sKc[x] = kc;
            double ph = double(kc.x) * double(cx) + double(kc.y) * double(cy) + double(kc.z) * double(cz);
            ph -= rint(ph);
            double sn, cs;
            sincospi(2.0 * ph, &sn, &cs);
            const double Sr = kS2[2 * kk], Si = kS2[2 * kk + 1];
            // conj(S) e^{i phi} = (Sr cs + Si sn) + i (Sr sn - Si cs)
            sB[x] = make_float2(float(Sr * cs + Si * sn), float(Sr * sn - Si * cs));
        }
        __syncwarp();
        for (int32_t x = 0; x < kn; ++x) {
            const float4 kc = sKc[x];
            if (kc.w == 0.f) {  // row start: direct evaluation; the finished row enters the sum
                kahan_add(acc, cacc, row);
                row = 0.f;
#pragma unroll
                for (int s = 0; s < NS; ++s) {
                    // the phase reduced to [-1/2, 1/2] turns, then the hardware sine and
                    // cosine (absolute error about 4e-7 on [-pi, pi])
                    float ph = fmaf(kc.z, dfr[3 * s + 2], fmaf(kc.y, dfr[3 * s + 1], kc.x * dfr[3 * s]));
                    ph -= rintf(ph);
                    __sincosf(6.28318530717958648f * ph, &ci[s], &cr[s]);
                }
            } else {  // next k-vector of the row
#pragma unroll
                for (int s = 0; s < NS; ++s) {
                    const float r = fmaf(cr[s], stc[s], -ci[s] * sts[s]);
                    ci[s] = fmaf(cr[s], sts[s], ci[s] * stc[s]);
                    cr[s] = r;
                }
            }
            float gr = 0.f, gi = 0.f;
#pragma unroll
            for (int s = 0; s < NS; ++s) { gr = fmaf(gqs[s], cr[s], gr); gi = fmaf(gqs[s], ci[s], gi); }
            const float2 B = sB[x];
            row = fmaf(B.x, gr, fmaf(-B.y, gi, row));
        }
        __syncwarp();
    }
    kahan_add(acc, cacc, row);
}

template <int NS, int RMODE>
__global__ void __launch_bounds__(32 * PA_WARPS32) k_recip(DevBatch<float> b, CallArgs ca, Work w) {
    __shared__ double2 s_B64[PA_WARPS32][PA_KCHUNK32];
    __shared__ float2 s_B32[PA_WARPS32][PA_KCHUNK32];
    __shared__ float4 s_kc[PA_WARPS32][PA_KCHUNK32];
    const int tid = threadIdx.x, lane = tid & 31, wp = tid >> 5;
    double gq64[NS];
    float gq32[NS];
#pragma unroll
    for (int s = 0; s < NS; ++s) { gq64[s] = b.gq64[s]; gq32[s] = b.gq[s]; }
    int32_t bin = 0, lo = 0, hi = 0;
    while (next_tile(w, b.nbins, lane, bin, lo, hi)) {
        const int32_t fw = b.bin_fw[bin];
        const bool active = lo + lane < hi;
        const int32_t li = active ? w.sorted[lo + lane] : 0;
        float cx, cy, cz;
        bin_centre(b, fw, bin, cx, cy, cz);
        const float4 pa = active ? w.pose_a[li] : make_float4(cx, cy, cz, 0.f);
        const float4 pq = active ? w.pose_b[li] : make_float4(0.f, 0.f, 0.f, 1.f);
        double E = 0.0;
        if (RMODE == 0) {
            // FP32 site offsets from the bin centre and FP32 rows over the whole table
            const float* iA = b.invcells + 9 * fw;
            const float d0 = pa.x - cx, d1 = pa.y - cy, d2 = pa.z - cz;
            float dfr[3 * NS], stc[NS], sts[NS];
            const float q[4] = {pq.x, pq.y, pq.z, pq.w};
            const float kst = b.kstep[fw];
#pragma unroll
            for (int s = 0; s < NS; ++s) {
                float g[3];
                const float gb[3] = {b.gsite[3 * s], b.gsite[3 * s + 1], b.gsite[3 * s + 2]};
                rotate_s(q, gb, g);
                dfr[3 * s + 0] = d0 + fmaf(iA[6], g[2], fmaf(iA[3], g[1], iA[0] * g[0]));
                dfr[3 * s + 1] = d1 + fmaf(iA[7], g[2], fmaf(iA[4], g[1], iA[1] * g[0]));
                dfr[3 * s + 2] = d2 + fmaf(iA[8], g[2], fmaf(iA[5], g[1], iA[2] * g[0]));
                sincospif(2.0f * kst * dfr[3 * s + 2], &sts[s], &stc[s]);
            }
            float acc = 0.f, cacc = 0.f;
            rows32<NS>(b.kcoef4, b.kS2, b.k_offsets[fw], b.k_offsets[fw + 1], dfr, stc, sts, gq32, cx, cy, cz, lane,
                       s_B32[wp], s_kc[wp], acc, cacc);
            E = double(acc) - double(cacc);
        } else {
            // FP64 site offsets from the bin centre
            const double* iA = b.invcells64 + 9 * fw;
            const double d0 = double(pa.x) - double(cx), d1 = double(pa.y) - double(cy), d2 = double(pa.z) - double(cz);
            double dfr[3 * NS], stc[NS], sts[NS];
            const double q[4] = {double(pq.x), double(pq.y), double(pq.z), double(pq.w)};
            const double kst = double(b.kstep[fw]);
#pragma unroll
            for (int s = 0; s < NS; ++s) {
                const double gb[3] = {b.gsite64[3 * s], b.gsite64[3 * s + 1], b.gsite64[3 * s + 2]};
                double g[3];
                rotate_s(q, gb, g);
                dfr[3 * s + 0] = d0 + fma(iA[6], g[2], fma(iA[3], g[1], iA[0] * g[0]));
                dfr[3 * s + 1] = d1 + fma(iA[7], g[2], fma(iA[4], g[1], iA[1] * g[0]));
                dfr[3 * s + 2] = d2 + fma(iA[8], g[2], fma(iA[5], g[1], iA[2] * g[0]));
                sincospi(2.0 * kst * dfr[3 * s + 2], &sts[s], &stc[s]);
            }
            if (RMODE == 1) {
                E = rows64<NS>(b.kcoef4, b.kS2, b.k_offsets[fw], b.k_offsets[fw + 1], dfr, stc, sts, gq64, cx, cy, cz,
                               lane, s_B64[wp], s_kc[wp]);
            } else {
                E = rows64<NS>(b.ks64_coef, b.ks64_S2, b.ks64_off[fw], b.ks64_off[fw + 1], dfr, stc, sts, gq64, cx, cy,
                               cz, lane, s_B64[wp], s_kc[wp]);
                // the FP32 rows from the FP64 offsets rounded once
                float dfr32[3 * NS], stc32[NS], sts32[NS];
#pragma unroll
                for (int s = 0; s < NS; ++s) {
                    dfr32[3 * s] = float(dfr[3 * s]); dfr32[3 * s + 1] = float(dfr[3 * s + 1]);
                    dfr32[3 * s + 2] = float(dfr[3 * s + 2]);
                    stc32[s] = float(stc[s]); sts32[s] = float(sts[s]);
                }
                float acc = 0.f, cacc = 0.f;
                rows32<NS>(b.ks32_coef, b.ks32_S2, b.ks32_off[fw], b.ks32_off[fw + 1], dfr32, stc32, sts32, gq32, cx,
                           cy, cz, lane, s_B32[wp], s_kc[wp], acc, cacc);
                E += double(acc) - double(cacc);
            }
        }
        if (active) w.dUr[li] = KE * E;
    }
}
