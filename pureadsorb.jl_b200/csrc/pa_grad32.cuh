// The adjoint pass: weighted sums of ∂ΔU/∂θ over the insertions that carry the Boltzmann weight.
//
// ln K_H = ln V - ln kT + ln <W>, W = exp(-ΔU/kT), so for any parameter θ of the energy
// d ln K_H / dθ = -<W ∂ΔU/∂θ> / (kT <W>). The forward pass leaves every survivor's pose, bin and
// ΔU in the workspace. The adjoint recomputes the pair terms of the insertions whose weight
// relative to their system's largest is at least exp(-window) and accumulates, per system:
//   - per (guest site a, host type t): Σ w Σ_j x(x - 1) and Σ w Σ_j x(2x - 1), x = (σ_at^2/r^2)^3,
//     over the LJ pairs inside the cutoff (∂u/∂ε_at = 4 x(x - 1) and ∂u/∂σ_at = (24 ε_at/σ_at)
//     x(2x - 1) for u = 4 ε_at (x^2 - x));
//   - per stored atom j: Σ w KE Σ_a q_a erfc(α r_aj)/r_aj over the pairs inside the Ewald cutoff
//     (the real-space part of ∂ΔU/∂q_j);
//   - per k-vector: G_k = Σ w S_g(k), S_g(k) = Σ_a q_a e^{ik·r_a} (the reciprocal part of
//     ∂ΔU/∂q_j is KE Σ_k 2 kpref_k Re(e^{-ik·r_j} G_k), formed per atom by k_charge_recip).
// Per-lane partial sums are FP32; every sum across lanes and insertions is an FP64 atomic add.
// Included by pa_kernels.cuh after pa_energy32.cuh.
#pragma once

#define PA_WARPSG 4

struct GradArgs {
    const double* xmax;       // nsys: the shift m_s; w = exp(-ΔU/kT - m_s)
    double kT;
    double window;            // insertions with -ΔU/kT >= m_s - window are recomputed
    const int64_t* sys_aoff;  // nsys+1: each system's first per-atom slot
    const int64_t* sys_koff;  // nsys+1: each system's first k slot
    int32_t nsys;
    int32_t lj_only;          // nonzero: no charge derivatives (real-space terms, G_k)
    int32_t skip_lj;          // nonzero: k_grad32 leaves the LJ sums (k_lj_reduce forms them)
    int32_t* heavy;           // n_act: local indices of the recomputed insertions
    int32_t* nheavy;          // count of heavy
    double* g_w;              // nsys: Σ w over the recomputed insertions
    double* g_lj;             // nsys*2*NS*nt: [s][0][a][t] = Σ w Σ x(x-1), [s][1][a][t] = Σ w Σ x(2x-1)
    double* g_q;              // sys_aoff[nsys]
    double* g_k;              // 2*sys_koff[nsys]: (re, im)
    const double* frac;       // 3*natoms: fractional coordinates of the stored atoms (FP64)
    const double* kpref2;     // nk: 2 kpref
};

// Selects the insertions the adjoint recomputes: survivors with x = -ΔU/kT >= m_s - window.
__global__ void __launch_bounds__(256) k_heavy(Work w, CallArgs ca, GradArgs g) {
    const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    bool keep = false;
    if (t < ca.n_act && w.bin_of[t] >= 0) {
        const int32_t s = find_system(ca.sys_off, g.nsys, ca.i_lo + t);
        keep = -w.dU[t] / g.kT >= g.xmax[s] - g.window;
    }
    const unsigned bal = __ballot_sync(0xffffffffu, keep);
    const int lane = threadIdx.x & 31;
    int32_t base = 0;
    if (lane == 0 && bal) base = atomicAdd(g.nheavy, __popc(bal));
    base = __shfl_sync(0xffffffffu, base, 0);
    if (keep) g.heavy[base + __popc(bal & ((1u << lane) - 1u))] = int32_t(t);
}

// One warp per recomputed insertion. For each guest site the lanes stride over the list of the
// bin holding that site (the forward pass's (insertion, site) items), with the forward kernel's
// site geometry operation for operation; then over the framework's k-vectors.
template <int NS>
__global__ void __launch_bounds__(32 * PA_WARPSG) k_grad32(DevBatch<float> b, CallArgs ca, Work w, GradArgs g) {
    extern __shared__ float s_dyn[];  // sig2 (NS*nt), then per warp 2*NS*nt accumulators
    const int tid = threadIdx.x, lane = tid & 31, wp = tid >> 5;
    const int nt = b.ntypes, nacc = 2 * NS * nt;
    float* s_sig2 = s_dyn;
    float* acc = s_dyn + NS * nt + wp * nacc;
    for (int x = tid; x < NS * nt; x += blockDim.x) s_sig2[x] = b.sig2[x];
    for (int x = lane; x < nacc; x += 32) acc[x] = 0.f;
    __syncthreads();
    float gqs[NS], gsb[3 * NS];
#pragma unroll
    for (int s = 0; s < NS; ++s) {
        gqs[s] = b.gq[s];
        gsb[3 * s] = b.gsite[3 * s]; gsb[3 * s + 1] = b.gsite[3 * s + 1]; gsb[3 * s + 2] = b.gsite[3 * s + 2];
    }
    const bool charged = b.has_charge != 0 && g.lj_only == 0;
    const int32_t nh = *g.nheavy;
    const int32_t nwarps = gridDim.x * PA_WARPSG;
    const float NLOG2E = -1.4426950408889634f;
    for (int32_t h = blockIdx.x * PA_WARPSG + wp; h < nh; h += nwarps) {
        const int32_t li = g.heavy[h];
        const int32_t sy = find_system(ca.sys_off, g.nsys, ca.i_lo + li);
        const double wgt = exp(-w.dU[li] / g.kT - g.xmax[sy]);
        const double wke = wgt * KE;
        const float4 pa = w.pose_a[li];
        const float4 pq = w.pose_b[li];
        const float q[4] = {pq.x, pq.y, pq.z, pq.w};
        const float rp[3] = {pa.x, pa.y, pa.z};
        const int32_t fw = b.framework_of[sy];
        const float* A = b.cells + 9 * fw;
        const float* iA = b.invcells + 9 * fw;
        const float rl2 = b.rl2, re2 = b.re2, alpha = float(b.alphas[fw]);
        double* gq_sys = g.g_q + g.sys_aoff[sy] - b.atom_offsets[fw];
        double fr[3 * NS];  // absolute fractional site positions (reciprocal phases)
#pragma unroll
        for (int s = 0; s < NS; ++s) {
            float gg[3], fs[3], sh[3];
            rotate_s(q, gsb + 3 * s, gg);
            site_frac32(rp, gg, iA, fs, sh);
#pragma unroll
            for (int r = 0; r < 3; ++r)
                fr[3 * s + r] = double(rp[r]) + double(fmaf(iA[6 + r], gg[2], fmaf(iA[3 + r], gg[1], iA[r] * gg[0])));
            // this site's bin and its position relative to the bin centre (as in k_energy32)
            const int32_t bin = w.item_bin[li * NS + s] / b.nsub;
            const int32_t l0 = b.list_offsets[bin], l1 = b.list_offsets[bin + 1];
            float cx, cy, cz;
            bin_centre(b, fw, bin, cx, cy, cz);
            const float d0 = float((double(pa.x) + double(sh[0])) - double(cx));
            const float d1 = float((double(pa.y) + double(sh[1])) - double(cy));
            const float d2 = float((double(pa.z) + double(sh[2])) - double(cz));
            const float px = fmaf(A[6], d2, fmaf(A[3], d1, A[0] * d0)) + gg[0];
            const float py = fmaf(A[7], d2, fmaf(A[4], d1, A[1] * d0)) + gg[1];
            const float pz = fmaf(A[8], d2, fmaf(A[5], d1, A[2] * d0)) + gg[2];
            // per-lane sums for the lane's current host type, flushed to the warp's shared
            // accumulators when the type changes (the list is type-major, so changes are rare)
            int32_t cur = -1;
            float P = 0.f, Q = 0.f;
            for (int32_t e = l0 + lane; e < l1; e += 32) {
                const float4 at = b.list_xyzq[e];
                const int32_t ty = b.list_type[e];
                if (ty != cur) {
                    if (cur >= 0) {
                        if (P != 0.f) atomicAdd(&acc[s * nt + cur], P);
                        if (Q != 0.f) atomicAdd(&acc[(NS + s) * nt + cur], Q);
                        P = 0.f; Q = 0.f;
                    }
                    cur = ty;
                }
                const float dx = px - at.x, dy = py - at.y, dz = pz - at.z;
                const float r2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
                if (!g.skip_lj && r2 < rl2) {
                    const float x = s_sig2[s * nt + ty] * rcp_nr(r2);
                    const float x3 = x * x * x;
                    P = fmaf(x3, x3 - 1.0f, P);
                    Q = fmaf(x3, fmaf(2.0f, x3, -1.0f), Q);
                }
                if (charged && r2 < re2) {
                    float ri = rsqrt_ftz(r2);
                    ri = ri * fmaf(-0.5f * r2 * ri, ri, 1.5f);
                    const float z = alpha * (r2 * ri);
                    const float tt = rcp_nr(fmaf(0.5f, z, 1.0f));
                    const float cf[PA_NERFC32] = PA_ERFC32_INIT;
                    float p = cf[PA_NERFC32 - 1];
#pragma unroll
                    for (int k = PA_NERFC32 - 2; k >= 0; --k) p = fmaf(p, tt, cf[k]);
                    const float cq = gqs[s] * (p * ex2_ftz((z * z) * NLOG2E) * ri);
                    if (cq != 0.f) atomicAdd(&gq_sys[b.list_atom[e]], wke * double(cq));
                }
            }
            if (cur >= 0) {
                if (P != 0.f) atomicAdd(&acc[s * nt + cur], P);
                if (Q != 0.f) atomicAdd(&acc[(NS + s) * nt + cur], Q);
            }
        }
        __syncwarp();
        double* glj = g.g_lj + int64_t(sy) * nacc;
        for (int x = lane; x < nacc; x += 32) {
            const float v = acc[x];
            if (v != 0.f) { atomicAdd(&glj[x], wgt * double(v)); acc[x] = 0.f; }
        }
        __syncwarp();
        // G_k += w S_g(k): the phase n.r_a of every site in FP64, one k-vector per lane
        if (charged) {
            const int32_t k0 = b.k_offsets[fw], k1 = b.k_offsets[fw + 1];
            double* gk = g.g_k + 2 * (g.sys_koff[sy] - k0);
            for (int32_t kk = k0 + lane; kk < k1; kk += 32) {
                const float4 kc = b.kcoef4[kk];
                double gr = 0.0, gi = 0.0;
#pragma unroll
                for (int s = 0; s < NS; ++s) {
                    double ph = double(kc.x) * fr[3 * s] + double(kc.y) * fr[3 * s + 1] + double(kc.z) * fr[3 * s + 2];
                    ph -= rint(ph);
                    double sn, cs;
                    sincospi(2.0 * ph, &sn, &cs);
                    gr = fma(double(gqs[s]), cs, gr);
                    gi = fma(double(gqs[s]), sn, gi);
                }
                atomicAdd(&gk[2 * kk], wgt * gr);
                atomicAdd(&gk[2 * kk + 1], wgt * gi);
            }
        }
        if (lane == 0) atomicAdd(&g.g_w[sy], wgt);
    }
}

// The LJ part of the adjoint from the forward pass's per-run sums (w.item_pq): per tile of 32
// sorted items of one bin, each item's weight w = exp(-ΔU/kT - m_s) times its runs' sums, reduced
// over the warp per (guest site, run) in a fixed order and added to the system's
// [s][0 or 1][site][type of the run] sums. Tiles are taken in order, warp by warp; every survivor
// enters (weights far below the largest underflow to zero).
template <int NS>
__global__ void __launch_bounds__(256) k_lj_reduce(DevBatch<float> b, CallArgs ca, Work wi, Work w, GradArgs g) {
    const int lane = threadIdx.x & 31;
    const int64_t warp = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = (int64_t(gridDim.x) * blockDim.x) >> 5;
    const int32_t total = wi.counters[1];
    const int nt = b.ntypes, rm = b.runs_per_bin, nacc = 2 * NS * nt;
    const unsigned FULL = 0xffffffffu;
    for (int64_t t = warp; t < total; t += nwarps) {
        const int32_t bin = find_bin(wi.tile_start, b.nbins, int32_t(t));
        const int32_t lo = wi.bin_start[bin] + (int32_t(t) - wi.tile_start[bin]) * PA_TILE32;
        const int32_t hi = min(lo + PA_TILE32, wi.bin_start[bin + 1]);
        const bool active = lo + lane < hi;
        const int32_t it = active ? wi.sorted[lo + lane] : 0;
        const int32_t li = it / NS, as = it - li * NS;
        const int32_t s = find_system(ca.sys_off, g.nsys, ca.i_lo + li);
        double wgt = 0.0;
        if (active) {
            const double x = -w.dU[li] / g.kT;
            if (x > -INFINITY) wgt = exp(x - g.xmax[s]);
        }
        const int32_t s0 = __shfl_sync(FULL, s, 0);
        const bool one = __all_sync(FULL, !active || s == s0);
        const int32_t l1 = b.list_offsets[bin + 1];
        const int2* runs = b.list_runs + int64_t(bin) * rm;
        const float2* pq = w.item_pq + int64_t(lo + lane) * rm;
        for (int32_t r = 0; r < rm; ++r) {
            const int2 run = runs[r];
            if (run.x >= l1) break;  // (warp-uniform) past the bin's last run
            float2 v = active ? pq[r] : make_float2(0.f, 0.f);
            const double vp = wgt * double(v.x), vq = wgt * double(v.y);
            if (one) {
#pragma unroll
                for (int a = 0; a < NS; ++a) {
                    double p = as == a ? vp : 0.0, q = as == a ? vq : 0.0;
#pragma unroll
                    for (int o = 16; o > 0; o >>= 1) {
                        p += __shfl_xor_sync(FULL, p, o);
                        q += __shfl_xor_sync(FULL, q, o);
                    }
                    if (lane == 0) {
                        double* acc = g.g_lj + int64_t(s0) * nacc;
                        if (p != 0.0) atomicAdd(&acc[a * nt + run.y], p);
                        if (q != 0.0) atomicAdd(&acc[(NS + a) * nt + run.y], q);
                    }
                }
            } else if (active) {  // a tile spanning systems that share a framework
                double* acc = g.g_lj + int64_t(s) * nacc;
                if (vp != 0.0) atomicAdd(&acc[as * nt + run.y], vp);
                if (vq != 0.0) atomicAdd(&acc[(NS + as) * nt + run.y], vq);
            }
        }
    }
}

// Reciprocal part of ∂ΔU/∂q_j per system and stored atom: g_q[s][j] += KE Σ_k 2 kpref_k
// (cos φ Re G_k + sin φ Im G_k), φ = 2π n_k·f_j in FP64. One thread per atom, blockIdx.y = system,
// the system's G_k staged through shared memory.
__global__ void __launch_bounds__(256) k_charge_recip(DevBatch<float> b, GradArgs g) {
    __shared__ double4 s_k[256];  // n1, n2, n3, 2 kpref
    __shared__ double2 s_g[256];
    const int32_t sy = blockIdx.y, fw = b.framework_of[sy];
    const int32_t a0 = b.atom_offsets[fw], a1 = b.atom_offsets[fw + 1];
    const int32_t k0 = b.k_offsets[fw], k1 = b.k_offsets[fw + 1];
    const int32_t j = a0 + blockIdx.x * blockDim.x + threadIdx.x;
    if (a0 + int32_t(blockIdx.x * blockDim.x) >= a1) return;  // the whole block is past this framework
    const double* gk = g.g_k + 2 * g.sys_koff[sy];
    double f0 = 0, f1 = 0, f2 = 0;
    if (j < a1) { f0 = g.frac[3 * j]; f1 = g.frac[3 * j + 1]; f2 = g.frac[3 * j + 2]; }
    double acc = 0.0;
    for (int32_t kb = k0; kb < k1; kb += 256) {
        const int32_t n = min(256, k1 - kb);
        __syncthreads();
        if (int32_t(threadIdx.x) < n) {
            const int32_t kk = kb + threadIdx.x;
            const float4 kc = b.kcoef4[kk];
            s_k[threadIdx.x] = make_double4(kc.x, kc.y, kc.z, g.kpref2[kk]);
            s_g[threadIdx.x] = make_double2(gk[2 * (kk - k0)], gk[2 * (kk - k0) + 1]);
        }
        __syncthreads();
        for (int32_t x = 0; x < n; ++x) {
            const double4 kc = s_k[x];
            double ph = kc.x * f0 + kc.y * f1 + kc.z * f2;
            ph -= rint(ph);
            double sn, cs;
            sincospi(2.0 * ph, &sn, &cs);
            acc = fma(kc.w, fma(cs, s_g[x].x, sn * s_g[x].y), acc);
        }
    }
    if (j < a1) g.g_q[g.sys_aoff[sy] + (j - a0)] += KE * acc;
}
