// Insertion into a loaded configuration (Widom along an NVT chain, `widom_chain_kernel!`,
// src/nvt.jl:85-124): the guest-guest real-space term of each test insertion.
//
// The host-guest terms of such an insertion are the FP32 path's own kernels (k_energy32 for the
// real space, k_recip against the system's running structure factor host + guests, which the
// call substitutes for the host's), and k_combine adds this kernel's term and the system's
// pose-independent constant. Here: for every live guest j of the insertion's system and every
// site pair (a of the test guest, b of guest j), one minimum image of the site-site vector
// (src/guest.jl:51-75: each pair its own image), Lennard-Jones inside the LJ cutoff and
// KE q_a q_b erfc(alpha r)/r inside the Ewald cutoff, with a compensated sum per lane and a
// fixed-order FP64 warp reduction. The geometry (test sites, site-site vectors, images, r^2) is
// FP64: the sites are absolute Cartesian positions across the cell, whose FP32 differences would
// lose about 1e-7 of the cell length; r^2 is then rounded once and the pair terms use the FP32
// arithmetic of k_energy32's rational form (guest-guest pairs have no near radius).
//
// One warp per insertion, lanes over the (live guest, guest site) pairs of the system (a system
// holds tens of guests, so lanes over guests alone would leave most of the warp idle). Included by
// pa_kernels.cuh after pa_energy32.cuh.
#pragma once

struct ChainArgs {
    const double* gsites;   // 3*N per live guest, guest-major: Cartesian site positions (A)
    const int32_t* goff;    // nsys+1: live guests of system s are [goff[s], goff[s+1])
    const int32_t* gtype;   // N: compact type of each guest site
    const double* cells;    // 9*nfw: FP64 cells (column-major)
    const double* invcells; // 9*nfw
};

template <int NS>
__global__ void __launch_bounds__(256) k_guest32(DevBatch<float> b, CallArgs ca, Work w, ChainArgs c) {
    const int lane = threadIdx.x & 31;
    const int64_t warp = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = (int64_t(gridDim.x) * blockDim.x) >> 5;
    const int nt = b.ntypes;
    const float NLOG2E = -1.4426950408889634f;
    for (int64_t t = warp; t < ca.n_act; t += nwarps) {
        if (w.bin_of[t] < 0) continue;  // rejected (warp-uniform)
        const int32_t s = find_system(ca.sys_off, b.nsys, ca.i_lo + t);
        const int32_t fw = b.framework_of[s];
        const int32_t j0 = c.goff[s], j1 = c.goff[s + 1];
        const float4 pa = w.pose_a[t];
        const float4 pq = w.pose_b[t];
        const double* A = c.cells + 9 * fw;
        const double* iA = c.invcells + 9 * fw;
        const float rl2 = b.rl2, re2 = b.re2, alpha = float(b.alphas[fw]);
        const float a2n = (alpha * alpha) * NLOG2E;
        // the test guest's sites: A rpos + rotate(q, site), FP64 from the FP32 pose
        double sx[NS], sy[NS], sz[NS];
        float sq[NS];
        {
            const double q[4] = {pq.x, pq.y, pq.z, pq.w};
            const double px = fma(A[6], double(pa.z), fma(A[3], double(pa.y), A[0] * double(pa.x)));
            const double py = fma(A[7], double(pa.z), fma(A[4], double(pa.y), A[1] * double(pa.x)));
            const double pz = fma(A[8], double(pa.z), fma(A[5], double(pa.y), A[2] * double(pa.x)));
#pragma unroll
            for (int a = 0; a < NS; ++a) {
                // v + 2 u x (u x v + w v) (src/energy.jl:13-16)
                const double v0 = b.gsite[3 * a], v1 = b.gsite[3 * a + 1], v2 = b.gsite[3 * a + 2];
                const double c0 = q[1] * v2 - q[2] * v1 + q[3] * v0;
                const double c1 = q[2] * v0 - q[0] * v2 + q[3] * v1;
                const double c2 = q[0] * v1 - q[1] * v0 + q[3] * v2;
                sx[a] = px + v0 + 2.0 * (q[1] * c2 - q[2] * c1);
                sy[a] = py + v1 + 2.0 * (q[2] * c0 - q[0] * c2);
                sz[a] = pz + v2 + 2.0 * (q[0] * c1 - q[1] * c0);
                sq[a] = float(KE * double(b.gq[a]));
            }
        }
        float esum = 0.f, ecmp = 0.f;
        bool hit = false;  // coincident sites: the pair energy diverges
        const int64_t p1 = int64_t(j1 - j0) * NS;
        for (int64_t p = lane; p < p1; p += 32) {
            {
                const int32_t bb = int32_t(p % NS);
                const double* o = c.gsites + 3 * (int64_t(j0) * NS + p);
                const double ox = o[0], oy = o[1], oz = o[2];
                const int32_t tb = c.gtype[bb];
                const float qb = b.gq[bb];
#pragma unroll
                for (int a = 0; a < NS; ++a) {
                    // minimum image of the site-site vector (FP64), r^2 rounded once
                    double dx = sx[a] - ox, dy = sy[a] - oy, dz = sz[a] - oz;
                    const double f0 = rint(fma(iA[6], dz, fma(iA[3], dy, iA[0] * dx)));
                    const double f1 = rint(fma(iA[7], dz, fma(iA[4], dy, iA[1] * dx)));
                    const double f2 = rint(fma(iA[8], dz, fma(iA[5], dy, iA[2] * dx)));
                    dx -= fma(A[6], f2, fma(A[3], f1, A[0] * f0));
                    dy -= fma(A[7], f2, fma(A[4], f1, A[1] * f0));
                    dz -= fma(A[8], f2, fma(A[5], f1, A[2] * f0));
                    const float r2 = float(fma(dz, dz, fma(dy, dy, dx * dx)));
                    if (!(r2 < rl2 || r2 < re2)) continue;
                    if (!(r2 > 0.f)) { hit = true; continue; }
                    float e = 0.f;
                    {
                        float ri = rsqrt_ftz(r2);
                        ri = ri * fmaf(-0.5f * r2 * ri, ri, 1.5f);
                        if (r2 < rl2) {
                            const float x = b.sig2[a * nt + tb] * (ri * ri);
                            const float x3 = x * x * x;
                            e = b.eps4[a * nt + tb] * (x3 * x3 - x3);
                        }
                        if (b.has_charge && r2 < re2) {
                            const float z = alpha * (r2 * ri);
                            const float tt = rcp_nr(fmaf(0.5f, z, 1.0f));
                            const float cf[PA_NERFC32] = PA_ERFC32_INIT;
                            float p = cf[PA_NERFC32 - 1];
#pragma unroll
                            for (int k = PA_NERFC32 - 2; k >= 0; --k) p = fmaf(p, tt, cf[k]);
                            e = fmaf(sq[a] * qb, p * ex2_ftz(r2 * a2n) * ri, e);
                        }
                    }
                    kahan_add(esum, ecmp, e);
                }
            }
        }
        // fixed-order FP64 reduction over the lanes
        double v = double(esum) - double(ecmp);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (__any_sync(0xffffffffu, hit)) v = INFINITY;
        if (lane == 0) w.dUg[t] = v;
    }
}
