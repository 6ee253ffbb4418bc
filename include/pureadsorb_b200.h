/*
 * pureadsorb_b200.h — C ABI of the B200 batched Widom insertion library.
 *
 * The library replaces the device half of PureAdsorb.jl's `widom` (src/widom.jl:290-442): the
 * host keeps building `FrameworkBatch` (src/batch.jl:237-432) and the rejection tables
 * (`build_rejection_tables`, src/widom.jl:202-253), validates the arguments
 * (src/widom.jl:302-364) and reduces the block sums (`_reduce`, src/widom.jl:451-492); this
 * library uploads the batch and runs pose generation, hard-core rejection, the insertion energy
 * and the Boltzmann-weight accumulation on one GPU.
 *
 * Conventions: plain pointers and sizes only. Every array is host memory owned by the caller and
 * read or written only during the call. Offsets are 0-based; LJ type indices, guest type
 * indices and framework indices are 1-based, exactly as `FrameworkBatch` stores them. Matrices
 * are 3x3 column-major (Julia's SMatrix layout); vectors of 3-vectors are interleaved
 * (SVector{3} layout); complex numbers are (re, im) pairs. Every entry point returns a
 * pa_status; none aborts or exits. pa_last_error gives the message of the last failure on a
 * context.
 */
#ifndef PUREADSORB_B200_H
#define PUREADSORB_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int32_t pa_status;
#define PA_OK 0
#define PA_ERR_ARG 1       /* invalid argument or inconsistent batch (ArgumentError/DimensionMismatch) */
#define PA_ERR_CUDA 2      /* a CUDA call failed */
#define PA_ERR_OVERFLOW 3  /* reserved: block sums overflowed (the host's _reduce reports it) */
#define PA_ERR_TIMEOUT 4   /* a bounded device wait gave up */
#define PA_ERR_NOMEM 5     /* device or host allocation failed */
#define PA_ERR_STATE 6     /* wrong object state (e.g. batch from another context) */

#define PA_PRECISION_F32 32 /* FP32 pair/Ewald arithmetic, FP64 constants and accumulation */
#define PA_PRECISION_F64 64 /* plain FP64 form of the reference algorithm */

#define PA_MAX_GUEST_SITES 8

typedef struct pa_context pa_context;
typedef struct pa_batch pa_batch;

/* Creates a context on CUDA device `device`: one stream, one workspace, one error slot.
 * Replaces the KernelAbstractions backend object passed as `backend` to `widom`
 * (src/widom.jl:298-301). */
pa_status pa_context_create(int32_t device, pa_context** out);
pa_status pa_context_destroy(pa_context* ctx);
/* Runs the context's work on an existing CUDA stream (a cudaStream_t passed as void*); NULL
 * restores the context's own stream. */
pa_status pa_context_set_stream(pa_context* ctx, void* stream);
/* Message of the last failed call on this context (empty if none); valid until the next call. */
const char* pa_last_error(const pa_context* ctx);
/* Enables per-kernel CUDA-event timing inside pa_widom (adds events, no synchronisation). */
pa_status pa_context_set_timing(pa_context* ctx, int32_t enable);
/* Total device milliseconds and launch counts per kernel class since timing was enabled.
 * Classes: 0 pose+phase-0, 1 scan/scatter, 2 energy (real space), 3 reduction, 4 neighbour-list
 * build, 5 adjoint (selection, recomputation, reciprocal charge term), 6 FP32 reciprocal term and
 * per-insertion sum, 7 guest-guest term of an insertion into a loaded configuration. */
pa_status pa_context_kernel_times(pa_context* ctx, double* ms /*8*/, int64_t* launches /*8*/);

/* Layout and launch choices of a context (no counterpart in the reference), set by the
 * autotuner or by hand. bin_width: edge in Å of the FP32 path's spatial bins, applied to batches
 * uploaded afterwards (0 selects 3.0). ctas_per_sm: persistent CTAs per SM of the FP32 energy
 * kernel, 1..8 (0 selects 8). use_graphs: 1 makes pa_widom capture its device sequence (kernels,
 * memsets and the copy of the segment sums into pinned host memory) in a CUDA graph and replay it
 * while the call's shape (batch, insertion range, workspace) repeats; seed and kT may change
 * between replays. A shape is captured on its second consecutive call (the first runs directly),
 * so a batch uploaded anew for every call never pays for a capture. Graphs are not used while
 * per-kernel timing is on. */
typedef struct pa_tuning {
    double bin_width;
    int32_t ctas_per_sm;
    int32_t use_graphs;
} pa_tuning;
pa_status pa_context_set_tuning(pa_context* ctx, const pa_tuning* tuning);
pa_status pa_context_get_tuning(const pa_context* ctx, pa_tuning* tuning);

/* Which parts of the FP32 path run in FP64 (no counterpart in the reference, whose Float32 batch
 * computes everything in Float32). near_radius: pairs of an (insertion, site) item closer than
 * this (Å), and pairs whose FP32 distance lies within 4e-6 rc^2 of a cutoff rc^2 (where FP32
 * rounding could flip the cutoff test), are evaluated in FP64 from FP64 list coordinates, FP64
 * site geometry and FP64 pair tables; every other pair stays FP32; 0 turns the FP64 pairs (and
 * the cutoff bands) off. fp64_reciprocal: 1 evaluates the reciprocal cross term (phase factors,
 * row recurrences, sums) in FP64, 0 in FP32. Applies to every later pa_widom / pa_widom_grad /
 * pa_widom_static call of the context; the defaults are PA_DEFAULT_NEAR_RADIUS and 1. */
#define PA_DEFAULT_NEAR_RADIUS 6.0
typedef struct pa_fp32_split {
    double near_radius;
    int32_t fp64_reciprocal;
    int32_t reserved;           /* 0 */
} pa_fp32_split;
pa_status pa_context_set_fp32_split(pa_context* ctx, const pa_fp32_split* split);
pa_status pa_context_get_fp32_split(const pa_context* ctx, pa_fp32_split* split);
/* The form of the FP32 screened-Coulomb pairs in the context's last FP32 energy launch (pa_widom,
 * pa_widom_grad or pa_widom_static): *exp_free = 1 when they were evaluated as
 * exp(-alpha^2 r^2) u H(u), u = 1/r^2, with H a degree-7 polynomial fitted on the host for the
 * batch's alpha over [1/rc^2, 1/near_radius^2] (used when every framework shares one alpha and the
 * fit, evaluated in FP32 as the kernel does, stays within 1.5e-7 relative; *fit_error is that
 * fit's largest relative error), 0 when they took the rational form exp(-z^2) P(t), t = 2/(2+z)
 * (*fit_error = 0). Both 0 before any such launch. */
pa_status pa_context_fp32_form(const pa_context* ctx, int32_t* exp_free, double* fit_error);

/*
 * The fields of a `FrameworkBatch` (src/batch.jl:72-104), as raw arrays. natoms = Σ atoms
 * (atom_offsets[nfw]); nk = Σ k-vectors (k_offsets[nfw]); N = nguest; nt = ntypes.
 * Floating-point arrays are FP64; a caller holding a FrameworkBatch{Float32} widens them.
 */
typedef struct pa_batch_desc {
    int32_t nsys, nfw, ntypes, nguest;
    const double* positions;        /* 3*natoms, cell-sorted per framework            */
    const int32_t* types;           /* natoms, compact 1-based                         */
    const double* charges;          /* natoms                                          */
    const int32_t* atom_offsets;    /* nfw+1                                           */
    const double* cells;            /* 9*nfw  (A, column-major, lattice vectors as columns) */
    const double* invcells;         /* 9*nfw                                           */
    const double* volumes;          /* nfw                                             */
    const double* alphas;           /* nfw                                             */
    const double* ks;               /* 3*nk Cartesian k-vectors                        */
    const double* kprefactor;       /* nk, w_k * pk(|k|^2, alpha, V)                   */
    const double* Shost;            /* 2*nk, (re, im)                                  */
    const int32_t* kcoeffs;         /* 3*nk integer (n1, n2, n3) with k = B*(n1,n2,n3); NULL
                                       makes the library recompute them as round(B^-1 k)    */
    const int32_t* k_offsets;       /* nfw+1                                           */
    const double* constant_offset;  /* nfw                                             */
    const int32_t* ncells;          /* 3*nfw cell-list grid                            */
    const int32_t* cell_offsets;    /* cellgrid_offsets[nfw]                           */
    const int32_t* cellgrid_offsets;/* nfw+1                                           */
    const double* sigma;            /* nt*nt column-major                              */
    const double* epsilon;          /* nt*nt column-major                              */
    const int32_t* guest_types;     /* N, compact 1-based                              */
    const double* guest_sites;      /* 3*N, body frame                                 */
    const double* guest_charges;    /* N                                               */
    double cutoff;                  /* LJ cutoff (A)                                   */
    double ewald_cutoff;            /* real-space Ewald cutoff (A)                     */
    const int32_t* framework_of;    /* nsys, 1-based                                   */
} pa_batch_desc;

/* Uploads a batch for the given precision (PA_PRECISION_F32 or _F64) and builds the device-side
 * tables the kernels read (per-framework spatial bins with their imaged neighbour lists for the
 * FP32 path). Replaces `adapt(backend, batch)` (src/widom.jl:368). The host arrays may be released
 * on return. The neighbour-list fill may still be running on return, on a second stream of the
 * context, so that it overlaps the next call's pose draw and phase 0: every later call that reads
 * the lists first orders the context's stream after the context's last fill (pa_widom just before
 * its energy kernel; an external event node when the stream is being captured). */
pa_status pa_batch_upload(pa_context* ctx, const pa_batch_desc* desc, int32_t precision, pa_batch** out);
pa_status pa_batch_free(pa_batch* batch);
/* Replaces an uploaded batch's LJ pair tables and per-framework constant offsets in place: the
 * parts of a FrameworkBatch that change when only the force field's LJ parameters do (a fitting
 * loop). No counterpart in the reference, which rebuilds the whole batch. sigma and epsilon are
 * nt*nt column-major as in pa_batch_desc; constant_offset has nfw entries. Geometry, bins,
 * neighbour lists and k tables stay. Waits for the copies. */
pa_status pa_batch_set_pair_tables(pa_context* ctx, pa_batch* batch, const double* sigma, const double* epsilon,
                                   const double* constant_offset);
/* Hard-core bound B_s of every framework of an uploaded batch (`hardcore_bound`,
 * src/reject.jl:95-124, which FrameworkBatch computes on the host, src/batch.jl:409-423),
 * evaluated on the device in FP64 from the batch's current pair tables: one root search per
 * attractive (site, atom) pair and a fixed-order sum per framework. For callers that change the
 * pair tables with pa_batch_set_pair_tables and need the bounds for pa_rejection_tables again.
 * Agrees with the host computation to rounding (a different erfc and summation order). bs gets
 * nfw values; PA_ERR_ARG when a root search fails. */
pa_status pa_batch_hardcore_bounds(pa_context* ctx, const pa_batch* batch, double* bs);
/* Size of the FP32 path's neighbour lists (entries over all bins) and the bin count. */
pa_status pa_batch_info(const pa_batch* batch, int64_t* list_entries, int64_t* nbins);

/* Arguments of one widom call. rho2/reach0 are `build_rejection_tables`'s output
 * (src/widom.jl:202-253): rho2 is nsys*N*nt (system s, site a, type t at
 * (s-1)*N*nt + (a-1)*nt + t, 1-based), reach0 is 3*nsys. With reject = 0 they may be NULL and
 * every insertion's energy is computed (`widom_singlephase`, src/widom.jl:296). */
/* A loaded configuration to insert into: Widom along an NVT chain (`widom_chain_kernel!`,
 * src/nvt.jl:85-124; the configuration as `SystemState` holds it, src/state.jl:5-126). Each test
 * insertion sees the host and every live guest of its system: host-guest real space, the
 * reciprocal cross term against the system's running structure factor (host plus guests, replacing
 * the host's), guest-guest real space (each site pair its own minimum image, src/guest.jl:51-75),
 * and the system's pose-independent term (`insertion_constant_term`, src/nvt.jl:45-66) in place of
 * the framework's constant offset. Needs an FP32 batch with one framework per system
 * (framework_of[s] == s + 1) and a single-phase call (reject = 0). */
typedef struct pa_chain_args {
    const double* Sk;             /* 2*nk (re, im): each system's running S(k) over its k table */
    const double* const_term;     /* nsys: each system's pose-independent term (eV)             */
    const int32_t* guest_offsets; /* nsys+1: the live guests of system s are
                                     [guest_offsets[s], guest_offsets[s+1])                    */
    const double* guest_sites;    /* 3*N per live guest, guest-major: Cartesian site positions */
    int64_t k_offset;             /* added to every insertion's per-system index: the cycle's
                                     insertions follow the previous cycles' in the pose stream  */
} pa_chain_args;

typedef struct pa_widom_args {
    double kT;          /* eV, already rounded to the batch's float type by the caller */
    int64_t ninsert;
    uint64_t seed;
    int32_t nblocks;
    int32_t run;        /* run length of the system assignment (src/widom.jl:34-53) */
    int32_t reject;     /* 1: two-phase (hard-core rejection), 0: single-phase */
    const double* rho2;
    const int32_t* reach0;
    /* Optional sharding over GPUs: this call processes only segments
     * [segment_begin, segment_end) of each block (segments of PA_SEGMENT insertions, in
     * per-system sample order); segment_end <= 0 means "to the end". */
    int64_t segment_begin;
    int64_t segment_end;
    const pa_chain_args* chain;  /* optional (NULL: insertion into the empty framework) */
} pa_widom_args;

#define PA_SEGMENT 2048

/* Block sums of one widom call. For system s and block b (0-based, row-major s*nblocks+b):
 * the block's Boltzmann sums are Σ W = exp(lse_max) * sum_w and Σ ΔU·W = exp(lse_max) * sum_uw,
 * accumulated in FP64 per PA_SEGMENT-insertion segment with a fixed reduction tree (so results
 * do not depend on how the work is scheduled). lse_max is -inf for a block whose every insertion
 * has zero weight. count is the number of insertions in the block. */
typedef struct pa_block_sums {
    double* lse_max;   /* nsys*nblocks */
    double* sum_w;     /* nsys*nblocks */
    double* sum_uw;    /* nsys*nblocks */
    int64_t* count;    /* nsys*nblocks */
    double* segments;  /* optional (may be NULL): 3 per segment of the whole job (max, Σ w,
                          Σ ΔU w, with x = -ΔU/kT and w = exp(x - max)), in global segment order;
                          a call writes the segments it processed. */
} pa_block_sums;

/* Number of PA_SEGMENT-insertion segments of a job (global order: system, block, position). */
pa_status pa_segment_count(int64_t ninsert, int32_t nsys, int32_t run, int32_t nblocks, int64_t* nseg);

/* Block sums from the segment triplets of a whole job (e.g. gathered from several GPUs that each
 * processed a contiguous segment range). Uses the same operation sequence as pa_widom, so the
 * result equals a single-GPU call bit for bit. */
pa_status pa_combine_segments(int64_t ninsert, int32_t nsys, int32_t run, int32_t nblocks, const double* segments,
                              pa_block_sums* sums);

/* Optional per-insertion outputs, in system-major, per-system sample order (insertion k of
 * system s at offset(s) + k - 1, offset = prefix sums of the per-system counts). Any pointer may
 * be NULL. dU: ΔU in eV including the constant offset, +inf for rejected insertions. flags: 1
 * if phase 0 rejected the insertion. poses: 7 per insertion, fractional position then
 * quaternion (x, y, z, w), widened to FP64. */
typedef struct pa_insertion_out {
    double* dU;
    uint8_t* flags;
    double* poses;
} pa_insertion_out;

/* One widom call: the whole chunk loop of src/widom.jl:399-440 on the device, with poses drawn
 * on the device from the counter-based stream (insertion k of system s draws words 0..5 of
 * ChainRNG(splitmix64(seed, s), k, 0); src/rng.jl:43-141, src/state.jl:225-230) instead of
 * the host Xoshiro stream of src/widom.jl:369. */
pa_status pa_widom(pa_context* ctx, const pa_batch* batch, const pa_widom_args* args, pa_block_sums* sums,
                   pa_insertion_out* per_insertion);

/* Rejection radii and phase-0 stencil reaches of one widom call, on the host
 * (`build_rejection_tables`, src/widom.jl:202-253): rho2 gets nsys*N*nt values, reach0 3*nsys.
 * bs and kmin are the batch's `bs` (nfw) and `kmin` (nfw*N*nt); eps_F is eps of the batch's
 * float type. Returns PA_ERR_ARG (and the 1-based system in *bad_system) when a system's margin
 * is not positive or a root search fails. Needs no device. */
pa_status pa_rejection_tables(const pa_batch_desc* desc, const double* bs, const double* kmin, double kT, double eps_F,
                              double* rho2, int32_t* reach0, int32_t* bad_system);

/* Batch construction on the device (pose-independent tables; the host builder computes the same
 * ones). Each call copies its host inputs, runs on the context's stream and returns once its
 * outputs are in host memory.
 *
 * pa_batch_rejection_tables: pa_rejection_tables for an uploaded batch, the root searches
 * (find_rho2, src/reject.jl:168-209) on the device, one thread per (system, site, type), with the
 * same operation sequence as the host, so rho2 and reach0 equal pa_rejection_tables' bit for bit.
 * bs (nfw) and kmin (nfw*N*nt) as for pa_rejection_tables; the pair tables and constant offsets
 * are the batch's (after any pa_batch_set_pair_tables). */
pa_status pa_batch_rejection_tables(pa_context* ctx, const pa_batch* batch, const double* bs, const double* kmin,
                                    double kT, double eps_F, double* rho2, int32_t* reach0, int32_t* bad_system);

/* The half-space k-vectors of one cell (`kvectors`, src/ewald.jl:142-157): n1 = 0..nmax[0],
 * n2 = -nmax[1]..nmax[1], n3 = -nmax[2]..nmax[2] (n3 fastest), (0,0,0) left out, |k| <= kmax,
 * with k = B (n1, n2, n3) for the reciprocal basis B (row-major 3x3, 2 pi (A^-1)^T), weight 1 for
 * n1 = 0 and 2 otherwise, and kpref = w (c2piv exp(-|k|^2 / four_a2) / |k|^2) (`pk`,
 * src/ewald.jl:36-39) with c2piv = 2 pi / V and four_a2 = 4 alpha^2. Outputs in enumeration order:
 * ks (3 per k-vector), weights, kpref, coeffs (3 per k-vector), and their number in *nk; the
 * arrays need room for (nmax[0]+1)(2nmax[1]+1)(2nmax[2]+1)-1 k-vectors (capacity). */
pa_status pa_kvectors(pa_context* ctx, const double* B, const int32_t* nmax, double kmax, double c2piv, double four_a2,
                      int64_t capacity, double* ks, double* weights, double* kpref, int32_t* coeffs, int64_t* nk);

/* kmin of one framework (`kmin_table`, src/reject.jl:134-145): kmin[a*ntypes + t] is the most
 * negative KE q_a q_h over its atoms h of compact type t+1 (types 1-based), or 0. */
pa_status pa_kmin_table(pa_context* ctx, const double* guest_charges, int32_t nguest, const int32_t* types,
                        const double* charges, int64_t natoms, int32_t ntypes, double* kmin);

/* The phase-0 cell list of one framework (`cell_sort`, src/cell.jl:96-118): the stable counting
 * sort of its atoms by the cell of their wrapped fractional coordinates (3 per atom) on an
 * ncells[0] x ncells[1] x ncells[2] grid (x fastest). perm[i] is the 0-based original index of the
 * i-th sorted atom; offsets (prod(ncells)+1) the start of every cell. */
pa_status pa_cell_sort(pa_context* ctx, const double* frac, int64_t natoms, const int32_t* ncells, int64_t* perm,
                       int32_t* offsets);

/* Allocation-free variant of pa_widom; no counterpart in the reference. For callers that may
 * not allocate device memory during the call (a host application that owns a fixed memory
 * budget, strict per-tenant accounting, or code that must avoid cudaMalloc's device-wide
 * synchronisation): every per-call scratch buffer is carved out of one file-scope device array of
 * 32 MiB that each GPU loading the library holds until the process exits. It computes what
 * pa_widom computes (the same poses, phase-0 flags, energy and reduction kernels, and the context's
 * FP32/FP64 split), except that on an FP32 batch the poses and phase 0 come from the fused
 * per-insertion kernel (k_pose) instead of the warp-cooperative pair k_draw32 + k_phase0_32; both
 * give the same poses and flags bit for bit. Limits: at most 131,072 insertions per call (and, for
 * an FP32 batch, 393,216 insertion-site pairs), 1,024 systems, 32,768 spatial bins and 65,536
 * rejection radii; larger calls return PA_ERR_ARG. Only per_insertion->dU may be requested.
 * All calls share the array (host calls are serialised by a mutex); device work of two calls must
 * not overlap. A call that returns an error after its device work began (a launch error, a
 * timed-out wait) leaves the array in use until that work finishes; until then later calls return
 * PA_ERR_STATE. The first call on a device looks up the array's address and creates an event,
 * and the CUDA runtime may load the library's device module then (which allocates device memory,
 * the array included): make one warm-up call before any stream capture and before the code that
 * must not allocate. */
pa_status pa_widom_static(pa_context* ctx, const pa_batch* batch, const pa_widom_args* args, pa_block_sums* sums,
                          pa_insertion_out* per_insertion);

/* Adjoint sums of one widom call; no counterpart in the reference, which has no gradients.
 * The Julia analogue is a ChainRulesCore rrule of ln K_H over the FrameworkBatch fields sigma,
 * epsilon and charges. With x_i = -ΔU_i/kT, m_s = max x over system s's survivors of this call
 * and w_i = exp(x_i - m_s), d ln K_H(s) / dθ = -(Σ_i w_i ∂ΔU_i/∂θ) / (kT Σ_i w_i). The library
 * returns the numerator sums for θ = the batch's pair tables and stored charges; the caller
 * adds the constant offset's dependence (tail correction, net-charge term) and folds the
 * pair tables onto per-type parameters (Lorentz-Berthelot). The sums are taken over every
 * survivor whose x_i >= m_s - window (0 selects 50, i.e. relative weights down to 2e-22);
 * lighter insertions are left out. Accumulation is FP32 per lane and FP64 across lanes and
 * insertions by atomic adds, so the last bits depend on scheduling. */
typedef struct pa_grad_sums {
    double* xmax;        /* nsys out: m_s (-inf for a system without survivors)               */
    double* sum_w;       /* nsys out: Σ_i w_i over every survivor of the call                  */
    double* d_epsilon;   /* nsys*N*nt out: [s][a][t] Σ_i w_i ∂ΔU_i/∂ε(guest type of site a, t) */
    double* d_sigma;     /* nsys*N*nt out: the same for σ                                      */
    double* d_charge;    /* Σ_s natoms(framework_of[s]) out: Σ_i w_i ∂ΔU_i/∂q_j per stored
                            atom j of the system's framework (desc order), system-major          */
    double* s_guest;     /* optional, 2*Σ_s nk(framework_of[s]): Σ_i w_i S_g,i(k) (re, im)      */
    double window;       /* in: the charge pass recomputes survivors within this many kT of the
                            system's largest weight (0: 50); the ε and σ sums cover every survivor */
    int64_t recomputed;  /* out: insertions the charge pass recomputed (0 with lj_only)          */
    int32_t lj_only;     /* in: nonzero skips the charge derivatives (d_charge and s_guest are
                            returned as zeros), for callers that only need ε and σ               */
} pa_grad_sums;

/* pa_widom plus the adjoint sums. FP32 batches only (the adjoint walks the FP32 path's bins and
 * neighbour lists). Arguments as for pa_widom; sums->segments and per_insertion may be given. */
pa_status pa_widom_grad(pa_context* ctx, const pa_batch* batch, const pa_widom_args* args, pa_block_sums* sums,
                        pa_grad_sums* grad, pa_insertion_out* per_insertion);

/* Host-side pose of insertion k of system s (the same stream as the device), for callers that
 * need the poses without a GPU (e.g. the self-term orientations of FrameworkBatch). precision
 * selects 32- or 64-bit draws; rpos gets 3 and quat 4 values widened to FP64. */
pa_status pa_pose_host(int32_t precision, uint64_t seed, uint64_t s, uint64_t k, double* rpos, double* quat);

/* FP64 structure factor S(k) = Σ_j q_j exp(i k·r_j) of one atom set on the device
 * (`structure_factor`, src/ewald.jl:159-170). S gets 2*nk values (re, im). */
pa_status pa_structure_factor(pa_context* ctx, const double* ks, int64_t nk, const double* positions,
                              const double* charges, int64_t natoms, double* S);

/* Guest self term of the batch's constant offset for a set of orientations (src/batch.jl:357-375):
 * samples[o] = Σ_k kpref_k |Σ_s q_s exp(i k·g_s(o))|^2 over the given k-vectors, in FP64 on the
 * device (without the KE factor). sites: norient*nguest*3 rotated body-frame site offsets. */
pa_status pa_self_term(pa_context* ctx, const double* ks, const double* kpref, int64_t nk, const double* sites,
                       const double* charges, int32_t nguest, int32_t norient, double* samples);

/* Library version string. */
const char* pa_version(void);

#ifdef __cplusplus
}
#endif
#endif /* PUREADSORB_B200_H */
