"""ctypes binding to the C ABI in include/pureadsorb_b200.h (libpureadsorb_b200.so, built
in-tree by build.py). Every call checks its status and raises with the library's message; a
missing library raises LibraryMissing: there is no fallback path."""
import atexit
import math
import ctypes
import os
import weakref

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpureadsorb_b200.so")

PA_OK, PA_ERR_ARG, PA_ERR_CUDA, PA_ERR_OVERFLOW, PA_ERR_TIMEOUT, PA_ERR_NOMEM, PA_ERR_STATE = range(7)
PA_PRECISION_F32, PA_PRECISION_F64 = 32, 64
PA_MAX_GUEST_SITES = 8
PA_SEGMENT = 2048
STATUS_NAMES = {0: "PA_OK", 1: "PA_ERR_ARG", 2: "PA_ERR_CUDA", 3: "PA_ERR_OVERFLOW", 4: "PA_ERR_TIMEOUT",
                5: "PA_ERR_NOMEM", 6: "PA_ERR_STATE"}

_p = ctypes.c_void_p
_i32, _i64, _u64, _f64 = ctypes.c_int32, ctypes.c_int64, ctypes.c_uint64, ctypes.c_double


class LibraryMissing(RuntimeError):
    """The compiled library is absent: build it (build.py / __graft_entry__.build())."""


class PAError(RuntimeError):
    def __init__(self, status, message):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


class BatchDesc(ctypes.Structure):
    _fields_ = [("nsys", _i32), ("nfw", _i32), ("ntypes", _i32), ("nguest", _i32),
                ("positions", _p), ("types", _p), ("charges", _p), ("atom_offsets", _p), ("cells", _p),
                ("invcells", _p), ("volumes", _p), ("alphas", _p), ("ks", _p), ("kprefactor", _p), ("Shost", _p),
                ("kcoeffs", _p), ("k_offsets", _p), ("constant_offset", _p), ("ncells", _p), ("cell_offsets", _p),
                ("cellgrid_offsets", _p), ("sigma", _p), ("epsilon", _p), ("guest_types", _p),
                ("guest_sites", _p), ("guest_charges", _p), ("cutoff", _f64), ("ewald_cutoff", _f64),
                ("framework_of", _p)]


class ChainArgs(ctypes.Structure):
    _fields_ = [("Sk", _p), ("const_term", _p), ("guest_offsets", _p), ("guest_sites", _p), ("k_offset", _i64)]


class WidomArgs(ctypes.Structure):
    _fields_ = [("kT", _f64), ("ninsert", _i64), ("seed", _u64), ("nblocks", _i32), ("run", _i32),
                ("reject", _i32), ("rho2", _p), ("reach0", _p), ("segment_begin", _i64), ("segment_end", _i64),
                ("chain", ctypes.POINTER(ChainArgs))]


class BlockSums(ctypes.Structure):
    _fields_ = [("lse_max", _p), ("sum_w", _p), ("sum_uw", _p), ("count", _p), ("segments", _p)]


class InsertionOut(ctypes.Structure):
    _fields_ = [("dU", _p), ("flags", _p), ("poses", _p)]


class Fp32Split(ctypes.Structure):
    _fields_ = [("near_radius", _f64), ("fp64_reciprocal", _i32), ("reserved", _i32)]


class Tuning(ctypes.Structure):
    _fields_ = [("bin_width", _f64), ("ctas_per_sm", _i32), ("use_graphs", _i32)]


class GradSums(ctypes.Structure):
    _fields_ = [("xmax", _p), ("sum_w", _p), ("d_epsilon", _p), ("d_sigma", _p), ("d_charge", _p),
                ("s_guest", _p), ("window", _f64), ("recomputed", _i64), ("lj_only", _i32)]


# (name, restype, argtypes): every entry point the header declares
SIGNATURES = [
    ("pa_context_create", _i32, [_i32, ctypes.POINTER(_p)]),
    ("pa_context_destroy", _i32, [_p]),
    ("pa_context_set_stream", _i32, [_p, _p]),
    ("pa_last_error", ctypes.c_char_p, [_p]),
    ("pa_context_set_timing", _i32, [_p, _i32]),
    ("pa_context_kernel_times", _i32, [_p, _p, _p]),
    ("pa_context_set_tuning", _i32, [_p, ctypes.POINTER(Tuning)]),
    ("pa_context_get_tuning", _i32, [_p, ctypes.POINTER(Tuning)]),
    ("pa_batch_rejection_tables", _i32, [_p, _p, _p, _p, _f64, _f64, _p, _p, _p]),
    ("pa_kvectors", _i32, [_p, _p, _p, _f64, _f64, _f64, _i64, _p, _p, _p, _p, _p]),
    ("pa_kmin_table", _i32, [_p, _p, _i32, _p, _p, _i64, _i32, _p]),
    ("pa_cell_sort", _i32, [_p, _p, _i64, _p, _p, _p]),
    ("pa_context_set_fp32_split", _i32, [_p, ctypes.POINTER(Fp32Split)]),
    ("pa_context_get_fp32_split", _i32, [_p, ctypes.POINTER(Fp32Split)]),
    ("pa_context_fp32_form", _i32, [_p, ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_double)]),
    ("pa_batch_upload", _i32, [_p, ctypes.POINTER(BatchDesc), _i32, ctypes.POINTER(_p)]),
    ("pa_batch_free", _i32, [_p]),
    ("pa_batch_set_pair_tables", _i32, [_p, _p, _p, _p, _p]),
    ("pa_batch_hardcore_bounds", _i32, [_p, _p, _p]),
    ("pa_batch_info", _i32, [_p, ctypes.POINTER(_i64), ctypes.POINTER(_i64)]),
    ("pa_widom", _i32, [_p, _p, ctypes.POINTER(WidomArgs), ctypes.POINTER(BlockSums), ctypes.POINTER(InsertionOut)]),
    ("pa_widom_static", _i32, [_p, _p, ctypes.POINTER(WidomArgs), ctypes.POINTER(BlockSums), ctypes.POINTER(InsertionOut)]),
    ("pa_widom_grad", _i32, [_p, _p, ctypes.POINTER(WidomArgs), ctypes.POINTER(BlockSums), ctypes.POINTER(GradSums),
                             ctypes.POINTER(InsertionOut)]),
    ("pa_rejection_tables", _i32, [ctypes.POINTER(BatchDesc), _p, _p, _f64, _f64, _p, _p, ctypes.POINTER(_i32)]),
    ("pa_segment_count", _i32, [_i64, _i32, _i32, _i32, ctypes.POINTER(_i64)]),
    ("pa_combine_segments", _i32, [_i64, _i32, _i32, _i32, _p, ctypes.POINTER(BlockSums)]),
    ("pa_pose_host", _i32, [_i32, _u64, _u64, _u64, _p, _p]),
    ("pa_self_term", _i32, [_p, _p, _p, _i64, _p, _p, _i32, _i32, _p]),
    ("pa_structure_factor", _i32, [_p, _p, _i64, _p, _p, _i64, _p]),
    ("pa_version", ctypes.c_char_p, []),
]

_lib = None
# live library objects, released in dependency order (batches, then contexts) before the
# interpreter shuts the CUDA runtime down
_live_contexts = weakref.WeakSet()


def _release_all():
    for ctx in list(_live_contexts):
        ctx.close()


atexit.register(_release_all)


def lib():
    """The loaded library (loaded once)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise LibraryMissing(f"{LIB_PATH} is not built; run build.py in the package or __graft_entry__.build()")
        L = ctypes.CDLL(LIB_PATH)
        for name, res, args in SIGNATURES:
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def ptr(a):
    """Raw data pointer of a contiguous numpy array (None for None)."""
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"], "array must be contiguous"
    return a.ctypes.data


def pose_host(precision, seed, s, k):
    """(rpos[3], quat[4]) of insertion k of system s (1-based), drawn on the host by the library."""
    r = np.zeros(3)
    q = np.zeros(4)
    st = lib().pa_pose_host(int(precision), int(seed) & (2**64 - 1), int(s), int(k), ptr(r), ptr(q))
    if st != PA_OK:
        raise PAError(st, "pa_pose_host")
    return r, q


class Context:
    """One CUDA device context of the library (a stream, a workspace, an error slot)."""

    def __init__(self, device=0):
        L = lib()
        h = _p()
        st = L.pa_context_create(int(device), ctypes.byref(h))
        if st != PA_OK:
            raise PAError(st, f"pa_context_create(device={device}) failed (is a CUDA device visible?)")
        self.handle = h.value
        self.device = device
        self.batches = weakref.WeakSet()
        _live_contexts.add(self)

    def check(self, st, what):
        if st != PA_OK:
            msg = lib().pa_last_error(self.handle)
            raise PAError(st, f"{what}: {msg.decode() if msg else ''}")

    def close(self):
        """Frees this context's batches, then the context."""
        for b in list(getattr(self, "batches", ())):
            b.free()
        if self.handle:
            lib().pa_context_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream_ptr):
        self.check(lib().pa_context_set_stream(self.handle, stream_ptr), "pa_context_set_stream")

    def set_timing(self, enable):
        self.check(lib().pa_context_set_timing(self.handle, int(bool(enable))), "pa_context_set_timing")

    def set_tuning(self, bin_width=None, ctas_per_sm=None, use_graphs=None):
        """Changes the given launch choices (pa_tuning); the others keep their values. A new
        bin width applies to batches uploaded afterwards."""
        t = self.tuning()
        if bin_width is not None:
            t.bin_width = float(bin_width)
        if ctas_per_sm is not None:
            t.ctas_per_sm = int(ctas_per_sm)
        if use_graphs is not None:
            t.use_graphs = int(bool(use_graphs))
        self.check(lib().pa_context_set_tuning(self.handle, ctypes.byref(t)), "pa_context_set_tuning")

    def tuning(self):
        t = Tuning()
        self.check(lib().pa_context_get_tuning(self.handle, ctypes.byref(t)), "pa_context_get_tuning")
        return t

    def set_fp32_split(self, near_radius=None, fp64_reciprocal=None):
        """FP32 path (pa_fp32_split): pairs closer than near_radius (Å), and pairs at a cutoff's
        rounding band, are evaluated in FP64 (0 keeps every pair in FP32); fp64_reciprocal selects
        the FP64 reciprocal term. Arguments left None keep their values."""
        sp = self.fp32_split()
        if near_radius is not None:
            sp.near_radius = float(near_radius)
        if fp64_reciprocal is not None:
            sp.fp64_reciprocal = int(bool(fp64_reciprocal))
        self.check(lib().pa_context_set_fp32_split(self.handle, ctypes.byref(sp)), "pa_context_set_fp32_split")

    def fp32_split(self):
        sp = Fp32Split()
        self.check(lib().pa_context_get_fp32_split(self.handle, ctypes.byref(sp)), "pa_context_get_fp32_split")
        return sp

    def fp32_form(self):
        """(exp_free, fit_error) of the last FP32 energy launch: whether its FP32 screened-Coulomb
        pairs took the exp-free form exp(-alpha^2 r^2) u H(u), and the accepted fit's largest
        relative error (pa_context_fp32_form)."""
        ef, err = ctypes.c_int32(0), ctypes.c_double(0.0)
        self.check(lib().pa_context_fp32_form(self.handle, ctypes.byref(ef), ctypes.byref(err)), "pa_context_fp32_form")
        return bool(ef.value), float(err.value)

    def kernel_times(self):
        ms = np.zeros(8)
        n = np.zeros(8, dtype=np.int64)
        self.check(lib().pa_context_kernel_times(self.handle, ptr(ms), ptr(n)), "pa_context_kernel_times")
        return ms, n

    def batch_bounds(self, batch):
        """Hard-core bounds B_s of every framework of `batch` from the device
        (pa_batch_hardcore_bounds), through the batch's upload to this context, which later calls
        reuse; for FrameworkBatch(..., bounds=ctx.batch_bounds)."""
        return batch.device(self).hardcore_bounds(batch.nframeworks())

    def self_term(self, ks, kpref, sites, charges):
        """Σ_k kpref |Σ_s q_s e^{i k·g_s(o)}|^2 for every orientation o of `sites` (norient x N x 3),
        on the device (pa_self_term)."""
        ks = np.ascontiguousarray(ks, dtype=np.float64).reshape(-1, 3)
        w = np.ascontiguousarray(kpref, dtype=np.float64)
        g = np.ascontiguousarray(sites, dtype=np.float64)
        q = np.ascontiguousarray(charges, dtype=np.float64)
        no, N = g.shape[0], g.shape[1]
        out = np.zeros(no)
        self.check(lib().pa_self_term(self.handle, ptr(ks), ptr(w), len(ks), ptr(g), ptr(q), N, no, ptr(out)),
                   "pa_self_term")
        return out

    def structure_factor(self, ks, positions, charges):
        ks = np.ascontiguousarray(ks, dtype=np.float64).reshape(-1, 3)
        pos = np.ascontiguousarray(positions, dtype=np.float64).reshape(-1, 3)
        q = np.ascontiguousarray(charges, dtype=np.float64)
        S = np.zeros(2 * len(ks))
        self.check(lib().pa_structure_factor(self.handle, ptr(ks), len(ks), ptr(pos), ptr(q), len(q), ptr(S)),
                   "pa_structure_factor")
        return S[0::2] + 1j * S[1::2]


    def kvectors(self, B, nmax, kmax, alpha, V):
        """The half-space k-vectors of one cell on the device (pa_kvectors): (ks (nk, 3), weights,
        kpref, coefficients (nk, 3)) in enumeration order, from the reciprocal basis B (3 x 3), the
        bounds nmax (3) and the cell's volume V; kpref = w 2 pi / V exp(-k^2 / 4 alpha^2) / k^2."""
        Bc = np.ascontiguousarray(B, dtype=np.float64).reshape(9)
        nm = np.ascontiguousarray(nmax, dtype=np.int32).reshape(3)
        cap = max(1, int((nm[0] + 1) * (2 * nm[1] + 1) * (2 * nm[2] + 1)) - 1)
        ks, w, kp = np.zeros(3 * cap), np.zeros(cap), np.zeros(cap)
        co = np.zeros(3 * cap, dtype=np.int32)
        nk = _i64()
        self.check(lib().pa_kvectors(self.handle, ptr(Bc), ptr(nm), float(kmax), 2 * math.pi / float(V),
                                     4 * float(alpha) ** 2, cap, ptr(ks), ptr(w), ptr(kp), ptr(co), ctypes.byref(nk)),
                   "pa_kvectors")
        n = nk.value
        return ks[:3 * n].reshape(n, 3), w[:n], kp[:n], co[:3 * n].reshape(n, 3)

    def kmin_table(self, guest_charges, types, charges, ntypes):
        """kmin (N x ntypes) of one framework's atoms (types 1-based) on the device (pa_kmin_table)."""
        g = np.ascontiguousarray(guest_charges, dtype=np.float64)
        t = np.ascontiguousarray(types, dtype=np.int32)
        q = np.ascontiguousarray(charges, dtype=np.float64)
        out = np.zeros(len(g) * int(ntypes))
        self.check(lib().pa_kmin_table(self.handle, ptr(g), len(g), ptr(t), ptr(q), len(q), int(ntypes), ptr(out)),
                   "pa_kmin_table")
        return out.reshape(len(g), int(ntypes))

    def cell_sort(self, frac, n):
        """(permutation, prod(n)+1 offsets) of the stable cell sort of one framework's atoms on the
        device (pa_cell_sort)."""
        f = np.ascontiguousarray(frac, dtype=np.float64).reshape(-1, 3)
        nn = np.ascontiguousarray(n, dtype=np.int32).reshape(3)
        perm = np.zeros(len(f), dtype=np.int64)
        off = np.zeros(int(nn[0]) * int(nn[1]) * int(nn[2]) + 1, dtype=np.int32)
        self.check(lib().pa_cell_sort(self.handle, ptr(f), len(f), ptr(nn), ptr(perm), ptr(off)), "pa_cell_sort")
        return perm, off


class DeviceBatch:
    """A batch uploaded to a context for one precision (pa_batch)."""

    def __init__(self, ctx, desc, keep, precision):
        self.ctx = ctx
        h = _p()
        ctx.check(lib().pa_batch_upload(ctx.handle, ctypes.byref(desc), int(precision), ctypes.byref(h)),
                  "pa_batch_upload")
        self.handle = h.value
        self.precision = precision
        self._keep = keep
        ctx.batches.add(self)

    def set_pair_tables(self, sigma, epsilon, constant_offset):
        """Replaces the LJ pair tables (nt x nt) and constant offsets (nfw) in place."""
        sg = np.ascontiguousarray(np.asarray(sigma, dtype=np.float64).T.reshape(-1))
        ep = np.ascontiguousarray(np.asarray(epsilon, dtype=np.float64).T.reshape(-1))
        co = np.ascontiguousarray(constant_offset, dtype=np.float64)
        self.ctx.check(lib().pa_batch_set_pair_tables(self.ctx.handle, self.handle, ptr(sg), ptr(ep), ptr(co)),
                       "pa_batch_set_pair_tables")

    def hardcore_bounds(self, nfw):
        """Hard-core bound of every framework from the uploaded pair tables, on the device."""
        bs = np.zeros(nfw)
        self.ctx.check(lib().pa_batch_hardcore_bounds(self.ctx.handle, self.handle, ptr(bs)), "pa_batch_hardcore_bounds")
        return bs

    def rejection_tables(self, bs, kmin, kT, eps_F, nsys, N, nt):
        """Rejection radii (nsys*N*nt) and stencil reaches (nsys x 3) of one call, the root searches
        on the device (pa_batch_rejection_tables); returns (rho2, reach0, bad system or 0)."""
        b = np.ascontiguousarray(bs, dtype=np.float64)
        k = np.ascontiguousarray(kmin, dtype=np.float64)
        rho2 = np.zeros(nsys * N * nt)
        reach0 = np.zeros((nsys, 3), dtype=np.int32)
        bad = _i32(0)
        st = lib().pa_batch_rejection_tables(self.ctx.handle, self.handle, ptr(b), ptr(k), float(kT), float(eps_F),
                                             ptr(rho2), ptr(reach0), ctypes.byref(bad))
        if st != PA_OK and bad.value == 0:
            self.ctx.check(st, "pa_batch_rejection_tables")
        return rho2, reach0, bad.value

    def info(self):
        a, b = _i64(), _i64()
        lib().pa_batch_info(self.handle, ctypes.byref(a), ctypes.byref(b))
        return a.value, b.value

    def free(self):
        if self.handle:
            lib().pa_batch_free(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass
