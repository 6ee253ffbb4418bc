"""ctypes wrapper of the oracle (oracle.cpp) — TEST INFRASTRUCTURE ONLY.

Imported only by tests/, __graft_entry__.smoke() (as the checker) and bench.py's CPU-baseline
leg. It restates PureAdsorb.jl's Widom path on the CPU in FP64; see the header of oracle.cpp
for the reference files it follows and the known-answer tests that pin it.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "liboracle.so")

_p = ctypes.c_void_p
_i32, _i64, _u64, _f64 = ctypes.c_int32, ctypes.c_int64, ctypes.c_uint64, ctypes.c_double


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB


class BatchView(ctypes.Structure):
    _fields_ = [("nsys", _i32), ("nfw", _i32), ("ntypes", _i32), ("nguest", _i32),
                ("positions", _p), ("types", _p), ("charges", _p), ("atom_offsets", _p),
                ("cells", _p), ("invcells", _p), ("volumes", _p), ("alphas", _p),
                ("ks", _p), ("kprefactor", _p), ("Shost", _p), ("k_offsets", _p),
                ("constant_offset", _p), ("ncells", _p), ("cell_offsets", _p), ("cellgrid_offsets", _p),
                ("sigma", _p), ("epsilon", _p), ("guest_types", _p), ("guest_sites", _p), ("guest_charges", _p),
                ("cutoff", _f64), ("ewald_cutoff", _f64), ("framework_of", _p)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(os.path.join(HERE, "oracle.cpp")):
            build()
        L = ctypes.CDLL(LIB)
        sig = {
            "or_splitmix64": (_u64, [_u64, _u64]), "or_mulhi64": (_u64, [_u64, _u64]),
            "or_chain_bits": (_u64, [_u64, _u64, _u64, _u64]), "or_unit_f64": (_f64, [_u64]),
            "or_unit_f32": (ctypes.c_float, [_u64]), "or_rand_range": (_i64, [_u64, _i64]),
            "or_sincos2pi_f64": (None, [_p, _i64, _p, _p]), "or_sincos2pi_f32": (None, [_p, _i64, _p, _p]),
            "or_poses_f64": (None, [_u64, _i64, _i64, _i64, _p, _p]),
            "or_poses_f32": (None, [_u64, _i64, _i64, _i64, _p, _p]),
            "or_theta_f64": (_f64, []), "or_theta_f32": (ctypes.c_float, []), "or_erfc": (_f64, [_f64]),
            "or_ewald_alpha": (_f64, [_f64, _f64]), "or_ewald_kmax": (_f64, [_f64, _f64]),
            "or_pk": (_f64, [_f64, _f64, _f64]),
            "or_kvectors": (_i64, [_p, _f64, _p, _p, _p, _i64]),
            "or_structure_factor": (None, [_p, _i64, _p, _p, _i64, _p]),
            "or_ewald_energy": (_f64, [_p, _p, _p, _p, _i64, _f64, _f64, _p, _p, _i64]),
            "or_find_r0": (_f64, [_f64, _f64, _f64, _f64, _f64, ctypes.POINTER(ctypes.c_int)]),
            "or_find_rho2": (_f64, [_f64, _f64, _f64, _f64, _f64, ctypes.POINTER(ctypes.c_int)]),
            "or_pair_energy": (_f64, [_f64, _f64, _f64, _f64, _f64]),
            "or_batch_build": (_p, [_i32, _p, _p, _p, _p, _p, _p, _i32, _p, _p, _f64, _i32, _i32, _p, _p, _p,
                                    _f64, _f64, _f64, _i32, _i32, _p]),
            "or_batch_error": (ctypes.c_char_p, [_p]), "or_batch_free": (None, [_p]),
            "or_batch_field": (_i64, [_p, ctypes.c_char_p, _p]),
            "or_system_counts": (_i64, [_i64, _i64, _i64, _p]), "or_sys_of_index": (_i32, [_i64, _i64, _i64]),
            "or_widom": (ctypes.c_int, [ctypes.POINTER(BatchView), _i32, _f64, _i64, _u64, _i32, _i64, _i32, _p, _p,
                                        _p, _p, _p, _p, _p, _p, _p, _i32]),
            "or_insertion_energy": (None, [ctypes.POINTER(BatchView), _i32, _i64, _p, _p, _p]),
            "or_chain_energy": (None, [ctypes.POINTER(BatchView), _i32, _i64, _p, _p, _i64, _p, _p]),
            "or_insertion_energy_reference": (_f64, [_p, _p, _i32, _p, _p, _p, _i32, _p, _p, _f64, _f64, _i64, _p,
                                                     _p, _p, _p, _f64, _i64, _p, _p, _p]),
            "or_hardcore_flags": (None, [ctypes.POINTER(BatchView), _i32, _i32, _i64, _p, _p, _p, _p, _i32, _p]),
            "or_rejection_tables": (_i32, [ctypes.POINTER(BatchView), _p, _p, _f64, _f64, _p, _p]),
            "or_grad_sums": (ctypes.c_int, [ctypes.POINTER(BatchView), _f64, _i64, _i64, _p, _p, _p, _p, _p, _p, _p,
                                            _p, _p, _i32]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def P(a):
    return None if a is None else a.ctypes.data


def c64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def c32i(a):
    return np.ascontiguousarray(a, dtype=np.int32)


# ---------------------------------------------------------------------------------------------
# small functions
# ---------------------------------------------------------------------------------------------
def poses(precision, seed, s, k0, n):
    """(rpos (n,3), quat (n,4)) of insertions k0..k0+n-1 of system s, widened to FP64."""
    if precision == 32:
        r = np.zeros((n, 3), np.float32)
        q = np.zeros((n, 4), np.float32)
        lib().or_poses_f32(seed, s, k0, n, P(r), P(q))
    else:
        r = np.zeros((n, 3))
        q = np.zeros((n, 4))
        lib().or_poses_f64(seed, s, k0, n, P(r), P(q))
    return r.astype(np.float64), q.astype(np.float64)


def kvectors(A, kmax):
    A = c64(np.asarray(A).T.reshape(-1))  # column-major
    n = lib().or_kvectors(P(A), kmax, None, None, None, 0)
    ks = np.zeros((n, 3))
    w = np.zeros(n)
    co = np.zeros((n, 3), np.int32)
    lib().or_kvectors(P(A), kmax, P(ks), P(w), P(co), n)
    return ks, w, co


def structure_factor(ks, pos, q):
    ks, pos, q = c64(ks), c64(pos), c64(q)
    S = np.zeros(2 * len(ks))
    lib().or_structure_factor(P(ks), len(ks), P(pos), P(q), len(q), P(S))
    return S[0::2] + 1j * S[1::2]


def ewald_energy(A, pos, q, mol, alpha, cutoff, ks, w):
    A = c64(np.asarray(A).T.reshape(-1))
    pos, q, ks, w = c64(pos), c64(q), c64(ks), c64(w)
    mol = c32i(mol)
    return lib().or_ewald_energy(P(A), P(pos), P(q), P(mol), len(q), alpha, cutoff, P(ks), P(w), len(w))


def find_r0(s, e, K, alpha, r_lj):
    err = ctypes.c_int(0)
    v = lib().or_find_r0(s, e, K, alpha, r_lj, ctypes.byref(err))
    if err.value:
        raise ValueError(f"find_r0 error {err.value}")
    return v


def find_rho2(s, e, kmin, margin, r_lj):
    err = ctypes.c_int(0)
    v = lib().or_find_rho2(s, e, kmin, margin, r_lj, ctypes.byref(err))
    if err.value:
        raise ValueError(f"find_rho2 error {err.value}")
    return v


# ---------------------------------------------------------------------------------------------
# batch construction (src/batch.jl:237-432)
# ---------------------------------------------------------------------------------------------
class OracleBatch:
    """The oracle's own FrameworkBatch, as numpy arrays in the reference layout."""

    FIELDS = ["positions", "types", "charges", "atom_offsets", "cells", "invcells", "volumes", "alphas", "ks",
              "kprefactor", "Shost", "kcoeffs", "k_offsets", "constant_offset", "self_term_halfrange", "ncells",
              "cell_offsets", "cellgrid_offsets", "sigma", "epsilon", "compact_to_orig", "guest_types", "bs", "kmin",
              "framework_of", "perm"]
    INT = {"types", "atom_offsets", "kcoeffs", "k_offsets", "ncells", "cell_offsets", "cellgrid_offsets",
           "compact_to_orig", "guest_types", "framework_of", "perm"}

    def __init__(self, frameworks, ff_names_sigma_eps, guest, ewald_cutoff, ewald_precision, cellwidth=2.0,
                 fullk=False, self_quats=None):
        """frameworks: list of (cell 3x3, frac (n,3), orig types (1-based), charges, replication);
        ff_names_sigma_eps: (sigma per type, epsilon per type, cutoff, tail);
        guest: (sites (N,3), orig types (1-based), charges)."""
        cells = c64(np.concatenate([np.asarray(f[0]).T.reshape(-1) for f in frameworks]))
        natoms = np.array([len(f[1]) for f in frameworks], dtype=np.int64)
        frac = c64(np.concatenate([np.asarray(f[1]).reshape(-1) for f in frameworks]))
        types = c32i(np.concatenate([np.asarray(f[2]).reshape(-1) for f in frameworks]))
        charges = c64(np.concatenate([np.asarray(f[3]).reshape(-1) for f in frameworks]))
        rep = c32i(np.concatenate([np.asarray(f[4]).reshape(-1) for f in frameworks]))
        sig, eps, cutoff, tail = ff_names_sigma_eps
        sig, eps = c64(sig), c64(eps)
        gs, gt, gq = c64(np.asarray(guest[0]).reshape(-1)), c32i(guest[1]), c64(guest[2])
        sq = c64(np.asarray(self_quats).reshape(-1)) if self_quats is not None else c64(np.zeros(0))
        nself = 0 if self_quats is None else len(self_quats)
        self.h = lib().or_batch_build(len(frameworks), P(cells), P(natoms), P(frac), P(types), P(charges), P(rep),
                                      len(sig), P(sig), P(eps), cutoff, int(tail), len(gq), P(gs), P(gt), P(gq),
                                      ewald_cutoff, ewald_precision, cellwidth, int(fullk), nself, P(sq))
        err = lib().or_batch_error(self.h).decode()
        if err:
            lib().or_batch_free(self.h)
            raise ValueError(err)
        for f in self.FIELDS:
            n = lib().or_batch_field(self.h, f.encode(), None)
            a = np.zeros(n, dtype=np.int32 if f in self.INT else np.float64)
            lib().or_batch_field(self.h, f.encode(), P(a))
            setattr(self, f, a)
        self.ntypes = lib().or_batch_field(self.h, b"ntypes", None)
        self.nsys = lib().or_batch_field(self.h, b"nsys", None)
        self.nfw = lib().or_batch_field(self.h, b"nfw", None)
        self.Shost = self.Shost[0::2] + 1j * self.Shost[1::2]
        self.positions = self.positions.reshape(-1, 3)
        self.ks = self.ks.reshape(-1, 3)
        self.kcoeffs = self.kcoeffs.reshape(-1, 3)
        self.cells = self.cells.reshape(-1, 3, 3).transpose(0, 2, 1)
        self.invcells = self.invcells.reshape(-1, 3, 3).transpose(0, 2, 1)
        nt = self.ntypes
        self.sigma = self.sigma.reshape(nt, nt).T
        self.epsilon = self.epsilon.reshape(nt, nt).T
        self.ncells = self.ncells.reshape(-1, 3)
        lib().or_batch_free(self.h)
        self.h = None


# ---------------------------------------------------------------------------------------------
# widom over any batch in the reference layout (product FrameworkBatch or OracleBatch)
# ---------------------------------------------------------------------------------------------
def view(b, guest_sites, guest_charges, cutoff, ewald_cutoff):
    """(BatchView, keep-alive arrays) of a batch object with the reference's field names."""
    col = lambda M: c64(np.transpose(np.asarray(M), (0, 2, 1)).reshape(-1))
    arr = dict(positions=c64(np.asarray(b.positions).reshape(-1)), types=c32i(b.types), charges=c64(b.charges),
               atom_offsets=c32i(b.atom_offsets), cells=col(b.cells), invcells=col(b.invcells), volumes=c64(b.volumes),
               alphas=c64(b.alphas), ks=c64(np.asarray(b.ks).reshape(-1)), kprefactor=c64(b.kprefactor),
               Shost=c64(np.stack([np.real(b.Shost), np.imag(b.Shost)], axis=1).reshape(-1)),
               k_offsets=c32i(b.k_offsets), constant_offset=c64(b.constant_offset),
               ncells=c32i(np.asarray(b.ncells).reshape(-1)), cell_offsets=c32i(b.cell_offsets),
               cellgrid_offsets=c32i(b.cellgrid_offsets), sigma=c64(np.asarray(b.sigma).T.reshape(-1)),
               epsilon=c64(np.asarray(b.epsilon).T.reshape(-1)), guest_types=c32i(b.guest_types),
               guest_sites=c64(np.asarray(guest_sites).reshape(-1)), guest_charges=c64(guest_charges),
               framework_of=c32i(b.framework_of))
    v = BatchView()
    v.nsys, v.nfw = int(len(b.framework_of)), int(len(b.volumes))
    v.ntypes, v.nguest = int(np.asarray(b.sigma).shape[0]), int(len(b.guest_types))
    for k, a in arr.items():
        setattr(v, k, P(a) if a.size else None)
    v.cutoff, v.ewald_cutoff = cutoff, ewald_cutoff
    return v, arr


def rejection_tables(v, bs, kmin, kT, eps_F):
    N, nt = v.nguest, v.ntypes
    rho2 = np.zeros(v.nsys * N * nt)
    reach0 = np.zeros(3 * v.nsys, np.int32)
    bs, kmin = c64(bs), c64(kmin)
    st = lib().or_rejection_tables(ctypes.byref(v), P(bs), P(kmin), kT, eps_F, P(rho2), P(reach0))
    if st != 0:
        raise ValueError(f"rejection tables failed for system {abs(st)}")
    return rho2, reach0.reshape(-1, 3)


def widom(v, precision, kT, ninsert, seed, nblocks, run, reject, rho2=None, reach0=None, nthreads=0,
          want_insertions=True):
    """Runs the oracle's widom path. Returns dict with sW, sUW, n (nsys x nblocks) and, if
    requested, per-insertion dU/flags/poses (system-major sample order) and pair counts."""
    nsys = v.nsys
    sW = np.zeros(nsys * nblocks)
    sUW = np.zeros(nsys * nblocks)
    n = np.zeros(nsys * nblocks, np.int64)
    dU = np.zeros(ninsert) if want_insertions else None
    flags = np.zeros(ninsert, np.uint8) if want_insertions else None
    poses_out = np.zeros((ninsert, 7)) if want_insertions else None
    pairs = np.zeros(2, np.int64)
    r2 = None if rho2 is None else c64(rho2)
    r0 = None if reach0 is None else c32i(np.asarray(reach0).reshape(-1))
    st = lib().or_widom(ctypes.byref(v), precision, kT, ninsert, seed & (2**64 - 1), nblocks, run, int(reject), P(r2),
                        P(r0), P(sW), P(sUW), P(n), P(dU), P(flags), P(poses_out), P(pairs), nthreads)
    if st != 0:
        raise ValueError(f"or_widom failed ({st})")
    out = dict(sW=sW.reshape(nsys, nblocks), sUW=sUW.reshape(nsys, nblocks), n=n.reshape(nsys, nblocks), pairs=pairs)
    if want_insertions:
        out.update(dU=dU, flags=flags, poses=poses_out)
    return out


def grad_sums(v, kT, ninsert, run, out, natoms_of, nk_of, nthreads=0):
    """Adjoint sums of one widom() result (its dU, flags and poses, system-major): per system
    xmax, sum_w, d_eps/d_sig (N x nt), d_charge (the system's framework atoms) and s_guest
    (complex per k-vector). natoms_of/nk_of: per-system atom and k-vector counts."""
    nsys, N, nt = v.nsys, v.nguest, v.ntypes
    na, nk = int(np.sum(natoms_of)), int(np.sum(nk_of))
    xmax, sum_w = np.zeros(nsys), np.zeros(nsys)
    d_eps, d_sig = np.zeros(nsys * N * nt), np.zeros(nsys * N * nt)
    d_q, sg = np.zeros(na), np.zeros(2 * nk)
    dU, flags, poses = c64(out["dU"]), np.ascontiguousarray(out["flags"], dtype=np.uint8), c64(out["poses"])
    st = lib().or_grad_sums(ctypes.byref(v), kT, ninsert, run, P(poses), P(dU), P(flags), P(xmax), P(sum_w),
                            P(d_eps), P(d_sig), P(d_q), P(sg), nthreads)
    if st != 0:
        raise ValueError(f"or_grad_sums failed ({st})")
    aoff = np.concatenate([[0], np.cumsum(natoms_of)]).astype(np.int64)
    koff = np.concatenate([[0], np.cumsum(nk_of)]).astype(np.int64)
    sgc = sg[0::2] + 1j * sg[1::2]
    return [dict(xmax=xmax[s], sum_w=sum_w[s], d_epsilon=d_eps.reshape(nsys, N, nt)[s],
                 d_sigma=d_sig.reshape(nsys, N, nt)[s], d_charge=d_q[aoff[s]:aoff[s + 1]],
                 s_guest=sgc[koff[s]:koff[s + 1]]) for s in range(nsys)]


def insertion_energy(v, fw, pos, quat):
    pos, quat = c64(np.asarray(pos).reshape(-1)), c64(np.asarray(quat).reshape(-1))
    n = len(pos) // 3
    out = np.zeros(n)
    lib().or_insertion_energy(ctypes.byref(v), fw, n, P(pos), P(quat), P(out))
    return out


def hardcore_flags(v, precision, s, rpos, quat, rho2, reach0, brute=False):
    rpos, quat = c64(np.asarray(rpos).reshape(-1)), c64(np.asarray(quat).reshape(-1))
    r2, r0 = c64(rho2), c32i(np.asarray(reach0).reshape(-1))
    n = len(rpos) // 3
    out = np.zeros(n, np.uint8)
    lib().or_hardcore_flags(ctypes.byref(v), precision, s, n, P(rpos), P(quat), P(r2), P(r0), int(brute), P(out))
    return out


def chain_energy(v, fw, pos, quat, gsites):
    """widom_chain_kernel!'s energy without the constant term at explicit poses of system fw (the
    view's Shost being that system's running S(k)); gsites: the live guests' sites (ng, N, 3)."""
    pos, quat = c64(np.asarray(pos).reshape(-1)), c64(np.asarray(quat).reshape(-1))
    g = c64(np.asarray(gsites).reshape(-1)) if np.asarray(gsites).size else c64(np.zeros(3))
    ng = int(np.asarray(gsites).size // (3 * v.nguest))
    n = len(pos) // 3
    out = np.zeros(n)
    lib().or_chain_energy(ctypes.byref(v), fw, n, P(pos), P(quat), ng, P(g), P(out))
    return out
