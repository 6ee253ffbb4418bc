"""Command-line Widom insertion from input files, without writing Python: P1 CIF frameworks,
a kUPS-style YAML force field and guest (the reference's readers, src/structure.jl:37-92 and
src/forcefield.jl:54-101), one FrameworkBatch, one widom call on a B200, one JSON line per system.

    python pureadsorb.jl_b200 widom --cif A.cif [--cif B.cif ...] --forcefield ff.yaml \\
        --guest co2.yaml --T 298.15 --ninsert 1000000 [--seed 0] [--nblocks 10] [--float32]

Each framework is replicated to the smallest supercell whose opposite faces are 2 (r_c + r_guest)
apart (the guard FrameworkBatch applies, src/batch.jl:252-265), unless --replicate gives the
factors. The Ewald real-space cutoff defaults to the force field's LJ cutoff."""
import argparse
import json
import math
import sys

import numpy as np

from .batch import FrameworkBatch
from .cell import min_multiplicity
from .errors import ArgumentError
from .ewald import EwaldParams
from .forcefield import read_forcefield, read_guest
from .structure import read_cif, replicate
from .widom import B200Backend, widom


def parser():
    p = argparse.ArgumentParser(prog="pureadsorb.jl_b200", description=__doc__.split("\n\n")[0])
    sub = p.add_subparsers(dest="command", required=True)
    w = sub.add_parser("widom", help="Henry coefficient, excess chemical potential and heat of adsorption")
    w.add_argument("--cif", action="append", required=True, help="P1 CIF framework (repeat for a batch)")
    w.add_argument("--forcefield", required=True, help="kUPS-style YAML force field")
    w.add_argument("--guest", required=True, help="kUPS-style YAML rigid guest")
    w.add_argument("--T", type=float, required=True, help="temperature (K)")
    w.add_argument("--ninsert", type=int, required=True, help="insertions over all systems")
    w.add_argument("--seed", type=int, default=0)
    w.add_argument("--nblocks", type=int, default=10)
    w.add_argument("--run", type=int, default=None, help="consecutive insertions per system (default as widom)")
    w.add_argument("--replicate", type=int, nargs=3, default=None, metavar=("NA", "NB", "NC"),
                   help="supercell factors for every framework (default: the smallest that passes the guard)")
    w.add_argument("--ewald-cutoff", type=float, default=None, help="real-space Ewald cutoff (A); default: LJ cutoff")
    w.add_argument("--ewald-precision", type=float, default=1.0e-6)
    w.add_argument("--float32", action="store_true", help="the FP32 path (default: FP64)")
    w.add_argument("--device", type=int, default=0)
    return p


def build_inputs(args):
    """(frameworks, force field, guest, Ewald parameters) from the command's files (host only)."""
    T = np.float32 if args.float32 else np.float64
    ff = read_forcefield(args.forcefield, T=T)
    guest = read_guest(args.guest, ff, T=T)
    ewald = EwaldParams(args.ewald_cutoff if args.ewald_cutoff is not None else ff.cutoff, args.ewald_precision)
    rc = max(ff.cutoff, ewald.cutoff)
    r_guest = float(np.max(np.linalg.norm(guest.sites, axis=1))) if len(guest.sites) else 0.0
    fws = []
    for path in args.cif:
        fw = read_cif(path, T=T)
        n = tuple(args.replicate) if args.replicate is not None else min_multiplicity(fw.cell, rc + r_guest)
        fws.append(replicate(fw, n) if n != (1, 1, 1) else fw)
    return fws, ff, guest, ewald


def result_record(path, r):
    return {"framework": path, "mu_ex_eV": r.mu_ex, "mu_ex_err_eV": r.mu_ex_err, "K_H": r.K_H,
            "K_H_err": r.K_H_err, "q_st_eV": r.q_st, "q_st_err_eV": r.q_st_err, "nsamples": r.nsamples,
            "nblocks": r.nblocks}


def main(argv=None, out=None):
    out = out or sys.stdout
    args = parser().parse_args(argv)
    try:
        fws, ff, guest, ewald = build_inputs(args)
        T = np.float32 if args.float32 else np.float64
        batch = FrameworkBatch(fws, ff, guest, ewald, T=T)
        res = widom(batch, guest, T=args.T, ninsert=args.ninsert, seed=args.seed, nblocks=args.nblocks,
                    run=args.run, backend=B200Backend(args.device))
    except ArgumentError as e:
        print(f"error: {e}", file=sys.stderr)
        return 2
    for path, r in zip(args.cif, res):
        rec = result_record(path, r)
        out.write(json.dumps({k: (v if not (isinstance(v, float) and not math.isfinite(v)) else str(v))
                              for k, v in rec.items()}) + "\n")
    return 0
