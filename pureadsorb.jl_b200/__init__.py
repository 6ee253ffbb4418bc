"""B200-native batched Widom insertion with the API of PureAdsorb.jl's `widom` path.

Public names mirror the reference's exports for this path (src/PureAdsorb.jl:33-37):
Framework, read_cif, replicate, ForceField, read_forcefield, Guest, read_guest, EwaldParams,
FrameworkBatch, widom, WidomResult; plus B200Backend, the device backend object.
"""
from .batch import FrameworkBatch, nframeworks
from .cell import cell_matrix, min_multiplicity, minimum_image, perpendicular_lengths, volume
from .constants import KB, KE
from .errors import ArgumentError, DimensionMismatch
from .ewald import EwaldParams, ewald_alpha, ewald_kmax, full_ktables, kvectors, pk, structure_factor
from .forcefield import ForceField, Guest, read_forcefield, read_guest, tail_delta
from .structure import Framework, cartesian, natoms, read_cif, replicate, total_charge
from . import synthetic
from . import adjoint
from .adjoint import WidomGrad, fold_replicas, widom_grad
from .tune import TuneReport, autotune
from . import fit
from . import chain
from . import cli
from .chain import SystemState, insertion_constant_term, widom_along_chain, widom_chain
from .widom import (B200Backend, WidomResult, _reduce, _widom, block_sums, boltzmann_weight, build_rejection_tables,
                    default_run, sys_of_index, system_counts, widom, widom_singlephase)

__all__ = ["Framework", "read_cif", "replicate", "ForceField", "read_forcefield", "Guest", "read_guest",
           "EwaldParams", "FrameworkBatch", "widom", "WidomResult", "B200Backend", "widom_grad", "WidomGrad",
           "SystemState", "widom_chain", "widom_along_chain", "insertion_constant_term"]
