/* Prints the size and field offsets of every struct of the library's C ABI
 * (include/pureadsorb_b200.h), one line each: "struct <name> <sizeof>" and
 * "field <struct> <field> <offsetof>". Built and read by tests/test_abi_layout.py, which compares
 * them with the Python ctypes mirrors (pureadsorb.jl_b200/_lib.py) and with the Julia structs of
 * the binding in INTEGRATION.md. */
#include <stddef.h>
#include <stdio.h>

#include "pureadsorb_b200.h"

#define S(T) printf("struct %s %zu\n", #T, sizeof(T))
#define F(T, f) printf("field %s %s %zu\n", #T, #f, offsetof(T, f))

int main(void) {
    S(pa_tuning); F(pa_tuning, bin_width); F(pa_tuning, ctas_per_sm); F(pa_tuning, use_graphs);
    S(pa_fp32_split); F(pa_fp32_split, near_radius); F(pa_fp32_split, fp64_reciprocal); F(pa_fp32_split, reserved);
    S(pa_batch_desc);
    F(pa_batch_desc, nsys); F(pa_batch_desc, nfw); F(pa_batch_desc, ntypes); F(pa_batch_desc, nguest);
    F(pa_batch_desc, positions); F(pa_batch_desc, types); F(pa_batch_desc, charges); F(pa_batch_desc, atom_offsets);
    F(pa_batch_desc, cells); F(pa_batch_desc, invcells); F(pa_batch_desc, volumes); F(pa_batch_desc, alphas);
    F(pa_batch_desc, ks); F(pa_batch_desc, kprefactor); F(pa_batch_desc, Shost); F(pa_batch_desc, kcoeffs);
    F(pa_batch_desc, k_offsets); F(pa_batch_desc, constant_offset); F(pa_batch_desc, ncells);
    F(pa_batch_desc, cell_offsets); F(pa_batch_desc, cellgrid_offsets); F(pa_batch_desc, sigma);
    F(pa_batch_desc, epsilon); F(pa_batch_desc, guest_types); F(pa_batch_desc, guest_sites);
    F(pa_batch_desc, guest_charges); F(pa_batch_desc, cutoff); F(pa_batch_desc, ewald_cutoff);
    F(pa_batch_desc, framework_of);
    S(pa_chain_args); F(pa_chain_args, Sk); F(pa_chain_args, const_term); F(pa_chain_args, guest_offsets);
    F(pa_chain_args, guest_sites); F(pa_chain_args, k_offset);
    S(pa_widom_args); F(pa_widom_args, kT); F(pa_widom_args, ninsert); F(pa_widom_args, seed);
    F(pa_widom_args, nblocks); F(pa_widom_args, run); F(pa_widom_args, reject); F(pa_widom_args, rho2);
    F(pa_widom_args, reach0); F(pa_widom_args, segment_begin); F(pa_widom_args, segment_end);
    F(pa_widom_args, chain);
    S(pa_block_sums); F(pa_block_sums, lse_max); F(pa_block_sums, sum_w); F(pa_block_sums, sum_uw);
    F(pa_block_sums, count); F(pa_block_sums, segments);
    S(pa_insertion_out); F(pa_insertion_out, dU); F(pa_insertion_out, flags); F(pa_insertion_out, poses);
    S(pa_grad_sums); F(pa_grad_sums, xmax); F(pa_grad_sums, sum_w); F(pa_grad_sums, d_epsilon);
    F(pa_grad_sums, d_sigma); F(pa_grad_sums, d_charge); F(pa_grad_sums, s_guest); F(pa_grad_sums, window);
    F(pa_grad_sums, recomputed); F(pa_grad_sums, lj_only);
    return 0;
}
