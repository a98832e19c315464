// FP64 spline-table build for the projected potential of potential_type 1-4 and 6 (see tables.cu).
#pragma once

#include <cuda_runtime.h>

#include <vector>

namespace mtb {

struct TableHead {
    double R_min, R_max, R_tap, tap_cf;
};

// potential_type values with a table build: 1-4 (Doyle-Turner, Peng 0-4, Peng 0-12, Kirkland) and
// 6 (Lobato)
bool potential_type_supported(int type);

// The charge whose coefficients an atom of element Z and charge q uses: q when Peng's ionic table
// has an entry for it, else 0 (neutral), as Atom_Type::charge_to_idx (src/types.cuh:4125-4137).
int effective_charge(int Z, int charge);

// FP64 header of element Z on the host: R_min = max(dR_min, rn_c), R_max from the Vr = Vrl root,
// R_tap and the taper factor (Atomic_Data::get_atom_coef, src/atomic_data.hpp:1590-1620).
TableHead element_head(int Z, int potential_type, float dR_min, float Vrl);

// Build the spline tables of the elements in Zs (with their heads; charges[i] the ionic charge of
// entry i, all neutral when empty; an ion's head is its element's) on the device in FP64. d_tab
// receives, per element, 5*nR floats: R2[nR], c0[nR], c1[nR], c2[nR], c3[nR] (the float tables
// the splat evaluates). Synchronises `stream`.
void build_tables(const std::vector<int>& Zs, int potential_type, const std::vector<TableHead>& heads, int nR,
                  float* d_tab, cudaStream_t stream, const std::vector<int>& charges = {});

// Same build without allocating: the kernel's scratch is a fixed file-scope device array (at most
// 128 elements per call), d_tab is the caller's device buffer, and the work is only enqueued on
// `stream` (no synchronisation). Calls that overlap on the GPU race on the shared scratch.
void build_tables_noalloc(const std::vector<int>& Zs, int potential_type, const std::vector<TableHead>& heads,
                          int nR, float* d_tab, cudaStream_t stream, const std::vector<int>& charges = {});

}  // namespace mtb
