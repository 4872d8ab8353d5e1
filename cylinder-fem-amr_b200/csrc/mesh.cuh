// The mesh handle: caller-owned device mesh + CSR pattern, and the assembly plan built from
// them (node -> element incidence sorted by element, and the CSR position of every
// element-local (row, column) pair, which replaces the per-entry binary search
// find_csr_index of src/cfa/fem_kernels.cuh:12-28).
#pragma once

#include "internal.cuh"

namespace cfa {

// Outlet condition (src/cfa/common.cuh:76-89)
struct OutletBc {
    int outlet_dirichlet = 0;   // 0: p = 0 on BC_OUTLET; 1: inflow parabola at the outlet, dp pinned
    int pin = -1;               // pinned node when outlet_dirichlet
    double outlet_scale = 1.0;  // outlet parabola factor
};

// pressure_dirichlet (src/cfa/common.cuh:87-89)
__device__ __forceinline__ bool pressure_dirichlet(int i, int tag, const OutletBc& bc) {
    return bc.outlet_dirichlet ? i == bc.pin : tag == BC_OUTLET;
}

}  // namespace cfa

struct cfa_mesh {
    int n = 0, ne = 0, nnz = 0;
    long long uid = 0;
    const int* ev = nullptr;     // [3 ne]
    const double* x = nullptr;
    const double* y = nullptr;
    const int* tag = nullptr;
    const int* rp = nullptr;
    const int* ci = nullptr;
    cfa::DevBuf<int> inc_ptr;    // [n + 1]
    cfa::DevBuf<int> inc;        // [3 ne]: element << 2 | local vertex, ascending element per node
    cfa::DevBuf<int> pos;        // [9 ne]: pos[3 s + b] = CSR index of (node of s, vertex b of its element)
    cfa::OutletBc bc;
};
