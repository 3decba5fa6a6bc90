// (b) full dipolar recompute as an implicit GEMM on the tcgen05 tensor cores.
#include "hs_common.cuh"
#include "hs_internal.h"

int64_t hs_igemm_scratch(const HsLattice &, int) { return 0; }

int hs_launch_igemm(const HsLattice &, int, void *, int64_t, cudaStream_t) {
    hs_set_error("hs_dipolar_full_igemm: not available in this build");
    return HS_EINVAL;
}
