// FP64 instantiations of the fused kernels and launchers, and the common
// helpers (wvlh_fused_impl.cuh).
#define WVLH_FUSED_F64
#define WVLH_FUSED_COMMON
#include "wvlh_fused_impl.cuh"
