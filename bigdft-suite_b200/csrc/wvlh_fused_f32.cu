// FP32 instantiations of the fused kernels and launchers (wvlh_fused_impl.cuh).
#define WVLH_FUSED_F32
#include "wvlh_fused_impl.cuh"
