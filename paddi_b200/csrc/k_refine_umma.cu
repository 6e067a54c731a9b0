// k_refine_umma.cu -- dense candidate refine on tcgen05 tensor cores
// (three-term split-BF16).  Placeholder until the kernel lands: reports the
// path as unavailable so PADDI_DIST_AUTO uses the FP32 refine.
#include "paddi_internal.cuh"

bool paddi_umma_supported(int device)
{
    (void)device;
    return false;
}

cudaError_t paddi_launch_refine_umma(const float *, const float4 *, const float *,
                                     const int32_t *, const int32_t *, const int32_t *,
                                     PaddiAttemptDev *, uint32_t *, uint8_t *, int32_t, int32_t,
                                     int32_t, int32_t, float, int32_t, cudaStream_t)
{
    return cudaErrorNotSupported;
}
