// mpcf_selftest.cu -- exhaustive device checks of the branch-free correctly
// rounded reciprocals (mpcf_ieee.cuh) against the compiler's IEEE division,
// over every float bit pattern.  Compiled like stage_ref.cu (no contraction,
// IEEE division), the translation unit whose kernels use them.
#include <cuda_runtime.h>
#include <math.h>
#include "mpcf_ieee.cuh"
#include "mpcf_launch.h"
#include "../../include/mpcf_b200.h"

namespace mpcf {

__device__ __forceinline__ bool same_bits(const double a, const double b)
{
    return __double_as_longlong(a) == __double_as_longlong(b) || (isnan(a) && isnan(b));
}
__device__ __forceinline__ bool same_bits(const float a, const float b)
{
    return __float_as_uint(a) == __float_as_uint(b) || (isnan(a) && isnan(b));
}

// which = 0: rcp_rn_f64_weight(10 x^2) against 1.0 / (10.0*x*x), the WENO
//            weights' denominators of the FP32 reference form (x = beta + eps);
// which = 1: rcp_rn_f32(x) against the IEEE quotient 1 / x.
// Every float bit pattern x once; mismatches counted, the first 8 recorded.
__global__ void __launch_bounds__(256) ieee_selftest_kernel(const int which, unsigned long long* bad, unsigned* first)
{
    const unsigned long long total = 1ull << 32;
    const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
    for (unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += stride)
    {
        const float x = __uint_as_float((unsigned)i);
        bool ok;
        if (which == 0)
        {
            const double d = 10.0 * (double)x * (double)x;
            ok = same_bits(rcp_rn_f64_weight(d), __drcp_rn(d)) && same_bits(__drcp_rn(d), 1.0 / d);
        }
        else ok = same_bits(rcp_rn_f32(x), __fdiv_rn(1.0f, x));
        if (!ok)
        {
            const unsigned long long k = atomicAdd(bad, 1ull);
            if (k < 8) first[k] = (unsigned)i;
        }
    }
}

} // namespace mpcf

extern "C" int mpcf_selftest_ieee(int which, int device, unsigned long long* mismatches, unsigned* first8)
{
    using namespace mpcf;
    if ((which != 0 && which != 1) || !mismatches) return mpcf_fail_external(MPCF_ERR_ARG, "bad self-test arguments");
    int prev = 0;
    cudaGetDevice(&prev);
    if (cudaSetDevice(device) != cudaSuccess) { cudaGetLastError(); return mpcf_fail_external(MPCF_ERR_CUDA, "cudaSetDevice(%d)", device); }
    void* buf = nullptr;
    int rc = MPCF_OK;
    cudaError_t e = cudaMalloc(&buf, sizeof(unsigned long long) + 8 * sizeof(unsigned));
    if (e == cudaSuccess) e = cudaMemset(buf, 0, sizeof(unsigned long long) + 8 * sizeof(unsigned));
    if (e == cudaSuccess)
    {
        int sms = 148;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
        ieee_selftest_kernel<<<sms * 8, 256>>>(which, (unsigned long long*)buf, (unsigned*)((char*)buf + 8));
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    unsigned char host[8 + 32] = {0};
    if (e == cudaSuccess) e = cudaMemcpy(host, buf, sizeof(host), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) rc = mpcf_fail_external(MPCF_ERR_CUDA, "self-test: %s", cudaGetErrorString(e));
    else
    {
        *mismatches = *(unsigned long long*)host;
        if (first8)
            for (int k = 0; k < 8; ++k) first8[k] = ((unsigned*)(host + 8))[k];
    }
    if (buf) cudaFree(buf);
    cudaSetDevice(prev);
    return rc;
}
