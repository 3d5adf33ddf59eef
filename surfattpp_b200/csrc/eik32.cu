// FP32 engine: sweep-precision media planes and the FP32 persistent batch
// kernel.  Sweeps run in FP32 (fast division and square root); T0 and T,
// residuals, adjoint coefficients, convergence sums and the kernel
// accumulation stay FP64 (see batch.cuh).
#include "batch.cuh"
#include "launch.h"

namespace sa {

__global__ void media32_kernel(size_t total, const double* __restrict__ fun64,
                               const double* __restrict__ a_f64, const double* __restrict__ b_p64,
                               const double* __restrict__ c_f64, float* fun32, float* a_f32,
                               float* b_p32, float* c_f32) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total;
         i += (size_t)gridDim.x * blockDim.x) {
        fun32[i] = (float)fun64[i];
        if (a_f64) {
            a_f32[i] = (float)a_f64[i];
            b_p32[i] = (float)b_p64[i];
            c_f32[i] = (float)c_f64[i];
        }
    }
}

cudaError_t launch_media32(int nx, int ny, int nper, const double* fun64, const double* a_f64,
                           const double* b_p64, const double* c_f64, float* fun32, float* a_f32,
                           float* b_p32, float* c_f32, cudaStream_t st) {
    const size_t total = (size_t)nx * ny * nper;
    const int threads = 256;
    const int blocks = (int)std::min<size_t>((total + threads - 1) / threads, 148 * 16);
    media32_kernel<<<blocks, threads, 0, st>>>(total, fun64, a_f64, b_p64, c_f64, fun32, a_f32,
                                               b_p32, c_f32);
    return cudaGetLastError();
}

size_t batch32_slot_bytes(int nx, int ny) { return slot_layout<float>(nx, ny).total; }

int batch32_max_slots(int device) {
    int nsm = 0, per_sm = 0;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batch_kernel<float>, 128, 0);
    if (per_sm < 1) per_sm = 1;
    return nsm * per_sm * 4;
}

cudaError_t launch_batch32(const BatchDesc& d, cudaStream_t st) {
    const BatchArgs<float> B = make_batch_args<float>(d);
    const int blocks = (d.sc.nslots + 3) / 4;
    batch_kernel<float><<<blocks, 128, 0, st>>>(B);
    return cudaGetLastError();
}

}  // namespace sa
