// FP32 engine: sweep-precision media planes and the FP32 persistent batch
// kernel.  Sweeps run in FP32 (fast division and square root); T0 and T,
// residuals, adjoint coefficients, convergence sums and the kernel
// accumulation stay FP64 (see batch.cuh).
#include <algorithm>
#include <vector>

#include "batch.cuh"
#include "launch.h"

namespace sa {

__global__ void media32_kernel(size_t total, const double* __restrict__ fun64,
                               const double* __restrict__ mt64, float* fun32, float* mt32) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total;
         i += (size_t)gridDim.x * blockDim.x) {
        fun32[i] = (float)fun64[i];
        if (mt64)
            for (int c = 0; c < 4; c++) mt32[4 * i + c] = (float)mt64[4 * i + c];
    }
}

cudaError_t launch_media32(int nx, int ny, int nper, const double* fun64, const double* mt64,
                           float* fun32, float* mt32, cudaStream_t st) {
    const size_t total = (size_t)nx * ny * nper;
    const int threads = 256;
    const int blocks = (int)std::min<size_t>((total + threads - 1) / threads, 148 * 16);
    media32_kernel<<<blocks, threads, 0, st>>>(total, fun64, mt64, fun32, mt32);
    return cudaGetLastError();
}

size_t batch32_slot_bytes(int nx, int ny, int maxr) {
    return slot_layout<float>(nx, ny, maxr).total;
}

int batch32_max_slots(int device) {
    int nsm = 0, per_sm = 0;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batch_kernel<float, true, 0>, 128, 0);
    if (per_sm < 1) per_sm = 1;
    return nsm * per_sm * 4;
}

namespace {
template <int VAR>
void launch_variant(const BatchDesc& d, const BatchArgs<float>& B, int blocks, cudaStream_t st) {
    if (d.iso) batch_kernel<float, true, VAR><<<blocks, 128, 0, st>>>(B);
    else batch_kernel<float, false, VAR><<<blocks, 128, 0, st>>>(B);
}
}  // namespace

cudaError_t launch_batch32(const BatchDesc& d, cudaStream_t st) {
    const BatchArgs<float> B = make_batch_args<float>(d);
    // with tail teams every resident warp runs (the slots in use are spread
    // over the blocks, the other warps start as helpers)
    const int blocks =
        (((d.variant & 4) ? std::max(d.sc.nwarps, d.sc.nslots) : d.sc.nslots) + 3) / 4;
    switch (d.variant) {
        case 1: launch_variant<1>(d, B, blocks, st); break;
        case 2: launch_variant<2>(d, B, blocks, st); break;
        case 3: launch_variant<3>(d, B, blocks, st); break;
        case 4: launch_variant<4>(d, B, blocks, st); break;
        case 5: launch_variant<5>(d, B, blocks, st); break;
        case 6: launch_variant<6>(d, B, blocks, st); break;
        case 7: launch_variant<7>(d, B, blocks, st); break;
        default: launch_variant<0>(d, B, blocks, st); break;
    }
    return cudaGetLastError();
}

// One launch over several plans' events (batch_multi_kernel): the levels'
// arguments are copied to `dev_args` (nlev BatchArgs<float>), `code` lists
// level << 24 | event in queue order.  One variant and one metric kind (iso
// or general) for all levels; no tail teams (variant bit 2 is ignored).
namespace {
template <int VAR>
void launch_multi_variant(bool iso, const BatchArgs<float>* args, unsigned ntotal,
                          const unsigned* code, const Scratch& sc, int blocks, cudaStream_t st) {
    if (iso) batch_multi_kernel<float, true, VAR><<<blocks, 128, 0, st>>>(args, ntotal, code, sc);
    else batch_multi_kernel<float, false, VAR><<<blocks, 128, 0, st>>>(args, ntotal, code, sc);
}
}  // namespace

cudaError_t launch_batch32_multi(const BatchDesc* d, int nlev, void* dev_args, unsigned ntotal,
                                 const unsigned* code, const Scratch& sc, cudaStream_t st) {
    std::vector<BatchArgs<float>> h(nlev);
    for (int i = 0; i < nlev; i++) h[i] = make_batch_args<float>(d[i]);
    cudaError_t e = cudaMemcpyAsync(dev_args, h.data(), nlev * sizeof(BatchArgs<float>),
                                    cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return e;
    const auto* args = static_cast<const BatchArgs<float>*>(dev_args);
    const int blocks = (sc.nslots + 3) / 4;
    const bool iso = d[0].iso != 0;
    switch (d[0].variant & 3) {
        case 1: launch_multi_variant<1>(iso, args, ntotal, code, sc, blocks, st); break;
        case 2: launch_multi_variant<2>(iso, args, ntotal, code, sc, blocks, st); break;
        case 3: launch_multi_variant<3>(iso, args, ntotal, code, sc, blocks, st); break;
        default: launch_multi_variant<0>(iso, args, ntotal, code, sc, blocks, st); break;
    }
    return cudaGetLastError();
}

size_t batch32_args_bytes() { return sizeof(BatchArgs<float>); }

}  // namespace sa
