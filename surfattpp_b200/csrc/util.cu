// Small device utilities: deterministic event-sum of the misfit and status
// folding.
#include "launch.h"

namespace sa {

// chi = sum over events of chi_ev (fixed-order tree: deterministic run to run).
__global__ void sum_events_kernel(int ne, const double* __restrict__ chi_ev, double* chi) {
    __shared__ double part[1024];
    double s = 0.0;
    for (int i = threadIdx.x; i < ne; i += blockDim.x) s += chi_ev[i];
    part[threadIdx.x] = s;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) part[threadIdx.x] += part[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) *chi = part[0];
}

// worst = max status over events (0 = all ok).
__global__ void fold_status_kernel(int ne, const int* __restrict__ st, int* worst) {
    __shared__ int part[1024];
    int s = 0;
    for (int i = threadIdx.x; i < ne; i += blockDim.x) s = max(s, st[i]);
    part[threadIdx.x] = s;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) part[threadIdx.x] = max(part[threadIdx.x], part[threadIdx.x + w]);
        __syncthreads();
    }
    if (threadIdx.x == 0) *worst = part[0];
}

// Status of one misfit-gradient evaluation: SA_ERR_NOROOT (4) when any column's
// dispersion root search failed, else the worst event status.
__global__ void grad_status_kernel(int ncol, const int* __restrict__ colst,
                                   const int* __restrict__ ev_worst, int* out) {
    __shared__ int any;
    if (threadIdx.x == 0) any = 0;
    __syncthreads();
    int s = 0;
    for (int i = threadIdx.x; i < ncol; i += blockDim.x) s |= colst[i];
    if (s) atomicOr(&any, 1);
    __syncthreads();
    if (threadIdx.x == 0) *out = any ? 4 : *ev_worst;
}

cudaError_t launch_grad_status(int ncol, const int* colst, const int* ev_worst, int* out,
                               cudaStream_t st) {
    grad_status_kernel<<<1, 1024, 0, st>>>(ncol, colst, ev_worst, out);
    return cudaGetLastError();
}

cudaError_t launch_sum_events(int ne, const double* chi_ev, double* chi, cudaStream_t st) {
    sum_events_kernel<<<1, 1024, 0, st>>>(ne, chi_ev, chi);
    return cudaGetLastError();
}

cudaError_t launch_fold_status(int ne, const int* status, int* worst, cudaStream_t st) {
    fold_status_kernel<<<1, 1024, 0, st>>>(ne, status, worst);
    return cudaGetLastError();
}

}  // namespace sa
