// Small device utilities: deterministic event-sum of the misfit and status
// folding.
#include <cub/cub.cuh>
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

// Sort key of each event for the next evaluation's queue: the previous
// evaluation's sweep work, forward sweeps weighted 3x (a forward cell update
// costs about three adjoint ones).
__global__ void event_cost_kernel(int ne, const int* __restrict__ fwd_it,
                                  const int* __restrict__ adj_it, unsigned int* key, int* idx) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ne) return;
    key[i] = 3u * (unsigned)fwd_it[i] + (unsigned)adj_it[i];
    idx[i] = i;
}

cudaError_t launch_event_cost(int ne, const int* fwd_it, const int* adj_it, unsigned int* key,
                              int* idx, cudaStream_t st) {
    event_cost_kernel<<<(ne + 255) / 256, 256, 0, st>>>(ne, fwd_it, adj_it, key, idx);
    return cudaGetLastError();
}

// Sort keys of one level's events in a multi-grid launch: the previous
// evaluation's sweep counts times the level's cell count (in units of 256
// cells), so solves of different grid sizes compare by work; code = level
// << 24 | event.
__global__ void multi_cost_kernel(int ne, const int* __restrict__ fwd_it,
                                  const int* __restrict__ adj_it, unsigned int scale, int lev,
                                  unsigned int* key, int* code) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ne) return;
    key[i] = (3u * (unsigned)fwd_it[i] + (unsigned)adj_it[i] + 1u) * scale;
    code[i] = (lev << 24) | i;
}

cudaError_t launch_multi_cost(int ne, const int* fwd_it, const int* adj_it, unsigned int scale,
                              int lev, unsigned int* key, int* code, cudaStream_t st) {
    if (ne <= 0) return cudaSuccess;
    multi_cost_kernel<<<(ne + 255) / 256, 256, 0, st>>>(ne, fwd_it, adj_it, scale, lev, key, code);
    return cudaGetLastError();
}

// Deterministic accumulation (src/preproc.cpp:28-31 in event order): for one
// chunk of events [e0, e0 + nchunk), adj_s[ip][k] += contrib[e - e0][k] over
// the chunk's events of period ip in event order (per_ptr / per_ev: the
// chunk's events grouped by period, ascending).  One thread per (ip, k).
__global__ void ordered_accumulate_kernel(size_t n, int nper, int e0,
                                          const int* __restrict__ per_ptr,
                                          const int* __restrict__ per_ev,
                                          const double* __restrict__ contrib, double* adj_s) {
    const size_t gid = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (gid >= n * nper) return;
    const int ip = (int)(gid / n);
    const size_t k = gid % n;
    double a = adj_s[gid];
    for (int j = per_ptr[ip]; j < per_ptr[ip + 1]; j++)
        a += contrib[(size_t)(per_ev[j] - e0) * n + k];
    adj_s[gid] = a;
}

// The misfit in event order, as the reference's event loop adds it
// (src/preproc.cpp:142).
__global__ void sum_events_ordered_kernel(int ne, const double* __restrict__ chi_ev, double* chi) {
    double s = 0.0;
    for (int i = 0; i < ne; i++) s += chi_ev[i];
    *chi = s;
}

cudaError_t launch_ordered_accumulate(size_t n, int nper, int e0, const int* per_ptr,
                                      const int* per_ev, const double* contrib, double* adj_s,
                                      cudaStream_t st) {
    const size_t total = n * nper;
    ordered_accumulate_kernel<<<(unsigned)((total + 255) / 256), 256, 0, st>>>(
        n, nper, e0, per_ptr, per_ev, contrib, adj_s);
    return cudaGetLastError();
}

cudaError_t launch_sum_events_ordered(int ne, const double* chi_ev, double* chi,
                                      cudaStream_t st) {
    sum_events_ordered_kernel<<<1, 1, 0, st>>>(ne, chi_ev, chi);
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

size_t sort_events_temp_bytes(int ne) {
    size_t bytes = 0;
    cub::DeviceRadixSort::SortPairsDescending(nullptr, bytes, (const unsigned int*)nullptr,
                                              (unsigned int*)nullptr, (const int*)nullptr,
                                              (int*)nullptr, ne);
    return bytes;
}

// order = events by descending key (stable: equal keys keep event order).
cudaError_t launch_sort_events(int ne, const unsigned int* key_in, unsigned int* key_out,
                               const int* idx_in, int* order, void* temp, size_t temp_bytes,
                               cudaStream_t st) {
    return cub::DeviceRadixSort::SortPairsDescending(temp, temp_bytes, key_in, key_out, idx_in,
                                                     order, ne, 0, 32, st);
}

}  // namespace sa
