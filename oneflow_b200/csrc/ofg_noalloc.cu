// ofg_residual_rms_noalloc: the residual RMS of a caller-owned residual array
// without allocating anything (the contract is in include/oneflow_b200.h).
//
// Scratch lives in this file's static __device__ object: one slot of partial
// sums per block and a ticket counter, 18,952 bytes per device.  Every call
// clears the ticket on its stream before its kernel (a 4-byte memset, no
// allocation), so a call that never finished cannot leave a stale count for
// the next one; the partial sums need no clearing, since every block writes
// its own slot before the ticket counts it.  Two calls that overlap in time on
// the same device share the scratch and race: callers serialise them (one
// stream, or an event between).
#include <cuda_runtime.h>

#include <atomic>
#include <cstddef>
#include <cstdint>

#include "../../include/oneflow_b200.h"

namespace {

constexpr int kBlocks = 296;     // blocks of the reduction (2 per SM) = partial-sum slots
constexpr int kThreads = 256;
constexpr int kMaxEq = OFG_NOALLOC_MAX_EQ;

struct Scratch {
    double partial[kBlocks * kMaxEq];   // per-block sums of squares
    unsigned int ticket;                // blocks finished; cleared by every call before its kernel
};
static_assert(sizeof(Scratch) <= 19 * 1024, "scratch stays small");

static __device__ __align__(256) Scratch g_scratch;

// Every block adds the squares of a contiguous range of cells in a fixed
// order; the last block to finish adds the block sums in block order and
// writes sqrt(sum / n) per equation to out (deterministic run to run).
__global__ void __launch_bounds__(kThreads) k_rms_noalloc(const double *res, long long n, int neq, double *out,
                                                          Scratch *sc) {
    __shared__ double red[kThreads / 32][kMaxEq];
    __shared__ bool last;
    double acc[kMaxEq];
#pragma unroll
    for (int e = 0; e < kMaxEq; ++e) acc[e] = 0.0;
    long long per = (n + gridDim.x - 1) / gridDim.x;
    long long b0 = (long long)blockIdx.x * per, b1 = b0 + per < n ? b0 + per : n;
    for (long long i = b0 + threadIdx.x; i < b1; i += blockDim.x)
#pragma unroll
        for (int e = 0; e < kMaxEq; ++e)
            if (e < neq) {
                double v = res[i * neq + e];
                acc[e] += v * v;
            }
    int w = threadIdx.x >> 5, l = threadIdx.x & 31;
#pragma unroll
    for (int e = 0; e < kMaxEq; ++e) {
        double x = acc[e];
        for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
        if (l == 0) red[w][e] = x;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int e = 0; e < neq; ++e) {
            double s = 0.0;
            for (int k = 0; k < kThreads / 32; ++k) s += red[k][e];
            sc->partial[blockIdx.x * kMaxEq + e] = s;
        }
        __threadfence();
        last = atomicAdd(&sc->ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last || threadIdx.x != 0) return;
    __threadfence();
    for (int e = 0; e < neq; ++e) {
        double s = 0.0;
        for (unsigned int k = 0; k < gridDim.x; ++k) s += __ldcg(&sc->partial[k * kMaxEq + e]);
        out[e] = sqrt(s / double(n));
    }
    sc->ticket = 0u;
}

// address of the scratch on each device, looked up once with that device
// current (host threads that race on the first call store the same value)
constexpr int kMaxDevices = 64;
std::atomic<Scratch *> g_scratch_addr[kMaxDevices];

}  // namespace

extern "C" int ofg_residual_rms_noalloc(const double *res, int64_t n_cells, int n_eq, double *rms_out,
                                        void *stream) {
    if (!res || !rms_out || n_cells <= 0 || n_eq < 1) return OFG_E_ARG;
    if (n_eq > OFG_NOALLOC_MAX_EQ) return OFG_E_SIZE;   // the scratch holds OFG_NOALLOC_MAX_EQ sums per block
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0) return OFG_E_CUDA;
    if (dev >= kMaxDevices) return OFG_E_SIZE;
    Scratch *sc = g_scratch_addr[dev].load(std::memory_order_acquire);
    if (!sc) {
        // first call on this device (with it current): resolve the scratch
        // address, which also loads this module on the device
        void *p = nullptr;
        if (cudaGetSymbolAddress(&p, g_scratch) != cudaSuccess || !p) return OFG_E_CUDA;
        sc = static_cast<Scratch *>(p);
        g_scratch_addr[dev].store(sc, std::memory_order_release);
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (cudaMemsetAsync(reinterpret_cast<char *>(sc) + offsetof(Scratch, ticket), 0, sizeof(unsigned int), st) !=
        cudaSuccess)
        return OFG_E_CUDA;
    long long nb = (n_cells + kThreads - 1) / kThreads;
    int blocks = nb < kBlocks ? int(nb) : kBlocks;
    k_rms_noalloc<<<blocks, kThreads, 0, st>>>(res, (long long)n_cells, n_eq, rms_out, sc);
    return cudaGetLastError() == cudaSuccess ? OFG_OK : OFG_E_CUDA;
}
