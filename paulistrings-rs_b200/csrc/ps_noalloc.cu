// ps_noalloc.cu -- ps_expectation_device_noalloc: the product-state expectation of a Pauli
// sum that the caller already holds in device memory, computed without allocating anything.
//
// Some callers cannot allocate device memory themselves: a host framework that owns all of
// the GPU's memory through its own pool (a stray cudaMalloc outside the pool can fail, or
// fragment the pool), a service that reserves its whole memory budget at start-up and forbids
// allocation afterwards (cudaMalloc/cudaFree can synchronize the device and stall a
// latency-bound loop), or a process under a fixed per-client memory limit.  Such a caller
// passes the store's packed keys and coefficients and an output slot, all in device memory it
// already has, and this entry point reduces them using only the scratch array below.
//
// The scratch is a file-scope device array of kNoAllocPartials float64 partial sums (512 KiB).
// Every GPU that loads this library holds one copy of it until the process exits.  Host code
// cannot use the array's name as a device address, so the first call on each device looks
// the address up with cudaGetSymbolAddress while that device is current; with the CUDA
// runtime's lazy module loading that lookup is also what loads this file's module on the
// device and reserves the array, so the first call belongs at start-up, before any stream
// capture.  All calls on a device share the array, so calls
// whose kernels overlap on the GPU race; serialize them (one stream, or events).  Nothing in
// the array needs clearing between calls: each call writes every partial it then reads.
#include <cstdint>
#include <cuda_runtime.h>
#include <mutex>

#include "../../include/paulistrings_b200.h"
#include "ps_device.cuh"

namespace {

constexpr int kNoAllocThreads = 256;
constexpr int kNoAllocTermsPerThread = 64;
constexpr uint64_t kNoAllocTermsPerBlock = (uint64_t)kNoAllocThreads * kNoAllocTermsPerThread;
constexpr int kNoAllocPartials = 65536;
static_assert(kNoAllocTermsPerBlock * kNoAllocPartials == PS_NOALLOC_MAX_TERMS, "limit");

static __device__ __align__(256) double g_noalloc_partials[kNoAllocPartials];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
double* g_partials_addr[kMaxDevices] = {};

template <int W>
struct NoAllocBasis {
    uint64_t ax[W], az[W], neg[W];
};

// Block b sums terms [b * kNoAllocTermsPerBlock, (b + 1) * kNoAllocTermsPerBlock) into partials[b].
template <int W, typename T>
__global__ void __launch_bounds__(kNoAllocThreads) k_expect_noalloc_blocks(const uint64_t* __restrict__ keys,
                                                                           const T* __restrict__ coef, uint64_t n,
                                                                           const NoAllocBasis<W> B,
                                                                           double* __restrict__ partials) {
    __shared__ double sh[kNoAllocThreads];
    const uint64_t base = (uint64_t)blockIdx.x * kNoAllocTermsPerBlock;
    double acc = 0.0;
    for (int q = 0; q < kNoAllocTermsPerThread; ++q) {
        const uint64_t i = base + (uint64_t)q * kNoAllocThreads + threadIdx.x;
        if (i >= n) break;
        uint64_t k[2 * W];
        psb::load_key<W>(keys, i, k);
        uint64_t mismatch = 0;
        uint32_t sign = 0;
#pragma unroll
        for (int w = 0; w < W; ++w) {
            const uint64_t sup = k[w] | k[W + w];
            mismatch |= (k[w] ^ (sup & B.ax[w])) | (k[W + w] ^ (sup & B.az[w]));
            sign += __popcll(sup & B.neg[w]);
        }
        if (mismatch) continue;
        const double c = psb::to_f64(coef[i]);
        acc = __dadd_rn(acc, (sign & 1u) ? -c : c);
    }
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int s = kNoAllocThreads / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) sh[threadIdx.x] = __dadd_rn(sh[threadIdx.x], sh[threadIdx.x + s]);
        __syncthreads();
    }
    if (threadIdx.x == 0) partials[blockIdx.x] = sh[0];
}

// One block sums partials[0, count) in a fixed order into *out.
__global__ void __launch_bounds__(kNoAllocThreads) k_expect_noalloc_final(const double* __restrict__ partials,
                                                                          uint32_t count, double* __restrict__ out) {
    __shared__ double sh[kNoAllocThreads];
    double acc = 0.0;
    for (uint32_t i = threadIdx.x; i < count; i += kNoAllocThreads) acc = __dadd_rn(acc, partials[i]);
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int s = kNoAllocThreads / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) sh[threadIdx.x] = __dadd_rn(sh[threadIdx.x], sh[threadIdx.x + s]);
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = sh[0];
}

// Device address of the scratch array on `device`, looked up once per device.
ps_status partials_for(int device, double** out) {
    if (device < 0 || device >= kMaxDevices) return PS_ERR_UNSUPPORTED;
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_partials_addr[device]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_partials);
        if (e != cudaSuccess || !p) {
            cudaGetLastError();
            return PS_ERR_DEVICE;
        }
        g_partials_addr[device] = static_cast<double*>(p);
    }
    *out = g_partials_addr[device];
    return PS_OK;
}

// Both launches go through cudaLaunchKernel, whose return value is that launch's own status: an
// error some earlier call of the caller's left pending is neither reported as this call's
// failure nor cleared from the caller's view.
template <int W, typename T>
ps_status launch(const uint64_t* keys, const void* coeffs, uint64_t n, const uint64_t* ax, const uint64_t* az,
                 const uint64_t* neg, double* out, cudaStream_t st, double* partials) {
    NoAllocBasis<W> B;
    for (int w = 0; w < W; ++w) {
        B.ax[w] = ax[w];
        B.az[w] = az[w];
        B.neg[w] = neg[w];
    }
    uint32_t blocks = (uint32_t)((n + kNoAllocTermsPerBlock - 1) / kNoAllocTermsPerBlock);
    const T* coef = static_cast<const T*>(coeffs);
    if (blocks) {
        void* args[] = {(void*)&keys, (void*)&coef, (void*)&n, (void*)&B, (void*)&partials};
        if (cudaLaunchKernel((const void*)k_expect_noalloc_blocks<W, T>, dim3(blocks), dim3(kNoAllocThreads), args, 0,
                             st) != cudaSuccess)
            return PS_ERR_DEVICE;
    }
    void* fargs[] = {(void*)&partials, (void*)&blocks, (void*)&out};
    if (cudaLaunchKernel((const void*)k_expect_noalloc_final, dim3(1), dim3(kNoAllocThreads), fargs, 0, st) !=
        cudaSuccess)
        return PS_ERR_DEVICE;
    return PS_OK;
}

}  // namespace

extern "C" {
#pragma GCC visibility push(default)

ps_status ps_expectation_device_noalloc(const uint64_t* keys, const void* coeffs, int32_t dtype, int32_t width,
                                        uint64_t n, const uint64_t* axis_x, const uint64_t* axis_z,
                                        const uint64_t* negative, double* out, void* stream) {
    if (!out || !axis_x || !axis_z || !negative || (n && (!keys || !coeffs))) return PS_ERR_INVALID;
    if (dtype != PS_F64 && dtype != PS_F32) return PS_ERR_INVALID;
    if (width != 1 && width != 2 && width != 4) return PS_ERR_UNSUPPORTED;
    if (n > PS_NOALLOC_MAX_TERMS) return PS_ERR_INVALID;  // the scratch holds one partial per 16,384 terms
    // The kernel reads a key as 16-byte vectors and a coefficient as one T, and writes one
    // double: a pointer off those boundaries would fault the device instead of failing here.
    const uintptr_t csize = dtype == PS_F64 ? sizeof(double) : sizeof(float);
    if ((reinterpret_cast<uintptr_t>(keys) & 15u) != 0 || (reinterpret_cast<uintptr_t>(coeffs) & (csize - 1)) != 0 ||
        (reinterpret_cast<uintptr_t>(out) & 7u) != 0)
        return PS_ERR_INVALID;
    int device = -1;
    if (cudaGetDevice(&device) != cudaSuccess) {
        cudaGetLastError();
        return PS_ERR_NO_DEVICE;
    }
    double* partials = nullptr;
    ps_status st = partials_for(device, &partials);
    if (st != PS_OK) return st;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (dtype == PS_F64) {
        switch (width) {
        case 1: return launch<1, double>(keys, coeffs, n, axis_x, axis_z, negative, out, s, partials);
        case 2: return launch<2, double>(keys, coeffs, n, axis_x, axis_z, negative, out, s, partials);
        default: return launch<4, double>(keys, coeffs, n, axis_x, axis_z, negative, out, s, partials);
        }
    }
    switch (width) {
    case 1: return launch<1, float>(keys, coeffs, n, axis_x, axis_z, negative, out, s, partials);
    case 2: return launch<2, float>(keys, coeffs, n, axis_x, axis_z, negative, out, s, partials);
    default: return launch<4, float>(keys, coeffs, n, axis_x, axis_z, negative, out, s, partials);
    }
}

#pragma GCC visibility pop
}  // extern "C"
