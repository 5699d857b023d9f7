// ps_rotlayer.cuh -- device helpers of a rotation layer's table shared by the layer kernels
// and the TopN compaction that classifies its output rows for the next layer: support pattern
// of a key, per-pattern amplitudes staged in shared memory, the partner test, divergence rank.
#pragma once

#include "ps_device.cuh"
#include "ps_kernels.h"

namespace psb {

// word `wi` of a key held in registers, by an unrolled select (a runtime index into a
// register array would move the array to local memory)
template <int W>
__device__ __forceinline__ uint64_t pick(const uint64_t* k, int wi) {
    uint64_t v = k[0];
#pragma unroll
    for (int w = 1; w < 2 * W; ++w) v = (w == wi) ? k[w] : v;
    return v;
}

// support pattern of key k (LocalPtm::support_bits, channel/prepared.rs:141-151)
template <int W>
__device__ __forceinline__ uint32_t pattern_of(const RotLayer<W>& L, const uint64_t* k) {
    uint32_t s = (uint32_t)((pick<W>(k, L.qw[0]) >> L.qb[0]) & 1u) |
                 (uint32_t)((pick<W>(k, W + L.qw[0]) >> L.qb[0]) & 1u) << 1 |
                 (uint32_t)((pick<W>(k, L.qw[1]) >> L.qb[1]) & 1u) << 2 |
                 (uint32_t)((pick<W>(k, W + L.qw[1]) >> L.qb[1]) & 1u) << 3;
    return s & L.pattern_mask;
}

template <typename T>
struct Amp;
template <>
struct Amp<double> {
    template <int W>
    __device__ static double a0(const RotLayer<W>& L, uint32_t s) { return L.a0[s]; }
    template <int W>
    __device__ static double a1(const RotLayer<W>& L, uint32_t s) { return L.a1[s]; }
    template <int W>
    __device__ static double cs(const RotLayer<W>& L) { return L.cos64; }
    template <int W>
    __device__ static double sn(const RotLayer<W>& L) { return L.sin64; }
};
template <>
struct Amp<float> {
    template <int W>
    __device__ static float a0(const RotLayer<W>& L, uint32_t s) { return L.a0f[s]; }
    template <int W>
    __device__ static float a1(const RotLayer<W>& L, uint32_t s) { return L.a1f[s]; }
    template <int W>
    __device__ static float cs(const RotLayer<W>& L) { return L.cos32; }
    template <int W>
    __device__ static float sn(const RotLayer<W>& L) { return L.sin32; }
};

// The layer's per-pattern amplitudes staged in shared memory: indexing the kernel-parameter
// copy with a per-lane pattern would serialize on the constant cache.
template <typename T>
struct AmpTab {
    T a0[16];
    T a1[16];
};

template <int W, typename T>
__device__ __forceinline__ void stage_amps(const RotLayer<W>& L, AmpTab<T>& t) {
    if (threadIdx.x < 16) {
        t.a0[threadIdx.x] = Amp<T>::a0(L, threadIdx.x);
        t.a1[threadIdx.x] = Amp<T>::a1(L, threadIdx.x);
    }
}

template <int W, typename T>
__device__ __forceinline__ bool emits_partner_regs(const RotLayer<W>& L, const AmpTab<T>& A,
                                                   const uint64_t (&k)[2 * W]) {
    if (L.wide) {
        uint64_t f = 0;
#pragma unroll
        for (int i = 0; i < W; ++i) f ^= (k[i] & L.gz[i]) ^ (k[W + i] & L.gx[i]);
        return (__popcll(f) & 1) != 0;
    }
    return A.a1[pattern_of<W>(L, k)] != T(0);
}

template <int W>
__device__ __forceinline__ uint32_t div_regs(const uint64_t (&a)[2 * W], const uint64_t (&b)[2 * W]) {
    uint32_t r = 0xFFFFu;
#pragma unroll
    for (int i = 2 * W - 1; i >= 0; --i) {
        uint64_t d = a[i] ^ b[i];
        if (d) r = 64u * i + (uint32_t)__clzll((long long)d);
    }
    return r;
}

}  // namespace psb
