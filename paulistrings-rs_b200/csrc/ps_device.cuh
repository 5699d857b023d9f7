// ps_device.cuh -- device-side building blocks shared by the layer kernels.
//
// Keys are 2W unsigned 64-bit words per term, x words then z words; the store is
// sorted lexicographically by those words (the reference's derived Ord on
// PauliString, crates/paulistrings/src/pauli_string.rs:13-20).  Bit b of word i
// has significance rank 64*i + (63 - b): rank 0 is the most significant bit.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "ps_kernels.h"

#ifndef PS_CHECKED
#define PS_CHECKED 0
#endif

namespace psb {

// ---------------------------------------------------------------------------
// error flags shared by all kernels of a handle (ps_ctl::err)
// ---------------------------------------------------------------------------
enum : uint32_t {
    ERR_TIMEOUT = 1u,     // a bounded spin gave up
    ERR_BOUNDS = 2u,      // checked builds: an index left its buffer (the access was skipped)
    ERR_KEY_RANGE = 4u,   // an uploaded key has a bit at or above num_qubits
    ERR_INTERNAL = 8u     // an invariant of the layer pipeline failed
};

// Default spin limit of every look-back / barrier wait (Ctl::spin_limit): a few seconds of
// polling, far beyond any legitimate wait, and still finite.
constexpr long long kSpinLimit = 1LL << 22;

__device__ __forceinline__ long long spin_limit(const Ctl* ctl) { return (long long)ctl->spin_limit; }

__device__ __forceinline__ void raise_err(Ctl* ctl, uint32_t bit, uint32_t info) {
    if ((atomicOr(&ctl->err, bit) & bit) == 0) atomicExch(&ctl->err_info, info);
}

// Always-on guard for data-dependent scatter positions: a failed check is recorded in the
// handle's flags (ERR_INTERNAL) and the access is skipped.
#define PS_GUARD(ctl, cond, info) \
    (((cond)) ? true : (::psb::raise_err((ctl), ::psb::ERR_INTERNAL, (info)), false))

#if PS_CHECKED
#define PS_BOUNDS(ctl, cond, info)                                                            \
    (((cond)) ? true : (::psb::raise_err((ctl), ::psb::ERR_BOUNDS, (info)), false))
#else
#define PS_BOUNDS(ctl, cond, info) true
#endif

// ---------------------------------------------------------------------------
// memory-model helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned long long ld_acquire_u64(const unsigned long long* p) {
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_u64(unsigned long long* p, unsigned long long v) {
    asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ unsigned int ld_acquire_u32(const unsigned int* p) {
    unsigned int v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_u32(unsigned int* p, unsigned int v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// ---------------------------------------------------------------------------
// TMA bulk copies (cp.async.bulk, sm_90+) completed on an mbarrier
// ---------------------------------------------------------------------------
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
// dst (shared) and src (global) 16-byte aligned, bytes a multiple of 16.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}
// dst (global) and src (shared) 16-byte aligned, bytes a multiple of 16; completes in the
// issuing thread's bulk group.
__device__ __forceinline__ void bulk_s2g(void* dst, const void* src, uint32_t bytes) {
    asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst), "r"(smem_u32(src)),
                 "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
// Wait until every committed bulk group of this thread has finished reading shared memory.
__device__ __forceinline__ void bulk_wait_read_all() {
    asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
}
// Order this thread's generic-proxy shared-memory writes before later async-proxy reads
// (a bulk copy out of shared memory issued after a barrier).
__device__ __forceinline__ void fence_proxy_async_shared() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait for the phase `parity` of `bar`; returns false (and flags ERR_TIMEOUT) if it gave up.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, Ctl* ctl, uint32_t info) {
    long long spins = 0;
    while (!mbar_try_wait(bar, parity)) {
        if (++spins > spin_limit(ctl)) {
            raise_err(ctl, ERR_TIMEOUT, info);
            return false;
        }
    }
    return true;
}

// After a bounded wait gave up: wait (with a fixed limit of its own, not the handle's, which a
// test may have shortened) for the phase `parity` of `bar`, so the bulk copies in flight into
// this block's shared memory have landed before the block reuses or releases it.
constexpr long long kDrainLimit = 1LL << 24;
__device__ __forceinline__ void mbar_drain(uint64_t* bar, uint32_t parity) {
    for (long long spins = 0; spins < kDrainLimit && !mbar_try_wait(bar, parity); ++spins) __nanosleep(64);
}

// Issue a bulk copy of `bytes` (rounded up to 16) from global `src` (16-B aligned) into shared `dst`.
// The caller sized the source allocation with >= 16 bytes of tail padding.
__device__ __forceinline__ uint32_t round16(uint32_t b) { return (b + 15u) & ~15u; }

// ---------------------------------------------------------------------------
// key algebra (crates/paulistrings/src/pauli_string.rs:68-123)
// ---------------------------------------------------------------------------
template <int W>
struct KeyT {
    uint64_t w[2 * W];
};

template <int W>
__device__ __forceinline__ void load_key(const uint64_t* __restrict__ base, uint64_t row, uint64_t (&k)[2 * W]) {
    const ulonglong2* p = reinterpret_cast<const ulonglong2*>(base + row * (2 * W));
#pragma unroll
    for (int q = 0; q < W; ++q) {
        ulonglong2 v = p[q];
        k[2 * q] = v.x;
        k[2 * q + 1] = v.y;
    }
}
template <int W>
__device__ __forceinline__ void store_key(uint64_t* __restrict__ base, uint64_t row, const uint64_t (&k)[2 * W]) {
    ulonglong2* p = reinterpret_cast<ulonglong2*>(base + row * (2 * W));
#pragma unroll
    for (int q = 0; q < W; ++q) p[q] = make_ulonglong2(k[2 * q], k[2 * q + 1]);
}

// a <= b lexicographically
template <int W>
__device__ __forceinline__ bool key_le(const uint64_t* a, const uint64_t* b) {
#pragma unroll
    for (int i = 0; i < 2 * W; ++i) {
        if (a[i] != b[i]) return a[i] < b[i];
    }
    return true;
}
template <int W>
__device__ __forceinline__ bool key_lt(const uint64_t* a, const uint64_t* b) {
#pragma unroll
    for (int i = 0; i < 2 * W; ++i) {
        if (a[i] != b[i]) return a[i] < b[i];
    }
    return false;
}
template <int W>
__device__ __forceinline__ bool key_eq(const uint64_t* a, const uint64_t* b) {
    uint64_t d = 0;
#pragma unroll
    for (int i = 0; i < 2 * W; ++i) d |= a[i] ^ b[i];
    return d == 0;
}
// Significance rank of the first differing bit of two distinct keys (0 = most significant).
template <int W>
__device__ __forceinline__ uint32_t divergence(const uint64_t* a, const uint64_t* b) {
#pragma unroll
    for (int i = 0; i < 2 * W; ++i) {
        uint64_t d = a[i] ^ b[i];
        if (d) return 64u * i + (uint32_t)__clzll((long long)d);
    }
    return 0xFFFFu;  // equal keys: cannot happen in a store with unique keys
}
template <int W>
__device__ __forceinline__ uint32_t key_weight(const uint64_t* k) {
    uint32_t w = 0;
#pragma unroll
    for (int i = 0; i < W; ++i) w += __popcll(k[i] | k[W + i]);
    return w;
}
// anticommutation with generator (gx, gz): parity of popcount(x&gz ^ z&gx)
template <int W>
__device__ __forceinline__ bool anticommutes(const uint64_t* k, const uint64_t* gx, const uint64_t* gz) {
    uint64_t f = 0;
#pragma unroll
    for (int i = 0; i < W; ++i) f ^= (k[i] & gz[i]) ^ (k[W + i] & gx[i]);
    return (__popcll(f) & 1) != 0;
}
// Phase exponent of k * g (mul_assign): 2bc + ab + cd - (a^c)(b^d) mod 4.
template <int W>
__device__ __forceinline__ uint32_t product_phase(const uint64_t* k, const uint64_t* gx, const uint64_t* gz) {
    uint32_t d = 0;
#pragma unroll
    for (int i = 0; i < W; ++i) {
        uint64_t a = k[i], b = k[W + i], c = gx[i], e = gz[i];
        d += 2u * __popcll(b & c) + __popcll(a & b) + __popcll(c & e) - __popcll((a ^ c) & (b ^ e));
    }
    return d & 3u;
}

// ---------------------------------------------------------------------------
// exact arithmetic wrappers: never contracted into FMA, so every product and sum
// rounds once, as the reference's host arithmetic does.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double to_f64(double a) { return a; }
__device__ __forceinline__ double to_f64(float a) { return (double)a; }

// TopN select key of a coefficient: 0 for NaN, else bits(|c|^2) + 1 (monotone in |c|^2, as the
// reference's norm_sqr ordering; crates/paulistrings/src/truncation/builtin.rs:107-110).
template <typename T>
__device__ __forceinline__ uint64_t mag_key(T c) {
    double v = to_f64(c);
    double m = __dmul_rn(v, v);
    if (isnan(m)) return 0ull;
    return (uint64_t)__double_as_longlong(m) + 1ull;
}

// TopN's first select digit, windowed: 2048 bins of 2^48 select-key units (1/16 of an octave
// of |c|^2) starting at `base`; keys below the window land in bin 0, above it in bin 2047.
__device__ __forceinline__ uint64_t window_key(uint64_t mk, uint64_t base) {
    if (mk < base) return 0ull;
    const uint64_t d = mk - base;
    return d > ((1ull << 59) - 1) ? ((1ull << 59) - 1) : d;
}

// ApproxTopN's octave of |c|^2: the exponent field of its f64 pattern, NaN counted in the top
// bin as the reference's histogram counts it (crates/paulistrings/src/truncation/builtin.rs:264-293).
template <typename T>
__device__ __forceinline__ uint32_t octave_bin(T c) {
    const double v = to_f64(c);
    const double m = __dmul_rn(v, v);
    if (isnan(m)) return 2047u;
    return (uint32_t)((uint64_t)__double_as_longlong(m) >> 52);
}

// Select key of the octave: 0 for NaN (never kept), else octave + 1.
template <typename T>
__device__ __forceinline__ uint64_t octave_key(T c) {
    const double v = to_f64(c);
    const double m = __dmul_rn(v, v);
    if (isnan(m)) return 0ull;
    return ((uint64_t)__double_as_longlong(m) >> 52) + 1ull;
}

// The learned pass's ranking: score = log|c| (floored at -200, so a zero coefficient stays
// finite) + the scorer's prediction f, as a select key: the score's order-preserving f32
// pattern shifted up (0 for a NaN score, never kept), larger kept first.
template <typename T>
__device__ __forceinline__ float log_abs_coeff(T c);
template <>
__device__ __forceinline__ float log_abs_coeff<double>(double c) {
    return fmaxf((float)log(fabs(c)), -200.0f);
}
template <>
__device__ __forceinline__ float log_abs_coeff<float>(float c) {
    return fmaxf(logf(fabsf(c)), -200.0f);
}
__device__ __forceinline__ uint64_t score_select_key(float y) {
    const uint32_t u = __float_as_uint(y);
    if (y != y) return 0;  // NaN: never kept
    const uint32_t order = (u & 0x80000000u) ? ~u : (u | 0x80000000u);
    return (uint64_t)order << 31;
}
template <typename T>
__device__ __forceinline__ uint64_t score_key(T c, float f) {
    return score_select_key(__fadd_rn(log_abs_coeff<T>(c), f));
}

// A coefficient's bit pattern in a 64-bit word and back, so a loop can issue all of its loads
// before it uses any of them.
__device__ __forceinline__ uint64_t raw_bits(double v) { return (uint64_t)__double_as_longlong(v); }
__device__ __forceinline__ uint64_t raw_bits(float v) { return (uint64_t)__float_as_uint(v); }
template <typename T>
__device__ __forceinline__ T from_raw(uint64_t r);
template <>
__device__ __forceinline__ double from_raw<double>(uint64_t r) { return __longlong_as_double((long long)r); }
template <>
__device__ __forceinline__ float from_raw<float>(uint64_t r) { return __uint_as_float((uint32_t)r); }

// Knuth TwoSum: s + e == a + b exactly.
template <typename T>
__device__ __forceinline__ void two_sum(T a, T b, T& s, T& e) {
    s = add_rn(a, b);
    T bb = add_rn(s, -a);
    T aa = add_rn(s, -bb);
    e = add_rn(add_rn(a, -aa), add_rn(b, -bb));
}

// ---------------------------------------------------------------------------
// keep program (postfix; KeepProgram, crates/paulistrings/src/engine/gpu/truncation.rs:24-102)
// ---------------------------------------------------------------------------
template <int W>
__device__ __forceinline__ bool keep_eval(const KeepProg& p, const uint64_t* k, double c) {
    switch (p.fast) {  // uniform across the grid
    case 0: return true;
    case 1: return p.fast_eps2 < 0.0 || __dmul_rn(c, c) > p.fast_eps2;
    case 2: return key_weight<W>(k) <= (uint64_t)p.fast_k;
    case 3: return (p.fast_eps2 < 0.0 || __dmul_rn(c, c) > p.fast_eps2) && key_weight<W>(k) <= (uint64_t)p.fast_k;
    default: break;
    }
    if (p.n == 0) return true;
    uint32_t stack = 0;  // bit stack
    int sp = 0;
    for (int i = 0; i < p.n; ++i) {
        int op = p.op[i];
        if (op == 0) {
            stack |= 1u << sp;
            ++sp;
        } else if (op == 1) {
            double e2 = p.eps2[i];
            bool v = (e2 < 0.0) || (__dmul_rn(c, c) > e2);
            stack = (stack & ~(1u << sp)) | ((uint32_t)v << sp);
            ++sp;
        } else if (op == 2) {
            bool v = key_weight<W>(k) <= (uint64_t)p.iarg[i];
            stack = (stack & ~(1u << sp)) | ((uint32_t)v << sp);
            ++sp;
        } else {
            bool b = (stack >> (sp - 1)) & 1u;
            bool a = (stack >> (sp - 2)) & 1u;
            sp -= 2;
            bool v = (op == 3) ? (a && b) : (a || b);
            stack = (stack & ~(1u << sp)) | ((uint32_t)v << sp);
            ++sp;
        }
    }
    return sp > 0 ? ((stack >> (sp - 1)) & 1u) != 0 : true;
}

// ---------------------------------------------------------------------------
// decoupled look-back over tiles for a 64-bit sum (flag in the top two bits)
// ---------------------------------------------------------------------------
constexpr unsigned long long kFlagAgg = 1ull << 62;
constexpr unsigned long long kFlagInc = 2ull << 62;
constexpr unsigned long long kValMask = (1ull << 62) - 1;

// Exclusive prefix of tile `tile`, computed by one full warp after the tile published its
// aggregate: each poll reads 32 predecessors at once, sums the aggregates up to the nearest
// inclusive prefix, and moves the window back only when none of the 32 holds one.
// Returns the same value in every lane.
// `limit` > 0 replaces the handle's spin limit for this wait (failure injection).
__device__ __forceinline__ unsigned long long lookback_sum_warp(const unsigned long long* status, unsigned int tile,
                                                               Ctl* ctl, uint32_t info, long long limit = 0) {
    const int lane = threadIdx.x & 31;
    unsigned long long acc = 0;
    long long base = (long long)tile - 1;
    long long spins = 0;
    while (base >= 0) {
        const long long t = base - lane;
        unsigned long long v = t >= 0 ? ld_acquire_u64(status + t) : kFlagInc;  // before tile 0: prefix 0
        const unsigned long long f = v & ~kValMask;
        const unsigned int empty = __ballot_sync(0xffffffffu, f == 0);
        const unsigned int inc = __ballot_sync(0xffffffffu, f == kFlagInc);
        const int first_inc = inc ? __ffs(inc) - 1 : 32;
        const unsigned int need = first_inc >= 31 ? 0xffffffffu : ((2u << first_inc) - 1u);
        if (empty & need) {
            if (++spins > (limit > 0 ? limit : spin_limit(ctl))) {
                if (lane == 0) raise_err(ctl, ERR_TIMEOUT, info);
                return acc;
            }
            __nanosleep(20);
            continue;
        }
        unsigned long long val = lane <= first_inc ? (v & kValMask) : 0ull;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) val += __shfl_xor_sync(0xffffffffu, val, o);
        acc += val;
        if (first_inc < 32) break;
        base -= 32;
    }
    return acc;
}

// Block-wide exclusive sum over threads (blockDim.x a multiple of 32, <= 1024).
template <int BLOCK>
__device__ __forceinline__ unsigned int block_exclusive_sum(unsigned int v, unsigned int* smem_warp,
                                                            unsigned int& total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        unsigned int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) smem_warp[warp] = x;
    __syncthreads();
    if (warp == 0) {
        unsigned int w = lane < BLOCK / 32 ? smem_warp[lane] : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            unsigned int y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        if (lane < BLOCK / 32) smem_warp[lane] = w;
    }
    __syncthreads();
    unsigned int warp_prefix = warp ? smem_warp[warp - 1] : 0u;
    total = smem_warp[BLOCK / 32 - 1];
    __syncthreads();
    return warp_prefix + x - v;
}

}  // namespace psb
