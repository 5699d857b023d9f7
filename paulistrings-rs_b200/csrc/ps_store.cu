// ps_store.cu -- ingest, readout and layer-pass kernels of the device store.
//
//   k_pack / k_unpack      host row layout (x[W], z[W]) <-> packed keys (x words, z words)
//   k_sort_hist, k_sort_pass
//                          onesweep LSD radix sort of (key, index) pairs: one upfront pass
//                          builds every 8-bit digit histogram in shared memory, then one
//                          scatter pass per digit ranks a tile stably (warp match_any) and
//                          finds its global bin offsets by a decoupled look-back per bin.
//                          Digits that are constant over the input are skipped.
//   k_dedup                sum runs of equal keys in input order, drop exact zeros (and keep
//                          rejects), compact with a look-back (BuildAccumulator::finalize,
//                          crates/paulistrings/src/pauli_sum/accumulator.rs:35-56)
//   k_topn_select_all      TopN select on the bit pattern of |c|^2 (NaN lowest) in one
//                          cooperative launch: a digit-1 bin from the merge's histogram, the bin's
//                          keys gathered, 13-bit digit rounds until at most 4096 keys remain, then
//                          an in-block radix select (TopN::finalize_layer,
//                          crates/paulistrings/src/truncation/builtin.rs:73-129); the multi-launch
//                          k_topn_hist1 / k_topn_cand / k_topn_hist_cand / k_topn_select path when
//                          the device cannot run it
//   k_topn_compact         order-preserving compaction keeping everything above the boundary and
//                          the first `quota` boundary ties in key order
//   k_topn_compact_cls     the same when every tie is kept, also listing the next rotation
//                          layer's partners (its idx, divergence ranks and partner count)
//   k_expect_*             <psi|O|psi> in a product state, float64 partial sums reduced in a
//                          fixed order (readout/product_state.rs:84-101)
#include "ps_device.cuh"
#include "ps_rotlayer.cuh"
#include "ps_store.h"

#include <algorithm>
#include <atomic>
#include <cstddef>
#include <type_traits>

namespace psb {

constexpr int kThreads = 256;

// Liveness of the rows e0, e0 + 32, e0 + 64, ... of a possibly slotted store (slots hold more
// than 32 rows), one division up front and a compare per step.
struct SlotWalk {
    uint32_t q = 0, r = 0;
    __device__ SlotWalk(const SlotMap& s, uint64_t e0) {
        if (s.count) {  // a slotted store spans fewer than 2^32 rows
            q = (uint32_t)e0 / s.rows;
            r = (uint32_t)e0 - q * s.rows;
        }
    }
    // call only for a row below the store's span
    __device__ bool live(const SlotMap& s) const { return !s.count || r < __ldg(s.count + q); }
    __device__ void step32(const SlotMap& s) {
        r += 32;
        if (r >= s.rows) {
            r -= s.rows;
            ++q;
        }
    }
};
__device__ __forceinline__ bool slot_live(const SlotMap& s, uint64_t e) {
    if (!s.count) return true;
    const uint32_t q = (uint32_t)e / s.rows;  // a slotted store spans fewer than 2^32 rows
    return (uint32_t)e - q * s.rows < __ldg(s.count + q);
}

// ---------------------------------------------------------------------------
// pack / unpack
// ---------------------------------------------------------------------------
template <int W, typename T>
__global__ void k_pack(const uint64_t* __restrict__ x, const uint64_t* __restrict__ z, const double* __restrict__ c,
                       uint64_t n, uint32_t num_qubits, uint64_t* __restrict__ keys, T* __restrict__ coef,
                       uint32_t* __restrict__ vals, Ctl* ctl) {
    uint64_t sup[W];
#pragma unroll
    for (int w = 0; w < W; ++w) sup[w] = 0;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t k[2 * W];
        uint64_t leak = 0;
#pragma unroll
        for (int w = 0; w < W; ++w) {
            k[w] = x[i * W + w];
            k[W + w] = z[i * W + w];
            sup[w] |= k[w] | k[W + w];
            uint32_t first = 64u * w;
            uint64_t live = num_qubits >= first + 64 ? ~0ull : (num_qubits <= first ? 0ull : ((1ull << (num_qubits - first)) - 1));
            leak |= (k[w] | k[W + w]) & ~live;
        }
        if (leak) raise_err(ctl, ERR_KEY_RANGE, 401);
        store_key<W>(keys, i, k);
        coef[i] = (T)c[i];
        vals[i] = (uint32_t)i;
    }
    // the union of the supports (ctl->support, cleared by the launcher), one atomic per warp and word
#pragma unroll
    for (int w = 0; w < W; ++w) {
        const uint32_t lo = __reduce_or_sync(0xffffffffu, (uint32_t)sup[w]);
        const uint32_t hi = __reduce_or_sync(0xffffffffu, (uint32_t)(sup[w] >> 32));
        const uint64_t v = (uint64_t)hi << 32 | lo;
        if ((threadIdx.x & 31) == 0 && v) atomicOr(&ctl->support[w], (unsigned long long)v);
    }
}

template <int W, typename T>
__global__ void k_unpack(const uint64_t* __restrict__ keys, const T* __restrict__ coef, uint64_t n,
                         uint64_t* __restrict__ x, uint64_t* __restrict__ z, double* __restrict__ c) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t k[2 * W];
        load_key<W>(keys, i, k);
#pragma unroll
        for (int w = 0; w < W; ++w) {
            x[i * W + w] = k[w];
            z[i * W + w] = k[W + w];
        }
        c[i] = to_f64(coef[i]);
    }
}

// Counts rows that break "strictly increasing keys, nonzero coefficients" into count[5];
// an upload that passes is already in store form and skips the sort.
template <int W, typename T>
__global__ void __launch_bounds__(kThreads) k_check_sorted(const uint64_t* __restrict__ keys,
                                                           const T* __restrict__ coef, uint64_t n, Ctl* ctl) {
    unsigned int bad = 0;
    for (uint64_t i = blockIdx.x * (uint64_t)kThreads + threadIdx.x; i < n; i += (uint64_t)gridDim.x * kThreads) {
        uint64_t k[2 * W];
        load_key<W>(keys, i, k);
        bool ok = coef[i] != T(0);
        if (i > 0) {
            uint64_t p[2 * W];
            load_key<W>(keys, i - 1, p);
            ok = ok && key_lt<W>(p, k);
        }
        bad += ok ? 0u : 1u;
    }
    bad = __reduce_add_sync(0xffffffffu, bad);
    if ((threadIdx.x & 31) == 0 && bad) atomicAdd(&ctl->count[5], (unsigned long long)bad);
}

// ---------------------------------------------------------------------------
// onesweep radix sort
// ---------------------------------------------------------------------------
template <int W>
__device__ __forceinline__ uint32_t digit_of(const uint64_t* k, int d) {
    int wi = 2 * W - 1 - (d >> 3);
    return (uint32_t)((k[wi] >> ((d & 7) * 8)) & 0xFFu);
}

template <int W>
__global__ void __launch_bounds__(kThreads) k_sort_hist(const uint64_t* __restrict__ keys, uint64_t n,
                                                        unsigned int* __restrict__ hist) {
    constexpr int ND = 16 * W;
    extern __shared__ unsigned int sh[];  // ND x 256
    for (int i = threadIdx.x; i < ND * 256; i += kThreads) sh[i] = 0;
    __syncthreads();
    for (uint64_t i = blockIdx.x * (uint64_t)kThreads + threadIdx.x; i < n; i += (uint64_t)gridDim.x * kThreads) {
        uint64_t k[2 * W];
        load_key<W>(keys, i, k);
#pragma unroll
        for (int d = 0; d < ND; ++d) atomicAdd(&sh[d * 256 + digit_of<W>(k, d)], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < ND * 256; i += kThreads)
        if (sh[i]) atomicAdd(&hist[i], sh[i]);
}

template <int W>
struct SortTile {
    static constexpr int ITEMS = W == 1 ? 8 : (W == 2 ? 4 : 2);
    static constexpr int TILE = kThreads * ITEMS;
};

constexpr unsigned int kSFlagAgg = 1u << 30;
constexpr unsigned int kSFlagInc = 2u << 30;
constexpr unsigned int kSValMask = (1u << 30) - 1;

template <int W>
__global__ void __launch_bounds__(kThreads) k_sort_pass(const uint64_t* __restrict__ kin, const uint32_t* __restrict__ vin,
                                                        uint64_t* __restrict__ kout, uint32_t* __restrict__ vout,
                                                        uint64_t n, int d, const unsigned int* __restrict__ bin_base,
                                                        unsigned int* status, Ctl* ctl) {
    constexpr int ITEMS = SortTile<W>::ITEMS;
    constexpr int TILE = SortTile<W>::TILE;
    constexpr int WARPS = kThreads / 32;
    __shared__ unsigned int s_tile;
    __shared__ unsigned int s_whist[WARPS][256];
    __shared__ unsigned int s_base[256];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int i = tid; i < WARPS * 256; i += kThreads) (&s_whist[0][0])[i] = 0;
    if (tid == 0) s_tile = atomicAdd(&ctl->tile_counter[4], 1u);
    __syncthreads();
    const unsigned int tile = s_tile;
    const uint64_t t0 = (uint64_t)tile * TILE;
    const unsigned int lanemask_lt = (1u << lane) - 1u;

    uint64_t k[ITEMS][2 * W];
    uint32_t v[ITEMS];
    uint32_t dig[ITEMS];
    uint32_t rank[ITEMS];
#pragma unroll
    for (int i = 0; i < ITEMS; ++i) {
        uint64_t e = t0 + (uint64_t)warp * 32 * ITEMS + (uint64_t)i * 32 + lane;
        bool valid = e < n;
        if (valid) {
            load_key<W>(kin, e, k[i]);
            v[i] = vin[e];
            dig[i] = digit_of<W>(k[i], d);
        } else {
            dig[i] = 256u + lane;  // unique sentinel, never counted
        }
        unsigned int peers = __match_any_sync(0xffffffffu, dig[i]);
        unsigned int before = 0;
        if (valid) before = s_whist[warp][dig[i]];
        __syncwarp();
        rank[i] = before + __popc(peers & lanemask_lt);
        if (valid && (peers & lanemask_lt) == 0) s_whist[warp][dig[i]] = before + __popc(peers);
        __syncwarp();
    }
    __syncthreads();
    // per bin: exclusive offsets over warps, tile count, global look-back
    {
        const int b = tid;  // kThreads == 256 bins
        unsigned int run = 0;
        for (int w = 0; w < WARPS; ++w) {
            unsigned int c = s_whist[w][b];
            s_whist[w][b] = run;
            run += c;
        }
        unsigned int* st = status + (size_t)tile * 256 + b;
        unsigned int prefix = 0;
        if (tile == 0) {
            st_release_u32(st, kSFlagInc | run);
        } else {
            st_release_u32(st, kSFlagAgg | run);
            long long spins = 0;
            for (int t = (int)tile - 1; t >= 0;) {
                unsigned int s = ld_acquire_u32(status + (size_t)t * 256 + b);
                unsigned int f = s & ~kSValMask;
                if (f == 0) {
                    if (++spins > spin_limit(ctl)) {
                        raise_err(ctl, ERR_TIMEOUT, 501);
                        break;
                    }
                    __nanosleep(32);
                    continue;
                }
                prefix += s & kSValMask;
                if (f == kSFlagInc) break;
                --t;
            }
            st_release_u32(st, kSFlagInc | (prefix + run));
        }
        s_base[b] = bin_base[b] + prefix;
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < ITEMS; ++i) {
        uint64_t e = t0 + (uint64_t)warp * 32 * ITEMS + (uint64_t)i * 32 + lane;
        if (e >= n) continue;
        uint64_t pos = (uint64_t)s_base[dig[i]] + s_whist[warp][dig[i]] + rank[i];
        if (!PS_GUARD(ctl, pos < n, 502)) continue;
        store_key<W>(kout, pos, k[i]);
        vout[pos] = v[i];
    }
}

// ---------------------------------------------------------------------------
// dedup after the sort: runs of equal keys summed in input (stable) order
// ---------------------------------------------------------------------------
template <int W, typename T>
__global__ void __launch_bounds__(kThreads) k_dedup(const uint64_t* __restrict__ keys, const uint32_t* __restrict__ vals,
                                                    const T* __restrict__ cin, uint64_t n, const KeepProg keep,
                                                    int compensated, uint64_t* __restrict__ okeys,
                                                    T* __restrict__ ocoef, unsigned long long* status, Ctl* ctl) {
    constexpr int ITEMS = 8;
    __shared__ unsigned int s_tile;
    __shared__ unsigned int s_warp[kThreads / 32];
    __shared__ unsigned long long s_off;
    const int tid = threadIdx.x;
    if (tid == 0) s_tile = atomicAdd(&ctl->tile_counter[5], 1u);
    __syncthreads();
    const unsigned int tile = s_tile;
    const uint64_t e0 = (uint64_t)tile * (kThreads * ITEMS) + (uint64_t)tid * ITEMS;
    T sums[ITEMS];
    uint32_t keepmask = 0;
#pragma unroll
    for (int i = 0; i < ITEMS; ++i) {
        uint64_t e = e0 + i;
        sums[i] = T(0);
        if (e >= n) continue;
        uint64_t k[2 * W];
        load_key<W>(keys, e, k);
        if (e > 0) {
            uint64_t p[2 * W];
            load_key<W>(keys, e - 1, p);
            if (key_eq<W>(p, k)) continue;  // not a run head
        }
        T s = add_rn(T(0), cin[vals[e]]);
        T comp = T(0);
        for (uint64_t f = e + 1; f < n; ++f) {
            uint64_t q[2 * W];
            load_key<W>(keys, f, q);
            if (!key_eq<W>(q, k)) break;
            T a = cin[vals[f]];
            if (compensated) {
                T hi, lo;
                two_sum(s, a, hi, lo);
                s = hi;
                comp = add_rn(comp, lo);
            } else {
                s = add_rn(s, a);
            }
        }
        if (compensated) s = add_rn(s, comp);
        sums[i] = s;
        if (s != T(0) && keep_eval<W>(keep, k, to_f64(s))) keepmask |= 1u << i;
    }
    unsigned int count = __popc(keepmask), total;
    unsigned int excl = block_exclusive_sum<kThreads>(count, s_warp, total);
    if (tid < 32) {
        unsigned long long p = 0;
        if (tile == 0) {
            if (tid == 0) st_release_u64(status + tile, kFlagInc | (unsigned long long)total);
        } else {
            if (tid == 0) st_release_u64(status + tile, kFlagAgg | (unsigned long long)total);
            p = lookback_sum_warp(status, tile, ctl, 601);
            if (tid == 0) st_release_u64(status + tile, kFlagInc | (p + total));
        }
        if (tid == 0) {
            s_off = p;
            if ((uint64_t)(tile + 1) * (kThreads * ITEMS) >= n) ctl->count[2] = p + total;
        }
    }
    __syncthreads();
    unsigned long long o = s_off + excl;
#pragma unroll
    for (int i = 0; i < ITEMS; ++i) {
        if (!((keepmask >> i) & 1u)) continue;
        uint64_t k[2 * W];
        load_key<W>(keys, e0 + i, k);
        if (PS_BOUNDS(ctl, o < n, 602)) {
            store_key<W>(okeys, o, k);
            ocoef[o] = sums[i];
        }
        ++o;
    }
}

// ---------------------------------------------------------------------------
// TopN radix-select on the bit pattern of |c|^2.  The select key is mag_key(c): 0 for NaN,
// else bits(|c|^2) + 1, so it is monotone in |c|^2 and NaN sorts lowest.  Digit 1 is
// key >> 52 (2048 bins, the octave of |c|^2); it is histogrammed by the merge kernel of
// the layer (or k_topn_hist1 when no merge ran), the boundary bin's keys are gathered into a
// candidate buffer, and the remaining 52 bits are selected over the candidates in four
// 13-bit digits.  aux[0] prefix, aux[1] mask, aux[2] remaining rank, aux[3] count above,
// count[4] candidates.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads) k_topn_hist1(const double* __restrict__ c64, const float* __restrict__ c32,
                                                         uint64_t n, unsigned int* __restrict__ hist, SlotMap slots,
                                                         const float* __restrict__ fpred) {
    __shared__ unsigned int sh[kTopnBins1];
    for (int i = threadIdx.x; i < kTopnBins1; i += kThreads) sh[i] = 0;
    __syncthreads();
    for (uint64_t i = blockIdx.x * (uint64_t)kThreads + threadIdx.x; i < n; i += (uint64_t)gridDim.x * kThreads) {
        if (!slot_live(slots, i)) continue;
        uint64_t mk;
        if (fpred)
            mk = c64 ? score_key<double>(c64[i], fpred[i]) : score_key<float>(c32[i], fpred[i]);
        else
            mk = c64 ? mag_key<double>(c64[i]) : mag_key<float>(c32[i]);
        atomicAdd(&sh[mk >> 52], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kTopnBins1; i += kThreads)
        if (sh[i]) atomicAdd(&hist[i], sh[i]);
}

// One block: pick the bin holding the remaining rank, counting from the top; clears the histogram.
template <int BINS>
__global__ void __launch_bounds__(1024) k_topn_select(unsigned int* __restrict__ hist, int shift, int bits, Ctl* ctl) {
    constexpr int PER = BINS / 1024;
    __shared__ unsigned long long s_part[1024];
    __shared__ int s_choice;
    __shared__ unsigned long long s_above;
    const int t = threadIdx.x;
    if (t == 0) {
        s_choice = 0;
        s_above = 0;
    }
    // thread t owns bins [BINS - (t + 1) * PER, BINS - t * PER), highest first
    unsigned long long mine = 0;
    for (int q = 0; q < PER; ++q) mine += hist[BINS - 1 - (t * PER + q)];
    s_part[t] = mine;
    __syncthreads();
    for (int o = 1; o < 1024; o <<= 1) {  // inclusive scan over threads (top bins first)
        unsigned long long v = t >= o ? s_part[t - o] : 0ull;
        __syncthreads();
        s_part[t] += v;
        __syncthreads();
    }
    const unsigned long long r = ctl->aux[2];
    const unsigned long long before = t ? s_part[t - 1] : 0ull;
    if (before < r && s_part[t] >= r) {
        unsigned long long acc = before;
        for (int q = 0; q < PER; ++q) {
            const int bin = BINS - 1 - (t * PER + q);
            const unsigned long long c = hist[bin];
            if (acc + c >= r) {
                s_choice = bin;
                s_above = acc;
                break;
            }
            acc += c;
        }
    }
    __syncthreads();
    for (int q = 0; q < PER; ++q) hist[t * PER + q] = 0;
    if (t == 0) {
        const unsigned long long above = s_above;
        ctl->aux[0] |= (unsigned long long)s_choice << shift;
        ctl->aux[1] |= ((1ull << bits) - 1ull) << shift;
        ctl->aux[2] = r - above;
        ctl->aux[3] += above;
    }
}

// ---------------------------------------------------------------------------
// The whole select in one cooperative launch (every block resident): block 0 picks the digit-1
// bin from the histogram the merge built, every block gathers the boundary bin's keys into its
// own candidate segment, then four 13-bit digits each histogram the candidates grid-wide and
// block 0 picks the bin.  Phases are separated by bounded grid barriers; a barrier that gives
// up flags ERR_TIMEOUT and every block returns.  Replaces ten launches per pass.
// ---------------------------------------------------------------------------
constexpr int kSelThreads = 256;

// Grid barrier on two words (arrivals, generation), zero at launch.  Bounded by the handle's
// spin limit.  Values other blocks wrote before the barrier are read after it with L1-bypassing
// loads (__ldcg): a line this SM cached before the barrier may be stale.
__device__ __forceinline__ bool grid_barrier(unsigned int* bar, Ctl* ctl, uint32_t info) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        s_ok = 1;
        const unsigned int gen = ld_acquire_u32(&bar[1]);  // before arriving: the release cannot come earlier
        __threadfence();
        if (atomicAdd(&bar[0], 1u) == gridDim.x - 1) {
            bar[0] = 0;  // every other block waits on the generation word
            __threadfence();
            st_release_u32(&bar[1], gen + 1);
        } else {
            long long spins = 0;
            while (ld_acquire_u32(&bar[1]) == gen) {
                if (++spins > spin_limit(ctl)) {
                    raise_err(ctl, ERR_TIMEOUT, info);
                    s_ok = 0;
                    break;
                }
                __nanosleep(32);
            }
        }
        __threadfence();
    }
    __syncthreads();
    return s_ok != 0;
}

// One block of kSelThreads: pick the bin of hist (BINS bins, counted from the top) holding the
// remaining rank aux[2]; update prefix, mask, rank and count above, record the bin's count in
// aux[4]; clear hist.
template <int BINS>
__device__ __forceinline__ void block_select(unsigned int* __restrict__ hist, int shift, int bits, Ctl* ctl,
                                             unsigned long long* s_part) {
    constexpr int PER = BINS / kSelThreads;
    __shared__ int s_choice;
    __shared__ unsigned long long s_above, s_count;
    const int t = threadIdx.x;
    if (t == 0) {
        s_choice = 0;
        s_above = 0;
        s_count = 0;
    }
    unsigned long long mine = 0;
    for (int q = 0; q < PER; ++q) mine += __ldcg(&hist[BINS - 1 - (t * PER + q)]);
    s_part[t] = mine;
    __syncthreads();
    for (int o = 1; o < kSelThreads; o <<= 1) {
        unsigned long long v = t >= o ? s_part[t - o] : 0ull;
        __syncthreads();
        s_part[t] += v;
        __syncthreads();
    }
    const unsigned long long r = __ldcg(&ctl->aux[2]);
    const unsigned long long before = t ? s_part[t - 1] : 0ull;
    if (before < r && s_part[t] >= r) {
        unsigned long long acc = before;
        for (int q = 0; q < PER; ++q) {
            const int bin = BINS - 1 - (t * PER + q);
            const unsigned long long c = __ldcg(&hist[bin]);
            if (acc + c >= r) {
                s_choice = bin;
                s_above = acc;
                s_count = c;
                break;
            }
            acc += c;
        }
    }
    __syncthreads();
    for (int q = 0; q < PER; ++q) hist[t * PER + q] = 0;
    if (t == 0) {
        const unsigned long long above = s_above;
        ctl->aux[0] |= (unsigned long long)s_choice << shift;
        ctl->aux[1] |= ((1ull << bits) - 1ull) << shift;
        ctl->aux[2] = r - above;
        ctl->aux[3] += above;
        ctl->aux[4] = s_count;  // keys in the chosen bin
    }
    __syncthreads();
}

// Block-wide (kSelThreads threads): the boundary of the `total` candidate keys in sk (shared
// memory) at rank r from the top (1 <= r <= total), by an in-block radix select of eight 8-bit
// digits (a histogram of the keys that match the digits fixed so far, and one warp finding the
// digit that holds the remaining rank).  Sets the select's final prefix (the boundary key
// itself, full mask), the rank left within the keys equal to it, adds the count of candidates
// strictly larger to the count above, and records the number of candidates equal to the
// boundary (aux[4]).
__device__ __forceinline__ void block_sort_boundary(const uint64_t* sk, unsigned int total, unsigned long long r,
                                                    Ctl* ctl) {
    static_assert(kSelThreads == 256, "one histogram bin per thread");
    __shared__ unsigned int h[256];
    __shared__ unsigned long long s_prefix, s_mask, s_r, s_above, s_pass_above;
    __shared__ unsigned int s_bin, s_cnt;
    const int tid = threadIdx.x, lane = tid & 31;
    if (tid == 0) {
        s_prefix = 0;
        s_mask = 0;
        s_r = r;
        s_above = 0;
        s_cnt = 0;
    }
    __syncthreads();
    for (int shift = 56; shift >= 0; shift -= 8) {
        h[tid] = 0;
        __syncthreads();
        const uint64_t pfx = s_prefix, msk = s_mask;
        for (unsigned int i = tid; i < total; i += kSelThreads) {
            const uint64_t k = sk[i];
            if ((k & msk) == pfx) atomicAdd(&h[(unsigned int)(k >> shift) & 255u], 1u);
        }
        __syncthreads();
        if (tid < 32) {
            // lane l holds the bins 255 - 8 l - j (j < 8), counted from the top
            unsigned int c[8], tot = 0;
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                c[j] = h[255 - (8 * lane + j)];
                tot += c[j];
            }
            unsigned int incl = tot;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const unsigned int v = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += v;
            }
            const unsigned long long rr = s_r;
            const unsigned int excl = incl - tot;
            if (excl < rr && incl >= rr) {  // exactly one lane: its bins hold the remaining rank
                unsigned int acc = excl;
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    if (acc + c[j] >= rr) {
                        s_bin = 255u - (unsigned int)(8 * lane + j);
                        s_pass_above = acc;
                        s_cnt = c[j];
                        break;
                    }
                    acc += c[j];
                }
            }
        }
        __syncthreads();
        if (tid == 0) {
            s_prefix |= (unsigned long long)s_bin << shift;
            s_mask |= 0xFFull << shift;
            s_r -= s_pass_above;
            s_above += s_pass_above;
        }
        __syncthreads();
    }
    if (tid == 0) {
        ctl->aux[0] = s_prefix;
        ctl->aux[1] = ~0ull;
        ctl->aux[2] = s_r;
        ctl->aux[3] += s_above;
        ctl->aux[4] = s_cnt;
    }
}

// SCORE: the learned pass's variant (select keys from score_key of the coefficient and the
// prediction); the plain variant stays within four resident blocks per SM, the scored one three.
template <typename T, bool SCORE>
__global__ void __launch_bounds__(kSelThreads, SCORE ? 3 : 4) k_topn_select_all(const T* __restrict__ coef,
                                                                 const uint64_t* __restrict__ sel, int window,
                                                                 uint64_t base, uint64_t n_arg, Ctl* ctl,
                                                                 unsigned int* __restrict__ hist,
                                                                 uint64_t* __restrict__ cand, uint64_t cand_cap,
                                                                 uint64_t seg_cap, unsigned int* __restrict__ seg_count,
                                                                 SlotMap slots, unsigned int* bar,
                                                                 const float* __restrict__ fpred,
                                                                 unsigned long long keep_n,
                                                                 unsigned long long* __restrict__ cstatus,
                                                                 uint32_t ncstatus, int deferred) {
    constexpr int ITEMS = 16;
    constexpr int CHUNK = kSelThreads * ITEMS;
    // deferred: the host launched this pass without reading the layer's counts; n_arg bounds the
    // rows (it sized the grid and the segments), the merge left the span, and a failed layer
    // (an error flag already set) writes nothing more
    if (deferred && ctl->err) return;
    const uint64_t n = deferred ? ctl->span : n_arg;
    __shared__ unsigned int sh[kTopnBinsN];
    __shared__ unsigned long long s_part[kSelThreads];
    __shared__ unsigned long long s_base;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const unsigned int lt = (1u << lane) - 1u;
    // the compaction's look-back words and dispenser, reset here for the launch that follows
    for (uint32_t i = blockIdx.x * kSelThreads + tid; i < ncstatus; i += gridDim.x * kSelThreads) cstatus[i] = 0;
    // digit 1 (block 0 first sets the select's state: no prefix, rank keep_n from the top).
    // Deferred, the live rows may fit the quota (the host checks that itself otherwise): then
    // every live row is kept, the histogram is cleared and nothing is selected.
    const bool keep_all = deferred && ctl->count[1] <= keep_n;
    if (blockIdx.x == 0) {
        if (tid < 8) ctl->aux[tid] = tid == 2 ? keep_n : 0ull;
        if (tid == 0) {
            ctl->tile_counter[6] = 0;
            ctl->topn_all = keep_all ? 1ull : 0ull;
            ctl->count[0] = 0;  // the compaction's partner count for the next layer (none when it lists none)
            ctl->count[3] = 0;  // its output count (no tile writes it when the span is empty)
        }
        __syncthreads();
        if (keep_all) {
            for (int q = tid; q < kTopnBins1; q += kSelThreads) hist[q] = 0;
        } else {
            block_select<kTopnBins1>(hist, window ? 48 : 52, window ? 11 : 12, ctl, s_part);
        }
    }
    if (keep_all) return;  // every block: the same decision, before any barrier
    if (!grid_barrier(bar, ctl, 720)) return;
    // the boundary bin's keys into this block's segment
    {
        const uint64_t prefix = __ldcg(&ctl->aux[0]), mask = __ldcg(&ctl->aux[1]);
        if (window && blockIdx.x == 0 && tid == 0) {
            const uint64_t bin = prefix >> 48;
            if (bin == 0 || bin == 2047) ctl->aux[5] = 1;  // the boundary left the window: retry in full range
        }
        if (tid == 0) s_base = 0;
        __syncthreads();
        for (uint64_t c0 = (uint64_t)blockIdx.x * CHUNK; c0 < n; c0 += (uint64_t)gridDim.x * CHUNK) {
            const uint64_t wbase = c0 + (uint64_t)warp * 32 * ITEMS;
            uint64_t key[ITEMS];
            float fp[SCORE ? ITEMS : 1];
#pragma unroll
            for (int i = 0; i < ITEMS; ++i) {
                const uint64_t e = wbase + (uint64_t)i * 32 + lane;
                key[i] = e < n ? (sel ? sel[e] : raw_bits(coef[e])) : 0ull;
                if constexpr (SCORE) fp[i] = e < n ? fpred[e] : 0.0f;
            }
            unsigned int ball[ITEMS];
            unsigned int wc = 0;
#pragma unroll
            for (int i = 0; i < ITEMS; ++i) {
                if (!sel) {
                    uint64_t mk;
                    if constexpr (SCORE)
                        mk = score_key<T>(from_raw<T>(key[i]), fp[i]);
                    else
                        mk = mag_key<T>(from_raw<T>(key[i]));
                    key[i] = window ? window_key(mk, base) : mk;
                }
                const uint64_t e = wbase + (uint64_t)i * 32 + lane;
                const bool hit = e < n && (key[i] & mask) == prefix && slot_live(slots, e);
                ball[i] = __ballot_sync(0xffffffffu, hit);
                wc += __popc(ball[i]);
            }
            // the warp's place in the block's segment: the order of the candidates does not
            // matter, so one shared atomic per warp replaces a block-wide scan (and its barriers)
            if (wc) {
                unsigned long long slot = 0;
                if (lane == 0) slot = atomicAdd(&s_base, (unsigned long long)wc);
                slot = __shfl_sync(0xffffffffu, slot, 0) + (uint64_t)blockIdx.x * seg_cap;
#pragma unroll
                for (int i = 0; i < ITEMS; ++i) {
                    if ((ball[i] >> lane) & 1u) {
                        const unsigned long long q = slot + __popc(ball[i] & lt);
                        if (PS_GUARD(ctl, q < cand_cap, 721)) cand[q] = key[i];
                    }
                    slot += __popc(ball[i]);
                }
            }
        }
        __syncthreads();
        if (tid == 0) seg_count[blockIdx.x] = (unsigned int)s_base;
    }
    if (!grid_barrier(bar, ctl, 722)) return;
    // Few candidates (the usual case at small sums): block 0 gathers them all into shared memory
    // and radix-selects the boundary there; no further grid barrier.  Every block sums the
    // segment lengths, so all take the same branch.
    {
        constexpr int kSortCap = kTopnBinsN / 2;  // 64-bit keys in the 8192-word histogram's space
        constexpr int SEGS_PER = 8;               // segments a thread of block 0 gathers (G <= 2048)
        unsigned long long mine = 0;
        for (unsigned int g = tid; g < gridDim.x; g += kSelThreads) mine += __ldcg(&seg_count[g]);
        s_part[tid] = mine;
        __syncthreads();
        for (int o = kSelThreads / 2; o > 0; o >>= 1) {
            if (tid < o) s_part[tid] += s_part[tid + o];
            __syncthreads();
        }
        const unsigned long long total = s_part[0];
        __syncthreads();
        const unsigned long long r = __ldcg(&ctl->aux[2]);
        if (total <= (unsigned long long)kSortCap && gridDim.x <= (unsigned int)(SEGS_PER * kSelThreads) && r >= 1 &&
            r <= total) {
            if (blockIdx.x != 0) return;
            uint64_t* sk = reinterpret_cast<uint64_t*>(sh);
            // gather: thread t takes segments [SEGS_PER t, SEGS_PER (t + 1)) at the exclusive sum of
            // the lengths before them
            unsigned int lens[SEGS_PER];
            unsigned long long own = 0;
#pragma unroll
            for (int q = 0; q < SEGS_PER; ++q) {
                const unsigned int g = (unsigned int)(SEGS_PER * tid + q);
                lens[q] = g < gridDim.x ? __ldcg(&seg_count[g]) : 0u;
                own += lens[q];
            }
            s_part[tid] = own;
            __syncthreads();
            for (int o = 1; o < kSelThreads; o <<= 1) {  // inclusive scan
                const unsigned long long v = tid >= o ? s_part[tid - o] : 0ull;
                __syncthreads();
                s_part[tid] += v;
                __syncthreads();
            }
            // each warp copies its 32 threads' segments in turn, its lanes side by side
            const unsigned long long first = s_part[tid] - own;
            for (int l = 0; l < 32; ++l) {
                unsigned long long at = __shfl_sync(0xffffffffu, first, l);
#pragma unroll
                for (int q = 0; q < SEGS_PER; ++q) {
                    const unsigned int len = __shfl_sync(0xffffffffu, lens[q], l);
                    const uint64_t* sg = cand + (uint64_t)(SEGS_PER * (warp * 32 + l) + q) * seg_cap;
                    for (unsigned int i = lane; i < len; i += 32) sk[at + i] = __ldcg(&sg[i]);
                    at += len;
                }
            }
            __syncthreads();
            block_sort_boundary(sk, (unsigned int)total, r, ctl);
            return;
        }
    }
    // four 13-bit digits over this block's own candidates (it reads what it wrote)
    const unsigned int len = seg_count[blockIdx.x];
    const uint64_t* seg = cand + (uint64_t)blockIdx.x * seg_cap;
    const int shifts[2][4] = {{39, 26, 13, 0}, {35, 22, 9, 0}};
    for (int d = 0; d < 4; ++d) {
        const int shift = shifts[window ? 1 : 0][d];
        for (int i = tid; i < kTopnBinsN; i += kSelThreads) sh[i] = 0;
        __syncthreads();
        const uint64_t prefix = __ldcg(&ctl->aux[0]), mask = __ldcg(&ctl->aux[1]);
        for (unsigned int i = tid; i < len; i += kSelThreads) {
            const uint64_t mk = seg[i];
            if ((mk & mask) == prefix) atomicAdd(&sh[(mk >> shift) & (kTopnBinsN - 1)], 1u);
        }
        __syncthreads();
        for (int i = tid; i < kTopnBinsN; i += kSelThreads)
            if (sh[i]) atomicAdd(&hist[i], sh[i]);
        if (!grid_barrier(bar, ctl, 723)) return;
        if (blockIdx.x == 0) block_select<kTopnBinsN>(hist, shift, 13, ctl, s_part);
        if (!grid_barrier(bar, ctl, 724)) return;
        // Once the chosen bin holds at most kSortCap keys, the remaining digits give way to one
        // block's select: every block appends its keys of the bin to a list in the (now zero)
        // histogram's space, and block 0 radix-selects among them, then zeroes the words it used.
        constexpr unsigned int kSortCap = kTopnBinsN / 2;
        const unsigned long long cnt = __ldcg(&ctl->aux[4]), r = __ldcg(&ctl->aux[2]);
        if (d < 3 && cnt <= kSortCap && r >= 1 && r <= cnt) {
            const uint64_t pfx = __ldcg(&ctl->aux[0]), msk = __ldcg(&ctl->aux[1]);
            uint64_t* list = reinterpret_cast<uint64_t*>(hist);
            unsigned long long* fill = &ctl->aux[6];
            for (unsigned int i0 = 0; i0 < len; i0 += kSelThreads) {
                const unsigned int i = i0 + tid;
                const uint64_t mk = i < len ? seg[i] : 0ull;
                const bool hit = i < len && (mk & msk) == pfx;
                const unsigned int b = __ballot_sync(0xffffffffu, hit);
                if (b) {
                    unsigned long long at = 0;
                    if (lane == 0) at = atomicAdd(fill, (unsigned long long)__popc(b));
                    at = __shfl_sync(0xffffffffu, at, 0) + __popc(b & lt);
                    if (hit && PS_GUARD(ctl, at < kSortCap, 725)) list[at] = mk;
                }
            }
            if (!grid_barrier(bar, ctl, 726)) return;
            if (blockIdx.x != 0) return;
            uint64_t* sk = reinterpret_cast<uint64_t*>(sh);
            const unsigned long long filled = __ldcg(fill);
            if (tid == 0) PS_GUARD(ctl, filled == cnt, 727);
            const unsigned int total = (unsigned int)min(cnt, (unsigned long long)kSortCap);
            const unsigned int used = (unsigned int)min(filled, (unsigned long long)kSortCap);
            for (unsigned int i = tid; i < total; i += kSelThreads) sk[i] = __ldcg(&list[i]);
            for (unsigned int i = tid; i < used; i += kSelThreads) list[i] = 0ull;
            __syncthreads();
            block_sort_boundary(sk, total, r, ctl);
            return;
        }
    }
}

// The compaction's key (key_mode): 0 mag_key of the coefficient, 1 a precomputed key (the
// scored TopN's score keys, same conventions: 0 never kept, larger kept first), 2 ApproxTopN's
// octave key, 3 none (every live row kept), 4 the learned score from the coefficient and the
// row's prediction.

// ApproxTopN's octave histogram of |c|^2 (2048 bins, NaN in the top one).
template <typename T>
__global__ void __launch_bounds__(kThreads) k_octave_hist(const T* __restrict__ coef, uint64_t n,
                                                          unsigned int* __restrict__ hist) {
    __shared__ unsigned int sh[kTopnBins1];
    for (int i = threadIdx.x; i < kTopnBins1; i += kThreads) sh[i] = 0;
    __syncthreads();
    for (uint64_t i = blockIdx.x * (uint64_t)kThreads + threadIdx.x; i < n; i += (uint64_t)gridDim.x * kThreads)
        atomicAdd(&sh[octave_bin<T>(coef[i])], 1u);
    __syncthreads();
    for (int i = threadIdx.x; i < kTopnBins1; i += kThreads)
        if (sh[i]) atomicAdd(&hist[i], sh[i]);
}

// Gather the keys of the boundary bin (order does not matter for the select): each block
// takes chunks of kThreads * 16 elements and appends their candidates to its own segment of
// the candidate buffer (seg_cap keys, room for every element of the block's chunks), so no
// counter is shared between blocks; seg_count[block] receives the segment's length.
template <typename T, bool SCORE>
__global__ void __launch_bounds__(kThreads) k_topn_cand(const T* __restrict__ coef, const uint64_t* __restrict__ sel,
                                                        int window, uint64_t base, uint64_t n, Ctl* ctl,
                                                        uint64_t* __restrict__ cand, uint64_t cand_cap,
                                                        uint64_t seg_cap, unsigned int* __restrict__ seg_count,
                                                        SlotMap slots, const float* __restrict__ fpred) {
    constexpr int ITEMS = 16;
    constexpr int CHUNK = kThreads * ITEMS;
    __shared__ unsigned int s_w[kThreads / 32];
    __shared__ unsigned long long s_base;
    const uint64_t prefix = ctl->aux[0], mask = ctl->aux[1];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const unsigned int lt = (1u << lane) - 1u;
    if (window && blockIdx.x == 0 && tid == 0) {
        const uint64_t bin = prefix >> 48;
        if (bin == 0 || bin == 2047) ctl->aux[5] = 1;  // the boundary left the window: retry in full range
    }
    if (tid == 0) s_base = 0;
    __syncthreads();
    for (uint64_t c0 = (uint64_t)blockIdx.x * CHUNK; c0 < n; c0 += (uint64_t)gridDim.x * CHUNK) {
        const uint64_t wbase = c0 + (uint64_t)warp * 32 * ITEMS;
        // every load of the chunk first, then the keys and ballots
        uint64_t key[ITEMS];
        float fp[SCORE ? ITEMS : 1];
#pragma unroll
        for (int i = 0; i < ITEMS; ++i) {
            const uint64_t e = wbase + (uint64_t)i * 32 + lane;
            key[i] = e < n ? (sel ? sel[e] : raw_bits(coef[e])) : 0ull;
            if constexpr (SCORE) fp[i] = e < n ? fpred[e] : 0.0f;
        }
        unsigned int ball[ITEMS];
        unsigned int wc = 0;
#pragma unroll
        for (int i = 0; i < ITEMS; ++i) {
            if (!sel) {
                uint64_t mk;
                if constexpr (SCORE)
                    mk = score_key<T>(from_raw<T>(key[i]), fp[i]);
                else
                    mk = mag_key<T>(from_raw<T>(key[i]));
                key[i] = window ? window_key(mk, base) : mk;
            }
            const uint64_t e = wbase + (uint64_t)i * 32 + lane;
            // a row in a slot's unused tail is no row: tested only for the few hits (a slot's
            // tail is allocated, so its value load above stays in bounds)
            const bool hit = e < n && (key[i] & mask) == prefix && slot_live(slots, e);
            ball[i] = __ballot_sync(0xffffffffu, hit);
            wc += __popc(ball[i]);
        }
        if (lane == 0) s_w[warp] = wc;
        __syncthreads();
        unsigned int wx = 0, tot = 0;
#pragma unroll
        for (int w = 0; w < kThreads / 32; ++w) {
            wx += w < warp ? s_w[w] : 0u;
            tot += s_w[w];
        }
        // this block's own segment of the candidate buffer: no counter shared between blocks
        const unsigned long long seg_used = s_base;
        __syncthreads();
        if (tid == 0) s_base = seg_used + tot;
        unsigned long long slot = (uint64_t)blockIdx.x * seg_cap + seg_used + wx;
#pragma unroll
        for (int i = 0; i < ITEMS; ++i) {
            if ((ball[i] >> lane) & 1u) {
                const unsigned long long q = slot + __popc(ball[i] & lt);
                if (PS_GUARD(ctl, q < cand_cap, 703)) cand[q] = key[i];
            }
            slot += __popc(ball[i]);
        }
        __syncthreads();
    }
    if (tid == 0) seg_count[blockIdx.x] = (unsigned int)s_base;
}

__global__ void __launch_bounds__(kThreads) k_topn_hist_cand(const uint64_t* __restrict__ cand, Ctl* ctl, int shift,
                                                             unsigned int* __restrict__ hist, uint64_t seg_cap,
                                                             const unsigned int* __restrict__ seg_count,
                                                             unsigned int nseg) {
    __shared__ unsigned int sh[kTopnBinsN];
    for (int i = threadIdx.x; i < kTopnBinsN; i += kThreads) sh[i] = 0;
    __syncthreads();
    const uint64_t prefix = ctl->aux[0], mask = ctl->aux[1];
    for (unsigned int g = blockIdx.x; g < nseg; g += gridDim.x) {
        const uint64_t* seg = cand + (uint64_t)g * seg_cap;
        const unsigned int len = seg_count[g];
        for (unsigned int i = threadIdx.x; i < len; i += kThreads) {
            const uint64_t mk = seg[i];
            if ((mk & mask) == prefix) atomicAdd(&sh[(mk >> shift) & (kTopnBinsN - 1)], 1u);
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kTopnBinsN; i += kThreads)
        if (sh[i]) atomicAdd(&hist[i], sh[i]);
}

// Order-preserving compaction, warp-striped: keeps keys above the boundary and the first
// `quota` boundary ties in key order, quota = keep_n - (count above the boundary), none when
// the boundary is NaN (the select leaves boundary and count above in aux[0] / aux[3]).
// key_mode 3 keeps every row.  Rows outside the slots of a slotted store are skipped.
// SCORE: the learned pass's variant (score keys from the prediction column, which the kept rows
// carry); the plain variant keeps its registers, and with them its residency, free of the log.
// One tile (the tile dispenser's next) per call.
template <int W, typename T, bool SCORE>
__device__ __forceinline__ void compact_tile(const uint64_t* __restrict__ keys, const T* __restrict__ coef,
                                             const uint64_t* __restrict__ sel, int key_mode, uint64_t base,
                                             uint64_t n, unsigned long long keep_n, uint64_t* __restrict__ okeys,
                                             T* __restrict__ ocoef, unsigned long long* status, Ctl* ctl,
                                             SlotMap slots, const float* __restrict__ fin, float* __restrict__ fout) {
    const unsigned long long quota = ctl->aux[0] == 0 ? 0ull : keep_n - ctl->aux[3];
    constexpr int ITEMS = 16;
    constexpr int TILE = kThreads * ITEMS;
    __shared__ unsigned int s_tile;
    __shared__ unsigned int s_wa[kThreads / 32], s_wt[kThreads / 32];
    __shared__ unsigned long long s_above, s_ties;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const unsigned int lt = (1u << lane) - 1u;
    if (tid == 0) s_tile = atomicAdd(&ctl->tile_counter[6], 1u);
    __syncthreads();
    const unsigned int tile = s_tile;
    if (tile > 0 && (uint64_t)tile * TILE >= n) return;  // past the span (a grid sized by a bound)
    const uint64_t boundary = ctl->aux[0] == 0 ? 0ull : ctl->aux[0] + base;  // a windowed select's key back in full range
    const uint64_t wbase = (uint64_t)tile * TILE + (uint64_t)warp * 32 * ITEMS;
    unsigned int ba[ITEMS], bt[ITEMS];
    unsigned int wa = 0, wt = 0;
    SlotWalk sw(slots, wbase + lane);
#pragma unroll
    for (int i = 0; i < ITEMS; ++i) {
        const uint64_t e = wbase + (uint64_t)i * 32 + lane;
        bool isa = false, ist = false;
        if (e < n) {
            // the key load does not wait for the liveness test (a slot's tail is allocated)
            uint64_t mk = 0ull;
            if (key_mode == 1)
                mk = sel[e];
            else if (key_mode == 2)
                mk = octave_key<T>(coef[e]);
            else if (key_mode == 0)
                mk = mag_key<T>(coef[e]);
            if constexpr (SCORE) {
                if (key_mode == 4) mk = score_key<T>(coef[e], fin[e]);
            }
            if (sw.live(slots)) {
                isa = key_mode == 3 || mk > boundary;  // key_mode 3 keeps every row (compacting slots)
                ist = key_mode != 3 && mk == boundary && boundary != 0;
            }
        }
        sw.step32(slots);
        ba[i] = __ballot_sync(0xffffffffu, isa);
        bt[i] = __ballot_sync(0xffffffffu, ist);
        wa += __popc(ba[i]);
        wt += __popc(bt[i]);
    }
    if (lane == 0) {
        s_wa[warp] = wa;
        s_wt[warp] = wt;
    }
    __syncthreads();
    unsigned int xa = 0, xt = 0, ta = 0, tt = 0;
#pragma unroll
    for (int w = 0; w < kThreads / 32; ++w) {
        xa += w < warp ? s_wa[w] : 0u;
        xt += w < warp ? s_wt[w] : 0u;
        ta += s_wa[w];
        tt += s_wt[w];
    }
    if (tid < 32) {
        unsigned long long agg = (unsigned long long)ta | ((unsigned long long)tt << 31);
        unsigned long long pre = 0;
        if (tile == 0) {
            if (tid == 0) st_release_u64(status + tile, kFlagInc | agg);
        } else {
            if (tid == 0) st_release_u64(status + tile, kFlagAgg | agg);
            pre = lookback_sum_warp(status, tile, ctl, 701);
            if (tid == 0) st_release_u64(status + tile, kFlagInc | (pre + agg));
        }
        if (tid == 0) {
            s_above = pre & ((1ull << 31) - 1);
            s_ties = pre >> 31;
            if ((uint64_t)(tile + 1) * TILE >= n) {
                unsigned long long tot_ties = s_ties + tt;
                ctl->count[3] = s_above + ta + (tot_ties < quota ? tot_ties : quota);
            }
        }
    }
    __syncthreads();
    unsigned long long arank = s_above + xa, trank = s_ties + xt;
#pragma unroll
    for (int i = 0; i < ITEMS; ++i) {
        const bool isa = (ba[i] >> lane) & 1u, ist = (bt[i] >> lane) & 1u;
        const unsigned long long ar = arank + __popc(ba[i] & lt), tr = trank + __popc(bt[i] & lt);
        if (isa || (ist && tr < quota)) {
            const unsigned long long pos = ar + (tr < quota ? tr : quota);
            const uint64_t e = wbase + (uint64_t)i * 32 + lane;
            uint64_t k[2 * W];
            load_key<W>(keys, e, k);
            if (PS_GUARD(ctl, pos < n, 702)) {
                store_key<W>(okeys, pos, k);
                ocoef[pos] = coef[e];
                if constexpr (SCORE) fout[pos] = fin[e];  // the learned pass's prediction travels with its row
            }
        }
        arank += __popc(ba[i]);
        trank += __popc(bt[i]);
    }
}

template <int W, typename T, bool SCORE>
__global__ void __launch_bounds__(kThreads) k_topn_compact(const uint64_t* __restrict__ keys, const T* __restrict__ coef,
                                                           const uint64_t* __restrict__ sel, int key_mode,
                                                           uint64_t base, uint64_t n, unsigned long long keep_n,
                                                           uint64_t* __restrict__ okeys, T* __restrict__ ocoef,
                                                           unsigned long long* status, Ctl* ctl, SlotMap slots,
                                                           const float* __restrict__ fin, float* __restrict__ fout,
                                                           int deferred) {
    // A select whose windowed boundary left the window writes nothing: the pass reruns in full
    // range and rewrites the output.  Deferred (see k_topn_select_all): the merge's span, no
    // write after a failed layer, and every live row kept when the select found them within the
    // quota.
    if (deferred) {
        if (ctl->err) return;
        n = ctl->span;
        if (ctl->topn_all) key_mode = 3;
    }
    if (key_mode != 2 && key_mode != 3 && ctl->aux[5]) return;
    compact_tile<W, T, SCORE>(keys, coef, sel, key_mode, base, n, keep_n, okeys, ocoef, status, ctl, slots, fin, fout);
}

// Plain TopN compaction that also classifies the kept rows for the next rotation layer (the work
// of that layer's k_classify, done while the keys are in registers).  When every key equal to the
// boundary is kept (the select's tie count aux[4] equals the rank left for the ties, aux[2]), a
// row is kept iff it is live and its key is at least the boundary, so a tile's kept count and its
// count of kept rows that emit a partner under the next layer are both local, and one look-back
// word carries the two (31 bits each).  The kept row goes to position pos; the j-th kept row that
// emits a partner gets idx[j] = pos and D[j] = its divergence rank from the (j-1)-th (unknown for
// the first of a warp, which k_level_reduce resolves), and the last tile publishes the partner
// count in count[0], as k_classify does.  Otherwise (the quota cuts the ties, or the boundary is
// NaN) the plain compaction runs and aux[7] tells the host that the next layer classifies itself.
// FLAGS: the layer's merge wrote each row's partner test under the next layer (nflag, one byte
// per row of the slotted store), so the first pass reads a byte instead of the key.
// SCORE: the inherited learned pass (keys score_key(c, f) from the carried predictions fin,
// which the kept rows carry to fout).
template <int W, typename T, bool FLAGS, bool SCORE = false>
__global__ void __launch_bounds__(kThreads, W == 1 ? (SCORE ? 4 : 8) : (W == 2 ? 4 : 2)) k_topn_compact_cls(const uint64_t* __restrict__ keys,
                                                               const T* __restrict__ coef, uint64_t base, uint64_t n,
                                                               unsigned long long keep_n, uint64_t* __restrict__ okeys,
                                                               T* __restrict__ ocoef, unsigned long long* status,
                                                               Ctl* ctl, SlotMap slots, const RotLayer<W> L,
                                                               uint32_t* __restrict__ idx, uint16_t* __restrict__ D,
                                                               const uint8_t* __restrict__ nflag, int deferred,
                                                               const float* __restrict__ fin = nullptr,
                                                               float* __restrict__ fout = nullptr) {
    // deferred: as k_topn_compact
    bool all = false;
    if (deferred) {
        if (ctl->err) return;
        n = ctl->span;
        all = ctl->topn_all != 0;
    }
    if (!all && ctl->aux[5]) return;  // the windowed boundary left the window: the pass reruns in full range
    if (!all && !(ctl->aux[0] != 0 && ctl->aux[4] == ctl->aux[2])) {
        if (blockIdx.x == 0 && threadIdx.x == 0) ctl->aux[7] = 1;
        compact_tile<W, T, SCORE>(keys, coef, nullptr, SCORE ? 4 : 0, base, n, keep_n, okeys, ocoef, status, ctl,
                                  slots, fin, fout);
        return;
    }
    constexpr int ITEMS = 16;
    constexpr int TILE = kThreads * ITEMS;
    constexpr unsigned long long kLow31 = (1ull << 31) - 1;
    __shared__ unsigned int s_tile;
    __shared__ unsigned int s_wk[kThreads / 32], s_wp[kThreads / 32];
    __shared__ unsigned long long s_kept, s_part;
    __shared__ AmpTab<T> A;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const unsigned int lt = (1u << lane) - 1u;
    if (tid == 0) s_tile = atomicAdd(&ctl->tile_counter[6], 1u);
    stage_amps<W, T>(L, A);
    __syncthreads();
    const unsigned int tile = s_tile;
    if (tile > 0 && (uint64_t)tile * TILE >= n) return;  // past the span (a grid sized by a bound)
    // a windowed select's key back in full range; every live row when all are kept
    const uint64_t boundary = all ? 0ull : ctl->aux[0] + base;
    const uint64_t wbase = (uint64_t)tile * TILE + (uint64_t)warp * 32 * ITEMS;
    unsigned int bk[ITEMS], bp[ITEMS];
    unsigned int wk = 0, wp = 0;
    SlotWalk sw(slots, wbase + lane);
#pragma unroll
    for (int i = 0; i < ITEMS; ++i) {
        const uint64_t e = wbase + (uint64_t)i * 32 + lane;
        bool kept = false, part = false;
        if (e < n) {
            // neither load waits for the liveness test (a slot's tail is allocated)
            uint64_t mk;
            if constexpr (SCORE)
                mk = score_key<T>(coef[e], fin[e]);
            else
                mk = mag_key<T>(coef[e]);
            if constexpr (FLAGS) {
                const bool f = nflag[e] != 0;
                if (sw.live(slots) && mk >= boundary) {
                    kept = true;
                    part = f;
                }
            } else {
                uint64_t k[2 * W];
                load_key<W>(keys, e, k);
                if (sw.live(slots) && mk >= boundary) {
                    kept = true;
                    part = emits_partner_regs<W, T>(L, A, k);
                }
            }
        }
        sw.step32(slots);
        bk[i] = __ballot_sync(0xffffffffu, kept);
        bp[i] = __ballot_sync(0xffffffffu, part);
        wk += __popc(bk[i]);
        wp += __popc(bp[i]);
    }
    if (lane == 0) {
        s_wk[warp] = wk;
        s_wp[warp] = wp;
    }
    __syncthreads();
    unsigned int xk = 0, xp = 0, tk = 0, tp = 0;
#pragma unroll
    for (int w = 0; w < kThreads / 32; ++w) {
        xk += w < warp ? s_wk[w] : 0u;
        xp += w < warp ? s_wp[w] : 0u;
        tk += s_wk[w];
        tp += s_wp[w];
    }
    if (tid < 32) {
        const unsigned long long agg = (unsigned long long)tk | ((unsigned long long)tp << 31);
        unsigned long long pre = 0;
        if (tile == 0) {
            if (tid == 0) st_release_u64(status + tile, kFlagInc | agg);
        } else {
            if (tid == 0) st_release_u64(status + tile, kFlagAgg | agg);
            pre = lookback_sum_warp(status, tile, ctl, 704);
            if (tid == 0) st_release_u64(status + tile, kFlagInc | (pre + agg));
        }
        if (tid == 0) {
            s_kept = pre & kLow31;
            s_part = pre >> 31;
            if ((uint64_t)(tile + 1) * TILE >= n) {
                ctl->count[3] = s_kept + tk;
                ctl->count[0] = s_part + tp;
            }
        }
    }
    __syncthreads();
    unsigned long long kr = s_kept + xk, pr = s_part + xp;
    uint64_t prev[2 * W];
#pragma unroll
    for (int w = 0; w < 2 * W; ++w) prev[w] = 0;
    bool have_prev = false;
#pragma unroll
    for (int i = 0; i < ITEMS; ++i) {
        const unsigned int b = bk[i], bq = bp[i];
        const uint64_t e = wbase + (uint64_t)i * 32 + lane;
        const unsigned long long pos = kr + __popc(b & lt);
        uint64_t k[2 * W];
#pragma unroll
        for (int w = 0; w < 2 * W; ++w) k[w] = 0;
        if ((b >> lane) & 1u) {
            load_key<W>(keys, e, k);
            if (PS_GUARD(ctl, pos < n, 702)) {
                store_key<W>(okeys, pos, k);
                ocoef[pos] = coef[e];
                if constexpr (SCORE) fout[pos] = fin[e];
            }
        }
        if (bq != 0) {  // warp-uniform: the rows that emit a partner, in order, with their ranks
            const unsigned int lower = bq & lt;
            const int src = lower ? 31 - __clz(lower) : lane;
            const int hi = 31 - __clz(bq);
            uint64_t pk[2 * W];
#pragma unroll
            for (int w = 0; w < 2 * W; ++w) pk[w] = __shfl_sync(0xffffffffu, k[w], src);
            if ((bq >> lane) & 1u) {
                const unsigned long long j = pr + __popc(lower);
                if (PS_BOUNDS(ctl, j < n, 705)) {
                    idx[j] = (uint32_t)pos;
                    uint16_t d;
                    if (lower)
                        d = (uint16_t)div_regs<W>(pk, k);
                    else if (have_prev)
                        d = (uint16_t)div_regs<W>(prev, k);
                    else
                        d = j == 0 ? kDivStart : kDivUnknown;
                    D[j] = d;
                }
            }
#pragma unroll
            for (int w = 0; w < 2 * W; ++w) prev[w] = __shfl_sync(0xffffffffu, k[w], hi);
            have_prev = true;
            pr += __popc(bq);
        }
        kr += __popc(b);
    }
}

// ---------------------------------------------------------------------------
// CollapseSample (crates/paulistrings/src/truncation/collapse_sample.rs): the terms' |c| laid
// end to end in key order, stretch boundaries accumulated per block of kCollapseBlock terms
// (the block's start plus a running sum from 0.0, as the reference accumulates per bucket),
// samples systematic points (u + k) * h; a term holding m points keeps sign(c) * m * h.
// ---------------------------------------------------------------------------
constexpr uint64_t kCollapseBlock = 1024;

// One thread per block: the block's sum of |c|, left to right from 0.0.
template <typename T>
__global__ void __launch_bounds__(kThreads) k_collapse_norms(const T* __restrict__ coef, uint64_t n,
                                                             double* __restrict__ norms) {
    const uint64_t b = blockIdx.x * (uint64_t)kThreads + threadIdx.x;
    const uint64_t lo = b * kCollapseBlock;
    if (lo >= n) return;
    const uint64_t hi = lo + kCollapseBlock < n ? lo + kCollapseBlock : n;
    double sum = 0.0;
    for (uint64_t i = lo; i < hi; ++i) sum = add_rn(sum, fabs(to_f64(coef[i])));
    norms[b] = sum;
}

// One thread per block: each term's multiplicity, walking the block's points from first[b]
// (systematic_resample, collapse_sample.rs:144-172).
template <typename T>
__global__ void __launch_bounds__(kThreads) k_collapse_mult(const T* __restrict__ coef, uint64_t n,
                                                            const double* __restrict__ starts,
                                                            const uint64_t* __restrict__ first, double u,
                                                            uint64_t samples, double total,
                                                            uint32_t* __restrict__ mult) {
    const uint64_t b = blockIdx.x * (uint64_t)kThreads + threadIdx.x;
    const uint64_t lo = b * kCollapseBlock;
    if (lo >= n) return;
    const uint64_t hi = lo + kCollapseBlock < n ? lo + kCollapseBlock : n;
    const double start = starts[b], step = total / (double)samples;
    uint64_t next = first[b];
    const uint64_t end = first[b + 1];
    double running = 0.0;
    for (uint64_t i = lo; i < hi; ++i) {
        if (next == end) {
            mult[i] = 0;
            continue;
        }
        running = add_rn(running, fabs(to_f64(coef[i])));
        const double boundary = add_rn(0.0, add_rn(start, running));
        uint64_t stop = end;
        if (boundary < total) {
            stop = next;
            while (stop < end && mul_rn(add_rn(u, (double)stop), step) < boundary) ++stop;
        }
        mult[i] = (uint32_t)(stop - next);
        next = stop;
    }
}

// Order-preserving compaction of the drawn terms, coefficient sign(c) * m * h (in f64, then T).
template <int W, typename T>
__global__ void __launch_bounds__(kThreads) k_collapse_compact(const uint64_t* __restrict__ keys,
                                                               const T* __restrict__ coef,
                                                               const uint32_t* __restrict__ mult, uint64_t n,
                                                               double step, uint64_t* __restrict__ okeys,
                                                               T* __restrict__ ocoef, unsigned long long* status,
                                                               Ctl* ctl) {
    constexpr int ITEMS = 16;
    constexpr int TILE = kThreads * ITEMS;
    __shared__ unsigned int s_tile;
    __shared__ unsigned int s_w[kThreads / 32];
    __shared__ unsigned long long s_off;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const unsigned int lt = (1u << lane) - 1u;
    if (tid == 0) s_tile = atomicAdd(&ctl->tile_counter[6], 1u);
    __syncthreads();
    const unsigned int tile = s_tile;
    const uint64_t wbase = (uint64_t)tile * TILE + (uint64_t)warp * 32 * ITEMS;
    unsigned int ball[ITEMS];
    unsigned int wc = 0;
#pragma unroll
    for (int i = 0; i < ITEMS; ++i) {
        const uint64_t e = wbase + (uint64_t)i * 32 + lane;
        ball[i] = __ballot_sync(0xffffffffu, e < n && mult[e] > 0);
        wc += __popc(ball[i]);
    }
    if (lane == 0) s_w[warp] = wc;
    __syncthreads();
    unsigned int wx = 0, tot = 0;
#pragma unroll
    for (int w = 0; w < kThreads / 32; ++w) {
        wx += w < warp ? s_w[w] : 0u;
        tot += s_w[w];
    }
    if (tid < 32) {
        unsigned long long p = 0;
        if (tile == 0) {
            if (tid == 0) st_release_u64(status + tile, kFlagInc | (unsigned long long)tot);
        } else {
            if (tid == 0) st_release_u64(status + tile, kFlagAgg | (unsigned long long)tot);
            p = lookback_sum_warp(status, tile, ctl, 721);
            if (tid == 0) st_release_u64(status + tile, kFlagInc | (p + tot));
        }
        if (tid == 0) {
            s_off = p;
            if ((uint64_t)(tile + 1) * TILE >= n) ctl->count[3] = p + tot;
        }
    }
    __syncthreads();
    unsigned long long o = s_off + wx;
#pragma unroll
    for (int i = 0; i < ITEMS; ++i) {
        if ((ball[i] >> lane) & 1u) {
            const uint64_t e = wbase + (uint64_t)i * 32 + lane;
            const unsigned long long pos = o + __popc(ball[i] & lt);
            const double c = to_f64(coef[e]);
            const double weight = mul_rn((double)mult[e], step);
            const double v = mul_rn(c / fabs(c), weight);  // drawn(), collapse_sample.rs:136-140
            uint64_t k[2 * W];
            load_key<W>(keys, e, k);
            if (PS_GUARD(ctl, pos < n, 722)) {
                store_key<W>(okeys, pos, k);
                ocoef[pos] = (T)v;
            }
        }
        o += __popc(ball[i]);
    }
}

// ---------------------------------------------------------------------------
// expectation in a product state
// ---------------------------------------------------------------------------
template <int W>
struct Basis {
    uint64_t ax[W], az[W], neg[W];
};

template <int W, typename T>
__global__ void __launch_bounds__(kThreads) k_expect_partial(const uint64_t* __restrict__ keys, const T* __restrict__ coef,
                                                             uint64_t n, const Basis<W> B, double* __restrict__ partial) {
    __shared__ double sh[kThreads];
    double acc = 0.0;
    for (uint64_t i = blockIdx.x * (uint64_t)kThreads + threadIdx.x; i < n; i += (uint64_t)gridDim.x * kThreads) {
        uint64_t k[2 * W];
        load_key<W>(keys, i, k);
        uint64_t mismatch = 0;
        uint32_t sign = 0;
#pragma unroll
        for (int w = 0; w < W; ++w) {
            uint64_t sup = k[w] | k[W + w];
            mismatch |= (k[w] ^ (sup & B.ax[w])) | (k[W + w] ^ (sup & B.az[w]));
            sign += __popcll(sup & B.neg[w]);
        }
        if (mismatch) continue;
        double c = to_f64(coef[i]);
        acc = __dadd_rn(acc, (sign & 1u) ? -c : c);
    }
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int s = kThreads / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) sh[threadIdx.x] = __dadd_rn(sh[threadIdx.x], sh[threadIdx.x + s]);
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.x] = sh[0];
}

__global__ void k_expect_final(const double* __restrict__ partial, int count, double* __restrict__ out) {
    __shared__ double sh[kThreads];
    double acc = 0.0;
    for (int i = threadIdx.x; i < count; i += kThreads) acc = __dadd_rn(acc, partial[i]);
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int s = kThreads / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) sh[threadIdx.x] = __dadd_rn(sh[threadIdx.x], sh[threadIdx.x + s]);
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = sh[0];
}

// ---------------------------------------------------------------------------
// host launchers
// ---------------------------------------------------------------------------
static inline unsigned int grid_for(uint64_t n, int sms) {
    uint64_t blocks = (n + kThreads - 1) / kThreads;
    uint64_t cap = (uint64_t)sms * 8;
    if (blocks > cap) blocks = cap;
    return (unsigned int)(blocks ? blocks : 1);
}

// Keys per block segment of the TopN candidate buffer: every element of the block's chunks.
static inline uint64_t topn_seg_cap(uint64_t n, int sms) {
    const uint64_t g = grid_for(n, sms), nchunks = (n + kThreads * 16 - 1) / (kThreads * 16);
    return (nchunks + g - 1) / g * (kThreads * 16);
}

// Words of the TopN candidate buffer: block segments holding every element of their chunks and
// the segment lengths, for any grid of at most 8 blocks per multiprocessor (the multi-launch
// select's grid_for and the cooperative select's resident grid).
uint64_t topn_cand_words(uint64_t n, int sms) {
    const uint64_t gmax = (uint64_t)(sms > 0 ? sms : 1) * 8, nchunks = (n + kThreads * 16 - 1) / (kThreads * 16);
    return (nchunks + gmax) * (kThreads * 16) + (gmax + 1) / 2;
}

template <int W, typename T>
cudaError_t StoreOps<W, T>::pack(const uint64_t* x, const uint64_t* z, const double* c, uint64_t n, uint32_t nq,
                                 uint64_t* keys, T* coef, uint32_t* vals, Ctl* ctl, int sms, cudaStream_t st,
                                 KernelProf* prof) {
    cudaMemsetAsync(&ctl->support[0], 0, sizeof(ctl->support), st);
    if (!n) return cudaSuccess;
    prof->begin(K_PACK, (double)n * (16 * W + 8 + 16 * W + sizeof(T) + 4), st);
    k_pack<W, T><<<grid_for(n, sms), kThreads, 0, st>>>(x, z, c, n, nq, keys, coef, vals, ctl);
    prof->end(st);
    return cudaGetLastError();
}

template <int W, typename T>
cudaError_t StoreOps<W, T>::check_sorted(const uint64_t* keys, const T* coef, uint64_t n, Ctl* ctl,
                                         unsigned long long* host_count, bool* sorted, int sms, cudaStream_t st,
                                         KernelProf* prof) {
    cudaMemsetAsync(&ctl->count[5], 0, sizeof(unsigned long long), st);
    prof->begin(K_PACK, (double)n * (16 * W + sizeof(T)), st);
    if (n) k_check_sorted<W, T><<<grid_for(n, sms), kThreads, 0, st>>>(keys, coef, n, ctl);
    prof->end(st);
    cudaMemcpyAsync(host_count, &ctl->count[5], sizeof(unsigned long long), cudaMemcpyDeviceToHost, st);
    cudaError_t e = spin_sync(st);
    *sorted = e == cudaSuccess && *host_count == 0;
    return e;
}

template <int W, typename T>
cudaError_t StoreOps<W, T>::unpack(const uint64_t* keys, const T* coef, uint64_t n, uint64_t* x, uint64_t* z,
                                   double* c, int sms, cudaStream_t st, KernelProf* prof) {
    if (!n) return cudaSuccess;
    prof->begin(K_UNPACK, (double)n * (16 * W + sizeof(T) + 16 * W + 8), st);
    k_unpack<W, T><<<grid_for(n, sms), kThreads, 0, st>>>(keys, coef, n, x, z, c);
    prof->end(st);
    return cudaGetLastError();
}

template <int W, typename T>
cudaError_t StoreOps<W, T>::sort_pairs(uint64_t* keys, uint32_t* vals, uint64_t* keys_alt, uint32_t* vals_alt,
                                       uint64_t n, SortScratch& s, Ctl* ctl, int sms, cudaStream_t st,
                                       bool& result_in_alt, KernelProf* prof) {
    result_in_alt = false;
    if (n <= 1) return cudaSuccess;
    constexpr int ND = 16 * W;
    cudaError_t e;
    cudaMemsetAsync(s.hist, 0, (size_t)ND * 256 * sizeof(unsigned int), st);
    prof->begin(K_SORT_HIST, (double)n * 16 * W, st);
    k_sort_hist<W><<<grid_for(n, sms), kThreads, (size_t)ND * 256 * sizeof(unsigned int), st>>>(keys, n, s.hist);
    prof->end(st);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    cudaMemcpyAsync(s.host_hist, s.hist, (size_t)ND * 256 * sizeof(unsigned int), cudaMemcpyDeviceToHost, st);
    if ((e = spin_sync(st)) != cudaSuccess) return e;
    constexpr int TILE = SortTile<W>::TILE;
    const uint32_t tiles = (uint32_t)((n + TILE - 1) / TILE);
    uint64_t *ka = keys, *kb = keys_alt;
    uint32_t *va = vals, *vb = vals_alt;
    for (int d = 0; d < ND; ++d) {
        const unsigned int* h = s.host_hist + d * 256;
        bool trivial = false;
        for (int b = 0; b < 256; ++b)
            if (h[b] == n) trivial = true;
        if (trivial) continue;
        unsigned int* base = s.host_base + d * 256;
        unsigned int run = 0;
        for (int b = 0; b < 256; ++b) {
            base[b] = run;
            run += h[b];
        }
        cudaMemcpyAsync(s.base + d * 256, base, 256 * sizeof(unsigned int), cudaMemcpyHostToDevice, st);
        cudaMemsetAsync(s.status, 0, (size_t)tiles * 256 * sizeof(unsigned int), st);
        cudaMemsetAsync(&ctl->tile_counter[4], 0, sizeof(unsigned int), st);
        prof->begin(K_SORT_PASS, (double)n * 2 * (16 * W + 4), st);
        k_sort_pass<W><<<tiles, kThreads, 0, st>>>(ka, va, kb, vb, n, d, s.base + d * 256, s.status, ctl);
        prof->end(st);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        uint64_t* tk = ka;
        ka = kb;
        kb = tk;
        uint32_t* tv = va;
        va = vb;
        vb = tv;
        result_in_alt = !result_in_alt;
    }
    // the host copies of the bases must outlive the async copies
    return spin_sync(st);
}

template <int W, typename T>
cudaError_t StoreOps<W, T>::dedup(const uint64_t* keys, const uint32_t* vals, const T* cin, uint64_t n,
                                  const KeepProg& keep, bool compensated, uint64_t* okeys, T* ocoef,
                                  unsigned long long* status, Ctl* ctl, unsigned long long* host_count,
                                  uint64_t* out_n, cudaStream_t st, KernelProf* prof) {
    if (!n) {
        *out_n = 0;
        return cudaSuccess;
    }
    const uint32_t tiles = (uint32_t)((n + kThreads * 8 - 1) / (kThreads * 8));
    cudaMemsetAsync(status, 0, (size_t)tiles * sizeof(unsigned long long), st);
    cudaMemsetAsync(&ctl->tile_counter[5], 0, sizeof(unsigned int), st);
    prof->begin(K_DEDUP, (double)n * (16 * W + 4 + sizeof(T)), st);
    k_dedup<W, T><<<tiles, kThreads, 0, st>>>(keys, vals, cin, n, keep, compensated ? 1 : 0, okeys, ocoef, status, ctl);
    prof->end(st);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    cudaMemcpyAsync(host_count, &ctl->count[2], sizeof(unsigned long long), cudaMemcpyDeviceToHost, st);
    if ((e = spin_sync(st)) != cudaSuccess) return e;
    *out_n = *host_count;
    prof->add_bytes(K_DEDUP, (double)*out_n * (16 * W + sizeof(T)));
    return cudaSuccess;
}

// Resident blocks per SM of the cooperative select (its plain or scored variant), looked up on
// first use; -1 when the device cannot run it.
template <typename T>
int select_blocks_per_sm(bool score) {
    static std::atomic<int> per_sm[2] = {{0}, {0}};
    std::atomic<int>& per_v = per_sm[score ? 1 : 0];
    int per = per_v.load(std::memory_order_relaxed);
    if (per == 0) {
        const void* kern = score ? (const void*)k_topn_select_all<T, true> : (const void*)k_topn_select_all<T, false>;
        int dev = 0, coop = 0;
        if (cudaGetDevice(&dev) != cudaSuccess ||
            cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev) != cudaSuccess || !coop ||
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, kSelThreads, 0) != cudaSuccess || per < 1)
            per = -1;
        cudaGetLastError();
        per_v.store(per, std::memory_order_relaxed);
    }
    return per;
}

template <int W, typename T>
bool StoreOps<W, T>::cooperative_select() {
    return select_blocks_per_sm<T>(false) > 0;
}

template <int W, typename T>
cudaError_t StoreOps<W, T>::topn(const uint64_t* keys, const T* coef, uint64_t n, uint64_t keep_n, uint64_t* okeys,
                                 T* ocoef, unsigned int* hist, bool hist_ready, uint64_t* cand, uint64_t cand_cap,
                                 unsigned long long* status, Ctl* ctl, unsigned long long* host_count,
                                 uint64_t* out_n, int sms, cudaStream_t st, KernelProf* prof, const uint64_t* sel,
                                 bool window, uint64_t base, SlotMap slots, const float* fpred, float* fout,
                                 const RotLayer<W>* next, uint32_t* next_idx, uint16_t* next_D,
                                 const uint8_t* next_flags, bool deferred) {
    const int dfr = deferred ? 1 : 0;
    // aux: prefix, mask, remaining rank, above, keys in the last chosen bin (after the select:
    // the keys equal to the boundary), window miss, keys gathered for the in-block select
    // (cooperative select), next layer not classified by the compaction; count[4]: candidates
    window = window && hist_ready && !sel;
    if (!window) base = 0;
    const unsigned int cgrid = grid_for(n, sms);
    const uint64_t seg_cap = topn_seg_cap(n, sms);
    const uint64_t key_cap = seg_cap * cgrid;  // segments, then the segment lengths
    if (key_cap + (cgrid + 1) / 2 > cand_cap) return cudaErrorInvalidValue;  // sized by topn_cand_words
    unsigned int* seg_count = reinterpret_cast<unsigned int*>(cand + key_cap);
    cudaError_t e;
    if (deferred && (!hist_ready || !slots.count)) return cudaErrorInvalidValue;  // needs the merge's histogram and slots
    if (!hist_ready) {
        cudaMemsetAsync(hist, 0, kTopnBins1 * sizeof(unsigned int), st);
        prof->begin(K_TOPN_HIST, (double)n * sizeof(T), st);
        k_topn_hist1<<<grid_for(n, sms), kThreads, 0, st>>>(std::is_same<T, double>::value ? (const double*)coef : nullptr,
                                                            std::is_same<T, float>::value ? (const float*)coef : nullptr,
                                                            n, hist, slots, sel ? nullptr : fpred);
        prof->end(st);
    }
    // the whole select in one cooperative launch when the device runs it (the multi-launch path
    // below otherwise)
    bool selected = false;
    {
        const float* fp = sel ? nullptr : fpred;
        const void* kern = fp ? (const void*)k_topn_select_all<T, true> : (const void*)k_topn_select_all<T, false>;
        const int per = select_blocks_per_sm<T>(fp != nullptr);
        if (per > 0) {
            const uint64_t nchunks = (n + kSelThreads * 16 - 1) / (kSelThreads * 16);
            const unsigned int G =
                (unsigned int)std::max<uint64_t>(1, std::min<uint64_t>(std::min<uint64_t>(grid_for(n, sms), nchunks),
                                                                       (uint64_t)per * (sms > 0 ? sms : 1)));
            const uint64_t gseg = (nchunks + G - 1) / G * (kSelThreads * 16);
            const uint64_t gkey = gseg * G;
            if (gkey + (G + 1) / 2 <= cand_cap) {
                unsigned int* gcount = reinterpret_cast<unsigned int*>(cand + gkey);
                unsigned int* bar = &ctl->tile_counter[4];
                cudaMemsetAsync(bar, 0, 2 * sizeof(unsigned int), st);
                const int win = window ? 1 : 0;
                unsigned long long kn = keep_n;
                const uint32_t ctiles = (uint32_t)((n + kThreads * 16 - 1) / (kThreads * 16));
                void* args[] = {(void*)&coef, (void*)&sel,  (void*)&win,   (void*)&base, (void*)&n,
                                (void*)&ctl,  (void*)&hist, (void*)&cand,  (void*)&gkey, (void*)&gseg,
                                (void*)&gcount, (void*)&slots, (void*)&bar, (void*)&fp, (void*)&kn,
                                (void*)&status, (void*)&ctiles, (void*)&dfr};
                prof->begin(K_TOPN_HIST, deferred ? 0.0 : (double)n * sizeof(T), st);
                e = cudaLaunchCooperativeKernel(kern, dim3(G), dim3(kSelThreads), args, 0, st);
                prof->end(st);
                selected = e == cudaSuccess;
                if (!selected) cudaGetLastError();  // not launched: the multi-launch path selects instead
                if (!selected && deferred) return cudaErrorNotSupported;  // the host does not know the span
            }
        }
    }
    if (!selected) {
        unsigned long long* init = host_count + 8;
        init[0] = 0ull;
        init[1] = 0ull;
        init[2] = (unsigned long long)keep_n;
        init[3] = 0ull;
        init[4] = 0ull;
        init[5] = 0ull;
        init[6] = 0ull;
        init[7] = 0ull;
        cudaMemcpyAsync(ctl->aux, init, 8 * sizeof(unsigned long long), cudaMemcpyHostToDevice, st);
        // digit 1: the select key's top 12 bits (key >> 52), or in a window the bin of 2^48 units;
        // then 13-bit digits down to bit 0 (a window's last digit overlaps bits already fixed)
        prof->begin(K_TOPN_STEP, kTopnBins1 * 8.0, st);
        k_topn_select<kTopnBins1><<<1, 1024, 0, st>>>(hist, window ? 48 : 52, window ? 11 : 12, ctl);
        prof->end(st);
        prof->begin(K_TOPN_HIST, (double)n * sizeof(T), st);
        if (!sel && fpred)
            k_topn_cand<T, true><<<cgrid, kThreads, 0, st>>>(coef, sel, window ? 1 : 0, base, n, ctl, cand, key_cap,
                                                             seg_cap, seg_count, slots, fpred);
        else
            k_topn_cand<T, false><<<cgrid, kThreads, 0, st>>>(coef, sel, window ? 1 : 0, base, n, ctl, cand, key_cap,
                                                              seg_cap, seg_count, slots, nullptr);
        prof->end(st);
        static const int kShifts[2][4] = {{39, 26, 13, 0}, {35, 22, 9, 0}};
        for (int d = 0; d < 4; ++d) {
            const int shift = kShifts[window ? 1 : 0][d];
            prof->begin(K_TOPN_HIST, 0.0, st);
            k_topn_hist_cand<<<2 * sms, kThreads, 0, st>>>(cand, ctl, shift, hist, seg_cap, seg_count, cgrid);
            prof->end(st);
            prof->begin(K_TOPN_STEP, kTopnBinsN * 8.0, st);
            k_topn_select<kTopnBinsN><<<1, 1024, 0, st>>>(hist, shift, 13, ctl);
            prof->end(st);
        }
    }
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    const uint32_t tiles = (uint32_t)((n + kThreads * 16 - 1) / (kThreads * 16));
    if (!selected) {  // the cooperative select reset these itself
        cudaMemsetAsync(status, 0, (size_t)tiles * sizeof(unsigned long long), st);
        cudaMemsetAsync(&ctl->tile_counter[6], 0, sizeof(unsigned int), st);
    }
    prof->begin(K_TOPN_COMPACT, deferred ? 0.0 : (double)n * sizeof(T), st);
    const bool classify = next && next_idx && next_D && !sel && (fpred != nullptr) == (fout != nullptr);
    if (classify && fpred)
        k_topn_compact_cls<W, T, false, true><<<tiles, kThreads, 0, st>>>(keys, coef, base, n,
                                                                          (unsigned long long)keep_n, okeys, ocoef,
                                                                          status, ctl, slots, *next, next_idx, next_D,
                                                                          nullptr, dfr, fpred, fout);
    else if (classify && next_flags)
        k_topn_compact_cls<W, T, true><<<tiles, kThreads, 0, st>>>(keys, coef, base, n, (unsigned long long)keep_n,
                                                                   okeys, ocoef, status, ctl, slots, *next, next_idx,
                                                                   next_D, next_flags, dfr);
    else if (classify)
        k_topn_compact_cls<W, T, false><<<tiles, kThreads, 0, st>>>(keys, coef, base, n, (unsigned long long)keep_n,
                                                                    okeys, ocoef, status, ctl, slots, *next, next_idx,
                                                                    next_D, nullptr, dfr);
    else if (fout)
        k_topn_compact<W, T, true><<<tiles, kThreads, 0, st>>>(keys, coef, sel, sel ? 1 : (fpred ? 4 : 0), base, n,
                                                               (unsigned long long)keep_n, okeys, ocoef, status, ctl,
                                                               slots, fpred, fout, dfr);
    else
        k_topn_compact<W, T, false><<<tiles, kThreads, 0, st>>>(keys, coef, sel, sel ? 1 : 0, base, n,
                                                                (unsigned long long)keep_n, okeys, ocoef, status, ctl,
                                                                slots, nullptr, nullptr, dfr);
    prof->end(st);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    // the one host synchronization of the pass: counts, error flags and the select's aux words
    // (and, deferred, the span the select read and whether it kept every live row)
    cudaMemcpyAsync(host_count, &ctl->count[0], offsetof(Ctl, spin_limit), cudaMemcpyDeviceToHost, st);
    if (deferred) cudaMemcpyAsync(host_count + 22, &ctl->span, 2 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st);
    if ((e = spin_sync(st)) != cudaSuccess) return e;
    *out_n = host_count[3];
    if (deferred) {  // the rows the select and the compaction read: the span, known now
        prof->add_bytes(K_TOPN_HIST, (double)host_count[22] * sizeof(T));
        prof->add_bytes(K_TOPN_COMPACT, (double)host_count[22] * sizeof(T));
    }
    if (classify && next_flags) prof->add_bytes(K_TOPN_COMPACT, (double)(deferred ? host_count[22] : n));
    prof->add_bytes(K_TOPN_COMPACT, (double)*out_n * (2 * 16 * W + sizeof(T)));
    if (classify && !topn_unclassified(host_count)) prof->add_bytes(K_TOPN_COMPACT, (double)host_count[0] * 6.0);
    return cudaSuccess;
}

template <int W, typename T>
cudaError_t StoreOps<W, T>::densify(const uint64_t* keys, const T* coef, uint64_t n, SlotMap slots, uint64_t* okeys,
                                    T* ocoef, unsigned long long* status, Ctl* ctl, unsigned long long* host_count,
                                    uint64_t* out_n, cudaStream_t st, KernelProf* prof, const float* fin, float* fout) {
    if (n == 0) {
        *out_n = 0;
        return cudaSuccess;
    }
    unsigned long long* init = host_count + 8;
    for (int q = 0; q < 4; ++q) init[q] = 0ull;  // no boundary, no quota
    cudaMemcpyAsync(ctl->aux, init, 4 * sizeof(unsigned long long), cudaMemcpyHostToDevice, st);
    const uint32_t tiles = (uint32_t)((n + kThreads * 16 - 1) / (kThreads * 16));
    cudaMemsetAsync(status, 0, (size_t)tiles * sizeof(unsigned long long), st);
    cudaMemsetAsync(&ctl->tile_counter[6], 0, sizeof(unsigned int), st);
    prof->begin(K_TOPN_COMPACT, 0.0, st);
    if (fout)
        k_topn_compact<W, T, true><<<tiles, kThreads, 0, st>>>(keys, coef, nullptr, 3, 0ull, n, 0ull, okeys, ocoef,
                                                               status, ctl, slots, fin, fout, 0);
    else
        k_topn_compact<W, T, false><<<tiles, kThreads, 0, st>>>(keys, coef, nullptr, 3, 0ull, n, 0ull, okeys, ocoef,
                                                                status, ctl, slots, nullptr, nullptr, 0);
    prof->end(st);
    cudaError_t e;
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    cudaMemcpyAsync(host_count, &ctl->count[0], offsetof(Ctl, err_info) + sizeof(unsigned int),
                    cudaMemcpyDeviceToHost, st);
    if ((e = spin_sync(st)) != cudaSuccess) return e;
    *out_n = host_count[3];
    prof->add_bytes(K_TOPN_COMPACT, (double)*out_n * (2 * 16 * W + 2 * sizeof(T)));
    return cudaSuccess;
}

template <int W, typename T>
cudaError_t StoreOps<W, T>::approx_topn(const uint64_t* keys, const T* coef, uint64_t n, uint64_t keep_n,
                                        uint64_t* okeys, T* ocoef, unsigned int* hist, bool hist_ready,
                                        unsigned int* host_hist, unsigned long long* status, Ctl* ctl,
                                        unsigned long long* host_count, uint64_t* out_n, int sms, cudaStream_t st,
                                        KernelProf* prof) {
    // octave_edge (crates/paulistrings/src/truncation/builtin.rs:312-353): walk the octaves from
    // the top; the first whose population overflows keep_n is the boundary, cut by a quota
    cudaError_t e;
    if (!hist_ready) {
        prof->begin(K_TOPN_HIST, (double)n * sizeof(T), st);
        k_octave_hist<T><<<grid_for(n, sms), kThreads, 0, st>>>(coef, n, hist);
        prof->end(st);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    cudaMemcpyAsync(host_hist, hist, kTopnBins1 * sizeof(unsigned int), cudaMemcpyDeviceToHost, st);
    cudaMemsetAsync(hist, 0, kTopnBins1 * sizeof(unsigned int), st);
    if ((e = spin_sync(st)) != cudaSuccess) return e;
    unsigned long long above = 0, bin = 0;
    bool found = false;
    for (int b = kTopnBins1 - 1; b >= 0; --b) {
        if (above + host_hist[b] > keep_n) {
            bin = (unsigned long long)b;
            found = true;
            break;
        }
        above += host_hist[b];
    }
    if (!found) {  // cannot happen for n > keep_n; keep everything rather than guess
        *out_n = n;
        return cudaErrorInvalidValue;
    }
    unsigned long long* init = host_count + 8;
    init[0] = bin + 1;  // octave keys are octave + 1
    init[1] = 0;
    init[2] = 0;
    init[3] = above;
    cudaMemcpyAsync(ctl->aux, init, 4 * sizeof(unsigned long long), cudaMemcpyHostToDevice, st);
    const uint32_t tiles = (uint32_t)((n + kThreads * 16 - 1) / (kThreads * 16));
    cudaMemsetAsync(status, 0, (size_t)tiles * sizeof(unsigned long long), st);
    cudaMemsetAsync(&ctl->tile_counter[6], 0, sizeof(unsigned int), st);
    prof->begin(K_TOPN_COMPACT, (double)n * sizeof(T), st);
    k_topn_compact<W, T, false><<<tiles, kThreads, 0, st>>>(keys, coef, nullptr, 2, 0ull, n, (unsigned long long)keep_n,
                                                     okeys, ocoef, status, ctl, SlotMap{nullptr, 0u}, nullptr, nullptr, 0);
    prof->end(st);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    cudaMemcpyAsync(host_count, &ctl->count[0], offsetof(Ctl, err_info) + sizeof(unsigned int),
                    cudaMemcpyDeviceToHost, st);
    if ((e = spin_sync(st)) != cudaSuccess) return e;
    *out_n = host_count[3];
    prof->add_bytes(K_TOPN_COMPACT, (double)*out_n * (2 * 16 * W + sizeof(T)));
    return cudaSuccess;
}

// The key-addressed stream of rng.rs: splitmix64 absorbs the key words, seeds xoshiro256++,
// and uniform() is the first output's top 53 bits (crates/paulistrings/src/rng.rs:1-62).
static uint64_t mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
static uint64_t splitmix64(uint64_t& state) {
    state += 0x9E3779B97F4A7C15ull;
    return mix64(state);
}
static double keyed_uniform(uint64_t k0, uint64_t k1) {
    const uint64_t key[2] = {k0, k1};
    uint64_t absorbed = 2;
    for (uint64_t w : key) {
        uint64_t t = absorbed ^ w;
        absorbed = splitmix64(t);
    }
    uint64_t st[4];
    for (auto& w : st) w = splitmix64(absorbed);
    if (!(st[0] | st[1] | st[2] | st[3])) st[0] = 1;
    auto rotl = [](uint64_t x, int r) { return (x << r) | (x >> (64 - r)); };
    const uint64_t out = rotl(st[0] + st[3], 23) + st[0];
    return (double)(out >> 11) * (1.0 / 9007199254740992.0);
}

template <int W, typename T>
cudaError_t StoreOps<W, T>::collapse_sample(const uint64_t* keys, const T* coef, uint64_t n, uint64_t samples,
                                            uint64_t seed, uint64_t call, uint64_t* okeys, T* ocoef,
                                            double* norms, double* host_norms, uint64_t* first,
                                            uint64_t* host_first, uint32_t* mult, unsigned long long* status,
                                            Ctl* ctl, unsigned long long* host_count, uint64_t* out_n,
                                            bool* drawable, cudaStream_t st, KernelProf* prof) {
    const uint64_t nb = (n + kCollapseBlock - 1) / kCollapseBlock;
    const unsigned int grid = (unsigned int)((nb + kThreads - 1) / kThreads);
    cudaError_t e;
    prof->begin(K_TOPN_HIST, (double)n * sizeof(T), st);
    k_collapse_norms<T><<<grid, kThreads, 0, st>>>(coef, n, norms);
    prof->end(st);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    cudaMemcpyAsync(host_norms, norms, nb * sizeof(double), cudaMemcpyDeviceToHost, st);
    if ((e = spin_sync(st)) != cudaSuccess) return e;
    // the blocks' starts, left to right from 0.0, and sum |c| (systematic_resample's `starts`)
    double* starts = host_norms + nb + 1;
    double prefix = 0.0;
    for (uint64_t b = 0; b < nb; ++b) {
        starts[b] = prefix;
        prefix += host_norms[b];
    }
    starts[nb] = prefix;
    const double total = prefix;
    *drawable = total > 0.0 && total <= 1.7976931348623157e308;  // assert_drawable: positive and finite
    if (!*drawable) return cudaSuccess;
    const double u = keyed_uniform(seed, call), step = total / (double)samples;
    auto below = [&](double boundary) {  // SystematicPoints::below
        if (boundary >= total) return samples;
        uint64_t lo = 0, hi = samples;
        while (lo < hi) {
            const uint64_t mid = lo + (hi - lo) / 2;
            if ((u + (double)mid) * step < boundary)
                lo = mid + 1;
            else
                hi = mid;
        }
        return lo;
    };
    for (uint64_t b = 0; b <= nb; ++b) host_first[b] = below(starts[b]);
    double* dstarts = norms + nb + 1;
    cudaMemcpyAsync(dstarts, starts, (nb + 1) * sizeof(double), cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(first, host_first, (nb + 1) * sizeof(uint64_t), cudaMemcpyHostToDevice, st);
    prof->begin(K_TOPN_STEP, (double)n * (sizeof(T) + 4), st);
    k_collapse_mult<T><<<grid, kThreads, 0, st>>>(coef, n, dstarts, first, u, samples, total, mult);
    prof->end(st);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    const uint32_t tiles = (uint32_t)((n + kThreads * 16 - 1) / (kThreads * 16));
    cudaMemsetAsync(status, 0, (size_t)tiles * sizeof(unsigned long long), st);
    cudaMemsetAsync(&ctl->tile_counter[6], 0, sizeof(unsigned int), st);
    prof->begin(K_TOPN_COMPACT, (double)n * (4 + sizeof(T)), st);
    k_collapse_compact<W, T><<<tiles, kThreads, 0, st>>>(keys, coef, mult, n, step, okeys, ocoef, status, ctl);
    prof->end(st);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    cudaMemcpyAsync(host_count, &ctl->count[0], offsetof(Ctl, err_info) + sizeof(unsigned int),
                    cudaMemcpyDeviceToHost, st);
    if ((e = spin_sync(st)) != cudaSuccess) return e;
    *out_n = host_count[3];
    return cudaSuccess;
}

template <int W, typename T>
cudaError_t StoreOps<W, T>::expectation(const uint64_t* keys, const T* coef, uint64_t n, const uint64_t* ax,
                                        const uint64_t* az, const uint64_t* neg, double* partial, double* out_dev,
                                        int sms, cudaStream_t st, KernelProf* prof) {
    Basis<W> B;
    for (int w = 0; w < W; ++w) {
        B.ax[w] = ax[w];
        B.az[w] = az[w];
        B.neg[w] = neg[w];
    }
    const int blocks = kExpectBlocks;
    prof->begin(K_EXPECT, (double)n * (16 * W + sizeof(T)), st);
    k_expect_partial<W, T><<<blocks, kThreads, 0, st>>>(keys, coef, n, B, partial);
    k_expect_final<<<1, kThreads, 0, st>>>(partial, blocks, out_dev);
    prof->end(st);
    ++prof->launches[K_EXPECT];
    (void)sms;
    return cudaGetLastError();
}

template <int W, typename T>
cudaError_t StoreOps<W, T>::configure() {
    return cudaFuncSetAttribute(k_sort_hist<W>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)(16 * W * 256 * sizeof(unsigned int)));
}

template <int W, typename T>
size_t StoreOps<W, T>::sort_tile() {
    return SortTile<W>::TILE;
}

template struct StoreOps<1, double>;
template struct StoreOps<1, float>;
template struct StoreOps<2, double>;
template struct StoreOps<2, float>;
template struct StoreOps<4, double>;
template struct StoreOps<4, float>;

}  // namespace psb
