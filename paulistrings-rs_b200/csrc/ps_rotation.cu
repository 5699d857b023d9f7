// ps_rotation.cu -- the rotation layer on a sorted device store.
//
// A rotation-shaped table (an identity entry and one generator entry g,
// crates/paulistrings/src/engine/bucketed/rotation_layer.rs:75-140) maps each
// term k to (k, c*a0[s]) and, when the generator entry reaches its support
// pattern s, to (k ^ g, c*a1[s]).  Partners of a sorted run, taken in the run's
// order, are sorted under an order that differs from key order only where two
// keys first differ on a bit of g (crates/paulistrings/src/engine/bucketed/
// partner_order.rs:10-14).  So the layer is:
//
//   k_layer_prep reset the layer's counts, tile dispensers and look-back words;
//   k_classify   stream the store keys (warp-striped coalesced loads), list
//                anticommuting rows with a decoupled look-back count and record
//                each one's divergence rank from its predecessor (skipped when the
//                TopN compaction before the layer already wrote that list);
//   level scans  (k_level_reduce per tile, k_level_scan over the tiles,
//                k_level_apply per partner): forward max-scan per bit of g (the
//                upper half of each group moves down by the lower half's size) and
//                backward min-scan (the lower half moves up by the upper half's
//                size); the last batch writes each partner at its sorted slot;
//   k_partition  merge-path split points (a warp per run of tiles, 32-way search);
//   k_merge      merge own rows and partners (TMA bulk copies into shared
//                memory), sum equal keys, drop exact zeros and keep-program
//                rejects, and write the tile at its look-back offset or, before
//                a TopN pass, at its fixed slot (with the first select digit, and
//                before a rotation layer each row's partner test under it).
//
// Key-preserving tables (depolarizing noise, quarter turns with sin = 0) run
// k_partition + k_merge with an empty partner stream.
#include <algorithm>
#include <atomic>
#include <type_traits>
#include <cstddef>

#include "ps_device.cuh"
#include "ps_kernels.h"
#include "ps_rotlayer.cuh"

namespace psb {

constexpr int kBlock = 256;
constexpr int kTopnHistBins = 2048;  // key >> 52 of |c|^2 (first TopN select digit)

template <int W>
struct RotTile {
    static constexpr int kClassifyItems = W == 1 ? 16 : (W == 2 ? 8 : (W == 4 ? 4 : 2));
    static constexpr int kClassifyTile = kBlock * kClassifyItems;
    // odd, so the threads' merge-path starts fall on different shared-memory bank groups
    static constexpr int kMergeItems = W == 1 ? 5 : (W == 2 ? 5 : (W == 4 ? 3 : 1));
    static constexpr int kMergeTile = kBlock * kMergeItems;
};
constexpr int kScanItems = 16;
constexpr int kLevelInf = 0x7fffffff;  // identity of the backward level scan
constexpr int kScanTile = kBlock * kScanItems;
constexpr int kApplyThreads = 512;  // k_level_apply block: 8 partners per thread
static_assert(kScanTile == (int)kScanTileRows, "scan tile");

// Does term k emit a partner?
template <int W, typename T>
__device__ __forceinline__ bool emits_partner(const RotLayer<W>& L, const AmpTab<T>& A, const uint64_t* k) {
    if (L.wide) return anticommutes<W>(k, L.gx, L.gz);
    return A.a1[pattern_of<W>(L, k)] != T(0);
}

// Own-row coefficient after the layer.
template <int W, typename T>
__device__ __forceinline__ T own_coeff(const RotLayer<W>& L, const AmpTab<T>& A, const uint64_t* k, T c) {
    if (L.wide) return anticommutes<W>(k, L.gx, L.gz) ? mul_rn(c, Amp<T>::cs(L)) : c;
    return mul_rn(c, A.a0[pattern_of<W>(L, k)]);
}

// Partner coefficient (DeltaEntry::emit / PreparedRotation::emit_generator).
template <int W, typename T>
__device__ __forceinline__ T partner_coeff(const RotLayer<W>& L, const AmpTab<T>& A, const uint64_t* k, T c) {
    if (L.wide) {
        uint32_t total = (1u + product_phase<W>(k, L.gx, L.gz)) & 3u;
        T m = (total & 2u) ? -c : c;  // real mul_phase, coefficient.rs:107-114
        return mul_rn(m, Amp<T>::sn(L));
    }
    return mul_rn(c, A.a1[pattern_of<W>(L, k)]);
}

// The folded noise channels, staged in shared memory (their factors are indexed by each lane's
// pattern).
template <typename T>
struct NoiseSmem {
    T f[kMaxNoise][4];
    uint16_t q[kMaxNoise];
    int n;
};

// The kernels that fold no noise take an empty argument in its place.
struct NoNoise {};
template <bool NOISE>
using NoiseArg = typename std::conditional<NOISE, NoiseList, NoNoise>::type;

// Before a TopN pass whose compaction lists the next rotation layer's partners: the merge
// writes, per output row (slot layout), whether the row emits a partner under that layer, so the
// compaction decides from one byte instead of reading the key twice.
template <int W>
struct NextFlagArg {
    RotLayer<W> L;
    uint8_t* flags;
};
struct NoNextFlag {};
template <int W, bool ON>
using NextArg = typename std::conditional<ON, NextFlagArg<W>, NoNextFlag>::type;

// Shared storage for the staged channels only in the kernels that fold noise.
template <typename T, bool ON>
struct NoiseShared {
    NoiseSmem<T> s;
    unsigned int drop[kMaxNoise + 1];
    __device__ NoiseSmem<T>* tab() { return &s; }
    __device__ unsigned int* drops() { return drop; }
};
template <typename T>
struct NoiseShared<T, false> {
    __device__ NoiseSmem<T>* tab() { return nullptr; }
    __device__ unsigned int* drops() { return nullptr; }
};

template <typename T>
__device__ __forceinline__ void stage_noise(const NoiseList& N, NoiseSmem<T>& S) {
    for (int i = threadIdx.x; i < N.n * 4; i += blockDim.x) {
        if constexpr (std::is_same<T, double>::value)
            S.f[i >> 2][i & 3] = N.f[i >> 2][i & 3];
        else
            S.f[i >> 2][i & 3] = N.ff[i >> 2][i & 3];
    }
    for (int i = threadIdx.x; i < N.n; i += blockDim.x) S.q[i] = N.q[i];
    if (threadIdx.x == 0) S.n = N.n;
}

// The folded channels applied to coefficient v of key k in order, as the separate layers would:
// a channel multiplies by its factor for k's pattern on its qubit (the identity's factor is 1,
// skipped), then the term must stay nonzero and pass the keep program.  Returns the index of the
// channel after which the term is dropped, or S.n when it survives all of them.
template <int W, typename T>
__device__ __forceinline__ int noise_apply(const NoiseSmem<T>& S, const KeepProg& keep, const uint64_t* k, T& v) {
    if (!(v != T(0) && keep_eval<W>(keep, k, to_f64(v)))) return 0;
    for (int j = 0; j < S.n; ++j) {
        const int q = S.q[j];
        const uint32_t s = (uint32_t)((pick<W>(k, q >> 6) >> (q & 63)) & 1u) |
                           (uint32_t)((pick<W>(k, W + (q >> 6)) >> (q & 63)) & 1u) << 1;
        if (s) {
            v = mul_rn(v, S.f[j][s]);
            if (!(v != T(0) && keep_eval<W>(keep, k, to_f64(v)))) return j;
        }
    }
    return S.n;
}

// ---------------------------------------------------------------------------
// k_classify: warp-striped (lane l of warp w reads row base_w + 32 i + l, coalesced 16W-byte
// loads), anticommuting rows compacted by ballot in row order; each listed row records its
// divergence rank from the previous listed row (shuffled from the lane that holds it).  The
// first listed row of each warp takes kDivUnknown and the forward k_level_reduce resolves it.
// ---------------------------------------------------------------------------
template <int W, typename T>
__global__ void __launch_bounds__(kBlock) k_classify(const uint64_t* __restrict__ keys, uint64_t n,
                                                     const RotLayer<W> L, uint32_t* __restrict__ idx,
                                                     uint16_t* __restrict__ D, unsigned long long* status,
                                                     Ctl* ctl) {
    constexpr int ITEMS = RotTile<W>::kClassifyItems;
    constexpr int TILE = RotTile<W>::kClassifyTile;
    __shared__ unsigned int s_tile;
    __shared__ unsigned int s_wcount[kBlock / 32];
    __shared__ unsigned long long s_prefix;
    __shared__ AmpTab<T> A;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const unsigned int lanemask_lt = (1u << lane) - 1u;
    if (tid == 0) s_tile = atomicAdd(&ctl->tile_counter[0], 1u);
    stage_amps<W, T>(L, A);
    __syncthreads();
    const unsigned int tile = s_tile;
    const uint64_t wbase = (uint64_t)tile * TILE + (uint64_t)warp * 32 * ITEMS;
    unsigned int ball[ITEMS];
    unsigned int wcount = 0;
#pragma unroll
    for (int i = 0; i < ITEMS; ++i) {
        const uint64_t row = wbase + (uint64_t)i * 32 + lane;
        bool e = false;
        if (row < n) {
            uint64_t kk[2 * W];
            load_key<W>(keys, row, kk);
            e = emits_partner_regs<W, T>(L, A, kk);
        }
        ball[i] = __ballot_sync(0xffffffffu, e);
        wcount += __popc(ball[i]);
    }
    if (lane == 0) s_wcount[warp] = wcount;
    __syncthreads();
    unsigned int wexcl = 0, total = 0;
#pragma unroll
    for (int w = 0; w < kBlock / 32; ++w) {
        unsigned int c = s_wcount[w];
        wexcl += w < warp ? c : 0u;
        total += c;
    }
    if (tid < 32) {
        unsigned long long p = 0;
        if (tile == 0) {
            if (tid == 0) st_release_u64(status + tile, kFlagInc | (unsigned long long)total);
        } else {
            if (tid == 0) st_release_u64(status + tile, kFlagAgg | (unsigned long long)total);
            p = lookback_sum_warp(status, tile, ctl, 102);
            if (tid == 0) st_release_u64(status + tile, kFlagInc | (p + total));
        }
        if (tid == 0) {
            s_prefix = p;
            if ((uint64_t)(tile + 1) * TILE >= n) ctl->count[0] = p + total;
        }
    }
    __syncthreads();
    const unsigned long long base = s_prefix + wexcl;
    uint64_t prev[2 * W];
    bool have_prev = false;
    unsigned int run = 0;
#pragma unroll
    for (int i = 0; i < ITEMS; ++i) {
        const unsigned int b = ball[i];
        if (b != 0) {  // warp-uniform
            const unsigned int lower = b & lanemask_lt;
            const int src = lower ? 31 - __clz(lower) : lane;
            const int hi = 31 - __clz(b);
            // keys are read again here (this tile was just streamed, so L2 holds it) rather
            // than kept in registers across the look-back
            const uint64_t row = wbase + (uint64_t)i * 32 + lane;
            uint64_t ki[2 * W];
            if (row < n)
                load_key<W>(keys, row, ki);
            else
#pragma unroll
                for (int w = 0; w < 2 * W; ++w) ki[w] = 0;
            uint64_t pk[2 * W];
#pragma unroll
            for (int w = 0; w < 2 * W; ++w) pk[w] = __shfl_sync(0xffffffffu, ki[w], src);
            if ((b >> lane) & 1u) {
                const unsigned long long j = base + run + __popc(lower);
                if (PS_BOUNDS(ctl, j < n, 103)) {
                    idx[j] = (uint32_t)(wbase + (uint64_t)i * 32 + lane);
                    uint16_t d;
                    if (lower)
                        d = (uint16_t)div_regs<W>(pk, ki);
                    else if (have_prev)
                        d = (uint16_t)div_regs<W>(prev, ki);
                    else
                        d = j == 0 ? kDivStart : kDivUnknown;
                    D[j] = d;
                }
            }
#pragma unroll
            for (int w = 0; w < 2 * W; ++w) prev[w] = __shfl_sync(0xffffffffu, ki[w], hi);
            have_prev = true;
            run += __popc(b);
        }
    }
}

// ---------------------------------------------------------------------------
// level scans.  For level rank L, a "group" is a maximal run of partners sharing
// every key bit more significant than L, and its "split" is the first row whose
// bit L is set.  Starts: j == 0 or D[j] < L.  Splits: D[j] == L.
// ---------------------------------------------------------------------------
// The level scans run in three phases with no look-back: k_level_reduce writes each tile's
// aggregates for both directions, k_level_scan (one block) combines them into each tile's
// exclusive prefix (forward, max) and suffix (backward, min), and k_level_apply finishes both
// scans per partner and, on the last batch of levels, places it.  With every tile of a scan in
// flight at once, a decoupled look-back would walk back hundreds of tiles.  Per-tile values
// (LevelTile: forward values at [0, 2LV), backward at [2LV, 4LV)) live in the caller's level
// slot buffer.

// One thread's aggregates over its kScanItems partners starting at j0 (those below m).
// Forward, agg[2l], agg[2l+1]: last start / last split of level l (identity -1, max).
// Backward, agg[2LV+2l], agg[2LV+2l+1]: first start after a group / first split (identity
// kLevelInf, min).
template <int LV, int IT = kScanItems>
__device__ __forceinline__ void level_thread_agg(const uint16_t (&d)[IT], uint32_t j0, uint32_t m,
                                                 const Levels& lv, int (&agg)[4 * LV]) {
    const int NL = lv.n;
#pragma unroll
    for (int l = 0; l < LV; ++l) {
        agg[2 * l] = agg[2 * l + 1] = -1;
        agg[2 * LV + 2 * l] = agg[2 * LV + 2 * l + 1] = kLevelInf;
        if (l < NL) {
            const uint32_t Lr = lv.rank[l];
#pragma unroll
            for (int i = 0; i < IT; ++i) {
                const uint32_t j = j0 + i;
                if (j < m) {
                    if (j == 0 || d[i] < Lr) agg[2 * l] = (int)j;
                    if (j != 0 && d[i] == Lr) agg[2 * l + 1] = (int)j;
                }
            }
#pragma unroll
            for (int i = IT - 1; i >= 0; --i) {
                const uint32_t j = j0 + i;
                if (j < m) {
                    if (j != 0 && d[i] < Lr) agg[2 * LV + 2 * l] = (int)j;
                    if (j != 0 && d[i] == Lr) agg[2 * LV + 2 * l + 1] = (int)j;
                }
            }
        }
    }
}

// value v of a LevelTile row combines by max (forward half) or min (backward half)
template <int LV>
__device__ __forceinline__ int level_comb(int v, int a, int b) {
    return v < 2 * LV ? max(a, b) : min(a, b);
}
template <int LV>
__device__ __forceinline__ int level_id(int v) {
    return v < 2 * LV ? -1 : kLevelInf;
}

// Phase 1: each tile's aggregates.  It also resolves the divergence ranks that k_classify left
// unknown (the first listed row of each warp), so the later phases read them.
template <int W, int LV>
__global__ void __launch_bounds__(kBlock) k_level_reduce(const uint32_t* __restrict__ idx, uint16_t* __restrict__ D,
                                                         const uint64_t* __restrict__ keys, uint64_t n, const Levels lv,
                                                         LevelTile* __restrict__ tiles, Ctl* ctl) {
    __shared__ int s_w[kBlock / 32][4 * LV];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t m = (uint32_t)ctl->count[0];  // partners, published by k_classify
    const uint32_t ntiles = (m + kScanTile - 1) / kScanTile;
    for (uint32_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const uint32_t j0 = tile * (uint32_t)kScanTile + (uint32_t)tid * kScanItems;
        uint16_t d[kScanItems];
        unsigned int unknown = 0;  // bit i: item i's rank is left for this kernel to resolve
#pragma unroll
        for (int i = 0; i < kScanItems; ++i) {
            const uint32_t j = j0 + i;
            d[i] = j < m ? D[j] : (uint16_t)0;
        }
#pragma unroll
        for (int i = 0; i < kScanItems; ++i)
            if (j0 + i < m && j0 + i > 0 && d[i] == kDivUnknown) unknown |= 1u << i;
        // one pass per unknown item of this thread (rarely more than one), its loads issued
        // together rather than item by item
        while (unknown) {
            const int i = __ffs(unknown) - 1;
            unknown &= unknown - 1;
            const uint32_t j = j0 + i;
            const uint32_t ra = idx[j - 1], rb = idx[j];
            uint16_t r = kDivUnknown;
            if (PS_GUARD(ctl, ra < n && rb < n, 201)) {
                uint64_t ka[2 * W], kb[2 * W];
                load_key<W>(keys, ra, ka);
                load_key<W>(keys, rb, kb);
                r = (uint16_t)divergence<W>(ka, kb);
                D[j] = r;
            }
#pragma unroll
            for (int q = 0; q < kScanItems; ++q)
                if (q == i) d[q] = r;
        }
        int agg[4 * LV];
        level_thread_agg<LV>(d, j0, m, lv, agg);
#pragma unroll
        for (int v = 0; v < 4 * LV; ++v) {
            int x = agg[v];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) x = level_comb<LV>(v, x, __shfl_xor_sync(0xffffffffu, x, o));
            if (lane == 0) s_w[warp][v] = x;
        }
        __syncthreads();
        if (tid < 4 * LV) {
            int x = level_id<LV>(tid);
            for (int w = 0; w < kBlock / 32; ++w) x = level_comb<LV>(tid, x, s_w[w][tid]);
            tiles[tile].agg[tid] = x;
        }
        __syncthreads();
    }
}

// Phase 2, one block of kScanThreads: pre = the forward aggregates of the tiles before (max)
// and the backward aggregates of the tiles after (min).  Rounds of kScanThreads tiles, one
// tile per thread with a block scan and a carry: ascending for the forward values, descending
// for the backward ones.
constexpr int kScanThreads = 1024;
template <bool kFwd, int LV>
__device__ __forceinline__ void level_scan_pass(LevelTile* __restrict__ tiles, uint32_t ntiles,
                                                int (&s_w)[kScanThreads / 32][2 * LV], int (&s_carry)[2 * LV]) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    constexpr int ID = kFwd ? -1 : kLevelInf;
    constexpr int OFF = kFwd ? 0 : 2 * LV;
    auto comb = [](int a, int b) { return kFwd ? max(a, b) : min(a, b); };
    if (tid < 2 * LV) s_carry[tid] = ID;
    const uint32_t rounds = (ntiles + kScanThreads - 1) / kScanThreads;
    for (uint32_t r = 0; r < rounds; ++r) {
        // forward: tile r * kScanThreads + tid; backward: counted from the last tile
        const long long pos = kFwd ? (long long)r * kScanThreads + tid
                                   : (long long)ntiles - 1 - ((long long)r * kScanThreads + tid);
        const bool have = kFwd ? pos < (long long)ntiles : pos >= 0;
        int x[2 * LV];
#pragma unroll
        for (int v = 0; v < 2 * LV; ++v) x[v] = have ? tiles[pos].agg[OFF + v] : ID;
        int excl[2 * LV];
#pragma unroll
        for (int v = 0; v < 2 * LV; ++v) {
            int y = x[v];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int z = __shfl_up_sync(0xffffffffu, y, o);
                if (lane >= o) y = comb(y, z);
            }
            const int e = __shfl_up_sync(0xffffffffu, y, 1);
            excl[v] = lane == 0 ? ID : e;
            if (lane == 31) s_w[warp][v] = y;
        }
        __syncthreads();
#pragma unroll
        for (int v = 0; v < 2 * LV; ++v) {
            int c = s_carry[v];
            for (int w = 0; w < warp; ++w) c = comb(c, s_w[w][v]);
            if (have) tiles[pos].pre[OFF + v] = comb(c, excl[v]);
        }
        __syncthreads();
        if (tid < 2 * LV) {
            int c = s_carry[tid];
            for (int w = 0; w < kScanThreads / 32; ++w) c = comb(c, s_w[w][tid]);
            s_carry[tid] = c;
        }
        __syncthreads();
    }
}

template <int LV>
__global__ void __launch_bounds__(kScanThreads) k_level_scan(LevelTile* __restrict__ tiles, Ctl* ctl) {
    __shared__ int s_w[kScanThreads / 32][2 * LV];
    __shared__ int s_carry[2 * LV];
    const uint32_t m = (uint32_t)ctl->count[0];
    const uint32_t ntiles = (m + kScanTile - 1) / kScanTile;
    level_scan_pass<true, LV>(tiles, ntiles, s_w, s_carry);
    level_scan_pass<false, LV>(tiles, ntiles, s_w, s_carry);
}

// Phase 3 (blocks of NT threads over the same 4096-partner tiles: at 8 partners per thread the
// apply's registers allow more resident warps to cover its gather latency): per partner j, F = sum over levels of -(split - start) for rows in an upper half
// (forward) plus (group end - split) for rows in a lower half (backward), added to the F of
// earlier batches; on the last batch each partner goes to j + F.
template <int W, typename T, int LV, int NT, bool NOISE>
__global__ void __launch_bounds__(NT) k_level_apply(const uint32_t* __restrict__ idx,
                                                        const uint16_t* __restrict__ D, int32_t* __restrict__ F,
                                                        const uint64_t* __restrict__ keys, const T* __restrict__ coef,
                                                        uint64_t n, const Levels lv, const RotLayer<W> L,
                                                        int accumulate, int scatter, uint64_t* __restrict__ Pk,
                                                        T* __restrict__ Pc, const LevelTile* __restrict__ tiles,
                                                        Ctl* ctl, const KeepProg keep, const NoiseArg<NOISE> N,
                                                        const float* __restrict__ Sf, float* __restrict__ Pf) {
    constexpr int IT = kScanTile / NT;  // partners per thread
    __shared__ int s_w[NT / 32][4 * LV];
    __shared__ AmpTab<T> A;
    __shared__ NoiseShared<T, NOISE> NSH;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    stage_amps<W, T>(L, A);
    if constexpr (NOISE) stage_noise<T>(N, *NSH.tab());
    __syncthreads();
    const uint32_t m = (uint32_t)ctl->count[0];
    const uint32_t ntiles = (m + kScanTile - 1) / kScanTile;
    const int NL = lv.n;
    for (uint32_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const uint32_t j0 = tile * (uint32_t)kScanTile + (uint32_t)tid * IT;
        uint16_t d[IT];
#pragma unroll
        for (int i = 0; i < IT; ++i) {
            const uint32_t j = j0 + i;
            d[i] = j < m ? D[j] : (uint16_t)0;
        }
        int agg[4 * LV];
        level_thread_agg<LV, IT>(d, j0, m, lv, agg);
        // exclusive scans over the block's threads (prefix max / suffix min), then the tile's pre
        int excl[4 * LV];
#pragma unroll
        for (int v = 0; v < 4 * LV; ++v) {
            const bool fwd = v < 2 * LV;
            int x = agg[v];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int y = fwd ? __shfl_up_sync(0xffffffffu, x, o) : __shfl_down_sync(0xffffffffu, x, o);
                if (fwd ? lane >= o : lane + o < 32) x = level_comb<LV>(v, x, y);
            }
            const int e = fwd ? __shfl_up_sync(0xffffffffu, x, 1) : __shfl_down_sync(0xffffffffu, x, 1);
            excl[v] = (fwd ? lane == 0 : lane == 31) ? level_id<LV>(v) : e;
            if (fwd ? lane == 31 : lane == 0) s_w[warp][v] = x;
        }
        __syncthreads();
#pragma unroll
        for (int v = 0; v < 4 * LV; ++v) {
            if (v < 2 * LV) {
                for (int w = 0; w < warp; ++w) excl[v] = max(excl[v], s_w[w][v]);
            } else {
                for (int w = warp + 1; w < NT / 32; ++w) excl[v] = min(excl[v], s_w[w][v]);
            }
            excl[v] = level_comb<LV>(v, excl[v], tiles[tile].pre[v]);
        }
        __syncthreads();  // s_w is rewritten by the next tile
        int f[IT];
#pragma unroll
        for (int i = 0; i < IT; ++i) {
            const uint32_t j = j0 + i;
            f[i] = 0;
#pragma unroll
            for (int l = 0; l < LV; ++l) {
                if (l < NL && j < m) {
                    const uint32_t Lr = lv.rank[l];
                    if (j == 0 || d[i] < Lr) excl[2 * l] = (int)j;
                    if (j != 0 && d[i] == Lr) excl[2 * l + 1] = (int)j;
                    const int st = excl[2 * l], sp = excl[2 * l + 1];
                    if (sp > st) f[i] -= (sp - st);
                }
            }
        }
#pragma unroll
        for (int i = IT - 1; i >= 0; --i) {
            const uint32_t j = j0 + i;
            if (j >= m) continue;
#pragma unroll
            for (int l = 0; l < LV; ++l) {
                if (l < NL) {
                    int* ex = excl + 2 * LV;
                    const int e = ex[2 * l] == kLevelInf ? (int)m : ex[2 * l];
                    const int q = ex[2 * l + 1];
                    if (q < e) f[i] += e - q;
                    const uint32_t Lr = lv.rank[l];
                    if (j != 0 && d[i] < Lr) ex[2 * l] = (int)j;
                    if (j != 0 && d[i] == Lr) ex[2 * l + 1] = (int)j;
                }
            }
            const int ft = accumulate ? F[j] + f[i] : f[i];
            if (!scatter) {
                F[j] = ft;
                continue;
            }
            const long long dest = (long long)j + ft;
            const uint32_t row = idx[j];
            if (!PS_GUARD(ctl, dest >= 0 && dest < (long long)m && row < n, 204)) continue;
            uint64_t k[2 * W];
            load_key<W>(keys, row, k);
            T c = coef[row];
            T pc;
            if constexpr (NOISE) {
                // a parent the folded noise drops has no partner: a zero partner adds nothing to
                // an equal own row and is dropped as an exact zero otherwise
                pc = noise_apply<W, T>(*NSH.tab(), keep, k, c) < NSH.tab()->n ? T(0) : partner_coeff<W, T>(L, A, k, c);
            } else {
                pc = partner_coeff<W, T>(L, A, k, c);
            }
#pragma unroll
            for (int w = 0; w < W; ++w) {
                k[w] ^= L.gx[w];
                k[W + w] ^= L.gz[w];
            }
            store_key<W>(Pk, (uint64_t)dest, k);
            Pc[dest] = pc;
            if (Pf) Pf[dest] = Sf[row];  // a partner inherits its parent's prediction
        }
    }
}

// ---------------------------------------------------------------------------
// merge-path partition: bounds[t] = (i, j) where tile t starts; pairs of equal keys
// (own row, partner) never straddle a boundary.
// ---------------------------------------------------------------------------
template <int W>
__device__ __forceinline__ bool mp_pred(const uint64_t* Sk, const uint64_t* Pk, uint64_t i, uint64_t d) {
    // S[i] <= P[d - 1 - i]
    return key_le<W>(Sk + i * 2 * W, Pk + (d - 1 - i) * 2 * W);
}

template <int W>
__global__ void k_partition(const uint64_t* __restrict__ Sk, uint64_t n, const uint64_t* __restrict__ Pk,
                            uint32_t tile_items, ulonglong2* __restrict__ bounds, const Ctl* ctl) {
    const int lane = threadIdx.x & 31;
    const uint64_t m = ctl->count[0];  // partners, published by k_classify (0 without partners)
    const uint32_t num_tiles = (uint32_t)((n + m + tile_items - 1) / tile_items);
    const uint32_t warps = gridDim.x * (blockDim.x >> 5);
    // Each warp takes a run of consecutive boundaries (the grid is sized by residency).  The
    // split moves by at most tile_items from one boundary to the next, so after the first of
    // the run the search starts in a window of that width, on keys the last search touched.
    const uint32_t per = (num_tiles + 1 + warps - 1) / warps;
    const uint32_t t0 = (blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) * per;
    uint64_t prev_i = 0;
    for (uint32_t t = t0; t <= num_tiles && t < t0 + per; ++t) {
        uint64_t dd = (uint64_t)t * tile_items;
        if (dd > n + m) dd = n + m;
        uint64_t lo = dd > m ? dd - m : 0, hi = dd < n ? dd : n;  // answer in [lo, hi]
        if (t > t0) {
            lo = lo > prev_i ? lo : prev_i;
            hi = hi < prev_i + tile_items ? hi : prev_i + tile_items;
        }
        while (hi - lo > 32) {
            uint64_t span = hi - lo;
            uint64_t p = lo + (span * (uint64_t)lane) / 32;  // p_0 = lo, all < hi
            bool f = mp_pred<W>(Sk, Pk, p, dd);
            unsigned int b = __ballot_sync(0xffffffffu, f);
            int c = __popc(b);
            if (c == 0) {
                hi = lo;
                break;
            }
            uint64_t pc1 = lo + (span * (uint64_t)(c - 1)) / 32;
            uint64_t pc = c < 32 ? lo + (span * (uint64_t)c) / 32 : hi;
            lo = pc1 + 1;
            hi = pc;
        }
        uint64_t span = hi - lo;
        bool f = (uint64_t)lane < span ? mp_pred<W>(Sk, Pk, lo + lane, dd) : false;
        unsigned int b = __ballot_sync(0xffffffffu, f);
        uint64_t i = lo + (uint64_t)__popc(b);
        uint64_t j = dd - i;
        prev_i = i;
        if (lane == 0) {
            if (i > 0 && j < m && key_eq<W>(Sk + (i - 1) * 2 * W, Pk + j * 2 * W)) ++j;
            bounds[t] = make_ulonglong2(i, j);
        }
    }
}

// ---------------------------------------------------------------------------
// k_merge
// ---------------------------------------------------------------------------
template <int W, typename T>
struct MergeSmem {
    static constexpr int TILE = RotTile<W>::kMergeTile;
    static constexpr int PAD = 16 / (int)sizeof(T);  // elements of alignment slack per stream
    static constexpr int KEY_ROWS = TILE + 4;
    static constexpr int COEF_SLOTS = TILE + 4 + 4 * PAD;
    static constexpr size_t key_bytes = (size_t)KEY_ROWS * 16 * W;
    static constexpr size_t coef_bytes = ((size_t)COEF_SLOTS * sizeof(T) + 15) / 16 * 16;
    static constexpr size_t bytes = key_bytes + coef_bytes;
    // the learned pass's prediction column (floats, 16-byte windows of 4), after the coefficients
    static constexpr int F_SLOTS = TILE + 4 + 16;
    static constexpr size_t f_bytes = ((size_t)F_SLOTS * sizeof(float) + 15) / 16 * 16;
};

template <int W>
__device__ __forceinline__ void ld_row(const uint64_t* base, uint32_t r, uint64_t (&k)[2 * W]) {
    const ulonglong2* p = reinterpret_cast<const ulonglong2*>(base + (size_t)r * 2 * W);
#pragma unroll
    for (int q = 0; q < W; ++q) {
        ulonglong2 v = p[q];
        k[2 * q] = v.x;
        k[2 * q + 1] = v.y;
    }
}

template <int W>
__device__ __forceinline__ bool le_regs(const uint64_t (&a)[2 * W], const uint64_t (&b)[2 * W]) {
#pragma unroll
    for (int i = 0; i < 2 * W; ++i)
        if (a[i] != b[i]) return a[i] < b[i];
    return true;
}
template <int W>
__device__ __forceinline__ bool eq_regs(const uint64_t (&a)[2 * W], const uint64_t (&b)[2 * W]) {
    uint64_t d = 0;
#pragma unroll
    for (int i = 0; i < 2 * W; ++i) d |= a[i] ^ b[i];
    return d == 0;
}

// Walk one thread's merge-path range once, with the two run heads held in registers (one
// shared load per consumed item).  Own row first, partner second when their keys are equal, as
// the reference's merge sums bucket-first.  A range holds at most ITEMS + 1 rows and an equal
// pair is consumed in one step, so STEPS = ITEMS + 1 unrolled steps cover it (the caller checks
// that nothing is left).  Step s leaves its output in ok[s] / ov[s] and sets bit s of the
// returned mask when the output is kept (nonzero and passing the keep program).
template <int W, typename T, int STEPS, bool NOISE, bool HASF>
__device__ __forceinline__ uint32_t merge_walk(const uint64_t* sSk, const T* sSc, const uint64_t* sPk, const T* sPc,
                                               uint32_t& i, uint32_t ie, uint32_t& j, uint32_t je,
                                               const RotLayer<W>& L, const AmpTab<T>& A, const KeepProg& keep,
                                               uint64_t (&ok)[STEPS][2 * W], T (&ov)[STEPS],
                                               const NoiseSmem<T>* NS, unsigned int* s_drop, const float* sSf,
                                               const float* sPf, float (&of)[STEPS]) {
    uint32_t mask = 0;
    uint64_t a[2 * W], b[2 * W];
    if (i < ie) ld_row<W>(sSk, i, a);
    if (j < je) ld_row<W>(sPk, j, b);
#pragma unroll
    for (int s = 0; s < STEPS; ++s) {
        if (i < ie || j < je) {
            const bool takeS = (j >= je) || (i < ie && le_regs<W>(a, b));
            T v;
            if (takeS) {
#pragma unroll
                for (int w = 0; w < 2 * W; ++w) ok[s][w] = a[w];
                if constexpr (HASF) of[s] = sSf[i];  // the string's own prediction
                if constexpr (NOISE) {
                    T c = sSc[i];
                    const int d = noise_apply<W, T>(*NS, keep, a, c);
                    if (d < NS->n) {
                        atomicAdd(&s_drop[d], 1u);
                        v = T(0);
                    } else {
                        v = own_coeff<W, T>(L, A, a, c);
                    }
                } else {
                    v = own_coeff<W, T>(L, A, a, sSc[i]);
                }
                if (j < je && eq_regs<W>(a, b)) {
                    v = add_rn(v, sPc[j]);
                    if (++j < je) ld_row<W>(sPk, j, b);
                }
                if (++i < ie) ld_row<W>(sSk, i, a);
            } else {
#pragma unroll
                for (int w = 0; w < 2 * W; ++w) ok[s][w] = b[w];
                if constexpr (HASF) of[s] = sPf[j];  // a new string: its parent's prediction
                v = sPc[j];
                if (++j < je) ld_row<W>(sPk, j, b);
            }
            ov[s] = v;
            if (v != T(0) && keep_eval<W>(keep, ok[s], to_f64(v))) mask |= 1u << s;
        }
    }
    return mask;
}

template <int W, typename T, bool NOISE, bool HASF, bool NEXTF = false>
__global__ void __launch_bounds__(kBlock, W == 1 ? 4 : 1) k_merge(const uint64_t* __restrict__ Sk, const T* __restrict__ Sc,
                                                  uint64_t n, const uint64_t* __restrict__ Pk,
                                                  const T* __restrict__ Pc, const ulonglong2* __restrict__ bounds,
                                                  const RotLayer<W> L, const KeepProg keep,
                                                  uint64_t* __restrict__ Ok, T* __restrict__ Oc, uint64_t out_cap,
                                                  unsigned long long* status, Ctl* ctl,
                                                  unsigned int* __restrict__ topn_hist, int hist_mode,
                                                  uint64_t hist_base, unsigned int* __restrict__ slot_count,
                                                  long long stall_limit, const NoiseArg<NOISE> N,
                                                  unsigned long long* __restrict__ noise_drops,
                                                  const float* __restrict__ Sf, const float* __restrict__ Pf,
                                                  float* __restrict__ Of, const NextArg<W, NEXTF> NX = {}) {
    using SM = MergeSmem<W, T>;
    constexpr int ITEMS = RotTile<W>::kMergeItems;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    uint64_t* sK = reinterpret_cast<uint64_t*>(smem_raw);
    T* sC = reinterpret_cast<T*>(smem_raw + SM::key_bytes);
    float* sF = reinterpret_cast<float*>(smem_raw + SM::bytes);  // HASF only
    __shared__ uint64_t bar;
    __shared__ unsigned int s_tile;
    __shared__ unsigned int s_warp[kBlock / 32];
    __shared__ unsigned int s_si[kBlock + 1], s_sj[kBlock + 1];
    __shared__ unsigned long long s_outoff;
    __shared__ unsigned int s_hist[kTopnHistBins];
    __shared__ AmpTab<T> A;
    __shared__ AmpTab<T> NA;  // the next layer's amplitudes (NEXTF)
    __shared__ NoiseShared<T, NOISE> NSH;
    NoiseSmem<T>* NS = NSH.tab();
    unsigned int* s_drop = NSH.drops();

    const int tid = threadIdx.x;
    if (tid == 0) mbar_init(&bar, 1);
    if (topn_hist)
        for (int q = tid; q < kTopnHistBins; q += kBlock) s_hist[q] = 0;
    stage_amps<W, T>(L, A);
    if constexpr (NEXTF) stage_amps<W, T>(NX.L, NA);
    if constexpr (NOISE) {
        stage_noise<T>(N, *NS);
        for (int q = tid; q <= kMaxNoise; q += kBlock) s_drop[q] = 0;
    }
    const uint64_t m = ctl->count[0];  // partners, published by k_classify (0 without partners)
    const uint32_t num_tiles = (uint32_t)((n + m + SM::TILE - 1) / SM::TILE);
    // a slotted output's span, for the TopN pass that reads it without the host knowing m
    if (slot_count && blockIdx.x == 0 && tid == 0) ctl->span = (unsigned long long)num_tiles * (SM::TILE + 2);
    uint32_t phase = 0;  // completed phases of `bar`
    // Persistent: each block takes tiles from the dispenser until none is left (the grid is
    // sized by residency, not by the tile count, which only the device knows).
    for (;;) {
        if (tid == 0) s_tile = atomicAdd(&ctl->tile_counter[3], 1u);
        __syncthreads();  // also: every thread is done with the previous tile's shared memory
        const unsigned int tile = s_tile;
        if (tile >= num_tiles) break;
        const ulonglong2 b0 = bounds[tile], b1 = bounds[tile + 1];
        if (!PS_GUARD(ctl, b1.x >= b0.x && b1.y >= b0.y && b1.x - b0.x + b1.y - b0.y <= (uint64_t)SM::TILE + 2 &&
                               b1.x <= n && b1.y <= m,
                      301))
            break;
        const uint32_t cs = (uint32_t)(b1.x - b0.x), cp = (uint32_t)(b1.y - b0.y);
        // stage the two input runs: keys packed (S then P), coefficients from 16-byte aligned windows
        const uint64_t sa = b0.x & ~(uint64_t)(SM::PAD - 1), pa = b0.y & ~(uint64_t)(SM::PAD - 1);
        const uint32_t s_off = (uint32_t)(b0.x - sa), p_off = (uint32_t)(b0.y - pa);
        const uint32_t sc_slots = (s_off + cs + SM::PAD - 1) / SM::PAD * SM::PAD;
        T* sSc = sC;             // S coefficient of local i at sSc[s_off + i]
        T* sPc = sC + sc_slots;  // P coefficient of local j at sPc[p_off + j]
        uint64_t* sSk = sK;
        uint64_t* sPk = sK + (size_t)cs * 2 * W;
        // the prediction column, in windows of 4 floats (16 bytes)
        const uint64_t fsa = b0.x & ~(uint64_t)3, fpa = b0.y & ~(uint64_t)3;
        const uint32_t fs_off = (uint32_t)(b0.x - fsa), fp_off = (uint32_t)(b0.y - fpa);
        const uint32_t sf_slots = (fs_off + cs + 3) / 4 * 4;
        float* sSf = sF;
        float* sPf = sF + sf_slots;
        if (tid == 0 && cs + cp) {
            bulk_wait_read_all();  // the previous tile's bulk store has read the staged rows
            uint32_t kbS = cs * 16u * W, kbP = cp * 16u * W;
            uint32_t cbS = cs ? round16((s_off + cs) * (uint32_t)sizeof(T)) : 0u;
            uint32_t cbP = cp ? round16((p_off + cp) * (uint32_t)sizeof(T)) : 0u;
            uint32_t fbS = 0, fbP = 0;
            if constexpr (HASF) {
                fbS = cs ? round16((fs_off + cs) * 4u) : 0u;
                fbP = cp ? round16((fp_off + cp) * 4u) : 0u;
            }
            mbar_arrive_expect_tx(&bar, kbS + kbP + cbS + cbP + fbS + fbP);
            if (kbS) bulk_g2s(sSk, Sk + b0.x * 2 * W, kbS, &bar);
            if (kbP) bulk_g2s(sPk, Pk + b0.y * 2 * W, kbP, &bar);
            if (cbS) bulk_g2s(sSc, Sc + sa, cbS, &bar);
            if (cbP) bulk_g2s(sPc, Pc + pa, cbP, &bar);
            if constexpr (HASF) {
                if (fbS) bulk_g2s(sSf, Sf + fsa, fbS, &bar);
                if (fbP) bulk_g2s(sPf, Pf + fpa, fbP, &bar);
            }
        }
        if (cs + cp) {  // block-uniform
            const bool ok = mbar_wait(&bar, phase & 1u, ctl, 302);
            // a wait that gave up (ERR_TIMEOUT is flagged) ends the block: its copies land first,
            // and nothing reads the unfilled tile or issues another copy into it
            if (__syncthreads_or(ok ? 0 : 1)) {
                if (tid == 0) mbar_drain(&bar, phase & 1u);
                break;
            }
            ++phase;
        }
        const T* Sc_l = sSc + s_off;
        const T* Pc_l = sPc + p_off;

        // per-thread merge-path start, equal pairs kept together
        {
            uint32_t dd = min((uint32_t)tid * ITEMS, cs + cp);
            uint32_t lo = dd > cp ? dd - cp : 0, hi = min(dd, cs);
            while (lo < hi) {
                uint32_t mid = (lo + hi) >> 1;
                if (key_le<W>(sSk + (size_t)mid * 2 * W, sPk + (size_t)(dd - 1 - mid) * 2 * W))
                    lo = mid + 1;
                else
                    hi = mid;
            }
            uint32_t i = lo, j = dd - lo;
            if (i > 0 && j < cp && key_eq<W>(sSk + (size_t)(i - 1) * 2 * W, sPk + (size_t)j * 2 * W)) ++j;
            s_si[tid] = i;
            s_sj[tid] = j;
            if (tid == 0) {
                s_si[kBlock] = cs;
                s_sj[kBlock] = cp;
            }
        }
        __syncthreads();
        const uint32_t i0 = s_si[tid], j0 = s_sj[tid];
        const uint32_t ie = max(s_si[tid + 1], i0), je = max(s_sj[tid + 1], j0);
        constexpr int STEPS = ITEMS + 1;
        uint64_t ok[STEPS][2 * W];
        T ov[STEPS];
        float of[STEPS];
        uint32_t i = i0, j = j0;
        const uint32_t mask = merge_walk<W, T, STEPS, NOISE, HASF>(sSk, Sc_l, sPk, Pc_l, i, ie, j, je, L, A, keep, ok,
                                                                  ov, NS, s_drop, sSf + fs_off, sPf + fp_off, of);
        PS_GUARD(ctl, i >= ie && j >= je, 305);
        unsigned int total;
        const unsigned int excl = block_exclusive_sum<kBlock>(__popc(mask), s_warp, total);
        // Every thread is past the walk, so the staged inputs are dead: stage the kept outputs
        // over them in output order (keys from sK, coefficients from sC) while warp 0 looks back.
        {
            uint32_t r = excl;
#pragma unroll
            for (int s = 0; s < STEPS; ++s) {
                if ((mask >> s) & 1u) {
                    store_key<W>(sK, r, ok[s]);
                    sC[r] = ov[s];
                    if constexpr (HASF) sF[r] = of[s];
                    ++r;
                }
            }
        }
        fence_proxy_async_shared();  // the bulk store below reads the staged keys through the async proxy
        if (slot_count) {
            // slotted output: the tile's slot is fixed, so it waits for no predecessor
            if (tid == 0) {
                s_outoff = (unsigned long long)tile * (SM::TILE + 2);
                slot_count[tile] = total;
                atomicAdd(&ctl->count[1], (unsigned long long)total);
            }
        } else if (tid < 32) {
            unsigned long long p = 0;
            if (tile == 0) {
                if (tid == 0) st_release_u64(status + tile, kFlagInc | (unsigned long long)total);
            } else {
                if (tid == 0) st_release_u64(status + tile, kFlagAgg | (unsigned long long)total);
                p = lookback_sum_warp(status, tile, ctl, 303, stall_limit);
                if (tid == 0) st_release_u64(status + tile, kFlagInc | (p + total));
            }
            if (tid == 0) {
                s_outoff = p;
                if (tile == num_tiles - 1) ctl->count[1] = p + total;
            }
        }
        __syncthreads();
        const unsigned long long off = s_outoff;
        if (!PS_GUARD(ctl, off + total <= out_cap, 304)) break;
        // keys: one bulk copy of the staged rows (16W bytes each, so both ends are 16-byte aligned)
        if (tid == 0 && total) {
            bulk_s2g(Ok + off * 2 * W, sK, total * 16u * W);
            bulk_commit();
        }
        // coefficients (and predictions): coalesced stores, with the fused first TopN digit
        for (uint32_t q = tid; q < total; q += kBlock) {
            const T v = sC[q];
            Oc[off + q] = v;
            if constexpr (NEXTF) {
                uint64_t k[2 * W];
                ld_row<W>(sK, q, k);
                NX.flags[off + q] = emits_partner_regs<W, T>(NX.L, NA, k) ? 1 : 0;
            }
            float fv = 0.0f;
            if constexpr (HASF) {
                fv = sF[q];
                Of[off + q] = fv;
            }
            if (topn_hist) {
                uint32_t bin;
                if (hist_mode == 1)
                    bin = octave_bin<T>(v);
                else if (hist_mode == 2)
                    bin = (uint32_t)(window_key(mag_key<T>(v), hist_base) >> 48);
                else if (hist_mode == 3)
                    bin = (uint32_t)(score_key<T>(v, fv) >> 52);
                else if (hist_mode == 4)
                    bin = (uint32_t)(window_key(score_key<T>(v, fv), hist_base) >> 48);
                else
                    bin = (uint32_t)(mag_key<T>(v) >> 52);
                atomicAdd(&s_hist[bin], 1u);
            }
        }
    }
    if (topn_hist) {
        __syncthreads();
        for (int q = tid; q < kTopnHistBins; q += kBlock)
            if (s_hist[q]) atomicAdd(&topn_hist[q], s_hist[q]);
    }
    if constexpr (NOISE) {
        __syncthreads();
        for (int q = tid; q <= kMaxNoise; q += kBlock)
            if (s_drop[q]) atomicAdd(&noise_drops[q], (unsigned long long)s_drop[q]);
    }
    if (tid == 0) bulk_wait_read_all();  // shared memory stays valid until the last copy has read it
}

// One launch resets what a rotation layer's kernels count on: the partner count (unless the
// partner list is already there) and the output count,
// the tile dispensers (the merge's starts at `merge_start`, 1 under failure injection), the
// look-back words of the classify and the merge (disjoint ranges of `status`) and the folded
// noise's drop counters.
__global__ void k_layer_prep(Ctl* ctl, unsigned long long* __restrict__ status, uint32_t nstatus,
                             unsigned int merge_start, unsigned long long* __restrict__ noise_drops, int keep_m) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < 2 && !(t == 0 && keep_m)) ctl->count[t] = 0;
    if (t < 4) ctl->tile_counter[t] = t == 3 ? merge_start : 0u;
    if (noise_drops && t <= (uint32_t)kMaxNoise) noise_drops[t] = 0;
    for (uint32_t i = t; i < nstatus; i += gridDim.x * blockDim.x) status[i] = 0;
}

// ---------------------------------------------------------------------------
// host launchers
// ---------------------------------------------------------------------------
// Resident blocks per SM of a kernel, looked up on first use and kept for the process (every
// device this library runs on is a B200, so one value serves all).
template <typename K>
int resident_blocks(K kernel, int threads, size_t smem, std::atomic<int>& cache) {
    int v = cache.load(std::memory_order_relaxed);
    if (v == 0) {
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, kernel, threads, smem) != cudaSuccess || v < 1) v = 1;
        cache.store(v, std::memory_order_relaxed);
    }
    return v;
}

template <int W, typename T>
cudaError_t launch_rotation_layer(const RotationArgs<W, T>& a, cudaStream_t st) {
    // One host synchronization per layer: k_classify publishes the partner count m on the
    // device and every later kernel reads it there, their grids sized for m = n (surplus blocks
    // return at once); the host reads m, the output count and the error flags in one copy at
    // the end.
    constexpr int CT = RotTile<W>::kClassifyTile;
    constexpr int MT = RotTile<W>::kMergeTile;
    Ctl* ctl = a.ctl;
    cudaError_t e;
    const uint64_t m_hi = a.L.partners ? a.n : 0;  // partners cannot outnumber the terms
    if (m_hi > a.p_cap) return cudaErrorMemoryAllocation;  // caller sized the partner buffers by n
    // look-back words: the classify's tiles first, then the merge's (when it is not slotted)
    const uint32_t ctiles = m_hi > 0 ? (uint32_t)((a.n + CT - 1) / CT) : 0u;
    const uint32_t mtiles_max = (uint32_t)((a.n + m_hi + MT - 1) / MT);
    unsigned long long* merge_status = a.status + ctiles;
    {
        const uint32_t nstatus = ctiles + (a.slot_count ? 0u : mtiles_max);
        const uint32_t blocks = std::max<uint32_t>(1u, std::min<uint32_t>((nstatus + 255) / 256, 4u * (uint32_t)a.sms));
        k_layer_prep<<<blocks, 256, 0, st>>>(ctl, a.status, nstatus, a.inject_stall ? 1u : 0u,
                                             a.noise ? a.noise_drops : nullptr, a.preclassified);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    if (m_hi > 0) {
        // 1. classify (unless the TopN compaction before this layer listed the partners)
        if (!a.preclassified) {
            const uint32_t tiles = ctiles;
            a.prof->begin(K_CLASSIFY, (double)a.n * 16 * W, st);
            k_classify<W, T><<<tiles, kBlock, 0, st>>>(a.Sk, a.n, a.L, a.idx, a.D, a.status, ctl);
            a.prof->end(st);
            if ((e = cudaGetLastError()) != cudaSuccess) return e;
        }
        // 2-3. level scans (batches of kMaxLevels; one batch of four covers every gate on at
        // most two qubits), scatter on the last batch
        const uint32_t stiles = (uint32_t)((m_hi + kScanTile - 1) / kScanTile);
        // grid-stride kernels over the scan tiles, at most the resident blocks of the apply
        // variant that runs
        static std::atomic<int> level_per_sm[2];
        const int per_sm = a.levels->n <= 4
                               ? resident_blocks(k_level_apply<W, T, 4, kApplyThreads, false>, kApplyThreads, 0,
                                                 level_per_sm[0])
                               : resident_blocks(k_level_apply<W, T, kMaxLevels, kApplyThreads, false>, kApplyThreads,
                                                 0, level_per_sm[1]);
        const uint32_t sgrid = std::min<uint32_t>(stiles, (uint32_t)per_sm * (uint32_t)(a.sms > 0 ? a.sms : 1));
        LevelTile* lt = reinterpret_cast<LevelTile*>(a.slots);
        const bool narrow = a.levels->n <= 4;
        const int per = narrow ? 4 : kMaxLevels;
        int nb = (a.levels->n + per - 1) / per;
        for (int b = 0; b < nb; ++b) {
            Levels lv{};
            lv.n = min(per, a.levels->n - b * per);
            for (int l = 0; l < lv.n; ++l) lv.rank[l] = a.levels->rank[b * per + l];
            const bool last = b == nb - 1;
            // forward and backward scans of this batch of levels; the last batch places the partners
            a.prof->begin(K_LEVEL_SCAN, 0.0, st);
            a.prof->more_launches(K_LEVEL_SCAN, 1);  // reduce and scan
            if (narrow) {
                k_level_reduce<W, 4><<<sgrid, kBlock, 0, st>>>(a.idx, a.D, a.Sk, a.n, lv, lt, ctl);
                k_level_scan<4><<<1, kScanThreads, 0, st>>>(lt, ctl);
            } else {
                k_level_reduce<W, kMaxLevels><<<sgrid, kBlock, 0, st>>>(a.idx, a.D, a.Sk, a.n, lv, lt, ctl);
                k_level_scan<kMaxLevels><<<1, kScanThreads, 0, st>>>(lt, ctl);
            }
            a.prof->end(st);
            if ((e = cudaGetLastError()) != cudaSuccess) return e;
            a.prof->begin(K_LEVEL_APPLY, 0.0, st);
            // the folded noise matters only where the partners are placed (the last batch)
            if (a.noise && last) {
                if (narrow)
                    k_level_apply<W, T, 4, kApplyThreads, true><<<sgrid, kApplyThreads, 0, st>>>(
                        a.idx, a.D, a.F, a.Sk, a.Sc, a.n, lv, a.L, b > 0, last, a.Pk, a.Pc, lt, ctl, a.keep, *a.noise,
                        a.Sf, a.Pf);
                else
                    k_level_apply<W, T, kMaxLevels, kApplyThreads, true><<<sgrid, kApplyThreads, 0, st>>>(
                        a.idx, a.D, a.F, a.Sk, a.Sc, a.n, lv, a.L, b > 0, last, a.Pk, a.Pc, lt, ctl, a.keep, *a.noise,
                        a.Sf, a.Pf);
            } else {
                if (narrow)
                    k_level_apply<W, T, 4, kApplyThreads, false><<<sgrid, kApplyThreads, 0, st>>>(
                        a.idx, a.D, a.F, a.Sk, a.Sc, a.n, lv, a.L, b > 0, last, a.Pk, a.Pc, lt, ctl, a.keep,
                        NoNoise{}, a.Sf, a.Pf);
                else
                    k_level_apply<W, T, kMaxLevels, kApplyThreads, false><<<sgrid, kApplyThreads, 0, st>>>(
                        a.idx, a.D, a.F, a.Sk, a.Sc, a.n, lv, a.L, b > 0, last, a.Pk, a.Pc, lt, ctl, a.keep,
                        NoNoise{}, a.Sf, a.Pf);
            }
            a.prof->end(st);
            if ((e = cudaGetLastError()) != cudaSuccess) return e;
        }
    }
    // 4. partition
    const uint64_t total_hi = a.n + m_hi;
    const uint32_t mtiles_hi = (uint32_t)((total_hi + MT - 1) / MT);
    if (mtiles_hi == 0) {
        *a.partners_out = 0;
        *a.out_count = 0;
        return cudaSuccess;
    }
    if ((a.slot_count ? (uint64_t)mtiles_hi * (MT + 2) : total_hi) > a.out_cap) return cudaErrorMemoryAllocation;
    {
        uint32_t warps = mtiles_hi + 1;
        uint32_t blocks = std::min<uint32_t>((warps + 7) / 8, 8u * (uint32_t)(a.sms > 0 ? a.sms : 1));
        a.prof->begin(K_PARTITION, 0.0, st);
        k_partition<W><<<blocks, 256, 0, st>>>(a.Sk, a.n, a.Pk, (uint32_t)MT, a.bounds, ctl);
        a.prof->end(st);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    // 5. merge (its look-back words and dispenser were reset by k_layer_prep; under failure
    // injection the dispenser starts at tile 1, so tile 0 never publishes and tile 1's bounded
    // look-back gives up)
    const size_t smem = MergeSmem<W, T>::bytes;
    static std::atomic<int> merge_per_sm[4];
    const long long stall = a.inject_stall ? (long long)a.stall_limit : 0ll;
    a.prof->begin(K_MERGE, 0.0, st);
    if (a.noise) {
        const int mper = resident_blocks(k_merge<W, T, true, false>, kBlock, smem, merge_per_sm[1]);
        const uint32_t mgrid = (uint32_t)std::min<uint64_t>(mtiles_hi, (uint64_t)mper * (a.sms > 0 ? a.sms : 1));
        k_merge<W, T, true, false><<<mgrid, kBlock, smem, st>>>(
            a.Sk, a.Sc, a.n, a.Pk, a.Pc, a.bounds, a.L, a.keep, a.Ok, a.Oc, a.out_cap, merge_status, ctl, a.topn_hist,
            a.topn_hist_mode, a.topn_hist_base, a.slot_count, stall, *a.noise, a.noise_drops, nullptr, nullptr, nullptr);
    } else if (a.Sf) {
        const size_t fsmem = smem + MergeSmem<W, T>::f_bytes;
        const int mper = resident_blocks(k_merge<W, T, false, true>, kBlock, fsmem, merge_per_sm[2]);
        const uint32_t mgrid = (uint32_t)std::min<uint64_t>(mtiles_hi, (uint64_t)mper * (a.sms > 0 ? a.sms : 1));
        k_merge<W, T, false, true><<<mgrid, kBlock, fsmem, st>>>(
            a.Sk, a.Sc, a.n, a.Pk, a.Pc, a.bounds, a.L, a.keep, a.Ok, a.Oc, a.out_cap, merge_status, ctl, a.topn_hist,
            a.topn_hist_mode, a.topn_hist_base, a.slot_count, stall, NoNoise{}, nullptr, a.Sf, a.Pf, a.Of);
    } else if (a.next_flags) {
        const int mper = resident_blocks(k_merge<W, T, false, false, true>, kBlock, smem, merge_per_sm[3]);
        const uint32_t mgrid = (uint32_t)std::min<uint64_t>(mtiles_hi, (uint64_t)mper * (a.sms > 0 ? a.sms : 1));
        NextFlagArg<W> nx;
        nx.L = a.next_L;
        nx.flags = a.next_flags;
        k_merge<W, T, false, false, true><<<mgrid, kBlock, smem, st>>>(
            a.Sk, a.Sc, a.n, a.Pk, a.Pc, a.bounds, a.L, a.keep, a.Ok, a.Oc, a.out_cap, merge_status, ctl, a.topn_hist,
            a.topn_hist_mode, a.topn_hist_base, a.slot_count, stall, NoNoise{}, nullptr, nullptr, nullptr, nullptr, nx);
    } else {
        const int mper = resident_blocks(k_merge<W, T, false, false>, kBlock, smem, merge_per_sm[0]);
        const uint32_t mgrid = (uint32_t)std::min<uint64_t>(mtiles_hi, (uint64_t)mper * (a.sms > 0 ? a.sms : 1));
        k_merge<W, T, false, false><<<mgrid, kBlock, smem, st>>>(
            a.Sk, a.Sc, a.n, a.Pk, a.Pc, a.bounds, a.L, a.keep, a.Ok, a.Oc, a.out_cap, merge_status, ctl, a.topn_hist,
            a.topn_hist_mode, a.topn_hist_base, a.slot_count, stall, NoNoise{}, nullptr, nullptr, nullptr, nullptr);
    }
    a.prof->end(st);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if (a.inject_flag) {  // as a failed device check would leave it (stream order: after the kernels)
        *reinterpret_cast<unsigned int*>(a.host_count + 60) = a.inject_flag;  // pinned, otherwise unused
        cudaMemcpyAsync(&ctl->err, a.host_count + 60, sizeof(unsigned int), cudaMemcpyHostToDevice, st);
    }
    if (a.defer_counts) {
        // the caller reads them after the TopN pass's synchronization (and books the bytes then)
        cudaMemcpyAsync(a.defer_counts, &ctl->count[0], offsetof(Ctl, err_info) + sizeof(unsigned int),
                        cudaMemcpyDeviceToHost, st);
        *a.partners_out = 0;
        *a.out_count = 0;
        *a.span_out = (a.n + m_hi + MT - 1) / MT * (uint64_t)(MT + 2);  // a bound: m is not known here
        *a.err_flags = 0;
        *a.err_info = 0;
        return cudaGetLastError();
    }
    // counts and error flags in one copy: count[0..7], tile_counter[0..7], err, err_info
    cudaMemcpyAsync(a.host_count, &ctl->count[0], offsetof(Ctl, err_info) + sizeof(unsigned int),
                    cudaMemcpyDeviceToHost, st);
    if (a.noise)
        cudaMemcpyAsync(a.host_noise_drops, a.noise_drops, (kMaxNoise + 1) * sizeof(unsigned long long),
                        cudaMemcpyDeviceToHost, st);
    if ((e = spin_sync(st)) != cudaSuccess) return e;
    const uint64_t m = a.host_count[0];
    *a.partners_out = m;
    *a.out_count = a.host_count[1];
    if (a.slot_count) *a.span_out = (a.n + m + MT - 1) / MT * (uint64_t)(MT + 2);
    const unsigned int* flags = reinterpret_cast<const unsigned int*>(
        reinterpret_cast<const unsigned char*>(a.host_count) + offsetof(Ctl, err));
    *a.err_flags = flags[0];
    *a.err_info = flags[1];
    book_rotation_bytes<W, T>(a.prof, a.n, m, *a.out_count, a.levels->n, !a.preclassified);
    if (a.next_flags) a.prof->add_bytes(K_MERGE, (double)*a.out_count);  // the partner-test bytes
    return cudaSuccess;
}

// The algorithmic bytes of a rotation layer's kernels, booked once m and the output count are
// known (after the layer's synchronization, or the TopN pass's when the layer did not wait).
template <int W, typename T>
void book_rotation_bytes(KernelProf* prof, uint64_t n, uint64_t m, uint64_t out_count, int nlv, bool classified) {
    constexpr int MT = RotTile<W>::kMergeTile;
    if (classified) prof->add_bytes(K_CLASSIFY, (double)m * 6);  // idx + divergence writes
    const int per = nlv <= 4 ? 4 : kMaxLevels;
    const int nb = m ? (nlv + per - 1) / per : 0;
    for (int b = 0; b < nb; ++b) {
        const bool last = b == nb - 1;
        prof->add_bytes(K_LEVEL_SCAN, (double)m * 2);  // divergence reads
        // divergence reads, earlier batches' F, then F written or (last) index, gather and place
        prof->add_bytes(K_LEVEL_APPLY, (double)m * (2 + (b > 0 ? 4 : 0) + (last ? 4 + 2.0 * (16 * W + sizeof(T)) : 4)));
    }
    prof->add_bytes(K_PARTITION, (double)((n + m + MT - 1) / MT + 1) * 16);
    prof->add_bytes(K_MERGE, (double)(n + m + out_count) * (16 * W + sizeof(T)));
}

template <int W>
uint32_t merge_slot_rows() {
    return (uint32_t)RotTile<W>::kMergeTile + 2;
}
template <int W>
uint64_t merge_span_rows(uint64_t rows_in) {
    return (rows_in + RotTile<W>::kMergeTile - 1) / RotTile<W>::kMergeTile * (uint64_t)merge_slot_rows<W>();
}
template uint32_t merge_slot_rows<1>();
template uint32_t merge_slot_rows<2>();
template uint32_t merge_slot_rows<4>();
template uint64_t merge_span_rows<1>(uint64_t);
template uint64_t merge_span_rows<2>(uint64_t);
template uint64_t merge_span_rows<4>(uint64_t);

template <int W, typename T>
cudaError_t configure_rotation_kernels() {
    cudaError_t e = cudaSuccess;
    const void* kernels[4] = {(const void*)k_merge<W, T, false, false>, (const void*)k_merge<W, T, true, false>,
                              (const void*)k_merge<W, T, false, true>, (const void*)k_merge<W, T, false, false, true>};
    for (const void* k : kernels) {
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)(MergeSmem<W, T>::bytes + MergeSmem<W, T>::f_bytes));
        // all of the unified L1 as shared memory, so residency is set by registers, not the carveout
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout,
                                     (int)cudaSharedmemCarveoutMaxShared);
    }
    return e;
}

#define PS_INSTANTIATE_ROT(W, T)                                                                 \
    template cudaError_t launch_rotation_layer<W, T>(const RotationArgs<W, T>&, cudaStream_t); \
    template void book_rotation_bytes<W, T>(KernelProf*, uint64_t, uint64_t, uint64_t, int, bool); \
    template cudaError_t configure_rotation_kernels<W, T>();

PS_INSTANTIATE_ROT(1, double)
PS_INSTANTIATE_ROT(1, float)
PS_INSTANTIATE_ROT(2, double)
PS_INSTANTIATE_ROT(2, float)
PS_INSTANTIATE_ROT(4, double)
PS_INSTANTIATE_ROT(4, float)

}  // namespace psb
