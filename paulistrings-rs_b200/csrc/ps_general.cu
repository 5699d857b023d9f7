// ps_general.cu -- the branch stage of a general-table layer (the sort path).
//
// A general local table (a two-qubit Clifford permutation, a dense unitary PTM, ...) sends
// each input term to the records of its support pattern s: (key ^ mask_e, c * a_e[s]) for
// every entry e whose amplitude at s is nonzero, in ascending entry order (DeltaEntry::emit,
// crates/paulistrings/src/channel/prepared.rs:50-68).  k_gen_branch writes the records in
// (term, entry) order with their own index as the sort value, so the stable LSD radix sort
// that follows and the run-summing dedup after it add each output key's contributions in the
// order the naive layer adds them (crates/paulistrings/src/test_support/oracle.rs:21-54):
// the result is bit-identical to it, sums of three or more contributions included.
//
//   k_gen_count    records the layer emits: one pass over the keys, a 16-entry count table
//   k_gen_branch   warp-striped rows, per-warp shuffle scan of the record counts, block scan,
//                  decoupled look-back across tiles, then every row writes its records
#include "ps_device.cuh"
#include "ps_kernels.h"

namespace psb {
namespace {

constexpr int kGenThreads = 256;

template <int W>
__host__ __device__ constexpr int gen_items() {
    return W == 4 ? 4 : 8;
}

template <int W, typename T>
__device__ __forceinline__ uint32_t gen_pattern(const GenLayer<W, T>& G, const uint64_t* __restrict__ k) {
    uint32_t s = (uint32_t)((k[G.qw[0]] >> G.qb[0]) & 1u) | (uint32_t)((k[W + G.qw[0]] >> G.qb[0]) & 1u) << 1 |
                 (uint32_t)((k[G.qw[1]] >> G.qb[1]) & 1u) << 2 | (uint32_t)((k[W + G.qw[1]] >> G.qb[1]) & 1u) << 3;
    return s & G.pattern_mask;
}

template <int W, typename T>
__global__ void __launch_bounds__(kGenThreads) k_gen_count(const uint64_t* __restrict__ keys, uint64_t n,
                                                           const GenLayer<W, T> G, Ctl* ctl) {
    __shared__ unsigned int s_cnt[16];
    __shared__ unsigned long long s_sum[kGenThreads / 32];
    if (threadIdx.x < 16) s_cnt[threadIdx.x] = G.cnt[threadIdx.x];
    __syncthreads();
    unsigned long long acc = 0;
    for (uint64_t r = (uint64_t)blockIdx.x * kGenThreads + threadIdx.x; r < n; r += (uint64_t)gridDim.x * kGenThreads)
        acc += s_cnt[gen_pattern<W, T>(G, keys + r * 2 * W)];
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, d);
    if ((threadIdx.x & 31) == 0) s_sum[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long t = 0;
        for (int w = 0; w < kGenThreads / 32; ++w) t += s_sum[w];
        if (t) atomicAdd(&ctl->count[6], t);
    }
}

template <int W, typename T>
__global__ void __launch_bounds__(kGenThreads) k_gen_branch(const uint64_t* __restrict__ keys,
                                                            const T* __restrict__ coef, uint64_t n,
                                                            const GenLayer<W, T> G, uint64_t* __restrict__ rkeys,
                                                            uint32_t* __restrict__ rvals, T* __restrict__ rcoef,
                                                            uint64_t m_cap, unsigned long long* status, Ctl* ctl) {
    constexpr int ITEMS = gen_items<W>();
    constexpr int TILE = kGenThreads * ITEMS;
    __shared__ T s_amp[16][16];
    __shared__ uint8_t s_ent[16][16];
    __shared__ unsigned int s_cnt[16];
    __shared__ uint64_t s_mask[16][2 * W];
    __shared__ unsigned int s_tile;
    __shared__ unsigned int s_warp[kGenThreads / 32];
    __shared__ unsigned long long s_off;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int i = tid; i < 256; i += kGenThreads) {
        s_amp[i >> 4][i & 15] = G.amp[i >> 4][i & 15];
        s_ent[i >> 4][i & 15] = G.ent[i >> 4][i & 15];
    }
    if (tid < 16) s_cnt[tid] = G.cnt[tid];
    for (int i = tid; i < 16 * 2 * W; i += kGenThreads) {
        const int e = i / (2 * W), w = i % (2 * W);
        s_mask[e][w] = w < W ? G.mx[e][w] : G.mz[e][w - W];
    }
    if (tid == 0) s_tile = atomicAdd(&ctl->tile_counter[7], 1u);
    __syncthreads();
    const unsigned int tile = s_tile;
    const uint64_t wbase = (uint64_t)tile * TILE + (uint64_t)warp * 32 * ITEMS;

    // record counts in row order (row = wbase + 32 i + lane), scanned per warp
    uint32_t pat[ITEMS];
    unsigned int excl[ITEMS];
    unsigned int run = 0;
#pragma unroll
    for (int i = 0; i < ITEMS; ++i) {
        const uint64_t row = wbase + (uint64_t)i * 32 + lane;
        unsigned int c = 0;
        pat[i] = 0;
        if (row < n) {
            pat[i] = gen_pattern<W, T>(G, keys + row * 2 * W);
            c = s_cnt[pat[i]];
        }
        unsigned int x = c;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const unsigned int y = __shfl_up_sync(0xffffffffu, x, d);
            if (lane >= d) x += y;
        }
        excl[i] = run + x - c;
        run += __shfl_sync(0xffffffffu, x, 31);
    }
    unsigned int total;
    const unsigned int wx = block_exclusive_sum<kGenThreads>(lane == 31 ? run : 0u, s_warp, total);
    const unsigned int warp_off = __shfl_sync(0xffffffffu, wx, 31);
    if (tid < 32) {
        unsigned long long p = 0;
        if (tile == 0) {
            if (tid == 0) st_release_u64(status + tile, kFlagInc | (unsigned long long)total);
        } else {
            if (tid == 0) st_release_u64(status + tile, kFlagAgg | (unsigned long long)total);
            p = lookback_sum_warp(status, tile, ctl, 801);
            if (tid == 0) st_release_u64(status + tile, kFlagInc | (p + total));
        }
        if (tid == 0) {
            s_off = p;
            if ((uint64_t)(tile + 1) * TILE >= n) ctl->count[7] = p + total;
        }
    }
    __syncthreads();
    const unsigned long long base = s_off + warp_off;
#pragma unroll
    for (int i = 0; i < ITEMS; ++i) {
        const uint64_t row = wbase + (uint64_t)i * 32 + lane;
        if (row >= n) continue;
        const uint32_t s = pat[i];
        const unsigned int c = s_cnt[s];
        if (!c) continue;
        const unsigned long long o = base + excl[i];
        if (!PS_GUARD(ctl, o + c <= m_cap, 802)) continue;
        uint64_t k[2 * W];
        load_key<W>(keys, row, k);
        const T v = coef[row];
        for (unsigned int j = 0; j < c; ++j) {
            const int e = s_ent[s][j];
            uint64_t out[2 * W];
#pragma unroll
            for (int w = 0; w < 2 * W; ++w) out[w] = k[w] ^ s_mask[e][w];
            store_key<W>(rkeys, o + j, out);
            rvals[o + j] = (uint32_t)(o + j);
            rcoef[o + j] = mul_rn(v, s_amp[s][j]);
        }
    }
}

inline unsigned int gen_grid(uint64_t n, int sms) {
    uint64_t blocks = (n + kGenThreads - 1) / kGenThreads;
    const uint64_t cap = (uint64_t)sms * 8;
    if (blocks > cap) blocks = cap;
    return (unsigned int)(blocks ? blocks : 1);
}

}  // namespace

template <int W, typename T>
size_t GeneralOps<W, T>::branch_tile() {
    return (size_t)kGenThreads * gen_items<W>();
}

template <int W, typename T>
cudaError_t GeneralOps<W, T>::count(const uint64_t* keys, uint64_t n, const GenLayer<W, T>& G, Ctl* ctl,
                                    unsigned long long* host_count, uint64_t* m, int sms, cudaStream_t st,
                                    KernelProf* prof) {
    cudaMemsetAsync(&ctl->count[6], 0, sizeof(unsigned long long), st);
    prof->begin(K_GEN_COUNT, (double)n * 16 * W, st);
    if (n) k_gen_count<W, T><<<gen_grid(n, sms), kGenThreads, 0, st>>>(keys, n, G, ctl);
    prof->end(st);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    cudaMemcpyAsync(host_count, &ctl->count[6], sizeof(unsigned long long), cudaMemcpyDeviceToHost, st);
    if ((e = spin_sync(st)) != cudaSuccess) return e;
    *m = *host_count;
    return cudaSuccess;
}

template <int W, typename T>
cudaError_t GeneralOps<W, T>::branch(const uint64_t* keys, const T* coef, uint64_t n, const GenLayer<W, T>& G,
                                     uint64_t* rkeys, uint32_t* rvals, T* rcoef, uint64_t m_cap,
                                     unsigned long long* status, Ctl* ctl, cudaStream_t st, KernelProf* prof) {
    if (!n) return cudaSuccess;
    const uint64_t tiles = (n + branch_tile() - 1) / branch_tile();
    cudaMemsetAsync(status, 0, (size_t)tiles * sizeof(unsigned long long), st);
    cudaMemsetAsync(&ctl->tile_counter[7], 0, sizeof(unsigned int), st);
    prof->begin(K_GEN_BRANCH, (double)n * (16 * W + sizeof(T)) + (double)m_cap * (16 * W + 4 + sizeof(T)), st);
    k_gen_branch<W, T><<<(unsigned int)tiles, kGenThreads, 0, st>>>(keys, coef, n, G, rkeys, rvals, rcoef, m_cap,
                                                                     status, ctl);
    prof->end(st);
    return cudaGetLastError();
}

template struct GeneralOps<1, double>;
template struct GeneralOps<2, double>;
template struct GeneralOps<4, double>;
template struct GeneralOps<1, float>;
template struct GeneralOps<2, float>;
template struct GeneralOps<4, float>;

}  // namespace psb
