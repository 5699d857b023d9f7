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
//   k_topn_hist/_step/_compact
//                          TopN by 8-bit radix-select on the bit pattern of |c|^2 (NaN lowest),
//                          then an order-preserving compaction keeping everything above the
//                          boundary and the first `quota` boundary ties in key order
//                          (TopN::finalize_layer, crates/paulistrings/src/truncation/builtin.rs:73-129)
//   k_expect_*             <psi|O|psi> in a product state, float64 partial sums reduced in a
//                          fixed order (readout/product_state.rs:84-101)
#include "ps_device.cuh"
#include "ps_store.h"

namespace psb {

constexpr int kThreads = 256;

// ---------------------------------------------------------------------------
// pack / unpack
// ---------------------------------------------------------------------------
template <int W, typename T>
__global__ void k_pack(const uint64_t* __restrict__ x, const uint64_t* __restrict__ z, const double* __restrict__ c,
                       uint64_t n, uint32_t num_qubits, uint64_t* __restrict__ keys, T* __restrict__ coef,
                       uint32_t* __restrict__ vals, Ctl* ctl) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t k[2 * W];
        uint64_t leak = 0;
#pragma unroll
        for (int w = 0; w < W; ++w) {
            k[w] = x[i * W + w];
            k[W + w] = z[i * W + w];
            uint32_t first = 64u * w;
            uint64_t live = num_qubits >= first + 64 ? ~0ull : (num_qubits <= first ? 0ull : ((1ull << (num_qubits - first)) - 1));
            leak |= (k[w] | k[W + w]) & ~live;
        }
        if (leak) raise_err(ctl, ERR_KEY_RANGE, 401);
        store_key<W>(keys, i, k);
        coef[i] = (T)c[i];
        vals[i] = (uint32_t)i;
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
                    if (++spins > kSpinLimit) {
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
// TopN radix-select on |c|^2 bits
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ uint64_t mag_key(T c) {
    double v = to_f64(c);
    double m = __dmul_rn(v, v);
    if (isnan(m)) return 0ull;  // NaN sorts below every number and is never kept
    return (uint64_t)__double_as_longlong(m) + 1ull;
}

template <typename T>
__global__ void __launch_bounds__(kThreads) k_topn_hist(const T* __restrict__ coef, uint64_t n, int byte,
                                                        Ctl* ctl, unsigned int* __restrict__ hist) {
    __shared__ unsigned int sh[256];
    sh[threadIdx.x] = 0;
    __syncthreads();
    const uint64_t prefix = ctl->aux[0], mask = ctl->aux[1];
    for (uint64_t i = blockIdx.x * (uint64_t)kThreads + threadIdx.x; i < n; i += (uint64_t)gridDim.x * kThreads) {
        uint64_t mk = mag_key<T>(coef[i]);
        if ((mk & mask) == prefix) atomicAdd(&sh[(mk >> (8 * byte)) & 0xFFu], 1u);
    }
    __syncthreads();
    if (sh[threadIdx.x]) atomicAdd(&hist[threadIdx.x], sh[threadIdx.x]);
}

// aux[0] prefix, aux[1] mask, aux[2] remaining rank (1-based, among prefix matches),
// aux[3] count strictly above the prefix so far.
__global__ void k_topn_step(unsigned int* __restrict__ hist, int byte, Ctl* ctl) {
    __shared__ unsigned int sh[256];
    const int b = threadIdx.x;
    sh[b] = hist[b];
    hist[b] = 0;
    __syncthreads();
    if (b == 0) {
        unsigned long long r = ctl->aux[2];
        unsigned long long above = 0;
        int chosen = 0;
        for (int q = 255; q >= 0; --q) {
            unsigned long long c = sh[q];
            if (above + c >= r) {
                chosen = q;
                break;
            }
            above += c;
        }
        ctl->aux[0] |= (unsigned long long)chosen << (8 * byte);
        ctl->aux[1] |= 0xFFull << (8 * byte);
        ctl->aux[2] = r - above;
        ctl->aux[3] += above;
    }
}

template <int W, typename T>
__global__ void __launch_bounds__(kThreads) k_topn_compact(const uint64_t* __restrict__ keys, const T* __restrict__ coef,
                                                           uint64_t n, unsigned long long quota,
                                                           uint64_t* __restrict__ okeys, T* __restrict__ ocoef,
                                                           unsigned long long* status, Ctl* ctl) {
    constexpr int ITEMS = 8;
    __shared__ unsigned int s_tile;
    __shared__ unsigned int s_warp[kThreads / 32];
    __shared__ unsigned long long s_above, s_ties;
    const int tid = threadIdx.x;
    if (tid == 0) s_tile = atomicAdd(&ctl->tile_counter[6], 1u);
    __syncthreads();
    const unsigned int tile = s_tile;
    const uint64_t boundary = ctl->aux[0];
    const uint64_t e0 = (uint64_t)tile * (kThreads * ITEMS) + (uint64_t)tid * ITEMS;
    uint32_t amask = 0, tmask = 0;
#pragma unroll
    for (int i = 0; i < ITEMS; ++i) {
        uint64_t e = e0 + i;
        if (e >= n) continue;
        uint64_t mk = mag_key<T>(coef[e]);
        if (mk > boundary) amask |= 1u << i;
        else if (mk == boundary && boundary != 0) tmask |= 1u << i;
    }
    unsigned int ta, tt;
    unsigned int ea = block_exclusive_sum<kThreads>(__popc(amask), s_warp, ta);
    unsigned int et = block_exclusive_sum<kThreads>(__popc(tmask), s_warp, tt);
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
            if ((uint64_t)(tile + 1) * (kThreads * ITEMS) >= n) {
                unsigned long long tot_ties = s_ties + tt;
                ctl->count[3] = s_above + ta + (tot_ties < quota ? tot_ties : quota);
            }
        }
    }
    __syncthreads();
    unsigned long long arank = s_above + ea, trank = s_ties + et;
#pragma unroll
    for (int i = 0; i < ITEMS; ++i) {
        bool isa = (amask >> i) & 1u, ist = (tmask >> i) & 1u;
        if (!isa && !ist) continue;
        bool keepit = isa || trank < quota;
        unsigned long long tie_before = trank < quota ? trank : quota;
        unsigned long long pos = arank + tie_before;
        if (keepit) {
            uint64_t k[2 * W];
            load_key<W>(keys, e0 + i, k);
            if (PS_GUARD(ctl, pos < n, 702)) {
                store_key<W>(okeys, pos, k);
                ocoef[pos] = coef[e0 + i];
            }
        }
        if (isa) ++arank;
        if (ist) ++trank;
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

template <int W, typename T>
cudaError_t StoreOps<W, T>::pack(const uint64_t* x, const uint64_t* z, const double* c, uint64_t n, uint32_t nq,
                                 uint64_t* keys, T* coef, uint32_t* vals, Ctl* ctl, int sms, cudaStream_t st,
                                 KernelProf* prof) {
    if (!n) return cudaSuccess;
    prof->begin(K_PACK, (double)n * (16 * W + 8 + 16 * W + sizeof(T) + 4), st);
    k_pack<W, T><<<grid_for(n, sms), kThreads, 0, st>>>(x, z, c, n, nq, keys, coef, vals, ctl);
    prof->end(st);
    return cudaGetLastError();
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
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return e;
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
    return cudaStreamSynchronize(st);
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
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return e;
    *out_n = *host_count;
    prof->add_bytes(K_DEDUP, (double)*out_n * (16 * W + sizeof(T)));
    return cudaSuccess;
}

template <int W, typename T>
cudaError_t StoreOps<W, T>::topn(const uint64_t* keys, const T* coef, uint64_t n, uint64_t keep_n, uint64_t* okeys,
                                 T* ocoef, unsigned int* hist, unsigned long long* status, Ctl* ctl,
                                 unsigned long long* host_count, uint64_t* out_n, int sms, cudaStream_t st,
                                 KernelProf* prof) {
    // aux: prefix, mask, remaining rank, above
    unsigned long long init[4] = {0ull, 0ull, (unsigned long long)keep_n, 0ull};
    cudaMemcpyAsync(ctl->aux, init, sizeof(init), cudaMemcpyHostToDevice, st);
    cudaMemsetAsync(hist, 0, 256 * sizeof(unsigned int), st);
    cudaError_t e;
    for (int byte = 7; byte >= 0; --byte) {
        prof->begin(K_TOPN_HIST, (double)n * sizeof(T), st);
        k_topn_hist<T><<<grid_for(n, sms), kThreads, 0, st>>>(coef, n, byte, ctl, hist);
        prof->end(st);
        prof->begin(K_TOPN_STEP, 2048.0, st);
        k_topn_step<<<1, 256, 0, st>>>(hist, byte, ctl);
        prof->end(st);
    }
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    unsigned long long aux[4];
    cudaMemcpyAsync(aux, ctl->aux, sizeof(aux), cudaMemcpyDeviceToHost, st);
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return e;
    unsigned long long quota = keep_n - aux[3];
    if (aux[0] == 0) quota = 0;  // NaN boundary: only the non-NaN terms stay
    const uint32_t tiles = (uint32_t)((n + kThreads * 8 - 1) / (kThreads * 8));
    cudaMemsetAsync(status, 0, (size_t)tiles * sizeof(unsigned long long), st);
    cudaMemsetAsync(&ctl->tile_counter[6], 0, sizeof(unsigned int), st);
    prof->begin(K_TOPN_COMPACT, (double)n * sizeof(T), st);
    k_topn_compact<W, T><<<tiles, kThreads, 0, st>>>(keys, coef, n, quota, okeys, ocoef, status, ctl);
    prof->end(st);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    cudaMemcpyAsync(host_count, &ctl->count[3], sizeof(unsigned long long), cudaMemcpyDeviceToHost, st);
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return e;
    *out_n = *host_count;
    prof->add_bytes(K_TOPN_COMPACT, (double)*out_n * 2 * (16 * W + sizeof(T)));
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
