// ps_scorer.cu -- the learned truncation scorer on the tcgen05 tensor cores.
//
// The scorer is a small MLP over one term: a one-hot I/X/Y/Z code per qubit and three scalar
// features (Pauli weight, log|c|, remaining depth) -> 128 -> GELU -> 128 -> GELU -> 1, with
// BF16 weights and FP32 accumulation.  The one-hot first layer is an embedding bag: the
// hidden pre-activation is b1 + the scalar features times their input columns + the embedding
// rows of the term's non-identity qubits (the identity columns fold into b1).  The second
// layer is a 128 x 128 GEMM per tile of 128 terms on the tensor cores: the tile's
// activations (operand A, 128 terms x 128) and the weight (operand B, 128 x 128) sit in shared
// memory in the canonical K-major layout without swizzle (8-row x 16-byte core matrices), one
// thread issues eight tcgen05.mma kind::f16 (M = N = 128, K = 16 each) into a 128-column
// TMEM accumulator, tcgen05.commit arrives on an mbarrier, and each of the four warps reads
// its 32 TMEM lanes (32 terms) back with tcgen05.ld for the GELU and the output dot product.
// Training adds the two backward GEMMs (dW2 = h1^T dz2 accumulated across a block's tiles in
// TMEM, dh1 = dz2 W2^T) and Adam on fp32 master weights.
//
// Every mbarrier wait is bounded; a block whose wait gives up records ERR_TIMEOUT, stops
// issuing, frees its TMEM and returns.
#include <algorithm>
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "ps_device.cuh"
#include "ps_scorer.h"
#include "ps_store.h"

namespace psb {
namespace {

constexpr int kScoreThreads = 128;   // one warpgroup: warp w owns TMEM lanes 32w .. 32w + 31
constexpr uint32_t kTileBytes = kScoreTile * kHid * 2;  // one bf16 128 x 128 operand

// instruction descriptor: kind::f16, D f32 (bit 4), A bf16 (bits 7-9), B bf16 (bits 10-12),
// both K-major, N >> 3 at bits 17-22, M >> 4 at bits 24-28
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(kHid >> 3) << 17) |
                            ((uint32_t)(kScoreTile >> 4) << 24);

__device__ __forceinline__ float bf2f(uint16_t b) { return __uint_as_float((uint32_t)b << 16); }
__device__ __forceinline__ uint16_t f2bf(float f) { return __bfloat16_as_ushort(__float2bfloat16_rn(f)); }
__device__ __forceinline__ uint32_t pack2(float a, float b) { return (uint32_t)f2bf(a) | ((uint32_t)f2bf(b) << 16); }

// Byte offset of element (row, k) of a 128 x 128 bf16 operand in the K-major no-swizzle
// canonical layout: core matrix (row / 8, k / 8) at (row / 8) * 2048 + (k / 8) * 128, its eight
// 16-byte rows contiguous.  The descriptor's leading byte offset (next core matrix along K) is
// 128 and its stride byte offset (next 8-row group) is 2048.
__device__ __forceinline__ uint32_t kmaj_off(int row, int k) {
    return (uint32_t)((row >> 3) * 2048 + (k >> 3) * 128 + (row & 7) * 16 + (k & 7) * 2);
}

__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t sbo = 2048u) {
    uint64_t d = (uint64_t)((saddr & 0x3FFFFu) >> 4);  // start address, bits 0-13
    d |= (uint64_t)(128u >> 4) << 16;                   // leading byte offset, bits 16-29
    d |= (uint64_t)(sbo >> 4) << 32;                    // stride byte offset, bits 32-45
    d |= (uint64_t)1 << 46;                             // descriptor version 1 (sm_100)
    return d;                                           // base offset 0, no swizzle
}

// kind::f16 with A and B both f16 (bits 7-12 zero): the inference kernel's second layer
constexpr uint32_t kIdescF16 = (1u << 4) | ((uint32_t)(kHid >> 3) << 17) | ((uint32_t)(kScoreTile >> 4) << 24);

// D (TMEM, 128 lanes x 128 f32 columns) (+)= A (128 x 128) * B^T, A and B K-major in shared
// memory.  K-step j starts 2 core matrices (256 bytes) further along K.
__device__ __forceinline__ void umma_tile(uint32_t d_tmem, uint32_t a_saddr, uint32_t b_saddr, bool accumulate,
                                          uint32_t idesc = kIdesc) {
    const uint64_t ad = umma_desc(a_saddr), bd = umma_desc(b_saddr);
#pragma unroll
    for (int j = 0; j < kHid / 16; ++j) {
        const uint32_t acc = (j > 0 || accumulate) ? 1u : 0u;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
            ::"r"(d_tmem), "l"(ad + 16ull * j), "l"(bd + 16ull * j), "r"(idesc), "r"(acc));
    }
}

__device__ __forceinline__ void umma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void tmem_alloc(uint32_t* dst, uint32_t cols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst)), "r"(cols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t cols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(cols) : "memory");
}

// 32 consecutive f32 columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// GELU, tanh form (Hendrycks & Gimpel 2016), and its derivative.  tanh is the hardware's
// single-instruction approximation (PTX tanh.approx.f32, maximum relative error about 2^-11):
// one SFU operation per hidden unit instead of a libm evaluation, which was the scorer's
// bottleneck; the network's inputs and weights are bf16, so 2^-11 is below their rounding.
constexpr float kGeluS = 0.7978845608028654f;  // sqrt(2 / pi)
constexpr float kGeluA = 0.044715f;
__device__ __forceinline__ float tanh_hw(float x) {
    float y;
    asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float gelu(float x) {
    const float t = tanh_hw(kGeluS * (x + kGeluA * x * x * x));
    return 0.5f * x * (1.0f + t);
}
__device__ __forceinline__ float gelu_grad(float x) {
    const float x2 = x * x;
    const float t = tanh_hw(kGeluS * (x + kGeluA * x2 * x));
    return 0.5f * (1.0f + t) + 0.5f * x * (1.0f - t * t) * kGeluS * (1.0f + 3.0f * kGeluA * x2);
}

// The inference kernel's GELU on two f16 lanes at once: tanh.approx.f16x2 and packed f16
// arithmetic (6 instructions per pair).  Its results feed an f16 operand (11 significant
// bits, finer than the bf16 operand of the other paths).  Beyond |x| ~ 40 the cube overflows
// to +-inf, where tanh gives +-1 and the GELU its exact limits x and 0.
__device__ __forceinline__ __half2 tanh_h2(__half2 x) {
    uint32_t in = *reinterpret_cast<uint32_t*>(&x), out;
    asm("tanh.approx.f16x2 %0, %1;" : "=r"(out) : "r"(in));
    return *reinterpret_cast<__half2*>(&out);
}
__device__ __forceinline__ __half2 gelu_h2(__half2 x) {
    const __half2 s = __float2half2_rn(kGeluS), sa = __float2half2_rn(kGeluS * kGeluA), h = __float2half2_rn(0.5f);
    const __half2 x2 = __hmul2(x, x);
    const __half2 u = __hmul2(x, __hfma2(x2, sa, s));
    const __half2 hx = __hmul2(x, h);
    return __hfma2(hx, tanh_h2(u), hx);
}
__device__ __forceinline__ uint32_t h2_bits(__half2 v) { return *reinterpret_cast<uint32_t*>(&v); }

// Column sums of a warp's 32 x 32 block: lane l holds row l's 32 values on entry and the sum
// of column l on exit (v[0]); 31 shuffles.
__device__ __forceinline__ float warp_column_sum(float (&v)[32]) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int s = 16; s >= 1; s >>= 1) {
        const bool upper = (lane & s) != 0;
#pragma unroll
        for (int i = 0; i < s; ++i) {
            const float send = upper ? v[i] : v[i + s];
            const float keep = upper ? v[i + s] : v[i];
            v[i] = keep + __shfl_xor_sync(0xffffffffu, send, s);
        }
    }
    return v[0];
}

template <int W>
__device__ __forceinline__ float term_features(const ScorerArgs& A, const ScoreInput& in, uint64_t row, bool valid,
                                               uint64_t (&k)[2 * W], float (&f)[3]) {
#pragma unroll
    for (int i = 0; i < 2 * W; ++i) k[i] = 0;
    f[0] = f[1] = f[2] = 0.0f;
    if (!valid) return 0.0f;
    load_key<W>(in.keys, row, k);
    int weight = 0;
#pragma unroll
    for (int w = 0; w < W; ++w) weight += __popcll(k[w] | k[W + w]);
    float logc;
    if (in.logc)
        logc = in.logc[row];
    else if (in.coef64)
        logc = (float)log(fabs(in.coef64[row]));
    else
        logc = logf(fabsf(in.coef32[row]));
    logc = fmaxf(logc, -200.0f);  // a zero coefficient must not feed -inf into the network
    const float rem = in.rem ? in.rem[row] : in.rem_uniform;
    f[0] = (float)weight * A.fscale[0];
    f[1] = logc * A.fscale[1];
    f[2] = rem * A.fscale[2];
    return logc;
}

__device__ __forceinline__ void load_bf16x32(const uint16_t* p, float (&v)[32]) {
    const uint4* q = reinterpret_cast<const uint4*>(p);
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const uint4 u = __ldg(q + i);
        const uint32_t w[4] = {u.x, u.y, u.z, u.w};
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            v[8 * i + 2 * j] = __uint_as_float(w[j] << 16);
            v[8 * i + 2 * j + 1] = __uint_as_float(w[j] & 0xFFFF0000u);
        }
    }
}

// Hidden pre-activation z1 for hidden units [32 c, 32 c + 32): b1 + f . u, then the embedding
// rows of the non-identity qubits in ascending qubit order.
template <int W>
__device__ __forceinline__ void z1_chunk(const ScorerArgs& A, const uint64_t (&k)[2 * W], const float (&f)[3], int c,
                                         float (&z)[32]) {
    float b[32], u0[32], u1[32], u2[32];
    load_bf16x32(A.p + A.L.b1 + 32 * c, b);
    load_bf16x32(A.p + A.L.u + 32 * c, u0);
    load_bf16x32(A.p + A.L.u + kHid + 32 * c, u1);
    load_bf16x32(A.p + A.L.u + 2 * kHid + 32 * c, u2);
#pragma unroll
    for (int j = 0; j < 32; ++j) z[j] = b[j] + f[0] * u0[j] + f[1] * u1[j] + f[2] * u2[j];
#pragma unroll
    for (int w = 0; w < W; ++w) {
        uint64_t live = k[w] | k[W + w];
        while (live) {
            const int bit = __ffsll((long long)live) - 1;
            live &= live - 1;
            const int q = A.site_row ? (int)A.site_row[64 * w + bit] : 64 * w + bit;
            if (q < 0) continue;
            const int p = (int)((k[w] >> bit) & 1u) | ((int)((k[W + w] >> bit) & 1u) << 1);
            float e[32];
            load_bf16x32(A.p + A.L.embed + ((size_t)q * 3 + (size_t)(p - 1)) * kHid + 32 * c, e);
#pragma unroll
            for (int j = 0; j < 32; ++j) z[j] += e[j];
        }
    }
}

// Write 32 bf16 values of row `row`, columns [32 c, 32 c + 32), into a K-major operand.
__device__ __forceinline__ void store_row_chunk(uint8_t* op, int row, int c, const float (&h)[32]) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        uint4 u;
        u.x = pack2(h[8 * q + 0], h[8 * q + 1]);
        u.y = pack2(h[8 * q + 2], h[8 * q + 3]);
        u.z = pack2(h[8 * q + 4], h[8 * q + 5]);
        u.w = pack2(h[8 * q + 6], h[8 * q + 7]);
        *reinterpret_cast<uint4*>(op + kmaj_off(row, 32 * c + 8 * q)) = u;
    }
}


// Shared prologue: B operand from w2 (transposed for the forward GEMM: element (out, in) = w2[in][out];
// as stored for dh1 = dz2 W2^T: element (in, out) = w2[in][out]).
__device__ __forceinline__ void stage_w2(const ScorerArgs& A, uint8_t* sB, bool transposed) {
    const uint16_t* w2 = A.p + A.L.w2;
    for (int i = threadIdx.x; i < kHid * kHid; i += blockDim.x) {
        const int r = i / kHid, c = i % kHid;  // w2[r][c], r = in, c = out
        *reinterpret_cast<uint16_t*>(sB + (transposed ? kmaj_off(c, r) : kmaj_off(r, c))) = w2[i];
    }
}

// ---------------------------------------------------------------------------
// inference (the scored TopN pass) and the training forward
// ---------------------------------------------------------------------------
template <int W, bool TRAIN>
__global__ void __launch_bounds__(kScoreThreads) k_score(const ScorerArgs A, const ScoreInput in,
                                                         float* __restrict__ scores, uint64_t* __restrict__ sel,
                                                         unsigned int* __restrict__ hist, const float* __restrict__ target,
                                                         float inv_batch, TrainScratch S, float* __restrict__ grads,
                                                         float* __restrict__ loss, Ctl* ctl, float* __restrict__ fout) {
    extern __shared__ __align__(128) uint8_t smem[];
    uint8_t* sA = smem;
    uint8_t* sB = smem + kTileBytes;
    float* s_b2 = reinterpret_cast<float*>(smem + 2 * kTileBytes);
    float* s_w3 = s_b2 + kHid;
    float* s_acc = s_w3 + kHid;  // TRAIN: db2[128], dw3[128], db3, loss
    unsigned int* s_hist = reinterpret_cast<unsigned int*>(s_acc + 2 * kHid + 2);
    __shared__ __align__(8) uint64_t s_bar;
    __shared__ uint32_t s_tmem;
    const int tid = threadIdx.x, warp = tid >> 5;

    stage_w2(A, sB, true);
    for (int i = tid; i < kHid; i += kScoreThreads) {
        s_b2[i] = bf2f(A.p[A.L.b2 + i]);
        s_w3[i] = bf2f(A.p[A.L.w3 + i]);
    }
    if (TRAIN)
        for (int i = tid; i < 2 * kHid + 2; i += kScoreThreads) s_acc[i] = 0.0f;
    if (hist)
        for (int i = tid; i < kTopnBins1; i += kScoreThreads) s_hist[i] = 0;
    const float b3 = bf2f(A.p[A.L.b3]);
    if (tid == 0) mbar_init(&s_bar, 1);
    if (warp == 0) tmem_alloc(&s_tmem, kHid);
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = s_tmem;
    const uint32_t lane_base = (uint32_t)(warp * 32) << 16;

    const uint64_t ntiles = (in.n + kScoreTile - 1) / kScoreTile;
    uint32_t phase = 0;
    for (uint64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const uint64_t row = tile * kScoreTile + tid;
        const bool valid = row < in.n;
        uint64_t k[2 * W];
        float f[3];
        const float logc = term_features<W>(A, in, row, valid, k, f);
#pragma unroll 1
        for (int c = 0; c < kHid / 32; ++c) {
            float z[32], h[32];
            z1_chunk<W>(A, k, f, c, z);
#pragma unroll
            for (int j = 0; j < 32; ++j) h[j] = gelu(z[j]);
            store_row_chunk(sA, tid, c, h);
            if (TRAIN && valid) {
                uint4* dh = reinterpret_cast<uint4*>(S.h1 + row * kHid + 32 * c);
                uint4* dg = reinterpret_cast<uint4*>(S.gz1 + row * kHid + 32 * c);
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    dh[q] = make_uint4(pack2(h[8 * q], h[8 * q + 1]), pack2(h[8 * q + 2], h[8 * q + 3]),
                                       pack2(h[8 * q + 4], h[8 * q + 5]), pack2(h[8 * q + 6], h[8 * q + 7]));
                    float g[8];
#pragma unroll
                    for (int j = 0; j < 8; ++j) g[j] = gelu_grad(z[8 * q + j]);
                    dg[q] = make_uint4(pack2(g[0], g[1]), pack2(g[2], g[3]), pack2(g[4], g[5]), pack2(g[6], g[7]));
                }
            }
        }
        fence_async_smem();
        tc_fence_before();
        __syncthreads();
        if (tid == 0) {
            tc_fence_after();
            umma_tile(tmem, smem_u32(sA), smem_u32(sB), false);
            umma_commit(&s_bar);
        }
        const bool ok = __syncthreads_and(mbar_wait(&s_bar, phase, ctl, 901) ? 1 : 0) != 0;
        phase ^= 1u;
        if (!ok) {
            mbar_drain(&s_bar, phase ^ 1u);  // let the issued MMAs drain before TMEM is freed
            break;
        }
        tc_fence_after();
        float y = b3;
#pragma unroll 1
        for (int c = 0; c < kHid / 32; ++c) {
            float z2[32];
            tmem_ld32(tmem + lane_base + 32u * c, z2);
#pragma unroll
            for (int j = 0; j < 32; ++j) y += gelu(z2[j] + s_b2[32 * c + j]) * s_w3[32 * c + j];
        }
        if (!TRAIN) {
            if (fout && valid) fout[row] = y;
            if (A.residual) y += logc;
            if (valid) {
                if (scores) scores[row] = y;
                if (sel) {
                    const uint64_t sk = score_select_key(y);
                    sel[row] = sk;
                    if (hist) atomicAdd(&s_hist[sk >> 52], 1u);
                }
            }
        } else {
            const float t = valid ? target[row] : 0.0f;
            const float err = valid ? (y - t) : 0.0f;
            const float dy = 2.0f * inv_batch * err;
            float e2 = err * err;
#pragma unroll
            for (int s = 16; s >= 1; s >>= 1) e2 += __shfl_xor_sync(0xffffffffu, e2, s);
            float dyw = dy;
#pragma unroll
            for (int s = 16; s >= 1; s >>= 1) dyw += __shfl_xor_sync(0xffffffffu, dyw, s);
            if ((tid & 31) == 0) {
                atomicAdd(&s_acc[2 * kHid], dyw);
                atomicAdd(&s_acc[2 * kHid + 1], e2);
            }
#pragma unroll 1
            for (int c = 0; c < kHid / 32; ++c) {
                float dz[32], dw[32];
                tmem_ld32(tmem + lane_base + 32u * c, dz);  // z2 again, one chunk at a time
#pragma unroll
                for (int j = 0; j < 32; ++j) {
                    const float x = dz[j] + s_b2[32 * c + j];
                    dz[j] = dy * s_w3[32 * c + j] * gelu_grad(x);
                    dw[j] = dy * gelu(x);
                }
                if (valid) {
                    uint4* dd = reinterpret_cast<uint4*>(S.dz2 + row * kHid + 32 * c);
#pragma unroll
                    for (int q = 0; q < 4; ++q)
                        dd[q] = make_uint4(pack2(dz[8 * q], dz[8 * q + 1]), pack2(dz[8 * q + 2], dz[8 * q + 3]),
                                           pack2(dz[8 * q + 4], dz[8 * q + 5]), pack2(dz[8 * q + 6], dz[8 * q + 7]));
                }
                const float sdz = warp_column_sum(dz);
                const float sdw = warp_column_sum(dw);
                atomicAdd(&s_acc[32 * c + (tid & 31)], sdz);
                atomicAdd(&s_acc[kHid + 32 * c + (tid & 31)], sdw);
            }
        }
        tc_fence_before();
        __syncthreads();
    }
    __syncthreads();
    if (hist)
        for (int i = tid; i < kTopnBins1; i += kScoreThreads)
            if (s_hist[i]) atomicAdd(&hist[i], s_hist[i]);
    if (TRAIN) {
        for (int i = tid; i < kHid; i += kScoreThreads) {
            atomicAdd(&grads[A.L.b2 + i], s_acc[i]);
            atomicAdd(&grads[A.L.w3 + i], s_acc[kHid + i]);
        }
        if (tid == 0) {
            atomicAdd(&grads[A.L.b3], s_acc[2 * kHid]);
            atomicAdd(loss, s_acc[2 * kHid + 1]);
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        tmem_dealloc(tmem, kHid);
    }
}

// ---------------------------------------------------------------------------
// training backward: dW2 = h1^T dz2 (TMEM columns 0-127, accumulated over the block's tiles),
// dh1 = dz2 W2^T (columns 128-255, per tile), then dz1 = dh1 * gelu'(z1) feeds db1, du and
// the embedding rows.
// ---------------------------------------------------------------------------
template <int W>
__global__ void __launch_bounds__(kScoreThreads) k_train_bwd(const ScorerArgs A, const ScoreInput in, TrainScratch S,
                                                             float* __restrict__ grads, Ctl* ctl) {
    extern __shared__ __align__(128) uint8_t smem[];
    uint8_t* sA1 = smem;                   // h1^T      (in, term)
    uint8_t* sB1 = smem + kTileBytes;      // dz2^T     (out, term)
    uint8_t* sA2 = smem + 2 * kTileBytes;  // dz2       (term, out)
    uint8_t* sB2 = smem + 3 * kTileBytes;  // w2        (in, out)
    float* s_acc = reinterpret_cast<float*>(smem + 4 * kTileBytes);  // db1[128], du[3][128]
    __shared__ __align__(8) uint64_t s_bar;
    __shared__ uint32_t s_tmem;
    const int tid = threadIdx.x, warp = tid >> 5;

    stage_w2(A, sB2, false);
    for (int i = tid; i < 4 * kHid; i += kScoreThreads) s_acc[i] = 0.0f;
    if (tid == 0) mbar_init(&s_bar, 1);
    if (warp == 0) tmem_alloc(&s_tmem, 2 * kHid);
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = s_tmem;
    const uint32_t lane_base = (uint32_t)(warp * 32) << 16;

    const uint64_t ntiles = (in.n + kScoreTile - 1) / kScoreTile;
    uint32_t phase = 0;
    int done = 0;
    bool ok = true;
    for (uint64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const uint64_t row = tile * kScoreTile + tid;
        const bool valid = row < in.n;
        // stage the operands; rows past the batch are zero
        for (int c = 0; c < kHid / 8; ++c) {
            uint4 h = make_uint4(0, 0, 0, 0), d = make_uint4(0, 0, 0, 0);
            if (valid) {
                h = *reinterpret_cast<const uint4*>(S.h1 + row * kHid + 8 * c);
                d = *reinterpret_cast<const uint4*>(S.dz2 + row * kHid + 8 * c);
            }
            *reinterpret_cast<uint4*>(sA2 + kmaj_off(tid, 8 * c)) = d;
            const uint32_t hw[4] = {h.x, h.y, h.z, h.w}, dw[4] = {d.x, d.y, d.z, d.w};
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int col = 8 * c + 2 * j;
                *reinterpret_cast<uint16_t*>(sA1 + kmaj_off(col, tid)) = (uint16_t)(hw[j] & 0xFFFFu);
                *reinterpret_cast<uint16_t*>(sA1 + kmaj_off(col + 1, tid)) = (uint16_t)(hw[j] >> 16);
                *reinterpret_cast<uint16_t*>(sB1 + kmaj_off(col, tid)) = (uint16_t)(dw[j] & 0xFFFFu);
                *reinterpret_cast<uint16_t*>(sB1 + kmaj_off(col + 1, tid)) = (uint16_t)(dw[j] >> 16);
            }
        }
        fence_async_smem();
        tc_fence_before();
        __syncthreads();
        if (tid == 0) {
            tc_fence_after();
            umma_tile(tmem, smem_u32(sA1), smem_u32(sB1), done > 0);
            umma_tile(tmem + kHid, smem_u32(sA2), smem_u32(sB2), false);
            umma_commit(&s_bar);
        }
        ok = __syncthreads_and(mbar_wait(&s_bar, phase, ctl, 902) ? 1 : 0) != 0;
        phase ^= 1u;
        if (!ok) {
            mbar_drain(&s_bar, phase ^ 1u);  // let the issued MMAs drain before TMEM is freed
            break;
        }
        ++done;
        tc_fence_after();
        uint64_t k[2 * W];
        float f[3];
        term_features<W>(A, in, row, valid, k, f);
#pragma unroll 1
        for (int c = 0; c < kHid / 32; ++c) {
            float dz[32], g[32];
            tmem_ld32(tmem + lane_base + kHid + 32u * c, dz);
            if (valid)
                load_bf16x32(S.gz1 + row * kHid + 32 * c, g);
            else
#pragma unroll
                for (int j = 0; j < 32; ++j) g[j] = 0.0f;
#pragma unroll
            for (int j = 0; j < 32; ++j) dz[j] *= g[j];
            if (valid) {
#pragma unroll
                for (int w = 0; w < W; ++w) {
                    uint64_t live = k[w] | k[W + w];
                    while (live) {
                        const int bit = __ffsll((long long)live) - 1;
                        live &= live - 1;
                        const int q = 64 * w + bit;
                        const int p = (int)((k[w] >> bit) & 1u) | ((int)((k[W + w] >> bit) & 1u) << 1);
                        float* e = grads + A.L.embed + ((size_t)q * 3 + (size_t)(p - 1)) * kHid + 32 * c;
#pragma unroll
                        for (int j = 0; j < 32; ++j) atomicAdd(e + j, dz[j]);
                    }
                }
            }
            float t0[32], t1[32], t2[32];
#pragma unroll
            for (int j = 0; j < 32; ++j) {
                t0[j] = dz[j] * f[0];
                t1[j] = dz[j] * f[1];
                t2[j] = dz[j] * f[2];
            }
            const int l = tid & 31;
            atomicAdd(&s_acc[32 * c + l], warp_column_sum(dz));
            atomicAdd(&s_acc[kHid + 32 * c + l], warp_column_sum(t0));
            atomicAdd(&s_acc[2 * kHid + 32 * c + l], warp_column_sum(t1));
            atomicAdd(&s_acc[3 * kHid + 32 * c + l], warp_column_sum(t2));
        }
        tc_fence_before();
        __syncthreads();
    }
    if (ok && done > 0) {
        tc_fence_after();
        // dW2[in][out]: this thread's lane is `in`, the columns are `out`
        const int in_row = tid;
#pragma unroll 1
        for (int c = 0; c < kHid / 32; ++c) {
            float v[32];
            tmem_ld32(tmem + lane_base + 32u * c, v);
#pragma unroll
            for (int j = 0; j < 32; ++j) atomicAdd(&grads[A.L.w2 + (size_t)in_row * kHid + 32 * c + j], v[j]);
        }
        __syncthreads();
        for (int i = tid; i < kHid; i += kScoreThreads) {
            atomicAdd(&grads[A.L.b1 + i], s_acc[i]);
            atomicAdd(&grads[A.L.u + i], s_acc[kHid + i]);
            atomicAdd(&grads[A.L.u + kHid + i], s_acc[2 * kHid + i]);
            atomicAdd(&grads[A.L.u + 2 * kHid + i], s_acc[3 * kHid + i]);
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        tmem_dealloc(tmem, 2 * kHid);
    }
}


// B operand of the inference kernel's layer 2 in f16: element (out, in) = w2[in][out] (every
// bf16 weight in f16's normal range converts exactly).
__device__ __forceinline__ void stage_w2_f16(const ScorerArgs& A, uint8_t* sB) {
    const uint16_t* w2 = A.p + A.L.w2;
    for (int i = threadIdx.x; i < kHid * kHid; i += blockDim.x) {
        const int r = i / kHid, c = i % kHid;  // w2[r][c], r = in, c = out
        *reinterpret_cast<__half*>(sB + kmaj_off(c, r)) = __float2half_rn(bf2f(w2[i]));
    }
}

// ---------------------------------------------------------------------------
// inference on the tensor cores (scorers of at most kTcRows embedding rows)
//
// Both layers are GEMMs per tile of 128 terms.  Layer 1: the tile's one-hot operand A1
// (128 terms x K1, K1 = 3 kTcRows + 16: the count of each (row, X/Z/Y) among the term's
// non-identity qubits, then the three scalar features each split into a bf16 high and low part,
// then a 1 for the bias) times B1 (128 hidden x K1: the embedding rows, the feature columns u
// twice, b1) gives z1 = b1 + f.u + the embedding bag, accumulated in f32 in TMEM.  The counts are
// small integers and the split features carry 16 significant bits, so the product equals the
// CUDA-core embedding bag up to the order of f32 additions.  Layer 2 is the 128 x 128 GEMM of the
// other kernel, in f16 here: both GELUs run on packed f16 pairs (gelu_h2), the first feeding the
// f16 operand directly, the second's outputs weighted and summed in f32.  A CTA holds two warpgroups, each owning one tile at a time (its own operand,
// mbarrier and 128 TMEM columns, shared by the two accumulators in turn) and synchronising on its
// own named barrier, so one warpgroup's GELUs overlap the other's MMAs.
// ---------------------------------------------------------------------------
constexpr int kK1 = 3 * kTcRows + 16;
constexpr uint32_t kK1Sbo = (uint32_t)(kK1 / 8) * 128u;     // bytes between 8-row groups (K1 wide)
constexpr uint32_t kOpA1Bytes = (uint32_t)kScoreTile * kK1 * 2u;
constexpr uint32_t kOpB1Bytes = (uint32_t)kHid * kK1 * 2u;
constexpr int kTcThreads = 256;
constexpr size_t kTcSmem = kOpB1Bytes + kTileBytes + 2 * (size_t)kOpA1Bytes + 2 * kHid * sizeof(float) +
                           kTopnBins1 * sizeof(unsigned int);

// Byte offset of element (row, k) of a K1-wide K-major operand (core matrix (row / 8, k / 8)).
__device__ __forceinline__ uint32_t kmaj1_off(int row, int k) {
    return (uint32_t)((row >> 3) * kK1Sbo + (k >> 3) * 128 + (row & 7) * 16 + (k & 7) * 2);
}

// Named barrier over one warpgroup (ids 1 and 2; 0 is __syncthreads).
__device__ __forceinline__ void wg_sync(int id) { asm volatile("bar.sync %0, 128;" ::"r"(id) : "memory"); }
__device__ __forceinline__ bool wg_and(int id, bool v) {
    uint32_t out;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\t"
        "setp.ne.u32 p, %1, 0;\n\t"
        "bar.red.and.pred q, %2, 128, p;\n\t"
        "selp.u32 %0, 1, 0, q;\n\t}"
        : "=r"(out)
        : "r"(v ? 1u : 0u), "r"(id)
        : "memory");
    return out != 0;
}

// D (TMEM) = A (128 x K1) * B1^T: K1 / 16 MMAs, each 2 core matrices (256 bytes) further along K.
__device__ __forceinline__ void umma_tile_k1(uint32_t d_tmem, uint32_t a_saddr, uint32_t b_saddr) {
    const uint64_t ad = umma_desc(a_saddr, kK1Sbo), bd = umma_desc(b_saddr, kK1Sbo);
#pragma unroll
    for (int j = 0; j < kK1 / 16; ++j) {
        const uint32_t acc = j > 0 ? 1u : 0u;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
            ::"r"(d_tmem), "l"(ad + 16ull * j), "l"(bd + 16ull * j), "r"(kIdesc), "r"(acc));
    }
}

__device__ __forceinline__ void split_bf16(float v, uint16_t& hi, uint16_t& lo) {
    hi = f2bf(v);
    lo = f2bf(v - bf2f(hi));
}

template <int W>
__global__ void __launch_bounds__(kTcThreads, 1) k_score_tc(const ScorerArgs A, const ScoreInput in,
                                                            float* __restrict__ scores, uint64_t* __restrict__ sel,
                                                            unsigned int* __restrict__ hist, Ctl* ctl,
                                                            float* __restrict__ fout) {
    extern __shared__ __align__(128) uint8_t smem[];
    uint8_t* sB1 = smem;
    uint8_t* sB2 = smem + kOpB1Bytes;
    float* s_b2 = reinterpret_cast<float*>(smem + kOpB1Bytes + kTileBytes + 2 * (size_t)kOpA1Bytes);
    float* s_w3 = s_b2 + kHid;
    unsigned int* s_hist = reinterpret_cast<unsigned int*>(s_w3 + kHid);
    __shared__ __align__(8) uint64_t s_bar[2];
    __shared__ uint32_t s_tmem;
    const int tid = threadIdx.x, warp = tid >> 5;
    const int g = tid >> 7, t = tid & 127;  // warpgroup, row of its tile
    uint8_t* sA = smem + kOpB1Bytes + kTileBytes + (size_t)g * kOpA1Bytes;

    // B1 (hidden n, input column k): embedding rows, u (twice: high and low feature parts), b1
    for (int i = tid; i < kHid * kK1; i += kTcThreads) {
        const int k = i / kHid, n = i % kHid;  // n fastest: the global reads are contiguous
        uint16_t v = 0;
        if (k < 3 * kTcRows) {
            if (k / 3 < A.nq) v = A.p[A.L.embed + (size_t)k * kHid + n];  // embed[q][p][n], k = 3 q + p
        } else if (k < 3 * kTcRows + 6) {
            v = A.p[A.L.u + (size_t)((k - 3 * kTcRows) >> 1) * kHid + n];
        } else if (k == 3 * kTcRows + 6) {
            v = A.p[A.L.b1 + n];
        }
        *reinterpret_cast<uint16_t*>(sB1 + kmaj1_off(n, k)) = v;
    }
    stage_w2_f16(A, sB2);
    for (int i = tid; i < kHid; i += kTcThreads) {
        s_b2[i] = bf2f(A.p[A.L.b2 + i]);
        s_w3[i] = bf2f(A.p[A.L.w3 + i]);
    }
    if (hist)
        for (int i = tid; i < kTopnBins1; i += kTcThreads) s_hist[i] = 0;
    const float b3 = bf2f(A.p[A.L.b3]);
    if (tid == 0) {
        mbar_init(&s_bar[0], 1);
        mbar_init(&s_bar[1], 1);
    }
    if (warp == 0) tmem_alloc(&s_tmem, 2 * kHid);
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = s_tmem + (uint32_t)(g * kHid);           // this warpgroup's columns
    const uint32_t lane_base = (uint32_t)((warp & 3) * 32) << 16;  // its warp's TMEM lanes
    const int bar_id = 1 + g;

    const uint64_t ntiles = (in.n + kScoreTile - 1) / kScoreTile;
    uint32_t phase = 0;
    for (uint64_t tile = 2 * (uint64_t)blockIdx.x + g; tile < ntiles; tile += 2 * (uint64_t)gridDim.x) {
        const uint64_t row = tile * kScoreTile + t;
        const bool valid = row < in.n;
        uint64_t k[2 * W];
        float f[3];
        const float logc = term_features<W>(A, in, row, valid, k, f);
        // A1 row t: zeros, the split scalar features and the bias column, then the counts
        {
            const uint4 zero = make_uint4(0, 0, 0, 0);
#pragma unroll
            for (int c = 0; c < 3 * kTcRows / 8; ++c) *reinterpret_cast<uint4*>(sA + kmaj1_off(t, 8 * c)) = zero;
            uint16_t h0, l0, h1, l1, h2, l2;
            split_bf16(f[0], h0, l0);
            split_bf16(f[1], h1, l1);
            split_bf16(f[2], h2, l2);
            const uint16_t one = valid ? f2bf(1.0f) : 0;
            *reinterpret_cast<uint4*>(sA + kmaj1_off(t, 3 * kTcRows)) =
                make_uint4((uint32_t)h0 | (uint32_t)l0 << 16, (uint32_t)h1 | (uint32_t)l1 << 16,
                           (uint32_t)h2 | (uint32_t)l2 << 16, (uint32_t)one);
            *reinterpret_cast<uint4*>(sA + kmaj1_off(t, 3 * kTcRows + 8)) = zero;
#pragma unroll
            for (int w = 0; w < W; ++w) {
                uint64_t live = k[w] | k[W + w];
                while (live) {
                    const int bit = __ffsll((long long)live) - 1;
                    live &= live - 1;
                    const int r = A.site_row ? (int)A.site_row[64 * w + bit] : 64 * w + bit;
                    if (r < 0 || r >= kTcRows) continue;
                    const int p = (int)((k[w] >> bit) & 1u) | ((int)((k[W + w] >> bit) & 1u) << 1);
                    uint16_t* e = reinterpret_cast<uint16_t*>(sA + kmaj1_off(t, 3 * r + p - 1));
                    *e = f2bf(bf2f(*e) + 1.0f);
                }
            }
        }
        fence_async_smem();
        tc_fence_before();
        wg_sync(bar_id);
        if (t == 0) {
            tc_fence_after();
            umma_tile_k1(tmem, smem_u32(sA), smem_u32(sB1));
            umma_commit(&s_bar[g]);
        }
        bool ok = wg_and(bar_id, mbar_wait(&s_bar[g], phase, ctl, 905));
        phase ^= 1u;
        if (!ok) {
            mbar_drain(&s_bar[g], phase ^ 1u);
            break;
        }
        tc_fence_after();
        // GELU(z1) as the f16 layer-2 operand, over the dead A1 (128-wide K-major layout)
#pragma unroll 1
        for (int c = 0; c < kHid / 32; ++c) {
            float z[32];
            tmem_ld32(tmem + lane_base + 32u * c, z);
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                uint4 u;
                u.x = h2_bits(gelu_h2(__floats2half2_rn(z[8 * q + 0], z[8 * q + 1])));
                u.y = h2_bits(gelu_h2(__floats2half2_rn(z[8 * q + 2], z[8 * q + 3])));
                u.z = h2_bits(gelu_h2(__floats2half2_rn(z[8 * q + 4], z[8 * q + 5])));
                u.w = h2_bits(gelu_h2(__floats2half2_rn(z[8 * q + 6], z[8 * q + 7])));
                *reinterpret_cast<uint4*>(sA + kmaj_off(t, 32 * c + 8 * q)) = u;
            }
        }
        fence_async_smem();
        tc_fence_before();
        wg_sync(bar_id);
        if (t == 0) {
            tc_fence_after();
            umma_tile(tmem, smem_u32(sA), smem_u32(sB2), false, kIdescF16);
            umma_commit(&s_bar[g]);
        }
        ok = wg_and(bar_id, mbar_wait(&s_bar[g], phase, ctl, 906));
        phase ^= 1u;
        if (!ok) {
            mbar_drain(&s_bar[g], phase ^ 1u);
            break;
        }
        tc_fence_after();
        float y = b3;
#pragma unroll 1
        for (int c = 0; c < kHid / 32; ++c) {
            float z2[32];
            tmem_ld32(tmem + lane_base + 32u * c, z2);
#pragma unroll
            for (int j = 0; j < 32; j += 2) {
                const float2 g = __half22float2(
                    gelu_h2(__floats2half2_rn(z2[j] + s_b2[32 * c + j], z2[j + 1] + s_b2[32 * c + j + 1])));
                y = __fmaf_rn(g.x, s_w3[32 * c + j], y);
                y = __fmaf_rn(g.y, s_w3[32 * c + j + 1], y);
            }
        }
        if (fout && valid) fout[row] = y;  // the network's own output (the prediction a row carries)
        if (A.residual) y += logc;
        if (valid) {
            if (scores) scores[row] = y;
            if (sel) {
                const uint64_t sk = score_select_key(y);
                sel[row] = sk;
                if (hist) atomicAdd(&s_hist[sk >> 52], 1u);
            }
        }
        tc_fence_before();
        wg_sync(bar_id);  // every lane has read the accumulator and left A before the next tile
    }
    __syncthreads();
    if (hist)
        for (int i = tid; i < kTopnBins1; i += kTcThreads)
            if (s_hist[i]) atomicAdd(&hist[i], s_hist[i]);
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        tmem_dealloc(s_tmem, 2 * kHid);
    }
}

__global__ void k_adam(float* __restrict__ master, uint16_t* __restrict__ bf, float* __restrict__ g,
                       float* __restrict__ m, float* __restrict__ v, size_t count, float lr, float b1, float b2,
                       float eps, float c1, float c2) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < count; i += (size_t)gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.0f - b1) * gi;
        const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        const float p = master[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
        master[i] = p;
        bf[i] = f2bf(p);
        g[i] = 0.0f;
    }
}

__global__ void k_to_bf16(const float* __restrict__ master, uint16_t* __restrict__ bf, size_t count) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < count; i += (size_t)gridDim.x * blockDim.x)
        bf[i] = f2bf(master[i]);
}

constexpr size_t kScoreSmem = 2 * kTileBytes + (4 * kHid + 2) * sizeof(float) + kTopnBins1 * sizeof(unsigned int);
constexpr size_t kBwdSmem = 4 * kTileBytes + 4 * kHid * sizeof(float);

inline unsigned int score_grid(uint64_t n, int sms, int per_sm) {
    const uint64_t tiles = (n + kScoreTile - 1) / kScoreTile;
    const uint64_t cap = (uint64_t)sms * per_sm;
    return (unsigned int)(tiles < cap ? (tiles ? tiles : 1) : cap);
}

}  // namespace

template <int W>
cudaError_t configure_scorer_kernels() {
    cudaError_t e = cudaFuncSetAttribute(k_score<W, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kScoreSmem);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_score_tc<W>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTcSmem);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_score<W, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kScoreSmem);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_train_bwd<W>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kBwdSmem);
    return e;
}

template <int W>
cudaError_t launch_score(const ScorerArgs& A, const ScoreInput& in, float* scores, uint64_t* sel_keys,
                         unsigned int* hist, Ctl* ctl, int sms, cudaStream_t st, KernelProf* prof, float* fout) {
    if (!in.n) return cudaSuccess;
    // 2 x (128 x 128) bf16 GEMM flops per term plus the output dot; bytes: key + coefficient
    prof->begin(K_SCORE, (double)in.n * (16 * W + 8 + (sel_keys ? 8 : 4)), st);
    TrainScratch none{nullptr, nullptr, nullptr};
    if (A.nq <= kTcRows) {
        // one CTA per SM (~200 KB of shared memory, 256 TMEM columns), two tiles in flight per CTA
        const uint64_t tiles = (in.n + kScoreTile - 1) / kScoreTile;
        const unsigned int grid = (unsigned int)std::min<uint64_t>((tiles + 1) / 2, (uint64_t)(sms > 0 ? sms : 1));
        k_score_tc<W><<<grid, kTcThreads, kTcSmem, st>>>(A, in, scores, sel_keys, hist, ctl, fout);
    } else {
        // three blocks per SM: 3 x 128 TMEM columns and 3 x ~75 KB of shared memory fit one SM
        k_score<W, false><<<score_grid(in.n, sms, 3), kScoreThreads, kScoreSmem, st>>>(A, in, scores, sel_keys, hist,
                                                                                      nullptr, 0.0f, none, nullptr,
                                                                                      nullptr, ctl, fout);
    }
    prof->end(st);
    return cudaGetLastError();
}

template <int W>
cudaError_t launch_train_batch(const ScorerArgs& A, const ScoreInput& in, const float* target, float inv_batch,
                               const TrainScratch& S, float* grads, float* loss, Ctl* ctl, int sms,
                               cudaStream_t st, KernelProf* prof) {
    if (!in.n) return cudaSuccess;
    prof->begin(K_SCORE_TRAIN, (double)in.n * (16 * W + 12 + 6 * kHid), st);
    k_score<W, true><<<score_grid(in.n, sms, 3), kScoreThreads, kScoreSmem, st>>>(A, in, nullptr, nullptr, nullptr,
                                                                                 target, inv_batch, S, grads, loss,
                                                                                 ctl, nullptr);
    // one block per SM: 256 TMEM columns and 130 KB of shared memory
    k_train_bwd<W><<<score_grid(in.n, sms, 1), kScoreThreads, kBwdSmem, st>>>(A, in, S, grads, ctl);
    prof->end(st);
    return cudaGetLastError();
}

cudaError_t launch_adam(float* master, uint16_t* bf16, float* grads, float* m, float* v, size_t count, float lr,
                        float beta1, float beta2, float eps, int step, cudaStream_t st) {
    const float c1 = 1.0f - powf(beta1, (float)step), c2 = 1.0f - powf(beta2, (float)step);
    k_adam<<<256, 256, 0, st>>>(master, bf16, grads, m, v, count, lr, beta1, beta2, eps, c1, c2);
    return cudaGetLastError();
}

cudaError_t launch_to_bf16(const float* master, uint16_t* bf16, size_t count, cudaStream_t st) {
    k_to_bf16<<<256, 256, 0, st>>>(master, bf16, count);
    return cudaGetLastError();
}

template cudaError_t configure_scorer_kernels<1>();
template cudaError_t configure_scorer_kernels<2>();
template cudaError_t configure_scorer_kernels<4>();
template cudaError_t launch_score<1>(const ScorerArgs&, const ScoreInput&, float*, uint64_t*, unsigned int*, Ctl*,
                                     int, cudaStream_t, KernelProf*, float*);
template cudaError_t launch_score<2>(const ScorerArgs&, const ScoreInput&, float*, uint64_t*, unsigned int*, Ctl*,
                                     int, cudaStream_t, KernelProf*, float*);
template cudaError_t launch_score<4>(const ScorerArgs&, const ScoreInput&, float*, uint64_t*, unsigned int*, Ctl*,
                                     int, cudaStream_t, KernelProf*, float*);
template cudaError_t launch_train_batch<1>(const ScorerArgs&, const ScoreInput&, const float*, float,
                                           const TrainScratch&, float*, float*, Ctl*, int, cudaStream_t, KernelProf*);
template cudaError_t launch_train_batch<2>(const ScorerArgs&, const ScoreInput&, const float*, float,
                                           const TrainScratch&, float*, float*, Ctl*, int, cudaStream_t, KernelProf*);
template cudaError_t launch_train_batch<4>(const ScorerArgs&, const ScoreInput&, const float*, float,
                                           const TrainScratch&, float*, float*, Ctl*, int, cudaStream_t, KernelProf*);

}  // namespace psb
