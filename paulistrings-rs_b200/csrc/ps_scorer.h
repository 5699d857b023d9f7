// ps_scorer.h -- the learned truncation scorer: parameter layout and kernel launchers.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include "ps_kernels.h"

namespace psb {

constexpr int kHid = 128;          // hidden width of both hidden layers
constexpr int kScoreTile = 128;    // terms per tensor-core tile (the MMA's M)

// Offsets (in parameters) of one scorer's flat parameter vector; the fp32 masters, the bf16
// copies the kernels read, the gradients and the Adam moments all share it.
//   embed [nq][3][kHid]  rows for X, Z, Y on qubit q (local index x | z << 1, minus one);
//                        the identity's one-hot column is folded into b1
//   u     [3][kHid]      input columns of the scalar features (weight, log|c|, remaining depth)
//   b1    [kHid]
//   w2    [kHid][kHid]   (in, out)
//   b2    [kHid]
//   w3    [kHid]
//   b3    [1]
struct ScorerLayout {
    size_t embed, u, b1, w2, b2, w3, b3, total;
};

inline ScorerLayout scorer_layout(int nq) {
    ScorerLayout L;
    L.embed = 0;
    L.u = L.embed + (size_t)nq * 3 * kHid;
    L.b1 = L.u + 3 * kHid;
    L.w2 = L.b1 + kHid;
    L.b2 = L.w2 + (size_t)kHid * kHid;
    L.w3 = L.b2 + kHid;
    L.b3 = L.w3 + kHid;
    L.total = L.b3 + 1;
    return L;
}

struct ScorerArgs {
    const uint16_t* p;        // bf16 parameters (device)
    ScorerLayout L;
    int nq;                   // embedding rows
    float fscale[3];          // feature scales: weight, log|c|, remaining depth
    int residual;             // scores = log|c| + output
    const int16_t* site_row;  // inference: embedding row of each qubit of the scored sums (-1: none);
                              // nullptr: qubit q uses row q
};

// Embedding rows the tensor-core inference kernel holds in its one-hot operand: scorers with at
// most this many rows (after a site map, any number of qubits) score on the tensor cores.
constexpr int kTcRows = 64;

// Per-term features: the key, and log|c| from a coefficient column (coef64 / coef32) or an
// array (logc); the remaining depth uniform (rem_uniform) or from an array (rem).
struct ScoreInput {
    const uint64_t* keys;
    const double* coef64;
    const float* coef32;
    const float* logc;
    const float* rem;
    float rem_uniform;
    uint64_t n;
};

// Select keys for the TopN machinery: (order-preserving bits of the score) << 31, 0 for NaN;
// also histograms their top 11 bits into hist (kTopnBins1 words, zero on entry) when non-null.
// fout (optional): the network's output per term, before the residual log|c| (the prediction a
// row carries through the layers of an inherited scored pass).
template <int W>
cudaError_t launch_score(const ScorerArgs& A, const ScoreInput& in, float* scores, uint64_t* sel_keys,
                         unsigned int* hist, Ctl* ctl, int sms, cudaStream_t st, KernelProf* prof,
                         float* fout = nullptr);

// Training: one minibatch.  Forward stores h1, gelu'(z1) and dz2 (bf16) per term and adds
// dw3, db2, db3 and the summed squared error; backward adds dW2 (tensor cores), db1, du and
// the embedding rows.  grads (fp32, layout above) accumulate; loss[0] += sum (y - t)^2.
struct TrainScratch {
    uint16_t* h1;     // [B][kHid] bf16
    uint16_t* gz1;    // [B][kHid] bf16, gelu'(z1)
    uint16_t* dz2;    // [B][kHid] bf16
};
template <int W>
cudaError_t launch_train_batch(const ScorerArgs& A, const ScoreInput& in, const float* target, float inv_batch,
                               const TrainScratch& S, float* grads, float* loss, Ctl* ctl, int sms,
                               cudaStream_t st, KernelProf* prof);

// Adam on the fp32 masters, bf16 copies refreshed, gradients cleared.
cudaError_t launch_adam(float* master, uint16_t* bf16, float* grads, float* m, float* v, size_t count, float lr,
                        float beta1, float beta2, float eps, int step, cudaStream_t st);
// bf16 copies of the fp32 masters.
cudaError_t launch_to_bf16(const float* master, uint16_t* bf16, size_t count, cudaStream_t st);

template <int W>
cudaError_t configure_scorer_kernels();

}  // namespace psb
