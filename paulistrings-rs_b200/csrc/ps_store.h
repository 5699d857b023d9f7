// ps_store.h -- launchers of the store kernels (ingest, readout, TopN).
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include "ps_kernels.h"

namespace psb {

constexpr int kExpectBlocks = 592;  // 4 x 148 SMs; fixed so the reduction order is fixed
constexpr int kTopnBins1 = 2048;    // first select digit: |c|^2 key >> 52
constexpr int kTopnBinsN = 8192;    // later digits: 13 bits over the boundary-bin candidates

struct SortScratch {
    unsigned int* hist;        // device, 16W x 256
    unsigned int* base;        // device, 16W x 256
    unsigned int* status;      // device, tiles x 256
    unsigned int* host_hist;   // pinned, 16W x 256
    unsigned int* host_base;   // pinned, 16W x 256
};

// 64-bit words the TopN candidate buffer needs for n terms (block segments and their lengths).
uint64_t topn_cand_words(uint64_t n, int sms);

// The select's boundary (full-range select key) and whether a windowed select missed, from
// the aux words StoreOps::topn leaves in host_count.
inline uint64_t topn_boundary(const unsigned long long* host_count, uint64_t base) {
    const unsigned long long* aux = reinterpret_cast<const unsigned long long*>(
        reinterpret_cast<const unsigned char*>(host_count) + offsetof(Ctl, aux));
    return aux[0] == 0 ? 0 : aux[0] + base;
}
// A topn call given the next layer: its compaction fell back to the plain one (aux[7]), so the
// next layer's partner list was not written.
inline bool topn_unclassified(const unsigned long long* host_count) {
    const unsigned long long* aux = reinterpret_cast<const unsigned long long*>(
        reinterpret_cast<const unsigned char*>(host_count) + offsetof(Ctl, aux));
    return aux[7] != 0;
}
inline bool topn_window_missed(const unsigned long long* host_count) {
    const unsigned long long* aux = reinterpret_cast<const unsigned long long*>(
        reinterpret_cast<const unsigned char*>(host_count) + offsetof(Ctl, aux));
    return aux[5] != 0;
}

// Error bits and check id left in host_count by StoreOps::topn.
inline void topn_flags(const unsigned long long* host_count, unsigned int* flags, unsigned int* info) {
    const unsigned int* f = reinterpret_cast<const unsigned int*>(reinterpret_cast<const unsigned char*>(host_count) +
                                                                  offsetof(Ctl, err));
    *flags = f[0];
    *info = f[1];
}

template <int W, typename T>
struct StoreOps {
    static cudaError_t configure();
    static size_t sort_tile();
    static cudaError_t pack(const uint64_t* x, const uint64_t* z, const double* c, uint64_t n, uint32_t nq,
                            uint64_t* keys, T* coef, uint32_t* vals, Ctl* ctl, int sms, cudaStream_t st, KernelProf* prof);
    // *sorted = keys strictly increasing and no zero coefficient (synchronizes)
    static cudaError_t check_sorted(const uint64_t* keys, const T* coef, uint64_t n, Ctl* ctl,
                                    unsigned long long* host_count, bool* sorted, int sms, cudaStream_t st,
                                    KernelProf* prof);
    static cudaError_t unpack(const uint64_t* keys, const T* coef, uint64_t n, uint64_t* x, uint64_t* z, double* c,
                              int sms, cudaStream_t st, KernelProf* prof);
    // LSD radix sort of (key, value) pairs; the sorted pairs end in (keys, vals) or, when
    // result_in_alt, in (keys_alt, vals_alt).
    static cudaError_t sort_pairs(uint64_t* keys, uint32_t* vals, uint64_t* keys_alt, uint32_t* vals_alt, uint64_t n,
                                  SortScratch& s, Ctl* ctl, int sms, cudaStream_t st, bool& result_in_alt,
                                  KernelProf* prof);
    static cudaError_t dedup(const uint64_t* keys, const uint32_t* vals, const T* cin, uint64_t n, const KeepProg& keep,
                             bool compensated, uint64_t* okeys, T* ocoef, unsigned long long* status, Ctl* ctl,
                             unsigned long long* host_count, uint64_t* out_n, cudaStream_t st, KernelProf* prof);
    // hist: kTopnBinsN words, zero on entry and on exit; when hist_ready its first kTopnBins1
    // words already hold the digit-1 histogram of coef (built by the layer's merge).
    // host_count: pinned scratch of at least 20 words; on return it holds the control block's
    // counts, tile counters and error words (read the flags with topn_flags).
    // sel: when non-null, precomputed select keys (larger kept first, 0 never) replace mag_key(c);
    // hist_ready must then hold their digit-1 histogram.  fpred: the learned pass's predictions;
    // the select key is then score_key(c, f) (windowed like mag_key when window), and the kept
    // rows' predictions are written to fout.  next (plain TopN only): the next rotation layer;
    // the compaction then also writes that layer's partner list (next_idx, next_D, n words each)
    // and its partner count in count[0], unless topn_unclassified says it could not; next_flags:
    // each row's partner test under that layer, written by the layer's merge (or nullptr).
    // deferred: the host has not read the layer's counts; n (and the scratch) bound the span,
    // which the kernels read from the control block with the live count (when it is within
    // keep_n every live row is kept), and a layer that failed is left alone; host_count[22] and
    // [23] receive the span and whether every live row was kept.  Needs cooperative_select().
    static cudaError_t topn(const uint64_t* keys, const T* coef, uint64_t n, uint64_t keep_n, uint64_t* okeys, T* ocoef,
                            unsigned int* hist, bool hist_ready, uint64_t* cand, uint64_t cand_cap,
                            unsigned long long* status, Ctl* ctl, unsigned long long* host_count, uint64_t* out_n,
                            int sms, cudaStream_t st, KernelProf* prof, const uint64_t* sel = nullptr,
                            bool window = false, uint64_t base = 0, SlotMap slots = SlotMap{nullptr, 0u},
                            const float* fpred = nullptr, float* fout = nullptr, const RotLayer<W>* next = nullptr,
                            uint32_t* next_idx = nullptr, uint16_t* next_D = nullptr,
                            const uint8_t* next_flags = nullptr, bool deferred = false);
    // Can topn run deferred (the whole select in one cooperative launch on this device)?
    static bool cooperative_select();
    // Compact the live rows of a slotted store of n rows (its span) into okeys / ocoef, in order;
    // *out_n = rows kept.  Reads the counts and error words into host_count (synchronizes).
    static cudaError_t densify(const uint64_t* keys, const T* coef, uint64_t n, SlotMap slots, uint64_t* okeys,
                               T* ocoef, unsigned long long* status, Ctl* ctl, unsigned long long* host_count,
                               uint64_t* out_n, cudaStream_t st, KernelProf* prof, const float* fin = nullptr,
                               float* fout = nullptr);
    // ApproxTopN (crates/paulistrings/src/truncation/builtin.rs:240-468): every octave of |c|^2
    // above the boundary octave kept, then the first quota boundary terms in key order.
    // hist: 2048 words, zero on entry and exit, holding the octave histogram when hist_ready;
    // host_hist: pinned, 2048 words.
    static cudaError_t approx_topn(const uint64_t* keys, const T* coef, uint64_t n, uint64_t keep_n, uint64_t* okeys,
                                   T* ocoef, unsigned int* hist, bool hist_ready, unsigned int* host_hist,
                                   unsigned long long* status, Ctl* ctl, unsigned long long* host_count,
                                   uint64_t* out_n, int sms, cudaStream_t st, KernelProf* prof);
    // CollapseSample's draw of `samples` points (the caller decides that n exceeds the cache).
    // norms: device, 2 * (blocks + 1) doubles; host_norms: pinned, 2 * (blocks + 1); first /
    // host_first: blocks + 1 words; mult: n words; blocks = ceil(n / 1024).  *drawable false
    // (nothing written) when sum |c| is zero or not finite.
    static cudaError_t collapse_sample(const uint64_t* keys, const T* coef, uint64_t n, uint64_t samples,
                                       uint64_t seed, uint64_t call, uint64_t* okeys, T* ocoef, double* norms,
                                       double* host_norms, uint64_t* first, uint64_t* host_first, uint32_t* mult,
                                       unsigned long long* status, Ctl* ctl, unsigned long long* host_count,
                                       uint64_t* out_n, bool* drawable, cudaStream_t st, KernelProf* prof);
    static cudaError_t expectation(const uint64_t* keys, const T* coef, uint64_t n, const uint64_t* ax,
                                   const uint64_t* az, const uint64_t* neg, double* partial, double* out_dev, int sms,
                                   cudaStream_t st, KernelProf* prof);
};

}  // namespace psb
