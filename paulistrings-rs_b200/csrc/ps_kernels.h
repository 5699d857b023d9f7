// ps_kernels.h -- plain data shapes shared by the host driver and the kernel launchers.
#pragma once

#include <chrono>
#include <cstddef>
#include <cstdint>
#include <cstdlib>
#include <sys/prctl.h>
#include <thread>
#include <cuda_runtime.h>

namespace psb {

// Wait for everything queued on `st`: the calling thread spins on an event for up to the spin
// budget (a layer's short waits end within it, where a sleeping thread's wake-up would cost more
// than the kernels it waited for), then polls the event between sleeps of 20 us with the
// thread's timer slack at 1 us (a thread that keeps spinning through a millisecond wait on a
// busy host is preempted and returns late; a blocking wait in the driver wakes up later still).
// The budget is PAULISTRINGS_B200_SPIN_US microseconds, read once (default 200; negative: spin
// without bound).  One event per device and host thread.
inline long long spin_budget_ns() {
    static const long long ns = [] {
        const char* v = std::getenv("PAULISTRINGS_B200_SPIN_US");
        const long long us = v && *v ? std::atoll(v) : 200;
        return us < 0 ? -1ll : us * 1000;
    }();
    return ns;
}
inline cudaError_t spin_sync(cudaStream_t st) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return cudaStreamSynchronize(st);
    thread_local cudaEvent_t events[64] = {};
    thread_local bool slack_set = false;
    if (!events[dev] && cudaEventCreateWithFlags(&events[dev], cudaEventDisableTiming) != cudaSuccess) {
        events[dev] = nullptr;
        return cudaStreamSynchronize(st);
    }
    cudaError_t e = cudaEventRecord(events[dev], st);
    if (e != cudaSuccess) return e;
    const long long budget = spin_budget_ns();
    const auto t0 = std::chrono::steady_clock::now();
    bool sleeping = false;
    while ((e = cudaEventQuery(events[dev])) == cudaErrorNotReady) {
        if (!sleeping && budget >= 0 &&
            std::chrono::duration_cast<std::chrono::nanoseconds>(std::chrono::steady_clock::now() - t0).count() > budget) {
            sleeping = true;
            if (!slack_set) {
                prctl(PR_SET_TIMERSLACK, 1000ul, 0ul, 0ul, 0ul);  // this thread's sleeps end within ~1 us
                slack_set = true;
            }
        }
        if (sleeping) std::this_thread::sleep_for(std::chrono::microseconds(20));
    }
    return e;
}

// Device-resident control block of one handle.
struct Ctl {
    unsigned long long count[8];   // counts published by kernels (partners, outputs, ...)
    unsigned int tile_counter[8];  // dynamic tile dispensers, reset before each launch
    unsigned int err;              // ERR_* bits
    unsigned int err_info;         // id of the first check that failed
    unsigned long long aux[8];     // small per-pass values (TopN boundary, quota, ...)
    unsigned long long spin_limit; // polls before a bounded device wait gives up
    unsigned long long support[4]; // ingest: OR of every key's x | z words (the qubits any term touches)
    unsigned long long span;       // a slotted merge's output: rows its slots span
    unsigned long long topn_all;   // a TopN select found the live rows within its quota: keep them all
};

// Lowered keep program (postfix), KeepProgram in the reference's device path.
struct KeepProg {
    int32_t n;
    int32_t op[15];     // 0 true, 1 coeff, 2 weight, 3 and, 4 or
    int64_t iarg[15];   // weight limit
    double eps2[15];    // eps * eps, or -1 when eps < 0 (keeps everything)
    // the common programs, recognised on the host: 0 keep all, 1 threshold, 2 weight,
    // 3 threshold and weight, 4 interpret op[]
    int32_t fast;
    double fast_eps2;
    int64_t fast_k;
};

constexpr int kMaxLevels = 8;
constexpr uint16_t kDivStart = 0xFFFE;    // divergence slot of the first partner
constexpr uint16_t kDivUnknown = 0xFFFF;  // predecessor lives in another classify tile

// The set bits of a partner delta, as significance ranks (0 = most significant key bit).
struct Levels {
    int32_t n;
    uint32_t rank[kMaxLevels];
};

// All set bits of a delta; launchers batch them by kMaxLevels.
struct LevelList {
    int32_t n;
    uint32_t rank[2 * 64 * 16];
};

// Device form of one rotation-shaped (or key-preserving) layer.
template <int W>
struct RotLayer {
    uint64_t gx[W], gz[W];   // partner delta (generator) x / z masks
    int32_t wide;            // 1: PreparedRotation (per-term phase), 0: LocalPtm lookup
    int32_t partners;        // 0: key-preserving, no partner stream
    int32_t qw[2], qb[2];    // support qubit j lives in word qw[j], bit qb[j]
    uint32_t pattern_mask;   // (1 << 2k) - 1
    double a0[16], a1[16];   // identity / generator amplitude per support pattern
    float a0f[16], a1f[16];
    double cos64, sin64;
    float cos32, sin32;
};

// Single-qubit key-preserving channels (depolarizing, dephasing, Pauli channels) that precede a
// rotation layer, folded into it: per channel its qubit and the factor of each pattern of that
// qubit (x | z << 1).  Applied in order to a term's coefficient, the keep program checked after
// each as the separate layers would, before the rotation's branches.
constexpr int kMaxNoise = 64;
struct NoiseList {
    int32_t n;
    uint16_t q[kMaxNoise];
    double f[kMaxNoise][4];
    float ff[kMaxNoise][4];
};

// Device form of a general local table (LocalPtm with any entries), per input support
// pattern s: the records it emits, in ascending entry order (DeltaEntry::emit,
// crates/paulistrings/src/channel/prepared.rs:50-68).
template <int W, typename T>
struct GenLayer {
    int32_t qw[2], qb[2];     // support qubit j lives in word qw[j], bit qb[j]
    uint32_t pattern_mask;    // (1 << 2k) - 1
    int32_t num_entries;
    uint64_t mx[16][W];       // entry e: x / z XOR masks
    uint64_t mz[16][W];
    uint8_t cnt[16];          // records emitted by pattern s
    uint8_t ent[16][16];      // entry of record j of pattern s
    T amp[16][16];            // amplitude of record j of pattern s
};

// Kernel ids of the per-kernel profile.
enum KernelId : int {
    K_CLASSIFY = 0,
    K_LEVEL_SCAN,   // k_level_reduce + k_level_scan
    K_LEVEL_APPLY,  // k_level_apply (places the partners)
    K_PARTITION,
    K_MERGE,
    K_TOPN_HIST,
    K_TOPN_STEP,
    K_TOPN_COMPACT,
    K_PACK,
    K_SORT_HIST,
    K_SORT_PASS,
    K_DEDUP,
    K_UNPACK,
    K_EXPECT,
    K_GEN_COUNT,
    K_GEN_BRANCH,
    K_SCORE,
    K_SCORE_TRAIN,
    K_NUM_KERNELS
};

// Counts every launch; with events enabled, times each launch with CUDA events on the
// launching stream and books its algorithmic bytes (resolved after the caller's sync).
struct KernelProf {
    static constexpr int kPool = 256;
    bool events = false;
    unsigned long long launches[K_NUM_KERNELS] = {};
    double ms[K_NUM_KERNELS] = {};
    double bytes[K_NUM_KERNELS] = {};
    unsigned long long timed[K_NUM_KERNELS] = {};
    cudaEvent_t ev[2 * kPool] = {};
    int pend_id[kPool] = {};
    double pend_bytes[kPool] = {};
    int npend = 0;
    bool ready = false;

    void begin(int id, double algo_bytes, cudaStream_t st) {
        ++launches[id];
        if (!events) return;
        if (!ready) {
            for (int i = 0; i < 2 * kPool; ++i) cudaEventCreate(&ev[i]);
            ready = true;
        }
        if (npend >= kPool) resolve();
        if (npend >= kPool) return;
        pend_id[npend] = id;
        pend_bytes[npend] = algo_bytes;
        cudaEventRecord(ev[2 * npend], st);
    }
    void end(cudaStream_t st) {
        if (!events || !ready || npend >= kPool) return;
        cudaEventRecord(ev[2 * npend + 1], st);
        ++npend;
    }
    // Accumulates the pending launches (waits for their end events).
    void resolve() {
        for (int i = 0; i < npend; ++i) {
            float t = 0.f;
            cudaEventSynchronize(ev[2 * i + 1]);
            cudaEventElapsedTime(&t, ev[2 * i], ev[2 * i + 1]);
            ms[pend_id[i]] += t;
            bytes[pend_id[i]] += pend_bytes[i];
            ++timed[pend_id[i]];
        }
        npend = 0;
    }
    // launches timed together with the one begin() opened (a group of kernels under one id)
    void more_launches(int id, unsigned k) { launches[id] += k; }
    void add_bytes(int id, double b) {
        if (events) bytes[id] += b;
    }
    void reset() {
        resolve();
        for (int i = 0; i < K_NUM_KERNELS; ++i) launches[i] = 0, ms[i] = 0, bytes[i] = 0, timed[i] = 0;
    }
    void destroy() {
        if (ready)
            for (int i = 0; i < 2 * kPool; ++i) cudaEventDestroy(ev[i]);
        ready = false;
    }
};

// A slotted store: row e is live when e % rows < count[e / rows] (tile e / rows of a slotted
// merge wrote count[e / rows] rows at the start of its slot).  count == nullptr: every row
// below n is live (a dense store).
struct SlotMap {
    const unsigned int* count;
    uint32_t rows;
};

template <int W, typename T>
struct RotationArgs {
    const uint64_t* Sk;          // sorted store keys (n rows of 2W words)
    const T* Sc;
    uint64_t n;
    RotLayer<W> L;
    const LevelList* levels;     // all delta bits
    KeepProg keep;
    uint32_t* idx;               // scratch, >= n
    uint16_t* D;                 // scratch, >= n
    int32_t* F;                  // scratch, >= n
    void* slots;                 // level-scan tile values (LevelTile), >= scan tiles
    unsigned long long* status;  // look-back words, >= classify / merge tiles
    ulonglong2* bounds;          // merge-path bounds, >= merge tiles + 1
    uint64_t* Pk;                // partner keys (sorted), capacity p_cap
    T* Pc;
    uint64_t p_cap;
    uint64_t* Ok;                // output store, capacity out_cap
    T* Oc;
    uint64_t out_cap;
    Ctl* ctl;
    unsigned long long* host_count;  // pinned host scratch, >= 16 words
    uint64_t* partners_out;
    uint64_t* out_count;
    unsigned int* err_flags;          // the control block's error bits after the layer
    unsigned int* err_info;
    KernelProf* prof;
    unsigned int* topn_hist;  // when set, the merge histograms its outputs into 2048 bins:
    int topn_hist_mode;       // 0 select key >> 52, 1 octave of |c|^2 (ApproxTopN),
    uint64_t topn_hist_base;  // 2 window_key(select key, topn_hist_base) >> 48
    int inject_stall;         // failure injection: the merge skips its first tile
    int preclassified;        // idx, D and count[0] already hold this layer's partner list (written
                              // by the TopN compaction before it): no classify pass
    RotLayer<W> next_L;       // with next_flags (slotted output only): the next rotation layer,
    uint8_t* next_flags;      // and per output row whether it emits a partner under it
    unsigned int inject_flag;          // failure injection: error bits written after the kernels
    unsigned long long* defer_counts;  // pinned: when set, the counts and error words are copied here
                                       // and the launcher returns without waiting (slotted output: the
                                       // TopN pass reads the span and live count on the device)
    unsigned long long stall_limit;  // ... and its look-back waits give up after this many polls
    unsigned int* slot_count; // when set, the merge writes tile t at rows t * merge_slot_rows<W>()
                              // and its row count to slot_count[t], with no look-back (slotted
                              // output, compacted by the TopN pass that follows); >= merge tiles
    uint64_t* span_out;       // slotted output: rows its slots span
    int sms;                  // multiprocessors of the device (persistent grids)
    const NoiseList* noise;   // host copy of the folded noise channels (nullptr: none)
    const float* Sf;          // the learned pass's predictions: of the store rows (nullptr: none),
    float* Pf;                // of the partners (inherited from their parents),
    float* Of;                // and of the output rows
    unsigned long long* noise_drops;       // device, kMaxNoise + 1: own rows first dropped after channel j
    unsigned long long* host_noise_drops;  // pinned, kMaxNoise + 1: the same, after the layer's sync
};

// Rows of one merge tile's output slot, and the rows a slotted merge of at most `rows_in`
// input rows (own rows plus partners) can span.
template <int W>
uint32_t merge_slot_rows();
template <int W>
uint64_t merge_span_rows(uint64_t rows_in);

template <int W, typename T>
cudaError_t launch_rotation_layer(const RotationArgs<W, T>& a, cudaStream_t st);
template <int W, typename T>
void book_rotation_bytes(KernelProf* prof, uint64_t n, uint64_t m, uint64_t out_count, int nlv, bool classified);
template <int W, typename T>
cudaError_t configure_rotation_kernels();

// General-table layer (branch records for the sort path).
template <int W, typename T>
struct GeneralOps {
    // records the layer emits (synchronizes)
    static cudaError_t count(const uint64_t* keys, uint64_t n, const GenLayer<W, T>& G, Ctl* ctl,
                             unsigned long long* host_count, uint64_t* m, int sms, cudaStream_t st, KernelProf* prof);
    // records (key ^ mask, c * amplitude, own index) in (term, entry) order; status >= tiles words
    static cudaError_t branch(const uint64_t* keys, const T* coef, uint64_t n, const GenLayer<W, T>& G,
                              uint64_t* rkeys, uint32_t* rvals, T* rcoef, uint64_t m_cap,
                              unsigned long long* status, Ctl* ctl, cudaStream_t st, KernelProf* prof);
    static size_t branch_tile();
};

// One level-scan tile's values for both scans of a batch of levels: its aggregates and the
// combined aggregates of the tiles before it (forward scan) and after it (backward scan).
struct LevelTile {
    int agg[4 * kMaxLevels];
    int pre[4 * kMaxLevels];
};

// Rows of the smallest tile of any look-back kernel (bounds every tile count).
constexpr size_t kMinTileRows = 256;
constexpr size_t kScanTileRows = 4096;

}  // namespace psb
