/*
 * paulistrings_b200.h -- C ABI of the B200 Pauli-propagation layer path.
 *
 * One opaque handle (ps_sum) owns a Pauli sum resident on one CUDA device: a
 * double-buffered store of packed symplectic keys (x words then z words, 16*W
 * bytes per term) plus a coefficient column (float64 or float32), kept sorted by
 * key with unique keys.  All entry points take plain pointers and sizes; no
 * torch or CUDA types cross the boundary.  Every call returns a ps_status; on
 * any error the store keeps the last completed layer and ps_last_error()
 * describes the failure.  One handle per host thread; each handle issues its
 * work on its own CUDA stream.
 *
 * Reference interfaces replaced (paths inside lkdvos/paulistrings-rs):
 *   PauliSum.propagate(..., device=)      crates/paulistrings-py/src/sum.rs:2132-2183
 *   GpuSum upload / to_host               crates/paulistrings/src/engine/gpu/sum.rs:118-253
 *   PartitionBackend::apply_layer         crates/paulistrings/src/engine/backend.rs:80
 *   PartitionBackend::finalize_layer      crates/paulistrings/src/engine/backend.rs:90
 *   PartitionStorage::{len, settle}       crates/paulistrings/src/engine/backend.rs:26-72
 *   Channel::prepare_for_layer / Prepared crates/paulistrings/src/channel/prepared.rs:345-350, 401-493
 *   KeepProgram (lowered policy)          crates/paulistrings/src/engine/gpu/truncation.rs:24-102
 *   run_layers (the layer loop)           crates/paulistrings/src/engine/driver.rs:319-592
 *   expectation_product                   crates/paulistrings/src/readout/product_state.rs:84-101
 */
#ifndef PAULISTRINGS_B200_H
#define PAULISTRINGS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PS_ABI_VERSION 1
#define PS_MAX_W 16          /* up to 1024 qubits, as the reference's widest monomorphization */
#define PS_MAX_ENTRIES 16    /* 4^2 local deltas of a two-qubit table */
#define PS_MAX_KEEP_NODES 15 /* as the reference's KeepProgram */
#define PS_MAX_PASSES 4

/* Status codes (GpuError variants, crates/paulistrings/src/engine/gpu/error.rs:9). */
typedef enum ps_status {
    PS_OK = 0,
    PS_ERR_OOM = 1,          /* device allocation failed; store unchanged */
    PS_ERR_UNSUPPORTED = 2,  /* channel or policy the device path does not run */
    PS_ERR_INVALID = 3,      /* bad argument (qubit out of range, bad dtype, NULL) */
    PS_ERR_DEVICE = 4,       /* CUDA error */
    PS_ERR_TIMEOUT = 5,      /* a bounded device-side wait gave up */
    PS_ERR_NO_DEVICE = 6     /* no CUDA device, or the ordinal does not exist */
} ps_status;

typedef enum ps_dtype { PS_F64 = 0, PS_F32 = 1 } ps_dtype;
typedef enum ps_direction { PS_FORWARD = 0, PS_HEISENBERG = 1 } ps_direction;

/* ---- policy: keep program (postfix) + ordered layer passes ------------------------
 * Lowered form of a BuiltinTruncation tree (crates/paulistrings/src/truncation/tree.rs:20-39):
 * And(a, b) keeps iff both keep and runs a's passes then b's; Or(a, b) takes per-term
 * filters only.  An empty program keeps every nonzero term. */
typedef enum ps_keep_op {
    PS_KEEP_TRUE = 0,
    PS_KEEP_COEFF = 1,   /* farg = epsilon: keep iff eps < 0 || |c|^2 > eps^2 (builtin.rs:28-31) */
    PS_KEEP_WEIGHT = 2,  /* iarg = k: keep iff Pauli weight <= k (builtin.rs:50-59) */
    PS_KEEP_AND = 3,
    PS_KEEP_OR = 4
} ps_keep_op;

typedef enum ps_pass_kind {
    PS_PASS_NONE = 0,
    PS_PASS_TOPN = 1,    /* keep the n largest |c|^2; ties first in key order (builtin.rs:73-129) */
    PS_PASS_SCORED_TOPN = 2, /* keep the n terms the handle's scorer ranks highest (ps_set_scorer);
                               ties first in key order, a NaN score never kept.  samples > 1 (a
                               residual scorer, the only pass of the policy): the scorer predicts
                               for every term only every `samples` layers; in between, each term
                               carries its prediction f (a partner its parent's) and ranks by
                               log|c| + f inside the layer's merge and select */
    PS_PASS_APPROX_TOPN = 3, /* ApproxTopN (builtin.rs:240-468): every octave of |c|^2 above the
                               boundary octave kept whole, then the first of the boundary octave
                               in key order up to n in all; a NaN never kept */
    PS_PASS_COLLAPSE_SAMPLE = 4 /* CollapseSample (collapse_sample.rs:1-240): above n terms, `samples`
                               systematic draws in proportion to |c| (one uniform from the
                               xoshiro256++ stream keyed (seed, call)); a drawn term keeps
                               sign(c) * multiplicity * sum|c| / samples.  Stretches accumulate in
                               key order per block of 1024 terms, as the reference accumulates
                               per bucket (target_bucket_len 1024). */
} ps_pass_kind;

typedef struct ps_keep_node {
    int32_t op;          /* ps_keep_op */
    int32_t reserved;
    int64_t iarg;
    double farg;
} ps_keep_node;

typedef struct ps_pass {
    int32_t kind;        /* ps_pass_kind */
    int32_t reserved;
    uint64_t n;          /* TopN / ApproxTopN / scored: terms kept; CollapseSample: the cache */
    uint64_t samples;    /* CollapseSample: draws per collapse (>= 1) */
    uint64_t seed;       /* CollapseSample: trajectory seed */
    uint64_t call;       /* CollapseSample: pass index of the first layer; ps_propagate's layer
                            i uses call + i, as the reference's policy counts its passes */
} ps_pass;

typedef struct ps_policy {
    int32_t num_nodes;
    int32_t num_passes;
    ps_keep_node nodes[PS_MAX_KEEP_NODES];
    ps_pass passes[PS_MAX_PASSES];
} ps_policy;

/* ---- channels (the Channel plug-in's built-ins, crates/paulistrings-py/src/circuit.rs:232-345,
 * crates/paulistrings/src/channel/ptm/{clifford,unitary,noise}.rs) */
typedef enum ps_channel_kind {
    PS_CH_PAULI_ROTATION = 1,    /* exp(-i param P / 2), P = paulis[j] ('X','Y','Z') on qubits[j] */
    PS_CH_DEPOLARIZING = 2,      /* one qubit, param = p: X, Y, Z scaled by 1 - 4p/3 (ptm/noise.rs:12-16) */
    PS_CH_HADAMARD = 3,          /* X -> Z, Z -> X, Y -> -Y */
    PS_CH_PHASE = 4,             /* S: X -> Y, Y -> -X */
    PS_CH_PHASE_DAGGER = 5,      /* S^dagger: X -> -Y, Y -> X */
    PS_CH_PAULI_X = 6,
    PS_CH_PAULI_Y = 7,
    PS_CH_PAULI_Z = 8,
    PS_CH_CNOT = 9,              /* qubits[0] control, qubits[1] target */
    PS_CH_CZ = 10,
    PS_CH_SWAP = 11,
    PS_CH_UNITARY = 12,          /* matrix: 2^k x 2^k complex, row-major, re/im interleaved, qubits[0] the
                                    more significant tensor factor; k = num_support in {1, 2} */
    PS_CH_DEPHASING = 13,        /* param = p: X, Y scaled by 1 - 2p */
    PS_CH_PAULI_CHANNEL = 14,    /* params = (px, py, pz) */
    PS_CH_DEPOLARIZING_2Q = 15,  /* two qubits, param = p: every non-identity Pauli scaled by 1 - 16p/15 */
    PS_CH_AMPLITUDE_DAMPING = 16 /* param = gamma */
} ps_channel_kind;

typedef struct ps_channel {
    int32_t kind;             /* ps_channel_kind */
    int32_t num_support;
    const uint32_t* qubits;
    const char* paulis;       /* PS_CH_PAULI_ROTATION: num_support characters */
    double param;
    const double* matrix;     /* PS_CH_UNITARY only */
    double params[3];         /* PS_CH_PAULI_CHANNEL only */
    int32_t adjoint;          /* nonzero: the channel's adjoint (PtmChannel::adjoint, ptm.rs:126-149;
                                 a rotation's negated angle), composed with the layer direction */
    int32_t reserved;
} ps_channel;

/* ---- prepared per-layer table (Prepared, crates/paulistrings/src/channel/prepared.rs:345-350) */
typedef enum ps_table_mode {
    PS_TABLE_LOCAL = 1,       /* LocalPtm: support <= 2 qubits, entries grouped by key delta */
    PS_TABLE_ROTATION = 2     /* PreparedRotation: wide generator, amplitudes per term */
} ps_table_mode;

typedef struct ps_table_entry {
    uint32_t local_delta;     /* bit 2j = x-bit of support qubit j, bit 2j+1 its z-bit */
    uint32_t reserved;
    uint64_t mask_x[PS_MAX_W];
    uint64_t mask_z[PS_MAX_W];
    double amplitude[PS_MAX_ENTRIES]; /* amplitude[s]: support pattern s -> s ^ local_delta */
} ps_table_entry;

typedef struct ps_table {
    int32_t mode;             /* ps_table_mode */
    int32_t k;                /* LOCAL: number of support qubits (0..2) */
    uint32_t qubits[2];       /* LOCAL: support qubits, ascending */
    int32_t num_entries;      /* LOCAL: ascending by local_delta; identity first when present */
    int32_t width;            /* W the masks are meaningful for */
    ps_table_entry entries[PS_MAX_ENTRIES];
    uint64_t gen_x[PS_MAX_W]; /* ROTATION: generator */
    uint64_t gen_z[PS_MAX_W];
    double cos_theta;         /* ROTATION: snapped cos/sin of the applied angle (rotation.rs:70-77) */
    double sin_theta;
} ps_table;

/* ---- per-layer and per-run statistics (PartitionTrace rows, engine/trace.rs:110-139) */
typedef enum ps_layer_path {
    PS_PATH_RESCALE = 1,      /* key-preserving rescale + keep */
    PS_PATH_ROTATION = 2,     /* partner reorder + merge-path join */
    PS_PATH_SORT = 3          /* general table: branch records + radix sort + segmented dedup */
} ps_layer_path;

typedef struct ps_layer_stats {
    uint64_t terms_in;
    uint64_t partners;        /* rows emitted besides each term's own row */
    uint64_t terms_out;       /* after the keep program */
    uint64_t terms_after_passes;
    int32_t path;             /* ps_layer_path */
    int32_t reserved;
} ps_layer_stats;

typedef struct ps_run_stats {
    uint64_t layers;
    uint64_t peak_terms;
    uint64_t final_terms;
    uint64_t total_terms_in;  /* sum over layers of terms_in */
    uint64_t kernel_launches; /* kernels this call launched */
    double device_ms;         /* CUDA-event time of the whole run */
    uint64_t collapses;       /* CollapseSample collapses performed */
    uint64_t layers_skipped;  /* layers that changed nothing and launched nothing: the table acts
                                 on qubits no term touches, maps the identity there to itself,
                                 and every term already passed the same keep program */
    uint64_t skipped_terms_in;/* sum of terms_in over those layers */
} ps_run_stats;

/* Per-kernel profile (the phase-timing counters, crates/paulistrings/src/engine/stats.rs:12 and
 * the device layer's CUDA events, engine/gpu/layer.rs:345-386): launches are always counted;
 * with profiling on, every launch is timed with CUDA events on the handle's stream and its
 * algorithmic bytes (reads + writes the kernel must do at its input/output sizes) are booked. */
typedef struct ps_kernel_profile {
    char name[32];
    uint64_t launches;
    uint64_t timed_launches;
    double total_ms;
    double algorithmic_bytes;
} ps_kernel_profile;

typedef struct ps_sum ps_sum;

/* Version of this ABI (PS_ABI_VERSION). */
int32_t ps_abi_version(void);

/* Number of visible CUDA devices (0 when none).  cuda_available(), python/paulistrings/__init__.py:18-22 */
int32_t ps_device_count(void);

/* Create an empty device sum.  GpuSum::from_host_with_options, engine/gpu/sum.rs:118-212.
 * num_qubits <= 64 * PS_MAX_W; the width W is the smallest of 1, 2, 4, 8, 16 that fits. */
ps_status ps_create(int32_t device, int32_t num_qubits, int32_t dtype, ps_sum** out);
ps_status ps_destroy(ps_sum* sum);
const char* ps_last_error(const ps_sum* sum);
int32_t ps_width(const ps_sum* sum);
int32_t ps_num_qubits(const ps_sum* sum);
int32_t ps_dtype_of(const ps_sum* sum);

/* Replace the contents from host arrays: x and z are n x W words (row-major), coeffs n doubles
 * (rounded once to float for PS_F32).  Duplicate keys are summed in input order and exact zeros
 * dropped (BuildAccumulator::finalize, crates/paulistrings/src/pauli_sum/accumulator.rs:35-56);
 * keys beyond num_qubits are rejected with PS_ERR_INVALID. */
ps_status ps_upload(ps_sum* sum, const uint64_t* x, const uint64_t* z, const double* coeffs, uint64_t n);

/* Number of terms (synchronizes the handle's stream).  PartitionStorage::exact_len. */
ps_status ps_len(ps_sum* sum, uint64_t* n);

/* Copy the sorted contents to host arrays of capacity cap (x, z: cap x W words; coeffs: cap
 * doubles).  *n receives the term count; PS_ERR_INVALID if cap < count.  GpuSum::to_host. */
ps_status ps_download(ps_sum* sum, uint64_t* x, uint64_t* z, double* coeffs, uint64_t cap, uint64_t* n);

/* Host-side table builder: a channel's per-layer engine form for this width and dtype, adjoint
 * when direction is Heisenberg.  Prepared::derive_local / PauliRotation::prepare_for_layer,
 * crates/paulistrings/src/channel/rotation.rs:105-124 and prepared.rs:214-233, 401-493. */
ps_status ps_prepare_channel(int32_t num_qubits, int32_t dtype, const ps_channel* channel, int32_t adjoint,
                             ps_table* out);

/* Apply one prepared layer and the keep program: every term's outputs are emitted, equal keys
 * summed, exact zeros and keep rejects dropped.  PartitionBackend::apply_layer. */
ps_status ps_apply_layer(ps_sum* sum, const ps_table* table, const ps_policy* policy, ps_layer_stats* stats);

/* Run the policy's layer passes (TopN).  PartitionBackend::finalize_layer. */
ps_status ps_finalize_layer(ps_sum* sum, const ps_policy* policy);

/* The whole layer loop: channels in order (forward) or reversed with adjoints (Heisenberg),
 * each applied then finalized.  run_layers, engine/driver.rs:319-592.  terms_after (optional,
 * num_channels entries) receives each layer's final length. */
ps_status ps_propagate(ps_sum* sum, const ps_channel* channels, uint64_t num_channels, const ps_policy* policy,
                       int32_t direction, uint64_t* terms_after, ps_run_stats* stats);

/* <psi|O|psi> in a product state: per qubit an axis (x-bit, z-bit of the axis Pauli) and a sign
 * bit (1 = the -1 eigenstate); W words each.  Summed in float64 on the device.
 * PauliSum::expectation_product, readout/product_state.rs:84-101. */
ps_status ps_expectation(ps_sum* sum, const uint64_t* axis_x, const uint64_t* axis_z, const uint64_t* negative,
                         double* out);

/* Turn per-kernel CUDA-event timing on or off; clears the profile.  PhaseStats, engine/stats.rs:12. */
ps_status ps_set_profiling(ps_sum* sum, int32_t enabled);

/* Copy up to cap kernel records; *count receives the number of kernels profiled. */
ps_status ps_read_profile(ps_sum* sum, ps_kernel_profile* out, int32_t cap, int32_t* count);

/* Largest n ps_expectation_device_noalloc accepts (its scratch holds one partial per 16,384 terms). */
#define PS_NOALLOC_MAX_TERMS (1ull << 30)

/* The product-state expectation (as ps_expectation) of a sum the caller already holds in device
 * memory, for callers that cannot allocate device memory themselves (a framework that owns the
 * GPU's memory through its own pool, a service that forbids allocation after start-up).  This
 * entry point allocates nothing: its scratch is a fixed 512 KiB device array inside the library,
 * held by every GPU that loads it until the process exits.  keys: n rows of 2*width u64 (x words
 * then z words) in device memory; coeffs: n float64 or float32 (dtype) in device memory; the
 * axis/sign masks are host arrays of width words; out: one float64 in device memory, written on
 * `stream` (a cudaStream_t, NULL for the default stream).  keys must be 16-byte aligned, coeffs
 * aligned to its element size and out to 8 bytes; a pointer off those boundaries, or n above
 * PS_NOALLOC_MAX_TERMS, is rejected with PS_ERR_INVALID before anything is launched.  The first
 * call on each device looks up the scratch address, which (with the CUDA runtime's lazy module
 * loading) is also when the library's module is loaded on that device and the array reserved:
 * make that first call at start-up, before any stream capture.  Calls on one device share the
 * scratch, so calls that overlap on the GPU race.  It has no counterpart in the reference. */
ps_status ps_expectation_device_noalloc(const uint64_t* keys, const void* coeffs, int32_t dtype, int32_t width,
                                        uint64_t n, const uint64_t* axis_x, const uint64_t* axis_z,
                                        const uint64_t* negative, double* out, void* stream);

/* Failure injection for tests (FaultPlan, crates/paulistrings/src/engine/gpu/partition.rs:33-45),
 * host-side only.  PS_FAULT_OOM: after `arg` more device allocations of this handle succeed,
 * every further one fails as if the device were out of memory, until PS_FAULT_NONE.  PS_FAULT_STALL: the next layer's
 * merge skips its first tile, so the following tile's output-offset wait sees a flag nothing
 * sets and gives up after `arg` polls (0: the default limit), reporting PS_ERR_TIMEOUT; the
 * shortened limit applies to that merge's output-offset waits only, and every other bounded
 * wait keeps the default.  PS_FAULT_FLAG: the next rotation layer's device error word is set
 * from the host, in stream order after its kernels, as a failed device check would set it
 * (`arg`: the flag bits, 0 for an internal-check failure); the layer reports PS_ERR_DEVICE (or
 * PS_ERR_TIMEOUT for the timeout bit), including a layer whose TopN pass was already queued
 * behind it.  PS_FAULT_NONE disarms them all.  Either way the layer fails and the store keeps
 * the last completed layer. */
typedef enum ps_fault_kind { PS_FAULT_NONE = 0, PS_FAULT_OOM = 1, PS_FAULT_STALL = 2, PS_FAULT_FLAG = 3 } ps_fault_kind;
ps_status ps_inject_fault(ps_sum* sum, int32_t kind, uint64_t arg);

/* Wait for the handle's stream.  PartitionStorage::settle. */
ps_status ps_synchronize(ps_sum* sum);

/* ---- learned truncation -------------------------------------------------------------
 * A scorer is a small MLP implementing a TruncationPolicy layer pass (the TruncationPolicy
 * trait, crates/paulistrings/src/truncation/mod.rs:30-107; no built-in counterpart in the
 * reference): from a term's per-qubit I/X/Y/Z code, its Pauli weight, log|c| and the remaining
 * depth it predicts log of the magnitude the term's descendants contribute to the final
 * expectation.  Architecture: one-hot (num_qubits x 4) + 3 scalar features -> 128 -> GELU ->
 * 128 -> GELU -> 1, BF16 weights, FP32 accumulation, the 128 x 128 layer on the tensor cores.
 * Parameters (fp32, this order): embed[num_qubits][3][128] (rows for X, Z, Y: local index
 * x | z << 1, minus one; the identity's one-hot column is folded into b1), u[3][128] (weight,
 * log|c|, remaining-depth columns), b1[128], w2[128][128] (in, out), b2[128], w3[128], b3.
 * Scalar features enter as weight * s0, log|c| * s1 and remaining * s2, with
 * remaining = layers still to apply / layers_per_unit. */
typedef struct ps_scorer ps_scorer;

typedef struct ps_scorer_config {
    int32_t num_qubits;       /* <= 256 */
    int32_t residual;         /* nonzero: the score is log|c| + the network's output (the network
                                 predicts the descendants' factor; train it on target - log|c|) */
    double layers_per_unit;   /* layers per unit of the remaining-depth feature (e.g. per Trotter step) */
    float feature_scale[3];   /* s0, s1, s2 */
    float init_scale;         /* standard deviation of the initial embedding and u weights */
    uint64_t seed;            /* initial weights (splitmix64 + Box-Muller) */
} ps_scorer_config;

ps_status ps_scorer_create(int32_t device, const ps_scorer_config* config, ps_scorer** out);
ps_status ps_scorer_destroy(ps_scorer* scorer);
const char* ps_scorer_last_error(const ps_scorer* scorer);
uint64_t ps_scorer_num_params(const ps_scorer* scorer);
ps_status ps_scorer_get_params(ps_scorer* scorer, float* out);      /* fp32 master weights */
ps_status ps_scorer_set_params(ps_scorer* scorer, const float* in);
/* Scores of n terms (keys: n rows of 2W words, x words then z words, W the scorer's width). */
ps_status ps_scorer_score(ps_scorer* scorer, const uint64_t* keys, const float* log_abs_c, const float* remaining,
                          uint64_t n, float* out);
/* Gradients of the mean squared error sum((y - target)^2) / n over one batch (n <= 65536),
 * without updating; *loss = that mean.  For checking the backward kernels. */
ps_status ps_scorer_gradients(ps_scorer* scorer, const uint64_t* keys, const float* log_abs_c, const float* remaining,
                              const float* target, uint64_t n, float* grads_out, float* loss);
/* Adam (beta 0.9 / 0.999, eps 1e-8) over shuffled minibatches of `batch` terms for `epochs`
 * passes; epoch_loss[e] = mean squared error over epoch e (optional). */
ps_status ps_scorer_train(ps_scorer* scorer, const uint64_t* keys, const float* log_abs_c, const float* remaining,
                          const float* target, uint64_t n, int32_t epochs, int32_t batch, float learning_rate,
                          float* epoch_loss);
/* Score sums of num_sites qubits (<= 256) with this scorer's embedding rows: site q of a term
 * adds embedding row row_of_site[q] (-1: the site is not an input), so one scorer trained on a
 * small register serves a larger one (e.g. a window of rows around the observable's site, the
 * sites beyond it clamped to the window's edge rows).  The weight, log|c| and remaining-depth
 * features are unchanged (the weight counts every site).  num_sites 0 or a NULL map restores
 * the identity (site q uses row q).  Training refuses a mapped scorer: its rows are the
 * embedding rows' own qubits.  No counterpart in the reference, which has no learned policy. */
ps_status ps_scorer_set_site_map(ps_scorer* scorer, int32_t num_sites, const int32_t* row_of_site);
/* Attach a scorer for PS_PASS_SCORED_TOPN passes; remaining_layers = layers still to apply.
 * Each ps_finalize_layer (and each layer of ps_propagate) first counts one layer down, then
 * scores with the remaining depth that is left.  NULL detaches. */
ps_status ps_set_scorer(ps_sum* sum, ps_scorer* scorer, double remaining_layers);

/* Sum each output key's contributions on the sort path (general tables, three or more
 * contributions per key) with TwoSum compensation: the rounding error of every addition is
 * carried and added back once at the end of the run.  Off by default, which adds in plain
 * arithmetic in the order of the reference's layer.  No counterpart in the reference; meant
 * for PS_F32 sums, where it keeps dense-table layers close to a float64 run.  The rotation and
 * rescale paths add at most two contributions per key, where compensation changes nothing. */
ps_status ps_set_compensated_sums(ps_sum* sum, int32_t enabled);

#ifdef __cplusplus
}
#endif
#endif
