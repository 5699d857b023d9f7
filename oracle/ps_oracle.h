/*
 * ps_oracle.h -- CPU oracle for the Pauli-propagation layer path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference
 * engine's semantics (lkdvos/paulistrings-rs), used by tests/ as the parity
 * checker and by bench.py as the timed CPU baseline.  Nothing in the product
 * library links or calls it.
 *
 * Semantics restated (reference file:line, paths inside the reference repo):
 *   key algebra         crates/paulistrings/src/pauli_string.rs:68-123
 *   real mul_phase      crates/paulistrings/src/coefficient.rs:107-114
 *   rotation apply      crates/paulistrings/src/channel/rotation.rs:43-77
 *   local table probe   crates/paulistrings/src/channel/prepared.rs:214-281, 401-493
 *   PTM channels        crates/paulistrings/src/channel/ptm.rs:126-149 (adjoint), 248-263
 *                       (transfer_matrix), ptm/clifford.rs:10-111, ptm/unitary.rs:13-127,
 *                       ptm/noise.rs:7-80; complex arithmetic as num-complex 0.4
 *                       (mul, add, division by (d, 0)); real conversion with |im| <= 1e-12
 *                       (coefficient.rs:20, 97-99)
 *   naive layer         crates/paulistrings/src/test_support/oracle.rs:21-54
 *   threshold / weight  crates/paulistrings/src/truncation/builtin.rs:28-59
 *   TopN (+NaN, ties)   crates/paulistrings/src/truncation/builtin.rs:73-129, 210-239
 *   ApproxTopN          crates/paulistrings/src/truncation/builtin.rs:240-468 (octave histogram
 *                       with NaN in the top bin, edge walk from the top, boundary quota)
 *   CollapseSample      crates/paulistrings/src/truncation/collapse_sample.rs:1-240 and the
 *                       key-addressed stream of crates/paulistrings/src/rng.rs:1-62; stretches
 *                       accumulated per 1024-term block of the store (the reference's buckets)
 *   And / Or            crates/paulistrings/src/truncation/builtin.rs:479-526, 604-625
 *   Heisenberg order    crates/paulistrings/src/engine/driver.rs:349-352
 *   product readout     crates/paulistrings/src/readout/product_state.rs:84-101
 *
 * Store order: keys sorted lexicographically by (x[0..W), z[0..W)) as unsigned
 * 64-bit words, which is the reference's derived Ord on PauliString
 * (crates/paulistrings/src/pauli_string.rs:1-20).  TopN boundary ties are kept
 * first in this key order (the reference keeps them "first in bucket order" and
 * documents that choice as not a semantic promise).
 */
#ifndef PS_ORACLE_H
#define PS_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PSO_MAX_W 16
#define PSO_F64 0
#define PSO_F32 1

/* keep-program node ops (postfix) */
#define PSO_KEEP_TRUE 0
#define PSO_KEEP_COEFF 1   /* farg = epsilon: keep iff eps < 0 || |c|^2 > eps^2 */
#define PSO_KEEP_WEIGHT 2  /* iarg = k: keep iff weight <= k */
#define PSO_KEEP_AND 3
#define PSO_KEEP_OR 4

/* layer passes */
#define PSO_PASS_TOPN 1    /* n = retained count */
#define PSO_PASS_APPROX_TOPN 3 /* ApproxTopN: octave cut, n = retained count */
#define PSO_PASS_COLLAPSE_SAMPLE 4 /* CollapseSample: above n terms, systematic resample by |c| */

typedef struct pso_policy {
    int32_t num_nodes;
    int32_t op[16];
    int64_t iarg[16];
    double farg[16];
    int32_t num_passes;
    int32_t pass_kind[4];
    uint64_t pass_n[4];
    uint64_t pass_samples[4];  /* CollapseSample: draws per collapse */
    uint64_t pass_seed[4];     /* CollapseSample: trajectory seed */
    uint64_t pass_call[4];     /* CollapseSample: pass index of the first layer */
} pso_policy;

/* channel kinds (same numbers as the product's C ABI) */
#define PSO_CH_ROTATION 1     /* exp(-i theta P / 2); paulis[j] in "XYZ" on qubits[j] */
#define PSO_CH_DEPOLARIZE 2   /* single-qubit depolarizing, param = p */
#define PSO_CH_HADAMARD 3
#define PSO_CH_PHASE 4
#define PSO_CH_PHASE_DAGGER 5
#define PSO_CH_PAULI_X 6
#define PSO_CH_PAULI_Y 7
#define PSO_CH_PAULI_Z 8
#define PSO_CH_CNOT 9         /* qubits[0] control */
#define PSO_CH_CZ 10
#define PSO_CH_SWAP 11
#define PSO_CH_UNITARY 12     /* matrix: 2^k x 2^k complex row-major, re/im interleaved */
#define PSO_CH_DEPHASING 13
#define PSO_CH_PAULI_CHANNEL 14 /* params = px, py, pz */
#define PSO_CH_DEPOLARIZING_2Q 15
#define PSO_CH_AMPLITUDE_DAMPING 16

typedef struct pso_channel {
    int32_t kind;
    int32_t num_support;
    uint32_t qubits[64];
    char paulis[64];
    double param;
    double params[3];
    double matrix[32];
    int32_t adjoint;          /* the channel's own adjoint, composed with the layer direction */
} pso_channel;

typedef struct pso_sum pso_sum;

pso_sum* pso_new(int W, int num_qubits, int dtype);
void pso_free(pso_sum* s);
size_t pso_len(const pso_sum* s);
int pso_width(const pso_sum* s);
/* Replace the contents: duplicates are summed in input order, exact zeros dropped, keys sorted.
 * keys: n rows of 2W words (x words then z words); coeffs: n doubles (rounded to f32 for PSO_F32). */
int pso_set(pso_sum* s, const uint64_t* keys, const double* coeffs, size_t n);
/* Copy out the sorted contents (keys n x 2W, coeffs as doubles). */
void pso_get(const pso_sum* s, uint64_t* keys, double* coeffs);

/* One channel layer (naive: emit, hash-accumulate, keep on sums, drop exact zeros, sort)
 * followed by the policy's layer passes.  adjoint != 0 applies the adjoint channel. */
int pso_apply_channel(pso_sum* s, const pso_channel* ch, int adjoint, const pso_policy* policy);
/* The prepared table of one channel (support, entries ascending by local delta, float64
 * amplitudes amps[16 * e + s]); wide rotations set *wide only.  -1 when the channel is
 * declined. */
int pso_prepare_table(const pso_channel* ch, int adjoint, int W, int nq, int* wide, int* k, uint32_t* qubits,
                      int* num_entries, uint32_t* deltas, double* amps);
/* Test hooks of the key-addressed stream (rng.rs). */
uint64_t pso_splitmix64_first(uint64_t state);
void pso_xoshiro_two(const uint64_t* state4, uint64_t* out2);
double pso_keyed_uniform(uint64_t seed, uint64_t call);
/* CollapseSample collapses performed by this process so far. */
uint64_t pso_collapses(void);
/* The policy's layer passes alone. */
void pso_finalize_layer(pso_sum* s, const pso_policy* policy);
/* The whole circuit; direction 0 = forward, 1 = heisenberg (reverse order, adjoint channels).
 * terms_after (optional, length num_channels) receives the length after each layer. */
int pso_propagate(pso_sum* s, const pso_channel* chans, size_t num_channels, const pso_policy* policy,
                  int direction, uint64_t* terms_after);
/* <psi|O|psi> for the product state given by per-qubit axis bits and sign bits (W words each). */
double pso_expectation(const pso_sum* s, const uint64_t* axis_x, const uint64_t* axis_z,
                       const uint64_t* negative);

/* Sorted-store CPU engine in the reference host engine's shape (rotation scan, linear
 * partner order, merge-join; OpenMP over chunks).  Same results as pso_apply_channel.
 * Used only as the timed CPU baseline. */
int pso_apply_channel_sorted(pso_sum* s, const pso_channel* ch, int adjoint, const pso_policy* policy);
int pso_propagate_sorted(pso_sum* s, const pso_channel* chans, size_t num_channels,
                         const pso_policy* policy, int direction, uint64_t* terms_after);
void pso_set_threads(int threads);

#ifdef __cplusplus
}
#endif
#endif
