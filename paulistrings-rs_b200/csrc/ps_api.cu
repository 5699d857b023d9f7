// ps_api.cu -- the C ABI (include/paulistrings_b200.h): device store, table builder,
// layer dispatch and the layer loop.
//
// The store is double-buffered: a layer reads the current buffer and writes the spare,
// and the handle flips to the spare only when every kernel of the layer finished without
// a device-side error, so a failed layer leaves the last completed layer in place
// (crates/paulistrings/src/engine/gpu/driver.rs:44).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/paulistrings_b200.h"
#include "ps_device.cuh"
#include "ps_kernels.h"
#include "ps_scorer.h"
#include "ps_store.h"

using namespace psb;

namespace {

constexpr size_t kPad = 256;  // tail slack of every buffer (bulk copies read up to 15 bytes past the end)

struct Buf {
    void* p = nullptr;
    size_t bytes = 0;
};

}  // namespace

struct ps_scorer {
    int device = 0;
    int nq = 0;
    int W = 1;
    int num_sites = 0;     // qubits of the sums it scores (nq unless a site map is set)
    int key_W = 1;         // their width
    Buf site_map;          // int16 embedding row per site (set by ps_scorer_set_site_map)
    bool mapped = false;
    int sms = 148;
    ps_scorer_config cfg{};
    ScorerLayout L{};
    cudaStream_t stream = nullptr;
    Ctl* ctl = nullptr;
    Buf master, bf, grads, m, v;                                   // parameters, Adam state
    Buf keys, logc, rem, target, h1, gz1, dz2, scores, loss;        // batch staging
    int step = 0;
    KernelProf prof;
    std::string err;
};

struct ps_sum {
    int device = 0;
    int nq = 0;
    int W = 1;
    int dtype = PS_F64;
    int sms = 148;
    cudaStream_t stream = nullptr;
    Ctl* ctl = nullptr;
    unsigned long long* hcount = nullptr;  // pinned
    double* hout = nullptr;                // pinned
    Buf keys[2], coef[2];
    uint64_t cap[2] = {0, 0};
    int cur = 0;
    uint64_t n = 0;
    Buf pk, pc;
    Buf idx, dv, fv, slots, status, bounds, hist, cand, partial, dout;
    bool hist_ready = false;  // hist holds the TopN digit-1 histogram of the current store
    int hist_kind = 0;        // ... of that pass kind: PS_PASS_TOPN or PS_PASS_APPROX_TOPN
    bool hist_window = false; // ... binned in the TopN window starting at hist_base
    uint64_t hist_base = 0;
    bool topn_window = false; // the next TopN histogram may use the window at topn_base, centred
    uint64_t topn_base = 0;   // on the last boundary (the boundary moves little between layers)
    unsigned int* hhist = nullptr;  // pinned, kTopnBins1 words
    bool compensated = false; // sort-path dedup sums runs with TwoSum compensation
    uint64_t pass_call = 0;        // CollapseSample: added to the policy's call (ps_propagate's layer)
    uint64_t collapses = 0;        // CollapseSample collapses performed
    Buf cnorms, cfirst;            // CollapseSample block sums / first points
    double* hnorms = nullptr;      // pinned, hnorms_cap doubles
    uint64_t* hfirst = nullptr;    // pinned, hfirst_cap words
    size_t hnorms_cap = 0, hfirst_cap = 0;
    ps_scorer* scorer = nullptr;   // PS_PASS_SCORED_TOPN
    double scorer_remaining = 0;   // layers still to apply
    Buf sel;                       // scored TopN select keys
    // Inherited scoring (a scored pass with a rescore interval above 1): each row carries the
    // scorer's prediction f (its score is log|c| + f) in fcol[buffer]; partners inherit their
    // parent's; every `interval` layers the scorer predicts afresh for every row.
    Buf fcol[2], pf;
    bool f_valid = false;          // fcol[cur] holds the current rows' predictions
    uint64_t f_age = 0;            // layers since the predictions were made
    bool score_window = false;     // the next score select may bin in the window at score_base
    uint64_t score_base = 0;
    SortScratch sort{};
    Buf sort_status;
    Buf up_x, up_z, up_c, up_k, up_v0, up_v1, up_c0, up_st;  // ingest / readout staging, grow-only
    LevelList* levels = nullptr;  // host scratch
    KernelProf prof;
    // Light-cone skip: `support` holds a superset of the qubits any term touches (exact after an
    // upload, widened by each layer's support), and keep_clean says every term already passed
    // the keep program clean_keep.  A layer whose support misses `support` and which maps the
    // identity pattern to itself with amplitude 1 leaves every term as it is; with the same keep
    // program it changes nothing and is skipped.
    uint64_t support[4] = {0, 0, 0, 0};
    bool support_known = false;
    bool keep_clean = false;
    uint64_t layers_skipped = 0;
    // The TopN compaction classifies its kept rows for the next rotation layer (ps_propagate
    // names that layer's table in next_table while it finalizes a layer); pre_valid: the store
    // of pre_n terms has its partner list for the table pre_table in idx / dv and count[0].
    const ps_table* next_table = nullptr;
    bool pre_valid = false;
    const ps_table* pre_table = nullptr;
    uint64_t pre_n = 0;
    // the merge before such a TopN pass: each output row's partner test under next_table
    Buf nflag;
    bool nflag_valid = false;
    const ps_table* nflag_table = nullptr;
    LevelList* levels_next = nullptr;  // host scratch for the next layer's table
    // A rotation layer whose plain TopN pass follows at once (inside ps_propagate) does not wait
    // for its counts: the pass reads the span and live count on the device, and one
    // synchronization after it serves both.  def_*: what the pass needs to finish the layer.
    unsigned int fault_flag = 0;  // PS_FAULT_FLAG: error bits the next rotation layer reports
    bool in_propagate = false;
    bool deferred = false;
    int def_prev_cur = 0;
    uint64_t def_n_in = 0;
    int def_nlv = 0;
    bool def_classified = false;
    bool def_flags = false;
    ps_layer_stats* def_stats = nullptr;
    Buf noise_drops;                      // folded noise: own rows first dropped after channel j
    unsigned long long* hnoise = nullptr; // pinned, kMaxNoise + 1 words
    KeepProg clean_keep{};
    long long fault_oom_after = -1;   // failure injection: allocations left before all fail
    bool fault_stall = false;         // failure injection: next merge skips its first tile
    unsigned long long stall_limit = 0;  // ... and its output-offset waits give up after this many polls
    // Slotted store: the last merge left each tile's rows at the start of a fixed slot of
    // slot_rows rows (n = the slots' span, live_n = rows in them) for the TopN pass that follows
    // to compact; every other reader compacts it first (Engine::densify).
    bool slotted = false;
    uint64_t live_n = 0;
    uint32_t slot_rows = 0;
    Buf slot_count;
    std::string err;
};

namespace {


ps_status set_err(ps_sum* s, ps_status st, const std::string& msg) {
    if (s) s->err = msg;
    return st;
}

ps_status cuda_fail(ps_sum* s, cudaError_t e, const char* where) {
    ps_status st = (e == cudaErrorMemoryAllocation) ? PS_ERR_OOM : PS_ERR_DEVICE;
    if (e == cudaErrorMemoryAllocation) cudaGetLastError();  // clear the sticky-free allocation error
    return set_err(s, st, std::string(where) + ": " + cudaGetErrorString(e));
}

// Grow-only buffer; contents are not preserved.  A buffer that must grow grows by half again
// at least (exactly to the request when that much does not fit), so a sum that grows a little
// every layer does not free and allocate -- two device-wide synchronizations -- every layer.
cudaError_t ensure(Buf& b, size_t bytes) {
    if (b.bytes >= bytes && b.p) return cudaSuccess;
    size_t cap = b.p && b.bytes ? std::max(bytes, b.bytes + b.bytes / 2) : bytes;
    if (b.p) cudaFree(b.p);
    b.p = nullptr;
    b.bytes = 0;
    cudaError_t e = cudaMalloc(&b.p, cap + kPad);
    if (e == cudaErrorMemoryAllocation && cap > bytes) {
        cudaGetLastError();
        cap = bytes;
        e = cudaMalloc(&b.p, cap + kPad);
    }
    if (e != cudaSuccess) {
        b.p = nullptr;
        return e;
    }
    b.bytes = cap;
    return cudaSuccess;
}

// ensure() through the handle, so an injected allocation failure can take its place.
cudaError_t ensure(ps_sum* s, Buf& b, size_t bytes) {
    if (b.bytes >= bytes && b.p) return cudaSuccess;
    if (s->fault_oom_after >= 0) {
        if (s->fault_oom_after == 0) return cudaErrorMemoryAllocation;  // until disarmed
        --s->fault_oom_after;
    }
    return ensure(b, bytes);
}

void release(Buf& b) {
    if (b.p) cudaFree(b.p);
    b.p = nullptr;
    b.bytes = 0;
}

int width_for(int nq) {
    for (int w : {1, 2, 4, 8, 16})
        if (nq <= 64 * w) return w;
    return 0;
}

// Status of device-side error flags already read back; clears them on the device when set.
ps_status flags_status(ps_sum* s, unsigned int flags, unsigned int info, const char* where) {
    if (flags == 0) return PS_OK;
    cudaMemsetAsync(&s->ctl->err, 0, 2 * sizeof(unsigned int), s->stream);
    cudaStreamSynchronize(s->stream);
    char msg[160];
    if (flags & ERR_KEY_RANGE) {
        snprintf(msg, sizeof msg, "%s: a key has a bit at or above num_qubits=%d", where, s->nq);
        return set_err(s, PS_ERR_INVALID, msg);
    }
    if (flags & ERR_TIMEOUT) {
        snprintf(msg, sizeof msg, "%s: a bounded device wait gave up (check %u)", where, info);
        return set_err(s, PS_ERR_TIMEOUT, msg);
    }
    snprintf(msg, sizeof msg, "%s: device check failed (flags %u, check %u)", where, flags, info);
    return set_err(s, PS_ERR_DEVICE, msg);
}

// Device-side error flags of the handle (synchronizes).
ps_status check_device_flags(ps_sum* s, const char* where) {
    unsigned int flags[2] = {0, 0};
    cudaError_t e = cudaMemcpyAsync(flags, &s->ctl->err, sizeof(flags), cudaMemcpyDeviceToHost, s->stream);
    if (e == cudaSuccess) e = spin_sync(s->stream);
    if (e != cudaSuccess) return cuda_fail(s, e, where);
    return flags_status(s, flags[0], flags[1], where);
}

// ---------------------------------------------------------------------------
// keep program lowering
// ---------------------------------------------------------------------------
ps_status lower_keep(const ps_policy* p, KeepProg& k, std::string& why) {
    std::memset(&k, 0, sizeof k);
    if (!p) return PS_OK;  // fast = 0: keep every nonzero term
    if (p->num_nodes < 0 || p->num_nodes > PS_MAX_KEEP_NODES || p->num_passes < 0 || p->num_passes > PS_MAX_PASSES) {
        why = "policy: bad node or pass count";
        return PS_ERR_INVALID;
    }
    int depth = 0;
    for (int i = 0; i < p->num_nodes; ++i) {
        const ps_keep_node& nd = p->nodes[i];
        k.op[i] = nd.op;
        switch (nd.op) {
        case PS_KEEP_TRUE: ++depth; break;
        case PS_KEEP_COEFF:
            k.eps2[i] = nd.farg < 0.0 ? -1.0 : nd.farg * nd.farg;
            ++depth;
            break;
        case PS_KEEP_WEIGHT:
            if (nd.iarg < 0) {
                why = "policy: negative weight limit";
                return PS_ERR_INVALID;
            }
            k.iarg[i] = nd.iarg;
            ++depth;
            break;
        case PS_KEEP_AND:
        case PS_KEEP_OR:
            if (depth < 2) {
                why = "policy: malformed keep program";
                return PS_ERR_INVALID;
            }
            --depth;
            break;
        default: why = "policy: unknown keep node"; return PS_ERR_UNSUPPORTED;
        }
    }
    if (p->num_nodes && depth != 1) {
        why = "policy: malformed keep program";
        return PS_ERR_INVALID;
    }
    k.n = p->num_nodes;
    // recognise the common programs so kernels skip the interpreter
    k.fast = 4;
    if (k.n == 0 || (k.n == 1 && k.op[0] == PS_KEEP_TRUE)) {
        k.fast = 0;
    } else if (k.n == 1 && k.op[0] == PS_KEEP_COEFF) {
        k.fast = 1;
        k.fast_eps2 = k.eps2[0];
    } else if (k.n == 1 && k.op[0] == PS_KEEP_WEIGHT) {
        k.fast = 2;
        k.fast_k = k.iarg[0];
    } else if (k.n == 3 && k.op[2] == PS_KEEP_AND &&
               ((k.op[0] == PS_KEEP_COEFF && k.op[1] == PS_KEEP_WEIGHT) ||
                (k.op[0] == PS_KEEP_WEIGHT && k.op[1] == PS_KEEP_COEFF))) {
        k.fast = 3;
        const int ci = k.op[0] == PS_KEEP_COEFF ? 0 : 1;
        k.fast_eps2 = k.eps2[ci];
        k.fast_k = k.iarg[1 - ci];
    }
    for (int i = 0; i < p->num_passes; ++i) {
        if (p->passes[i].kind == PS_PASS_COLLAPSE_SAMPLE && p->passes[i].samples == 0) {
            why = "policy: CollapseSample needs at least one sample";
            return PS_ERR_INVALID;
        }
        if (p->passes[i].kind != PS_PASS_TOPN && p->passes[i].kind != PS_PASS_SCORED_TOPN &&
            p->passes[i].kind != PS_PASS_APPROX_TOPN && p->passes[i].kind != PS_PASS_COLLAPSE_SAMPLE &&
            p->passes[i].kind != PS_PASS_NONE) {
            why = "policy: unknown layer pass";
            return PS_ERR_UNSUPPORTED;
        }
    }
    return PS_OK;
}

// ---------------------------------------------------------------------------
// table builder (restates channel/rotation.rs:43-124 and channel/prepared.rs:214-493)
// ---------------------------------------------------------------------------
void sin_cos_snapped(double theta, double& sn, double& cs) {
    const double kSnap = 1e-15;
    double s = std::sin(theta), c = std::cos(theta);
    if (std::fabs(s) < kSnap) {
        sn = 0.0;
        cs = std::isnan(c) ? c : std::copysign(1.0, c);
    } else if (std::fabs(c) < kSnap) {
        sn = std::isnan(s) ? s : std::copysign(1.0, s);
        cs = 0.0;
    } else {
        sn = s;
        cs = c;
    }
}

struct HostKey {
    uint64_t x[PS_MAX_W], z[PS_MAX_W];
};

bool host_anticommutes(const HostKey& a, const uint64_t* gx, const uint64_t* gz, int W) {
    uint64_t f = 0;
    for (int i = 0; i < W; ++i) f ^= (a.x[i] & gz[i]) ^ (a.z[i] & gx[i]);
    return (__builtin_popcountll(f) & 1) != 0;
}

unsigned host_phase(const HostKey& k, const uint64_t* gx, const uint64_t* gz, int W) {
    unsigned d = 0;
    for (int i = 0; i < W; ++i) {
        uint64_t a = k.x[i], b = k.z[i], c = gx[i], e = gz[i];
        d += 2u * __builtin_popcountll(b & c) + __builtin_popcountll(a & b) + __builtin_popcountll(c & e) -
             __builtin_popcountll((a ^ c) & (b ^ e));
    }
    return d & 3u;
}

HostKey lift_local(const ps_table& t, unsigned d) {
    HostKey k;
    std::memset(&k, 0, sizeof k);
    for (int j = 0; j < t.k; ++j) {
        uint32_t q = t.qubits[j];
        if ((d >> (2 * j)) & 1u) k.x[q / 64] |= 1ull << (q % 64);
        if ((d >> (2 * j + 1)) & 1u) k.z[q / 64] |= 1ull << (q % 64);
    }
    return k;
}

unsigned local_bits(const ps_table& t, const HostKey& k) {
    unsigned s = 0;
    for (int j = 0; j < t.k; ++j) {
        uint32_t q = t.qubits[j];
        s |= (unsigned)((k.x[q / 64] >> (q % 64)) & 1u) << (2 * j);
        s |= (unsigned)((k.z[q / 64] >> (q % 64)) & 1u) << (2 * j + 1);
    }
    return s;
}

void push_deltas(ps_table& t, const double (&table)[16][16], int W) {
    int dim = 1 << (2 * t.k);
    bool has[16] = {false};
    for (int s = 0; s < dim; ++s)
        for (int u = 0; u < dim; ++u)
            if (table[s][u] != 0.0) has[s ^ u] = true;
    t.num_entries = 0;
    for (int d = 0; d < dim; ++d) {
        if (!has[d]) continue;
        ps_table_entry& e = t.entries[t.num_entries++];
        std::memset(&e, 0, sizeof e);
        e.local_delta = (uint32_t)d;
        HostKey m = lift_local(t, (unsigned)d);
        for (int w = 0; w < W; ++w) {
            e.mask_x[w] = m.x[w];
            e.mask_z[w] = m.z[w];
        }
        for (int s = 0; s < dim; ++s) e.amplitude[s] = table[s][s ^ d];
    }
}

// ---------------------------------------------------------------------------
// PTM channels (crates/paulistrings/src/channel/ptm.rs:248-263, ptm/clifford.rs,
// ptm/unitary.rs, ptm/noise.rs).  Local index per qubit: x | z << 1 (I 0, X 1, Z 2, Y 3);
// the constructor's first qubit in the low two bits.  ptm[s][t]: input s -> output t in the
// Schroedinger map; the adjoint reads the transpose.
// ---------------------------------------------------------------------------
struct Cx {
    double re, im;
};
inline Cx cmul(Cx a, Cx b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
inline Cx cadd(Cx a, Cx b) { return {a.re + b.re, a.im + b.im}; }

// Pauli matrix of local index (I, X, Z, Y order), 2x2
void pauli_mat(int idx, Cx (&m)[2][2]) {
    const Cx z{0, 0}, o{1, 0}, mo{-1, 0}, i{0, 1}, mi{0, -1};
    switch (idx) {
    case 0: m[0][0] = o; m[0][1] = z; m[1][0] = z; m[1][1] = o; break;
    case 1: m[0][0] = z; m[0][1] = o; m[1][0] = o; m[1][1] = z; break;
    case 2: m[0][0] = o; m[0][1] = z; m[1][0] = z; m[1][1] = mo; break;
    default: m[0][0] = z; m[0][1] = mi; m[1][0] = i; m[1][1] = z; break;
    }
}

// P_s as a 2^k x 2^k matrix; for k = 2, kron(P(s & 3), P(s >> 2)), the first qubit the more
// significant tensor factor (ptm/unitary.rs:42)
void local_pauli(int k, int s, Cx (&m)[4][4]) {
    Cx a[2][2], b[2][2];
    if (k == 1) {
        pauli_mat(s, a);
        for (int r = 0; r < 2; ++r)
            for (int c = 0; c < 2; ++c) m[r][c] = a[r][c];
        return;
    }
    pauli_mat(s & 3, a);
    pauli_mat(s >> 2, b);
    for (int r = 0; r < 4; ++r)
        for (int c = 0; c < 4; ++c) m[r][c] = cmul(a[r / 2][c / 2], b[r % 2][c % 2]);
}

// ptm[s][t] = tr(P_t U P_s U^dagger) / 2^k, parts within 1e-12 of zero snapped to zero
// (ptm/unitary.rs:13-53, 123-127); false if U is not unitary to 1e-10 or an entry is complex.
bool unitary_ptm(int k, const double* mat, double (&ptm)[16][16], std::string& why) {
    const int d = 1 << k, dim = 1 << (2 * k);
    Cx U[4][4], Ud[4][4];
    for (int r = 0; r < d; ++r)
        for (int c = 0; c < d; ++c) {
            U[r][c] = {mat[2 * (r * d + c)], mat[2 * (r * d + c) + 1]};
            if (!std::isfinite(U[r][c].re) || !std::isfinite(U[r][c].im)) {
                why = "unitary: non-finite entry";
                return false;
            }
        }
    for (int r = 0; r < d; ++r)
        for (int c = 0; c < d; ++c) Ud[r][c] = {U[c][r].re, -U[c][r].im};
    double dev = 0.0;
    for (int r = 0; r < d; ++r)
        for (int c = 0; c < d; ++c) {
            Cx acc{0, 0};
            for (int q = 0; q < d; ++q) acc = cadd(acc, cmul(Ud[r][q], U[q][c]));
            acc.re -= (r == c) ? 1.0 : 0.0;
            dev = std::max(dev, std::hypot(acc.re, acc.im));
        }
    if (!(dev <= 1e-10)) {
        why = "unitary: the matrix is not unitary to 1e-10";
        return false;
    }
    for (int s = 0; s < dim; ++s) {
        Cx Ps[4][4], T1[4][4], C[4][4];
        local_pauli(k, s, Ps);
        for (int r = 0; r < d; ++r)
            for (int c = 0; c < d; ++c) {
                Cx acc{0, 0};
                for (int q = 0; q < d; ++q) acc = cadd(acc, cmul(U[r][q], Ps[q][c]));
                T1[r][c] = acc;
            }
        for (int r = 0; r < d; ++r)
            for (int c = 0; c < d; ++c) {
                Cx acc{0, 0};
                for (int q = 0; q < d; ++q) acc = cadd(acc, cmul(T1[r][q], Ud[q][c]));
                C[r][c] = acc;
            }
        for (int t = 0; t < dim; ++t) {
            Cx Pt[4][4];
            local_pauli(k, t, Pt);
            Cx tr{0, 0};
            for (int r = 0; r < d; ++r)
                for (int q = 0; q < d; ++q) tr = cadd(tr, cmul(Pt[r][q], C[q][r]));
            double re = tr.re / d, im = tr.im / d;
            if (std::fabs(re) < 1e-12) re = 0.0;
            if (std::fabs(im) < 1e-12) im = 0.0;
            if (!(std::fabs(im) <= 1e-12)) {  // Coefficient::from_complex64, coefficient.rs:97-99
                why = "unitary: complex transfer-matrix entry (a real coefficient type needs a real PTM)";
                return false;
            }
            ptm[s][t] = re;
        }
    }
    return true;
}

// The named PTM channels as ptm[s][t] in constructor order; k = support size.
bool named_ptm(const ps_channel* ch, int& k, double (&ptm)[16][16], std::string& why) {
    std::memset(ptm, 0, sizeof ptm);
    auto signed_perm_1q = [&](const int (&image)[4], unsigned negated) {
        k = 1;
        for (int s = 0; s < 4; ++s) ptm[s][image[s]] = ((negated >> s) & 1u) ? -1.0 : 1.0;
    };
    auto prob = [&](double v, const char* name) {
        if (!(v >= 0.0 && v <= 1.0)) {
            why = std::string(name) + " must lie in [0, 1]";
            return false;
        }
        return true;
    };
    static const double kCnot[32] = {1, 0, 0, 0, 0, 0, 0, 0, 0, 0, 1, 0, 0, 0, 0, 0,
                                     0, 0, 0, 0, 0, 0, 1, 0, 0, 0, 0, 0, 1, 0, 0, 0};
    static const double kCz[32] = {1, 0, 0, 0, 0, 0, 0, 0, 0, 0, 1, 0, 0, 0, 0, 0,
                                   0, 0, 0, 0, 1, 0, 0, 0, 0, 0, 0, 0, 0, 0, -1, 0};
    static const double kSwap[32] = {1, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 1, 0, 0, 0,
                                     0, 0, 1, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 1, 0};
    switch (ch->kind) {
    case PS_CH_HADAMARD: signed_perm_1q({0, 2, 1, 3}, 0b1000u); return true;
    case PS_CH_PHASE: signed_perm_1q({0, 3, 2, 1}, 0b1000u); return true;
    case PS_CH_PHASE_DAGGER: {  // the transpose of S
        signed_perm_1q({0, 3, 2, 1}, 0b1000u);
        double t[16][16];
        std::memcpy(t, ptm, sizeof t);
        for (int a = 0; a < 4; ++a)
            for (int b = 0; b < 4; ++b) ptm[a][b] = t[b][a];
        return true;
    }
    case PS_CH_PAULI_X: signed_perm_1q({0, 1, 2, 3}, 0b1100u); return true;
    case PS_CH_PAULI_Y: signed_perm_1q({0, 1, 2, 3}, 0b0110u); return true;
    case PS_CH_PAULI_Z: signed_perm_1q({0, 1, 2, 3}, 0b1010u); return true;
    case PS_CH_CNOT: k = 2; return unitary_ptm(2, kCnot, ptm, why);
    case PS_CH_CZ: k = 2; return unitary_ptm(2, kCz, ptm, why);
    case PS_CH_SWAP: k = 2; return unitary_ptm(2, kSwap, ptm, why);
    case PS_CH_UNITARY:
        k = ch->num_support;
        if (k != 1 && k != 2) {
            why = "unitary: one or two qubits";
            return false;
        }
        if (!ch->matrix) {
            why = "unitary: missing matrix";
            return false;
        }
        return unitary_ptm(k, ch->matrix, ptm, why);
    case PS_CH_DEPHASING: {
        if (!prob(ch->param, "dephasing: p")) return false;
        k = 1;
        const double sc = 1.0 - 2.0 * ch->param;
        ptm[0][0] = 1.0;
        ptm[1][1] = sc;
        ptm[2][2] = 1.0;
        ptm[3][3] = sc;
        return true;
    }
    case PS_CH_PAULI_CHANNEL: {
        const double px = ch->params[0], py = ch->params[1], pz = ch->params[2];
        if (!prob(px, "pauli_channel: px") || !prob(py, "pauli_channel: py") || !prob(pz, "pauli_channel: pz"))
            return false;
        if (!(px + py + pz <= 1.0)) {
            why = "pauli_channel: px + py + pz must be at most 1";
            return false;
        }
        k = 1;
        ptm[0][0] = 1.0;
        ptm[1][1] = 1.0 - 2.0 * (py + pz);
        ptm[2][2] = 1.0 - 2.0 * (px + py);
        ptm[3][3] = 1.0 - 2.0 * (px + pz);
        return true;
    }
    case PS_CH_DEPOLARIZING_2Q: {
        if (!prob(ch->param, "depolarizing_2q: p")) return false;
        k = 2;
        const double sc = 1.0 - 16.0 * ch->param / 15.0;
        for (int q = 0; q < 16; ++q) ptm[q][q] = q ? sc : 1.0;
        return true;
    }
    case PS_CH_AMPLITUDE_DAMPING: {
        const double g = ch->param;
        if (!prob(g, "amplitude_damping: gamma")) return false;
        k = 1;
        const double tr = std::sqrt(1.0 - g);
        ptm[0][0] = 1.0;
        ptm[0][2] = g;
        ptm[1][1] = tr;
        ptm[2][2] = 1.0 - g;
        ptm[3][3] = tr;
        return true;
    }
    default: why = "unknown channel kind"; return false;
    }
}

ps_status build_table(int nq, const ps_channel* ch, int adjoint, ps_table* out, std::string& why) {
    const int W = width_for(nq);
    if (!W) {
        why = "num_qubits out of range";
        return PS_ERR_INVALID;
    }
    std::memset(out, 0, sizeof *out);
    out->width = W;
    if (!ch || ch->num_support < 0 || ch->num_support > 64 * PS_MAX_W || (ch->num_support && !ch->qubits)) {
        why = "channel: bad support";
        return PS_ERR_INVALID;
    }
    adjoint = (adjoint != 0) != (ch->adjoint != 0);
    if (ch->kind == PS_CH_PAULI_ROTATION) {
        if (ch->num_support && !ch->paulis) {
            why = "pauli_rotation: missing Pauli labels";
            return PS_ERR_INVALID;
        }
        uint64_t gx[PS_MAX_W] = {0}, gz[PS_MAX_W] = {0};
        for (int j = 0; j < ch->num_support; ++j) {
            uint32_t q = ch->qubits[j];
            if ((int)q >= nq) {
                why = "pauli_rotation: qubit " + std::to_string(q) + " is outside the " + std::to_string(nq) +
                      "-qubit register";
                return PS_ERR_INVALID;
            }
            uint64_t bit = 1ull << (q % 64);
            if ((gx[q / 64] | gz[q / 64]) & bit) {
                why = "pauli_rotation: repeated qubit " + std::to_string(q);
                return PS_ERR_INVALID;
            }
            char p = ch->paulis[j];
            if (p == 'X' || p == 'x')
                gx[q / 64] |= bit;
            else if (p == 'Y' || p == 'y') {
                gx[q / 64] |= bit;
                gz[q / 64] |= bit;
            } else if (p == 'Z' || p == 'z')
                gz[q / 64] |= bit;
            else if (p != 'I' && p != 'i') {
                why = std::string("pauli_rotation: bad Pauli label '") + p + "'";
                return PS_ERR_INVALID;
            }
        }
        if (!std::isfinite(ch->param)) {
            why = "pauli_rotation: angle must be finite";
            return PS_ERR_INVALID;
        }
        double sn, cs;
        sin_cos_snapped(adjoint ? -ch->param : ch->param, sn, cs);
        int weight = 0;
        for (int w = 0; w < W; ++w) weight += __builtin_popcountll(gx[w] | gz[w]);
        if (weight > 2) {
            out->mode = PS_TABLE_ROTATION;
            for (int w = 0; w < W; ++w) {
                out->gen_x[w] = gx[w];
                out->gen_z[w] = gz[w];
            }
            out->cos_theta = cs;
            out->sin_theta = sn;
            return PS_OK;
        }
        out->mode = PS_TABLE_LOCAL;
        int k = 0;
        for (int w = 0; w < W; ++w) {
            uint64_t live = gx[w] | gz[w];
            while (live) {
                out->qubits[k++] = (uint32_t)(64 * w + __builtin_ctzll(live));
                live &= live - 1;
            }
        }
        out->k = k;
        double table[16][16];
        std::memset(table, 0, sizeof table);
        int dim = 1 << (2 * k);
        for (int s = 0; s < dim; ++s) {
            HostKey in = lift_local(*out, (unsigned)s);
            if (!host_anticommutes(in, gx, gz, W)) {
                table[s][s] += 1.0;
                continue;
            }
            table[s][s] += 1.0 * cs;
            unsigned total = (1u + host_phase(in, gx, gz, W)) & 3u;
            HostKey o = in;
            for (int w = 0; w < W; ++w) {
                o.x[w] ^= gx[w];
                o.z[w] ^= gz[w];
            }
            table[s][local_bits(*out, o)] += ((total & 2u) ? -1.0 : 1.0) * sn;
        }
        push_deltas(*out, table, W);
        return PS_OK;
    }
    if (ch->kind == PS_CH_DEPOLARIZING) {
        if (ch->num_support != 1) {
            why = "depolarizing: exactly one qubit";
            return PS_ERR_INVALID;
        }
        if ((int)ch->qubits[0] >= nq) {
            why = "depolarizing: qubit outside the register";
            return PS_ERR_INVALID;
        }
        double p = ch->param;
        if (!(p >= 0.0 && p <= 1.0)) {
            why = "depolarizing: p must lie in [0, 1]";
            return PS_ERR_INVALID;
        }
        double scale = 1.0 - 4.0 * p / 3.0;
        out->mode = PS_TABLE_LOCAL;
        out->k = 1;
        out->qubits[0] = ch->qubits[0];
        double table[16][16];
        std::memset(table, 0, sizeof table);
        table[0][0] = 1.0;
        table[1][1] = scale;
        table[2][2] = scale;
        table[3][3] = scale;
        push_deltas(*out, table, W);
        return PS_OK;
    }
    if (ch->kind >= PS_CH_HADAMARD && ch->kind <= PS_CH_AMPLITUDE_DAMPING) {
        double ptm[16][16];
        int k = 0;
        if (!named_ptm(ch, k, ptm, why)) return PS_ERR_INVALID;
        if (ch->num_support != k) {
            why = "channel: expected " + std::to_string(k) + " qubit(s)";
            return PS_ERR_INVALID;
        }
        for (int j = 0; j < k; ++j)
            if ((int)ch->qubits[j] >= nq) {
                why = "channel: qubit outside the register";
                return PS_ERR_INVALID;
            }
        if (k == 2 && ch->qubits[0] == ch->qubits[1]) {
            why = "channel: the two qubits must differ";
            return PS_ERR_INVALID;
        }
        // transfer_matrix (ptm.rs:248-263): transposed for the adjoint, reordered to
        // ascending-qubit local indices
        const bool reversed = k == 2 && ch->qubits[0] > ch->qubits[1];
        auto reorder = [&](int idx) { return reversed ? (((idx & 3) << 2) | (idx >> 2)) : idx; };
        double table[16][16];
        std::memset(table, 0, sizeof table);
        const int dim = 1 << (2 * k);
        for (int a = 0; a < dim; ++a)
            for (int b = 0; b < dim; ++b) {
                if (ptm[a][b] == 0.0) continue;
                const int row = adjoint ? b : a, col = adjoint ? a : b;
                table[reorder(row)][reorder(col)] += ptm[a][b];
            }
        out->mode = PS_TABLE_LOCAL;
        out->k = k;
        out->qubits[0] = reversed ? ch->qubits[1] : ch->qubits[0];
        out->qubits[1] = k == 2 ? (reversed ? ch->qubits[0] : ch->qubits[1]) : 0;
        push_deltas(*out, table, W);
        return PS_OK;
    }
    why = "unknown channel kind";
    return PS_ERR_UNSUPPORTED;
}

// ---------------------------------------------------------------------------
// table -> device layer
// ---------------------------------------------------------------------------
// Rotation-shaped tables run on the partner path: the identity entry scales every term in
// place and one more entry (delta g) sends some terms to k ^ g, so every output key gets at
// most two contributions and their order cannot change the sum.  The reference takes the
// tables RotationLayer::of accepts (crates/paulistrings/src/engine/bucketed/rotation_layer.rs:
// 101-140) this way; this path also takes the two-entry tables that rule declines only because
// a non-emitting pattern is scaled (Hadamard's Y -> -Y) or a partner is one-sided (amplitude
// damping's Z -> I), which are rotation-shaped in the sense above.  Every other local table
// sets *general and runs on the sort path.
template <int W, typename T>
ps_status to_rot_layer(const ps_table& t, RotLayer<W>& L, LevelList& lv, std::string& why, bool* general) {
    std::memset(&L, 0, sizeof L);
    lv.n = 0;
    *general = false;
    uint64_t dx[W] = {0}, dz[W] = {0};
    if (t.mode == PS_TABLE_ROTATION) {
        L.wide = 1;
        L.partners = t.sin_theta != 0.0 ? 1 : 0;
        for (int w = 0; w < W; ++w) {
            L.gx[w] = dx[w] = t.gen_x[w];
            L.gz[w] = dz[w] = t.gen_z[w];
        }
        L.cos64 = t.cos_theta;
        L.sin64 = t.sin_theta;
        L.cos32 = (float)t.cos_theta;
        L.sin32 = (float)t.sin_theta;
        L.pattern_mask = 0;
    } else if (t.mode == PS_TABLE_LOCAL) {
        if (t.k < 0 || t.k > 2) {
            why = "table: support above two qubits";
            return PS_ERR_INVALID;
        }
        for (int j = 0; j < 2; ++j) {
            uint32_t q = t.qubits[j < t.k ? j : 0];
            if (t.k == 0) q = 0;
            L.qw[j] = (int)(q / 64);
            L.qb[j] = (int)(q % 64);
        }
        L.pattern_mask = (1u << (2 * t.k)) - 1u;
        const int dim = 1 << (2 * t.k);
        if (t.num_entries == 1 && t.entries[0].local_delta == 0) {
            L.partners = 0;
            for (int s = 0; s < 16; ++s) {
                double a = s < dim ? t.entries[0].amplitude[s] : 1.0;
                L.a0[s] = a;
                L.a0f[s] = (float)a;
            }
        } else if (t.num_entries == 2 && t.entries[0].local_delta == 0) {
            const ps_table_entry &e0 = t.entries[0], &e1 = t.entries[1];
            const unsigned delta = e1.local_delta;
            // RotationLayer::of's shape test (bucketed/rotation_layer.rs:101-140), per
            // coefficient type; its Clifford residue rule applies only to the tables it accepts
            bool ref_shaped = true;
            for (int s = 0; s < dim; ++s) {
                T a0 = (T)e0.amplitude[s], a1 = (T)e1.amplitude[s];
                if (a1 == T(0)) {
                    if (a0 != T(1)) ref_shaped = false;
                } else if ((T)e1.amplitude[s ^ delta] == T(0)) {
                    ref_shaped = false;
                }
            }
            bool clifford = ref_shaped;
            const double eps = 2.220446049250313e-16;
            for (int s = 0; s < dim; ++s) {
                double a0 = (double)(T)e0.amplitude[s], a1 = (double)(T)e1.amplitude[s];
                if (a1 != 0.0) clifford = clifford && (a0 * a0 <= eps * eps * (a1 * a1));
            }
            L.partners = 1;
            for (int w = 0; w < W; ++w) {
                L.gx[w] = dx[w] = e1.mask_x[w];
                L.gz[w] = dz[w] = e1.mask_z[w];
            }
            for (int s = 0; s < 16; ++s) {
                double a0 = s < dim ? e0.amplitude[s] : 1.0;
                double a1 = s < dim ? e1.amplitude[s] : 0.0;
                if (clifford && (T)a1 != T(0)) a0 = 0.0;
                L.a0[s] = a0;
                L.a1[s] = a1;
                L.a0f[s] = (float)a0;
                L.a1f[s] = (float)a1;
            }
        } else {
            *general = true;
            return PS_OK;
        }
    } else {
        why = "table: unknown mode";
        return PS_ERR_INVALID;
    }
    if (L.partners) {
        for (int w = 0; w < W; ++w) {
            uint64_t bits = dx[w];
            while (bits) {
                int b = 63 - __builtin_clzll(bits);
                lv.rank[lv.n++] = (uint32_t)(64 * w + (63 - b));
                bits &= ~(1ull << b);
            }
        }
        for (int w = 0; w < W; ++w) {
            uint64_t bits = dz[w];
            while (bits) {
                int b = 63 - __builtin_clzll(bits);
                lv.rank[lv.n++] = (uint32_t)(64 * (W + w) + (63 - b));
                bits &= ~(1ull << b);
            }
        }
    }
    return PS_OK;
}

// A local table as per-pattern record lists (ascending entry order, zero amplitudes in the
// coefficient type skipped, as DeltaEntry::emit skips them).
template <int W, typename T>
void to_gen_layer(const ps_table& t, GenLayer<W, T>& G) {
    std::memset(&G, 0, sizeof G);
    for (int j = 0; j < 2; ++j) {
        uint32_t q = t.k ? t.qubits[j < t.k ? j : 0] : 0;
        G.qw[j] = (int)(q / 64);
        G.qb[j] = (int)(q % 64);
    }
    G.pattern_mask = (1u << (2 * t.k)) - 1u;
    G.num_entries = t.num_entries;
    for (int e = 0; e < t.num_entries; ++e)
        for (int w = 0; w < W; ++w) {
            G.mx[e][w] = t.entries[e].mask_x[w];
            G.mz[e][w] = t.entries[e].mask_z[w];
        }
    const int dim = 1 << (2 * t.k);
    for (int s = 0; s < dim; ++s) {
        int c = 0;
        for (int e = 0; e < t.num_entries; ++e) {
            const T a = (T)t.entries[e].amplitude[s];
            if (a == T(0)) continue;
            G.ent[s][c] = (uint8_t)e;
            G.amp[s][c] = a;
            ++c;
        }
        G.cnt[s] = (uint8_t)c;
    }
}

// The qubits a table acts on, as W words (its generator for a wide rotation).
template <int W>
void table_support(const ps_table& t, uint64_t (&out)[W]) {
    for (int w = 0; w < W; ++w) out[w] = 0;
    if (t.mode == PS_TABLE_ROTATION) {
        for (int w = 0; w < W; ++w) out[w] = t.gen_x[w] | t.gen_z[w];
        return;
    }
    for (int j = 0; j < t.k && j < 2; ++j)
        if (t.qubits[j] < 64u * W) out[t.qubits[j] / 64] |= 1ull << (t.qubits[j] % 64);
}

// The rescore interval of an inherited scored pass (the policy's first and only pass is a
// scored TopN whose `samples` field is above 1, with a residual scorer attached), else 0.
uint64_t inherit_interval(const ps_policy* p, const ps_sum* s) {
    if (!p || p->num_passes != 1 || p->passes[0].kind != PS_PASS_SCORED_TOPN || p->passes[0].samples <= 1) return 0;
    if (!s->scorer || !s->scorer->cfg.residual) return 0;
    return p->passes[0].samples;
}

// ---------------------------------------------------------------------------
// per-width / per-dtype operations
// ---------------------------------------------------------------------------
template <int W, typename T>
struct Engine {
    static constexpr size_t kKeyBytes = 16 * W;

    static cudaError_t reserve_store(ps_sum* s, int which, uint64_t rows) {
        if (s->cap[which] >= rows && s->keys[which].p) return cudaSuccess;
        uint64_t want = rows < 1024 ? 1024 : rows;
        // grow by 1.5x so a slowly growing sum does not reallocate every layer
        if (s->cap[which] && want < s->cap[which] + s->cap[which] / 2) want = s->cap[which] + s->cap[which] / 2;
        cudaError_t e = ensure(s, s->keys[which], want * kKeyBytes);
        if (e == cudaSuccess) e = ensure(s, s->coef[which], want * sizeof(T));
        if (e != cudaSuccess) {
            release(s->keys[which]);
            release(s->coef[which]);
            s->cap[which] = 0;
            cudaGetLastError();
            // retry at the exact size
            want = rows < 1024 ? 1024 : rows;
            e = ensure(s, s->keys[which], want * kKeyBytes);
            if (e == cudaSuccess) e = ensure(s, s->coef[which], want * sizeof(T));
            if (e != cudaSuccess) {
                release(s->keys[which]);
                release(s->coef[which]);
                return e;
            }
        }
        s->cap[which] = want;
        return cudaSuccess;
    }

    static uint64_t* K(ps_sum* s, int w) { return static_cast<uint64_t*>(s->keys[w].p); }
    static float* F(ps_sum* s, int w) { return static_cast<float*>(s->fcol[w].p); }
    // a prediction column as long as store buffer w
    static cudaError_t reserve_f(ps_sum* s, int w) { return ensure(s, s->fcol[w], s->cap[w] * sizeof(float)); }

    // Can this layer be skipped (see ps_sum::support)?  identity0: the table maps the identity
    // pattern to itself alone with amplitude 1.
    static bool skippable(const ps_sum* s, const uint64_t (&lsup)[W], const KeepProg& keep, bool identity0) {
        if (!identity0 || !s->support_known || !s->keep_clean || s->slotted) return false;
        if (std::memcmp(&keep, &s->clean_keep, sizeof keep) != 0) return false;
        for (int w = 0; w < W; ++w)
            if (lsup[w] & s->support[w]) return false;
        return true;
    }
    // A layer ran with keep program `keep`: every term passed it; the support grows by the
    // layer's own (partner rows live on it).
    static void layer_done(ps_sum* s, const uint64_t (&lsup)[W], const KeepProg& keep, bool widens) {
        s->keep_clean = true;
        s->clean_keep = keep;
        if (widens)
            for (int w = 0; w < W; ++w) s->support[w] |= lsup[w];
    }
    static void skipped(ps_sum* s, ps_layer_stats* stats, int path) {
        if (s->hist_ready) {
            cudaMemsetAsync(s->hist.p, 0, kTopnBinsN * sizeof(unsigned int), s->stream);
            s->hist_ready = false;
        }
        if (stats) {
            stats->terms_in = s->n;
            stats->partners = 0;
            stats->terms_out = s->n;
            stats->terms_after_passes = s->n;
            stats->path = path;
        }
        ++s->layers_skipped;
    }
    static T* C(ps_sum* s, int w) { return static_cast<T*>(s->coef[w].p); }

    static ps_status upload(ps_sum* s, const uint64_t* x, const uint64_t* z, const double* c, uint64_t n) {
        if (n >= (1ull << 30)) return set_err(s, PS_ERR_UNSUPPORTED, "upload: at most 2^30 - 1 terms per upload");
        const int spare = 1 - s->cur;
        if (n == 0) {
            s->n = 0;
            s->slotted = false;
            for (int w = 0; w < W; ++w) s->support[w] = 0;
            s->support_known = true;
            s->keep_clean = false;
            s->f_valid = false;
            return PS_OK;
        }
        cudaError_t e = cudaSuccess;
        if ((e = ensure(s, s->up_x, n * W * 8)) != cudaSuccess || (e = ensure(s, s->up_z, n * W * 8)) != cudaSuccess ||
            (e = ensure(s, s->up_c, n * 8)) != cudaSuccess || (e = ensure(s, s->up_v0, n * 4)) != cudaSuccess ||
            (e = reserve_store(s, spare, n)) != cudaSuccess)
            return cuda_fail(s, e, "upload: allocation");
        cudaMemcpyAsync(s->up_x.p, x, n * W * 8, cudaMemcpyHostToDevice, s->stream);
        cudaMemcpyAsync(s->up_z.p, z, n * W * 8, cudaMemcpyHostToDevice, s->stream);
        cudaMemcpyAsync(s->up_c.p, c, n * 8, cudaMemcpyHostToDevice, s->stream);
        // pack straight into the spare store; an input already in store form (sorted, unique,
        // no zeros, as every download is) needs nothing more
        e = StoreOps<W, T>::pack((uint64_t*)s->up_x.p, (uint64_t*)s->up_z.p, (double*)s->up_c.p, n, (uint32_t)s->nq,
                                 K(s, spare), C(s, spare), (uint32_t*)s->up_v0.p, s->ctl, s->sms, s->stream, &s->prof);
        if (e != cudaSuccess) return cuda_fail(s, e, "upload: pack");
        s->support_known = false;
        s->keep_clean = false;
        s->f_valid = false;
        e = cudaMemcpyAsync(s->hcount + 48, &s->ctl->support[0], sizeof(s->ctl->support), cudaMemcpyDeviceToHost,
                            s->stream);
        if (e != cudaSuccess) return cuda_fail(s, e, "upload: support");
        ps_status fs = check_device_flags(s, "upload");  // synchronizes: the support words have landed
        if (fs != PS_OK) return fs;
        for (int w = 0; w < W; ++w) s->support[w] = s->hcount[48 + w];
        s->support_known = true;
        bool sorted = false;
        e = StoreOps<W, T>::check_sorted(K(s, spare), C(s, spare), n, s->ctl, s->hcount, &sorted, s->sms, s->stream,
                                         &s->prof);
        if (e != cudaSuccess) return cuda_fail(s, e, "upload: check");
        uint64_t out_n = n;
        if (!sorted) {
            const size_t tiles = (n + StoreOps<W, T>::sort_tile() - 1) / StoreOps<W, T>::sort_tile();
            if ((e = ensure(s, s->up_k, 2 * n * kKeyBytes)) != cudaSuccess || (e = ensure(s, s->up_v1, n * 4)) != cudaSuccess ||
                (e = ensure(s, s->up_c0, n * sizeof(T))) != cudaSuccess ||
                (e = ensure(s, s->up_st, (n / 2048 + 2) * sizeof(unsigned long long))) != cudaSuccess ||
                (e = ensure(s, s->sort_status, tiles * 256 * sizeof(unsigned int))) != cudaSuccess)
                return cuda_fail(s, e, "upload: sort scratch");
            s->sort.status = static_cast<unsigned int*>(s->sort_status.p);
            uint64_t* k0 = (uint64_t*)s->up_k.p;
            uint64_t* k1 = k0 + n * 2 * W;
            cudaMemcpyAsync(k0, K(s, spare), n * kKeyBytes, cudaMemcpyDeviceToDevice, s->stream);
            cudaMemcpyAsync(s->up_c0.p, C(s, spare), n * sizeof(T), cudaMemcpyDeviceToDevice, s->stream);
            bool alt = false;
            e = StoreOps<W, T>::sort_pairs(k0, (uint32_t*)s->up_v0.p, k1, (uint32_t*)s->up_v1.p, n, s->sort, s->ctl,
                                           s->sms, s->stream, alt, &s->prof);
            if (e != cudaSuccess) return cuda_fail(s, e, "upload: sort");
            KeepProg none;
            std::memset(&none, 0, sizeof none);
            e = StoreOps<W, T>::dedup(alt ? k1 : k0, alt ? (uint32_t*)s->up_v1.p : (uint32_t*)s->up_v0.p,
                                      (T*)s->up_c0.p, n, none, false, K(s, spare), C(s, spare),
                                      (unsigned long long*)s->up_st.p, s->ctl, s->hcount, &out_n, s->stream, &s->prof);
            if (e != cudaSuccess) return cuda_fail(s, e, "upload: dedup");
            fs = check_device_flags(s, "upload");
            if (fs != PS_OK) return fs;
        }
        s->cur = spare;
        s->n = out_n;
        s->slotted = false;
        if (s->hist_ready) {
            cudaMemsetAsync(s->hist.p, 0, kTopnBinsN * sizeof(unsigned int), s->stream);
            s->hist_ready = false;
        }
        return PS_OK;
    }

    // Compact a slotted store into the spare buffer (a no-op on a dense store).
    static ps_status densify(ps_sum* s, const char* what) {
        if (!s->slotted) return PS_OK;
        const int spare = 1 - s->cur;
        cudaError_t e = reserve_store(s, spare, s->live_n);
        if (e == cudaSuccess) e = ensure(s, s->status, (s->n / 4096 + 4) * sizeof(unsigned long long));
        if (e != cudaSuccess) return cuda_fail(s, e, what);
        if (e == cudaSuccess && s->f_valid) e = reserve_f(s, spare);
        if (e != cudaSuccess) return cuda_fail(s, e, what);
        uint64_t out_n = 0;
        e = StoreOps<W, T>::densify(K(s, s->cur), C(s, s->cur), s->n, slot_map(s), K(s, spare), C(s, spare),
                                    (unsigned long long*)s->status.p, s->ctl, s->hcount, &out_n, s->stream, &s->prof,
                                    s->f_valid ? F(s, s->cur) : nullptr, s->f_valid ? F(s, spare) : nullptr);
        s->prof.resolve();
        if (e != cudaSuccess) return cuda_fail(s, e, what);
        unsigned int fl = 0, fi = 0;
        topn_flags(s->hcount, &fl, &fi);
        ps_status ps = flags_status(s, fl, fi, what);
        if (ps != PS_OK) return ps;
        if (out_n != s->live_n) return set_err(s, PS_ERR_DEVICE, std::string(what) + ": slotted store lost rows");
        s->cur = spare;
        s->n = out_n;
        s->slotted = false;
        return PS_OK;
    }

    static SlotMap slot_map(const ps_sum* s) {
        return s->slotted ? SlotMap{(const unsigned int*)s->slot_count.p, s->slot_rows} : SlotMap{nullptr, 0u};
    }

    static ps_status download(ps_sum* s, uint64_t* x, uint64_t* z, double* c, uint64_t cap, uint64_t* nout) {
        {
            ps_status ps = densify(s, "download");
            if (ps != PS_OK) return ps;
        }
        if (nout) *nout = s->n;
        if (cap < s->n) return set_err(s, PS_ERR_INVALID, "download: capacity below the term count");
        if (s->n == 0) return PS_OK;
        cudaError_t e;
        if ((e = ensure(s, s->up_x, s->n * W * 8)) != cudaSuccess || (e = ensure(s, s->up_z, s->n * W * 8)) != cudaSuccess ||
            (e = ensure(s, s->up_c, s->n * 8)) != cudaSuccess)
            return cuda_fail(s, e, "download: allocation");
        e = StoreOps<W, T>::unpack(K(s, s->cur), C(s, s->cur), s->n, (uint64_t*)s->up_x.p, (uint64_t*)s->up_z.p,
                                   (double*)s->up_c.p, s->sms, s->stream, &s->prof);
        if (e == cudaSuccess && x) e = cudaMemcpyAsync(x, s->up_x.p, s->n * W * 8, cudaMemcpyDeviceToHost, s->stream);
        if (e == cudaSuccess && z) e = cudaMemcpyAsync(z, s->up_z.p, s->n * W * 8, cudaMemcpyDeviceToHost, s->stream);
        if (e == cudaSuccess && c) e = cudaMemcpyAsync(c, s->up_c.p, s->n * 8, cudaMemcpyDeviceToHost, s->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
        if (e != cudaSuccess) return cuda_fail(s, e, "download");
        return PS_OK;
    }

    // Does table t run on the partner path with a partner stream (where noise can be folded)?
    static bool folds_noise(const ps_table& t) {
        RotLayer<W> L;
        LevelList* lv = new LevelList();
        std::string why;
        bool general = false;
        const bool ok = to_rot_layer<W, T>(t, L, *lv, why, &general) == PS_OK && !general && L.partners;
        delete lv;
        return ok;
    }

    // noise (optional): single-qubit key-preserving channels to fold in before the table, in
    // order; noise_after[j] receives the terms left after channel j.
    static ps_status apply(ps_sum* s, const ps_table& t, const ps_policy* policy, ps_layer_stats* stats,
                           const NoiseList* noise = nullptr, uint64_t* noise_after = nullptr) {
        KeepProg keep;
        std::string why;
        // the last TopN pass wrote this layer's partner list (the store is as it left it)
        const bool preclassified = s->pre_valid && s->pre_table == &t && !s->slotted && s->n == s->pre_n;
        s->pre_valid = false;
        ps_status ps = lower_keep(policy, keep, why);
        if (ps != PS_OK) return set_err(s, ps, why);
        if ((ps = densify(s, "apply")) != PS_OK) return ps;
        RotationArgs<W, T> a;
        std::memset(&a, 0, sizeof a);
        bool general = false;
        ps = to_rot_layer<W, T>(t, a.L, *s->levels, why, &general);
        if (ps != PS_OK) return set_err(s, ps, why);
        uint64_t lsup[W];
        table_support<W>(t, lsup);
        if (general) return apply_general(s, t, keep, policy, stats, lsup);
        {
            // a commuting term keeps c exactly on the wide path; a local table must leave the
            // identity pattern alone
            const bool identity0 = a.L.wide || ((T)a.L.a1[0] == T(0) && (T)a.L.a0[0] == T(1));
            if (!noise && skippable(s, lsup, keep, identity0)) {
                skipped(s, stats, a.L.partners ? PS_PATH_ROTATION : PS_PATH_RESCALE);
                return PS_OK;
            }
        }
        const uint64_t n = s->n;
        if (n >= (1ull << 31) - 1) return set_err(s, PS_ERR_UNSUPPORTED, "apply: at most 2^31 - 2 terms");
        const int spare = 1 - s->cur;
        const uint64_t out_rows = a.L.partners ? 2 * n : n;
        // the first layer pass is TopN (or ApproxTopN) and could trigger: the merge builds its
        // first select digit (the octave histogram); before plain TopN the merge writes slots
        const int first_pass = policy && policy->num_passes > 0 ? policy->passes[0].kind : PS_PASS_NONE;
        // an inherited scored pass: the predictions ride along with the rows (folded noise cannot)
        const bool carry_f = inherit_interval(policy, s) > 1 && s->f_valid && !noise;
        if (!carry_f) s->f_valid = false;
        const bool scored_fuse = carry_f && first_pass == PS_PASS_SCORED_TOPN;
        const bool fuse_topn = (first_pass == PS_PASS_TOPN || first_pass == PS_PASS_APPROX_TOPN || scored_fuse) &&
                               out_rows > policy->passes[0].n;
        const uint64_t span_rows = merge_span_rows<W>(out_rows);
        // (the TopN kernels index a slotted store's rows in 32 bits)
        const bool slotted = fuse_topn && (first_pass == PS_PASS_TOPN || scored_fuse) && !s->fault_stall &&
                             span_rows < (1ull << 32);
        cudaError_t e = reserve_store(s, spare, slotted ? span_rows : out_rows);
        if (e == cudaSuccess && carry_f) e = reserve_f(s, spare);
        if (e == cudaSuccess && carry_f && a.L.partners) e = ensure(s, s->pf, n * sizeof(float));
        if (e == cudaSuccess && slotted)
            e = ensure(s, s->slot_count, (span_rows / merge_slot_rows<W>() + 1) * sizeof(unsigned int));
        if (e != cudaSuccess) return cuda_fail(s, e, "apply: output store");
        // a plain TopN pass alone follows and a rotation layer (with partners) comes next: the
        // merge also writes each output row's partner test under that layer, for the compaction
        s->nflag_valid = false;
        if (slotted && first_pass == PS_PASS_TOPN && policy->num_passes == 1 && s->next_table && !carry_f &&
            !(noise && noise->n > 0) && a.L.partners && policy->passes[0].n < (1ull << 31) - 1) {
            std::string why_next;
            bool general_next = false;
            if (to_rot_layer<W, T>(*s->next_table, a.next_L, *s->levels_next, why_next, &general_next) == PS_OK &&
                !general_next && a.next_L.partners) {
                if ((e = ensure(s, s->nflag, span_rows)) != cudaSuccess) return cuda_fail(s, e, "apply: partner flags");
                a.next_flags = static_cast<uint8_t*>(s->nflag.p);
                s->nflag_valid = true;
                s->nflag_table = s->next_table;
            }
        }
        const uint64_t tiles_hi = out_rows / kMinTileRows + 4;
        if ((e = ensure(s, s->status, tiles_hi * sizeof(unsigned long long))) != cudaSuccess ||
            (e = ensure(s, s->bounds, (tiles_hi + 2) * sizeof(ulonglong2))) != cudaSuccess)
            return cuda_fail(s, e, "apply: scratch");
        if (a.L.partners) {
            if ((e = ensure(s, s->pk, n * kKeyBytes)) != cudaSuccess || (e = ensure(s, s->pc, n * sizeof(T))) != cudaSuccess ||
                (e = ensure(s, s->idx, n * 4)) != cudaSuccess || (e = ensure(s, s->dv, n * 2)) != cudaSuccess ||
                (e = ensure(s, s->fv, n * 4)) != cudaSuccess ||
                (e = ensure(s, s->slots, (n / kScanTileRows + 4) * sizeof(LevelTile))) != cudaSuccess)
                return cuda_fail(s, e, "apply: partner scratch");
        }
        a.Sk = K(s, s->cur);
        a.Sc = C(s, s->cur);
        a.n = n;
        a.preclassified = preclassified && a.L.partners && !noise ? 1 : 0;
        a.levels = s->levels;
        a.keep = keep;
        a.idx = (uint32_t*)s->idx.p;
        a.D = (uint16_t*)s->dv.p;
        a.F = (int32_t*)s->fv.p;
        a.slots = s->slots.p;
        a.status = (unsigned long long*)s->status.p;
        a.bounds = (ulonglong2*)s->bounds.p;
        a.Pk = (uint64_t*)s->pk.p;
        a.Pc = (T*)s->pc.p;
        a.p_cap = a.L.partners ? n : 0;
        a.Ok = K(s, spare);
        a.Oc = C(s, spare);
        a.out_cap = s->cap[spare];
        a.ctl = s->ctl;
        a.host_count = s->hcount;
        uint64_t partners = 0, out_n = 0;
        unsigned int err_flags = 0, err_info = 0;
        a.partners_out = &partners;
        a.out_count = &out_n;
        a.err_flags = &err_flags;
        a.err_info = &err_info;
        a.prof = &s->prof;
        const bool window = (first_pass == PS_PASS_TOPN && s->topn_window) || (scored_fuse && s->score_window);
        a.topn_hist_mode = first_pass == PS_PASS_APPROX_TOPN ? 1 : (scored_fuse ? (window ? 4 : 3) : (window ? 2 : 0));
        a.topn_hist_base = window ? (scored_fuse ? s->score_base : s->topn_base) : 0;
        if (carry_f) {
            a.Sf = F(s, s->cur);
            a.Pf = a.L.partners ? static_cast<float*>(s->pf.p) : nullptr;
            a.Of = F(s, spare);
        }
        if (s->hist_ready) {
            cudaMemsetAsync(s->hist.p, 0, kTopnBinsN * sizeof(unsigned int), s->stream);
            s->hist_ready = false;
        }
        a.topn_hist = fuse_topn ? (unsigned int*)s->hist.p : nullptr;
        a.inject_stall = s->fault_stall ? 1 : 0;
        a.stall_limit = s->fault_stall ? s->stall_limit : 0;
        s->fault_stall = false;
        uint64_t span = 0;
        a.slot_count = slotted ? (unsigned int*)s->slot_count.p : nullptr;
        a.sms = s->sms;
        a.span_out = &span;
        if (noise && noise->n > 0) {
            if (!a.L.partners) return set_err(s, PS_ERR_INVALID, "apply: noise folded into a layer without partners");
            if ((e = ensure(s, s->noise_drops, (kMaxNoise + 1) * sizeof(unsigned long long))) != cudaSuccess)
                return cuda_fail(s, e, "apply: noise scratch");
            if (!s->hnoise && (e = cudaMallocHost(&s->hnoise, (kMaxNoise + 1) * sizeof(unsigned long long))) != cudaSuccess) {
                s->hnoise = nullptr;
                return cuda_fail(s, e, "apply: noise scratch");
            }
            a.noise = noise;
            a.noise_drops = static_cast<unsigned long long*>(s->noise_drops.p);
            a.host_noise_drops = s->hnoise;
        }
        // the TopN pass that follows reads the span and live count on the device and waits once
        // for both (one cooperative select, the merge's histogram and slots; no folded noise)
        // (or an inherited learned pass between rescorings, whose select reads the carried scores)
        const bool defer_pass = (first_pass == PS_PASS_TOPN && !carry_f) ||
                                (scored_fuse && s->f_age + 1 < inherit_interval(policy, s));
        const bool defer = s->in_propagate && slotted && fuse_topn && defer_pass && policy->num_passes == 1 &&
                           policy->passes[0].n > 0 && !a.noise && a.L.partners &&
                           StoreOps<W, T>::cooperative_select();
        if (defer) a.defer_counts = s->hcount + 32;
        a.inject_flag = s->fault_flag;
        s->fault_flag = 0;
        s->deferred = false;
        e = launch_rotation_layer<W, T>(a, s->stream);
        s->prof.resolve();
        if (e != cudaSuccess) return cuda_fail(s, e, "apply: rotation layer");
        ps = flags_status(s, err_flags, err_info, "apply");
        if (ps != PS_OK) {
            if (fuse_topn) cudaMemsetAsync(s->hist.p, 0, kTopnBinsN * sizeof(unsigned int), s->stream);
            return ps;
        }
        s->hist_ready = fuse_topn;
        s->hist_kind = first_pass;
        s->hist_window = fuse_topn && window;
        s->hist_base = a.topn_hist_base;
        uint64_t n_rot = n;  // terms entering the rotation, after the folded noise
        if (a.noise) {
            for (int j = 0; j < noise->n; ++j) {
                n_rot -= s->hnoise[j];
                if (noise_after) noise_after[j] = n_rot;
            }
        }
        if (stats) {
            stats->terms_in = n_rot;
            stats->partners = partners;
            stats->terms_out = out_n;
            stats->terms_after_passes = out_n;
            stats->path = a.L.partners ? PS_PATH_ROTATION : PS_PATH_RESCALE;
        }
        if (defer) {
            // counts, statistics and the error check come with the TopN pass's synchronization
            s->deferred = true;
            s->def_prev_cur = s->cur;
            s->def_n_in = n;
            s->def_nlv = s->levels->n;
            s->def_classified = !a.preclassified;
            s->def_flags = a.next_flags != nullptr;
            s->def_stats = stats;
            if (stats) std::memset(stats, 0, sizeof *stats);
        }
        s->cur = spare;
        s->n = slotted ? span : out_n;  // deferred: a bound on the span
        s->slotted = slotted;
        s->live_n = out_n;              // deferred: not known yet
        s->slot_rows = slotted ? merge_slot_rows<W>() : 0u;
        layer_done(s, lsup, keep, a.L.partners != 0);
        return PS_OK;
    }

    // The deferred layer's counts, read after the TopN pass's synchronization (host_count + 32
    // holds the copy the layer queued before the pass): statistics, byte bookkeeping and its
    // error check.  A failed layer's pass wrote nothing, so its input is restored as the store.
    static ps_status finish_deferred(ps_sum* s, uint64_t span) {
        s->deferred = false;
        const unsigned long long* c = s->hcount + 32;
        const unsigned int* f = reinterpret_cast<const unsigned int*>(reinterpret_cast<const unsigned char*>(c) +
                                                                      offsetof(Ctl, err));
        if (f[0]) {
            s->cur = s->def_prev_cur;
            s->n = s->def_n_in;
            s->slotted = false;
            s->live_n = 0;
            cudaMemsetAsync(s->hist.p, 0, kTopnBinsN * sizeof(unsigned int), s->stream);  // the pass left it
            s->hist_ready = false;
            return flags_status(s, f[0], f[1], "apply");
        }
        const uint64_t m = c[0], out = c[1];
        book_rotation_bytes<W, T>(&s->prof, s->def_n_in, m, out, s->def_nlv, s->def_classified);
        if (s->def_flags) s->prof.add_bytes(K_MERGE, (double)out);  // the partner-test bytes
        if (s->def_stats) {
            s->def_stats->terms_in = s->def_n_in;
            s->def_stats->partners = m;
            s->def_stats->terms_out = out;
            s->def_stats->terms_after_passes = out;
            s->def_stats->path = PS_PATH_ROTATION;
        }
        s->n = span;
        s->live_n = out;
        return PS_OK;
    }

    // A deferred layer whose pass cannot run on the device's counts: wait for them here.
    static ps_status settle_deferred(ps_sum* s) {
        cudaMemcpyAsync(s->hcount + 22, &s->ctl->span, sizeof(unsigned long long), cudaMemcpyDeviceToHost, s->stream);
        cudaError_t e = spin_sync(s->stream);
        if (e != cudaSuccess) return cuda_fail(s, e, "apply: counts");
        return finish_deferred(s, s->hcount[22]);
    }

    // The sort path: branch records, LSD radix sort of (key, record index), run-summing dedup
    // with the keep program (apply_layer_body's general tables, engine/gpu/layer.rs:614-763).
    static ps_status apply_general(ps_sum* s, const ps_table& t, const KeepProg& keep, const ps_policy* policy,
                                   ps_layer_stats* stats, const uint64_t (&lsup)[W]) {
        (void)policy;
        GenLayer<W, T> G;
        to_gen_layer<W, T>(t, G);
        s->f_valid = false;  // the sort path carries no predictions
        {
            bool identity0 = G.cnt[0] == 1 && G.amp[0][0] == T(1);
            for (int w = 0; identity0 && w < W; ++w)
                identity0 = G.mx[G.ent[0][0]][w] == 0 && G.mz[G.ent[0][0]][w] == 0;
            if (skippable(s, lsup, keep, identity0)) {
                skipped(s, stats, PS_PATH_SORT);
                return PS_OK;
            }
        }
        const uint64_t n = s->n;
        if (s->hist_ready) {
            cudaMemsetAsync(s->hist.p, 0, kTopnBinsN * sizeof(unsigned int), s->stream);
            s->hist_ready = false;
        }
        uint64_t m = 0;
        cudaError_t e = GeneralOps<W, T>::count(K(s, s->cur), n, G, s->ctl, s->hcount, &m, s->sms, s->stream, &s->prof);
        s->prof.resolve();
        if (e != cudaSuccess) return cuda_fail(s, e, "apply: record count");
        if (m >= (1ull << 32) - 1)
            return set_err(s, PS_ERR_UNSUPPORTED, "apply: a general layer emits at most 2^32 - 2 records");
        const int spare = 1 - s->cur;
        uint64_t out_n = 0;
        if (m) {
            const size_t sort_tiles = (m + StoreOps<W, T>::sort_tile() - 1) / StoreOps<W, T>::sort_tile();
            const size_t branch_tiles = (n + GeneralOps<W, T>::branch_tile() - 1) / GeneralOps<W, T>::branch_tile();
            if ((e = reserve_store(s, spare, m)) != cudaSuccess || (e = ensure(s, s->up_k, 2 * m * kKeyBytes)) != cudaSuccess ||
                (e = ensure(s, s->up_v0, m * 4)) != cudaSuccess || (e = ensure(s, s->up_v1, m * 4)) != cudaSuccess ||
                (e = ensure(s, s->up_c0, m * sizeof(T))) != cudaSuccess ||
                (e = ensure(s, s->up_st, (m / 2048 + 2) * sizeof(unsigned long long))) != cudaSuccess ||
                (e = ensure(s, s->status, (branch_tiles + 2) * sizeof(unsigned long long))) != cudaSuccess ||
                (e = ensure(s, s->sort_status, sort_tiles * 256 * sizeof(unsigned int))) != cudaSuccess)
                return cuda_fail(s, e, "apply: sort-path scratch");
            s->sort.status = static_cast<unsigned int*>(s->sort_status.p);
            uint64_t* k0 = (uint64_t*)s->up_k.p;
            uint64_t* k1 = k0 + m * 2 * W;
            uint32_t* v0 = (uint32_t*)s->up_v0.p;
            uint32_t* v1 = (uint32_t*)s->up_v1.p;
            T* rc = (T*)s->up_c0.p;
            e = GeneralOps<W, T>::branch(K(s, s->cur), C(s, s->cur), n, G, k0, v0, rc, m,
                                         (unsigned long long*)s->status.p, s->ctl, s->stream, &s->prof);
            if (e != cudaSuccess) return cuda_fail(s, e, "apply: branch");
            bool alt = false;
            e = StoreOps<W, T>::sort_pairs(k0, v0, k1, v1, m, s->sort, s->ctl, s->sms, s->stream, alt, &s->prof);
            if (e != cudaSuccess) return cuda_fail(s, e, "apply: sort");
            ps_status fs = check_device_flags(s, "apply");
            if (fs != PS_OK) return fs;
            e = StoreOps<W, T>::dedup(alt ? k1 : k0, alt ? v1 : v0, rc, m, keep, s->compensated, K(s, spare),
                                      C(s, spare), (unsigned long long*)s->up_st.p, s->ctl, s->hcount, &out_n,
                                      s->stream, &s->prof);
            s->prof.resolve();
            if (e != cudaSuccess) return cuda_fail(s, e, "apply: dedup");
            fs = check_device_flags(s, "apply");
            if (fs != PS_OK) return fs;
        }
        if (stats) {
            stats->terms_in = n;
            stats->partners = m > n ? m - n : 0;
            stats->terms_out = out_n;
            stats->terms_after_passes = out_n;
            stats->path = PS_PATH_SORT;
        }
        s->cur = spare;
        s->n = out_n;
        layer_done(s, lsup, keep, true);
        return PS_OK;
    }

    static ps_status finalize(ps_sum* s, const ps_policy* policy) {
        const uint64_t interval = inherit_interval(policy, s);
        const bool deferrable = policy && policy->num_passes > 0 &&
                                (policy->passes[0].kind == PS_PASS_TOPN ||
                                 (policy->passes[0].kind == PS_PASS_SCORED_TOPN && interval > 1));
        if (s->deferred && !deferrable) {  // a pass that needs the layer's counts on the host
            ps_status ps = settle_deferred(s);
            if (ps != PS_OK) return ps;
        }
        if (!(policy && policy->num_passes > 0 && (policy->passes[0].kind == PS_PASS_TOPN || interval > 1))) {
            ps_status ps = densify(s, "finalize");
            if (ps != PS_OK) return ps;
        }
        bool ready = s->hist_ready;
        if (ready) s->hist_ready = false;
        if (s->scorer) s->scorer_remaining -= 1.0;
        ps_status result = PS_OK;
        for (int i = 0; policy && i < policy->num_passes; ++i) {
            const ps_pass& p = policy->passes[i];
            if (p.kind == PS_PASS_SCORED_TOPN) {
                if (interval > 1) {
                    ps_status ps = scored_inherited(s, p.n, interval,
                                                    ready && i == 0 && s->hist_kind == PS_PASS_SCORED_TOPN,
                                                    i == policy->num_passes - 1);
                    if (ps != PS_OK) return ps;
                    continue;
                }
                if (ready && i == 0) cudaMemsetAsync(s->hist.p, 0, kTopnBinsN * sizeof(unsigned int), s->stream);
                ps_status ps = scored_topn(s, p.n);
                if (ps != PS_OK) return ps;
                continue;
            }
            if (p.kind == PS_PASS_COLLAPSE_SAMPLE) {
                if (ready && i == 0) cudaMemsetAsync(s->hist.p, 0, kTopnBinsN * sizeof(unsigned int), s->stream);
                ps_status ps = collapse(s, p.n, p.samples, p.seed, p.call + s->pass_call);
                if (ps != PS_OK) return ps;
                continue;
            }
            if (p.kind == PS_PASS_APPROX_TOPN) {
                ps_status ps = approx_topn(s, p.n, ready && i == 0 && s->hist_kind == PS_PASS_APPROX_TOPN,
                                           ready && i == 0);
                if (ps != PS_OK) return ps;
                continue;
            }
            if (p.kind != PS_PASS_TOPN) continue;
            if (ready && i == 0 && s->hist_kind != PS_PASS_TOPN) {  // a histogram of another pass kind
                cudaMemsetAsync(s->hist.p, 0, kTopnBinsN * sizeof(unsigned int), s->stream);
                ready = false;
            }
            const bool use_hist = ready && i == 0;
            // the layer before did not wait for its counts: the select decides on the device
            // whether the live rows fit (the layer keeps a pass of n > 0 only, with its histogram)
            const bool dfr = s->deferred && i == 0 && use_hist;
            if (s->deferred && !dfr) {
                ps_status ps = settle_deferred(s);
                if (ps != PS_OK) return ps;
            }
            if (!dfr && (s->slotted ? s->live_n : s->n) <= p.n) {
                if (use_hist) cudaMemsetAsync(s->hist.p, 0, kTopnBinsN * sizeof(unsigned int), s->stream);
                ps_status ps = densify(s, "topn");
                if (ps != PS_OK) return ps;
                continue;
            }
            if (p.n == 0) {
                if (use_hist) cudaMemsetAsync(s->hist.p, 0, kTopnBinsN * sizeof(unsigned int), s->stream);
                s->n = 0;
                s->slotted = false;
                continue;
            }
            const int spare = 1 - s->cur;
            cudaError_t e = reserve_store(s, spare, p.n);
            if (e == cudaSuccess) e = ensure(s, s->cand, topn_cand_words(s->n, s->sms) * sizeof(uint64_t));
            if (e == cudaSuccess) e = ensure(s, s->status, (s->n / 4096 + 4) * sizeof(unsigned long long));
            // the layer's last pass, with a rotation layer (with partners) next: the compaction also
            // writes that layer's partner list, so it skips its own classify pass
            RotLayer<W> next_L;
            bool classify = false;
            if (e == cudaSuccess && s->next_table && i == policy->num_passes - 1 && p.n < (1ull << 31) - 1) {
                std::string why_next;
                bool general = false;
                classify = to_rot_layer<W, T>(*s->next_table, next_L, *s->levels, why_next, &general) == PS_OK &&
                           !general && next_L.partners;
                if (classify) e = ensure(s, s->idx, p.n * 4);
                if (classify && e == cudaSuccess) e = ensure(s, s->dv, p.n * 2);
            }
            if (e != cudaSuccess) {
                if (use_hist) cudaMemsetAsync(s->hist.p, 0, kTopnBinsN * sizeof(unsigned int), s->stream);
                return cuda_fail(s, e, "topn: scratch");
            }
            // the merge wrote the rows' partner tests under that layer
            const bool flags_ok = classify && i == 0 && s->slotted && s->nflag_valid && s->nflag_table == s->next_table;
            s->nflag_valid = false;
            uint64_t out_n = 0;
            // a histogram binned in the window around the last boundary selects in 1/16 octaves
            // (few candidates); when the boundary left the window, the pass reruns in full range
            const bool window = use_hist && s->hist_window;
            bool kept_all = false;
            for (int attempt = 0; attempt < 2; ++attempt) {
                const bool win = window && attempt == 0;
                const bool dfr_now = dfr && attempt == 0;
                e = StoreOps<W, T>::topn(K(s, s->cur), C(s, s->cur), s->n, p.n, K(s, spare), C(s, spare),
                                         (unsigned int*)s->hist.p, use_hist && attempt == 0, (uint64_t*)s->cand.p,
                                         topn_cand_words(s->n, s->sms), (unsigned long long*)s->status.p, s->ctl,
                                         s->hcount, &out_n, s->sms,
                                         s->stream, &s->prof, nullptr, win, win ? s->hist_base : 0, slot_map(s),
                                         nullptr, nullptr, classify ? &next_L : nullptr,
                                         classify ? (uint32_t*)s->idx.p : nullptr,
                                         classify ? (uint16_t*)s->dv.p : nullptr, classify && flags_ok ?
                                         static_cast<const uint8_t*>(s->nflag.p) : nullptr, dfr_now);
                s->prof.resolve();
                if (e != cudaSuccess) return cuda_fail(s, e, "topn");
                if (dfr_now) {  // the layer's own counts and error check, then the pass's
                    ps_status ps = finish_deferred(s, s->hcount[22]);
                    if (ps != PS_OK) return ps;
                    kept_all = s->hcount[23] != 0;
                }
                unsigned int fl = 0, fi = 0;
                topn_flags(s->hcount, &fl, &fi);
                ps_status ps = flags_status(s, fl, fi, "topn");
                if (ps != PS_OK) {
                    cudaMemsetAsync(s->hist.p, 0, kTopnBinsN * sizeof(unsigned int), s->stream);
                    return ps;
                }
                if (kept_all) break;  // no boundary: the window stays where it was
                if (!(win && topn_window_missed(s->hcount))) {
                    const uint64_t boundary = topn_boundary(s->hcount, win ? s->hist_base : 0);
                    const uint64_t half = 1024ull << 48;
                    s->topn_window = boundary != 0;
                    s->topn_base = boundary > half ? boundary - half : 0;
                    break;
                }
            }
            s->cur = spare;
            s->n = out_n;
            s->slotted = false;
            if (classify && !topn_unclassified(s->hcount)) {
                s->pre_valid = true;
                s->pre_table = s->next_table;
                s->pre_n = out_n;
            }
        }
        return result;
    }

    // CollapseSample: above `cache` terms, a systematic resample of `samples` points.
    static ps_status collapse(ps_sum* s, uint64_t cache, uint64_t samples, uint64_t seed, uint64_t call) {
        if (s->n <= cache) return PS_OK;
        const uint64_t n = s->n, nb = (n + 1023) / 1024;
        const int spare = 1 - s->cur;
        cudaError_t e = reserve_store(s, spare, n);
        if (e == cudaSuccess) e = ensure(s, s->cnorms, 2 * (nb + 1) * sizeof(double));
        if (e == cudaSuccess) e = ensure(s, s->cfirst, (nb + 1) * sizeof(uint64_t));
        if (e == cudaSuccess) e = ensure(s, s->idx, n * sizeof(uint32_t));
        if (e == cudaSuccess) e = ensure(s, s->status, (n / 4096 + 4) * sizeof(unsigned long long));
        if (e == cudaSuccess && s->hnorms_cap < 2 * (nb + 1)) {
            if (s->hnorms) cudaFreeHost(s->hnorms);
            s->hnorms = nullptr;
            s->hnorms_cap = 0;
            e = cudaMallocHost(&s->hnorms, 2 * (nb + 1) * sizeof(double));
            if (e == cudaSuccess) s->hnorms_cap = 2 * (nb + 1);
        }
        if (e == cudaSuccess && s->hfirst_cap < nb + 1) {
            if (s->hfirst) cudaFreeHost(s->hfirst);
    if (s->hnoise) cudaFreeHost(s->hnoise);
            s->hfirst = nullptr;
            s->hfirst_cap = 0;
            e = cudaMallocHost(&s->hfirst, (nb + 1) * sizeof(uint64_t));
            if (e == cudaSuccess) s->hfirst_cap = nb + 1;
        }
        if (e != cudaSuccess) return cuda_fail(s, e, "CollapseSample: scratch");
        uint64_t out_n = 0;
        bool drawable = true;
        e = StoreOps<W, T>::collapse_sample(K(s, s->cur), C(s, s->cur), n, samples, seed, call, K(s, spare),
                                            C(s, spare), (double*)s->cnorms.p, s->hnorms, (uint64_t*)s->cfirst.p,
                                            s->hfirst, (uint32_t*)s->idx.p, (unsigned long long*)s->status.p,
                                            s->ctl, s->hcount, &out_n, &drawable, s->stream, &s->prof);
        s->prof.resolve();
        if (e != cudaSuccess) return cuda_fail(s, e, "CollapseSample");
        if (!drawable)
            return set_err(s, PS_ERR_INVALID,
                           "CollapseSample: cannot draw by |c| from " + std::to_string(n) +
                               " terms whose sum of |c| is zero or not finite");
        unsigned int fl = 0, fi = 0;
        topn_flags(s->hcount, &fl, &fi);
        ps_status ps = flags_status(s, fl, fi, "CollapseSample");
        if (ps != PS_OK) return ps;
        s->cur = spare;
        s->n = out_n;
        ++s->collapses;
        s->keep_clean = false;  // the drawn terms carry new coefficients
        s->f_valid = false;
        return PS_OK;
    }

    // ApproxTopN: the octave histogram (fused into the layer's merge when use_hist), the edge
    // walk on the host, one compaction.  held: the hist buffer holds some histogram to clear.
    static ps_status approx_topn(ps_sum* s, uint64_t keep_n, bool use_hist, bool held) {
        if (held && !use_hist) cudaMemsetAsync(s->hist.p, 0, kTopnBinsN * sizeof(unsigned int), s->stream);
        if (s->n <= keep_n) {
            if (use_hist) cudaMemsetAsync(s->hist.p, 0, kTopnBinsN * sizeof(unsigned int), s->stream);
            return PS_OK;
        }
        if (keep_n == 0) {
            if (use_hist) cudaMemsetAsync(s->hist.p, 0, kTopnBinsN * sizeof(unsigned int), s->stream);
            s->n = 0;
            return PS_OK;
        }
        const int spare = 1 - s->cur;
        cudaError_t e = reserve_store(s, spare, keep_n);
        if (e == cudaSuccess) e = ensure(s, s->status, (s->n / 4096 + 4) * sizeof(unsigned long long));
        if (e != cudaSuccess) {
            if (use_hist) cudaMemsetAsync(s->hist.p, 0, kTopnBinsN * sizeof(unsigned int), s->stream);
            return cuda_fail(s, e, "approx TopN: scratch");
        }
        uint64_t out_n = 0;
        e = StoreOps<W, T>::approx_topn(K(s, s->cur), C(s, s->cur), s->n, keep_n, K(s, spare), C(s, spare),
                                        (unsigned int*)s->hist.p, use_hist, s->hhist,
                                        (unsigned long long*)s->status.p, s->ctl, s->hcount, &out_n, s->sms,
                                        s->stream, &s->prof);
        s->prof.resolve();
        if (e != cudaSuccess) return cuda_fail(s, e, "approx TopN");
        unsigned int fl = 0, fi = 0;
        topn_flags(s->hcount, &fl, &fi);
        ps_status ps = flags_status(s, fl, fi, "approx TopN");
        if (ps != PS_OK) return ps;
        s->cur = spare;
        s->n = out_n;
        return PS_OK;
    }

    // The inherited learned pass.  Every `interval` layers (and whenever the rows carry no valid
    // predictions) the scorer predicts afresh for every row, writing the predictions, the select
    // keys and their first-digit histogram in one pass, and the select runs on those keys; in
    // the layers between, the merge carried each row's prediction (partners their parent's) and
    // histogrammed log|c| + f, and the select computes the same score from the coefficient and
    // the prediction.  Either way the compaction carries the predictions with the kept rows.
    // hist_ok: the layer's merge left a histogram of the scores in s->hist.
    static ps_status scored_inherited(ps_sum* s, uint64_t keep_n, uint64_t interval, bool hist_ok, bool last_pass) {
        ps_scorer* sc = s->scorer;
        const bool rescore = !s->f_valid || s->f_age + 1 >= interval;
        // the layer did not wait for its counts: the select reads them (between rescorings)
        const bool dfr = s->deferred && !rescore && hist_ok && keep_n > 0;
        if (s->deferred && !dfr) {
            ps_status ps = settle_deferred(s);
            if (ps != PS_OK) return ps;
        }
        const uint64_t live = s->slotted ? s->live_n : s->n;
        auto drop_hist = [&]() {
            if (hist_ok) cudaMemsetAsync(s->hist.p, 0, kTopnBinsN * sizeof(unsigned int), s->stream);
            hist_ok = false;
        };
        cudaError_t e;
        if (rescore) {
            drop_hist();
            if ((e = ensure(s, s->fcol[s->cur], s->cap[s->cur] * sizeof(float))) != cudaSuccess ||
                (e = ensure(s, s->sel, std::max<uint64_t>(s->n, 1) * sizeof(uint64_t))) != cudaSuccess)
                return cuda_fail(s, e, "scored TopN: scratch");
            if (s->n) {
                ScorerArgs A;
                A.p = static_cast<const uint16_t*>(sc->bf.p);
                A.L = sc->L;
                A.nq = sc->nq;
                for (int f = 0; f < 3; ++f) A.fscale[f] = sc->cfg.feature_scale[f];
                A.residual = 1;
                A.site_row = sc->mapped ? static_cast<const int16_t*>(sc->site_map.p) : nullptr;
                ScoreInput in{};
                in.keys = K(s, s->cur);
                in.coef64 = std::is_same<T, double>::value ? (const double*)C(s, s->cur) : nullptr;
                in.coef32 = std::is_same<T, float>::value ? (const float*)C(s, s->cur) : nullptr;
                in.rem_uniform = (float)(s->scorer_remaining / sc->cfg.layers_per_unit);
                in.n = s->n;  // a slotted store's gaps are scored too and never read
                e = launch_score<W>(A, in, nullptr, (uint64_t*)s->sel.p, (unsigned int*)s->hist.p, s->ctl, s->sms,
                                    s->stream, &s->prof, F(s, s->cur));
                if (e != cudaSuccess) return cuda_fail(s, e, "scored TopN: score");
                hist_ok = true;
            }
            s->f_valid = true;
            s->f_age = 0;
        } else {
            ++s->f_age;
        }
        if (!dfr && (live <= keep_n || keep_n == 0)) {
            drop_hist();
            if (keep_n == 0 && live > 0) {
                s->n = 0;
                s->slotted = false;
                return PS_OK;
            }
            return densify(s, "scored TopN");
        }
        const int spare = 1 - s->cur;
        e = reserve_store(s, spare, keep_n);
        if (e == cudaSuccess) e = reserve_f(s, spare);
        if (e == cudaSuccess) e = ensure(s, s->cand, topn_cand_words(s->n, s->sms) * sizeof(uint64_t));
        if (e == cudaSuccess) e = ensure(s, s->status, (s->n / 4096 + 4) * sizeof(unsigned long long));
        if (e != cudaSuccess) {
            drop_hist();
            return cuda_fail(s, e, "scored TopN: scratch");
        }
        // the layer's last pass between rescorings, a rotation layer (with partners) next: the
        // compaction also lists that layer's partners (as the plain TopN pass's does)
        RotLayer<W> next_L;
        bool classify = false;
        if (last_pass && !rescore && s->next_table && keep_n < (1ull << 31) - 1) {
            std::string why_next;
            bool general = false;
            classify = to_rot_layer<W, T>(*s->next_table, next_L, *s->levels, why_next, &general) == PS_OK &&
                       !general && next_L.partners;
            if (classify) e = ensure(s, s->idx, keep_n * 4);
            if (classify && e == cudaSuccess) e = ensure(s, s->dv, keep_n * 2);
            if (e != cudaSuccess) {
                drop_hist();
                return cuda_fail(s, e, "scored TopN: scratch");
            }
        }
        uint64_t out_n = 0;
        const bool window = !rescore && hist_ok && s->score_window;
        bool kept_all = false;
        for (int attempt = 0; attempt < 2; ++attempt) {
            const bool win = window && attempt == 0;
            const bool dfr_now = dfr && attempt == 0;
            e = StoreOps<W, T>::topn(K(s, s->cur), C(s, s->cur), s->n, keep_n, K(s, spare), C(s, spare),
                                     (unsigned int*)s->hist.p, hist_ok && attempt == 0, (uint64_t*)s->cand.p,
                                     topn_cand_words(s->n, s->sms), (unsigned long long*)s->status.p, s->ctl, s->hcount,
                                     &out_n, s->sms, s->stream, &s->prof, rescore ? (const uint64_t*)s->sel.p : nullptr,
                                     win, win ? s->score_base : 0, slot_map(s), F(s, s->cur), F(s, spare),
                                     classify ? &next_L : nullptr, classify ? (uint32_t*)s->idx.p : nullptr,
                                     classify ? (uint16_t*)s->dv.p : nullptr, nullptr, dfr_now);
            s->prof.resolve();
            if (e != cudaSuccess) return cuda_fail(s, e, "scored TopN");
            if (dfr_now) {  // the layer's own counts and error check, then the pass's
                ps_status ps = finish_deferred(s, s->hcount[22]);
                if (ps != PS_OK) return ps;
                kept_all = s->hcount[23] != 0;
            }
            unsigned int fl = 0, fi = 0;
            topn_flags(s->hcount, &fl, &fi);
            ps_status ps = flags_status(s, fl, fi, "scored TopN");
            if (ps != PS_OK) {
                cudaMemsetAsync(s->hist.p, 0, kTopnBinsN * sizeof(unsigned int), s->stream);
                return ps;
            }
            if (kept_all) break;  // no boundary: the window stays where it was
            if (!(win && topn_window_missed(s->hcount))) {
                const uint64_t boundary = topn_boundary(s->hcount, win ? s->score_base : 0);
                const uint64_t half = 1024ull << 48;
                s->score_window = boundary != 0;
                s->score_base = boundary > half ? boundary - half : 0;
                break;
            }
        }
        s->cur = spare;
        s->n = out_n;
        s->slotted = false;
        if (classify && !topn_unclassified(s->hcount)) {
            s->pre_valid = true;
            s->pre_table = s->next_table;
            s->pre_n = out_n;
        }
        return PS_OK;
    }

    // The learned pass: the attached scorer scores every term (tensor-core MLP, select keys and
    // their first-digit histogram written in the same pass), then the TopN select and the
    // order-preserving compaction run on the score keys.
    static ps_status scored_topn(ps_sum* s, uint64_t keep_n) {
        ps_scorer* sc = s->scorer;
        if (!sc) return set_err(s, PS_ERR_INVALID, "scored TopN: no scorer attached (ps_set_scorer)");
        if (s->n <= keep_n) return PS_OK;
        if (keep_n == 0) {
            s->n = 0;
            return PS_OK;
        }
        const int spare = 1 - s->cur;
        cudaError_t e = reserve_store(s, spare, keep_n);
        if (e == cudaSuccess) e = ensure(s, s->sel, s->n * sizeof(uint64_t));
        if (e == cudaSuccess) e = ensure(s, s->cand, topn_cand_words(s->n, s->sms) * sizeof(uint64_t));
        if (e == cudaSuccess) e = ensure(s, s->status, (s->n / 4096 + 4) * sizeof(unsigned long long));
        if (e != cudaSuccess) return cuda_fail(s, e, "scored TopN: scratch");
        ScorerArgs A;
        A.p = static_cast<const uint16_t*>(sc->bf.p);
        A.L = sc->L;
        A.nq = sc->nq;
        for (int f = 0; f < 3; ++f) A.fscale[f] = sc->cfg.feature_scale[f];
        A.residual = sc->cfg.residual ? 1 : 0;
        A.site_row = sc->mapped ? static_cast<const int16_t*>(sc->site_map.p) : nullptr;
        ScoreInput in{};
        in.keys = K(s, s->cur);
        in.coef64 = std::is_same<T, double>::value ? (const double*)C(s, s->cur) : nullptr;
        in.coef32 = std::is_same<T, float>::value ? (const float*)C(s, s->cur) : nullptr;
        in.rem_uniform = (float)(s->scorer_remaining / sc->cfg.layers_per_unit);
        in.n = s->n;
        cudaMemsetAsync(s->hist.p, 0, kTopnBins1 * sizeof(unsigned int), s->stream);
        e = launch_score<W>(A, in, nullptr, (uint64_t*)s->sel.p, (unsigned int*)s->hist.p, s->ctl, s->sms,
                            s->stream, &s->prof);
        if (e != cudaSuccess) return cuda_fail(s, e, "scored TopN: score");
        ps_status ps = check_device_flags(s, "scored TopN");
        if (ps != PS_OK) {
            cudaMemsetAsync(s->hist.p, 0, kTopnBinsN * sizeof(unsigned int), s->stream);
            return ps;
        }
        uint64_t out_n = 0;
        e = StoreOps<W, T>::topn(K(s, s->cur), C(s, s->cur), s->n, keep_n, K(s, spare), C(s, spare),
                                 (unsigned int*)s->hist.p, true, (uint64_t*)s->cand.p, topn_cand_words(s->n, s->sms),
                                 (unsigned long long*)s->status.p, s->ctl, s->hcount, &out_n, s->sms, s->stream,
                                 &s->prof, (const uint64_t*)s->sel.p);
        s->prof.resolve();
        if (e != cudaSuccess) return cuda_fail(s, e, "scored TopN");
        unsigned int fl = 0, fi = 0;
        topn_flags(s->hcount, &fl, &fi);
        ps = flags_status(s, fl, fi, "scored TopN");
        if (ps != PS_OK) {
            cudaMemsetAsync(s->hist.p, 0, kTopnBinsN * sizeof(unsigned int), s->stream);
            return ps;
        }
        s->cur = spare;
        s->n = out_n;
        return PS_OK;
    }

    static ps_status expectation(ps_sum* s, const uint64_t* ax, const uint64_t* az, const uint64_t* neg, double* out) {
        {
            ps_status ps = densify(s, "expectation");
            if (ps != PS_OK) return ps;
        }
        cudaError_t e = ensure(s, s->partial, kExpectBlocks * sizeof(double));
        if (e == cudaSuccess) e = ensure(s, s->dout, sizeof(double));
        if (e != cudaSuccess) return cuda_fail(s, e, "expectation: scratch");
        e = StoreOps<W, T>::expectation(K(s, s->cur), C(s, s->cur), s->n, ax, az, neg, (double*)s->partial.p,
                                        (double*)s->dout.p, s->sms, s->stream, &s->prof);
        if (e == cudaSuccess) e = cudaMemcpyAsync(s->hout, s->dout.p, sizeof(double), cudaMemcpyDeviceToHost, s->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
        if (e != cudaSuccess) return cuda_fail(s, e, "expectation");
        *out = *s->hout;
        return PS_OK;
    }

    static cudaError_t configure() {
        cudaError_t e = configure_rotation_kernels<W, T>();
        if (e == cudaSuccess) e = StoreOps<W, T>::configure();
        return e;
    }
};

template <template <int, typename> class Op, typename F>
ps_status dispatch(ps_sum* s, F&& f) {
    if (s->dtype == PS_F64) {
        switch (s->W) {
        case 1: return f(Op<1, double>());
        case 2: return f(Op<2, double>());
        case 4: return f(Op<4, double>());
        default: break;
        }
    } else {
        switch (s->W) {
        case 1: return f(Op<1, float>());
        case 2: return f(Op<2, float>());
        case 4: return f(Op<4, float>());
        default: break;
        }
    }
    return set_err(s, PS_ERR_UNSUPPORTED, "widths above 4 words (256 qubits) are not built");
}

// A single-qubit key-preserving channel whose factors can be folded into the next layer: it
// leaves the identity alone and shrinks no coefficient's magnitude by less than nothing
// (|factor| <= 1), so the keep program passes after it only if it passed before it.
bool foldable_noise(const ps_table& t, int nq) {
    if (t.mode != PS_TABLE_LOCAL || t.k != 1 || t.num_entries != 1 || t.entries[0].local_delta != 0) return false;
    if (t.qubits[0] >= (uint32_t)nq || t.entries[0].amplitude[0] != 1.0) return false;
    for (int s = 1; s < 4; ++s)
        if (!(std::fabs(t.entries[0].amplitude[s]) <= 1.0)) return false;
    return true;
}

// Would every layer pass of the policy leave a sum of the handle's current size (or smaller)
// unchanged?  Then folding noise layers skips only passes that would have done nothing.
bool passes_idle(const ps_policy* p, const ps_sum* s) {
    const uint64_t n = s->slotted ? s->live_n : s->n;
    for (int i = 0; p && i < p->num_passes; ++i)
        if (p->passes[i].kind != PS_PASS_NONE && n > p->passes[i].n) return false;
    return true;
}

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

}  // namespace

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {
#pragma GCC visibility push(default)

int32_t ps_abi_version(void) { return PS_ABI_VERSION; }

int32_t ps_device_count(void) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}

ps_status ps_create(int32_t device, int32_t num_qubits, int32_t dtype, ps_sum** out) {
    if (!out) return PS_ERR_INVALID;
    *out = nullptr;
    if (num_qubits < 1 || num_qubits > 64 * PS_MAX_W || (dtype != PS_F64 && dtype != PS_F32)) return PS_ERR_INVALID;
    const int W = width_for(num_qubits);
    if (W > 4) return PS_ERR_UNSUPPORTED;
    int count = ps_device_count();
    if (count == 0 || device < 0 || device >= count) return PS_ERR_NO_DEVICE;
    DeviceGuard g(device);
    ps_sum* s = new ps_sum();
    s->device = device;
    s->nq = num_qubits;
    s->W = W;
    s->dtype = dtype;
    cudaDeviceGetAttribute(&s->sms, cudaDevAttrMultiProcessorCount, device);
    cudaError_t e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMalloc(&s->ctl, sizeof(Ctl));
    if (e == cudaSuccess) e = cudaMemsetAsync(s->ctl, 0, sizeof(Ctl), s->stream);
    if (e == cudaSuccess) {
        static const unsigned long long limit = (unsigned long long)kSpinLimit;
        e = cudaMemcpy(&s->ctl->spin_limit, &limit, sizeof(limit), cudaMemcpyHostToDevice);
    }
    if (e == cudaSuccess) e = cudaMallocHost(&s->hcount, 64 * sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMallocHost(&s->hout, 8 * sizeof(double));
    if (e == cudaSuccess) e = cudaMallocHost(&s->hhist, kTopnBins1 * sizeof(unsigned int));
    if (e == cudaSuccess) e = cudaMalloc(&s->sort.hist, 16 * W * 256 * sizeof(unsigned int));
    if (e == cudaSuccess) e = cudaMalloc(&s->sort.base, 16 * W * 256 * sizeof(unsigned int));
    if (e == cudaSuccess) e = cudaMallocHost(&s->sort.host_hist, 16 * W * 256 * sizeof(unsigned int));
    if (e == cudaSuccess) e = cudaMallocHost(&s->sort.host_base, 16 * W * 256 * sizeof(unsigned int));
    if (e == cudaSuccess) e = ensure(s->hist, kTopnBinsN * sizeof(unsigned int));
    if (e == cudaSuccess) e = cudaMemsetAsync(s->hist.p, 0, kTopnBinsN * sizeof(unsigned int), s->stream);
    if (e == cudaSuccess) {
        ps_status st = dispatch<Engine>(s, [&](auto op) {
            cudaError_t ce = decltype(op)::configure();
            return ce == cudaSuccess ? PS_OK : cuda_fail(s, ce, "configure");
        });
        if (st != PS_OK) e = cudaErrorInvalidValue;
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
    if (e != cudaSuccess) {
        ps_destroy(s);
        cudaGetLastError();
        return e == cudaErrorMemoryAllocation ? PS_ERR_OOM : PS_ERR_DEVICE;
    }
    s->levels = new LevelList();
    s->levels_next = new LevelList();
    *out = s;
    return PS_OK;
}

ps_status ps_destroy(ps_sum* s) {
    if (!s) return PS_OK;
    DeviceGuard g(s->device);
    if (s->stream) cudaStreamSynchronize(s->stream);
    for (Buf* b : {&s->fcol[0], &s->fcol[1], &s->pf})
        release(*b);
    for (Buf* b : {&s->keys[0], &s->keys[1], &s->coef[0], &s->coef[1], &s->pk, &s->pc, &s->idx, &s->dv, &s->fv,
                   &s->slots, &s->status, &s->bounds, &s->hist, &s->cand, &s->partial, &s->dout, &s->sort_status,
                   &s->up_x, &s->up_z, &s->up_c, &s->up_k, &s->up_v0, &s->up_v1, &s->up_c0, &s->up_st, &s->sel,
                   &s->cnorms, &s->cfirst, &s->slot_count, &s->noise_drops, &s->nflag})
        release(*b);
    if (s->ctl) cudaFree(s->ctl);
    if (s->sort.hist) cudaFree(s->sort.hist);
    if (s->sort.base) cudaFree(s->sort.base);
    if (s->sort.host_hist) cudaFreeHost(s->sort.host_hist);
    if (s->sort.host_base) cudaFreeHost(s->sort.host_base);
    if (s->hcount) cudaFreeHost(s->hcount);
    if (s->hout) cudaFreeHost(s->hout);
    if (s->hhist) cudaFreeHost(s->hhist);
    if (s->hnorms) cudaFreeHost(s->hnorms);
    if (s->hfirst) cudaFreeHost(s->hfirst);
    s->prof.destroy();
    if (s->stream) cudaStreamDestroy(s->stream);
    delete s->levels;
    delete s->levels_next;
    delete s;
    return PS_OK;
}

const char* ps_last_error(const ps_sum* s) { return s ? s->err.c_str() : "null handle"; }
int32_t ps_width(const ps_sum* s) { return s ? s->W : 0; }
int32_t ps_num_qubits(const ps_sum* s) { return s ? s->nq : 0; }
int32_t ps_dtype_of(const ps_sum* s) { return s ? s->dtype : -1; }

ps_status ps_upload(ps_sum* s, const uint64_t* x, const uint64_t* z, const double* coeffs, uint64_t n) {
    if (!s) return PS_ERR_INVALID;
    if (n && (!x || !z || !coeffs)) return set_err(s, PS_ERR_INVALID, "upload: NULL array");
    DeviceGuard g(s->device);
    return dispatch<Engine>(s, [&](auto op) { return decltype(op)::upload(s, x, z, coeffs, n); });
}

ps_status ps_len(ps_sum* s, uint64_t* n) {
    if (!s || !n) return PS_ERR_INVALID;
    *n = s->slotted ? s->live_n : s->n;
    return PS_OK;
}

ps_status ps_download(ps_sum* s, uint64_t* x, uint64_t* z, double* coeffs, uint64_t cap, uint64_t* n) {
    if (!s) return PS_ERR_INVALID;
    DeviceGuard g(s->device);
    return dispatch<Engine>(s, [&](auto op) { return decltype(op)::download(s, x, z, coeffs, cap, n); });
}

ps_status ps_prepare_channel(int32_t num_qubits, int32_t dtype, const ps_channel* channel, int32_t adjoint,
                             ps_table* out) {
    (void)dtype;
    if (!out || !channel) return PS_ERR_INVALID;
    std::string why;
    return build_table(num_qubits, channel, adjoint, out, why);
}

ps_status ps_apply_layer(ps_sum* s, const ps_table* table, const ps_policy* policy, ps_layer_stats* stats) {
    if (!s || !table) return PS_ERR_INVALID;
    if (table->width != s->W) return set_err(s, PS_ERR_INVALID, "apply: table built for another width");
    DeviceGuard g(s->device);
    return dispatch<Engine>(s, [&](auto op) { return decltype(op)::apply(s, *table, policy, stats); });
}

ps_status ps_finalize_layer(ps_sum* s, const ps_policy* policy) {
    if (!s) return PS_ERR_INVALID;
    DeviceGuard g(s->device);
    KeepProg k;
    std::string why;
    ps_status ps = lower_keep(policy, k, why);
    if (ps != PS_OK) return set_err(s, ps, why);
    return dispatch<Engine>(s, [&](auto op) { return decltype(op)::finalize(s, policy); });
}

ps_status ps_propagate(ps_sum* s, const ps_channel* channels, uint64_t num_channels, const ps_policy* policy,
                       int32_t direction, uint64_t* terms_after, ps_run_stats* stats) {
    if (!s || (num_channels && !channels)) return PS_ERR_INVALID;
    if (direction != PS_FORWARD && direction != PS_HEISENBERG) return set_err(s, PS_ERR_INVALID, "bad direction");
    DeviceGuard g(s->device);
    KeepProg k;
    std::string why;
    ps_status ps = lower_keep(policy, k, why);
    if (ps != PS_OK) return set_err(s, ps, why);
    const bool adjoint = direction == PS_HEISENBERG;
    // Every channel is prepared before the first layer, so a bad channel fails the call
    // with the input untouched.
    std::vector<ps_table> tables(num_channels);
    for (uint64_t li = 0; li < num_channels; ++li) {
        uint64_t ci = adjoint ? num_channels - 1 - li : li;
        ps = build_table(s->nq, &channels[ci], adjoint ? 1 : 0, &tables[li], why);
        if (ps != PS_OK) return set_err(s, ps, "channel " + std::to_string(ci) + ": " + why);
    }
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, s->stream);
    s->pre_valid = false;  // a partner list (or flags) names a table of this call only
    s->nflag_valid = false;
    s->in_propagate = true;
    ps_run_stats rs;
    std::memset(&rs, 0, sizeof rs);
    rs.peak_terms = s->n;
    unsigned long long launches0 = 0;
    for (int i = 0; i < K_NUM_KERNELS; ++i) launches0 += s->prof.launches[i];
    const uint64_t collapses0 = s->collapses;
    for (uint64_t li = 0; li < num_channels; ++li) {
        ps_layer_stats ls;
        // A run of single-qubit noise channels folds into the rotation layer that follows it:
        // their factors are applied, in order and with the keep program after each, to every term
        // as the rotation reads it, so the run costs no pass of its own.
        uint64_t fj = li;
        while (fj < num_channels && fj - li < (uint64_t)kMaxNoise && foldable_noise(tables[fj], s->nq)) ++fj;
        if (fj > li && fj < num_channels && passes_idle(policy, s) && inherit_interval(policy, s) <= 1 &&
            dispatch<Engine>(s, [&](auto op) { return decltype(op)::folds_noise(tables[fj]) ? PS_OK : PS_ERR_UNSUPPORTED; }) ==
                PS_OK) {
            NoiseList N;
            std::memset(&N, 0, sizeof N);
            N.n = (int32_t)(fj - li);
            for (uint64_t q = li; q < fj; ++q) {
                const ps_table& t = tables[q];
                N.q[q - li] = (uint16_t)t.qubits[0];
                for (int p = 0; p < 4; ++p) {
                    N.f[q - li][p] = t.entries[0].amplitude[p];
                    N.ff[q - li][p] = (float)t.entries[0].amplitude[p];
                }
            }
            uint64_t after[kMaxNoise];
            const uint64_t n0 = s->n;
            s->next_table = fj + 1 < num_channels ? &tables[fj + 1] : nullptr;
            ps = dispatch<Engine>(s, [&](auto op) { return decltype(op)::apply(s, tables[fj], policy, &ls, &N, after); });
            if (ps == PS_OK && s->scorer) s->scorer_remaining -= (double)(fj - li);  // the folded layers' count-downs
            s->pass_call = fj;
            if (ps == PS_OK) ps = ps_finalize_layer(s, policy);
            s->next_table = nullptr;
            s->pass_call = 0;
            if (ps != PS_OK) {
                s->err = "layer " + std::to_string(fj) + " (with the noise of layers " + std::to_string(li) + "-" +
                         std::to_string(fj - 1) + " folded in): " + s->err;
                break;
            }
            for (uint64_t q = li; q < fj; ++q) {
                rs.total_terms_in += q == li ? n0 : after[q - li - 1];
                if (terms_after) terms_after[q] = after[q - li];
                ++rs.layers;
            }
            rs.total_terms_in += after[fj - li - 1];
            if (ls.terms_out > rs.peak_terms) rs.peak_terms = ls.terms_out;
            if (terms_after) terms_after[fj] = s->n;
            ++rs.layers;
            li = fj;
            continue;
        }
        rs.total_terms_in += s->n;
        const uint64_t skipped0 = s->layers_skipped, n_in = s->n;
        s->next_table = li + 1 < num_channels ? &tables[li + 1] : nullptr;
        ps = ps_apply_layer(s, &tables[li], policy, &ls);
        if (s->layers_skipped != skipped0) {
            ++rs.layers_skipped;
            rs.skipped_terms_in += n_in;
        }
        s->pass_call = li;  // CollapseSample's pass index of this layer
        if (ps == PS_OK) ps = ps_finalize_layer(s, policy);
        s->next_table = nullptr;
        s->pass_call = 0;
        if (ps != PS_OK) {
            s->err = "layer " + std::to_string(li) + ": " + s->err;
            break;
        }
        if (ls.terms_out > rs.peak_terms) rs.peak_terms = ls.terms_out;
        if (terms_after) terms_after[li] = s->n;
        ++rs.layers;
    }
    s->pre_valid = false;
    s->nflag_valid = false;
    s->next_table = nullptr;
    s->in_propagate = false;
    s->deferred = false;
    cudaEventRecord(e1, s->stream);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    rs.final_terms = s->n;
    rs.device_ms = ms;
    unsigned long long launches1 = 0;
    for (int i = 0; i < K_NUM_KERNELS; ++i) launches1 += s->prof.launches[i];
    rs.kernel_launches = launches1 - launches0;
    rs.collapses = s->collapses - collapses0;
    if (stats) *stats = rs;
    return ps;
}

ps_status ps_expectation(ps_sum* s, const uint64_t* axis_x, const uint64_t* axis_z, const uint64_t* negative,
                         double* out) {
    if (!s || !axis_x || !axis_z || !negative || !out) return PS_ERR_INVALID;
    DeviceGuard g(s->device);
    return dispatch<Engine>(s, [&](auto op) { return decltype(op)::expectation(s, axis_x, axis_z, negative, out); });
}

ps_status ps_set_profiling(ps_sum* s, int32_t enabled) {
    if (!s) return PS_ERR_INVALID;
    DeviceGuard g(s->device);
    s->prof.reset();
    s->prof.events = enabled != 0;
    return PS_OK;
}

ps_status ps_read_profile(ps_sum* s, ps_kernel_profile* out, int32_t cap, int32_t* count) {
    if (!s || !count || (cap > 0 && !out)) return PS_ERR_INVALID;
    static const char* kNames[K_NUM_KERNELS] = {"k_classify",     "k_level_scan", "k_level_apply", "k_partition",
                                                "k_merge",        "k_topn_hist",  "k_topn_step",  "k_topn_compact",
                                                "k_pack",         "k_sort_hist",  "k_sort_pass",  "k_dedup",
                                                "k_unpack",       "k_expect",     "k_gen_count",  "k_gen_branch",
                                                "k_score",        "k_score_train"};
    DeviceGuard g(s->device);
    s->prof.resolve();
    *count = K_NUM_KERNELS;
    for (int i = 0; i < K_NUM_KERNELS && i < cap; ++i) {
        std::memset(&out[i], 0, sizeof out[i]);
        std::strncpy(out[i].name, kNames[i], sizeof(out[i].name) - 1);
        out[i].launches = s->prof.launches[i];
        out[i].timed_launches = s->prof.timed[i];
        out[i].total_ms = s->prof.ms[i];
        out[i].algorithmic_bytes = s->prof.bytes[i];
    }
    return PS_OK;
}

ps_status ps_inject_fault(ps_sum* s, int32_t kind, uint64_t arg) {
    if (!s) return PS_ERR_INVALID;
    switch (kind) {
    case PS_FAULT_NONE:
        s->fault_oom_after = -1;
        s->fault_stall = false;
        s->stall_limit = 0;
        s->fault_flag = 0;
        break;
    case PS_FAULT_FLAG:
        s->fault_flag = arg ? (unsigned int)arg : 8u;  // ERR_INTERNAL
        break;
    case PS_FAULT_OOM:
        s->fault_oom_after = (long long)arg;
        break;
    case PS_FAULT_STALL:
        // the shortened limit reaches only the stalled merge's output-offset waits; every other
        // bounded wait of the handle keeps kSpinLimit
        s->fault_stall = true;
        s->stall_limit = arg ? arg : (unsigned long long)kSpinLimit;
        break;
    default: return PS_ERR_INVALID;
    }
    return PS_OK;
}

ps_status ps_synchronize(ps_sum* s) {
    if (!s) return PS_ERR_INVALID;
    DeviceGuard g(s->device);
    cudaError_t e = cudaStreamSynchronize(s->stream);
    return e == cudaSuccess ? PS_OK : cuda_fail(s, e, "synchronize");
}

ps_status ps_set_compensated_sums(ps_sum* s, int32_t enabled) {
    if (!s) return PS_ERR_INVALID;
    s->compensated = enabled != 0;
    return PS_OK;
}

// ---------------------------------------------------------------------------
// learned truncation: the scorer
// ---------------------------------------------------------------------------
ps_status ps_scorer_create(int32_t device, const ps_scorer_config* cfg, ps_scorer** out) {
    if (!out || !cfg) return PS_ERR_INVALID;
    *out = nullptr;
    if (cfg->num_qubits < 1 || cfg->num_qubits > 256 || !(cfg->layers_per_unit > 0.0)) return PS_ERR_INVALID;
    int count = ps_device_count();
    if (count == 0 || device < 0 || device >= count) return PS_ERR_NO_DEVICE;
    DeviceGuard g(device);
    ps_scorer* sc = new ps_scorer();
    sc->device = device;
    sc->nq = cfg->num_qubits;
    sc->W = width_for(cfg->num_qubits);
    sc->num_sites = sc->nq;
    sc->key_W = sc->W;
    sc->cfg = *cfg;
    sc->L = scorer_layout(sc->nq);
    cudaDeviceGetAttribute(&sc->sms, cudaDevAttrMultiProcessorCount, device);
    const size_t np = sc->L.total;
    // initial weights: N(0, init_scale) for the embedding rows and feature columns, N(0, 1/sqrt(128))
    // for the two dense layers, zero biases (splitmix64 stream, Box-Muller)
    std::vector<float> init(np, 0.0f);
    uint64_t state = cfg->seed;
    auto next = [&]() {
        uint64_t z = (state += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    };
    auto normal = [&]() {
        const double u1 = ((next() >> 11) + 1.0) * (1.0 / 9007199254740993.0), u2 = (next() >> 11) * (1.0 / 9007199254740992.0);
        return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
    };
    for (size_t i = sc->L.embed; i < sc->L.b1; ++i) init[i] = (float)(cfg->init_scale * normal());
    const double dense = 1.0 / std::sqrt((double)kHid);
    for (size_t i = sc->L.w2; i < sc->L.b2; ++i) init[i] = (float)(dense * normal());
    for (size_t i = sc->L.w3; i < sc->L.b3; ++i) init[i] = (float)(dense * normal());
    cudaError_t e = cudaStreamCreateWithFlags(&sc->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMalloc(&sc->ctl, sizeof(Ctl));
    if (e == cudaSuccess) e = cudaMemset(sc->ctl, 0, sizeof(Ctl));
    if (e == cudaSuccess) {
        static const unsigned long long limit = (unsigned long long)kSpinLimit;
        e = cudaMemcpy(&sc->ctl->spin_limit, &limit, sizeof(limit), cudaMemcpyHostToDevice);
    }
    if (e == cudaSuccess) e = ensure(sc->master, np * 4);
    if (e == cudaSuccess) e = ensure(sc->bf, np * 2);
    if (e == cudaSuccess) e = ensure(sc->grads, np * 4);
    if (e == cudaSuccess) e = ensure(sc->m, np * 4);
    if (e == cudaSuccess) e = ensure(sc->v, np * 4);
    if (e == cudaSuccess) e = ensure(sc->loss, 16);
    if (e == cudaSuccess) e = cudaMemcpy(sc->master.p, init.data(), np * 4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(sc->grads.p, 0, np * 4);
    if (e == cudaSuccess) e = cudaMemset(sc->m.p, 0, np * 4);
    if (e == cudaSuccess) e = cudaMemset(sc->v.p, 0, np * 4);
    if (e == cudaSuccess) e = launch_to_bf16((const float*)sc->master.p, (uint16_t*)sc->bf.p, np, sc->stream);
    if (e == cudaSuccess) {
        switch (sc->W) {
        case 1: e = configure_scorer_kernels<1>(); break;
        case 2: e = configure_scorer_kernels<2>(); break;
        default: e = configure_scorer_kernels<4>(); break;
        }
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(sc->stream);
    if (e != cudaSuccess) {
        ps_scorer_destroy(sc);
        cudaGetLastError();
        return e == cudaErrorMemoryAllocation ? PS_ERR_OOM : PS_ERR_DEVICE;
    }
    *out = sc;
    return PS_OK;
}

ps_status ps_scorer_destroy(ps_scorer* sc) {
    if (!sc) return PS_OK;
    DeviceGuard g(sc->device);
    if (sc->stream) cudaStreamSynchronize(sc->stream);
    for (Buf* b : {&sc->master, &sc->bf, &sc->grads, &sc->m, &sc->v, &sc->keys, &sc->logc, &sc->rem, &sc->target,
                   &sc->h1, &sc->gz1, &sc->dz2, &sc->scores, &sc->loss, &sc->site_map})
        release(*b);
    if (sc->ctl) cudaFree(sc->ctl);
    sc->prof.destroy();
    if (sc->stream) cudaStreamDestroy(sc->stream);
    delete sc;
    return PS_OK;
}

const char* ps_scorer_last_error(const ps_scorer* sc) { return sc ? sc->err.c_str() : "null scorer"; }
uint64_t ps_scorer_num_params(const ps_scorer* sc) { return sc ? (uint64_t)sc->L.total : 0; }

}  // extern "C"

namespace {

ps_status scorer_fail(ps_scorer* sc, ps_status st, const std::string& msg) {
    sc->err = msg;
    return st;
}

ps_status scorer_cuda(ps_scorer* sc, cudaError_t e, const char* where) {
    if (e == cudaErrorMemoryAllocation) cudaGetLastError();
    return scorer_fail(sc, e == cudaErrorMemoryAllocation ? PS_ERR_OOM : PS_ERR_DEVICE,
                       std::string(where) + ": " + cudaGetErrorString(e));
}

ps_status scorer_flags(ps_scorer* sc, const char* where) {
    unsigned int flags[2] = {0, 0};
    cudaError_t e = cudaMemcpyAsync(flags, &sc->ctl->err, sizeof(flags), cudaMemcpyDeviceToHost, sc->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(sc->stream);
    if (e != cudaSuccess) return scorer_cuda(sc, e, where);
    if (flags[0] == 0) return PS_OK;
    cudaMemsetAsync(&sc->ctl->err, 0, 2 * sizeof(unsigned int), sc->stream);
    cudaStreamSynchronize(sc->stream);
    char msg[160];
    snprintf(msg, sizeof msg, "%s: device check failed (flags %u, check %u)", where, flags[0], flags[1]);
    return scorer_fail(sc, (flags[0] & ERR_TIMEOUT) ? PS_ERR_TIMEOUT : PS_ERR_DEVICE, msg);
}

// inference: the site map applies; training (inference = false): always the identity
ScorerArgs scorer_args(const ps_scorer* sc, bool inference) {
    ScorerArgs A;
    A.p = static_cast<const uint16_t*>(sc->bf.p);
    A.L = sc->L;
    A.nq = sc->nq;
    for (int f = 0; f < 3; ++f) A.fscale[f] = sc->cfg.feature_scale[f];
    A.residual = sc->cfg.residual ? 1 : 0;
    A.site_row = inference && sc->mapped ? static_cast<const int16_t*>(sc->site_map.p) : nullptr;
    return A;
}

// Host feature arrays of n terms into the scorer's staging buffers.
cudaError_t scorer_stage(ps_scorer* sc, const uint64_t* keys, const float* logc, const float* rem, const float* target,
                         uint64_t n, int key_W = 0) {
    const size_t kb = (size_t)n * 16 * (key_W ? key_W : sc->W);
    cudaError_t e = ensure(sc->keys, kb ? kb : 16);
    if (e == cudaSuccess) e = ensure(sc->logc, n * 4 + 16);
    if (e == cudaSuccess) e = ensure(sc->rem, n * 4 + 16);
    if (e == cudaSuccess && target) e = ensure(sc->target, n * 4 + 16);
    if (e != cudaSuccess) return e;
    if (!n) return cudaSuccess;
    e = cudaMemcpyAsync(sc->keys.p, keys, kb, cudaMemcpyHostToDevice, sc->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(sc->logc.p, logc, n * 4, cudaMemcpyHostToDevice, sc->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(sc->rem.p, rem, n * 4, cudaMemcpyHostToDevice, sc->stream);
    if (e == cudaSuccess && target)
        e = cudaMemcpyAsync(sc->target.p, target, n * 4, cudaMemcpyHostToDevice, sc->stream);
    return e;
}

cudaError_t scorer_batch(ps_scorer* sc, uint64_t offset, uint64_t nb) {
    ScoreInput in{};
    in.keys = static_cast<const uint64_t*>(sc->keys.p) + offset * 2 * sc->W;
    in.logc = static_cast<const float*>(sc->logc.p) + offset;
    in.rem = static_cast<const float*>(sc->rem.p) + offset;
    in.n = nb;
    TrainScratch S{static_cast<uint16_t*>(sc->h1.p), static_cast<uint16_t*>(sc->gz1.p),
                   static_cast<uint16_t*>(sc->dz2.p)};
    const float* tgt = static_cast<const float*>(sc->target.p) + offset;
    const ScorerArgs A = scorer_args(sc, false);
    float* grads = static_cast<float*>(sc->grads.p);
    float* loss = static_cast<float*>(sc->loss.p);
    switch (sc->W) {
    case 1: return launch_train_batch<1>(A, in, tgt, 1.0f / (float)nb, S, grads, loss, sc->ctl, sc->sms, sc->stream, &sc->prof);
    case 2: return launch_train_batch<2>(A, in, tgt, 1.0f / (float)nb, S, grads, loss, sc->ctl, sc->sms, sc->stream, &sc->prof);
    default: return launch_train_batch<4>(A, in, tgt, 1.0f / (float)nb, S, grads, loss, sc->ctl, sc->sms, sc->stream, &sc->prof);
    }
}

cudaError_t scorer_train_scratch(ps_scorer* sc, uint64_t batch) {
    cudaError_t e = ensure(sc->h1, batch * kHid * 2);
    if (e == cudaSuccess) e = ensure(sc->gz1, batch * kHid * 2);
    if (e == cudaSuccess) e = ensure(sc->dz2, batch * kHid * 2);
    return e;
}

}  // namespace

extern "C" {

ps_status ps_scorer_get_params(ps_scorer* sc, float* out) {
    if (!sc || !out) return PS_ERR_INVALID;
    DeviceGuard g(sc->device);
    cudaError_t e = cudaMemcpyAsync(out, sc->master.p, sc->L.total * 4, cudaMemcpyDeviceToHost, sc->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(sc->stream);
    return e == cudaSuccess ? PS_OK : scorer_cuda(sc, e, "get_params");
}

ps_status ps_scorer_set_params(ps_scorer* sc, const float* in) {
    if (!sc || !in) return PS_ERR_INVALID;
    DeviceGuard g(sc->device);
    cudaError_t e = cudaMemcpyAsync(sc->master.p, in, sc->L.total * 4, cudaMemcpyHostToDevice, sc->stream);
    if (e == cudaSuccess) e = launch_to_bf16((const float*)sc->master.p, (uint16_t*)sc->bf.p, sc->L.total, sc->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(sc->stream);
    return e == cudaSuccess ? PS_OK : scorer_cuda(sc, e, "set_params");
}

ps_status ps_scorer_score(ps_scorer* sc, const uint64_t* keys, const float* logc, const float* rem, uint64_t n,
                          float* out) {
    if (!sc || (n && (!keys || !logc || !rem || !out))) return PS_ERR_INVALID;
    DeviceGuard g(sc->device);
    cudaError_t e = scorer_stage(sc, keys, logc, rem, nullptr, n, sc->key_W);
    if (e == cudaSuccess) e = ensure(sc->scores, n * 4 + 16);
    if (e != cudaSuccess) return scorer_cuda(sc, e, "score: staging");
    if (!n) return PS_OK;
    ScoreInput in{};
    in.keys = static_cast<const uint64_t*>(sc->keys.p);
    in.logc = static_cast<const float*>(sc->logc.p);
    in.rem = static_cast<const float*>(sc->rem.p);
    in.n = n;
    const ScorerArgs A = scorer_args(sc, true);
    float* sco = static_cast<float*>(sc->scores.p);
    switch (sc->key_W) {
    case 1: e = launch_score<1>(A, in, sco, nullptr, nullptr, sc->ctl, sc->sms, sc->stream, &sc->prof); break;
    case 2: e = launch_score<2>(A, in, sco, nullptr, nullptr, sc->ctl, sc->sms, sc->stream, &sc->prof); break;
    default: e = launch_score<4>(A, in, sco, nullptr, nullptr, sc->ctl, sc->sms, sc->stream, &sc->prof); break;
    }
    if (e != cudaSuccess) return scorer_cuda(sc, e, "score");
    ps_status ps = scorer_flags(sc, "score");
    if (ps != PS_OK) return ps;
    e = cudaMemcpyAsync(out, sco, n * 4, cudaMemcpyDeviceToHost, sc->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(sc->stream);
    return e == cudaSuccess ? PS_OK : scorer_cuda(sc, e, "score: readback");
}

ps_status ps_scorer_gradients(ps_scorer* sc, const uint64_t* keys, const float* logc, const float* rem,
                              const float* target, uint64_t n, float* grads_out, float* loss) {
    if (!sc || !n || n > 65536 || !keys || !logc || !rem || !target || !grads_out) return PS_ERR_INVALID;
    if (sc->mapped) return scorer_fail(sc, PS_ERR_INVALID, "gradients: clear the site map first (training rows use the embedding rows' own qubits)");
    DeviceGuard g(sc->device);
    cudaError_t e = scorer_stage(sc, keys, logc, rem, target, n);
    if (e == cudaSuccess) e = scorer_train_scratch(sc, n);
    if (e != cudaSuccess) return scorer_cuda(sc, e, "gradients: staging");
    cudaMemsetAsync(sc->grads.p, 0, sc->L.total * 4, sc->stream);
    cudaMemsetAsync(sc->loss.p, 0, 16, sc->stream);
    e = scorer_batch(sc, 0, n);
    if (e != cudaSuccess) return scorer_cuda(sc, e, "gradients");
    ps_status ps = scorer_flags(sc, "gradients");
    if (ps != PS_OK) return ps;
    float l = 0.f;
    e = cudaMemcpyAsync(grads_out, sc->grads.p, sc->L.total * 4, cudaMemcpyDeviceToHost, sc->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&l, sc->loss.p, 4, cudaMemcpyDeviceToHost, sc->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(sc->stream);
    cudaMemsetAsync(sc->grads.p, 0, sc->L.total * 4, sc->stream);
    if (e != cudaSuccess) return scorer_cuda(sc, e, "gradients: readback");
    if (loss) *loss = l / (float)n;
    return PS_OK;
}

ps_status ps_scorer_train(ps_scorer* sc, const uint64_t* keys, const float* logc, const float* rem, const float* target,
                          uint64_t n, int32_t epochs, int32_t batch, float lr, float* epoch_loss) {
    if (!sc || !n || !keys || !logc || !rem || !target || epochs < 1 || batch < 1 || batch > 65536 || !(lr > 0.f))
        return PS_ERR_INVALID;
    if (sc->mapped) return scorer_fail(sc, PS_ERR_INVALID, "train: clear the site map first (training rows use the embedding rows' own qubits)");
    DeviceGuard g(sc->device);
    const int K = 2 * sc->W;
    std::vector<uint64_t> pk((size_t)n * K);
    std::vector<float> pl(n), pr(n), pt(n);
    std::vector<uint64_t> perm(n);
    for (uint64_t i = 0; i < n; ++i) perm[i] = i;
    uint64_t state = sc->cfg.seed ^ 0xA5A5A5A5DEADBEEFull;
    auto next = [&]() {
        uint64_t z = (state += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    };
    cudaError_t e = scorer_train_scratch(sc, (uint64_t)batch);
    if (e != cudaSuccess) return scorer_cuda(sc, e, "train: scratch");
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    for (int ep = 0; ep < epochs; ++ep) {
        for (uint64_t i = n - 1; i > 0; --i) std::swap(perm[i], perm[next() % (i + 1)]);  // Fisher-Yates
        for (uint64_t i = 0; i < n; ++i) {
            const uint64_t j = perm[i];
            std::memcpy(&pk[i * K], &keys[j * K], K * sizeof(uint64_t));
            pl[i] = logc[j];
            pr[i] = rem[j];
            pt[i] = target[j];
        }
        e = scorer_stage(sc, pk.data(), pl.data(), pr.data(), pt.data(), n);
        if (e != cudaSuccess) return scorer_cuda(sc, e, "train: staging");
        cudaMemsetAsync(sc->loss.p, 0, 16, sc->stream);
        for (uint64_t off = 0; off < n; off += (uint64_t)batch) {
            const uint64_t nb = std::min<uint64_t>((uint64_t)batch, n - off);
            e = scorer_batch(sc, off, nb);
            if (e == cudaSuccess)
                e = launch_adam((float*)sc->master.p, (uint16_t*)sc->bf.p, (float*)sc->grads.p, (float*)sc->m.p,
                                (float*)sc->v.p, sc->L.total, lr, b1, b2, eps, ++sc->step, sc->stream);
            if (e != cudaSuccess) return scorer_cuda(sc, e, "train: step");
        }
        ps_status ps = scorer_flags(sc, "train");
        if (ps != PS_OK) return ps;
        float l = 0.f;
        e = cudaMemcpyAsync(&l, sc->loss.p, 4, cudaMemcpyDeviceToHost, sc->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(sc->stream);
        if (e != cudaSuccess) return scorer_cuda(sc, e, "train: loss");
        if (epoch_loss) epoch_loss[ep] = l / (float)n;
    }
    return PS_OK;
}

ps_status ps_scorer_set_site_map(ps_scorer* sc, int32_t num_sites, const int32_t* row_of_site) {
    if (!sc) return PS_ERR_INVALID;
    DeviceGuard g(sc->device);
    if (num_sites == 0 || !row_of_site) {
        sc->mapped = false;
        sc->num_sites = sc->nq;
        sc->key_W = sc->W;
        return PS_OK;
    }
    if (num_sites < 1 || num_sites > 256) return scorer_fail(sc, PS_ERR_INVALID, "set_site_map: 1 to 256 sites");
    std::vector<int16_t> rows(num_sites);
    for (int q = 0; q < num_sites; ++q) {
        if (row_of_site[q] < -1 || row_of_site[q] >= sc->nq)
            return scorer_fail(sc, PS_ERR_INVALID, "set_site_map: site " + std::to_string(q) + " maps outside the embedding rows");
        rows[q] = (int16_t)row_of_site[q];
    }
    const int kw = width_for(num_sites);
    cudaError_t e = ensure(sc->site_map, (size_t)num_sites * sizeof(int16_t) + 16);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(sc->site_map.p, rows.data(), (size_t)num_sites * sizeof(int16_t), cudaMemcpyHostToDevice,
                            sc->stream);
    if (e == cudaSuccess) {
        switch (kw) {
        case 1: e = configure_scorer_kernels<1>(); break;
        case 2: e = configure_scorer_kernels<2>(); break;
        default: e = configure_scorer_kernels<4>(); break;
        }
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(sc->stream);
    if (e != cudaSuccess) return scorer_cuda(sc, e, "set_site_map");
    sc->mapped = true;
    sc->num_sites = num_sites;
    sc->key_W = kw;
    return PS_OK;
}

ps_status ps_set_scorer(ps_sum* s, ps_scorer* sc, double remaining_layers) {
    if (!s) return PS_ERR_INVALID;
    if (sc && (sc->device != s->device || sc->num_sites != s->nq))
        return set_err(s, PS_ERR_INVALID, "set_scorer: the scorer was built (or site-mapped) for another device or qubit count");
    if (sc != s->scorer) s->f_valid = false;  // predictions of another scorer
    s->scorer = sc;
    s->scorer_remaining = remaining_layers;
    return PS_OK;
}

}  // extern "C"
