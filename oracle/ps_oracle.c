/*
 * ps_oracle.c -- CPU oracle for the Pauli-propagation layer path.
 *
 * TEST INFRASTRUCTURE ONLY (parity checker and timed CPU baseline); the product
 * library never links or calls it.  See ps_oracle.h for the reference
 * file:line each part restates.  Build with -ffp-contract=off: every product
 * and sum below must round exactly once, as the reference's Rust does.
 */
#include "ps_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

struct pso_sum {
    int W;
    int nq;
    int dtype;
    size_t n;
    size_t cap;
    uint64_t* keys; /* n x 2W */
    double* c64;
    float* c32;
};

/* ------------------------------------------------------------------------ */
/* key algebra: crates/paulistrings/src/pauli_string.rs                      */
/* ------------------------------------------------------------------------ */

static int key_cmp(const uint64_t* a, const uint64_t* b, int W) {
    for (int i = 0; i < 2 * W; ++i) {
        if (a[i] != b[i]) return a[i] < b[i] ? -1 : 1;
    }
    return 0;
}

/* commutes_with (pauli_string.rs:116-123): XOR-fold then one popcount. */
static int anticommutes(const uint64_t* k, const uint64_t* gx, const uint64_t* gz, int W) {
    uint64_t f = 0;
    for (int i = 0; i < W; ++i) f ^= (k[i] & gz[i]) ^ (k[W + i] & gx[i]);
    return __builtin_popcountll(f) & 1;
}

/* mul_assign phase exponent (pauli_string.rs:73-93): delta = 2bc + ab + cd - (a^c)(b^d) mod 4,
 * (a,b) = self (x,z), (c,d) = other (x,z). */
static unsigned product_phase(const uint64_t* k, const uint64_t* gx, const uint64_t* gz, int W) {
    unsigned d = 0;
    for (int i = 0; i < W; ++i) {
        uint64_t a = k[i], b = k[W + i], c = gx[i], e = gz[i];
        d += 2u * (unsigned)__builtin_popcountll(b & c);
        d += (unsigned)__builtin_popcountll(a & b);
        d += (unsigned)__builtin_popcountll(c & e);
        d -= (unsigned)__builtin_popcountll((a ^ c) & (b ^ e));
    }
    return d & 3u;
}

static unsigned key_weight(const uint64_t* k, int W) {
    unsigned w = 0;
    for (int i = 0; i < W; ++i) w += (unsigned)__builtin_popcountll(k[i] | k[W + i]);
    return w;
}

/* ------------------------------------------------------------------------ */
/* sum storage                                                              */
/* ------------------------------------------------------------------------ */

static void sum_reserve(pso_sum* s, size_t cap) {
    if (cap <= s->cap) return;
    size_t c = s->cap ? s->cap : 16;
    while (c < cap) c *= 2;
    s->keys = (uint64_t*)realloc(s->keys, c * 2 * (size_t)s->W * sizeof(uint64_t));
    if (s->dtype == PSO_F64)
        s->c64 = (double*)realloc(s->c64, c * sizeof(double));
    else
        s->c32 = (float*)realloc(s->c32, c * sizeof(float));
    s->cap = c;
}

pso_sum* pso_new(int W, int num_qubits, int dtype) {
    if (W < 1 || W > PSO_MAX_W || num_qubits < 1 || num_qubits > 64 * W) return NULL;
    if (dtype != PSO_F64 && dtype != PSO_F32) return NULL;
    pso_sum* s = (pso_sum*)calloc(1, sizeof(pso_sum));
    s->W = W;
    s->nq = num_qubits;
    s->dtype = dtype;
    return s;
}

void pso_free(pso_sum* s) {
    if (!s) return;
    free(s->keys);
    free(s->c64);
    free(s->c32);
    free(s);
}

size_t pso_len(const pso_sum* s) { return s->n; }
int pso_width(const pso_sum* s) { return s->W; }

void pso_get(const pso_sum* s, uint64_t* keys, double* coeffs) {
    if (keys) memcpy(keys, s->keys, s->n * 2 * (size_t)s->W * sizeof(uint64_t));
    if (coeffs) {
        for (size_t i = 0; i < s->n; ++i) coeffs[i] = s->dtype == PSO_F64 ? s->c64[i] : (double)s->c32[i];
    }
}

/* ------------------------------------------------------------------------ */
/* hash accumulator (the naive oracle's HashMap, test_support/oracle.rs:28-41) */
/* ------------------------------------------------------------------------ */

typedef struct {
    int W;
    int dtype;
    size_t mask;
    size_t used;
    uint64_t* keys;
    unsigned char* full;
    double* v64;
    float* v32;
    size_t* order; /* insertion order, for a deterministic walk */
} accum;

static uint64_t key_hash(const uint64_t* k, int W) {
    uint64_t h = 0x9E3779B97F4A7C15ull;
    for (int i = 0; i < 2 * W; ++i) {
        uint64_t v = k[i] + 0x9E3779B97F4A7C15ull * (uint64_t)(i + 1);
        v ^= v >> 30;
        v *= 0xBF58476D1CE4E5B9ull;
        v ^= v >> 27;
        v *= 0x94D049BB133111EBull;
        v ^= v >> 31;
        h = (h ^ v) * 0x100000001B3ull;
    }
    return h ^ (h >> 29);
}

static void accum_init(accum* a, int W, int dtype, size_t expect) {
    size_t cap = 64;
    while (cap < 2 * expect + 16) cap *= 2;
    a->W = W;
    a->dtype = dtype;
    a->mask = cap - 1;
    a->used = 0;
    a->keys = (uint64_t*)malloc(cap * 2 * (size_t)W * sizeof(uint64_t));
    a->full = (unsigned char*)calloc(cap, 1);
    a->v64 = dtype == PSO_F64 ? (double*)malloc(cap * sizeof(double)) : NULL;
    a->v32 = dtype == PSO_F32 ? (float*)malloc(cap * sizeof(float)) : NULL;
    a->order = (size_t*)malloc(cap * sizeof(size_t));
}

static void accum_free(accum* a) {
    free(a->keys);
    free(a->full);
    free(a->v64);
    free(a->v32);
    free(a->order);
}

static void accum_grow(accum* a);

static void accum_add(accum* a, const uint64_t* k, double v64, float v32) {
    if (2 * (a->used + 1) > a->mask + 1) accum_grow(a);
    int K = 2 * a->W;
    size_t h = (size_t)key_hash(k, a->W) & a->mask;
    while (a->full[h]) {
        if (memcmp(a->keys + h * K, k, (size_t)K * 8) == 0) {
            if (a->dtype == PSO_F64)
                a->v64[h] = a->v64[h] + v64;
            else
                a->v32[h] = a->v32[h] + v32;
            return;
        }
        h = (h + 1) & a->mask;
    }
    a->full[h] = 1;
    memcpy(a->keys + h * K, k, (size_t)K * 8);
    /* OR-insert ZERO then += out_c, as the reference's entry().or_insert(ZERO) += c */
    if (a->dtype == PSO_F64)
        a->v64[h] = 0.0 + v64;
    else
        a->v32[h] = 0.0f + v32;
    a->order[a->used++] = h;
}

static void accum_grow(accum* a) {
    accum b;
    accum_init(&b, a->W, a->dtype, a->mask + 1);
    int K = 2 * a->W;
    for (size_t i = 0; i < a->used; ++i) {
        size_t h = a->order[i];
        size_t g = (size_t)key_hash(a->keys + h * K, a->W) & b.mask;
        while (b.full[g]) g = (g + 1) & b.mask;
        b.full[g] = 1;
        memcpy(b.keys + g * K, a->keys + h * K, (size_t)K * 8);
        if (a->dtype == PSO_F64)
            b.v64[g] = a->v64[h];
        else
            b.v32[g] = a->v32[h];
        b.order[b.used++] = g;
    }
    accum_free(a);
    *a = b;
}

/* sort helper: indices into a key array */
static const uint64_t* g_sort_keys;
static int g_sort_W;
static int idx_cmp(const void* pa, const void* pb) {
    size_t a = *(const size_t*)pa, b = *(const size_t*)pb;
    return key_cmp(g_sort_keys + a * 2 * g_sort_W, g_sort_keys + b * 2 * g_sort_W, g_sort_W);
}

/* keep program (postfix), CoefficientThreshold / WeightCutoff / And / Or. */
static int keep_eval(const pso_policy* p, const uint64_t* k, int W, double c) {
    if (!p || p->num_nodes == 0) return 1;
    int stack[16];
    int sp = 0;
    for (int i = 0; i < p->num_nodes; ++i) {
        switch (p->op[i]) {
        case PSO_KEEP_TRUE: stack[sp++] = 1; break;
        case PSO_KEEP_COEFF: {
            double eps = p->farg[i];
            /* builtin.rs:29-31: eps < 0 || c.norm_sqr() > eps * eps, norm_sqr in f64 */
            stack[sp++] = (eps < 0.0) || (c * c > eps * eps);
            break;
        }
        case PSO_KEEP_WEIGHT: stack[sp++] = key_weight(k, W) <= (unsigned)p->iarg[i]; break;
        case PSO_KEEP_AND: {
            int b = stack[--sp], a = stack[--sp];
            stack[sp++] = a && b;
            break;
        }
        case PSO_KEEP_OR: {
            int b = stack[--sp], a = stack[--sp];
            stack[sp++] = a || b;
            break;
        }
        default: return 1;
        }
    }
    return sp ? stack[sp - 1] : 1;
}

/* Drain an accumulator into the sum: keep on the summed coefficient, drop exact zeros, sort. */
static void accum_drain(accum* a, pso_sum* s, const pso_policy* policy) {
    int W = s->W, K = 2 * W;
    size_t kept = 0;
    size_t* idx = (size_t*)malloc((a->used + 1) * sizeof(size_t));
    for (size_t i = 0; i < a->used; ++i) {
        size_t h = a->order[i];
        double v = a->dtype == PSO_F64 ? a->v64[h] : (double)a->v32[h];
        if (v != 0.0 && keep_eval(policy, a->keys + h * K, W, v)) idx[kept++] = h;
    }
    g_sort_keys = a->keys;
    g_sort_W = W;
    qsort(idx, kept, sizeof(size_t), idx_cmp);
    s->n = 0;
    sum_reserve(s, kept);
    for (size_t i = 0; i < kept; ++i) {
        memcpy(s->keys + i * K, a->keys + idx[i] * K, (size_t)K * 8);
        if (s->dtype == PSO_F64)
            s->c64[i] = a->v64[idx[i]];
        else
            s->c32[i] = a->v32[idx[i]];
    }
    s->n = kept;
    free(idx);
}

int pso_set(pso_sum* s, const uint64_t* keys, const double* coeffs, size_t n) {
    accum a;
    accum_init(&a, s->W, s->dtype, n);
    for (size_t i = 0; i < n; ++i) accum_add(&a, keys + i * 2 * (size_t)s->W, coeffs[i], (float)coeffs[i]);
    accum_drain(&a, s, NULL);
    accum_free(&a);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* prepared tables: channel/rotation.rs, channel/prepared.rs, ptm/noise.rs   */
/* ------------------------------------------------------------------------ */

typedef struct {
    unsigned local_delta;
    uint64_t mx[PSO_MAX_W], mz[PSO_MAX_W];
    double a64[16];
    float a32[16];
} entry_t;

typedef struct {
    int wide;               /* Prepared::Rotation (support > 2) */
    int k;                  /* support size for a local table */
    uint32_t q[2];
    int num_entries;
    entry_t e[16];
    /* wide rotation */
    uint64_t gx[PSO_MAX_W], gz[PSO_MAX_W];
    double cos64, sin64;
    float cos32, sin32;
} prepared_t;

/* rotation.rs:70-77: sin_cos with quarter turns snapped (signum as Rust: +0 -> +1, -0 -> -1). */
static void sin_cos_snap(double theta, double* sn, double* cs) {
    const double SNAP = 1e-15;
    double s = sin(theta), c = cos(theta);
    if (fabs(s) < SNAP) {
        *sn = 0.0;
        *cs = isnan(c) ? c : copysign(1.0, c);
    } else if (fabs(c) < SNAP) {
        *sn = isnan(s) ? s : copysign(1.0, s);
        *cs = 0.0;
    } else {
        *sn = s;
        *cs = c;
    }
}

static void lift(const prepared_t* p, unsigned d, uint64_t* mx, uint64_t* mz, int W) {
    memset(mx, 0, sizeof(uint64_t) * W);
    memset(mz, 0, sizeof(uint64_t) * W);
    for (int j = 0; j < p->k; ++j) {
        uint32_t q = p->q[j];
        if ((d >> (2 * j)) & 1u) mx[q / 64] |= 1ull << (q % 64);
        if ((d >> (2 * j + 1)) & 1u) mz[q / 64] |= 1ull << (q % 64);
    }
}

static unsigned support_bits(const prepared_t* p, const uint64_t* k, int W) {
    unsigned s = 0;
    for (int j = 0; j < p->k; ++j) {
        uint32_t q = p->q[j];
        s |= (unsigned)((k[q / 64] >> (q % 64)) & 1u) << (2 * j);
        s |= (unsigned)((k[W + q / 64] >> (q % 64)) & 1u) << (2 * j + 1);
    }
    return s;
}

static int build_generator(const pso_channel* ch, int W, int nq, uint64_t* gx, uint64_t* gz) {
    memset(gx, 0, sizeof(uint64_t) * W);
    memset(gz, 0, sizeof(uint64_t) * W);
    for (int j = 0; j < ch->num_support; ++j) {
        uint32_t q = ch->qubits[j];
        if ((int)q >= nq) return -1;
        uint64_t bit = 1ull << (q % 64);
        if ((gx[q / 64] | gz[q / 64]) & bit) return -1; /* repeated qubit */
        switch (ch->paulis[j]) {
        case 'X': gx[q / 64] |= bit; break;
        case 'Y': gx[q / 64] |= bit; gz[q / 64] |= bit; break;
        case 'Z': gz[q / 64] |= bit; break;
        case 'I': break;
        default: return -1;
        }
    }
    return 0;
}

/* ------------------------------------------------------------------------ */
/* PTM channels: ptm.rs, ptm/clifford.rs, ptm/unitary.rs, ptm/noise.rs       */
/* ------------------------------------------------------------------------ */

/* num-complex 0.4 arithmetic: (a+bi)(c+di) = (ac-bd) + (ad+bc)i, parts rounded once */
typedef struct {
    double re, im;
} cplx;

static cplx cx(double re, double im) {
    cplx v;
    v.re = re;
    v.im = im;
    return v;
}
static cplx cx_mul(cplx a, cplx b) { return cx(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re); }
static cplx cx_add(cplx a, cplx b) { return cx(a.re + b.re, a.im + b.im); }
static int cx_zero(cplx a) { return a.re == 0.0 && a.im == 0.0; }
/* a / (c + 0i): ((a.re c + a.im 0) / (c c + 0 0), (a.im c - a.re 0) / (c c + 0 0)) */
static cplx cx_div_real(cplx a, double c) {
    double nrm = c * c + 0.0 * 0.0;
    return cx((a.re * c + a.im * 0.0) / nrm, (a.im * c - a.re * 0.0) / nrm);
}

/* pauli_matrix (unitary.rs:82-90), I, X, Z, Y index order */
static void pauli_2x2(int idx, cplx* m) {
    cplx o = cx(1, 0), z = cx(0, 0), mo = cx(-1, 0), i = cx(0, 1), mi = cx(0, -1);
    cplx t[4][4] = {{o, z, z, o}, {z, o, o, z}, {o, z, z, mo}, {z, mi, i, z}};
    for (int q = 0; q < 4; ++q) m[q] = t[idx][q];
}

/* matmul (unitary.rs:92-106): zero a[i][k] skipped, sums from zero in k order */
static void cx_matmul(int N, const cplx* a, const cplx* b, cplx* out) {
    for (int q = 0; q < N * N; ++q) out[q] = cx(0, 0);
    for (int i = 0; i < N; ++i)
        for (int k = 0; k < N; ++k) {
            cplx aik = a[i * N + k];
            if (cx_zero(aik)) continue;
            for (int j = 0; j < N; ++j) out[i * N + j] = cx_add(out[i * N + j], cx_mul(aik, b[k * N + j]));
        }
}

/* the 2^k x 2^k matrix of local Pauli s; kron(P(s & 3), P(s >> 2)) for k = 2 (unitary.rs:37, 116-121) */
static void local_pauli_matrix(int k, int s, cplx* m) {
    cplx a[4], b[4];
    if (k == 1) {
        pauli_2x2(s, m);
        return;
    }
    pauli_2x2(s & 3, a);
    pauli_2x2(s >> 2, b);
    for (int r = 0; r < 4; ++r)
        for (int c = 0; c < 4; ++c) m[r * 4 + c] = cx_mul(a[(r / 2) * 2 + c / 2], b[(r % 2) * 2 + c % 2]);
}

/* unitary_1q / unitary_2q (unitary.rs:13-53): assert_unitary (1e-10, NaN fails), then
 * ptm[s][t] = clean(tr(P_t . U P_s U^dagger) / 2^k), clean snapping parts below 1e-12. */
static int unitary_ptm(int k, const double* mat, cplx ptm[16][16]) {
    int d = 1 << k, dim = 1 << (2 * k);
    cplx U[16], Ud[16], prod[16];
    for (int r = 0; r < d; ++r)
        for (int c = 0; c < d; ++c) U[r * d + c] = cx(mat[2 * (r * d + c)], mat[2 * (r * d + c) + 1]);
    for (int r = 0; r < d; ++r)
        for (int c = 0; c < d; ++c) Ud[r * d + c] = cx(U[c * d + r].re, -U[c * d + r].im);
    cx_matmul(d, Ud, U, prod);
    double largest = 0.0;
    for (int r = 0; r < d; ++r)
        for (int c = 0; c < d; ++c) {
            double dr = prod[r * d + c].re - (r == c ? 1.0 : 0.0), di = prod[r * d + c].im;
            double e = hypot(dr, di);
            if (e > largest || isnan(e)) largest = e;
        }
    if (!(largest <= 1e-10)) return -1;
    for (int s = 0; s < dim; ++s) {
        cplx Ps[16], t1[16], conj[16];
        local_pauli_matrix(k, s, Ps);
        cx_matmul(d, U, Ps, t1);
        cx_matmul(d, t1, Ud, conj);
        for (int t = 0; t < dim; ++t) {
            cplx Pt[16], m[16], tr = cx(0, 0);
            local_pauli_matrix(k, t, Pt);
            cx_matmul(d, Pt, conj, m);
            for (int i = 0; i < d; ++i) tr = cx_add(tr, m[i * d + i]);
            cplx v = cx_div_real(tr, (double)d);
            if (fabs(v.re) < 1e-12) v.re = 0.0;
            if (fabs(v.im) < 1e-12) v.im = 0.0;
            ptm[s][t] = v;
        }
    }
    return 0;
}

/* clifford_2q (clifford.rs:83-111): the signed permutation multiplied out from the images of
 * X0, Z0, X1, Z1 (packed x0 | z0 << 1 | x1 << 2 | z1 << 3), one i per input Y. */
static void clifford_2q_table(const unsigned images[4], cplx ptm[16][16]) {
    for (int index = 0; index < 16; ++index) {
        uint64_t prod[2] = {0, 0}; /* one-word key on qubits 0 and 1 */
        unsigned phase = 0;
        for (int g = 0; g < 4; ++g) {
            if (!((index >> g) & 1)) continue;
            unsigned im = images[g];
            uint64_t ox = (uint64_t)(im & 1u) | ((uint64_t)((im >> 2) & 1u) << 1);
            uint64_t oz = (uint64_t)((im >> 1) & 1u) | ((uint64_t)((im >> 3) & 1u) << 1);
            phase += product_phase(prod, &ox, &oz, 1);
            prod[0] ^= ox;
            prod[1] ^= oz;
        }
        unsigned y_count = (unsigned)(((index & 1) & ((index >> 1) & 1)) + (((index >> 2) & 1) & ((index >> 3) & 1)));
        phase = (phase + y_count) & 3u;
        unsigned t = (unsigned)((prod[0] & 1u) | ((prod[1] & 1u) << 1) | (((prod[0] >> 1) & 1u) << 2) |
                                (((prod[1] >> 1) & 1u) << 3));
        ptm[index][t] = cx(phase == 2u ? -1.0 : 1.0, 0.0);
    }
}

static void signed_perm_1q(const unsigned image[4], unsigned negated, cplx ptm[16][16]) {
    for (int s = 0; s < 4; ++s) ptm[s][image[s]] = cx(((negated >> s) & 1u) ? -1.0 : 1.0, 0.0);
}

static int in_unit(double v) { return v >= 0.0 && v <= 1.0; }

/* The constructor-order PTM of a named channel (k support qubits); -1 when the
 * constructor would panic. */
static int named_ptm(const pso_channel* ch, int* k_out, cplx ptm[16][16]) {
    for (int a = 0; a < 16; ++a)
        for (int b = 0; b < 16; ++b) ptm[a][b] = cx(0, 0);
    static const unsigned H[4] = {0, 2, 1, 3}, S[4] = {0, 3, 2, 1}, ID[4] = {0, 1, 2, 3};
    /* packed generator images: pack(x0, z0, x1, z1) = x0 | z0 << 1 | x1 << 2 | z1 << 3 */
    static const unsigned CNOT[4] = {1u | 4u, 2u, 4u, 2u | 8u};
    static const unsigned CZ[4] = {1u | 8u, 2u, 2u | 4u, 8u};
    static const unsigned SWAP[4] = {4u, 8u, 1u, 2u};
    int k = 1;
    switch (ch->kind) {
    case PSO_CH_DEPOLARIZE: {
        if (!in_unit(ch->param)) return -1;
        double sc = 1.0 - 4.0 * ch->param / 3.0;
        ptm[0][0] = cx(1, 0);
        for (int q = 1; q < 4; ++q) ptm[q][q] = cx(sc, 0);
        break;
    }
    case PSO_CH_HADAMARD: signed_perm_1q(H, 0x8u, ptm); break;
    case PSO_CH_PHASE: signed_perm_1q(S, 0x8u, ptm); break;
    case PSO_CH_PHASE_DAGGER: {
        /* phase_gate(q).adjoint(): the inverse signed permutation (ptm.rs:128-137) */
        unsigned inv[4], neg = 0;
        for (unsigned s = 0; s < 4; ++s) {
            inv[S[s]] = s;
            neg |= ((0x8u >> s) & 1u) << S[s];
        }
        signed_perm_1q(inv, neg, ptm);
        break;
    }
    case PSO_CH_PAULI_X: signed_perm_1q(ID, 0xCu, ptm); break;
    case PSO_CH_PAULI_Y: signed_perm_1q(ID, 0x6u, ptm); break;
    case PSO_CH_PAULI_Z: signed_perm_1q(ID, 0xAu, ptm); break;
    case PSO_CH_CNOT: k = 2; clifford_2q_table(CNOT, ptm); break;
    case PSO_CH_CZ: k = 2; clifford_2q_table(CZ, ptm); break;
    case PSO_CH_SWAP: k = 2; clifford_2q_table(SWAP, ptm); break;
    case PSO_CH_UNITARY:
        k = ch->num_support;
        if (k != 1 && k != 2) return -1;
        if (unitary_ptm(k, ch->matrix, ptm)) return -1;
        break;
    case PSO_CH_DEPHASING: {
        if (!in_unit(ch->param)) return -1;
        double sc = 1.0 - 2.0 * ch->param;
        ptm[0][0] = cx(1, 0);
        ptm[1][1] = cx(sc, 0);
        ptm[2][2] = cx(1, 0);
        ptm[3][3] = cx(sc, 0);
        break;
    }
    case PSO_CH_PAULI_CHANNEL: {
        double px = ch->params[0], py = ch->params[1], pz = ch->params[2];
        if (!in_unit(px) || !in_unit(py) || !in_unit(pz) || !(px + py + pz <= 1.0)) return -1;
        ptm[0][0] = cx(1, 0);
        ptm[1][1] = cx(1.0 - 2.0 * (py + pz), 0);
        ptm[2][2] = cx(1.0 - 2.0 * (px + py), 0);
        ptm[3][3] = cx(1.0 - 2.0 * (px + pz), 0);
        break;
    }
    case PSO_CH_DEPOLARIZING_2Q: {
        if (!in_unit(ch->param)) return -1;
        k = 2;
        double sc = 1.0 - 16.0 * ch->param / 15.0;
        for (int q = 0; q < 16; ++q) ptm[q][q] = cx(q ? sc : 1.0, 0);
        break;
    }
    case PSO_CH_AMPLITUDE_DAMPING: {
        double g = ch->param;
        if (!in_unit(g)) return -1;
        double tr = sqrt(1.0 - g);
        ptm[0][0] = cx(1, 0);
        ptm[0][2] = cx(g, 0);
        ptm[1][1] = cx(tr, 0);
        ptm[2][2] = cx(1.0 - g, 0);
        ptm[3][3] = cx(tr, 0);
        break;
    }
    default: return -1;
    }
    *k_out = k;
    return 0;
}

/* push_deltas (prepared.rs:257-281) then convert to the real type (prepared.rs:214-233):
 * one entry per local delta the table reaches, ascending; an imaginary part above 1e-12
 * declines the table. */
static int push_table(prepared_t* p, cplx table[16][16], int W) {
    int dim = 1 << (2 * p->k);
    int has[16] = {0};
    for (int s = 0; s < dim; ++s)
        for (int t = 0; t < dim; ++t)
            if (!cx_zero(table[s][t])) has[s ^ t] = 1;
    for (int d = 0; d < dim; ++d) {
        if (!has[d]) continue;
        entry_t* e = &p->e[p->num_entries++];
        e->local_delta = (unsigned)d;
        lift(p, (unsigned)d, e->mx, e->mz, W);
        for (int s = 0; s < dim; ++s) {
            cplx a = table[s][s ^ d];
            if (!(fabs(a.im) <= 1e-12)) return -1;
            e->a64[s] = a.re;
            e->a32[s] = (float)a.re;
        }
    }
    return 0;
}

/* RotationLayer::of Clifford residue rule (bucketed/rotation_layer.rs:101-122): on a
 * rotation-shaped table whose identity amplitudes are rounding residues of the generator
 * amplitudes, strings move instead of splitting. */
static void clifford_residue(prepared_t* p) {
    if (p->num_entries != 2 || p->e[0].local_delta != 0) return;
    int dim = 1 << (2 * p->k);
    entry_t* e0 = &p->e[0];
    entry_t* e1 = &p->e[1];
    unsigned delta = e1->local_delta;
    const double eps = 2.220446049250313e-16;
    for (int prec = 0; prec < 2; ++prec) {
        int clifford = 1, shaped = 1;
        for (int s = 0; s < dim; ++s) {
            double a0 = prec ? (double)e0->a32[s] : e0->a64[s];
            double a1 = prec ? (double)e1->a32[s] : e1->a64[s];
            double b1 = prec ? (double)e1->a32[s ^ delta] : e1->a64[s ^ delta];
            if (a1 == 0.0) {
                if (a0 != 1.0) shaped = 0;
            } else {
                if (b1 == 0.0) shaped = 0;
                clifford &= (a0 * a0 <= eps * eps * (a1 * a1));
            }
        }
        if (shaped && clifford) {
            for (int s = 0; s < dim; ++s) {
                if ((prec ? (double)e1->a32[s] : e1->a64[s]) == 0.0) continue;
                if (prec)
                    e0->a32[s] = 0.0f;
                else
                    e0->a64[s] = 0.0;
            }
        }
    }
}

static int prepare(const pso_channel* ch, int adjoint, int W, int nq, prepared_t* p) {
    memset(p, 0, sizeof(*p));
    adjoint = (adjoint != 0) ^ (ch->adjoint != 0);
    cplx table[16][16];
    for (int a = 0; a < 16; ++a)
        for (int b = 0; b < 16; ++b) table[a][b] = cx(0, 0);
    if (ch->kind == PSO_CH_ROTATION) {
        uint64_t gx[PSO_MAX_W], gz[PSO_MAX_W];
        if (build_generator(ch, W, nq, gx, gz)) return -1;
        double theta = adjoint ? -ch->param : ch->param;
        double sn, cs;
        sin_cos_snap(theta, &sn, &cs);
        unsigned weight = 0;
        for (int i = 0; i < W; ++i) weight += (unsigned)__builtin_popcountll(gx[i] | gz[i]);
        if (weight > 2) {
            /* Prepared::Rotation (rotation.rs:114-122, prepared.rs:387-397) */
            p->wide = 1;
            memcpy(p->gx, gx, sizeof(uint64_t) * W);
            memcpy(p->gz, gz, sizeof(uint64_t) * W);
            p->cos64 = cs;
            p->sin64 = sn;
            p->cos32 = (float)cs;
            p->sin32 = (float)sn;
            return 0;
        }
        /* LocalPtm::on_support: support qubits ascending */
        int k = 0;
        for (int w = 0; w < W; ++w) {
            uint64_t live = gx[w] | gz[w];
            while (live) {
                p->q[k++] = (uint32_t)(64 * w + __builtin_ctzll(live));
                live &= live - 1;
            }
        }
        p->k = k;
        int dim = 1 << (2 * k);
        /* probe_table: apply on each local basis Pauli with coefficient 1 */
        for (int s = 0; s < dim; ++s) {
            uint64_t key[2 * PSO_MAX_W];
            lift(p, (unsigned)s, key, key + W, W);
            if (!anticommutes(key, gx, gz, W)) {
                table[s][s].re += 1.0;
                continue;
            }
            table[s][s].re += 1.0 * cs;
            unsigned total = (1u + product_phase(key, gx, gz, W)) & 3u;
            double sgn = (total & 2u) ? -1.0 : 1.0; /* real mul_phase: even phase only */
            uint64_t out[2 * PSO_MAX_W];
            for (int i = 0; i < W; ++i) {
                out[i] = key[i] ^ gx[i];
                out[W + i] = key[W + i] ^ gz[i];
            }
            unsigned t = support_bits(p, out, W);
            table[s][t].re += sgn * sn;
        }
    } else {
        /* a PtmChannel: transfer_matrix (ptm.rs:248-263), transposed for the adjoint and
         * reordered to ascending-qubit local indices */
        cplx ptm[16][16];
        int k = 0;
        if (named_ptm(ch, &k, ptm)) return -1;
        if (ch->num_support != k) return -1;
        for (int j = 0; j < k; ++j)
            if ((int)ch->qubits[j] >= nq) return -1;
        if (k == 2 && ch->qubits[0] == ch->qubits[1]) return -1;
        int reversed = k == 2 && ch->qubits[0] > ch->qubits[1];
        p->k = k;
        p->q[0] = reversed ? ch->qubits[1] : ch->qubits[0];
        p->q[1] = k == 2 ? (reversed ? ch->qubits[0] : ch->qubits[1]) : 0;
        int dim = 1 << (2 * k);
        for (int s = 0; s < dim; ++s)
            for (int t = 0; t < dim; ++t) {
                if (cx_zero(ptm[s][t])) continue;
                int row = adjoint ? t : s, col = adjoint ? s : t;
                if (reversed) {
                    row = ((row & 3) << 2) | (row >> 2);
                    col = ((col & 3) << 2) | (col >> 2);
                }
                table[row][col] = cx_add(table[row][col], ptm[s][t]);
            }
    }
    if (push_table(p, table, W)) return -1;
    clifford_residue(p);
    return 0;
}

/* The prepared table of one channel, for comparing table builders: wide rotations report
 * wide = 1 and nothing else; local tables their support, entries (ascending local delta) and
 * float64 amplitudes amps[16 * e + s]. */
int pso_prepare_table(const pso_channel* ch, int adjoint, int W, int nq, int* wide, int* k, uint32_t* qubits,
                      int* num_entries, uint32_t* deltas, double* amps) {
    prepared_t p;
    if (W < 1 || W > PSO_MAX_W || prepare(ch, adjoint, W, nq, &p)) return -1;
    *wide = p.wide;
    *k = p.k;
    qubits[0] = p.q[0];
    qubits[1] = p.q[1];
    *num_entries = p.num_entries;
    for (int e = 0; e < p.num_entries; ++e) {
        deltas[e] = p.e[e].local_delta;
        for (int s = 0; s < 16; ++s) amps[16 * e + s] = p.e[e].a64[s];
    }
    return 0;
}

/* ------------------------------------------------------------------------ */
/* TopN (truncation/builtin.rs:73-129, 210-239)                              */
/* ------------------------------------------------------------------------ */

static double coef_at(const pso_sum* s, size_t i) { return s->dtype == PSO_F64 ? s->c64[i] : (double)s->c32[i]; }

static int mag_desc_cmp(const void* pa, const void* pb) {
    double a = *(const double*)pa, b = *(const double*)pb;
    /* descending, NaN last */
    int an = isnan(a), bn = isnan(b);
    if (an || bn) return an - bn;
    return (a < b) - (a > b);
}

static void topn(pso_sum* s, uint64_t n) {
    if (s->n <= n) return;
    if (n == 0) {
        s->n = 0;
        return;
    }
    size_t total = s->n;
    double* m = (double*)malloc(total * sizeof(double));
    for (size_t i = 0; i < total; ++i) {
        double c = coef_at(s, i);
        m[i] = c * c;
    }
    /* n-th largest |c|^2 by quickselect on a copy (select_nth_unstable, builtin.rs:107-111),
     * NaN ordered below every number */
    double* sel = (double*)malloc(total * sizeof(double));
    memcpy(sel, m, total * sizeof(double));
    size_t lo = 0, hi = total - 1, kth = (size_t)n - 1;
    while (lo < hi) {
        double pivot = sel[lo + (hi - lo) / 2];
        size_t i = lo, j = hi;
        while (i <= j) {
            while (mag_desc_cmp(&sel[i], &pivot) < 0) ++i;
            while (mag_desc_cmp(&sel[j], &pivot) > 0) --j;
            if (i <= j) {
                double t = sel[i];
                sel[i] = sel[j];
                sel[j] = t;
                ++i;
                if (j == 0) break;
                --j;
            }
        }
        if (kth <= j)
            hi = j;
        else if (kth >= i)
            lo = i;
        else
            break;
    }
    double boundary = sel[kth];
    free(sel);
    size_t above = 0;
    for (size_t i = 0; i < total; ++i)
        if (!isnan(m[i]) && (isnan(boundary) || m[i] > boundary)) ++above;
    size_t quota = (size_t)n - above;
    int K = 2 * s->W;
    size_t w = 0;
    for (size_t i = 0; i < total; ++i) {
        int side; /* +1 above, 0 at, -1 below */
        if (isnan(m[i]))
            side = -1;
        else if (isnan(boundary))
            side = 1;
        else
            side = m[i] > boundary ? 1 : (m[i] == boundary ? 0 : -1);
        int at = side == 0 && quota > 0;
        if (at) --quota;
        if (side == 1 || at) {
            if (w != i) {
                memmove(s->keys + w * K, s->keys + i * K, (size_t)K * 8);
                if (s->dtype == PSO_F64)
                    s->c64[w] = s->c64[i];
                else
                    s->c32[w] = s->c32[i];
            }
            ++w;
        }
    }
    s->n = w;
    free(m);
}

/* ApproxTopN (builtin.rs:240-468): octave = bits(|c|^2) >> 52, the histogram counting NaN in
 * the top bin; walk from the top, the first octave that overflows n is the boundary; keep
 * every non-NaN term above it and its first `quota` non-NaN terms in store (key) order. */
static void approx_topn(pso_sum* s, uint64_t n) {
    if (s->n <= n) return;
    if (n == 0) {
        s->n = 0;
        return;
    }
    static uint64_t hist[2048];
    memset(hist, 0, sizeof hist);
    size_t total = s->n;
    unsigned* oct = (unsigned*)malloc(total * sizeof(unsigned));
    unsigned char* nan = (unsigned char*)malloc(total);
    for (size_t i = 0; i < total; ++i) {
        double c = coef_at(s, i);
        double m = c * c;
        uint64_t bits;
        memcpy(&bits, &m, 8);
        nan[i] = (unsigned char)isnan(m);
        oct[i] = nan[i] ? 2047u : (unsigned)(bits >> 52);
        hist[oct[i]]++;
    }
    uint64_t above = 0;
    unsigned bin = 0;
    for (int b = 2047; b >= 0; --b) {
        if (above + hist[b] > n) {
            bin = (unsigned)b;
            break;
        }
        above += hist[b];
    }
    uint64_t quota = n - above;
    int K = 2 * s->W;
    size_t w = 0;
    for (size_t i = 0; i < total; ++i) {
        int keep = 0;
        if (!nan[i]) {
            if (oct[i] > bin)
                keep = 1;
            else if (oct[i] == bin && quota > 0) {
                keep = 1;
                --quota;
            }
        }
        if (!keep) continue;
        if (w != i) {
            memmove(s->keys + w * K, s->keys + i * K, (size_t)K * 8);
            if (s->dtype == PSO_F64)
                s->c64[w] = s->c64[i];
            else
                s->c32[w] = s->c32[i];
        }
        ++w;
    }
    s->n = w;
    free(oct);
    free(nan);
}

/* rng.rs: splitmix64 absorbs the key words, seeds xoshiro256++; uniform() is the first
 * output's top 53 bits scaled by 2^-53. */
static uint64_t rng_mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
static uint64_t rng_splitmix(uint64_t* state) {
    *state += 0x9E3779B97F4A7C15ull;
    return rng_mix64(*state);
}
static uint64_t rng_rotl(uint64_t x, int r) { return (x << r) | (x >> (64 - r)); }
static double keyed_uniform(uint64_t seed, uint64_t call) {
    uint64_t key[2] = {seed, call};
    uint64_t absorbed = 2;
    for (int i = 0; i < 2; ++i) {
        uint64_t t = absorbed ^ key[i];
        absorbed = rng_splitmix(&t);
    }
    uint64_t st[4];
    for (int i = 0; i < 4; ++i) st[i] = rng_splitmix(&absorbed);
    if (!(st[0] | st[1] | st[2] | st[3])) st[0] = 1;
    uint64_t out = rng_rotl(st[0] + st[3], 23) + st[0];
    return (double)(out >> 11) * (1.0 / 9007199254740992.0);
}

/* Test hooks for the stream: splitmix64's first output from `state`, xoshiro256++'s first two
 * outputs from `st`, and the keyed uniform. */
uint64_t pso_splitmix64_first(uint64_t state) { return rng_splitmix(&state); }
void pso_xoshiro_two(const uint64_t* st_in, uint64_t* out) {
    uint64_t st[4] = {st_in[0], st_in[1], st_in[2], st_in[3]};
    for (int k = 0; k < 2; ++k) {
        out[k] = rng_rotl(st[0] + st[3], 23) + st[0];
        uint64_t t = st[1] << 17;
        st[2] ^= st[0];
        st[3] ^= st[1];
        st[1] ^= st[2];
        st[0] ^= st[3];
        st[2] ^= t;
        st[3] = rng_rotl(st[3], 45);
    }
}
double pso_keyed_uniform(uint64_t seed, uint64_t call) { return keyed_uniform(seed, call); }

static uint64_t g_call_offset = 0; /* pso_propagate's layer index, added to the policy's call */
static uint64_t g_collapses = 0;
uint64_t pso_collapses(void) { return g_collapses; }

/* CollapseSample (collapse_sample.rs:80-172): the store's |c| end to end in key order, each
 * 1024-term block's start the left-to-right sum of the blocks before it and each boundary the
 * block start plus a running sum from 0.0; points (u + k) * h, h = sum / samples; a term holding
 * m points keeps (c / |c|) * (m * h). */
static void collapse_sample(pso_sum* s, uint64_t cache, uint64_t samples, uint64_t seed, uint64_t call) {
    size_t n = s->n;
    if (n <= cache || samples == 0) return;
    size_t nb = (n + 1023) / 1024;
    double* starts = (double*)malloc((nb + 1) * sizeof(double));
    double prefix = 0.0;
    for (size_t b = 0; b < nb; ++b) {
        size_t lo = b * 1024, hi = lo + 1024 < n ? lo + 1024 : n;
        double norm = 0.0;
        for (size_t i = lo; i < hi; ++i) norm = norm + fabs(coef_at(s, i));
        starts[b] = prefix;
        prefix = prefix + norm;
    }
    starts[nb] = prefix;
    double total = prefix;
    if (!(total > 0.0 && total <= 1.7976931348623157e308)) { /* assert_drawable */
        free(starts);
        return;
    }
    double u = keyed_uniform(seed, call), step = total / (double)samples;
    uint64_t* first = (uint64_t*)malloc((nb + 1) * sizeof(uint64_t));
    for (size_t b = 0; b <= nb; ++b) { /* SystematicPoints::below */
        double boundary = starts[b];
        if (boundary >= total) {
            first[b] = samples;
            continue;
        }
        uint64_t lo = 0, hi = samples;
        while (lo < hi) {
            uint64_t mid = lo + (hi - lo) / 2;
            if ((u + (double)mid) * step < boundary)
                lo = mid + 1;
            else
                hi = mid;
        }
        first[b] = lo;
    }
    int K = 2 * s->W;
    size_t w = 0;
    for (size_t b = 0; b < nb; ++b) {
        size_t lo = b * 1024, hi = lo + 1024 < n ? lo + 1024 : n;
        uint64_t next = first[b], end = first[b + 1];
        double running = 0.0;
        for (size_t i = lo; i < hi; ++i) {
            if (next == end) continue;
            double c = coef_at(s, i);
            double mag = fabs(c);
            running = running + mag;
            double boundary = 0.0 + (starts[b] + running);
            uint64_t stop = end;
            if (boundary < total) {
                stop = next;
                while (stop < end && (u + (double)stop) * step < boundary) ++stop;
            }
            uint64_t m = stop - next;
            next = stop;
            if (!m) continue;
            double v = (c / mag) * ((double)m * step);
            memmove(s->keys + w * K, s->keys + i * K, (size_t)K * 8);
            if (s->dtype == PSO_F64)
                s->c64[w] = v;
            else
                s->c32[w] = (float)v;
            ++w;
        }
    }
    s->n = w;
    ++g_collapses;
    free(first);
    free(starts);
}

void pso_finalize_layer(pso_sum* s, const pso_policy* policy) {
    if (!policy) return;
    for (int i = 0; i < policy->num_passes; ++i) {
        if (policy->pass_kind[i] == PSO_PASS_TOPN) topn(s, policy->pass_n[i]);
        if (policy->pass_kind[i] == PSO_PASS_APPROX_TOPN) approx_topn(s, policy->pass_n[i]);
        if (policy->pass_kind[i] == PSO_PASS_COLLAPSE_SAMPLE)
            collapse_sample(s, policy->pass_n[i], policy->pass_samples[i], policy->pass_seed[i],
                            policy->pass_call[i] + g_call_offset);
    }
}

/* ------------------------------------------------------------------------ */
/* the naive layer (test_support/oracle.rs:21-54)                            */
/* ------------------------------------------------------------------------ */

static void emit(accum* a, const uint64_t* k, int W, int dtype, double v64, float v32) {
    (void)W;
    (void)dtype;
    accum_add(a, k, v64, v32);
}

int pso_apply_channel(pso_sum* s, const pso_channel* ch, int adjoint, const pso_policy* policy) {
    prepared_t p;
    int W = s->W, K = 2 * W;
    if (prepare(ch, adjoint, W, s->nq, &p)) return -1;
    accum a;
    accum_init(&a, W, s->dtype, s->n * 2);
    uint64_t out[2 * PSO_MAX_W];
    for (size_t i = 0; i < s->n; ++i) {
        const uint64_t* k = s->keys + i * K;
        double c64 = s->dtype == PSO_F64 ? s->c64[i] : 0.0;
        float c32 = s->dtype == PSO_F32 ? s->c32[i] : 0.0f;
        if (p.wide) {
            /* rotation.rs:43-67 with the prepared cos/sin */
            if (!anticommutes(k, p.gx, p.gz, W)) {
                emit(&a, k, W, s->dtype, c64, c32);
                continue;
            }
            emit(&a, k, W, s->dtype, c64 * p.cos64, c32 * p.cos32);
            unsigned total = (1u + product_phase(k, p.gx, p.gz, W)) & 3u;
            for (int j = 0; j < W; ++j) {
                out[j] = k[j] ^ p.gx[j];
                out[W + j] = k[W + j] ^ p.gz[j];
            }
            double m64 = (total & 2u) ? -c64 : c64;
            float m32 = (total & 2u) ? -c32 : c32;
            emit(&a, out, W, s->dtype, m64 * p.sin64, m32 * p.sin32);
            continue;
        }
        /* DeltaEntry::emit (prepared.rs:50-68) */
        unsigned sp = support_bits(&p, k, W);
        for (int e = 0; e < p.num_entries; ++e) {
            const entry_t* en = &p.e[e];
            if (s->dtype == PSO_F64 ? en->a64[sp] == 0.0 : en->a32[sp] == 0.0f) continue;
            for (int j = 0; j < W; ++j) {
                out[j] = k[j] ^ en->mx[j];
                out[W + j] = k[W + j] ^ en->mz[j];
            }
            emit(&a, out, W, s->dtype, c64 * en->a64[sp], c32 * en->a32[sp]);
        }
    }
    accum_drain(&a, s, policy);
    accum_free(&a);
    pso_finalize_layer(s, policy);
    return 0;
}

int pso_propagate(pso_sum* s, const pso_channel* chans, size_t num_channels, const pso_policy* policy,
                  int direction, uint64_t* terms_after) {
    for (size_t li = 0; li < num_channels; ++li) {
        size_t ci = direction ? num_channels - 1 - li : li;
        g_call_offset = li;
        int rc = pso_apply_channel(s, &chans[ci], direction, policy);
        g_call_offset = 0;
        if (rc) return -1;
        if (terms_after) terms_after[li] = s->n;
    }
    return 0;
}

/* product_state.rs:84-101, summed in key order in f64 */
double pso_expectation(const pso_sum* s, const uint64_t* axis_x, const uint64_t* axis_z,
                       const uint64_t* negative) {
    int W = s->W, K = 2 * W;
    double acc = 0.0;
    for (size_t i = 0; i < s->n; ++i) {
        const uint64_t* k = s->keys + i * K;
        uint64_t mismatch = 0;
        unsigned sign = 0;
        for (int w = 0; w < W; ++w) {
            uint64_t sup = k[w] | k[W + w];
            mismatch |= (k[w] ^ (sup & axis_x[w])) | (k[W + w] ^ (sup & axis_z[w]));
            sign += (unsigned)__builtin_popcountll(sup & negative[w]);
        }
        if (mismatch) continue;
        double c = coef_at(s, i);
        acc += (sign & 1u) ? -c : c;
    }
    return acc;
}

/* ------------------------------------------------------------------------ */
/* sorted-store engine for CPU timing, in the reference host engine's shape:  */
/* rotation scan, linear partner order, merge-join with keep_term, all       */
/* parallel over chunks (crates/paulistrings/src/engine/bucketed.rs:376-490, */
/* bucketed/rotation_layer.rs:159-229, bucketed/partner_order.rs:16-140).    */
/* Same results as pso_apply_channel, bit for bit.                           */
/* ------------------------------------------------------------------------ */

static int g_threads = 0;
void pso_set_threads(int threads) { g_threads = threads; }

static int nthreads(void) {
#ifdef _OPENMP
    return g_threads > 0 ? g_threads : omp_get_max_threads();
#else
    return 1;
#endif
}

/* first differing bit rank (0 = most significant) of two distinct keys */
static unsigned div_rank(const uint64_t* a, const uint64_t* b, int W) {
    for (int i = 0; i < 2 * W; ++i) {
        uint64_t d = a[i] ^ b[i];
        if (d) return 64u * (unsigned)i + (unsigned)__builtin_clzll(d);
    }
    return 0xFFFFFFFFu;
}

typedef struct {
    int W, dtype;
    size_t n, cap;
    uint64_t* keys;
    double* c64;
    float* c32;
} cols_t;

static void cols_reserve(cols_t* c, size_t cap) {
    if (cap <= c->cap) return;
    c->keys = (uint64_t*)realloc(c->keys, cap * 2 * (size_t)c->W * 8);
    if (c->dtype == PSO_F64)
        c->c64 = (double*)realloc(c->c64, cap * sizeof(double));
    else
        c->c32 = (float*)realloc(c->c32, cap * sizeof(float));
    c->cap = cap;
}

/* pattern amplitude of the own row (identity entry) and partner (generator entry) */
static void rot_amps(const prepared_t* p, const uint64_t* k, int W, int dtype, double* a0, double* a1, float* f0,
                     float* f1, int* emits) {
    if (p->wide) {
        int ac = anticommutes(k, p->gx, p->gz, W);
        *emits = ac;
        *a0 = ac ? p->cos64 : 1.0;
        *f0 = ac ? p->cos32 : 1.0f;
        if (ac) {
            unsigned total = (1u + product_phase(k, p->gx, p->gz, W)) & 3u;
            *a1 = (total & 2u) ? -p->sin64 : p->sin64;
            *f1 = (total & 2u) ? -p->sin32 : p->sin32;
        } else {
            *a1 = 0.0;
            *f1 = 0.0f;
        }
        return;
    }
    unsigned sp = support_bits(p, k, W);
    *a0 = p->e[0].a64[sp];
    *f0 = p->e[0].a32[sp];
    if (p->num_entries > 1) {
        *a1 = p->e[1].a64[sp];
        *f1 = p->e[1].a32[sp];
    } else {
        *a1 = 0.0;
        *f1 = 0.0f;
    }
    *emits = dtype == PSO_F64 ? (*a1 != 0.0) : (*f1 != 0.0f);
}

int pso_apply_channel_sorted(pso_sum* s, const pso_channel* ch, int adjoint, const pso_policy* policy) {
    prepared_t p;
    const int W = s->W, K = 2 * W;
    if (prepare(ch, adjoint, W, s->nq, &p)) return -1;
    const int rotation = p.wide || (p.num_entries == 2 && p.e[0].local_delta == 0) ||
                         (p.num_entries == 1 && p.e[0].local_delta == 0);
    if (!rotation) return pso_apply_channel(s, ch, adjoint, policy);  /* general tables: naive path */
    const size_t n = s->n;
    const int T = nthreads();
    const uint64_t* gx = p.wide ? p.gx : p.e[p.num_entries > 1 ? 1 : 0].mx;
    const uint64_t* gz = p.wide ? p.gz : p.e[p.num_entries > 1 ? 1 : 0].mz;

    /* 1. scan: anticommuting rows, in row order, per chunk then concatenated */
    size_t* cnt = (size_t*)calloc((size_t)T + 1, sizeof(size_t));
    uint32_t* hit = (uint32_t*)malloc((n + 1) * sizeof(uint32_t));
#pragma omp parallel num_threads(T)
    {
#ifdef _OPENMP
        int t = omp_get_thread_num();
#else
        int t = 0;
#endif
        size_t lo = n * (size_t)t / (size_t)T, hi = n * (size_t)(t + 1) / (size_t)T, c = 0;
        for (size_t i = lo; i < hi; ++i) {
            double a0, a1;
            float f0, f1;
            int e;
            rot_amps(&p, s->keys + i * K, W, s->dtype, &a0, &a1, &f0, &f1, &e);
            c += (size_t)e;
        }
        cnt[t + 1] = c;
#pragma omp barrier
#pragma omp single
        for (int q = 0; q < T; ++q) cnt[q + 1] += cnt[q];
        size_t o = cnt[t];
        for (size_t i = lo; i < hi; ++i) {
            double a0, a1;
            float f0, f1;
            int e;
            rot_amps(&p, s->keys + i * K, W, s->dtype, &a0, &a1, &f0, &f1, &e);
            if (e) hit[o++] = (uint32_t)i;
        }
    }
    const size_t m = cnt[T];
    free(cnt);

    /* 2. partner order: slot of each partner in key order of k ^ g (linear scans over the
     * first-difference ranks; partner_order.rs:10-14) */
    uint32_t levels[2 * 64 * PSO_MAX_W];
    int nl = 0;
    for (int wi = 0; wi < K; ++wi) {
        uint64_t bits = wi < W ? gx[wi] : gz[wi - W];
        while (bits) {
            int b = 63 - __builtin_clzll(bits);
            levels[nl++] = 64u * (unsigned)wi + (unsigned)(63 - b);
            bits &= ~(1ull << b);
        }
    }
    int64_t* shift = (int64_t*)calloc(m + 1, sizeof(int64_t));
    uint32_t* dv = (uint32_t*)malloc((m + 1) * sizeof(uint32_t));
    dv[0] = 0;
#pragma omp parallel for num_threads(T) schedule(static)
    for (size_t j = 1; j < m; ++j) dv[j] = div_rank(s->keys + (size_t)hit[j - 1] * K, s->keys + (size_t)hit[j] * K, W);
    for (int l = 0; l < nl; ++l) {
        const uint32_t L = levels[l];
        size_t st = 0, sp = (size_t)-1;
        for (size_t j = 0; j < m; ++j) {   /* forward: upper halves move down */
            if (j == 0 || dv[j] < L) st = j;
            if (j != 0 && dv[j] == L) sp = j;
            if (sp != (size_t)-1 && sp > st) shift[j] -= (int64_t)(sp - st);
        }
        size_t e = m, q = m;
        for (size_t jj = m; jj-- > 0;) {   /* backward: lower halves move up */
            if (q < e) shift[jj] += (int64_t)(e - q);
            if (jj != 0 && dv[jj] < L) e = jj;
            if (jj != 0 && dv[jj] == L) q = jj;
        }
    }
    cols_t P = {W, s->dtype, 0, 0, NULL, NULL, NULL};
    cols_reserve(&P, m + 1);
#pragma omp parallel for num_threads(T) schedule(static)
    for (size_t j = 0; j < m; ++j) {
        const size_t row = hit[j], d = (size_t)((int64_t)j + shift[j]);
        const uint64_t* k = s->keys + row * K;
        double a0, a1;
        float f0, f1;
        int e;
        rot_amps(&p, k, W, s->dtype, &a0, &a1, &f0, &f1, &e);
        for (int w = 0; w < W; ++w) {
            P.keys[d * K + w] = k[w] ^ gx[w];
            P.keys[d * K + W + w] = k[W + w] ^ gz[w];
        }
        if (s->dtype == PSO_F64)
            P.c64[d] = s->c64[row] * a1;
        else
            P.c32[d] = s->c32[row] * f1;
    }
    P.n = m;
    free(shift);
    free(dv);
    free(hit);

    /* 3. merge-join own rows (scaled by a0) with the partners, own first on equal keys, keep
     * on the sum, drop exact zeros; merge-path split across threads */
    cols_t O = {W, s->dtype, 0, 0, NULL, NULL, NULL};
    cols_reserve(&O, n + m + 1);
    size_t* ocnt = (size_t*)calloc((size_t)T + 1, sizeof(size_t));
    size_t* obase = (size_t*)calloc((size_t)T + 1, sizeof(size_t));
#pragma omp parallel num_threads(T)
    {
#ifdef _OPENMP
        int t = omp_get_thread_num();
#else
        int t = 0;
#endif
        size_t tot = n + m;
        size_t d0 = tot * (size_t)t / (size_t)T, d1 = tot * (size_t)(t + 1) / (size_t)T;
        size_t bnd[2][2];
        for (int side = 0; side < 2; ++side) {
            size_t dd = side ? d1 : d0;
            size_t lo = dd > m ? dd - m : 0, hi = dd < n ? dd : n;
            while (lo < hi) {
                size_t mid = (lo + hi) / 2;
                if (key_cmp(s->keys + mid * K, P.keys + (dd - 1 - mid) * K, W) <= 0)
                    lo = mid + 1;
                else
                    hi = mid;
            }
            size_t i = lo, j = dd - lo;
            if (i > 0 && j < m && key_cmp(s->keys + (i - 1) * K, P.keys + j * K, W) == 0) ++j;
            bnd[side][0] = i;
            bnd[side][1] = j;
        }
        size_t i = bnd[0][0], j = bnd[0][1], ie = bnd[1][0], je = bnd[1][1];
        /* thread-local output, then one copy at the thread's offset */
        size_t cap = (ie - i) + (je > j ? je - j : 0) + 1;
        uint64_t* lk = (uint64_t*)malloc(cap * K * 8);
        double* l64 = (double*)malloc(cap * sizeof(double));
        float* l32 = (float*)malloc(cap * sizeof(float));
        size_t c = 0;
        while (i < ie || j < je) {
            int takeS = (j >= je) || (i < ie && key_cmp(s->keys + i * K, P.keys + j * K, W) <= 0);
            const uint64_t* k;
            double v64 = 0.0;
            float v32 = 0.0f;
            if (takeS) {
                k = s->keys + i * K;
                double a0, a1;
                float f0, f1;
                int e;
                rot_amps(&p, k, W, s->dtype, &a0, &a1, &f0, &f1, &e);
                v64 = s->dtype == PSO_F64 ? s->c64[i] * a0 : 0.0;
                v32 = s->dtype == PSO_F32 ? s->c32[i] * f0 : 0.0f;
                if (j < je && key_cmp(k, P.keys + j * K, W) == 0) {
                    if (s->dtype == PSO_F64)
                        v64 = v64 + P.c64[j];
                    else
                        v32 = v32 + P.c32[j];
                    ++j;
                }
                ++i;
            } else {
                k = P.keys + j * K;
                v64 = s->dtype == PSO_F64 ? P.c64[j] : 0.0;
                v32 = s->dtype == PSO_F32 ? P.c32[j] : 0.0f;
                ++j;
            }
            double v = s->dtype == PSO_F64 ? v64 : (double)v32;
            if (v != 0.0 && keep_eval(policy, k, W, v)) {
                memcpy(lk + c * K, k, (size_t)K * 8);
                l64[c] = v64;
                l32[c] = v32;
                ++c;
            }
        }
        ocnt[t + 1] = c;
#pragma omp barrier
#pragma omp single
        for (int q = 0; q < T; ++q) obase[q + 1] = obase[q] + ocnt[q + 1];
        size_t o = obase[t];
        memcpy(O.keys + o * K, lk, c * K * 8);
        if (s->dtype == PSO_F64)
            memcpy(O.c64 + o, l64, c * sizeof(double));
        else
            memcpy(O.c32 + o, l32, c * sizeof(float));
        free(lk);
        free(l64);
        free(l32);
    }
    O.n = obase[T];
    free(ocnt);
    free(obase);
    free(P.keys);
    free(P.c64);
    free(P.c32);
    /* swap in */
    free(s->keys);
    free(s->c64);
    free(s->c32);
    s->keys = O.keys;
    s->c64 = O.c64;
    s->c32 = O.c32;
    s->n = O.n;
    s->cap = O.cap;
    pso_finalize_layer(s, policy);
    return 0;
}

int pso_propagate_sorted(pso_sum* s, const pso_channel* chans, size_t num_channels,
                         const pso_policy* policy, int direction, uint64_t* terms_after) {
    for (size_t li = 0; li < num_channels; ++li) {
        size_t ci = direction ? num_channels - 1 - li : li;
        g_call_offset = li;
        int rc = pso_apply_channel_sorted(s, &chans[ci], direction, policy);
        g_call_offset = 0;
        if (rc) return -1;
        if (terms_after) terms_after[li] = s->n;
    }
    return 0;
}
