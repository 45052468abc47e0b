/*
 * CPU oracle for the Orion commitment (expander encode + SHA-256 Merkle tree)
 * -- TEST INFRASTRUCTURE ONLY. Only tests/ and bench.py's cpu_baseline leg
 * load it; the shipped library never links or calls it.
 *
 * Restates, in plain C:
 *   - glibc rand() (TYPE_3 additive feedback generator, the published glibc
 *     algorithm: 34-word state seeded by the 16807 LCG, 310 discarded outputs,
 *     r[i] = r[i-31] + r[i-3], output r[i] >> 1); the reference never seeds it,
 *     so its stream starts from seed 1 (TruePix-main/Orion/Orion_nonzk/include/
 *     linear_code/expanders.h:19-60 is its first consumer);
 *   - the expander graphs (expanders.h:19-60, parameter.h: alpha 0.238, r 1.72,
 *     degrees 10 / 20, distance threshold 13) and the recursive encoder
 *     (include/linear_code/linear_code_encode.h:8-72);
 *   - SHA-256 (FIPS 180-4) of one 64-byte block, as my_hhash
 *     (include/infrastructure/my_hhash.h:46-54 over flo-shani);
 *   - commit (src/VPD/linearPC.cpp:97-197): 128 columns of N/128 elements, row
 *     leaves chained over the 64 column pairs, h <- SHA256(h || x || y) with
 *     field elements as LE64(img) || LE64(real); padded rows use the zero-element
 *     chain; Merkle tree in heap order (src/infrastructure/merkle_tree.cpp:28-84).
 *
 * Parity pin: tests/golden/orion_golden.npz holds roots produced by the
 * reference sources themselves (oracle/orion_ref_harness.cpp, built by
 * `make -C oracle ref`), checked by tests/test_oracle.py.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef uint64_t u64;
typedef uint32_t u32;
typedef unsigned __int128 u128;
#define P61 ((u64)0x1FFFFFFFFFFFFFFFull)

/* ---- field (Fp2 = Fp[i]/(i^2+1)), elements stored as (img, real) ---- */
static inline u64 canon(u64 x) { return x >= P61 ? x - P61 : x; }
static inline u64 fadd(u64 a, u64 b) { return canon(a + b); }
static inline u64 fmul(u64 a, u64 b)
{
    u128 t = (u128)a * b;
    return canon(((u64)t & P61) + (u64)(t >> 61));
}
typedef struct { u64 img, real; } fe;
static inline fe feadd(fe a, fe b) { fe r = {fadd(a.img, b.img), fadd(a.real, b.real)}; return r; }
static inline fe femul(fe a, fe b)
{
    fe r;
    r.real = canon(fmul(a.real, b.real) + (P61 - fmul(a.img, b.img)));
    r.img = fadd(fmul(a.real, b.img), fmul(a.img, b.real));
    return r;
}

/* ---- glibc rand() ---- */
typedef struct { u32 r[34]; int i; } grand;

void oracle_glibc_seed(grand* g, u32 seed)
{
    int32_t r[34];
    r[0] = (int32_t)seed;
    for (int i = 1; i < 31; ++i) {
        long long v = (16807LL * r[i - 1]) % 2147483647LL;
        if (v < 0) v += 2147483647LL;
        r[i] = (int32_t)v;
    }
    for (int i = 31; i < 34; ++i) r[i] = r[i - 31];
    for (int i = 0; i < 34; ++i) g->r[i] = (u32)r[i];
    g->i = 34;
    /* discard 310 outputs */
    for (int k = 0; k < 310; ++k) {
        u32 v = g->r[(g->i - 31) % 34] + g->r[(g->i - 3) % 34];
        g->r[g->i % 34] = v;
        g->i++;
    }
}

static inline int grand_next(grand* g)
{
    u32 v = g->r[(g->i - 31) % 34] + g->r[(g->i - 3) % 34];
    g->r[g->i % 34] = v;
    g->i++;
    return (int)(v >> 1);
}

void oracle_glibc_stream(u32 seed, int n, int* out)
{
    grand g;
    oracle_glibc_seed(&g, seed);
    for (int i = 0; i < n; ++i) out[i] = grand_next(&g);
}

/* ---- expander graphs and encoder ---- */
#define CN 10
#define DN 20
#define THRESH 13
typedef struct { long long L, R; int degree; long long* nb; fe* w; } graph;
typedef struct { graph C[64], D[64]; int depth; } expanders;

static void gen_graph(grand* g, graph* gr, long long L, long long R, int d)
{
    gr->L = L;
    gr->R = R;
    gr->degree = d;
    gr->nb = (long long*)malloc(sizeof(long long) * (size_t)(L * d > 0 ? L * d : 1));
    gr->w = (fe*)malloc(sizeof(fe) * (size_t)(L * d > 0 ? L * d : 1));
    for (long long i = 0; i < L; ++i)
        for (int j = 0; j < d; ++j) {
            long long t = (long long)grand_next(g) % R;
            fe w;
            w.real = (u64)grand_next(g) % P61;
            w.img = (u64)grand_next(g) % P61;
            gr->nb[i * d + j] = t;
            gr->w[i * d + j] = w;
        }
}

static long long exp_init(grand* g, expanders* E, long long n, int dep)
{
    if (n <= THRESH) {
        if (dep > E->depth) E->depth = dep;
        return n;
    }
    long long R = (long long)(0.238 * (double)n);
    gen_graph(g, &E->C[dep], n, R, CN);
    long long L = exp_init(g, E, R, dep + 1);
    long long RD = (long long)((double)n * (1.72 - 1) - (double)L);
    gen_graph(g, &E->D[dep], L, RD, DN);
    return n + L + RD;
}

static long long enc_len(const expanders* E, long long n, int dep)
{
    if (n <= THRESH) return n;
    long long R = (long long)(0.238 * (double)n);
    long long L = enc_len(E, R, dep + 1);
    return n + L + E->D[dep].R;
}

static long long encode(const expanders* E, const fe* src, fe* dst, long long n, int dep)
{
    if (n <= THRESH) {
        memcpy(dst, src, sizeof(fe) * (size_t)n);
        return n;
    }
    const graph* C = &E->C[dep];
    const graph* D = &E->D[dep];
    long long R = (long long)(0.238 * (double)n);
    fe* y = (fe*)calloc((size_t)R + 1, sizeof(fe));
    for (long long i = 0; i < n; ++i)
        for (int d = 0; d < C->degree; ++d) {
            long long t = C->nb[i * C->degree + d];
            y[t] = feadd(y[t], femul(C->w[i * C->degree + d], src[i]));
        }
    memcpy(dst, src, sizeof(fe) * (size_t)n);
    long long L = encode(E, y, dst + n, R, dep + 1);
    free(y);
    fe* out = dst + n + L;
    memset(out, 0, sizeof(fe) * (size_t)D->R);
    for (long long i = 0; i < L; ++i)
        for (int d = 0; d < D->degree; ++d) {
            long long t = D->nb[i * D->degree + d];
            out[t] = feadd(out[t], femul(dst[n + i], D->w[i * D->degree + d]));
        }
    return n + L + D->R;
}

static void free_expanders(expanders* E)
{
    for (int d = 0; d < 64; ++d) {
        free(E->C[d].nb); free(E->C[d].w);
        free(E->D[d].nb); free(E->D[d].w);
    }
}

/* ---- SHA-256 (FIPS 180-4) of one 64-byte message ---- */
static const u32 K256[64] = {
    0x428a2f98, 0x71374491, 0xb5c0fbcf, 0xe9b5dba5, 0x3956c25b, 0x59f111f1, 0x923f82a4, 0xab1c5ed5,
    0xd807aa98, 0x12835b01, 0x243185be, 0x550c7dc3, 0x72be5d74, 0x80deb1fe, 0x9bdc06a7, 0xc19bf174,
    0xe49b69c1, 0xefbe4786, 0x0fc19dc6, 0x240ca1cc, 0x2de92c6f, 0x4a7484aa, 0x5cb0a9dc, 0x76f988da,
    0x983e5152, 0xa831c66d, 0xb00327c8, 0xbf597fc7, 0xc6e00bf3, 0xd5a79147, 0x06ca6351, 0x14292967,
    0x27b70a85, 0x2e1b2138, 0x4d2c6dfc, 0x53380d13, 0x650a7354, 0x766a0abb, 0x81c2c92e, 0x92722c85,
    0xa2bfe8a1, 0xa81a664b, 0xc24b8b70, 0xc76c51a3, 0xd192e819, 0xd6990624, 0xf40e3585, 0x106aa070,
    0x19a4c116, 0x1e376c08, 0x2748774c, 0x34b0bcb5, 0x391c0cb3, 0x4ed8aa4a, 0x5b9cca4f, 0x682e6ff3,
    0x748f82ee, 0x78a5636f, 0x84c87814, 0x8cc70208, 0x90befffa, 0xa4506ceb, 0xbef9a3f7, 0xc67178f2};
#define ROR(x, n) (((x) >> (n)) | ((x) << (32 - (n))))

static void sha_block(u32 st[8], const unsigned char* blk)
{
    u32 w[64];
    for (int t = 0; t < 16; ++t)
        w[t] = ((u32)blk[4 * t] << 24) | ((u32)blk[4 * t + 1] << 16) | ((u32)blk[4 * t + 2] << 8) |
               blk[4 * t + 3];
    for (int t = 16; t < 64; ++t) {
        u32 s0 = ROR(w[t - 15], 7) ^ ROR(w[t - 15], 18) ^ (w[t - 15] >> 3);
        u32 s1 = ROR(w[t - 2], 17) ^ ROR(w[t - 2], 19) ^ (w[t - 2] >> 10);
        w[t] = w[t - 16] + s0 + w[t - 7] + s1;
    }
    u32 a = st[0], b = st[1], c = st[2], d = st[3], e = st[4], f = st[5], g = st[6], h = st[7];
    for (int t = 0; t < 64; ++t) {
        u32 t1 = h + (ROR(e, 6) ^ ROR(e, 11) ^ ROR(e, 25)) + ((e & f) ^ (~e & g)) + K256[t] + w[t];
        u32 t2 = (ROR(a, 2) ^ ROR(a, 13) ^ ROR(a, 22)) + ((a & b) ^ (a & c) ^ (b & c));
        h = g; g = f; f = e; e = d + t1; d = c; c = b; b = a; a = t1 + t2;
    }
    st[0] += a; st[1] += b; st[2] += c; st[3] += d; st[4] += e; st[5] += f; st[6] += g; st[7] += h;
}

void oracle_sha256_64(const unsigned char* in, unsigned char* out)
{
    u32 st[8] = {0x6a09e667, 0xbb67ae85, 0x3c6ef372, 0xa54ff53a,
                 0x510e527f, 0x9b05688c, 0x1f83d9ab, 0x5be0cd19};
    unsigned char pad[64];
    memset(pad, 0, 64);
    pad[0] = 0x80;
    pad[62] = 0x02;  /* 512 bits, big-endian length */
    sha_block(st, in);
    sha_block(st, pad);
    for (int i = 0; i < 8; ++i) {
        out[4 * i] = (unsigned char)(st[i] >> 24);
        out[4 * i + 1] = (unsigned char)(st[i] >> 16);
        out[4 * i + 2] = (unsigned char)(st[i] >> 8);
        out[4 * i + 3] = (unsigned char)st[i];
    }
}

static void put_fe(unsigned char* p, fe x)
{
    for (int i = 0; i < 8; ++i) p[i] = (unsigned char)(x.img >> (8 * i));
    for (int i = 0; i < 8; ++i) p[8 + i] = (unsigned char)(x.real >> (8 * i));
}

/* ---- commit ---- */
long long oracle_encode_len(long long col_len)
{
    grand g;
    expanders E;
    memset(&E, 0, sizeof(E));
    oracle_glibc_seed(&g, 1);
    long long n = exp_init(&g, &E, col_len, 0);
    free_expanders(&E);
    return n;
}

/* codeword of one column of n elements (graphs from the default seed); dst
 * holds oracle_encode_len(n) elements. Returns that length. */
long long oracle_encode(const u64* src, long long n, u64* dst)
{
    grand g;
    expanders E;
    memset(&E, 0, sizeof(E));
    oracle_glibc_seed(&g, 1);
    exp_init(&g, &E, n, 0);
    long long len = encode(&E, (const fe*)src, (fe*)dst, n, 0);
    free_expanders(&E);
    return len;
}

/* src: N elements as (img, real) u64 pairs; writes the 32-byte root. Optionally
 * returns the leaves (rows x 32 bytes) when leaves != NULL. */
int oracle_orion_commit(const u64* src, long long N, unsigned char* root, unsigned char* leaves)
{
    if (N % 128 != 0) return -1;
    const long long col_len = N / 128, rows = 2 * col_len;
    grand g;
    expanders E;
    memset(&E, 0, sizeof(E));
    oracle_glibc_seed(&g, 1);
    const long long cw_len = exp_init(&g, &E, col_len, 0);
    if (cw_len != enc_len(&E, col_len, 0)) return -2;
    fe* cw = (fe*)calloc((size_t)(128 * (cw_len + 1)), sizeof(fe));
    for (int c = 0; c < 128; ++c)
        encode(&E, (const fe*)src + (size_t)c * col_len, cw + (size_t)c * cw_len, col_len, 0);
    unsigned char* stash = (unsigned char*)calloc((size_t)rows, 32);
    unsigned char blk[64];
    for (long long r = 0; r < cw_len; ++r) {
        unsigned char* h = stash + 32 * r;
        for (int j = 0; j < 64; ++j) {
            memcpy(blk, h, 32);
            put_fe(blk + 32, cw[(size_t)(2 * j) * cw_len + r]);
            put_fe(blk + 48, cw[(size_t)(2 * j + 1) * cw_len + r]);
            oracle_sha256_64(blk, h);
        }
    }
    unsigned char zl[32];
    memset(zl, 0, 32);
    for (int j = 0; j < 64; ++j) {
        memcpy(blk, zl, 32);
        memset(blk + 32, 0, 32);
        oracle_sha256_64(blk, zl);
    }
    for (long long r = cw_len; r < rows; ++r) memcpy(stash + 32 * r, zl, 32);
    if (leaves) memcpy(leaves, stash, (size_t)rows * 32);
    long long size = 1;
    while (size < rows) size *= 2;
    unsigned char* tree = (unsigned char*)calloc((size_t)(2 * size), 32);
    memcpy(tree + 32 * size, stash, (size_t)rows * 32);
    for (long long i = rows; i < size; ++i) {  /* padded leaves: SHA256(0^64) */
        memset(blk, 0, 64);
        oracle_sha256_64(blk, tree + 32 * (size + i));
    }
    for (long long k = size - 1; k >= 1; --k) {
        memcpy(blk, tree + 32 * (2 * k), 32);
        memcpy(blk + 32, tree + 32 * (2 * k + 1), 32);
        oracle_sha256_64(blk, tree + 32 * k);
    }
    memcpy(root, tree + 32, 32);
    free(tree);
    free(stash);
    free(cw);
    free_expanders(&E);
    return 0;
}

/* ---- Fp2 NTT (TruePix-main/Orion/Orion_nonzk/src/infrastructure/RS_polynomial.cpp:46-206) ----
 * fft: result[i] = P(w^i), i < order, P given by coef_len coefficients, w the
 * order-th root of unity of get_root_of_unity (src/linear_gkr/prime_field.cpp:60-73:
 * g = (real 2147483648, img 1033321771269002680) squared 62 - log2(order) times).
 * ifft: the coef_len coefficients whose evaluations on the coef_len-th roots of
 * unity are evals[i * (order / coef_len)]. Any exact transform gives the same
 * values; this one splits the order points into order/coef_len cosets. */
static fe fe_pow(fe a, u64 e)
{
    fe r = {0, 1};
    while (e) {
        if (e & 1) r = femul(r, a);
        a = femul(a, a);
        e >>= 1;
    }
    return r;
}

static fe root_of_unity(int lg)
{
    fe g = {1033321771269002680ull, 2147483648ull};
    for (int i = 0; i < 62 - lg; ++i) g = femul(g, g);
    return g;
}

static int ilog2(long long n)
{
    int k = 0;
    while ((1LL << k) < n) ++k;
    return k;
}

/* in-place radix-2 DFT of length m = 2^k: a[t] <- sum_j a[j] w^(jt) */
static void dft_inplace(fe* a, long long m, fe w)
{
    int k = ilog2(m);
    for (long long i = 1, j = 0; i < m; ++i) {
        long long bit = m >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) { fe t = a[i]; a[i] = a[j]; a[j] = t; }
    }
    for (int s = 1; s <= k; ++s) {
        long long len = 1LL << s, half = len >> 1;
        fe wl = fe_pow(w, (u64)(m / len));
        for (long long b = 0; b < m; b += len) {
            fe x = {0, 1};
            for (long long j = 0; j < half; ++j) {
                fe u = a[b + j], v = femul(a[b + j + half], x);
                a[b + j] = feadd(u, v);
                fe nv = {canon(P61 - v.img), canon(P61 - v.real)};
                a[b + j + half] = feadd(u, nv);
                x = femul(x, wl);
            }
        }
    }
}

int oracle_fft(const u64* coef, long long coef_len, long long order, u64* result)
{
    if (coef_len < 1 || order < coef_len || (coef_len & (coef_len - 1)) || (order & (order - 1)) ||
        order > (1LL << 27))
        return -1;
    const fe* c = (const fe*)coef;
    fe* out = (fe*)result;
    const fe w = root_of_unity(ilog2(order));
    const long long b = order / coef_len;
    const fe wb = fe_pow(w, (u64)b);
    fe* t = (fe*)malloc(sizeof(fe) * (size_t)coef_len);
    for (long long s = 0; s < b; ++s) {
        fe ws = fe_pow(w, (u64)s), x = {0, 1};
        for (long long j = 0; j < coef_len; ++j) { t[j] = femul(c[j], x); x = femul(x, ws); }
        dft_inplace(t, coef_len, wb);
        for (long long q = 0; q < coef_len; ++q) out[s + b * q] = t[q];
    }
    free(t);
    return 0;
}

int oracle_ifft(const u64* evals, long long coef_len, long long order, u64* result)
{
    if (coef_len < 1 || order < coef_len || (coef_len & (coef_len - 1)) || (order & (order - 1)) ||
        order > (1LL << 27))
        return -1;
    const fe* e = (const fe*)evals;
    fe* out = (fe*)result;
    const long long b = order / coef_len;
    for (long long i = 0; i < coef_len; ++i) out[i] = e[i * b];
    const int k = ilog2(coef_len);
    fe wi = fe_pow(root_of_unity(k), (u64)(coef_len - 1));  /* inverse root */
    dft_inplace(out, coef_len, wi);
    const fe inv_n = {0, k ? (1ull << (61 - k)) : 1ull};     /* 2^-k = 2^(61-k) mod p */
    for (long long i = 0; i < coef_len; ++i) out[i] = femul(out[i], inv_n);
    return 0;
}

/* ---- RS commit (include/poly_commitment/poly_commit.h:42-96 + src/VPD/fri.cpp:36-123) ----
 * 64 slices of 2^(L-6) elements; slice i -> IFFT -> FFT onto 2^(L-1) points
 * (l_eval[i][.]); codeword interleaved as w[(j << 7) | (i << 1) | h] =
 * l_eval[i][j + h * 2^(L-2)]; leaf j = chain over its 64 pairs of
 * h <- SHA256(x || y || h) from zero; Merkle tree over the 2^(L-2) leaves. */
int oracle_rs_commit(const u64* src, int log_len, unsigned char* root, u64* l_eval_out)
{
    if (log_len < 6 || log_len > 28) return -1;
    const long long real_cnt = 1LL << (log_len - 6), slice = 1LL << (log_len - 1);
    const long long total = slice * 64, n_leaves = slice / 2;
    fe* lev = (fe*)malloc(sizeof(fe) * (size_t)total);
    fe* tmp = (fe*)malloc(sizeof(fe) * (size_t)real_cnt);
    for (int i = 0; i < 64; ++i) {
        oracle_ifft(src + 2 * i * real_cnt, real_cnt, real_cnt, (u64*)tmp);
        oracle_fft((const u64*)tmp, real_cnt, slice, (u64*)(lev + i * slice));
    }
    free(tmp);
    if (l_eval_out) memcpy(l_eval_out, lev, sizeof(fe) * (size_t)total);
    unsigned char* tree = (unsigned char*)calloc((size_t)(2 * n_leaves), 32);
    unsigned char blk[64];
    for (long long j = 0; j < n_leaves; ++j) {
        unsigned char h[32];
        memset(h, 0, 32);
        for (int i = 0; i < 64; ++i) {
            put_fe(blk, lev[i * slice + j]);
            put_fe(blk + 16, lev[i * slice + j + n_leaves]);
            memcpy(blk + 32, h, 32);
            oracle_sha256_64(blk, h);
        }
        memcpy(tree + 32 * (n_leaves + j), h, 32);
    }
    for (long long k = n_leaves - 1; k >= 1; --k) {
        memcpy(blk, tree + 32 * (2 * k), 32);
        memcpy(blk + 32, tree + 32 * (2 * k + 1), 32);
        oracle_sha256_64(blk, tree + 32 * k);
    }
    memcpy(root, tree + 32, 32);
    free(tree);
    free(lev);
    return 0;
}

/* ---- tensor-product opening, prover side (src/VPD/linearPC.cpp:480-531,569-571) ----
 * combined[t] = sum_j r0[j] * codeword_j[t] (t < cw_len; its first N/128 entries
 * are combined_message); leaves i < 2 N/128 = SHA256(combined[i] || 0^48) (zero
 * element beyond cw_len; merkle_tree.cpp:5-13), tree as in the commit;
 * answer = sum_{i < N/128} r1[i] * combined[i]. r0: 128 elements, r1: N/128. */
int oracle_orion_combine(const u64* src, long long N, const u64* r0, const u64* r1, u64* combined_out,
                         unsigned char* root, u64* answer)
{
    if (N % 128 != 0) return -1;
    const long long col_len = N / 128, rows = 2 * col_len;
    grand g;
    expanders E;
    memset(&E, 0, sizeof(E));
    oracle_glibc_seed(&g, 1);
    const long long cw_len = exp_init(&g, &E, col_len, 0);
    fe* cw = (fe*)calloc((size_t)(cw_len + 1), sizeof(fe));
    fe* comb = (fe*)calloc((size_t)(cw_len + 1), sizeof(fe));
    for (int c = 0; c < 128; ++c) {
        encode(&E, (const fe*)src + (size_t)c * col_len, cw, col_len, 0);
        const fe r = ((const fe*)r0)[c];
        for (long long t = 0; t < cw_len; ++t) comb[t] = feadd(comb[t], femul(r, cw[t]));
    }
    if (combined_out) memcpy(combined_out, comb, sizeof(fe) * (size_t)cw_len);
    fe ans = {0, 0};
    for (long long i = 0; i < col_len; ++i) ans = feadd(ans, femul(((const fe*)r1)[i], comb[i]));
    answer[0] = ans.img;
    answer[1] = ans.real;
    long long size = 1;
    while (size < rows) size *= 2;
    unsigned char* tree = (unsigned char*)calloc((size_t)(2 * size), 32);
    unsigned char blk[64];
    for (long long i = 0; i < size; ++i) {
        memset(blk, 0, 64);
        if (i < rows) {
            fe x = {0, 0};
            if (i < cw_len) x = comb[i];
            put_fe(blk, x);
        }
        oracle_sha256_64(blk, tree + 32 * (size + i));
    }
    for (long long k = size - 1; k >= 1; --k) {
        memcpy(blk, tree + 32 * (2 * k), 32);
        memcpy(blk + 32, tree + 32 * (2 * k + 1), 32);
        oracle_sha256_64(blk, tree + 32 * k);
    }
    memcpy(root, tree + 32, 32);
    free(tree);
    free(comb);
    free(cw);
    free_expanders(&E);
    return 0;
}

/* ---- Virgo sumcheck round (src/linear_gkr/prover.cpp:576-644, 935-1006) ----
 * tables of n linear_poly {a, b} (two elements each); folded into n/2 entries;
 * ret = {a, b, c} of the round polynomial over the folded tables. */
static void fold_lp(const fe* t, long long i, fe r, int bit, fe* ya, fe* yb)
{
    const fe a0 = t[4 * i], b0 = t[4 * i + 1], a1 = t[4 * i + 2], b1 = t[4 * i + 3];
    fe neg;
    if (!bit) {
        *yb = b0;
        neg.img = canon(P61 - b0.img);
        neg.real = canon(P61 - b0.real);
        *ya = feadd(b1, neg);
    } else {
        *yb = feadd(femul(a0, r), b0);
        neg.img = canon(P61 - yb->img);
        neg.real = canon(P61 - yb->real);
        *ya = feadd(feadd(femul(a1, r), b1), neg);
    }
}

int oracle_virgo_update(const u64* vma, const u64* addv, const u64* ams, long long n, const u64* r, int bit,
                        u64* vma_out, u64* addv_out, u64* ams_out, u64* ret)
{
    if (n < 2 || (n & 1)) return -1;
    const fe R = {r[0], r[1]};
    fe qa = {0, 0}, qb = {0, 0}, qc = {0, 0};
    for (long long i = 0; i < n / 2; ++i) {
        fe va, vb, da, db, ma, mb;
        fold_lp((const fe*)vma, i, R, bit, &va, &vb);
        fold_lp((const fe*)addv, i, R, bit, &da, &db);
        fold_lp((const fe*)ams, i, R, bit, &ma, &mb);
        ((fe*)vma_out)[2 * i] = va; ((fe*)vma_out)[2 * i + 1] = vb;
        ((fe*)addv_out)[2 * i] = da; ((fe*)addv_out)[2 * i + 1] = db;
        ((fe*)ams_out)[2 * i] = ma; ((fe*)ams_out)[2 * i + 1] = mb;
        qa = feadd(qa, femul(ma, va));
        qb = feadd(qb, feadd(feadd(femul(ma, vb), femul(mb, va)), da));
        qc = feadd(qc, feadd(femul(mb, vb), db));
    }
    ret[0] = qa.img; ret[1] = qa.real;
    ret[2] = qb.img; ret[3] = qb.real;
    ret[4] = qc.img; ret[5] = qc.real;
    return 0;
}

/* ---- FRI commit-phase step (src/VPD/fri.cpp:316-420) ----
 * Previous witness in the interleaved layout w[(k << 7) | (j << 1) | h] = slice
 * j's value at k + h M/2 (M = 2^log_m per slice, k < M/2). For i < M/2:
 * v[i][j] = 2^-1 ((x + y) + w_M^-i r (x - y)), x = w[(i<<7)|(j<<1)], y = the
 * next one; re-interleaved: next[(i<<7)|(j<<1)|h] = v[i + h M/4][j], i < M/4;
 * leaf i = chain over j of SHA256(next[..|0] || next[..|1] || h); tree. */
int oracle_fri_step(const u64* w, int log_m, const u64* r, u64* next, unsigned char* root)
{
    if (log_m < 2 || log_m > 26) return -1;
    const long long M = 1LL << log_m, nxt = M / 2, nl = nxt / 2;
    const fe* W = (const fe*)w;
    fe* N = (fe*)next;
    const fe R = {r[0], r[1]};
    const fe omega = root_of_unity(log_m);
    const fe inv_omega = fe_pow(omega, (u64)(M - 1));
    const fe inv2 = {0, 1ull << 60};
    fe inv_mu = {0, 1};   /* w^-i, i = 0 */
    for (long long i = 0; i < nxt; ++i) {
        const fe t = femul(inv_mu, R);
        for (int j = 0; j < 64; ++j) {
            const fe x = W[(i << 7) | (j << 1)], y = W[(i << 7) | (j << 1) | 1];
            fe d;
            d.img = canon(x.img + (P61 - y.img));
            d.real = canon(x.real + (P61 - y.real));
            const fe v = femul(inv2, feadd(feadd(x, y), femul(t, d)));
            if (i < nl)
                N[(i << 7) | (j << 1)] = v;
            else
                N[((i - nl) << 7) | (j << 1) | 1] = v;
        }
        inv_mu = femul(inv_mu, inv_omega);
    }
    unsigned char* tree = (unsigned char*)calloc((size_t)(2 * nl), 32);
    unsigned char blk[64];
    for (long long i = 0; i < nl; ++i) {
        unsigned char h[32];
        memset(h, 0, 32);
        for (int j = 0; j < 64; ++j) {
            put_fe(blk, N[(i << 7) | (j << 1)]);
            put_fe(blk + 16, N[(i << 7) | (j << 1) | 1]);
            memcpy(blk + 32, h, 32);
            oracle_sha256_64(blk, h);
        }
        memcpy(tree + 32 * (nl + i), h, 32);
    }
    for (long long k = nl - 1; k >= 1; --k) {
        memcpy(blk, tree + 32 * (2 * k), 32);
        memcpy(blk + 32, tree + 32 * (2 * k + 1), 32);
        oracle_sha256_64(blk, tree + 32 * k);
    }
    memcpy(root, tree + 32, 32);
    free(tree);
    return 0;
}

/*
 * The polynomial of a frame in TruePix's layout, optionally masked
 * (TruePix-main/Orion/Orion_zk/include/truepix/truepix_gkr.h: load_coefs
 * :157-206, mask_hides_index / fill_mask :333-362, alloc_masked_from_seed
 * :374-384). out[f], f < padded * W, real parts only (the imaginary parts are 0):
 *   mode 0: pixel[copy * cs + wire] for wire < cs, const_val at const_idx
 *           (copy < copies), 0 elsewhere;
 *   mode 1: mode 0 + mask; mode 2: the mask.
 * The mask walks the indices in order with one splitmix64 state (seeded with
 * `seed`) and draws the next output, reduced mod p, at each private wire
 * (wire < cs, copy < copies); it is 0 elsewhere.
 */
static u64 splitmix64_next(u64* state)
{
    *state += 0x9E3779B97F4A7C15ULL;
    u64 z = *state;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

int oracle_frame_vector(const unsigned char* pix, int copies, int padded, int cs, int W, int const_idx,
                        u64 const_val, u64 seed, int mode, u64* out)
{
    if (mode < 0 || mode > 2 || copies > padded || cs > W) return -1;
    u64 state = seed;
    const long long n = (long long)padded * W;
    for (long long f = 0; f < n; ++f) {
        const long long copy = f / W;
        const int wire = (int)(f % W);
        u64 v = 0;
        if (copy < copies && mode != 2) {
            if (wire < cs) v = pix[copy * cs + wire];
            else if (wire == const_idx) v = const_val;
        }
        if (mode != 0 && copy < copies && wire < cs) v = fadd(v, splitmix64_next(&state) % P61);
        out[f] = v;
    }
    return 0;
}

/* ---- Virgo layer inits (zk_prover::sumcheck_phase1_init, prover.cpp:246-570;
 * sumcheck_phase2_init, prover.cpp:645-930) ----
 * A layer of n_gates = 2^length_g gates (type ty, inputs u, v; type 14 gates
 * carry (src, weight) lists comb_src/comb_w[comb_ptr[g] .. comb_ptr[g+1])) over a
 * previous layer of total_uv = 2^length_u values. Tables are linear_poly arrays
 * {a, b} of total_uv entries. tmp_g(i) = alpha eq(r0, i) + beta eq(r1, i), eq with
 * bit k of i <-> r[k]. Unknown gate types contribute nothing (the reference
 * prints a warning and skips them). Returns -1 on an index outside its range. */
static fe fe_of(const u64* p) { fe x = {p[0], p[1]}; return x; }
static void put_lp(u64* t, long long i, fe a, fe b) { t[4 * i] = a.img; t[4 * i + 1] = a.real; t[4 * i + 2] = b.img; t[4 * i + 3] = b.real; }
static fe fesub(fe a, fe b) { fe r = {fadd(a.img, canon(P61 - b.img)), fadd(a.real, canon(P61 - b.real))}; return r; }

static fe eq_at(const u64* r, int len, long long i, fe s)
{
    const fe one = {0, 1};
    for (int k = 0; k < len; ++k) s = femul(s, ((i >> k) & 1) ? fe_of(r + 2 * k) : fesub(one, fe_of(r + 2 * k)));
    return s;
}

static int virgo_layer_ok(long long n_gates, const int* ty, const long long* u, const long long* v, const int* comb_ptr,
                          const int* comb_src, int length_g, int length_u)
{
    const long long G = 1LL << length_g, U = 1LL << length_u;
    if (n_gates != G) return 0;
    for (long long g = 0; g < G; ++g) {
        switch (ty[g]) {
        case 0: case 1: case 6: case 7: case 8: case 9: case 10: case 13:
            if (u[g] < 0 || u[g] >= U || v[g] < 0 || v[g] >= U) return 0;
            break;
        case 4:   /* u indexes both the gate randoms and the table */
            if (u[g] < 0 || u[g] >= G || u[g] >= U || v[g] < 0 || v[g] >= U) return 0;
            break;
        case 5:
            if (u[g] < 0 || v[g] > U || u[g] > v[g]) return 0;
            break;
        case 12:
            if (u[g] < 0 || v[g] >= U || u[g] > v[g] + 1) return 0;
            break;
        case 14:
            if (!comb_ptr) return 0;
            for (int k = comb_ptr[g]; k < comb_ptr[g + 1]; ++k)
                if (comb_src[k] < 0 || comb_src[k] >= U) return 0;
            break;
        default:
            break;
        }
    }
    return 1;
}

int oracle_virgo_phase1_init(long long n_gates, const int* ty, const long long* u, const long long* v, const int* comb_ptr,
                             const int* comb_src, const u64* comb_w, int length_g, int length_u, const u64* values,
                             const u64* r0, const u64* r1, const u64* alpha, const u64* beta, u64* vma, u64* addv,
                             u64* ams)
{
    if (!virgo_layer_ok(n_gates, ty, u, v, comb_ptr, comb_src, length_g, length_u)) return -1;
    const long long U = 1LL << length_u;
    const fe zero = {0, 0};
    fe* A = (fe*)calloc((size_t)U, sizeof(fe));   /* addV_array[.].b */
    fe* M = (fe*)calloc((size_t)U, sizeof(fe));   /* add_mult_sum[.].b */
    if (!A || !M) { free(A); free(M); return -1; }
    const fe al = fe_of(alpha), be = fe_of(beta);
    for (long long g = 0; g < n_gates; ++g) {
        const int t = ty[g];
        if (t == 2) continue;
        const long long at = t == 4 ? u[g] : g;
        const fe tmp = feadd(eq_at(r0, length_g, at, al), eq_at(r1, length_g, at, be));
        const long long uu = u[g];
        switch (t) {
        case 0: { const fe tv = femul(fe_of(values + 2 * v[g]), tmp); A[uu] = feadd(A[uu], tv); M[uu] = feadd(M[uu], tmp); break; }
        case 1: { M[uu] = feadd(M[uu], femul(fe_of(values + 2 * v[g]), tmp)); break; }
        case 4: { M[uu] = feadd(M[uu], tmp); break; }
        case 5: for (long long j = uu; j < v[g]; ++j) M[j] = feadd(M[j], tmp); break;
        case 12: { fe x = tmp; for (long long j = uu; j <= v[g]; ++j) { M[j] = feadd(M[j], x); x = feadd(x, x); } break; }
        case 14:
            for (int k = comb_ptr[g]; k < comb_ptr[g + 1]; ++k)
                M[comb_src[k]] = feadd(M[comb_src[k]], femul(fe_of(comb_w + 2 * k), tmp));
            break;
        case 6: { M[uu] = fesub(M[uu], tmp); A[uu] = feadd(A[uu], tmp); break; }
        case 7: { const fe tv = femul(fe_of(values + 2 * v[g]), tmp); A[uu] = fesub(A[uu], tv); M[uu] = feadd(M[uu], tmp); break; }
        case 8: { const fe tv = femul(tmp, fe_of(values + 2 * v[g])); A[uu] = feadd(A[uu], tv); M[uu] = fesub(fesub(feadd(M[uu], tmp), tv), tv); break; }
        case 13: { const fe tv = femul(tmp, fe_of(values + 2 * v[g])); M[uu] = feadd(fesub(M[uu], tv), tmp); break; }
        case 9: { const fe tv = femul(tmp, fe_of(values + 2 * v[g])); A[uu] = feadd(A[uu], tv); M[uu] = fesub(M[uu], tv); break; }
        case 10: { M[uu] = feadd(M[uu], tmp); break; }
        default: break;
        }
    }
    for (long long i = 0; i < U; ++i) {
        put_lp(vma, i, zero, fe_of(values + 2 * i));
        put_lp(addv, i, zero, A[i]);
        put_lp(ams, i, zero, M[i]);
    }
    free(A);
    free(M);
    return 0;
}

int oracle_virgo_phase2_init(long long n_gates, const int* ty, const long long* u, const long long* v, const int* comb_ptr,
                             const int* comb_src, const u64* comb_w, int length_g, int length_u, const u64* values,
                             const u64* r0, const u64* r1, const u64* alpha, const u64* beta, const u64* vma0,
                             const u64* prev_r, const u64* r_u, u64* vma, u64* addv, u64* ams)
{
    if (!virgo_layer_ok(n_gates, ty, u, v, comb_ptr, comb_src, length_g, length_u)) return -1;
    const long long U = 1LL << length_u;
    const fe zero = {0, 0}, one = {0, 1};
    fe* A = (fe*)calloc((size_t)U, sizeof(fe));
    fe* M = (fe*)calloc((size_t)U, sizeof(fe));
    if (!A || !M) { free(A); free(M); return -1; }
    const fe al = fe_of(alpha), be = fe_of(beta);
    const fe v_u = feadd(femul(fe_of(vma0), fe_of(prev_r)), fe_of(vma0 + 2));
    for (long long g = 0; g < n_gates; ++g) {
        const int t = ty[g];
        if (t == 2 || t == 4) continue;
        const fe tg = feadd(eq_at(r0, length_g, g, al), eq_at(r1, length_g, g, be));
        const long long vv = v[g];
        if (t == 5 || t == 12 || t == 14) {
            fe x = femul(tg, v_u);
            if (t == 5) {
                for (long long j = u[g]; j < vv; ++j) A[0] = feadd(A[0], femul(x, eq_at(r_u, length_u, j, one)));
            } else if (t == 12) {
                for (long long j = u[g]; j <= vv; ++j) { A[0] = feadd(A[0], femul(x, eq_at(r_u, length_u, j, one))); x = feadd(x, x); }
            } else {
                for (int k = comb_ptr[g]; k < comb_ptr[g + 1]; ++k)
                    A[0] = feadd(A[0], femul(femul(x, eq_at(r_u, length_u, comb_src[k], one)), fe_of(comb_w + 2 * k)));
            }
            continue;
        }
        const fe tgu = femul(tg, eq_at(r_u, length_u, u[g], one));
        const fe tv = femul(tgu, v_u);
        switch (t) {
        case 1: M[vv] = feadd(M[vv], tv); break;
        case 0: M[vv] = feadd(M[vv], tgu); A[vv] = feadd(A[vv], tv); break;
        case 6: A[vv] = feadd(A[vv], fesub(tgu, tv)); break;
        case 7: M[vv] = fesub(M[vv], tgu); A[vv] = feadd(A[vv], tv); break;
        case 8: M[vv] = feadd(M[vv], fesub(fesub(tgu, tv), tv)); A[vv] = feadd(A[vv], tv); break;
        case 13: M[vv] = fesub(M[vv], tv); A[vv] = feadd(A[vv], tv); break;
        case 9: M[vv] = feadd(M[vv], fesub(tgu, tv)); break;
        case 10: A[vv] = feadd(A[vv], tv); break;
        default: break;
        }
    }
    for (long long i = 0; i < U; ++i) {
        put_lp(vma, i, zero, fe_of(values + 2 * i));
        put_lp(addv, i, zero, A[i]);
        put_lp(ams, i, zero, M[i]);
    }
    free(A);
    free(M);
    return 0;
}
