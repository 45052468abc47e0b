// The ./fft_gkr program's work on the device: the GKR proof of the inverse-FFT
// and evaluation circuit that Orion's polynomial-commitment verifier runs as a
// subprocess (TruePix-main/Orion/Orion_nonzk/src/VPD/fft_circuit_GKR.cpp,
// called through system("./fft_gkr <lg> log_fftgkr.txt") at
// src/VPD/vpd_verifier.cpp:80-89).
//
// The circuit (build_circuit, :22-112), for L = lg and n = 2^L:
//   layer 0       [1]
//   layers 1..L   tensor expansion of L random points r: layer L at index i is
//                 prod_k (bit k of i ? 1 - r[L-1-k] : r[L-1-k])
//   layers L+1..2L  an inverse FFT of size n, one butterfly layer each: for
//                 the layer of stride 2^d (d = L-1 down to 0), k < n / 2^(d+1),
//                 j < 2^d, x = (w^-1)^(2^d k) with w the order-n root of unity:
//                 cur[k 2^d + j]          = pre[k 2^(d+1) + j] + x pre[k 2^(d+1) + 2^d + j]
//                 cur[(k + n/2^(d+1)) 2^d + j] = the same with -
//   layer 2L+1    the inverse FFT's output times n^-1
//   layer 2L+2    64 n values: value j of polynomial i is layer(2L+1)[j] e_i^j
//                 for 64 random evaluation points e_i
//   layer 2L+3    the 64 sums over j
// and the sumcheck rounds engage_gkr (:770-825) runs over it: the addition
// layer (L + 6 rounds), the multiplication layer (L rounds), the scaling layer
// (no rounds) and two phases of L rounds per inverse-FFT layer; extension_gkr
// only counts proof bytes. Each round polynomial is checked (p(0) + p(1) equal
// to the running claim) and each layer ends with the reference's closed-form
// wiring check.
//
// The reference draws the verifier's randomness from glibc rand() in its
// unseeded state (prime_field::random, src/linear_gkr/prime_field.cpp:35-40)
// and nothing it draws depends on computed values, so here every draw is made
// up front on the host in the reference's order (same values), the whole
// prover runs on one stream without a host round trip (tables, round
// polynomials and the end-of-phase table entries stay on the device), and the
// host checks everything after one copy back.
//
// Device work: the circuit's layers (one kernel each), the table inits of each
// phase (one kernel each; the gate wiring of every layer is fixed, so an init
// writes each table entry directly instead of scattering gates), and the
// rounds through virgo::update, which is the reference's
// sumcheck_phase1_update / sumcheck_phase2_update (:172-236).
#include <chrono>
#include <cstdio>
#include <cstring>
#include <vector>

#include "fp2.cuh"
#include "glibc_rand.h"
#include "ntt.h"
#include "runtime.h"
#include "virgo.h"

namespace tp {
namespace fftgkr {

namespace {

constexpr int kThreads = 256;
constexpr int kPolys = 64;        // evaluation points of layer 2L+2 (fft_circuit_GKR.cpp:83-86)
constexpr int kPolyBits = 6;
constexpr int kMaxLg = 20;
constexpr long long kQuadBytes = 48;   // sizeof(quadratic_poly): three 16-byte elements

// ---- device helpers ---------------------------------------------------------

__device__ __forceinline__ fp2 ld(const ulonglong2* t, long long i)
{
    const ulonglong2 v = t[i];
    return mk(v.y, v.x);
}
__device__ __forceinline__ void st(ulonglong2* t, long long i, fp2 x)
{
    x = l2canon(x);
    t[i] = make_ulonglong2(x.im, x.re);
}
// linear_poly {0, b} at table entry i
__device__ __forceinline__ void st_lin(ulonglong2* t, long long i, fp2 b)
{
    t[2 * i] = make_ulonglong2(0, 0);
    st(t, 2 * i + 1, b);
}
__device__ __forceinline__ fp2 pw(fp2 x, long long e)
{
    fp2 r = mk(1, 0);
    while (e) {
        if (e & 1) r = l2mul(r, x);
        x = l2mul(x, x);
        e >>= 1;
    }
    return r;
}
// eq(z, i) = prod_k (bit k of i ? z_k : 1 - z_k), z: k < bits (canonical)
__device__ __forceinline__ fp2 eq(const fp2* z, int bits, long long i)
{
    fp2 r = mk(1, 0);
    for (int k = 0; k < bits; ++k) r = l2mul(r, ((i >> k) & 1) ? z[k] : l2sub(mk(1, 0), z[k]));
    return r;
}

// layer L of the tensor expansion: sel[2k] = r[L-1-k] (bit 0), sel[2k+1] = 1 - r[L-1-k]
__global__ void tensor_kernel(ulonglong2* out, int bits, const fp2* __restrict__ sel)
{
    const long long i = (long long)blockIdx.x * kThreads + threadIdx.x;
    if (i >= (1LL << bits)) return;
    fp2 v = mk(1, 0);
    for (int k = 0; k < bits; ++k) v = l2mul(v, sel[2 * k + ((i >> k) & 1)]);
    st(out, i, v);
}

// one inverse-FFT butterfly layer of stride 2^d (t < n / 2)
__global__ void butterfly_kernel(const ulonglong2* __restrict__ pre, ulonglong2* __restrict__ cur, int L, int d, fp2 w)
{
    const long long t = (long long)blockIdx.x * kThreads + threadIdx.x;
    if (t >= (1LL << (L - 1))) return;
    const long long j = t & ((1LL << d) - 1), k = t >> d, half = 1LL << (L - d - 1);
    const fp2 x = pw(w, k);
    const fp2 l = ld(pre, (k << (d + 1)) | j), r = l2mul(x, ld(pre, (k << (d + 1)) | (1LL << d) | j));
    st(cur, (k << d) | j, l2add(l, r));
    st(cur, ((k + half) << d) | j, l2sub(l, r));
}

// layer 2L+1 (scaled) and layer 2L+2 (evaluations): t < 64 n
__global__ void eval_kernel(const ulonglong2* __restrict__ ifft_out, int L, fp2 inv_n, const fp2* __restrict__ ep,
                            ulonglong2* __restrict__ scaled, ulonglong2* __restrict__ evals)
{
    const long long t = (long long)blockIdx.x * kThreads + threadIdx.x;
    if (t >= ((long long)kPolys << L)) return;
    const long long j = t & ((1LL << L) - 1), i = t >> L;
    const fp2 s = l2mul(ld(ifft_out, j), inv_n);
    if (i == 0) st(scaled, j, s);
    st(evals, t, l2mul(s, pw(ep[i], j)));
}

// layer 2L+3: one CTA per polynomial
__global__ void __launch_bounds__(kThreads) output_kernel(const ulonglong2* __restrict__ evals, int L,
                                                          ulonglong2* __restrict__ out)
{
    __shared__ fp2 red[kThreads];
    fp2 s = f2zero();
    for (long long j = threadIdx.x; j < (1LL << L); j += kThreads) s = l2add(s, ld(evals, ((long long)blockIdx.x << L) + j));
    red[threadIdx.x] = s;
    __syncthreads();
    for (int o = kThreads / 2; o; o >>= 1) {
        if (threadIdx.x < o) red[threadIdx.x] = l2add(red[threadIdx.x], red[threadIdx.x + o]);
        __syncthreads();
    }
    if (threadIdx.x == 0) st(out, blockIdx.x, red[0]);
}

// addition layer (addition_layer, :238-279): V_mult_add = the evaluations,
// add_mult_sum[i] = beta_g(i >> L) (bg: 64 host values), addV_array = 0
__global__ void init_add_kernel(const ulonglong2* __restrict__ evals, int L, const fp2* __restrict__ bg,
                                ulonglong2* vma, ulonglong2* addv, ulonglong2* ams)
{
    const long long i = (long long)blockIdx.x * kThreads + threadIdx.x;
    if (i >= ((long long)kPolys << L)) return;
    st_lin(vma, i, ld(evals, i));
    st_lin(addv, i, f2zero());
    st_lin(ams, i, bg[i >> L]);
}

// multiplication layer (mult_layer, :363-428): for i < n,
// add_mult_sum[i] = sum_j (eq(r0lo, i) c0[j] + eq(r1lo, i) c1[j]) e_j^i with
// c0[j] = alpha eq(r0hi, j), c1[j] = beta eq(r1hi, j) (host values)
__global__ void init_mult_kernel(const ulonglong2* __restrict__ scaled, int L, const fp2* __restrict__ r0lo,
                                 const fp2* __restrict__ r1lo, const fp2* __restrict__ c0, const fp2* __restrict__ c1,
                                 const fp2* __restrict__ ep, ulonglong2* vma, ulonglong2* addv, ulonglong2* ams)
{
    const long long i = (long long)blockIdx.x * kThreads + threadIdx.x;
    if (i >= (1LL << L)) return;
    const fp2 e0 = eq(r0lo, L, i), e1 = eq(r1lo, L, i);
    fp2 s = f2zero();
    for (int j = 0; j < kPolys; ++j)
        s = l2add(s, l2mul(l2add(l2mul(e0, c0[j]), l2mul(e1, c1[j])), pw(ep[j], i)));
    st_lin(vma, i, ld(scaled, i));
    st_lin(addv, i, f2zero());
    st_lin(ams, i, s);
}

// bg[g] = a eq(z0, g) + b eq(z1, g), g < 2^bits (the beta_g tables of a layer)
__global__ void beta_kernel(const fp2* __restrict__ z0, const fp2* __restrict__ z1, int bits, fp2 a, fp2 b,
                            ulonglong2* __restrict__ out)
{
    const long long g = (long long)blockIdx.x * kThreads + threadIdx.x;
    if (g >= (1LL << bits)) return;
    st(out, g, l2add(l2mul(a, eq(z0, bits, g)), l2mul(b, eq(z1, bits, g))));
}

// inverse-FFT layer of stride 2^d, phase 1 (ifft_gkr, :537-601): for u with bit d
// clear, g1 = k 2^d + j, g2 = g1 + n/2 (u = k 2^(d+1) + j, v = u + 2^d, x = w^k):
//   add_mult_sum[u] = bg[g1] + bg[g2],  addV_array[u] = (bg[g1] - bg[g2]) x pre[v]
// entries with bit d set stay zero; V_mult_add = pre
__global__ void init_ifft1_kernel(const ulonglong2* __restrict__ pre, const ulonglong2* __restrict__ bg, int L, int d,
                                  fp2 w, ulonglong2* vma, ulonglong2* addv, ulonglong2* ams)
{
    const long long u = (long long)blockIdx.x * kThreads + threadIdx.x;
    if (u >= (1LL << L)) return;
    st_lin(vma, u, ld(pre, u));
    if ((u >> d) & 1) {
        st_lin(addv, u, f2zero());
        st_lin(ams, u, f2zero());
        return;
    }
    const long long j = u & ((1LL << d) - 1), k = u >> (d + 1);
    const long long g1 = (k << d) | j, g2 = g1 + (1LL << (L - 1));
    const fp2 b1 = ld(bg, g1), b2 = ld(bg, g2);
    st_lin(ams, u, l2add(b1, b2));
    st_lin(addv, u, l2mul(l2mul(l2sub(b1, b2), pw(w, k)), ld(pre, u | (1LL << d))));
}

// phase 2 (:619-673): for v with bit d set, u = v - 2^d, tu = eq(r_u, u),
// v_u = last.a r_last + last.b (the one-entry V_mult_add phase 1 left):
//   add_mult_sum[v] = (bg[g1] - bg[g2]) tu x,  addV_array[v] = (bg[g1] + bg[g2]) tu v_u
// entries with bit d clear stay zero; V_mult_add = pre
__global__ void init_ifft2_kernel(const ulonglong2* __restrict__ pre, const ulonglong2* __restrict__ bg,
                                  const ulonglong2* __restrict__ equ, int L, int d, fp2 w,
                                  const ulonglong2* __restrict__ last, fp2 r_last, ulonglong2* vma, ulonglong2* addv,
                                  ulonglong2* ams)
{
    const long long v = (long long)blockIdx.x * kThreads + threadIdx.x;
    if (v >= (1LL << L)) return;
    st_lin(vma, v, ld(pre, v));
    if (!((v >> d) & 1)) {
        st_lin(addv, v, f2zero());
        st_lin(ams, v, f2zero());
        return;
    }
    const long long u = v ^ (1LL << d);
    const long long j = u & ((1LL << d) - 1), k = u >> (d + 1);
    const long long g1 = (k << d) | j, g2 = g1 + (1LL << (L - 1));
    const fp2 b1 = ld(bg, g1), b2 = ld(bg, g2), tu = ld(equ, u);
    const fp2 v_u = l2add(l2mul(ld(last, 0), r_last), ld(last, 1));
    st_lin(ams, v, l2mul(l2mul(l2sub(b1, b2), tu), pw(w, k)));
    st_lin(addv, v, l2mul(l2mul(l2add(b1, b2), tu), v_u));
}

unsigned grid(long long n) { return (unsigned)((n + kThreads - 1) / kThreads); }

// ---- host arithmetic ---------------------------------------------------------

fp2 one() { return mk(1, 0); }
fp2 omr(fp2 x) { return f2sub(one(), x); }
fp2 heq(const fp2* z, int bits, long long i)
{
    fp2 r = one();
    for (int k = 0; k < bits; ++k) r = f2mul(r, ((i >> k) & 1) ? z[k] : omr(z[k]));
    return r;
}
struct Quad {
    fp2 a, b, c;
    fp2 at(fp2 x) const { return f2add(f2mul(f2add(f2mul(a, x), b), x), c); }   // quadratic_poly::eval
};

// the verifier's randomness, in the reference's draw order
struct Draws {
    std::vector<fp2> r, ep, r0, r1, ru_a, rv_a, ru_m, rv_m;
    std::vector<std::vector<fp2>> ru, rv;
    std::vector<fp2> alpha, beta;
};

Draws draw_all(int L)
{
    GlibcRand g(1);
    auto rnd = [&]() {                  // prime_field::random: real, then imaginary part
        const u64 re = (u64)g.next() % P61;
        const u64 im = (u64)g.next() % P61;
        return mk(re, im);
    };
    auto many = [&](int k) {
        std::vector<fp2> v(k);
        for (auto& x : v) x = rnd();
        return v;
    };
    Draws D;
    D.r = many(L);                      // main (:835-837)
    D.ep = many(kPolys);                // build_circuit (:86-88)
    D.r0 = many(L + 10);                // engage_gkr (:790-791)
    D.r1 = many(L + 10);
    D.ru_a = many(L + kPolyBits);       // addition_layer (:283-284)
    D.rv_a = many(L + kPolyBits);
    D.ru_m = many(L);                   // mult_layer (:432-433)
    D.rv_m = many(L);
    for (int d = 0; d < L; ++d) {       // ifft_gkr, per layer (:603-604, 757-758)
        D.ru.push_back(many(L));
        D.rv.push_back(many(L));
        D.alpha.push_back(rnd());
        D.beta.push_back(rnd());
    }
    return D;
}

long long count_proof_bytes(int L)
{
    long long rounds = (L + kPolyBits) + L + 2LL * L * L;   // addition, multiplication, inverse-FFT phases
    for (int i = 1; i <= L; ++i) rounds += i;               // extension_gkr (:762-768)
    return rounds * kQuadBytes;
}

double wall() { return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count(); }

struct DevBuf {
    void* p = nullptr;
    ~DevBuf() { if (p) cudaFree(p); }
    template <class T> T* as() const { return static_cast<T*>(p); }
};

// a pair of timing events, destroyed with the scope
struct EventPair {
    cudaEvent_t a = nullptr, b = nullptr;
    ~EventPair()
    {
        if (a) cudaEventDestroy(a);
        if (b) cudaEventDestroy(b);
    }
    bool create()
    {
        return !cuda_failed(cudaEventCreate(&a), "fft_gkr event") && !cuda_failed(cudaEventCreate(&b), "fft_gkr event");
    }
};

bool dalloc(DevBuf& b, size_t bytes, const char* what)
{
    if (cuda_failed(cudaMalloc(&b.p, bytes), what)) return false;
    return true;
}

}  // namespace

int run(int L, double* v_time, long long* proof_size, double* p_time, int* accepted, const char* trace_path)
{
    if (L < 0 || L > kMaxLg) {
        set_error(TP_ERR_ARG, "fft_gkr: lg %d outside [0, %d]", L, kMaxLg);
        return -1;
    }
    Ctx* c = ctx();
    if (!c) return -1;
    cudaStream_t s = c->stream;
    const long long n = 1LL << L, N = (long long)kPolys << L;
    const Draws D = draw_all(L);
    FILE* tr = nullptr;
    if (trace_path && !(tr = fopen(trace_path, "w"))) {
        set_error(TP_ERR_ARG, "fft_gkr: cannot write %s", trace_path);
        return -1;
    }
    struct Closer { FILE* f; ~Closer() { if (f) fclose(f); } } closer{tr};

    // rounds and their polynomial slots
    const int rounds_add = L + kPolyBits, rounds_mult = L;
    const long long n_rounds = rounds_add + rounds_mult + 2LL * L * L;
    // device memory: layers L..2L (n each), scaled (n), evaluations (64 n), outputs,
    // two sets of three tables, the beta tables, small inputs, the record
    DevBuf layers, scaled, evals, outs, tabA, tabB, bgt, equ, small, rec, sel;
    const size_t fe = sizeof(ulonglong2);
    if (!dalloc(layers, fe * n * (L + 1), "fft_gkr layers") || !dalloc(scaled, fe * n, "fft_gkr scaled") ||
        !dalloc(evals, fe * N, "fft_gkr evaluations") || !dalloc(outs, fe * kPolys, "fft_gkr outputs") ||
        !dalloc(tabA, 3 * 2 * fe * N, "fft_gkr tables") || !dalloc(tabB, 3 * fe * N, "fft_gkr tables") ||
        !dalloc(bgt, fe * n, "fft_gkr beta") || !dalloc(equ, fe * n, "fft_gkr eq"))
        return -1;
    // the record: round polynomials (3 elements each), then per phase the last
    // V_mult_add entry (2 elements), then the last phase's three entries (6)
    const long long n_phases = 2 + 2LL * L;
    const long long rec_elems = 3 * n_rounds + 2 * n_phases + 6;
    if (!dalloc(rec, fe * rec_elems, "fft_gkr record") || cuda_failed(cudaMemsetAsync(rec.p, 0, fe * rec_elems, s), "fft_gkr record"))
        return -1;
    ulonglong2* R = rec.as<ulonglong2>();
    ulonglong2* polys = R;
    ulonglong2* lasts = R + 3 * n_rounds;
    ulonglong2* finals = lasts + 2 * n_phases;

    // small host-known inputs in one upload: tensor selectors, evaluation points,
    // the multiplication layer's eq halves and the per-layer beta points
    std::vector<fp2> h_sel(2 * (size_t)(L > 0 ? L : 1));
    for (int k = 0; k < L; ++k) {
        h_sel[2 * k] = D.r[L - 1 - k];
        h_sel[2 * k + 1] = omr(D.r[L - 1 - k]);
    }
    std::vector<fp2> h_small;
    auto put = [&](const std::vector<fp2>& v) { size_t o = h_small.size(); h_small.insert(h_small.end(), v.begin(), v.end()); return o; };
    const size_t o_sel = put(h_sel), o_ep = put(D.ep);
    // addition layer beta_g over the 64 polynomials (alpha = 1, beta = 0 at that point)
    const fp2 alpha0 = one(), beta0 = f2zero();
    std::vector<fp2> bg64(kPolys);
    for (int i = 0; i < kPolys; ++i)
        bg64[i] = f2add(f2mul(alpha0, heq(D.r0.data(), kPolyBits, i)), f2mul(beta0, heq(D.r1.data(), kPolyBits, i)));
    const size_t o_bg64 = put(bg64);
    // multiplication layer: r0 = ru_a, r1 = rv_a (their first L + 6)
    std::vector<fp2> c0(kPolys), c1(kPolys);
    for (int j = 0; j < kPolys; ++j) {
        c0[j] = f2mul(alpha0, heq(D.ru_a.data() + L, kPolyBits, j));
        c1[j] = f2mul(beta0, heq(D.rv_a.data() + L, kPolyBits, j));
    }
    const size_t o_c0 = put(c0), o_c1 = put(c1);
    const size_t o_r0lo = put(std::vector<fp2>(D.ru_a.begin(), D.ru_a.begin() + L));
    const size_t o_r1lo = put(std::vector<fp2>(D.rv_a.begin(), D.rv_a.begin() + L));
    // inverse-FFT layers: layer d's r0, r1 are the previous layer's r_u, r_v
    // (for d = 0 the multiplication layer's), its r_u for the eq table
    std::vector<size_t> o_z0(L), o_z1(L), o_u(L);
    for (int d = 0; d < L; ++d) {
        o_z0[d] = put(d ? D.ru[d - 1] : D.ru_m);
        o_z1[d] = put(d ? D.rv[d - 1] : D.rv_m);
        o_u[d] = put(D.ru[d]);
    }
    if (!dalloc(small, sizeof(fp2) * (h_small.size() + 1), "fft_gkr inputs") ||
        cuda_failed(cudaMemcpyAsync(small.p, h_small.data(), sizeof(fp2) * h_small.size(), cudaMemcpyHostToDevice, s),
                    "fft_gkr inputs"))
        return -1;
    const fp2* S = small.as<fp2>();

    const fp2 rou = ntt::root_of_unity(L);
    const fp2 inv_rou = f2inv(rou);
    const fp2 inv_n = mk(finv((u64)n % P61), 0);
    std::vector<fp2> rot(L > 0 ? L : 1);
    if (L > 0) rot[0] = inv_rou;
    for (int d = 1; d < L; ++d) rot[d] = f2mul(rot[d - 1], rot[d - 1]);

    ulonglong2* Lay = layers.as<ulonglong2>();
    auto layer = [&](int t) { return Lay + (size_t)t * n; };   // layer L + t
    auto ok = [&](const char* what) { return !cuda_failed(cudaGetLastError(), what); };

    // ---- the circuit
    tensor_kernel<<<grid(n), kThreads, 0, s>>>(layer(0), L, S + o_sel);
    if (!ok("fft_gkr tensor")) return -1;
    for (int d = L - 1, t = 1; d >= 0; --d, ++t) {
        butterfly_kernel<<<grid(n / 2), kThreads, 0, s>>>(layer(t - 1), layer(t), L, d, rot[d]);
        if (!ok("fft_gkr butterfly")) return -1;
    }
    eval_kernel<<<grid(N), kThreads, 0, s>>>(layer(L), L, inv_n, S + o_ep, scaled.as<ulonglong2>(), evals.as<ulonglong2>());
    output_kernel<<<kPolys, kThreads, 0, s>>>(evals.as<ulonglong2>(), L, outs.as<ulonglong2>());
    if (!ok("fft_gkr evaluations")) return -1;
    if (cuda_failed(cudaStreamSynchronize(s), "fft_gkr circuit")) return -1;
    if (tr && L <= 6) {
        // the layers as the reference numbers them (0 .. 2L+3); the tensor
        // layers below L are made here for the dump only
        auto dump = [&](int id, const void* d, long long len) {
            std::vector<ulonglong2> h(len);
            if (cuda_failed(cudaMemcpy(h.data(), d, fe * len, cudaMemcpyDeviceToHost), "fft_gkr dump")) return false;
            fprintf(tr, "layer %d %lld", id, len);
            for (const ulonglong2& e : h) fprintf(tr, " %llu %llu", (unsigned long long)e.y, (unsigned long long)e.x);
            fprintf(tr, "\n");
            return true;
        };
        for (int k = 0; k < L; ++k) {
            std::vector<fp2> sk(2 * (size_t)(k > 0 ? k : 1));
            for (int m = 0; m < k; ++m) {
                sk[2 * m] = D.r[k - 1 - m];
                sk[2 * m + 1] = omr(D.r[k - 1 - m]);
            }
            DevBuf ds;
            if (!dalloc(ds, sizeof(fp2) * sk.size() + fe * (1LL << k), "fft_gkr dump")) return -1;
            ulonglong2* out = reinterpret_cast<ulonglong2*>(ds.as<fp2>() + sk.size());
            if (cuda_failed(cudaMemcpy(ds.p, sk.data(), sizeof(fp2) * sk.size(), cudaMemcpyHostToDevice), "fft_gkr dump"))
                return -1;
            tensor_kernel<<<grid(1LL << k), kThreads, 0, s>>>(out, k, ds.as<fp2>());
            if (!ok("fft_gkr dump") || cuda_failed(cudaStreamSynchronize(s), "fft_gkr dump") || !dump(k, out, 1LL << k))
                return -1;
        }
        for (int t = 0; t <= L; ++t)
            if (!dump(L + t, layer(t), n)) return -1;
        if (!dump(2 * L + 1, scaled.p, n) || !dump(2 * L + 2, evals.p, N) || !dump(2 * L + 3, outs.p, kPolys)) return -1;
    }

    // ---- the prover: every phase's init and rounds, no host round trip
    EventPair ev;
    if (!ev.create()) return -1;
    const double t0 = wall();
    cudaEventRecord(ev.a, s);
    ulonglong2 *A = tabA.as<ulonglong2>(), *B = tabB.as<ulonglong2>();
    long long round = 0, phase = 0;
    // runs the rounds of one phase over tables of `len` entries starting in set A;
    // records the last V_mult_add entry; returns the set holding the final tables
    auto phase_rounds = [&](long long len, int k, const std::vector<fp2>& rr) -> ulonglong2* {
        ulonglong2 *src = A, *dst = B;
        long long m = len;
        for (int i = 0; i < k; ++i) {
            const fp2 prev = i ? rr[i - 1] : f2zero();
            const long long h = m / 2;
            if (!virgo::update(src, src + 2 * m, src + 4 * m, m, prev, i, dst, dst + 2 * h, dst + 4 * h,
                               polys + 3 * round, s))
                return nullptr;
            ++round;
            std::swap(src, dst);
            m = h;
            // the next round reads the tables just written: set sizes follow m
        }
        if (cuda_failed(cudaMemcpyAsync(lasts + 2 * phase, src, 2 * fe, cudaMemcpyDeviceToDevice, s), "fft_gkr record"))
            return nullptr;
        ++phase;
        return src;
    };
    // tables of a set: V_mult_add at 0, addV_array at 2 len, add_mult_sum at 4 len
    // (two elements per entry); phase_rounds passes the running length along
    {
        init_add_kernel<<<grid(N), kThreads, 0, s>>>(evals.as<ulonglong2>(), L, S + o_bg64, A, A + 2 * N, A + 4 * N);
        if (!ok("fft_gkr addition init") || !phase_rounds(N, rounds_add, D.ru_a)) return -1;
    }
    {
        init_mult_kernel<<<grid(n), kThreads, 0, s>>>(scaled.as<ulonglong2>(), L, S + o_r0lo, S + o_r1lo, S + o_c0,
                                                       S + o_c1, S + o_ep, A, A + 2 * n, A + 4 * n);
        if (!ok("fft_gkr multiplication init")) return -1;
        ulonglong2* fin = phase_rounds(n, rounds_mult, D.ru_m);
        if (!fin) return -1;
        if (L == 0 && cuda_failed(cudaMemcpyAsync(finals, fin, 6 * fe, cudaMemcpyDeviceToDevice, s), "fft_gkr record"))
            return -1;
    }
    for (int d = 0; d < L; ++d) {
        const int dep = d;   // ifft_gkr's dep: stride 2^dep, pre = layer 2L - dep - 1
        ulonglong2* pre = layer(L - dep - 1);
        const fp2 a = d ? D.alpha[d - 1] : alpha0, b = d ? D.beta[d - 1] : beta0;
        beta_kernel<<<grid(n), kThreads, 0, s>>>(S + o_z0[d], S + o_z1[d], L, a, b, bgt.as<ulonglong2>());
        init_ifft1_kernel<<<grid(n), kThreads, 0, s>>>(pre, bgt.as<ulonglong2>(), L, dep, rot[dep], A, A + 2 * n,
                                                       A + 4 * n);
        if (!ok("fft_gkr inverse-FFT phase 1 init")) return -1;
        ulonglong2* fin1 = phase_rounds(n, L, D.ru[d]);
        if (!fin1) return -1;
        // the one-entry V_mult_add of phase 1 is read from the record
        const ulonglong2* last = lasts + 2 * (phase - 1);
        beta_kernel<<<grid(n), kThreads, 0, s>>>(S + o_u[d], S + o_u[d], L, one(), f2zero(), equ.as<ulonglong2>());
        init_ifft2_kernel<<<grid(n), kThreads, 0, s>>>(pre, bgt.as<ulonglong2>(), equ.as<ulonglong2>(), L, dep,
                                                       rot[dep], last, D.ru[d][L - 1], A, A + 2 * n, A + 4 * n);
        if (!ok("fft_gkr inverse-FFT phase 2 init")) return -1;
        ulonglong2* fin2 = phase_rounds(n, L, D.rv[d]);
        if (!fin2) return -1;
        if (d == L - 1 && cuda_failed(cudaMemcpyAsync(finals, fin2, 6 * fe, cudaMemcpyDeviceToDevice, s), "fft_gkr record"))
            return -1;
    }
    cudaEventRecord(ev.b, s);
    std::vector<ulonglong2> h_rec(rec_elems), h_out(kPolys);
    if (cuda_failed(cudaMemcpyAsync(h_rec.data(), rec.p, fe * rec_elems, cudaMemcpyDeviceToHost, s), "fft_gkr record") ||
        cuda_failed(cudaMemcpyAsync(h_out.data(), outs.p, fe * kPolys, cudaMemcpyDeviceToHost, s), "fft_gkr outputs") ||
        cuda_failed(cudaStreamSynchronize(s), "fft_gkr prover"))
        return -1;
    float dev_ms = 0;
    cudaEventElapsedTime(&dev_ms, ev.a, ev.b);

    // ---- the verifier's side (host)
    auto el = [&](long long i) { return mk(h_rec[i].y, h_rec[i].x); };
    auto poly = [&](long long k) { return Quad{el(3 * k), el(3 * k + 1), el(3 * k + 2)}; };
    auto last_eval = [&](long long ph, fp2 r) { return f2add(f2mul(el(3 * n_rounds + 2 * ph), r), el(3 * n_rounds + 2 * ph + 1)); };
    double vt = 0;
    bool good = true;
    long long k = 0;
    // one phase's round checks: p(0) + p(1) == claim, claim = p(r_i)
    auto rounds_ok = [&](fp2& claim, int cnt, const std::vector<fp2>& rr) {
        for (int i = 0; i < cnt; ++i, ++k) {
            const Quad q = poly(k);
            if (!(f2add(q.at(f2zero()), q.at(one())).re == claim.re && f2add(q.at(f2zero()), q.at(one())).im == claim.im))
                good = false;
            claim = q.at(rr[i]);
        }
    };
    auto same = [](fp2 x, fp2 y) { return x.re == y.re && x.im == y.im; };
    auto trace_claim = [&](const char* tag, fp2 x) {
        if (tr) fprintf(tr, "claim %s %llu %llu\n", tag, (unsigned long long)x.re, (unsigned long long)x.im);
    };
    // V_output (:134-151): the 64 outputs folded LSB first at r0
    std::vector<fp2> o(kPolys);
    for (int i = 0; i < kPolys; ++i) o[i] = mk(h_out[i].y, h_out[i].x);
    for (int b = 0, m = kPolys; b < kPolyBits; ++b, m /= 2)
        for (int j = 0; j < m / 2; ++j) o[j] = f2add(f2mul(o[2 * j], omr(D.r0[b])), f2mul(o[2 * j + 1], D.r0[b]));
    fp2 claim = o[0];
    trace_claim("a0", claim);
    std::vector<fp2> r0 = D.r0, r1 = D.r1;
    fp2 alpha = alpha0, beta = beta0;
    // addition layer
    rounds_ok(claim, rounds_add, D.ru_a);
    fp2 v_u = last_eval(0, rounds_add ? D.ru_a[rounds_add - 1] : f2zero());
    {
        const double t = wall();
        fp2 sum = f2zero();
        for (int i = 0; i < kPolys; ++i) sum = f2add(sum, f2mul(bg64[i], heq(D.ru_a.data() + L, kPolyBits, i)));
        vt += wall() - t;
        if (!same(claim, f2mul(sum, v_u))) good = false;
    }
    for (int i = 0; i < L + kPolyBits; ++i) { r0[i] = D.ru_a[i]; r1[i] = D.rv_a[i]; }
    claim = f2mul(alpha, v_u);
    trace_claim("add", claim);
    // multiplication layer
    rounds_ok(claim, rounds_mult, D.ru_m);
    v_u = last_eval(1, rounds_mult ? D.ru_m[rounds_mult - 1] : f2zero());
    {
        const double t = wall();
        fp2 sum = f2zero();
        for (int i = 0; i < kPolys; ++i) {
            fp2 g0 = alpha, g1 = beta;
            for (int j = 0; j < kPolyBits; ++j) {
                const bool bit = (i >> j) & 1;
                g0 = f2mul(g0, bit ? r0[L + j] : omr(r0[L + j]));
                g1 = f2mul(g1, bit ? r1[L + j] : omr(r1[L + j]));
            }
            fp2 u0 = one(), u1 = one(), x = D.ep[i];
            for (int j = 0; j < L; ++j) {
                const fp2 ru = D.ru_m[j];
                u0 = f2mul(u0, f2add(f2mul(f2mul(r0[j], ru), x), f2mul(omr(r0[j]), omr(ru))));
                u1 = f2mul(u1, f2add(f2mul(f2mul(r1[j], ru), x), f2mul(omr(r1[j]), omr(ru))));
                x = f2mul(x, x);
            }
            sum = f2add(sum, f2add(f2mul(g0, u0), f2mul(g1, u1)));
        }
        vt += wall() - t;
        if (!same(claim, f2mul(sum, v_u))) good = false;
    }
    for (int i = 0; i < L; ++i) { r0[i] = D.ru_m[i]; r1[i] = D.rv_m[i]; }
    claim = f2mul(alpha, v_u);
    trace_claim("mult", claim);
    // scaling layer (intermediate_layer, :497-502)
    claim = f2mul(claim, mk((u64)n % P61, 0));
    if (!same(f2mul(mk((u64)n % P61, 0), inv_n), one())) good = false;
    trace_claim("inter", claim);
    // inverse-FFT layers
    for (int d = 0; d < L; ++d) {
        const std::vector<fp2>&ru = D.ru[d], &rv = D.rv[d];
        rounds_ok(claim, L, ru);
        v_u = last_eval(2 + 2 * d, ru[L - 1]);
        rounds_ok(claim, L, rv);
        const fp2 v_v = last_eval(3 + 2 * d, rv[L - 1]);
        const double t = wall();
        // the closed form of :709-753
        const int lj = d, lk = L - d - 1;
        const fp2 base = f2mul(omr(ru[lj]), rv[lj]);
        fp2 A0u = f2mul(f2mul(omr(r0[L - 1]), base), alpha), A1u = f2mul(f2mul(omr(r1[L - 1]), base), beta);
        fp2 A0v = A0u, A1v = A1u;
        fp2 B0u = f2mul(f2mul(r0[L - 1], base), alpha), B1u = f2mul(f2mul(r1[L - 1], base), beta);
        fp2 B0v = B0u, B1v = B1u;
        fp2 x = rot[d];
        for (int i = 0; i < lk; ++i) {
            const fp2 uu = ru[lj + 1 + i], vv = rv[lj + 1 + i];
            const fp2 e0 = f2mul(f2mul(r0[lj + i], uu), vv), f0 = f2mul(f2mul(omr(r0[lj + i]), omr(uu)), omr(vv));
            const fp2 e1 = f2mul(f2mul(r1[lj + i], uu), vv), f1 = f2mul(f2mul(omr(r1[lj + i]), omr(uu)), omr(vv));
            A0u = f2mul(A0u, f2add(e0, f0));
            A1u = f2mul(A1u, f2add(e1, f1));
            A0v = f2mul(A0v, f2add(f2mul(e0, x), f0));
            A1v = f2mul(A1v, f2add(f2mul(e1, x), f1));
            B0u = f2mul(B0u, f2add(e0, f0));
            B1u = f2mul(B1u, f2add(e1, f1));
            B0v = f2mul(B0v, f2add(f0, f2mul(e0, x)));
            B1v = f2mul(B1v, f2add(f1, f2mul(e1, x)));
            x = f2mul(x, x);
        }
        for (int i = 0; i < lj; ++i) {
            const fp2 t0 = f2add(f2mul(f2mul(r0[i], ru[i]), rv[i]), f2mul(f2mul(omr(r0[i]), omr(ru[i])), omr(rv[i])));
            const fp2 t1 = f2add(f2mul(f2mul(r1[i], ru[i]), rv[i]), f2mul(f2mul(omr(r1[i]), omr(ru[i])), omr(rv[i])));
            A0u = f2mul(A0u, t0); A0v = f2mul(A0v, t0); B0u = f2mul(B0u, t0); B0v = f2mul(B0v, t0);
            A1u = f2mul(A1u, t1); A1v = f2mul(A1v, t1); B1u = f2mul(B1u, t1); B1v = f2mul(B1v, t1);
        }
        const fp2 want = f2add(f2mul(f2add(f2add(A0u, A1u), f2add(B0u, B1u)), v_u),
                               f2mul(f2sub(f2add(A0v, A1v), f2add(B0v, B1v)), v_v));
        vt += wall() - t;
        if (!same(claim, want)) good = false;
        for (int i = 0; i < L; ++i) { r0[i] = ru[i]; r1[i] = rv[i]; }
        alpha = D.alpha[d];
        beta = D.beta[d];
        claim = f2add(f2mul(alpha, v_u), f2mul(beta, v_v));
    }
    trace_claim("ifft", claim);
    const double t1 = wall();

    if (tr) {
        fprintf(tr, "final");
        for (int i = 0; i < 6; ++i) {
            const ulonglong2 e = h_rec[3 * n_rounds + 2 * n_phases + i];
            fprintf(tr, " %llu %llu", (unsigned long long)e.y, (unsigned long long)e.x);
        }
        fprintf(tr, "\nresult %d\nproof_size %lld\ndevice_ms %.4f\n", good ? 1 : 0, count_proof_bytes(L), dev_ms);
    }
    if (v_time) *v_time = vt;
    if (p_time) *p_time = t1 - t0;
    if (proof_size) *proof_size = count_proof_bytes(L);
    if (accepted) *accepted = good ? 1 : 0;
    return 0;
}

}  // namespace fftgkr
}  // namespace tp

extern "C" int tp_fft_gkr(int lg, double* v_time, long long* proof_size, double* p_time, int* accepted,
                          const char* trace_path)
{
    tp::clear_error();
    return tp::fftgkr::run(lg, v_time, proof_size, p_time, accepted, trace_path);
}
