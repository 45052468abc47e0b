// C ABI of libnative_fp2_gpu.so: the 14 entry points of the reference native_fp2
// library (TruePix-main/native_fp2/native_fp2.cu:824-1022, same prototypes as
// native_fp2.cpp:11-160) plus device-buffer and error-reporting extensions.
//
// Host-buffer entry points follow the reference contract: caller-owned host
// arrays (SoA real[]/imag[]), consumed and written before the call returns.
// Unlike the reference there is no host fallback: on failure the void entry
// points leave their outputs untouched and record an error that
// tp_last_error_code()/tp_last_error() report; session entry points return -1
// or NULL as in the reference.
#include <stdint.h>
#include <string.h>

#include <vector>

#include "gkr.h"
#include "runtime.h"
#include "../../include/native_fp2.h"

using tp::fp2;
using tp::mk;
using tp::u64;

namespace {

// A few pool buffers freed (stream-ordered) when the scope ends.
struct Scratch {
    cudaStream_t s;
    std::vector<void*> ptrs;
    bool ok = true;
    explicit Scratch(cudaStream_t st) : s(st) {}
    template <typename T>
    T* get(size_t n)
    {
        void* p = tp::dev_alloc(sizeof(T) * (n ? n : 1), s);
        if (!p) ok = false;
        ptrs.push_back(p);
        return reinterpret_cast<T*>(p);
    }
    ~Scratch()
    {
        for (void* p : ptrs) tp::dev_free(p, s);
    }
};

bool h2d(void* d, const void* h, size_t bytes, cudaStream_t s) { return tp::host_to_device(d, h, bytes, s); }
bool d2h(void* h, const void* d, size_t bytes, cudaStream_t s) { return tp::device_to_host(h, d, bytes, s); }
bool sync(cudaStream_t s) { return !tp::cuda_failed(cudaStreamSynchronize(s), "synchronize"); }

// NULL is the CUDA default stream, as everywhere in CUDA; callers that mix these
// entry points with other work on that stream (torch's default stream, for one)
// stay ordered with it
cudaStream_t pick(void* stream, tp::Ctx*)
{
    return reinterpret_cast<cudaStream_t>(stream);
}

// uint64_t (unsigned long) and tp::u64 (unsigned long long) have the same layout
inline const u64* U(const uint64_t* p) { return reinterpret_cast<const u64*>(p); }
inline u64* U(uint64_t* p) { return reinterpret_cast<u64*>(p); }

std::vector<fp2> pack_host(const uint64_t* re, const uint64_t* im, size_t n)
{
    std::vector<fp2> v(n);
    for (size_t i = 0; i < n; ++i) v[i] = mk(re[i], im[i]);
    return v;
}

tp::ClaimWorkspace g_batch_ws;

}  // namespace

extern "C" {

int native_fp2_init(void)
{
    tp::device_present();
    return 0;
}

int native_fp2_cuda_available(void) { return tp::device_present() ? 1 : 0; }

const char* tp_last_error(void) { return tp::error_text(); }
int tp_last_error_code(void) { return tp::error_code(); }
void tp_clear_error(void) { tp::clear_error(); }
int tp_last_launch_count(void) { return tp::last_launch_count(); }

void native_fp2_fold(const uint64_t* in_real, const uint64_t* in_imag, size_t n_out,
                     uint64_t r_real, uint64_t r_imag, uint64_t* out_real, uint64_t* out_imag)
{
    tp::clear_error();
    tp::Ctx* c = tp::ctx();
    if (!c || n_out == 0) return;
    cudaStream_t s = c->stream;
    Scratch sc(s);
    u64* ir = sc.get<u64>(2 * n_out);
    u64* ii = sc.get<u64>(2 * n_out);
    u64* orr = sc.get<u64>(n_out);
    u64* oi = sc.get<u64>(n_out);
    if (!sc.ok) return;
    if (!h2d(ir, in_real, 16 * n_out, s) || !h2d(ii, in_imag, 16 * n_out, s)) return;
    if (!tp::launch_fold_soa(ir, ii, n_out, mk(r_real, r_imag), orr, oi, s)) return;
    if (!d2h(out_real, orr, 8 * n_out, s) || !d2h(out_imag, oi, 8 * n_out, s)) return;
    sync(s);
}

void native_fp2_expand(const uint64_t* in_real, const uint64_t* in_imag, size_t n_src,
                       size_t ncopies, uint64_t* out_real, uint64_t* out_imag)
{
    tp::clear_error();
    tp::Ctx* c = tp::ctx();
    const size_t n = n_src * ncopies;
    if (!c || n == 0) return;
    cudaStream_t s = c->stream;
    Scratch sc(s);
    u64* ir = sc.get<u64>(n_src);
    u64* ii = sc.get<u64>(n_src);
    u64* orr = sc.get<u64>(n);
    u64* oi = sc.get<u64>(n);
    if (!sc.ok) return;
    if (!h2d(ir, in_real, 8 * n_src, s) || !h2d(ii, in_imag, 8 * n_src, s)) return;
    if (!tp::launch_expand_soa(ir, ii, n_src, ncopies, orr, oi, s)) return;
    if (!d2h(out_real, orr, 8 * n, s) || !d2h(out_imag, oi, 8 * n, s)) return;
    sync(s);
}

void native_fp2_sumcheck_early(int n_gates, const int* gate_type, const int* in0, const int* in1,
                               const uint64_t* z1_real, const uint64_t* z1_imag, int n_copies,
                               int n_wires, const uint64_t* values_real,
                               const uint64_t* values_imag, const uint64_t* fact0_real,
                               const uint64_t* fact0_imag, const uint64_t* fact1_real,
                               const uint64_t* fact1_imag, const uint64_t* beta_real,
                               const uint64_t* beta_imag, const uint64_t* beta_f0_real,
                               const uint64_t* beta_f0_imag, const uint64_t* beta_f1_real,
                               const uint64_t* beta_f1_imag, uint64_t out8[8])
{
    tp::clear_error();
    tp::Ctx* c = tp::ctx();
    if (!c) return;
    if (n_copies <= 0 || n_gates <= 0) {
        memset(out8, 0, 64);  // empty sums
        return;
    }
    if (n_copies & 1) {
        tp::set_error(tp::TP_ERR_ARG, "sumcheck_early needs an even n_copies (got %d)", n_copies);
        return;
    }
    if (n_wires <= 0) {
        tp::set_error(tp::TP_ERR_ARG, "sumcheck_early needs n_wires > 0");
        return;
    }
    tp::GateForm g;
    if (!tp::build_gate_form(n_gates, gate_type, in0, in1, U(z1_real), U(z1_imag), n_wires, g)) return;
    cudaStream_t s = c->stream;
    tp::DevGateForm dg;
    if (!tp::upload_gate_form(g, dg, s)) {
        tp::free_gate_form(dg, s);
        return;
    }
    const size_t n = (size_t)n_copies, h = n / 2, W = (size_t)n_wires;
    const size_t sizes[12] = {W * n, W * n, W * h, W * h, W * h, W * h, n, n, h, h, h, h};
    const uint64_t* src[12] = {values_real, values_imag, fact0_real, fact0_imag, fact1_real,
                               fact1_imag, beta_real, beta_imag, beta_f0_real, beta_f0_imag,
                               beta_f1_real, beta_f1_imag};
    {
        Scratch sc(s);
        const u64* t[12];
        bool ok = true;
        for (int i = 0; i < 12 && ok; ++i) {
            u64* d = sc.get<u64>(sizes[i]);
            ok = sc.ok && h2d(d, src[i], 8 * sizes[i], s);
            t[i] = d;
        }
        if (ok && tp::launch_claim_explicit(dg, n_copies, t, g_batch_ws, s)) {
            u64 host[8];
            if (d2h(host, g_batch_ws.out8, 64, s) && sync(s)) memcpy(out8, host, 64);
        }
    }
    tp::free_gate_form(dg, s);
}

void native_fp2_compute_beta(const uint64_t* z_real, const uint64_t* z_imag, int n_z,
                             uint64_t init_real, uint64_t init_imag, uint64_t* out_real,
                             uint64_t* out_imag)
{
    tp::clear_error();
    tp::Ctx* c = tp::ctx();
    if (!c || n_z <= 0) return;
    if (n_z > 40) {
        tp::set_error(tp::TP_ERR_ARG, "compute_beta: n_z = %d is too large", n_z);
        return;
    }
    cudaStream_t s = c->stream;
    const size_t n = (size_t)1 << n_z;
    std::vector<fp2> z = pack_host(z_real, z_imag, (size_t)n_z);
    Scratch sc(s);
    fp2* dz = sc.get<fp2>((size_t)n_z);
    u64* orr = sc.get<u64>(n);
    u64* oi = sc.get<u64>(n);
    if (!sc.ok) return;
    if (!h2d(dz, z.data(), sizeof(fp2) * z.size(), s)) return;
    if (!tp::launch_beta(dz, n_z, mk(init_real, init_imag), orr, oi, nullptr, s)) return;
    if (!d2h(out_real, orr, 8 * n, s) || !d2h(out_imag, oi, 8 * n, s)) return;
    sync(s);
}

void native_fp2_mle_eval_base(const uint64_t* inputs, const uint64_t* z_real,
                              const uint64_t* z_imag, int n_z, uint64_t* out_real,
                              uint64_t* out_imag)
{
    tp::clear_error();
    tp::Ctx* c = tp::ctx();
    if (!c) return;
    if (n_z <= 0) {
        // reference: the first input as is (no reduction), imaginary part 0
        *out_real = inputs ? inputs[0] : 0;
        *out_imag = 0;
        return;
    }
    if (!inputs || n_z > 40) {
        tp::set_error(tp::TP_ERR_ARG, "mle_eval_base: bad inputs (n_z = %d)", n_z);
        return;
    }
    cudaStream_t s = c->stream;
    const size_t n = (size_t)1 << n_z;
    std::vector<fp2> z = pack_host(z_real, z_imag, (size_t)n_z);
    Scratch sc(s);
    u64* din = sc.get<u64>(n);
    fp2* dz = sc.get<fp2>((size_t)n_z);
    fp2* dout = sc.get<fp2>(1);
    if (!sc.ok) return;
    if (!h2d(din, inputs, 8 * n, s) || !h2d(dz, z.data(), sizeof(fp2) * z.size(), s)) return;
    if (!tp::launch_mle_base(din, dz, n_z, dout, s)) return;
    fp2 host;
    if (!d2h(&host, dout, sizeof(fp2), s) || !sync(s)) return;
    *out_real = host.re;
    *out_imag = host.im;
}

void* native_fp2_early_create(int n_gates, const int* gate_type, const int* in0, const int* in1,
                              const uint64_t* z1_real, const uint64_t* z1_imag, int n_copies,
                              int n_wires, const uint64_t* values_real,
                              const uint64_t* values_imag, const uint64_t* beta_real,
                              const uint64_t* beta_imag)
{
    tp::clear_error();
    tp::Ctx* c = tp::ctx();
    if (!c) return nullptr;
    tp::Batch* S = tp::session_create(n_gates, gate_type, in0, in1, U(z1_real), U(z1_imag),
                                      n_copies, n_wires, c->stream);
    if (!S) return nullptr;
    if (!tp::batch_load_host(S, 0, U(values_real), U(values_imag), U(beta_real), U(beta_imag))) {
        tp::batch_destroy(S);
        return nullptr;
    }
    return S;
}

int native_fp2_early_claim(void* handle, uint64_t out8[8])
{
    tp::clear_error();
    if (!handle) return -1;
    return tp::session_claim(static_cast<tp::Batch*>(handle), U(out8)) ? 0 : -1;
}

int native_fp2_early_fold(void* handle, uint64_t r_real, uint64_t r_imag)
{
    tp::clear_error();
    if (!handle) return -1;
    return tp::batch_fold(static_cast<tp::Batch*>(handle), 0, mk(r_real, r_imag)) ? 0 : -1;
}

int native_fp2_early_finish(void* handle, uint64_t* wire_real, uint64_t* wire_imag,
                            uint64_t* beta_real, uint64_t* beta_imag)
{
    tp::clear_error();
    if (!handle) return -1;
    return tp::session_finish(static_cast<tp::Batch*>(handle), U(wire_real), U(wire_imag),
                              U(beta_real), U(beta_imag)) ? 0 : -1;
}

int native_fp2_early_n_copies(void* handle)
{
    return handle ? static_cast<tp::Batch*>(handle)->frames[0]->n_copies : 0;
}

int native_fp2_early_n_wires(void* handle)
{
    return handle ? static_cast<tp::Batch*>(handle)->frames[0]->n_wires : 0;
}

void native_fp2_early_destroy(void* handle) { tp::batch_destroy(static_cast<tp::Batch*>(handle)); }

// ---- host-only inspection ----------------------------------------------------

int tp_gate_form(int n_gates, const int* gate_type, const int* in0, const int* in1,
                 const uint64_t* z1_real, const uint64_t* z1_imag, int n_wires, uint64_t* k0,
                 uint64_t* lin, int max_terms, int* term_ab, uint64_t* term_c)
{
    tp::clear_error();
    tp::GateForm g;
    if (n_wires <= 0 ||
        !tp::build_gate_form(n_gates, gate_type, in0, in1, U(z1_real), U(z1_imag), n_wires, g))
        return -1;
    k0[0] = g.K0.re;
    k0[1] = g.K0.im;
    for (int w = 0; w < n_wires; ++w) {
        lin[2 * w] = g.L[w].re;
        lin[2 * w + 1] = g.L[w].im;
    }
    const int nt = (int)g.tc.size();
    for (int i = 0; i < nt && i < max_terms; ++i) {
        term_ab[2 * i] = g.ta[i];
        term_ab[2 * i + 1] = g.tb[i];
        term_c[2 * i] = g.tc[i].re;
        term_c[2 * i + 1] = g.tc[i].im;
    }
    return nt;
}

// ---- device-buffer extensions ------------------------------------------------

void* tp_early_create_dev(int n_gates, const int* gate_type, const int* in0, const int* in1,
                          const uint64_t* z1_real, const uint64_t* z1_imag, int n_copies,
                          int n_wires, const void* d_values, const void* d_beta, int borrow,
                          void* stream)
{
    tp::clear_error();
    tp::Ctx* c = tp::ctx();
    if (!c) return nullptr;
    tp::Batch* S = tp::session_create(n_gates, gate_type, in0, in1, U(z1_real), U(z1_imag),
                                      n_copies, n_wires, pick(stream, c));
    if (!S) return nullptr;
    if (!tp::batch_load_device(S, 0, static_cast<const fp2*>(d_values),
                               static_cast<const fp2*>(d_beta), borrow != 0)) {
        tp::batch_destroy(S);
        return nullptr;
    }
    return S;
}

int tp_early_claim_dev(void* handle, void* d_out8)
{
    tp::clear_error();
    if (!handle) return -1;
    u64* p = static_cast<u64*>(d_out8);
    return tp::batch_claim(static_cast<tp::Batch*>(handle), &p) ? 0 : -1;
}

int tp_early_finish_dev(void* handle, void* d_wires, void* d_beta)
{
    tp::clear_error();
    if (!handle) return -1;
    fp2* w = static_cast<fp2*>(d_wires);
    fp2* b = static_cast<fp2*>(d_beta);
    return tp::batch_finish(static_cast<tp::Batch*>(handle), &w, &b) ? 0 : -1;
}

int tp_early_launches(void* handle)
{
    return handle ? static_cast<tp::Batch*>(handle)->launches : 0;
}

int tp_fold_dev(const void* d_in, size_t n_out, uint64_t r_real, uint64_t r_imag, void* d_out,
                void* stream)
{
    tp::clear_error();
    tp::Ctx* c = tp::ctx();
    if (!c) return -1;
    return tp::launch_fold_aos(static_cast<const fp2*>(d_in), n_out, mk(r_real, r_imag),
                               static_cast<fp2*>(d_out), pick(stream, c)) ? 0 : -1;
}

int tp_compute_beta_dev(const void* d_z, int n_z, uint64_t init_real, uint64_t init_imag,
                        void* d_out, void* stream)
{
    tp::clear_error();
    tp::Ctx* c = tp::ctx();
    if (!c) return -1;
    return tp::launch_beta(static_cast<const fp2*>(d_z), n_z, mk(init_real, init_imag), nullptr,
                           nullptr, static_cast<fp2*>(d_out), pick(stream, c)) ? 0 : -1;
}

int tp_mle_eval_base_dev(const void* d_inputs, const void* d_z, int n_z, void* d_out,
                         void* stream)
{
    tp::clear_error();
    tp::Ctx* c = tp::ctx();
    if (!c) return -1;
    if (n_z <= 0 || n_z > 40) {
        tp::set_error(tp::TP_ERR_ARG, "tp_mle_eval_base_dev: n_z must be in [1, 40]");
        return -1;
    }
    return tp::launch_mle_base(static_cast<const u64*>(d_inputs), static_cast<const fp2*>(d_z), n_z,
                               static_cast<fp2*>(d_out), pick(stream, c)) ? 0 : -1;
}

int tp_table_from_pixels(const void* d_pixels, int n_copies, int n_copies_padded, int copy_size,
                         int n_wires, int const_idx, uint64_t const_val, void* d_table,
                         void* d_inputs, void* stream)
{
    tp::clear_error();
    tp::Ctx* c = tp::ctx();
    if (!c) return -1;
    return tp::launch_table_from_pixels(static_cast<const unsigned char*>(d_pixels), n_copies,
                                        n_copies_padded, copy_size, n_wires, const_idx, const_val,
                                        static_cast<fp2*>(d_table), static_cast<u64*>(d_inputs),
                                        pick(stream, c)) ? 0 : -1;
}

void* tp_early_create_pixels(int n_gates, const int* gate_type, const int* in0, const int* in1,
                             const uint64_t* z1_real, const uint64_t* z1_imag,
                             const void* d_pixels, int n_copies, int n_copies_padded,
                             int copy_size, int n_wires, int const_idx, uint64_t const_val,
                             const void* d_beta, void* stream)
{
    tp::clear_error();
    tp::Ctx* c = tp::ctx();
    if (!c) return nullptr;
    tp::Batch* S = tp::session_create(n_gates, gate_type, in0, in1, U(z1_real), U(z1_imag),
                                      n_copies_padded, n_wires, pick(stream, c));
    if (!S) return nullptr;
    tp::PixSrc px;
    px.pix = static_cast<const unsigned char*>(d_pixels);
    px.n_real = n_copies;
    px.cs = copy_size;
    px.const_idx = const_idx;
    px.const_val = const_val;
    if (!tp::batch_load_pixels(S, 0, px, static_cast<const fp2*>(d_beta))) {
        tp::batch_destroy(S);
        return nullptr;
    }
    return S;
}

int tp_mle_eval_pixels(const void* d_pixels, int n_copies, int n_copies_padded, int copy_size,
                       int n_wires, int const_idx, uint64_t const_val, const void* d_z,
                       void* d_out, void* stream)
{
    tp::clear_error();
    tp::Ctx* c = tp::ctx();
    if (!c) return -1;
    tp::PixSrc px;
    px.pix = static_cast<const unsigned char*>(d_pixels);
    px.n_real = n_copies;
    px.cs = copy_size;
    px.const_idx = const_idx;
    px.const_val = const_val;
    int launches = 0;
    return tp::launch_mle_pixels(px, n_copies_padded, n_wires, static_cast<const fp2*>(d_z),
                                 static_cast<fp2*>(d_out), pick(stream, c), &launches) ? 0 : -1;
}

int tp_early_rounds_dev(void* handle, int n_rounds, const uint64_t* challenges, void* d_claims)
{
    tp::clear_error();
    if (!handle || n_rounds < 0) return -1;
    tp::Batch* S = static_cast<tp::Batch*>(handle);
    u64* out = static_cast<u64*>(d_claims);
    for (int k = 0; k < n_rounds; ++k) {
        u64* p = out ? out + 8 * (size_t)k : nullptr;
        if (!tp::batch_claim(S, &p)) return -1;
        if (!tp::batch_fold(S, 0, mk(challenges[2 * k], challenges[2 * k + 1]))) return -1;
    }
    return 0;
}

// ---- batches of frames -------------------------------------------------------

void* tp_batch_create(int n_frames, void* stream)
{
    tp::clear_error();
    tp::Ctx* c = tp::ctx();
    if (!c) return nullptr;
    return tp::batch_create(n_frames, pick(stream, c));
}

int tp_batch_set_pixels(void* batch, int i, int n_gates, const int* gate_type, const int* in0,
                        const int* in1, const uint64_t* z1_real, const uint64_t* z1_imag,
                        const void* d_pixels, int n_copies, int n_copies_padded, int copy_size,
                        int n_wires, int const_idx, uint64_t const_val, const void* d_beta)
{
    tp::clear_error();
    if (!batch) return -1;
    tp::Batch* B = static_cast<tp::Batch*>(batch);
    if (!tp::batch_set_gates(B, i, n_gates, gate_type, in0, in1, U(z1_real), U(z1_imag),
                             n_copies_padded, n_wires))
        return -1;
    tp::PixSrc px;
    px.pix = static_cast<const unsigned char*>(d_pixels);
    px.n_real = n_copies;
    px.cs = copy_size;
    px.const_idx = const_idx;
    px.const_val = const_val;
    return tp::batch_load_pixels(B, i, px, static_cast<const fp2*>(d_beta)) ? 0 : -1;
}

int tp_batch_set_table(void* batch, int i, int n_gates, const int* gate_type, const int* in0,
                       const int* in1, const uint64_t* z1_real, const uint64_t* z1_imag,
                       int n_copies, int n_wires, const void* d_values, const void* d_beta,
                       int borrow)
{
    tp::clear_error();
    if (!batch) return -1;
    tp::Batch* B = static_cast<tp::Batch*>(batch);
    if (!tp::batch_set_gates(B, i, n_gates, gate_type, in0, in1, U(z1_real), U(z1_imag), n_copies,
                             n_wires))
        return -1;
    return tp::batch_load_device(B, i, static_cast<const fp2*>(d_values),
                                 static_cast<const fp2*>(d_beta), borrow != 0) ? 0 : -1;
}

int tp_batch_claim(void* batch, void* d_claims)
{
    tp::clear_error();
    if (!batch) return -1;
    tp::Batch* B = static_cast<tp::Batch*>(batch);
    std::vector<u64*> ptrs(B->frames.size(), nullptr);
    if (d_claims)
        for (size_t i = 0; i < ptrs.size(); ++i) ptrs[i] = static_cast<u64*>(d_claims) + 8 * i;
    return tp::batch_claim(B, ptrs.data()) ? 0 : -1;
}

int tp_batch_fold(void* batch, const uint64_t* challenges)
{
    tp::clear_error();
    if (!batch) return -1;
    tp::Batch* B = static_cast<tp::Batch*>(batch);
    for (size_t i = 0; i < B->frames.size(); ++i) {
        if (B->frames[i]->n_copies < 2) continue;
        if (!tp::batch_fold(B, (int)i, mk(challenges[2 * i], challenges[2 * i + 1]))) return -1;
    }
    return 0;
}

int tp_batch_fold_dev(void* batch, const void* d_challenges)
{
    tp::clear_error();
    if (!batch || !d_challenges) {
        tp::set_error(tp::TP_ERR_ARG, "tp_batch_fold_dev: null batch or challenges");
        return -1;
    }
    tp::Batch* B = static_cast<tp::Batch*>(batch);
    const tp::fp2* d = static_cast<const tp::fp2*>(d_challenges);
    for (size_t i = 0; i < B->frames.size(); ++i) {
        if (B->frames[i]->n_copies < 2) continue;
        if (!tp::batch_fold_dev(B, (int)i, d + i)) return -1;
    }
    return 0;
}

int tp_batch_n_copies(void* batch, int i)
{
    if (!batch) return 0;
    tp::Batch* B = static_cast<tp::Batch*>(batch);
    if (i < 0 || i >= (int)B->frames.size()) return 0;
    return B->frames[(size_t)i]->n_copies;
}

int tp_batch_finish(void* batch, void* d_wires, void* d_beta)
{
    tp::clear_error();
    if (!batch) return -1;
    tp::Batch* B = static_cast<tp::Batch*>(batch);
    const size_t n = B->frames.size();
    std::vector<fp2*> w(n, nullptr), b(n, nullptr);
    for (size_t i = 0; i < n; ++i) {
        if (d_wires) w[i] = static_cast<fp2*>(d_wires) + i * (size_t)B->frames[i]->n_wires;
        if (d_beta) b[i] = static_cast<fp2*>(d_beta) + i;
    }
    return tp::batch_finish(B, w.data(), b.data()) ? 0 : -1;
}

int tp_batch_vole_rounds_graph(void* batch, void* d_claims, void* d_fs_states, void* d_vole_states, const void* d_u,
                               const void* d_v, long long count, int layer, void* d_challenges, void* d_proof,
                               void* d_wires, void* d_beta)
{
    tp::clear_error();
    if (!batch || !d_claims || !d_fs_states || !d_vole_states || !d_u || !d_v || count < 4 || !d_challenges ||
        !d_wires || !d_beta) {
        tp::set_error(tp::TP_ERR_ARG, "tp_batch_vole_rounds_graph: bad arguments");
        return -1;
    }
    tp::Batch* B = static_cast<tp::Batch*>(batch);
    const size_t n = B->frames.size();
    std::vector<fp2*> w(n, nullptr), b(n, nullptr);
    for (size_t i = 0; i < n; ++i) {
        w[i] = static_cast<fp2*>(d_wires) + i * (size_t)B->frames[i]->n_wires;
        b[i] = static_cast<fp2*>(d_beta) + i;
    }
    return tp::batch_vole_rounds_graph(B, static_cast<u64*>(d_claims), d_fs_states, d_vole_states,
                                       static_cast<const fp2*>(d_u), static_cast<const fp2*>(d_v), count, layer,
                                       static_cast<fp2*>(d_challenges), static_cast<fp2*>(d_proof), w.data(),
                                       b.data())
               ? 0
               : -1;
}

int tp_batch_graph_replays(void* batch)
{
    return batch ? static_cast<tp::Batch*>(batch)->graph_replays : 0;
}

int tp_batch_autotune(int on)
{
    tp::clear_error();
    tp::batch_tune_enable(on != 0);
    return 0;
}

int tp_batch_tune_table(int* kind, int* bucket, int* ctas_per_sm, int max)
{
    tp::clear_error();
    if (!tp::ctx()) return -1;
    if (max > 0 && (!kind || !bucket || !ctas_per_sm)) {
        tp::set_error(tp::TP_ERR_ARG, "tp_batch_tune_table: null outputs");
        return -1;
    }
    return tp::batch_tune_table(kind, bucket, ctas_per_sm, max);
}

int tp_batch_tune_set(int kind, int bucket, int ctas_per_sm)
{
    tp::clear_error();
    return tp::batch_tune_set(kind, bucket, ctas_per_sm) ? 0 : -1;
}

int tp_batch_finish_frame(void* batch, int i, void* d_wires, void* d_beta)
{
    tp::clear_error();
    if (!batch) return -1;
    return tp::batch_finish_frame(static_cast<tp::Batch*>(batch), i, static_cast<fp2*>(d_wires),
                                  static_cast<fp2*>(d_beta))
               ? 0
               : -1;
}

void tp_batch_release(void* batch, int i, int free_buffers)
{
    if (batch) tp::batch_release(static_cast<tp::Batch*>(batch), i, free_buffers != 0);
}

int tp_batch_launches(void* batch) { return batch ? static_cast<tp::Batch*>(batch)->launches : 0; }

void tp_batch_destroy(void* batch) { tp::batch_destroy(static_cast<tp::Batch*>(batch)); }

int tp_timer_enable(int max_pairs) { return tp::timer_enable(max_pairs) ? 0 : -1; }
void tp_timer_disable(void) { tp::timer_disable(); }
void tp_timer_reset(void) { tp::timer_reset(); }
int tp_timer_read(float* ms, int* tags, int max_pairs) { return tp::timer_read(ms, tags, max_pairs); }

void tp_batch_reset(void* batch)
{
    if (batch) tp::batch_reset(static_cast<tp::Batch*>(batch));
}

int tp_compute_beta_batch_dev(const void* d_z, int n_z, int n_frames, void* d_out, void* stream)
{
    tp::clear_error();
    tp::Ctx* c = tp::ctx();
    if (!c) return -1;
    if (n_z <= 0 || n_z > 30 || n_frames <= 0) {
        tp::set_error(tp::TP_ERR_ARG, "beta batch: n_z %d, frames %d", n_z, n_frames);
        return -1;
    }
    int launches = 0;
    return tp::launch_beta_batch(static_cast<const fp2*>(d_z), n_z, n_frames,
                                 static_cast<fp2*>(d_out), pick(stream, c), &launches) ? 0 : -1;
}

int tp_mle_eval_pixels_batch(int n_frames, const void* const* d_pixels, const int* n_copies,
                             int n_copies_padded, int copy_size, int n_wires, int const_idx,
                             uint64_t const_val, const void* d_points, void* d_out, void* stream)
{
    tp::clear_error();
    tp::Ctx* c = tp::ctx();
    if (!c) return -1;
    std::vector<tp::MleFrame> fr((size_t)std::max(0, n_frames));
    for (int i = 0; i < n_frames; ++i) {
        fr[(size_t)i].pix = static_cast<const unsigned char*>(d_pixels[i]);
        fr[(size_t)i].n_real = n_copies[i];
        fr[(size_t)i].pad_ = 0;
    }
    int launches = 0;
    return tp::launch_mle_pixels_batch(fr.data(), n_frames, n_copies_padded, copy_size, n_wires,
                                       const_idx, const_val, static_cast<const fp2*>(d_points),
                                       static_cast<fp2*>(d_out), pick(stream, c), &launches) ? 0 : -1;
}

}  // extern "C"
