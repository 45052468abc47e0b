// C ABI of the Fp2 NTT and the Reed-Solomon commit (include/orion_gpu.h).
#include <stdint.h>

#include <vector>

#include "ntt.h"
#include "virgo.h"
#include "runtime.h"
#include "../../include/orion_gpu.h"

namespace {

struct DevBuf {
    void* p = nullptr;
    cudaStream_t s;
    explicit DevBuf(size_t bytes, cudaStream_t st) : s(st) { p = tp::dev_alloc(bytes, st); }
    ~DevBuf()
    {
        if (p) tp::dev_free(p, s);
    }
};

bool canonical(const uint64_t* a, long long words, const char* who)
{
    for (long long i = 0; i < words; ++i)
        if (a[i] >= tp::P61) {
            tp::set_error(tp::TP_ERR_ARG, "%s: element %lld is not canonical", who, i / 2);
            return false;
        }
    return true;
}

bool pow2(long long n) { return n > 0 && (n & (n - 1)) == 0; }

int host_transform(const uint64_t* in, int coef_len, int order, uint64_t* out, bool inv)
{
    tp::clear_error();
    tp::Ctx* c = tp::ctx();
    if (!c) return -1;
    const char* who = inv ? "tp_ifft" : "tp_fft";
    if (!in || !out || !pow2(coef_len) || !pow2(order) || coef_len > order || order > (1 << tp::ntt::kMaxLog)) {
        tp::set_error(tp::TP_ERR_ARG, "%s: need powers of two coef_len %d <= order %d <= 2^%d", who, coef_len,
                      order, tp::ntt::kMaxLog);
        return -1;
    }
    const long long n_in = inv ? order : coef_len, n_out = inv ? coef_len : order;
    if (!canonical(in, 2 * n_in, who)) return -1;
    cudaStream_t s = c->stream;
    DevBuf d_in(16 * (size_t)n_in, s), d_out(16 * (size_t)n_out, s);
    if (!d_in.p || !d_out.p) return -1;
    if (!tp::host_to_device(d_in.p, in, 16 * (size_t)n_in, s)) return -1;
    const ulonglong2* di = static_cast<const ulonglong2*>(d_in.p);
    ulonglong2* dout = static_cast<ulonglong2*>(d_out.p);
    const bool ok = inv ? tp::ntt::inverse(di, coef_len, order, dout, 1, 0, 0, nullptr, s)
                        : tp::ntt::forward(di, coef_len, order, dout, 1, 0, 0, nullptr, s);
    if (!ok) return -1;
    return tp::device_to_host(out, d_out.p, 16 * (size_t)n_out, s) ? 0 : -1;
}

}  // namespace

extern "C" {

int tp_fft(const uint64_t* coef, int coef_len, int order, uint64_t* result)
{
    return host_transform(coef, coef_len, order, result, false);
}

int tp_ifft(const uint64_t* evals, int coef_len, int order, uint64_t* result)
{
    return host_transform(evals, coef_len, order, result, true);
}

int tp_fft_dev(const void* d_coef, long long coef_len, long long order, void* d_out, int batch,
               long long in_stride, long long out_stride, void* stream)
{
    tp::clear_error();
    if (!tp::ctx()) return -1;
    if (!d_coef || !d_out) {
        tp::set_error(tp::TP_ERR_ARG, "tp_fft_dev: null buffer");
        return -1;
    }
    return tp::ntt::forward(static_cast<const ulonglong2*>(d_coef), coef_len, order, static_cast<ulonglong2*>(d_out),
                            batch, in_stride, out_stride, nullptr, reinterpret_cast<cudaStream_t>(stream))
               ? 0
               : -1;
}

int tp_ifft_dev(const void* d_evals, long long coef_len, long long order, void* d_out, int batch,
                long long in_stride, long long out_stride, void* stream)
{
    tp::clear_error();
    if (!tp::ctx()) return -1;
    if (!d_evals || !d_out) {
        tp::set_error(tp::TP_ERR_ARG, "tp_ifft_dev: null buffer");
        return -1;
    }
    return tp::ntt::inverse(static_cast<const ulonglong2*>(d_evals), coef_len, order, static_cast<ulonglong2*>(d_out),
                            batch, in_stride, out_stride, nullptr, reinterpret_cast<cudaStream_t>(stream))
               ? 0
               : -1;
}

int tp_ntt_autotune(int log_n, int batch, int* digits_out, float* ms_out)
{
    tp::clear_error();
    if (!tp::ctx()) return -1;
    std::vector<int> best;
    float ms = 0.f;
    if (!tp::ntt::autotune(log_n, batch, best, &ms)) return -1;
    for (size_t i = 0; i < 3; ++i)
        if (digits_out) digits_out[i] = i < best.size() ? best[i] : 0;
    if (ms_out) *ms_out = ms;
    return (int)best.size();
}

int tp_fri_commit_step_dev(const void* d_witness, int log_m, uint64_t r_real, uint64_t r_imag, void* d_next,
                           void* d_tree, void* stream)
{
    tp::clear_error();
    if (!tp::ctx()) return -1;
    if (!d_witness || !d_next || !d_tree) {
        tp::set_error(tp::TP_ERR_ARG, "tp_fri_commit_step_dev: null buffer");
        return -1;
    }
    return tp::rs::fri_step(static_cast<const ulonglong2*>(d_witness), log_m, tp::mk(r_real, r_imag),
                            static_cast<ulonglong2*>(d_next), static_cast<unsigned char*>(d_tree),
                            reinterpret_cast<cudaStream_t>(stream))
               ? 0
               : -1;
}

int tp_rs_commit_dev(const void* d_src, int log_len, void* d_l_eval, void* d_tree, void* stream)
{
    tp::clear_error();
    if (!tp::ctx()) return -1;
    if (!d_src || !d_l_eval || !d_tree) {
        tp::set_error(tp::TP_ERR_ARG, "tp_rs_commit_dev: null buffer");
        return -1;
    }
    return tp::rs::commit(static_cast<const ulonglong2*>(d_src), log_len, static_cast<ulonglong2*>(d_l_eval),
                          static_cast<unsigned char*>(d_tree), reinterpret_cast<cudaStream_t>(stream))
               ? 0
               : -1;
}

int tp_rs_commit(const uint64_t* src, int log_len, uint64_t* l_eval_out, unsigned char* tree_out)
{
    tp::clear_error();
    tp::Ctx* c = tp::ctx();
    if (!c) return -1;
    if (!src || !tree_out || log_len < tp::rs::kMinLog || log_len > tp::rs::kMaxLog) {
        tp::set_error(tp::TP_ERR_ARG, "tp_rs_commit: need src, tree_out and %d <= log_len <= %d", tp::rs::kMinLog,
                      tp::rs::kMaxLog);
        return -1;
    }
    const long long n = 1LL << log_len, n_eval = n << 5, n_tree = n >> 1;
    if (!canonical(src, 2 * n, "tp_rs_commit")) return -1;
    cudaStream_t s = c->stream;
    DevBuf d_src(16 * (size_t)n, s), d_eval(16 * (size_t)n_eval, s), d_tree(32 * (size_t)n_tree, s);
    if (!d_src.p || !d_eval.p || !d_tree.p) return -1;
    if (!tp::host_to_device(d_src.p, src, 16 * (size_t)n, s)) return -1;
    if (!tp::rs::commit(static_cast<const ulonglong2*>(d_src.p), log_len, static_cast<ulonglong2*>(d_eval.p),
                        static_cast<unsigned char*>(d_tree.p), s))
        return -1;
    if (!tp::device_to_host(tree_out, d_tree.p, 32 * (size_t)n_tree, s)) return -1;
    if (l_eval_out && !tp::device_to_host(l_eval_out, d_eval.p, 16 * (size_t)n_eval, s)) return -1;
    return 0;
}

int tp_virgo_sumcheck_update_dev(const void* d_vma, const void* d_addv, const void* d_ams, long long total_uv,
                                 uint64_t r_real, uint64_t r_imag, int current_bit, void* d_vma_out,
                                 void* d_addv_out, void* d_ams_out, void* d_ret, void* stream)
{
    tp::clear_error();
    if (!tp::ctx()) return -1;
    if (!d_vma || !d_addv || !d_ams || !d_vma_out || !d_addv_out || !d_ams_out || !d_ret) {
        tp::set_error(tp::TP_ERR_ARG, "tp_virgo_sumcheck_update_dev: null buffer");
        return -1;
    }
    return tp::virgo::update(static_cast<const ulonglong2*>(d_vma), static_cast<const ulonglong2*>(d_addv),
                             static_cast<const ulonglong2*>(d_ams), total_uv, tp::mk(r_real, r_imag), current_bit,
                             static_cast<ulonglong2*>(d_vma_out), static_cast<ulonglong2*>(d_addv_out),
                             static_cast<ulonglong2*>(d_ams_out), static_cast<ulonglong2*>(d_ret),
                             reinterpret_cast<cudaStream_t>(stream))
               ? 0
               : -1;
}

void* tp_virgo_layer_create(int length_g, int length_u, const int* ty, const long long* u, const long long* v,
                            const int* comb_ptr, const int* comb_src, const uint64_t* comb_w)
{
    tp::clear_error();
    return tp::virgo::layer_create(length_g, length_u, ty, u, v, comb_ptr, comb_src, comb_w);
}

void tp_virgo_layer_destroy(void* layer) { tp::virgo::layer_destroy(static_cast<tp::virgo::Layer*>(layer)); }

int tp_virgo_phase1_init_dev(void* layer, const void* d_values, const uint64_t* r0, const uint64_t* r1,
                             const uint64_t* alpha, const uint64_t* beta, void* d_vma, void* d_addv, void* d_ams,
                             void* stream)
{
    tp::clear_error();
    if (!tp::ctx()) return -1;
    if (!layer || !d_values || !d_vma || !d_addv || !d_ams) {
        tp::set_error(tp::TP_ERR_ARG, "tp_virgo_phase1_init_dev: null layer or buffer");
        return -1;
    }
    return tp::virgo::phase1_init(*static_cast<tp::virgo::Layer*>(layer), static_cast<const ulonglong2*>(d_values),
                                  r0, r1, alpha, beta, static_cast<ulonglong2*>(d_vma),
                                  static_cast<ulonglong2*>(d_addv), static_cast<ulonglong2*>(d_ams),
                                  reinterpret_cast<cudaStream_t>(stream))
               ? 0
               : -1;
}

int tp_virgo_phase2_init_dev(void* layer, const void* d_values, const uint64_t* r0, const uint64_t* r1,
                             const uint64_t* alpha, const uint64_t* beta, const void* d_vma0, const uint64_t* prev_r,
                             const uint64_t* r_u, void* d_vma, void* d_addv, void* d_ams, void* stream)
{
    tp::clear_error();
    if (!tp::ctx()) return -1;
    if (!layer || !d_values || !d_vma || !d_addv || !d_ams) {
        tp::set_error(tp::TP_ERR_ARG, "tp_virgo_phase2_init_dev: null layer or buffer");
        return -1;
    }
    return tp::virgo::phase2_init(*static_cast<tp::virgo::Layer*>(layer), static_cast<const ulonglong2*>(d_values),
                                  r0, r1, alpha, beta, static_cast<const ulonglong2*>(d_vma0), prev_r, r_u,
                                  static_cast<ulonglong2*>(d_vma), static_cast<ulonglong2*>(d_addv),
                                  static_cast<ulonglong2*>(d_ams), reinterpret_cast<cudaStream_t>(stream))
               ? 0
               : -1;
}

}  // extern "C"
