// Host side of the early-round sessions: a Batch of frames advanced round by
// round, one kernel launch per round (per source kind) for all frames.
//
// State machine per frame (TruePix-main/native_fp2/native_fp2_core.hpp:163-298
// for the single-session semantics): claim() evaluates the round polynomial at
// 0, 1, -1, 2 over the current copies; fold(r) records r and is applied by the
// next claim in the same pass (fold + claim fused), by a second fold, or by
// finish(). The first table of a frame may be its uint8 bytes; it is then
// never materialised.
#include "gkr.h"
#include "gkr_internal.cuh"
#include "runtime.h"

#include <algorithm>
#include <cstring>

namespace tp {

namespace {

// (re)use the frame's buffers: grow only when a configuration needs more
bool frame_alloc(Frame* f, size_t rows0, size_t rows1, cudaStream_t s)
{
    const size_t n = (size_t)f->n_copies0;
    if (f->borrowed0) {
        f->buf[0] = nullptr;
        f->cap0 = 0;
        f->borrowed0 = false;
    }
    if (rows0 > f->cap0) {
        dev_free(f->buf[0], s);
        f->buf[0] = (fp2*)dev_alloc(sizeof(fp2) * rows0, s);
        f->cap0 = f->buf[0] ? rows0 : 0;
    }
    if (rows1 > f->cap1) {
        dev_free(f->buf[1], s);
        f->buf[1] = (fp2*)dev_alloc(sizeof(fp2) * rows1, s);
        f->cap1 = f->buf[1] ? rows1 : 0;
    }
    if (n > f->capb) {
        dev_free(f->beta[0], s);
        dev_free(f->beta[1], s);
        f->beta[0] = (fp2*)dev_alloc(sizeof(fp2) * n, s);
        f->beta[1] = (fp2*)dev_alloc(sizeof(fp2) * n, s);
        f->capb = (f->beta[0] && f->beta[1]) ? n : 0;
    }
    f->cur = 0;
    f->pending = false;
    f->r_dev = nullptr;
    f->pix_cur = false;
    return (!rows0 || f->buf[0]) && f->buf[1] && f->beta[0] && f->beta[1];
}

// apply a recorded fold without a claim
bool apply_fold(Frame* f, cudaStream_t s, int* launches)
{
    const int n_out = f->n_phys >> 1;
    if (f->pix_cur) {
        if (!launch_fold_pixels(f->px, f->W_rows, n_out, f->r, f->buf[1], f->beta[0], f->beta[1], s,
                                launches))
            return false;
        f->pix_cur = false;
        f->cur = 1;
    } else {
        const int nxt = f->cur ^ 1;
        if (!launch_fold_rows(f->buf[f->cur], f->n_phys, f->buf[nxt], f->W_rows, f->beta[f->cur],
                              f->beta[nxt], f->r, s, launches))
            return false;
        f->cur = nxt;
    }
    f->n_phys = n_out;
    f->pending = false;
    return true;
}

bool ensure_workspace(Batch* B, size_t jobs, size_t ctas)
{
    cudaStream_t s = B->stream;
    if (jobs > B->cap_jobs) {
        dev_free(B->d_jobs, s);
        B->cap_jobs = std::max<size_t>(jobs, 16);
        B->d_jobs = (Job*)dev_alloc(sizeof(Job) * B->cap_jobs, s);
        if (!B->d_jobs) return false;
    }
    if (jobs > B->cap_tickets) {
        dev_free(B->tickets, s);
        B->cap_tickets = std::max<size_t>(jobs, 16);
        B->tickets = (unsigned*)dev_alloc(sizeof(unsigned) * B->cap_tickets, s);
        if (!B->tickets) return false;
        TP_CUDA_OK(cudaMemsetAsync(B->tickets, 0, sizeof(unsigned) * B->cap_tickets, s), "tickets");
    }
    if (ctas > B->cap_partials) {
        dev_free(B->partials, s);
        B->cap_partials = std::max<size_t>(ctas, 4096);
        B->partials = (fp2*)dev_alloc(sizeof(fp2) * 4 * B->cap_partials, s);
        if (!B->partials) return false;
    }
    return true;
}

// A job whose frame's pending fold takes its challenge from device memory gets
// it written into the uploaded job array, in stream order, before the launch.
struct RPatch {
    const fp2* r;
    long long job;
};

__global__ void patch_r_kernel(Job* __restrict__ jobs, const RPatch* __restrict__ p, int n)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) jobs[p[i].job].r = *p[i].r;
}

bool upload_jobs(Batch* B, const Job* jobs, size_t n, const std::vector<const fp2*>& rdev)
{
    if (!upload_async(B->d_jobs, jobs, sizeof(Job) * n, B->stream)) return false;
    std::vector<RPatch> p;
    for (size_t q = 0; q < n && q < rdev.size(); ++q)
        if (rdev[q]) p.push_back(RPatch{rdev[q], (long long)q});
    if (p.empty()) return true;
    if (p.size() > B->cap_patch) {
        dev_free(B->d_patch, B->stream);
        B->cap_patch = std::max<size_t>(p.size(), 64);
        B->d_patch = dev_alloc(sizeof(RPatch) * B->cap_patch, B->stream);
        if (!B->d_patch) {
            B->cap_patch = 0;
            return false;
        }
    }
    if (!upload_async(B->d_patch, p.data(), sizeof(RPatch) * p.size(), B->stream)) return false;
    patch_r_kernel<<<(unsigned)((p.size() + 127) / 128), 128, 0, B->stream>>>(
        B->d_jobs, static_cast<const RPatch*>(B->d_patch), (int)p.size());
    ++B->launches;
    return !cuda_failed(cudaGetLastError(), "challenge patch");
}

bool device_fold_blocked(const Frame* f)
{
    if (f->pending && f->r_dev) {
        set_error(TP_ERR_ARG, "a fold with a device challenge needs a claim or finish before the next fold");
        return true;
    }
    return false;
}

Job base_job(const Frame* f)
{
    Job j;
    memset(&j, 0, sizeof(j));
    j.L = f->form.L;
    j.ab = f->form.ab;
    j.cf = f->form.c;
    j.n_terms = f->form.n_terms;
    j.K0 = f->form.K0;
    j.Lc = f->Lc;
    j.r = f->r;
    j.W = f->n_wires;
    j.W_rows = f->W_rows;
    j.n_in = f->n_phys;
    j.beta = f->beta[f->cur];
    if (f->pix_cur) {
        j.pix = f->px.pix;
        j.n_real = f->px.n_real;
        j.cs = f->px.cs;
        j.const_idx = f->px.const_idx;
        j.const_val = f->px.const_val;
    } else {
        j.A = f->buf[f->cur];
    }
    return j;
}

}  // namespace

Batch* batch_create(int n_frames, cudaStream_t s)
{
    if (n_frames <= 0) {
        set_error(TP_ERR_ARG, "a batch needs at least one frame");
        return nullptr;
    }
    if (!ctx()) return nullptr;
    Batch* B = new Batch();
    B->stream = s;
    for (int i = 0; i < n_frames; ++i) B->frames.push_back(new Frame());
    return B;
}

bool batch_set_gates(Batch* B, int i, int n_gates, const int* type, const int* in0,
                     const int* in1, const u64* z_re, const u64* z_im, int n_copies, int n_wires)
{
    if (i < 0 || i >= (int)B->frames.size()) {
        set_error(TP_ERR_ARG, "frame index %d outside the batch", i);
        return false;
    }
    if (n_gates <= 0 || n_wires <= 0 || n_copies < 2 || (n_copies & (n_copies - 1)) != 0) {
        set_error(TP_ERR_ARG, "early session needs n_gates > 0, n_wires > 0 and n_copies a "
                              "power of two >= 2 (got %d, %d, %d)", n_gates, n_wires, n_copies);
        return false;
    }
    Frame* f = B->frames[(size_t)i];
    if (f->configured) {
        set_error(TP_ERR_ARG, "frame %d is already configured (tp_batch_reset first)", i);
        return false;
    }
    GateForm g;
    if (!build_gate_form(n_gates, type, in0, in1, z_re, z_im, n_wires, g)) return false;
    free_gate_form(f->form, B->stream);
    f->n_wires = f->W_rows = n_wires;
    f->n_copies0 = f->n_copies = f->n_phys = n_copies;
    f->L_host = g.L;
    f->Lc = f2zero();
    if (!upload_gate_form(g, f->form, B->stream)) return false;
    if ((size_t)n_wires + 1 > f->capfin) {
        dev_free(f->fin, B->stream);
        f->fin = (fp2*)dev_alloc(sizeof(fp2) * ((size_t)n_wires + 1), B->stream);
        f->capfin = f->fin ? (size_t)n_wires + 1 : 0;
    }
    if (!f->out8) f->out8 = (u64*)dev_alloc(64, B->stream);
    f->configured = f->fin && f->out8;
    return f->configured;
}

bool batch_load_host(Batch* B, int i, const u64* v_re, const u64* v_im, const u64* b_re,
                     const u64* b_im)
{
    Frame* f = B->frames[(size_t)i];
    cudaStream_t s = B->stream;
    const size_t vn = (size_t)f->n_wires * (size_t)f->n_copies0;
    if (!frame_alloc(f, vn, vn / 2, s)) return false;
    // stage the real limbs in the half-size buffer (exactly vn u64), the
    // imaginary limbs in a temporary, then pack
    u64* stage_re = reinterpret_cast<u64*>(f->buf[1]);
    u64* stage_im = (u64*)dev_alloc(sizeof(u64) * vn, s);
    if (!stage_im) return false;
    int launches = 0;
    bool ok = host_to_device(stage_re, v_re, 8 * vn, s) && host_to_device(stage_im, v_im, 8 * vn, s) &&
              launch_pack(stage_re, stage_im, vn, f->buf[0], s, &launches);
    const size_t n = (size_t)f->n_copies0;
    u64* bst = reinterpret_cast<u64*>(f->beta[1]);  // 16 B x n: room for both limb arrays
    ok = ok && !cuda_failed(cudaMemcpyAsync(bst, b_re, 8 * n, cudaMemcpyHostToDevice, s), "H2D beta") &&
         !cuda_failed(cudaMemcpyAsync(bst + n, b_im, 8 * n, cudaMemcpyHostToDevice, s), "H2D beta") &&
         launch_pack(bst, bst + n, n, f->beta[0], s, &launches);
    B->launches += launches;
    dev_free(stage_im, s);
    // the reference contract: host inputs are consumed before the call returns
    return ok && !cuda_failed(cudaStreamSynchronize(s), "load tables");
}

bool batch_load_device(Batch* B, int i, const fp2* d_values, const fp2* d_beta, bool borrow)
{
    Frame* f = B->frames[(size_t)i];
    cudaStream_t s = B->stream;
    const size_t vn = (size_t)f->n_wires * (size_t)f->n_copies0;
    if (!frame_alloc(f, borrow ? 0 : vn, vn / 2, s)) return false;
    if (borrow) {
        f->buf[0] = const_cast<fp2*>(d_values);
        f->borrowed0 = true;
    } else {
        TP_CUDA_OK(cudaMemcpyAsync(f->buf[0], d_values, sizeof(fp2) * vn, cudaMemcpyDeviceToDevice, s),
                   "copy values");
    }
    TP_CUDA_OK(cudaMemcpyAsync(f->beta[0], d_beta, sizeof(fp2) * (size_t)f->n_copies0,
                               cudaMemcpyDeviceToDevice, s), "copy beta");
    return true;
}

bool batch_load_pixels(Batch* B, int i, const PixSrc& px, const fp2* d_beta)
{
    Frame* f = B->frames[(size_t)i];
    if (!pixsrc_valid(px, f->n_copies0, f->n_wires)) return false;
    cudaStream_t s = B->stream;
    f->px = px;
    f->W_rows = pixsrc_rows(px);
    const size_t C = (size_t)f->n_copies0, R = (size_t)f->W_rows;
    // first fold writes R x C/2 into buf[1]; later folds alternate with buf[0]
    if (!frame_alloc(f, R * std::max<size_t>(1, C / 4), R * (C / 2), s)) return false;
    f->pix_cur = true;
    if (px.const_idx >= 0) f->Lc = f2scale(f->L_host[(size_t)px.const_idx], px.const_val);
    TP_CUDA_OK(cudaMemcpyAsync(f->beta[0], d_beta, sizeof(fp2) * C, cudaMemcpyDeviceToDevice, s),
               "copy beta");
    return true;
}

bool batch_claim(Batch* B, u64* const* d_claims)
{
    Ctx* c = ctx();
    if (!c) return false;
    std::vector<Job> by_kind[4];
    std::vector<Frame*> fr[4];
    for (size_t i = 0; i < B->frames.size(); ++i) {
        Frame* f = B->frames[i];
        if (!f->configured) continue;
        if (!f->buf[1]) {
            set_error(TP_ERR_ARG, "frame %zu has no table", i);
            return false;
        }
        if (f->n_copies < 2) continue;
        Job j = base_job(f);
        j.kind = (f->pix_cur ? 2 : 0) + (f->pending ? 1 : 0);
        if (f->pending) {
            const int nxt = f->pix_cur ? 1 : (f->cur ^ 1);
            j.Aout = f->buf[nxt];
            j.beta_out = f->beta[nxt];
        }
        j.n_pairs = f->n_copies / 2;
        j.out8 = (d_claims && d_claims[i]) ? d_claims[i] : f->out8;
        by_kind[j.kind].push_back(j);
        fr[j.kind].push_back(f);
    }
    if (B->frames.size() == 1 && by_kind[0].empty() && by_kind[1].empty() && by_kind[2].empty() &&
        by_kind[3].empty()) {
        set_error(TP_ERR_ARG, "claim needs at least 2 copies (have %d)", B->frames[0]->n_copies);
        return false;
    }
    const int target = 4 * c->n_sm;
    for (int k = 0; k < 4; ++k) {
        std::vector<Job>& jobs = by_kind[k];
        if (jobs.empty()) continue;
        double total = 0;
        for (const Job& j : jobs) total += (double)j.n_pairs * (k < 2 ? j.W_rows : j.cs);
        int cta = 0;
        for (size_t q = 0; q < jobs.size(); ++q) {
            Job& j = jobs[q];
            const double w = (double)j.n_pairs * (k < 2 ? j.W_rows : j.cs);
            plan_job(j, std::max(1, (int)(target * w / total + 0.5)));
            j.cta0 = cta;
            cta += j.tiles * j.groups;
        }
        if (!ensure_workspace(B, jobs.size(), (size_t)cta)) return false;
        for (size_t q = 0; q < jobs.size(); ++q) {
            jobs[q].partials = B->partials + 4 * (size_t)jobs[q].cta0;
            jobs[q].ticket = B->tickets + q;
        }
        std::vector<const fp2*> rdev(jobs.size(), nullptr);
        for (size_t q = 0; q < jobs.size(); ++q)
            if (fr[k][q]->pending) rdev[q] = fr[k][q]->r_dev;
        if (!upload_jobs(B, jobs.data(), jobs.size(), rdev)) return false;
        int lg = 0;
        while ((1 << lg) < 2 * jobs[0].n_pairs) ++lg;
        timer_begin(B->stream, 1000 * (k >> 1) + 100 * (k & 1) + lg);
        const bool ok = launch_round(B->d_jobs, jobs, k, B->stream, &B->launches);
        timer_end(B->stream);
        if (!ok) return false;
        for (Frame* f : fr[k]) {
            if (f->pending) {
                f->cur = f->pix_cur ? 1 : (f->cur ^ 1);
                f->pix_cur = false;
                f->n_phys >>= 1;
                f->pending = false;
                f->r_dev = nullptr;
            }
        }
    }
    return true;
}

bool batch_fold(Batch* B, int i, fp2 r)
{
    if (i < 0 || i >= (int)B->frames.size()) {
        set_error(TP_ERR_ARG, "frame index %d outside the batch", i);
        return false;
    }
    Frame* f = B->frames[(size_t)i];
    if (f->n_copies < 2) {
        set_error(TP_ERR_ARG, "fold needs at least 2 copies (have %d)", f->n_copies);
        return false;
    }
    if (r.re >= P61 || r.im >= P61) {
        set_error(TP_ERR_ARG, "fold challenge is not a canonical field element");
        return false;
    }
    if (device_fold_blocked(f)) return false;
    if (f->pending && !apply_fold(f, B->stream, &B->launches)) return false;
    f->pending = true;
    f->r = r;
    f->r_dev = nullptr;
    f->n_copies >>= 1;
    return true;
}

bool batch_fold_dev(Batch* B, int i, const fp2* d_r)
{
    if (i < 0 || i >= (int)B->frames.size()) {
        set_error(TP_ERR_ARG, "frame index %d outside the batch", i);
        return false;
    }
    Frame* f = B->frames[(size_t)i];
    if (f->n_copies < 2) {
        set_error(TP_ERR_ARG, "fold needs at least 2 copies (have %d)", f->n_copies);
        return false;
    }
    if (!d_r) {
        set_error(TP_ERR_ARG, "null device challenge");
        return false;
    }
    if (f->pending) {
        set_error(TP_ERR_ARG, "a fold with a device challenge needs a claim or finish after the previous fold");
        return false;
    }
    f->pending = true;
    f->r = f2zero();
    f->r_dev = d_r;
    f->n_copies >>= 1;
    return true;
}

bool batch_finish(Batch* B, fp2* const* d_wires, fp2* const* d_beta)
{
    std::vector<Job> jobs;
    std::vector<const fp2*> rdev;
    int max_w = 0;
    for (size_t i = 0; i < B->frames.size(); ++i) {
        Frame* f = B->frames[i];
        if (!f->configured) continue;
        if (!f->buf[1]) {
            set_error(TP_ERR_ARG, "frame %zu has no table", i);
            return false;
        }
        if (f->pending && f->n_phys > 2 && (device_fold_blocked(f) || !apply_fold(f, B->stream, &B->launches)))
            return false;
        Job j = base_job(f);
        j.kind = f->pending ? 1 : 0;  // a pending fold of the last two copies
        j.fin = (d_wires && d_wires[i]) ? d_wires[i] : f->fin;
        j.fin_beta = (d_beta && d_beta[i]) ? d_beta[i] : f->fin + f->n_wires;
        max_w = std::max(max_w, f->n_wires);
        jobs.push_back(j);
        rdev.push_back(f->pending ? f->r_dev : nullptr);
    }
    if (!ensure_workspace(B, jobs.size(), 1)) return false;
    if (!upload_jobs(B, jobs.data(), jobs.size(), rdev)) return false;
    return launch_finish(B->d_jobs, (int)jobs.size(), max_w, B->stream, &B->launches);
}

bool batch_finish_frame(Batch* B, int i, fp2* d_wires, fp2* d_beta)
{
    if (i < 0 || i >= (int)B->frames.size()) {
        set_error(TP_ERR_ARG, "frame index %d outside the batch", i);
        return false;
    }
    Frame* f = B->frames[(size_t)i];
    if (!f->configured || !f->buf[1]) {
        set_error(TP_ERR_ARG, "frame %d is not configured", i);
        return false;
    }
    if (f->pending && f->n_phys > 2 && (device_fold_blocked(f) || !apply_fold(f, B->stream, &B->launches)))
        return false;
    Job j = base_job(f);
    j.kind = f->pending ? 1 : 0;
    j.fin = d_wires ? d_wires : f->fin;
    j.fin_beta = d_beta ? d_beta : f->fin + f->n_wires;
    if (!ensure_workspace(B, 1, 1)) return false;
    if (!upload_jobs(B, &j, 1, std::vector<const fp2*>{f->pending ? f->r_dev : nullptr})) return false;
    if (!launch_finish(B->d_jobs, 1, f->n_wires, B->stream, &B->launches)) return false;
    batch_release(B, i, false);
    return true;
}

void batch_release(Batch* B, int i, bool free_buffers)
{
    if (i < 0 || i >= (int)B->frames.size()) return;
    Frame* f = B->frames[(size_t)i];
    f->configured = false;
    f->n_copies = 0;
    f->pending = false;
    f->r_dev = nullptr;
    if (free_buffers) {
        cudaStream_t s = B->stream;
        if (!f->borrowed0) dev_free(f->buf[0], s);
        dev_free(f->buf[1], s);
        dev_free(f->beta[0], s);
        dev_free(f->beta[1], s);
        f->buf[0] = f->buf[1] = f->beta[0] = f->beta[1] = nullptr;
        f->cap0 = f->cap1 = f->capb = 0;
        f->borrowed0 = false;
    }
}

void batch_reset(Batch* B)
{
    for (Frame* f : B->frames) {
        f->configured = false;
        f->n_copies = 0;
    }
}

void batch_destroy(Batch* B)
{
    if (!B) return;
    cudaStream_t s = B->stream;
    for (Frame* f : B->frames) {
        if (!f->borrowed0) dev_free(f->buf[0], s);
        dev_free(f->buf[1], s);
        dev_free(f->beta[0], s);
        dev_free(f->beta[1], s);
        dev_free(f->fin, s);
        dev_free(f->out8, s);
        free_gate_form(f->form, s);
        delete f;
    }
    dev_free(B->d_jobs, s);
    dev_free(B->partials, s);
    dev_free(B->tickets, s);
    dev_free(B->d_patch, s);
    delete B;
}

Batch* session_create(int n_gates, const int* type, const int* in0, const int* in1,
                      const u64* z_re, const u64* z_im, int n_copies, int n_wires, cudaStream_t s)
{
    Batch* B = batch_create(1, s);
    if (!B) return nullptr;
    if (!batch_set_gates(B, 0, n_gates, type, in0, in1, z_re, z_im, n_copies, n_wires)) {
        batch_destroy(B);
        return nullptr;
    }
    return B;
}

bool session_claim(Batch* B, u64 out8[8])
{
    if (!batch_claim(B, nullptr)) return false;
    TP_CUDA_OK(cudaMemcpyAsync(out8, B->frames[0]->out8, 64, cudaMemcpyDeviceToHost, B->stream),
               "D2H claim");
    TP_CUDA_OK(cudaStreamSynchronize(B->stream), "claim");
    return true;
}

bool session_finish(Batch* B, u64* w_re, u64* w_im, u64* b_re, u64* b_im)
{
    if (!batch_finish(B, nullptr, nullptr)) return false;
    Frame* f = B->frames[0];
    std::vector<fp2> h((size_t)f->n_wires + 1);
    TP_CUDA_OK(cudaMemcpyAsync(h.data(), f->fin, sizeof(fp2) * h.size(), cudaMemcpyDeviceToHost,
                               B->stream), "D2H finish");
    TP_CUDA_OK(cudaStreamSynchronize(B->stream), "finish");
    for (int w = 0; w < f->n_wires; ++w) {
        w_re[w] = h[w].re;
        w_im[w] = h[w].im;
    }
    *b_re = h[f->n_wires].re;
    *b_im = h[f->n_wires].im;
    return true;
}

}  // namespace tp
