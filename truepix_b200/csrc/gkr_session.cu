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
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>

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

namespace {

// ---- round planning ----------------------------------------------------------
// A round launch is planned on the host from the frames' state (which it then
// advances as the launch will), before anything is uploaded: the immediate path
// uploads and launches it at once, the graph path plans every round of a proof
// first and replays them from one device job table.

// work of a launch, for the autotuner's size buckets
int work_bucket(const std::vector<Job>& jobs, int kind)
{
    double total = 0;
    for (const Job& j : jobs) total += (double)j.n_pairs * (kind < 2 ? j.W_rows : j.cs);
    int b = 0;
    while (b < 62 && (double)(1ull << (b + 1)) <= total) ++b;
    return b;
}

// The claim/fold launch split: a round launch of one kind spreads `target` CTAs
// over its jobs in proportion to their work (pair tiles x row groups,
// plan_job). The autotuner measures the target, as CTAs per SM, per (kind, work
// bucket) on the device and keeps the fastest; 4 per SM until it has.
constexpr int kTuneMults[] = {2, 3, 4, 6, 8, 12, 16};

// one planned launch: a round kind (0..3) or the finish (kind 4)
struct RoundLaunch {
    int kind = 0;
    std::vector<Job> jobs;
    std::vector<const fp2*> rdev;   // per job: the device challenge patched into it, or null
    int bucket = 0;
    int timer_tag = 0;
    int max_w = 0;                  // finish: the widest frame
};

struct TuneKey {
    int device, kind, bucket;
    bool operator<(const TuneKey& o) const
    {
        return device != o.device ? device < o.device : kind != o.kind ? kind < o.kind : bucket < o.bucket;
    }
};
std::map<TuneKey, int>& tune_table()
{
    static std::map<TuneKey, int> t;
    return t;
}
std::mutex& tune_mutex()
{
    static std::mutex m;
    return m;
}
bool g_tune_on = false;

bool tune_known(int kind, int bucket)
{
    Ctx* c = ctx();
    std::lock_guard<std::mutex> lk(tune_mutex());
    return tune_table().count(TuneKey{c ? c->device : 0, kind, bucket}) != 0;
}

int tuned_mult(int kind, int bucket)
{
    Ctx* c = ctx();
    std::lock_guard<std::mutex> lk(tune_mutex());
    auto it = tune_table().find(TuneKey{c ? c->device : 0, kind, bucket});
    return it == tune_table().end() ? 4 : it->second;
}

void plan_jobs(std::vector<Job>& jobs, int kind, int target)
{
    double total = 0;
    for (const Job& j : jobs) total += (double)j.n_pairs * (kind < 2 ? j.W_rows : j.cs);
    int cta = 0;
    for (Job& j : jobs) {
        const double w = (double)j.n_pairs * (kind < 2 ? j.W_rows : j.cs);
        plan_job(j, std::max(1, (int)(target * w / total + 0.5)));
        j.cta0 = cta;
        cta += j.tiles * j.groups;
    }
}

size_t launch_ctas(const std::vector<Job>& jobs)
{
    size_t n = 0;
    for (const Job& j : jobs) n += (size_t)j.tiles * j.groups;
    return n;
}

void set_workspace_ptrs(Batch* B, std::vector<Job>& jobs)
{
    for (size_t q = 0; q < jobs.size(); ++q) {
        jobs[q].partials = B->partials + 4 * (size_t)jobs[q].cta0;
        jobs[q].ticket = B->tickets + q;
    }
}

// the claim launches of one round: per kind, its jobs and the device challenges
// of their pending folds; advances the frames past the round's folds
bool plan_claims(Batch* B, u64* const* d_claims, std::vector<RoundLaunch>& out)
{
    Ctx* c = ctx();
    if (!c) return false;
    RoundLaunch by_kind[4];
    std::vector<Frame*> fr[4];
    for (int k = 0; k < 4; ++k) by_kind[k].kind = k;
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
        by_kind[j.kind].jobs.push_back(j);
        by_kind[j.kind].rdev.push_back(f->pending ? f->r_dev : nullptr);
        fr[j.kind].push_back(f);
    }
    if (B->frames.size() == 1 && by_kind[0].jobs.empty() && by_kind[1].jobs.empty() && by_kind[2].jobs.empty() &&
        by_kind[3].jobs.empty()) {
        set_error(TP_ERR_ARG, "claim needs at least 2 copies (have %d)", B->frames[0]->n_copies);
        return false;
    }
    for (int k = 0; k < 4; ++k) {
        RoundLaunch& L = by_kind[k];
        if (L.jobs.empty()) continue;
        L.bucket = work_bucket(L.jobs, k);
        plan_jobs(L.jobs, k, tuned_mult(k, L.bucket) * c->n_sm);
        int lg = 0;
        while ((1 << lg) < 2 * L.jobs[0].n_pairs) ++lg;
        L.timer_tag = 1000 * (k >> 1) + 100 * (k & 1) + lg;
        for (Frame* f : fr[k]) {
            if (f->pending) {
                f->cur = f->pix_cur ? 1 : (f->cur ^ 1);
                f->pix_cur = false;
                f->n_phys >>= 1;
                f->pending = false;
                f->r_dev = nullptr;
            }
        }
        out.push_back(std::move(L));
    }
    return true;
}

// time one round launch under each candidate split, keep the fastest for its
// (kind, bucket); the launches rerun the same jobs (a claim or fold + claim
// reads its source and rewrites the same outputs)
bool tune_launch(Batch* B, RoundLaunch& L)
{
    Ctx* c = ctx();
    cudaStream_t s = B->stream;
    float best_ms = 0;
    int best = 4;
    cudaEvent_t e0, e1;
    TP_CUDA_OK(cudaEventCreate(&e0), "tune event");
    TP_CUDA_OK(cudaEventCreate(&e1), "tune event");
    bool ok = true;
    for (int mult : kTuneMults) {
        std::vector<Job> jobs = L.jobs;
        plan_jobs(jobs, L.kind, mult * c->n_sm);
        if (!ensure_workspace(B, jobs.size(), launch_ctas(jobs))) {
            ok = false;
            break;
        }
        set_workspace_ptrs(B, jobs);
        if (!upload_jobs(B, jobs.data(), jobs.size(), L.rdev)) {
            ok = false;
            break;
        }
        int dummy = 0;
        ok = launch_round(B->d_jobs, jobs, L.kind, s, &dummy);   // warm
        ok = ok && !cuda_failed(cudaEventRecord(e0, s), "tune event");
        for (int rep = 0; ok && rep < 3; ++rep) ok = launch_round(B->d_jobs, jobs, L.kind, s, &dummy);
        ok = ok && !cuda_failed(cudaEventRecord(e1, s), "tune event") &&
             !cuda_failed(cudaEventSynchronize(e1), "tune sync");
        if (!ok) break;
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        if (best_ms == 0 || ms < best_ms) {
            best_ms = ms;
            best = mult;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (!ok) return false;
    {
        std::lock_guard<std::mutex> lk(tune_mutex());
        tune_table()[TuneKey{c->device, L.kind, L.bucket}] = best;
    }
    plan_jobs(L.jobs, L.kind, best * c->n_sm);
    return true;
}

bool launch_planned(Batch* B, RoundLaunch& L)
{
    if (g_tune_on && !tune_known(L.kind, L.bucket) && !tune_launch(B, L)) return false;
    if (!ensure_workspace(B, L.jobs.size(), launch_ctas(L.jobs))) return false;
    set_workspace_ptrs(B, L.jobs);
    if (!upload_jobs(B, L.jobs.data(), L.jobs.size(), L.rdev)) return false;
    timer_begin(B->stream, L.timer_tag);
    const bool ok = launch_round(B->d_jobs, L.jobs, L.kind, B->stream, &B->launches);
    timer_end(B->stream);
    return ok;
}

}  // namespace

bool batch_claim(Batch* B, u64* const* d_claims)
{
    std::vector<RoundLaunch> plan;
    if (!plan_claims(B, d_claims, plan)) return false;
    for (RoundLaunch& L : plan)
        if (!launch_planned(B, L)) return false;
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

namespace {

// the finish launch: wires and beta of every configured frame (a pending fold of
// the last two copies applied by it); a pending fold of more copies is applied
// first (host challenges only)
bool plan_finish(Batch* B, fp2* const* d_wires, fp2* const* d_beta, RoundLaunch& L)
{
    L.kind = 4;
    L.max_w = 0;
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
        L.max_w = std::max(L.max_w, f->n_wires);
        L.jobs.push_back(j);
        L.rdev.push_back(f->pending ? f->r_dev : nullptr);
    }
    return true;
}

}  // namespace

bool batch_finish(Batch* B, fp2* const* d_wires, fp2* const* d_beta)
{
    RoundLaunch L;
    if (!plan_finish(B, d_wires, d_beta, L)) return false;
    if (!ensure_workspace(B, L.jobs.size(), 1)) return false;
    if (!upload_jobs(B, L.jobs.data(), L.jobs.size(), L.rdev)) return false;
    return launch_finish(B->d_jobs, (int)L.jobs.size(), L.max_w, B->stream, &B->launches);
}

namespace {

struct GraphOp {
    int type = 0;          // 0 round launch, 1 VOLE round, 2 finish
    RoundLaunch L;
    size_t job_off = 0, patch_off = 0, n_patch = 0;
    int round = 0;
};

template <class T>
bool grow_dev(T*& p, size_t& cap, size_t n, cudaStream_t s)
{
    if (n <= cap) return true;
    dev_free(p, s);
    cap = std::max(n, cap * 2);
    p = static_cast<T*>(dev_alloc(sizeof(T) * cap, s));
    if (!p) cap = 0;
    return p != nullptr;
}

}  // namespace

bool batch_vole_rounds_graph(Batch* B, u64* d_claims, void* d_states, void* d_vole_states, const fp2* d_u,
                             const fp2* d_v, long long count, int layer, fp2* d_chal, fp2* d_proof,
                             fp2* const* d_wires, fp2* const* d_beta)
{
    Ctx* c = ctx();
    if (!c) return false;
    cudaStream_t s = B->stream;
    if (!s) {
        set_error(TP_ERR_ARG, "the graph path needs a stream of the caller's (the legacy stream cannot capture)");
        return false;
    }
    const int nB = (int)B->frames.size();
    // rounds per frame; frames of different sizes (uneven batches) leave the
    // round loop after their own last round: their VOLE round is skipped (the
    // frame's entry in a device array of rounds) and they get no more claims
    int rounds = 0;
    bool uneven = false;
    std::vector<int> fr_rounds((size_t)nB);
    for (int i = 0; i < nB; ++i) {
        Frame* f = B->frames[(size_t)i];
        if (!f->configured || f->n_copies < 2) {
            set_error(TP_ERR_ARG, "every frame of the batch needs at least one round");
            return false;
        }
        int r = 0;
        while ((2 << r) <= f->n_copies) ++r;
        fr_rounds[(size_t)i] = r;
        if (i && r != rounds) uneven = true;
        rounds = std::max(rounds, r);
    }
    // ---- plan every launch (advances the frames as the launches will)
    std::vector<GraphOp> ops;
    std::vector<u64*> claim_ptrs((size_t)nB);
    for (int k = 0; k < rounds; ++k) {
        for (int i = 0; i < nB; ++i) claim_ptrs[(size_t)i] = d_claims + 8 * ((size_t)nB * k + i);
        std::vector<RoundLaunch> plan;
        if (!plan_claims(B, claim_ptrs.data(), plan)) return false;
        for (RoundLaunch& L : plan) {
            GraphOp op;
            op.type = 0;
            op.L = std::move(L);
            ops.push_back(std::move(op));
        }
        GraphOp v;
        v.type = 1;
        v.round = k;
        ops.push_back(v);
        for (int i = 0; i < nB; ++i)
            if (k < fr_rounds[(size_t)i] && !batch_fold_dev(B, i, d_chal + (size_t)nB * k + i)) return false;
    }
    {
        GraphOp fin;
        fin.type = 2;
        if (!plan_finish(B, d_wires, d_beta, fin.L)) return false;
        ops.push_back(std::move(fin));
    }
    // ---- workspace, one job table and one patch table
    size_t max_jobs = 1, max_ctas = 1, n_jobs = 0, n_patch = 0;
    for (GraphOp& op : ops) {
        if (op.type == 1) continue;
        max_jobs = std::max(max_jobs, op.L.jobs.size());
        if (op.type == 0) max_ctas = std::max(max_ctas, launch_ctas(op.L.jobs));
    }
    if (!ensure_workspace(B, max_jobs, max_ctas)) return false;
    for (GraphOp& op : ops) {
        if (op.type == 1) continue;
        if (op.type == 0) set_workspace_ptrs(B, op.L.jobs);
        op.job_off = n_jobs;
        op.patch_off = n_patch;
        for (const fp2* r : op.L.rdev) op.n_patch += r ? 1 : 0;
        n_jobs += op.L.jobs.size();
        n_patch += op.n_patch;
    }
    struct Patch {
        const fp2* r;
        long long job;
    };
    static_assert(sizeof(Patch) == 16, "patch layout (patch_r_kernel's RPatch)");
    // the patch table, then (uneven batches) the rounds of each frame
    const size_t bytes_jobs = sizeof(Job) * n_jobs, bytes_patch_only = sizeof(Patch) * std::max<size_t>(1, n_patch);
    const size_t bytes_patch = bytes_patch_only + (uneven ? sizeof(int) * (size_t)nB : 0);
    if (!grow_dev(B->d_table, B->cap_table, n_jobs, s)) return false;
    {
        unsigned char* pt = static_cast<unsigned char*>(B->d_ptable);
        size_t cap = B->cap_ptable;
        if (!grow_dev(pt, cap, bytes_patch, s)) return false;
        B->d_ptable = pt;
        B->cap_ptable = cap;
    }
    if (!B->staged) TP_CUDA_OK(cudaEventCreateWithFlags(&B->staged, cudaEventDisableTiming), "stage event");
    TP_CUDA_OK(cudaEventSynchronize(B->staged), "stage reuse");   // the previous upload has read the stage
    if (bytes_jobs + bytes_patch > B->cap_stage) {
        if (B->h_stage) cudaFreeHost(B->h_stage);
        B->cap_stage = std::max(bytes_jobs + bytes_patch, 2 * B->cap_stage);
        if (cuda_failed(cudaMallocHost(&B->h_stage, B->cap_stage), "pinned stage")) {
            B->h_stage = nullptr;
            B->cap_stage = 0;
            return false;
        }
    }
    Job* hj = static_cast<Job*>(B->h_stage);
    Patch* hp = reinterpret_cast<Patch*>(static_cast<unsigned char*>(B->h_stage) + bytes_jobs);
    for (const GraphOp& op : ops) {
        if (op.type == 1) continue;
        std::memcpy(hj + op.job_off, op.L.jobs.data(), sizeof(Job) * op.L.jobs.size());
        size_t q = op.patch_off;
        for (size_t j = 0; j < op.L.rdev.size(); ++j)
            if (op.L.rdev[j]) hp[q++] = Patch{op.L.rdev[j], (long long)(op.job_off + j)};
    }
    int* d_rounds = nullptr;
    if (uneven) {
        std::memcpy(reinterpret_cast<unsigned char*>(hp) + bytes_patch_only, fr_rounds.data(), sizeof(int) * (size_t)nB);
        d_rounds = reinterpret_cast<int*>(static_cast<unsigned char*>(B->d_ptable) + bytes_patch_only);
    }
    TP_CUDA_OK(cudaMemcpyAsync(B->d_table, hj, bytes_jobs, cudaMemcpyHostToDevice, s), "job table");
    if (n_patch || uneven)
        TP_CUDA_OK(cudaMemcpyAsync(B->d_ptable, hp, bytes_patch, cudaMemcpyHostToDevice, s), "patch table");
    TP_CUDA_OK(cudaEventRecord(B->staged, s), "stage event");
    // ---- the graph: captured once per shape, replayed after
    std::vector<long long> key = {(long long)(size_t)s, (long long)(size_t)B->d_table, (long long)(size_t)B->d_ptable,
                                  (long long)(size_t)d_states, (long long)(size_t)d_vole_states,
                                  (long long)(size_t)d_u, (long long)(size_t)d_v, count, layer,
                                  (long long)(size_t)d_chal, (long long)(size_t)d_proof, (long long)nB,
                                  (long long)uneven};
    int kernels = 0;
    for (const GraphOp& op : ops) {
        key.push_back(op.type);
        key.push_back(op.L.kind);
        key.push_back((long long)op.job_off);
        key.push_back((long long)op.L.jobs.size());
        key.push_back((long long)op.patch_off);
        key.push_back((long long)op.n_patch);
        key.push_back(op.L.max_w);
        for (const Job& j : op.L.jobs) {
            key.push_back(j.tiles);
            key.push_back(j.groups);
            key.push_back(j.wpg);
            key.push_back(j.pw);
        }
        kernels += (op.type == 1) ? 1 : 1 + (op.n_patch ? 1 : 0);
    }
    if (!B->graph || key != B->graph_key) {
        if (B->graph) {
            cudaGraphExecDestroy(B->graph);
            B->graph = nullptr;
        }
        if (!prepare_round_kernels()) return false;
        TP_CUDA_OK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal), "begin capture");
        bool ok = true;
        int dummy = 0;
        for (const GraphOp& op : ops) {
            if (!ok) break;
            if (op.type == 1) {
                char label[40];
                std::snprintf(label, sizeof(label), "sc-%d-%d", layer, op.round);
                ok = launch_vole_round_batch(d_states, d_vole_states, nB, d_claims + 8 * (size_t)nB * op.round,
                                             d_u, d_v, count, label, d_chal + (size_t)nB * op.round,
                                             d_proof ? d_proof + 5 * (size_t)nB * op.round : nullptr, s, d_rounds,
                                             op.round);
                continue;
            }
            if (op.n_patch) {
                patch_r_kernel<<<(unsigned)((op.n_patch + 127) / 128), 128, 0, s>>>(
                    B->d_table, static_cast<const RPatch*>(B->d_ptable) + op.patch_off, (int)op.n_patch);
                ok = !cuda_failed(cudaGetLastError(), "challenge patch");
            }
            if (!ok) break;
            if (op.type == 0)
                ok = launch_round(B->d_table + op.job_off, op.L.jobs, op.L.kind, s, &dummy);
            else
                ok = launch_finish(B->d_table + op.job_off, (int)op.L.jobs.size(), op.L.max_w, s, &dummy);
        }
        cudaGraph_t g = nullptr;
        const cudaError_t e = cudaStreamEndCapture(s, &g);
        if (!ok || cuda_failed(e, "end capture")) {
            if (g) cudaGraphDestroy(g);
            return false;
        }
        const cudaError_t ie = cudaGraphInstantiate(&B->graph, g, 0);
        cudaGraphDestroy(g);
        if (cuda_failed(ie, "graph instantiate")) {
            B->graph = nullptr;
            return false;
        }
        B->graph_key = key;
        B->graph_kernels = kernels;
    }
    TP_CUDA_OK(cudaGraphLaunch(B->graph, s), "graph launch");
    B->launches += B->graph_kernels;
    ++B->graph_replays;
    return true;
}

void batch_tune_enable(bool on) { g_tune_on = on; }

int batch_tune_table(int* kind, int* bucket, int* ctas_per_sm, int max)
{
    Ctx* c = ctx();
    std::lock_guard<std::mutex> lk(tune_mutex());
    int n = 0;
    for (const auto& kv : tune_table()) {
        if (c && kv.first.device != c->device) continue;
        if (n < max) {
            kind[n] = kv.first.kind;
            bucket[n] = kv.first.bucket;
            ctas_per_sm[n] = kv.second;
        }
        ++n;
    }
    return n;
}

bool batch_tune_set(int kind, int bucket, int ctas_per_sm)
{
    Ctx* c = ctx();
    if (!c) return false;
    if (kind < 0 || kind > 3 || bucket < 0 || bucket > 62 || ctas_per_sm < 1 || ctas_per_sm > 64) {
        set_error(TP_ERR_ARG, "tune entry (%d, %d, %d) out of range", kind, bucket, ctas_per_sm);
        return false;
    }
    std::lock_guard<std::mutex> lk(tune_mutex());
    tune_table()[TuneKey{c->device, kind, bucket}] = ctas_per_sm;
    return true;
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
    dev_free(B->d_table, s);
    dev_free(B->d_ptable, s);
    if (B->graph) cudaGraphExecDestroy(B->graph);
    if (B->staged) {
        cudaEventSynchronize(B->staged);
        cudaEventDestroy(B->staged);
    }
    if (B->h_stage) cudaFreeHost(B->h_stage);
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
