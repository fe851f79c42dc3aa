// ensemble.cu — batched PM steps over many boxes (C-ABI hgpm_ens_*).
//
// An ensemble holds size classes; a class is nslots boxes of one (ng, np)
// whose particle state, density accumulator, spectra and force grids live in
// slabs with a fixed per-slot stride.  One batched step launches each phase
// of the step ONCE per class, every launch covering all slots of the class
// (the slot is a grid dimension; idle slots' CTAs return at once), so a
// class of 32 small boxes costs the launches of one box and fills the GPU.
// Classes run on their own streams (forked from and joined to the ensemble
// stream), and the whole step can be captured in one CUDA graph.
//
// Each slot runs its own time line: hgpm_ens_start precomputes the slot's
// kick/drift scalars for every step (the host FP64 time stepper, exactly as
// hgpm_run_steps advances it) into a device table, and a per-slot step
// counter on the device selects the row; a slot that has run its steps goes
// idle by itself.  A slot is also a regular context (a "view"): ICs, state
// I/O and P(k) of one box go through the single-box C-ABI on it.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "hgpm_ctx.h"
#include "multi_class.h"

namespace {

struct EnsClass {
    int ng = 0, np = 0, nslots = 0, zs = 0, zs_np = 0, blk = 8;
    size_t ncell = 0, npart = 0, spec_elems = 0, force_elems = 0, part_stride = 0;
    void* slab = nullptr;      // one allocation: particles, rho64, spectra, force grids
    void* part_block = nullptr;
    unsigned long long* rho64 = nullptr;
    float2* spec = nullptr;
    float2* fspec = nullptr;
    float* force = nullptr;
    float2* tw_ng = nullptr;
    float2* tw_np = nullptr;
    double* cosq = nullptr;
    float* sk = nullptr;
    float* pkw = nullptr;
    int* d_err = nullptr;
    int* d_active = nullptr;   // [nslots] 1 while the slot has steps to run
    int* d_step = nullptr;     // [nslots] steps done
    int* d_nsteps = nullptr;   // [nslots]
    float4* d_sched = nullptr; // [nslots][HGPM_MAX_STEPS]
    int* blkwin = nullptr;     // [nslots][window_records] per-block CIC windows
    size_t win_stride = 0;
    int* spill = nullptr;      // counters [4][nslots], then queues [2][nslots][nblocks]
    SpillList dep_spill, kick_spill;
    int* h_mirror = nullptr;   // pinned: active[nslots], step[nslots], start staging
    float4* h_sched = nullptr; // pinned: one schedule row per slot
    // scratch the slot views share (their calls are ordered on one stream)
    float* stage = nullptr;
    double* pk_part = nullptr;
    unsigned long long* pk_pcnt = nullptr;
    double* pk_sum = nullptr;
    unsigned long long* pk_cnt = nullptr;
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr;     // after the class's last step queued by hgpm_ens_step_class
    cudaEvent_t join = nullptr;     // joins the class back in hgpm_ens_step (also inside its graph)
    cudaEvent_t setup = nullptr;    // slot set-up on the ensemble stream before hgpm_ens_step_class
    cudaGraphExec_t exec = nullptr; // one step of this class alone (hgpm_ens_step_class)
    std::vector<hgpm_ctx*> views;
    std::vector<int> in_use;   // host: slot started and not released
};

}  // namespace

struct hgpm_ensemble {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t fork = nullptr;
    std::vector<EnsClass> cls;
    bool use_graph = false;
    cudaGraphExec_t exec = nullptr;
    int kick_choice = 0;   // kick and deposit candidates (HGPM_KICK / HGPM_DEPOSIT)
    int dep_choice = -1;
    // hgpm_ens_step as one launch per phase across all classes (multi_class.h)
    // when every class is supported; else one launch per phase per class
    bool multi = true;
    int64_t launches = 0;
    std::string err;
};

static int efail(hgpm_ensemble* e, int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    if (e) e->err = buf;
    return code;
}

#define ECK(call)                                                                                        \
    do {                                                                                                 \
        cudaError_t e_ = (call);                                                                         \
        if (e_ != cudaSuccess)                                                                           \
            return efail(E, e_ == cudaErrorMemoryAllocation ? HGPM_ERR_OOM : HGPM_ERR_CUDA, "%s failed: %s (%s:%d)", \
                         #call, cudaGetErrorString(e_), __FILE__, __LINE__);                             \
    } while (0)

static int even16(int v) { return (v + 15) / 16 * 16; }

static void class_geometry(EnsClass& k) {
    k.ncell = (size_t)k.ng * k.ng * k.ng;
    k.npart = (size_t)k.np * k.np * k.np;
    k.zs = even16(k.ng / 2 + 1);
    k.zs_np = even16(k.np / 2 + 1);
    k.blk = block_side(k.np, k.ng);
    // per-slot sizes as a single context sizes them (runtime.cu hgpm_create);
    // strides rounded to 64 elements so every slot starts 256-byte aligned
    auto r64 = [](size_t v) { return (v + 63) / 64 * 64; };
    k.spec_elems = r64(std::max((size_t)k.ng * k.ng * k.zs, (size_t)k.np * k.np * k.zs_np));
    k.force_elems = r64(4 * std::max(k.ncell, k.npart));  // float4 grid; ICs use 3 planes of npart
    k.part_stride = r64(k.npart);
}

extern "C" size_t hgpm_ens_footprint_bytes(int ng, int np, int nslots) {
    EnsClass k;
    k.ng = ng;
    k.np = np;
    class_geometry(k);
    size_t per = k.part_stride * 7 * 4 + k.ncell * 8 + k.spec_elems * 8 * 4 + k.force_elems * 4 +
                 (size_t)window_records(np, ng) * 4;
    const size_t shared = k.npart * 6 * 4 + (size_t)(4 * 148 + 1) * 1024 * 16 + (size_t)ng * 64;
    return per * (size_t)nslots + (size_t)nslots * (HGPM_MAX_STEPS * 16 + 64) + shared;
}

static std::vector<float2> twiddle_table(int n) {
    std::vector<float2> t(n);
    for (int m = 0; m < n; ++m) {
        double ang = -2.0 * M_PI * (double)m / (double)n;
        t[m] = make_float2((float)cos(ang), (float)sin(ang));
    }
    return t;
}

static int make_class(hgpm_ensemble* E, EnsClass& k, int priority) {
    class_geometry(k);
    const size_t S = (size_t)k.nslots;
    ECK(cudaStreamCreateWithPriority(&k.stream, cudaStreamNonBlocking, priority));
    ECK(cudaEventCreateWithFlags(&k.done, cudaEventDisableTiming));
    ECK(cudaEventCreateWithFlags(&k.join, cudaEventDisableTiming));
    ECK(cudaEventCreateWithFlags(&k.setup, cudaEventDisableTiming));
    {
        auto a256 = [](size_t v) { return (v + 255) / 256 * 256; };
        const size_t b_part = a256(k.part_stride * 7 * 4 * S), b_rho = a256(k.ncell * 8 * S);
        const size_t b_spec = a256(k.spec_elems * 8 * S), b_fspec = a256(3 * k.spec_elems * 8 * S);
        const size_t b_force = a256(k.force_elems * 4 * S);
        ECK(cudaMalloc(&k.slab, b_part + b_rho + b_spec + b_fspec + b_force));
        char* q = (char*)k.slab;
        k.part_block = q;
        k.rho64 = (unsigned long long*)(q + b_part);
        k.spec = (float2*)(q + b_part + b_rho);
        k.fspec = (float2*)(q + b_part + b_rho + b_spec);
        k.force = (float*)(q + b_part + b_rho + b_spec + b_fspec);
    }
    ECK(cudaMemsetAsync(k.rho64, 0, k.ncell * 8 * S, E->stream));
    ECK(cudaMalloc(&k.stage, k.npart * 6 * sizeof(float)));
    {
        const int nparts = 4 * 148;
        ECK(cudaMalloc(&k.pk_part, (size_t)nparts * pk_max_bins() * 8));
        ECK(cudaMalloc(&k.pk_pcnt, (size_t)nparts * pk_max_bins() * 8));
        ECK(cudaMalloc(&k.pk_sum, pk_max_bins() * 8));
        ECK(cudaMalloc(&k.pk_cnt, pk_max_bins() * 8));
    }
    ECK(cudaMalloc(&k.tw_ng, k.ng * 8));
    ECK(cudaMalloc(&k.tw_np, k.np * 8));
    ECK(cudaMalloc(&k.cosq, k.ng * 8));
    ECK(cudaMalloc(&k.sk, k.ng * 4));
    ECK(cudaMalloc(&k.pkw, k.ng * 4));
    ECK(cudaMalloc(&k.d_err, 8));
    ECK(cudaMemsetAsync(k.d_err, 0, 8, E->stream));
    ECK(cudaMalloc(&k.d_active, 4 * S));
    ECK(cudaMalloc(&k.d_step, 4 * S));
    ECK(cudaMalloc(&k.d_nsteps, 4 * S));
    ECK(cudaMemsetAsync(k.d_active, 0, 4 * S, E->stream));
    ECK(cudaMemsetAsync(k.d_step, 0, 4 * S, E->stream));
    ECK(cudaMemsetAsync(k.d_nsteps, 0, 4 * S, E->stream));
    ECK(cudaMalloc(&k.d_sched, sizeof(float4) * HGPM_MAX_STEPS * S));
    k.win_stride = (size_t)window_records(k.np, k.ng);
    ECK(cudaMalloc(&k.blkwin, k.win_stride * 4 * S));
    {
        const int nblocks = (int)(k.win_stride / 8);
        ECK(cudaMalloc(&k.spill, (4 * S + 2 * S * (size_t)nblocks) * 4));
        // counters: deposit queues, kick queues, blocks over the kick's cap,
        // the kick's work counters
        k.dep_spill = SpillList{k.spill, k.spill + 4 * S, nblocks, k.spill + 2 * S, k.spill + 3 * S};
        k.kick_spill = SpillList{k.spill + S, k.spill + 4 * S + S * (size_t)nblocks, nblocks, k.spill + 2 * S,
                                 k.spill + 3 * S};
    }
    ECK(cudaMallocHost(&k.h_mirror, sizeof(int) * (2 * S + 4 * S)));
    ECK(cudaMallocHost(&k.h_sched, sizeof(float4) * HGPM_MAX_STEPS * S));
    memset(k.h_mirror, 0, sizeof(int) * 6 * S);
    const std::vector<float2> t1 = twiddle_table(k.ng), t2 = twiddle_table(k.np);
    ECK(cudaMemcpy(k.tw_ng, t1.data(), k.ng * 8, cudaMemcpyHostToDevice));
    ECK(cudaMemcpy(k.tw_np, t2.data(), k.np * 8, cudaMemcpyHostToDevice));
    ECK(launch_ktables(k.ng, k.cosq, k.sk, k.pkw, E->stream));
    E->launches += 1;
    ECK(cudaStreamSynchronize(E->stream));
    k.in_use.assign(S, 0);
    k.views.assign(S, nullptr);
    return HGPM_OK;
}

static void free_class(EnsClass& k) {
    for (hgpm_ctx* v : k.views)
        if (v) hgpm_destroy(v);
    void* d[] = {k.slab, k.tw_ng, k.tw_np, k.cosq, k.sk, k.pkw, k.d_err, k.d_active, k.d_step, k.d_nsteps,
                 k.d_sched, k.stage, k.pk_part, k.pk_pcnt, k.pk_sum, k.pk_cnt, k.blkwin, k.spill};
    for (void* q : d)
        if (q) cudaFree(q);
    if (k.h_mirror) cudaFreeHost(k.h_mirror);
    if (k.h_sched) cudaFreeHost(k.h_sched);
    if (k.exec) cudaGraphExecDestroy(k.exec);
    if (k.done) cudaEventDestroy(k.done);
    if (k.join) cudaEventDestroy(k.join);
    if (k.setup) cudaEventDestroy(k.setup);
    if (k.stream) cudaStreamDestroy(k.stream);
}

extern "C" void hgpm_ens_destroy(hgpm_ensemble* E) {
    if (!E) return;
    if (E->stream) cudaStreamSynchronize(E->stream);
    for (auto& k : E->cls)
        if (k.stream) cudaStreamSynchronize(k.stream);
    if (E->exec) cudaGraphExecDestroy(E->exec);
    for (auto& k : E->cls) free_class(k);
    if (E->fork) cudaEventDestroy(E->fork);
    if (E->stream) cudaStreamDestroy(E->stream);
    delete E;
}

extern "C" int hgpm_ens_create(int nclass, const int* ng, const int* np, const int* nslots, int device,
                               hgpm_ensemble** out) {
    if (!out || nclass <= 0 || !ng || !np || !nslots) return HGPM_ERR_ARG;
    hgpm_ensemble* E = new hgpm_ensemble();
    *out = E;
    E->device = device;
    for (int i = 0; i < nclass; ++i) {
        if (!fft_size_supported(ng[i]) || !fft_size_supported(np[i]))
            return efail(E, HGPM_ERR_ARG, "class %d: NG/NP must be one of " HGPM_SIZES_TEXT, i);
        if (nslots[i] <= 0 || nslots[i] > 65535 / 3) return efail(E, HGPM_ERR_ARG, "class %d: bad slot count", i);
    }
    const char* kv = getenv("HGPM_KICK");
    if (kv && kv[0] >= '0' && kv[0] <= '9' && atoi(kv) < kick_candidates(np[0], ng[0])) E->kick_choice = atoi(kv);
    const char* dv = getenv("HGPM_DEPOSIT");
    if (dv && dv[0] >= '0' && dv[0] <= '9') E->dep_choice = atoi(dv);
    ECK(cudaSetDevice(device));
    ECK(cudaStreamCreateWithFlags(&E->stream, cudaStreamNonBlocking));
    ECK(cudaEventCreateWithFlags(&E->fork, cudaEventDisableTiming));
    E->cls.resize(nclass);
    // stream priority by class size, smaller boxes first: their steps are
    // short, so they finish at close to their own pace while the large
    // classes take the rest of the GPU (serving p50 0.04 s against 0.23 s
    // with equal priorities).  HGPM_ENS_PRIO=n: all equal; l: larger first.
    int least = 0, greatest = 0;
    ECK(cudaDeviceGetStreamPriorityRange(&least, &greatest));
    const char* pv = getenv("HGPM_ENS_PRIO");
    const char mode = pv ? pv[0] : 's';
    for (int i = 0; i < nclass; ++i) {
        EnsClass& k = E->cls[i];
        k.ng = ng[i];
        k.np = np[i];
        k.nslots = nslots[i];
        int rank = 0;  // classes with fewer cells + particles
        const double w = (double)ng[i] * ng[i] * ng[i] + (double)np[i] * np[i] * np[i];
        for (int j = 0; j < nclass; ++j)
            if ((double)ng[j] * ng[j] * ng[j] + (double)np[j] * np[j] * np[j] < w) ++rank;
        int prio = least;
        if (mode == 's') prio = std::max(greatest, least - (nclass - 1 - rank));
        if (mode == 'l') prio = std::max(greatest, least - rank);
        int rc = make_class(E, k, prio);
        if (rc) return rc;
    }
    return HGPM_OK;
}

extern "C" const char* hgpm_ens_last_error(const hgpm_ensemble* E) { return E ? E->err.c_str() : "null ensemble"; }
extern "C" void* hgpm_ens_stream(hgpm_ensemble* E) { return E ? (void*)E->stream : nullptr; }
extern "C" int64_t hgpm_ens_kernel_launches(hgpm_ensemble* E, int reset) {
    if (!E) return 0;
    int64_t n = E->launches;
    for (auto& k : E->cls)
        for (hgpm_ctx* v : k.views)
            if (v) {
                n += v->launches;
                if (reset) v->launches = 0;
            }
    if (reset) E->launches = 0;
    return n;
}

static int check_slot(hgpm_ensemble* E, int ci, int slot) {
    if (!E || ci < 0 || ci >= (int)E->cls.size()) return E ? efail(E, HGPM_ERR_ARG, "no class %d", ci) : HGPM_ERR_ARG;
    if (slot < 0 || slot >= E->cls[ci].nslots) return efail(E, HGPM_ERR_ARG, "class %d has no slot %d", ci, slot);
    return HGPM_OK;
}

extern "C" int hgpm_ens_slot(hgpm_ensemble* E, int ci, int slot, const hgpm_params* p, hgpm_ctx** view) {
    int rc = check_slot(E, ci, slot);
    if (rc) return rc;
    if (!p || !view) return efail(E, HGPM_ERR_ARG, "null params or view");
    EnsClass& k = E->cls[ci];
    if (p->ng != k.ng || p->np != k.np)
        return efail(E, HGPM_ERR_ARG, "params NG %d NP %d do not fit class %d (NG %d NP %d)", p->ng, p->np, ci, k.ng,
                     k.np);
    if (p->rl <= 0) return efail(E, HGPM_ERR_ARG, "RL must be positive");
    if (k.in_use[slot]) return efail(E, HGPM_ERR_STATE, "class %d slot %d is running; release it first", ci, slot);
    hgpm_ctx* c = k.views[slot];
    if (!c) {
        c = new hgpm_ctx();
        c->view = true;
        c->device = E->device;
        c->stream = E->stream;
        c->ng = k.ng;
        c->np = k.np;
        c->zs = k.zs;
        c->zs_np = k.zs_np;
        c->blk = k.blk;
        c->ncell = k.ncell;
        c->npart = k.npart;
        c->nspec = (size_t)k.ng * k.ng * k.zs;
        char* b = (char*)k.part_block;
        const size_t a = k.part_stride * 4 * (size_t)k.nslots;  // bytes per particle array slab
        const size_t o = k.part_stride * 4 * (size_t)slot;
        c->part.cell = (uint32_t*)(b + o);
        c->part.ox = (float*)(b + a + o);
        c->part.oy = (float*)(b + 2 * a + o);
        c->part.oz = (float*)(b + 3 * a + o);
        c->part.vx = (float*)(b + 4 * a + o);
        c->part.vy = (float*)(b + 5 * a + o);
        c->part.vz = (float*)(b + 6 * a + o);
        c->rho64 = k.rho64 + k.ncell * slot;
        c->spec = k.spec + k.spec_elems * slot;
        c->fspec = k.fspec + 3 * k.spec_elems * slot;
        c->force = k.force + k.force_elems * slot;
        c->tw_ng = k.tw_ng;
        c->tw_np = k.tw_np;
        c->cosq = k.cosq;
        c->sk = k.sk;
        c->pkw = k.pkw;
        c->d_err = k.d_err;
        c->blkwin = k.blkwin + k.win_stride * slot;
        c->dep_spill = SpillList{k.dep_spill.cnt + slot, k.dep_spill.items + (size_t)slot * k.dep_spill.nblocks,
                                 k.dep_spill.nblocks, k.dep_spill.over + slot, k.dep_spill.next + slot};
        c->kick_spill = SpillList{k.kick_spill.cnt + slot, k.kick_spill.items + (size_t)slot * k.kick_spill.nblocks,
                                  k.kick_spill.nblocks, k.kick_spill.over + slot, k.kick_spill.next + slot};
        c->stage = k.stage;
        c->pk_part = k.pk_part;
        c->pk_pcnt = k.pk_pcnt;
        c->pk_sum = k.pk_sum;
        c->pk_cnt = k.pk_cnt;
        c->pk_nparts = 4 * 148;
        c->tma = false;  // batched passes are the plain ones; views match them
        c->xmode = 0;
        c->kick_choice = E->kick_choice;
        c->dep_choice = E->dep_choice;
        k.views[slot] = c;
    }
    c->p = *p;
    c->err.clear();
    c->have_state = false;
    c->rho_dirty = false;
    if (!c->p.ref_quirks) {
        // the class tables hold the reference-rounded cos; exact-cos boxes
        // need a class of their own
        return efail(E, HGPM_ERR_ARG, "ensemble slots use the reference-rounded Green's function (ref_quirks = 1)");
    }
    rc = ctx_set_rl_tables(c);
    if (rc) return efail(E, rc, "%s", c->err.c_str());
    *view = c;
    return HGPM_OK;
}

// Start slot `slot` of class ci: it must hold a particle state (ICs or a
// loaded state).  *ts is the time stepper as hgpm_run_steps takes it; on
// return it has advanced through all nsteps, as hgpm_run_steps leaves it.
extern "C" int hgpm_ens_start(hgpm_ensemble* E, int ci, int slot, hgpm_timestepper* ts, int nsteps) {
    int rc = check_slot(E, ci, slot);
    if (rc) return rc;
    EnsClass& k = E->cls[ci];
    hgpm_ctx* c = k.views[slot];
    if (!ts || nsteps <= 0 || nsteps > HGPM_MAX_STEPS) return efail(E, HGPM_ERR_ARG, "nsteps must be in [1, %d]", HGPM_MAX_STEPS);
    if (!c || !c->have_state) return efail(E, HGPM_ERR_STATE, "class %d slot %d holds no particle state", ci, slot);
    if (k.in_use[slot]) return efail(E, HGPM_ERR_STATE, "class %d slot %d is already running", ci, slot);
    // the schedule: the scalars hgpm_run_steps computes, step by step
    float4* row = k.h_sched + (size_t)slot * HGPM_MAX_STEPS;
    const float pf0 = hgpm_ts_drift_prefactor(ts, 0.5f);
    for (int s = 0; s < nsteps; ++s) {
        hgpm_ts_advance_half(ts);
        const double dt = ts->deltaT, fs = ts->fscal;
        hgpm_ts_advance_half(ts);
        const float pf = hgpm_ts_drift_prefactor(ts, 0.5f);
        row[s] = make_float4((float)(dt * fs), pf, pf, s + 1 < nsteps ? 2.f : 1.f);
    }
    int* st = k.h_mirror + 2 * k.nslots + 4 * slot;  // staging for this slot's counters
    // the counters below must not change under a step of this class still
    // queued on its own stream (hgpm_ens_step_class)
    ECK(cudaStreamWaitEvent(E->stream, k.done, 0));
    st[0] = 1;
    st[1] = 0;
    st[2] = nsteps;
    ECK(cudaMemcpyAsync(k.d_sched + (size_t)slot * HGPM_MAX_STEPS, row, sizeof(float4) * nsteps,
                        cudaMemcpyHostToDevice, E->stream));
    // the first drift of the run (driver_pm.cpp:114), on the slot's view
    rc = hgpm_drift(c, pf0);
    if (rc) return efail(E, rc, "%s", c->err.c_str());
    ECK(cudaMemcpyAsync(k.d_step + slot, st + 1, 4, cudaMemcpyHostToDevice, E->stream));
    ECK(cudaMemcpyAsync(k.d_nsteps + slot, st + 2, 4, cudaMemcpyHostToDevice, E->stream));
    ECK(cudaMemcpyAsync(k.d_active + slot, st + 0, 4, cudaMemcpyHostToDevice, E->stream));
    k.in_use[slot] = 1;
    k.h_mirror[slot] = 1;
    k.h_mirror[k.nslots + slot] = 0;
    return HGPM_OK;
}

extern "C" int hgpm_ens_release(hgpm_ensemble* E, int ci, int slot) {
    int rc = check_slot(E, ci, slot);
    if (rc) return rc;
    EnsClass& k = E->cls[ci];
    if (k.in_use[slot] && k.h_mirror[slot])
        return efail(E, HGPM_ERR_STATE, "class %d slot %d still has steps to run", ci, slot);
    k.in_use[slot] = 0;
    return HGPM_OK;
}

// Kernels of one class step besides the kick: deposit 2, z forward, y
// forward, x potential, y inverse, z inverse, gradient, slot advance.
constexpr int kStepKernels = 9;

// All phases of one step for every slot of class k, on stream s.
static int class_step(hgpm_ensemble* E, EnsClass& k, cudaStream_t s) {
    const int ng = k.ng, M = ng / 2, S = k.nslots;
    const float mass = ctx_cic_mass(ng, k.np);
    const double mean = (double)mass * (double)k.npart / (double)k.ncell;
    ParticleSoA p;
    char* b = (char*)k.part_block;
    const size_t a = k.part_stride * 4 * (size_t)S;
    p.cell = (uint32_t*)b;
    p.ox = (float*)(b + a);
    p.oy = (float*)(b + 2 * a);
    p.oz = (float*)(b + 3 * a);
    p.vx = (float*)(b + 4 * a);
    p.vy = (float*)(b + 5 * a);
    p.vz = (float*)(b + 6 * a);
    const int* act = k.d_active;
    ECK(launch_deposit(p, k.np, ng, mass, k.rho64, k.blkwin, k.dep_spill, s,
                       Slots{act, k.part_stride, k.ncell, k.win_stride}, S, E->dep_choice));
    ECK(launch_zfwd(ng, k.rho64, true, k.spec, ng * ng, k.zs, mean, k.tw_ng, s, Slots{act, k.ncell, k.spec_elems}, S));
    ECK(launch_strided(ng, false, k.spec, M + 1, (size_t)k.zs, (size_t)ng * k.zs, ng, 0, 1, k.tw_ng, s,
                       Slots{act, k.spec_elems, 0}, S));
    ECK(launch_xpotential(ng, k.spec, k.fspec, M + 1, (size_t)ng * k.zs, (size_t)k.zs, ng, k.tw_ng, k.cosq,
                          0.5 / ((double)ng * ng * ng), s, Slots{act, k.spec_elems, 3 * k.spec_elems}, S));
    ECK(launch_strided(ng, true, k.fspec, M + 1, (size_t)k.zs, (size_t)ng * k.zs, ng, 0, 1, k.tw_ng, s,
                       Slots{act, 3 * k.spec_elems, 0}, S));
    float4* f4 = reinterpret_cast<float4*>(k.force);
    float* phi = reinterpret_cast<float*>(k.fspec + k.spec_elems);  // as a single context places it
    ECK(launch_zinv(ng, k.fspec, phi, ng * ng, k.zs, 0, 0, 1, 1.0f, k.tw_ng, s,
                    Slots{act, 3 * k.spec_elems, 6 * k.spec_elems}, S));
    ECK(launch_gradient(ng, phi, f4, s, Slots{act, 6 * k.spec_elems, k.force_elems / 4}, S));
    ECK(launch_kick_drift(p, k.np, ng, f4, 0.0, 0.0, 0.f, 0.f, 0, E->kick_choice, k.blkwin, true, k.kick_spill, s,
                          Slots{act, k.part_stride, k.force_elems / 4, k.win_stride},
                          KickSched{k.d_sched, k.d_step, HGPM_MAX_STEPS}, S));
    ECK(launch_slots_advance(k.d_active, k.d_step, k.d_nsteps, S, s));
    E->launches += kStepKernels + kick_kernels(E->kick_choice, k.np, ng);
    return HGPM_OK;
}

static bool multi_ok(const hgpm_ensemble* E) {
    if (!E->multi || E->cls.empty() || E->cls.size() > (size_t)kMaxMC) return false;
    for (const auto& k : E->cls)
        if (!mc_class_supported(k.ng, k.np)) return false;
    return true;
}

// The classes as a multi-class table (multi_class.h), the largest boxes
// first: CTAs are dispatched in unit order, so the last ones to start, which
// set a launch's tail, are the smallest.
static MCTable multi_table(hgpm_ensemble* E) {
    MCTable t;
    t.n = (int)E->cls.size();
    std::vector<int> order(t.n);
    for (int i = 0; i < t.n; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
        return (double)E->cls[a].np * E->cls[a].np * E->cls[a].np > (double)E->cls[b].np * E->cls[b].np * E->cls[b].np;
    });
    for (int i = 0; i < t.n; ++i) {
        EnsClass& k = E->cls[order[i]];
        MCClass& c = t.c[i];
        const int S = k.nslots;
        c.ng = k.ng;
        c.np = k.np;
        c.nslots = S;
        c.nblocks = (k.np / 16) * (k.np / 16) * (k.np / 16);
        c.zs = k.zs;
        c.mass = ctx_cic_mass(k.ng, k.np);
        c.mean = (double)c.mass * (double)k.npart / (double)k.ncell;
        c.active = k.d_active;
        c.step = k.d_step;
        c.nsteps = k.d_nsteps;
        char* b = (char*)k.part_block;
        const size_t a = k.part_stride * 4 * (size_t)S;
        c.p.cell = (uint32_t*)b;
        c.p.ox = (float*)(b + a);
        c.p.oy = (float*)(b + 2 * a);
        c.p.oz = (float*)(b + 3 * a);
        c.p.vx = (float*)(b + 4 * a);
        c.p.vy = (float*)(b + 5 * a);
        c.p.vz = (float*)(b + 6 * a);
        c.part_stride = k.part_stride;
        c.rho64 = k.rho64;
        c.ncell = k.ncell;
        c.spec = k.spec;
        c.fspec = k.fspec;
        c.spec_elems = k.spec_elems;
        c.force = k.force;
        c.force_elems = k.force_elems;
        c.blkwin = k.blkwin;
        c.win_stride = k.win_stride;
        c.spill = k.dep_spill;
        c.tw = k.tw_ng;
        c.cosq = k.cosq;
        c.sched = k.d_sched;
        c.pitch = HGPM_MAX_STEPS;
    }
    return t;
}

// Fork the class streams off the ensemble stream, run every class that has a
// started slot, join back (or, multi-class, every phase once on the ensemble
// stream).
static int enqueue_step(hgpm_ensemble* E, bool all_classes) {
    if (multi_ok(E)) {
        ECK(mc_step(multi_table(E), E->stream));
        E->launches += kMCStepLaunches;
        return HGPM_OK;
    }
    ECK(cudaEventRecord(E->fork, E->stream));
    for (auto& k : E->cls) {
        bool any = all_classes;
        for (int s = 0; s < k.nslots && !any; ++s) any = k.in_use[s] != 0;
        if (!any) continue;
        ECK(cudaStreamWaitEvent(k.stream, E->fork, 0));
        int rc = class_step(E, k, k.stream);
        if (rc) return rc;
        ECK(cudaEventRecord(k.join, k.stream));
        ECK(cudaStreamWaitEvent(E->stream, k.join, 0));
    }
    return HGPM_OK;
}

extern "C" int hgpm_ens_multi_launch(hgpm_ensemble* E, int on) {
    if (!E) return HGPM_ERR_ARG;
    E->multi = on != 0;
    if (E->exec) {  // the captured step was made for the other form
        cudaGraphExecDestroy(E->exec);
        E->exec = nullptr;
    }
    return multi_ok(E) ? 1 : 0;
}

extern "C" int hgpm_ens_use_graph(hgpm_ensemble* E, int on) {
    if (!E) return HGPM_ERR_ARG;
    if (E->exec) {
        cudaGraphExecDestroy(E->exec);
        E->exec = nullptr;
    }
    for (auto& k : E->cls) {
        if (k.exec) cudaGraphExecDestroy(k.exec);
        k.exec = nullptr;
    }
    E->use_graph = on != 0;
    return HGPM_OK;
}

extern "C" int hgpm_ens_step(hgpm_ensemble* E, int nsteps) {
    if (!E || nsteps < 0) return HGPM_ERR_ARG;
    if (E->use_graph) {
        if (!E->exec) {
            // the graph covers every class (idle slots cost one early-exit CTA
            // row per launch), so it stays valid as slots start and finish
            cudaGraph_t g = nullptr;
            ECK(cudaStreamBeginCapture(E->stream, cudaStreamCaptureModeRelaxed));
            const int64_t before = E->launches;
            int rc = enqueue_step(E, true);
            cudaError_t ce = cudaStreamEndCapture(E->stream, &g);
            if (rc) {
                if (g) cudaGraphDestroy(g);
                return rc;
            }
            ECK(ce);
            E->launches = before;
            cudaError_t ie = cudaGraphInstantiate(&E->exec, g, 0);
            cudaGraphDestroy(g);
            ECK(ie);
        }
        int per = 0;
        if (multi_ok(E)) per = kMCStepLaunches;
        else
            for (auto& k : E->cls) per += kStepKernels + kick_kernels(E->kick_choice, k.np, k.ng);
        for (int i = 0; i < nsteps; ++i) {
            ECK(cudaGraphLaunch(E->exec, E->stream));
            E->launches += per;
        }
        return HGPM_OK;
    }
    for (int i = 0; i < nsteps; ++i) {
        int rc = enqueue_step(E, false);
        if (rc) return rc;
    }
    return HGPM_OK;
}

// ---- one class at a time (serving) ----------------------------------------
// nsteps steps of class ci on the class's own stream, after the slot set-up
// queued on the ensemble stream so far, not joined back: the classes of a
// serving loop advance at their own pace.  hgpm_ens_class_done polls,
// hgpm_ens_sync_class waits and refreshes the class's slot status.
static int class_valid(hgpm_ensemble* E, int ci) {
    if (!E) return HGPM_ERR_ARG;
    if (ci < 0 || ci >= (int)E->cls.size()) return efail(E, HGPM_ERR_ARG, "no class %d", ci);
    return HGPM_OK;
}

extern "C" int hgpm_ens_step_class(hgpm_ensemble* E, int ci, int nsteps) {
    int rc = class_valid(E, ci);
    if (rc) return rc;
    if (nsteps < 0) return efail(E, HGPM_ERR_ARG, "nsteps < 0");
    EnsClass& k = E->cls[ci];
    ECK(cudaEventRecord(k.setup, E->stream));
    ECK(cudaStreamWaitEvent(k.stream, k.setup, 0));
    if (E->use_graph) {
        if (!k.exec) {
            cudaGraph_t g = nullptr;
            ECK(cudaStreamBeginCapture(k.stream, cudaStreamCaptureModeRelaxed));
            const int64_t before = E->launches;
            rc = class_step(E, k, k.stream);
            cudaError_t ce = cudaStreamEndCapture(k.stream, &g);
            E->launches = before;
            if (rc) {
                if (g) cudaGraphDestroy(g);
                return rc;
            }
            ECK(ce);
            cudaError_t ie = cudaGraphInstantiate(&k.exec, g, 0);
            cudaGraphDestroy(g);
            ECK(ie);
        }
        for (int i = 0; i < nsteps; ++i) {
            ECK(cudaGraphLaunch(k.exec, k.stream));
            E->launches += kStepKernels + kick_kernels(E->kick_choice, k.np, k.ng);
        }
    } else {
        for (int i = 0; i < nsteps; ++i)
            if ((rc = class_step(E, k, k.stream))) return rc;
    }
    ECK(cudaEventRecord(k.done, k.stream));
    return HGPM_OK;
}

extern "C" int hgpm_ens_class_done(hgpm_ensemble* E, int ci, int* done) {
    int rc = class_valid(E, ci);
    if (rc) return rc;
    if (!done) return HGPM_ERR_ARG;
    const cudaError_t q = cudaEventQuery(E->cls[ci].done);
    if (q == cudaErrorNotReady) {
        *done = 0;
        return HGPM_OK;
    }
    ECK(q);
    *done = 1;
    return HGPM_OK;
}

extern "C" int hgpm_ens_sync_class(hgpm_ensemble* E, int ci) {
    int rc = class_valid(E, ci);
    if (rc) return rc;
    EnsClass& k = E->cls[ci];
    ECK(cudaMemcpyAsync(k.h_mirror, k.d_active, 4 * k.nslots, cudaMemcpyDeviceToHost, k.stream));
    ECK(cudaMemcpyAsync(k.h_mirror + k.nslots, k.d_step, 4 * k.nslots, cudaMemcpyDeviceToHost, k.stream));
    ECK(cudaStreamSynchronize(k.stream));
    int herr[2] = {0, 0};
    ECK(cudaMemcpy(herr, k.d_err, 8, cudaMemcpyDeviceToHost));
    if (herr[1]) return efail(E, HGPM_ERR_CUDA, "a bounded wait of an FFT pass timed out (results invalid)");
    return HGPM_OK;
}

// Wait for the ensemble's work and refresh the host copy of every slot's
// state (active flag, steps done).
extern "C" int hgpm_ens_sync(hgpm_ensemble* E) {
    if (!E) return HGPM_ERR_ARG;
    for (auto& k : E->cls) {
        ECK(cudaStreamWaitEvent(E->stream, k.done, 0));  // steps queued per class too
        ECK(cudaMemcpyAsync(k.h_mirror, k.d_active, 4 * k.nslots, cudaMemcpyDeviceToHost, E->stream));
        ECK(cudaMemcpyAsync(k.h_mirror + k.nslots, k.d_step, 4 * k.nslots, cudaMemcpyDeviceToHost, E->stream));
    }
    ECK(cudaStreamSynchronize(E->stream));
    for (auto& k : E->cls) {
        int herr[2] = {0, 0};
        ECK(cudaMemcpy(herr, k.d_err, 8, cudaMemcpyDeviceToHost));
        if (herr[1]) return efail(E, HGPM_ERR_CUDA, "a bounded wait of an FFT pass timed out (results invalid)");
    }
    return HGPM_OK;
}

// Slot state as of the last hgpm_ens_sync: *running 1 while steps remain,
// *steps_done the steps completed.
extern "C" int hgpm_ens_status(hgpm_ensemble* E, int ci, int slot, int* running, int* steps_done) {
    int rc = check_slot(E, ci, slot);
    if (rc) return rc;
    EnsClass& k = E->cls[ci];
    if (running) *running = k.in_use[slot] ? k.h_mirror[slot] : 0;
    if (steps_done) *steps_done = k.h_mirror[k.nslots + slot];
    return HGPM_OK;
}
