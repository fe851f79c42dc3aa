// hgpm_ctx.h — the context behind the C-ABI's opaque hgpm_ctx handle, shared
// by the host runtime (runtime.cu) and the batched ensemble (ensemble.cu).
// Not part of the public C-ABI.
#pragma once
#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdio>
#include <string>
#include <vector>

#include "../../include/hgpm_c.h"
#include "hgpm_internal.h"

using namespace hgpm;

struct PhaseRec {
    int phase;
    cudaEvent_t a, b;
};

struct hgpm_ctx {
    hgpm_params p;
    int device = 0;
    cudaStream_t stream = nullptr;
    int ng = 0, np = 0, zs = 0, zs_np = 0, blk = 8;
    size_t ncell = 0, npart = 0, nspec = 0;
    ParticleSoA part{};
    void* part_block = nullptr;
    unsigned long long* rho64 = nullptr;
    bool rho_dirty = false;
    float2* spec = nullptr;
    float2* fspec = nullptr;
    float* force = nullptr;
    float2* tw_ng = nullptr;
    float2* tw_np = nullptr;
    double* cosq = nullptr;
    float* sk = nullptr;
    float* pkw = nullptr;
    float* kf_pk = nullptr;
    float* kf_ic = nullptr;
    float* kf_fold = nullptr;  // k table of the last folded P(k) (lazy)
    int* d_err = nullptr;
    int* blkwin = nullptr;   // per-block CIC windows of the last deposit
    SpillList dep_spill, kick_spill;  // blocks too wide for the windows
    bool win_valid = false;  // blkwin describes the current positions
    // the real potential of the last solve (in the second force spectrum's
    // space) is current; the float4 force grid has been formed from it (a
    // kick that gathers the potential leaves it to hgpm_get_force)
    bool phi_valid = false;
    bool force_valid = false;
    bool phi2_valid = false;  // the paired potential, in the force grid's space
    // kernel variants (environment, read at creation): HGPM_NO_TMA=1 selects the
    // plain strided y passes, HGPM_XTMA=0|1|2 the fused x pass: plain, TMA-fed,
    // or plain with twice the columns per CTA (the default: 0.43 ms against
    // 0.48 TMA-fed at 512^3, 4.3 against 6.2 plain at 1024^3).  The deposit
    // and kick candidates (bit-identical results) are chosen by the autotuner
    // (hgpm_autotune, or its cache), else HGPM_DEPOSIT / HGPM_KICK, else the
    // built-in defaults (-1 / 0).
    bool tma = true;
    int xmode = 2;
    // HGPM_PLANE=1: the z and y passes as one kernel with a thread-block
    // cluster per x plane (launch_zy_fwd / launch_yz_inv_pair) at the sides
    // that have it; 0 (the default, faster) the separate passes
    bool plane = false;
    int dep_choice = -1;
    int kick_choice = 0;
    float* stage = nullptr;     // AoS float3 x, v staging (lazy)
    double* pk_part = nullptr;  // P(k) partial sums (lazy)
    unsigned long long* pk_pcnt = nullptr;
    double* pk_sum = nullptr;
    unsigned long long* pk_cnt = nullptr;
    int pk_nparts = 0;
    double* ic_table = nullptr;  // device copy of the .ipk table (lazy, grows)
    int ic_table_cap = 0;
    // a slot view of an ensemble: the particle, grid and spectrum buffers,
    // the per-size tables, d_err, the staging and P(k) scratch and the
    // stream belong to the ensemble
    bool view = false;
    bool have_state = false;
    bool timing = false;
    std::vector<PhaseRec> recs;
    std::vector<cudaEvent_t> free_events;
    double phase_ms[HGPM_NPHASE] = {0};
    int64_t phase_launch[HGPM_NPHASE] = {0};
    int64_t launches = 0;
    std::string err;
};

static int fail(hgpm_ctx* c, int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    if (c) c->err = buf;
    return code;
}

#define CK(call)                                                                                  \
    do {                                                                                          \
        cudaError_t e_ = (call);                                                                  \
        if (e_ != cudaSuccess)                                                                    \
            return fail(c, e_ == cudaErrorMemoryAllocation ? HGPM_ERR_OOM : HGPM_ERR_CUDA,        \
                        "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
    } while (0)

static cudaEvent_t take_event(hgpm_ctx* c) {
    if (!c->free_events.empty()) {
        cudaEvent_t e = c->free_events.back();
        c->free_events.pop_back();
        return e;
    }
    cudaEvent_t e;
    cudaEventCreate(&e);
    return e;
}

struct PhaseScope {
    hgpm_ctx* c;
    int phase;
    cudaEvent_t a = nullptr;
    PhaseScope(hgpm_ctx* c_, int ph) : c(c_), phase(ph) {
        if (c->timing) {
            a = take_event(c);
            cudaEventRecord(a, c->stream);
        }
    }
    ~PhaseScope() {
        if (c->timing) {
            cudaEvent_t b = take_event(c);
            cudaEventRecord(b, c->stream);
            c->recs.push_back({phase, a, b});
        }
    }
};

static void count(hgpm_ctx* c, int phase, int n) {
    c->launches += n;
    c->phase_launch[phase] += n;
}

enum { PH_DRIFT = 0, PH_DEPOSIT, PH_ZFWD, PH_YFWD, PH_POISSON, PH_YINV, PH_ZINV, PH_KICK, PH_PK };
static_assert(PH_PK + 1 == HGPM_NPHASE, "phase ids");

// Per-box tables that depend on RL (P(k) and IC wavenumbers); (re)computed
// when a context is created or a slot view is rebound to new params.
int ctx_set_rl_tables(hgpm_ctx* c);
// Unit-mass CIC weight scale (ng/np)^3 of pm_actions.cpp:229-230.
float ctx_cic_mass(int ng, int np);
// Apply the autotuner's cached entry for this context's size and device
// (autotune.cu); returns 1 if one was applied.
int ctx_apply_tuned(hgpm_ctx* c);
