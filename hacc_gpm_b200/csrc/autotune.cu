// autotune.cu — picks a context's kernel configurations by timing them.
//
// The reference has one launch knob, BLOCK_SIZE (params.cpp:164), applied to
// every kernel (InvokeGPUKernel, haccgpm.hpp:59).  Here each PM phase has a
// small set of configurations that give bit-identical results and differ
// only in speed, which depends on the box size and on how clustered the
// particles are:
//   deposit  window kernel, threads per CTA, window cap, load ring depth
//            (launch_deposit candidates),
//   kick     flat / windowed gathers from the force grid, or gathers from
//            the real potential (no force grid: the gradient kernel's time
//            is charged to the others), CTA shape, units per CTA turn
//            (launch_kick_drift candidates),
//   y pass   TMA-fed persistent or plain strided transform,
//   x pass   TMA-fed persistent or plain fused Poisson transform.
// hgpm_autotune times every candidate on the context's own current state
// (CUDA events on its stream), keeps the default unless another candidate
// is faster by more than the noise margin, applies the winners to the
// context and records them in a cache file keyed by (device name, SM
// count, ng, np); hgpm_create applies a cached entry to every new context
// of that size on that device.  The particle state is left unchanged: the
// kick candidates run with zero kick and drift factors (v + 0, x + 0 exactly).
#include <cuda_runtime.h>
#include <dlfcn.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "hgpm_ctx.h"

namespace {

std::mutex g_cache_mu;

// Device name with blanks replaced (one token in the cache file) and SM
// count, looked up once per device (cudaGetDeviceProperties takes
// milliseconds, and every context creation consults the cache).
struct DeviceKey {
    bool known = false;
    std::string name;
    int sms = 0;
};
std::mutex g_dev_mu;
DeviceKey g_dev[64];

const DeviceKey& device_key(int dev) {
    static const DeviceKey unknown{true, "unknown", 0};
    if (dev < 0 || dev >= 64) return unknown;
    std::lock_guard<std::mutex> g(g_dev_mu);
    DeviceKey& k = g_dev[dev];
    if (!k.known) {
        cudaDeviceProp prop;
        k.name = cudaGetDeviceProperties(&prop, dev) == cudaSuccess ? std::string(prop.name) : "unknown";
        for (auto& ch : k.name)
            if (ch == ' ' || ch == '\t') ch = '_';
        if (cudaDeviceGetAttribute(&k.sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) k.sms = 0;
        k.known = true;
    }
    return k;
}

std::string lib_dir_cache() {
    Dl_info info;
    if (dladdr(reinterpret_cast<void*>(&hgpm_autotune), &info) && info.dli_fname) {
        std::string p(info.dli_fname);
        const size_t slash = p.rfind('/');
        return (slash == std::string::npos ? std::string(".") : p.substr(0, slash)) + "/tune_cache.txt";
    }
    return "tune_cache.txt";
}

// The cache file: $HGPM_TUNE_CACHE, else tune_cache.txt beside the library.
std::string cache_path() {
    const char* env = getenv("HGPM_TUNE_CACHE");
    if (env && env[0]) return env;
    static std::string beside_lib;
    static std::once_flag once;
    std::call_once(once, [] { beside_lib = lib_dir_cache(); });
    return beside_lib;
}


}  // namespace

extern "C" int hgpm_tune_pick(const double* ms, int n, int def, double tol) {
    if (!ms || n <= 0) return -1;
    if (def < 0 || def >= n) def = 0;
    int best = def;
    for (int i = 0; i < n; ++i)
        if (ms[i] > 0 && (ms[best] <= 0 || ms[i] < ms[best])) best = i;
    // the default stays unless the fastest beats it by more than tol
    if (ms[def] > 0 && ms[best] >= ms[def] * (1.0 - tol)) return def;
    return best;
}

extern "C" int hgpm_tune_cache_lookup(const char* path, const char* device, int sms, int ng, int np,
                                      int choices[HGPM_TUNE_KNOBS]) {
    if (!path || !device || !choices) return HGPM_ERR_ARG;
    std::lock_guard<std::mutex> g(g_cache_mu);
    FILE* f = fopen(path, "r");
    if (!f) return 0;
    char line[512];
    int found = 0;
    while (fgets(line, sizeof(line), f)) {
        char dev[256];
        int s_sms, s_ng, s_np, c[HGPM_TUNE_KNOBS];
        if (sscanf(line, "v1 %255s %d %d %d %d %d %d %d", dev, &s_sms, &s_ng, &s_np, &c[0], &c[1], &c[2], &c[3]) != 8)
            continue;
        if (strcmp(dev, device) || s_sms != sms || s_ng != ng || s_np != np) continue;
        for (int k = 0; k < HGPM_TUNE_KNOBS; ++k) choices[k] = c[k];
        found = 1;  // the last matching line wins
    }
    fclose(f);
    return found;
}

extern "C" int hgpm_tune_cache_store(const char* path, const char* device, int sms, int ng, int np,
                                     const int choices[HGPM_TUNE_KNOBS], const double ms[HGPM_TUNE_KNOBS]) {
    if (!path || !device || !choices || !ms) return HGPM_ERR_ARG;
    for (const char* q = device; *q; ++q)
        if (*q == ' ' || *q == '\t' || *q == '\n') return HGPM_ERR_ARG;
    std::lock_guard<std::mutex> g(g_cache_mu);
    FILE* f = fopen(path, "a");
    if (!f) return HGPM_ERR_IO;
    fprintf(f, "v1 %s %d %d %d %d %d %d %d %.4f %.4f %.4f %.4f\n", device, sms, ng, np, choices[0], choices[1],
            choices[2], choices[3], ms[0], ms[1], ms[2], ms[3]);
    fclose(f);
    return HGPM_OK;
}

// Apply a cached entry for this context's size and device, if one exists
// and the environment does not pin the choice.  Called by hgpm_create.
int ctx_apply_tuned(hgpm_ctx* c) {
    if (getenv("HGPM_NO_TUNE_CACHE")) return 0;
    int ch[HGPM_TUNE_KNOBS];
    const DeviceKey& dk = device_key(c->device);
    if (hgpm_tune_cache_lookup(cache_path().c_str(), dk.name.c_str(), dk.sms, c->ng, c->np, ch) != 1) return 0;
    if (!getenv("HGPM_DEPOSIT") && ch[HGPM_TUNE_DEPOSIT] >= 0 && ch[HGPM_TUNE_DEPOSIT] < deposit_candidates(c->np, c->ng))
        c->dep_choice = ch[HGPM_TUNE_DEPOSIT];
    if (!getenv("HGPM_KICK") && ch[HGPM_TUNE_KICK] >= 0 && ch[HGPM_TUNE_KICK] < kick_candidates(c->np, c->ng))
        c->kick_choice = ch[HGPM_TUNE_KICK];
    if (!getenv("HGPM_NO_TMA")) c->tma = ch[HGPM_TUNE_YPASS] != 0;
    if (!getenv("HGPM_XTMA") && ch[HGPM_TUNE_XPASS] >= 0 && ch[HGPM_TUNE_XPASS] <= 2) c->xmode = ch[HGPM_TUNE_XPASS];
    return 1;
}

namespace {

// ms per launch of `fn` over `reps` launches after one warm-up launch.
template <class F>
double time_launches(hgpm_ctx* c, int reps, const F& fn, cudaError_t* err) {
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    *err = fn();
    cudaEventRecord(a, c->stream);
    for (int r = 0; r < reps && *err == cudaSuccess; ++r) *err = fn();
    cudaEventRecord(b, c->stream);
    cudaEventSynchronize(b);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return *err == cudaSuccess ? (double)ms / reps : -1.0;
}

}  // namespace

extern "C" int hgpm_autotune(hgpm_ctx* c, int reps, int store, int choices[HGPM_TUNE_KNOBS],
                             double best_ms[HGPM_TUNE_KNOBS]) {
    if (!c || reps <= 0) return HGPM_ERR_ARG;
    if (c->view) return fail(c, HGPM_ERR_STATE, "hgpm_autotune: an ensemble slot view has no tuning of its own");
    if (!c->have_state) return fail(c, HGPM_ERR_STATE, "no particle state loaded");
    CK(cudaSetDevice(c->device));
    const double tol = 0.02;  // the noise margin: a candidate must win by 2 %
    const int ng = c->ng, np = c->np, M = ng / 2;
    const float mass = ctx_cic_mass(ng, np);
    const double mean = (double)mass * (double)c->npart / (double)c->ncell;
    cudaError_t e = cudaSuccess;
    int pick[HGPM_TUNE_KNOBS];
    double pms[HGPM_TUNE_KNOBS];

    // deposit (the accumulator is cleared before each candidate; a candidate's
    // repeated launches add into it, which costs the same)
    {
        const int n = deposit_candidates(np, ng);
        std::vector<double> ms(n, -1.0);
        for (int i = 0; i < n; ++i) {
            CK(cudaMemsetAsync(c->rho64, 0, c->ncell * 8, c->stream));
            ms[i] = time_launches(c, reps, [&] {
                return launch_deposit(c->part, np, ng, mass, c->rho64, c->blkwin, c->dep_spill, c->stream, Slots{},
                                      1, i);
            }, &e);
            CK(e);
        }
        pick[HGPM_TUNE_DEPOSIT] = hgpm_tune_pick(ms.data(), n, deposit_default(np, ng), tol);
        pms[HGPM_TUNE_DEPOSIT] = ms[pick[HGPM_TUNE_DEPOSIT]];
    }
    // the density of the winner, then the z pass (consumes the accumulator)
    CK(cudaMemsetAsync(c->rho64, 0, c->ncell * 8, c->stream));
    CK(launch_deposit(c->part, np, ng, mass, c->rho64, c->blkwin, c->dep_spill, c->stream, Slots{}, 1,
                      pick[HGPM_TUNE_DEPOSIT]));
    CK(launch_zfwd(ng, c->rho64, true, c->spec, ng * ng, c->zs, mean, c->tw_ng, c->stream));
    // y pass: 1 = TMA-fed, 0 = plain (in place on the spectrum: timing only;
    // the spectrum is rebuilt below)
    {
        double ms[2];
        for (int t = 0; t < 2; ++t) {
            ms[t] = time_launches(c, reps, [&] {
                return t ? launch_strided_tma(ng, false, false, c->spec, M + 1, c->zs, 0, 1, c->tw_ng, c->d_err + 1,
                                              c->stream)
                         : launch_strided(ng, false, c->spec, M + 1, (size_t)c->zs, (size_t)ng * c->zs, ng, 0, 1,
                                          c->tw_ng, c->stream);
            }, &e);
            CK(e);
        }
        pick[HGPM_TUNE_YPASS] = hgpm_tune_pick(ms, 2, 1, tol);
        pms[HGPM_TUNE_YPASS] = ms[pick[HGPM_TUNE_YPASS]];
    }
    // x pass with the Green's function: 0 = plain, 1 = TMA-fed, 2 = plain
    // with twice the columns per CTA
    {
        double ms[3];
        const double coeff = 0.5 / ((double)ng * ng * ng);
        for (int t = 0; t < 3; ++t) {
            ms[t] = time_launches(c, reps, [&] {
                if (t == 1)
                    return launch_xpotential_tma(ng, c->spec, c->fspec, M + 1, c->zs, c->tw_ng, c->cosq, coeff,
                                                 c->d_err + 1, c->stream);
                if (t == 2)
                    return launch_xpotential_wide(ng, c->spec, c->fspec, M + 1, (size_t)ng * c->zs, (size_t)c->zs,
                                                  ng, c->tw_ng, c->cosq, coeff, c->stream);
                return launch_xpotential(ng, c->spec, c->fspec, M + 1, (size_t)ng * c->zs, (size_t)c->zs, ng,
                                         c->tw_ng, c->cosq, coeff, c->stream);
            }, &e);
            CK(e);
        }
        pick[HGPM_TUNE_XPASS] = hgpm_tune_pick(ms, 3, 2, tol);
        pms[HGPM_TUNE_XPASS] = ms[pick[HGPM_TUNE_XPASS]];
    }
    c->dep_choice = pick[HGPM_TUNE_DEPOSIT];
    c->tma = pick[HGPM_TUNE_YPASS] != 0;
    c->xmode = pick[HGPM_TUNE_XPASS];
    // a real force grid from the current positions for the kick candidates
    c->rho_dirty = true;
    int rc = hgpm_deposit(c);
    if (rc) return rc;
    rc = hgpm_solve_gradient(c);
    if (rc) return rc;
    rc = hgpm_sync(c);
    if (rc) return rc;
    {
        // the potential from the spectrum of the solve above, then the force
        // grid (both formed here whichever kick the context had); a candidate
        // that gathers the force grid is charged the gradient kernel that
        // makes it
        float* phi = reinterpret_cast<float*>(c->fspec + (size_t)ng * ng * c->zs);
        float4* f4 = reinterpret_cast<float4*>(c->force);
        const double z1 = time_launches(c, reps, [&] {
            return launch_zinv(ng, c->fspec, phi, ng * ng, c->zs, 0, 0, 1, 1.0f, c->tw_ng, c->stream);
        }, &e);
        CK(e);
        const double grad_ms = time_launches(c, reps, [&] { return launch_gradient(ng, phi, f4, c->stream); }, &e);
        CK(e);
        const int n = kick_candidates(np, ng);
        std::vector<double> ms(n, -1.0);
        auto time_kick = [&](int i, const float* pot) {
            const double t = time_launches(c, reps, [&] {
                // zero kick and drift factors: v + 0 and x + 0 leave the state as it is
                return launch_kick_drift(c->part, np, ng, f4, 0.0, 0.0, 0.f, 0.f, 2, i, c->blkwin, c->win_valid,
                                         c->kick_spill, c->stream, Slots{}, KickSched{}, 1, pot);
            }, &e);
            return t;
        };
        for (int i = 0; i < n; ++i) {
            if (kick_uses_phi2(i)) continue;
            ms[i] = time_kick(i, phi);
            CK(e);
            if (!kick_uses_phi(i)) ms[i] += grad_ms;
        }
        // the paired potential (in the force grid's space, so after the
        // candidates that gather the grid), charged the extra bytes its z
        // pass writes over the plain one
        const double z2 = time_launches(c, reps, [&] { return launch_zinv_pair(ng, c->fspec, c->force, c->zs, c->tw_ng, c->stream); }, &e);
        CK(e);
        for (int i = 0; i < n; ++i) {
            if (!kick_uses_phi2(i)) continue;
            ms[i] = time_kick(i, c->force) + (z2 - z1);
            CK(e);
        }
        pick[HGPM_TUNE_KICK] = hgpm_tune_pick(ms.data(), n, kick_default(np, ng), tol);
        pms[HGPM_TUNE_KICK] = ms[pick[HGPM_TUNE_KICK]];
    }
    c->kick_choice = pick[HGPM_TUNE_KICK];
    // the potential is the current one; the force grid's space now holds the
    // paired potential
    c->phi_valid = true;
    c->force_valid = false;
    c->phi2_valid = true;
    CK(cudaStreamSynchronize(c->stream));
    if (choices)
        for (int k = 0; k < HGPM_TUNE_KNOBS; ++k) choices[k] = pick[k];
    if (best_ms)
        for (int k = 0; k < HGPM_TUNE_KNOBS; ++k) best_ms[k] = pms[k];
    if (store) {
        const DeviceKey& dk = device_key(c->device);
        if (hgpm_tune_cache_store(cache_path().c_str(), dk.name.c_str(), dk.sms, ng, np, pick, pms))
            return fail(c, HGPM_ERR_IO, "hgpm_autotune: cannot write the cache %s", cache_path().c_str());
    }
    return HGPM_OK;
}

extern "C" int hgpm_tuned_choices(const hgpm_ctx* c, int choices[HGPM_TUNE_KNOBS]) {
    if (!c || !choices) return HGPM_ERR_ARG;
    choices[HGPM_TUNE_DEPOSIT] = c->dep_choice >= 0 ? c->dep_choice : deposit_default(c->np, c->ng);
    choices[HGPM_TUNE_KICK] = c->kick_choice;
    choices[HGPM_TUNE_YPASS] = c->tma ? 1 : 0;
    choices[HGPM_TUNE_XPASS] = c->xmode;
    return HGPM_OK;
}
