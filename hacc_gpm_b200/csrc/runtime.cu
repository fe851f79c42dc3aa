// runtime.cu — host runtime of the PM step behind the C-ABI (include/hgpm_c.h):
// params parser, FP64 time stepper and growth factors, device memory of a
// context, and the phase sequencing that launches the kernels of
// particles.cu and fft_passes.cu on the context's stream.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <algorithm>
#include <map>
#include <mutex>
#include <string>
#include <utility>
#include <vector>

#include "../../include/hgpm_c.h"
#include "hgpm_ctx.h"
#include "hgpm_internal.h"

// ===========================================================================
// params (src/simulation/params.cpp)
// ===========================================================================
static void set_err(char* err, size_t errlen, const char* fmt, ...) {
    if (!err || errlen == 0) return;
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(err, errlen, fmt, ap);
    va_end(ap);
}

static void params_defaults(hgpm_params* p) {
    memset(p, 0, sizeof(*p));
    p->block_size = 64;
    p->w_de = -1.0;
    p->t_cmb = 2.726;
    p->neff_massless = 3.04;
    p->z_ini = 200.0;
    p->ol = 1.0;
    p->pk_bins = 221;  // params.cpp:91
    p->last_step = -1;
    p->ref_quirks = 1;
}

static double atof_f(const char* s) { return (double)(float)atof(s); }

extern "C" void hgpm_params_derive(hgpm_params* p) {
    // params.cpp:237-245
    p->overload = p->rl != 0.0 ? (int)ceil(((double)p->ng) / (p->rl) * p->ol) : 0;
    p->omega_baryon = p->deut / p->hubble / p->hubble;
    p->omega_cb = p->omega_cdm + p->omega_baryon;
    p->omega_matter = p->omega_cb + p->omega_nu;
    p->omega_radiation = 2.471e-5 * pow(p->t_cmb / 2.725f, 4.0f) / pow(p->hubble, 2.0f);
    p->f_nu_massless = p->neff_massless * 7.0 / 8.0 * pow(4.0 / 11.0, 4.0 / 3.0);
    p->f_nu_massive = p->neff_massive * 7.0 / 8.0 * pow(4.0 / 11.0, 4.0 / 3.0);
}

static int mark_steps(unsigned char* arr, const char* value, char* err, size_t errlen, const char* key) {
    if (strcmp(value, "all") == 0) {
        for (int i = 0; i < HGPM_MAX_STEPS; ++i) arr[i] = 1;
        return HGPM_OK;
    }
    std::string v(value);
    size_t pos = 0;
    while (pos <= v.size()) {
        size_t c = v.find(',', pos);
        std::string tok = v.substr(pos, c == std::string::npos ? std::string::npos : c - pos);
        if (!tok.empty()) {
            int s = atoi(tok.c_str());
            if (s < 0 || s >= HGPM_MAX_STEPS) {
                set_err(err, errlen, "%s step %d outside [0, %d)", key, s, HGPM_MAX_STEPS);
                return HGPM_ERR_ARG;
            }
            arr[s] = 1;
        }
        if (c == std::string::npos) break;
        pos = c + 1;
    }
    return HGPM_OK;
}

extern "C" int hgpm_params_parse(const char* text, hgpm_params* out, char* err, size_t errlen) {
    if (!text || !out) return HGPM_ERR_ARG;
    hgpm_params p;
    params_defaults(&p);
    const char* cur = text;
    while (*cur) {
        const char* nl = strchr(cur, '\n');
        size_t len = nl ? (size_t)(nl - cur) : strlen(cur);
        std::string line(cur, len);
        cur = nl ? nl + 1 : cur + len;
        char key[200] = {0}, value[200] = {0};
        int got = sscanf(line.c_str(), "%199s %199s", key, value);
        if (got < 1) continue;
        if (!strcmp(key, "OMEGA_CDM")) p.omega_cdm = atof_f(value);
        else if (!strcmp(key, "DEUT")) p.deut = atof_f(value);
        else if (!strcmp(key, "OMEGA_NU")) p.omega_nu = atof_f(value);
        else if (!strcmp(key, "HUBBLE")) p.hubble = atof_f(value);
        else if (!strcmp(key, "SS8")) p.ss8 = atof_f(value);
        else if (!strcmp(key, "NS")) p.ns = atof_f(value);
        else if (!strcmp(key, "W_DE")) p.w_de = atof_f(value);
        else if (!strcmp(key, "WA_DE")) p.wa_de = atof_f(value);
        else if (!strcmp(key, "T_CMB")) p.t_cmb = atof_f(value);
        else if (!strcmp(key, "N_EFF_MASSLESS")) p.neff_massless = atof_f(value);
        else if (!strcmp(key, "N_EFF_MASSIVE")) p.neff_massive = atof_f(value);
        else if (!strcmp(key, "OUTPUT_BASE_NAME")) snprintf(p.prefix, sizeof(p.prefix), "%s", value);
        else if (!strcmp(key, "Z_IN")) p.z_ini = atof_f(value);
        else if (!strcmp(key, "Z_FIN")) p.z_fin = atof_f(value);
        else if (!strcmp(key, "N_STEPS")) p.nsteps = atoi(value);
        else if (!strcmp(key, "NG")) p.ng = atoi(value);
        else if (!strcmp(key, "NP")) p.np = atoi(value);
        else if (!strcmp(key, "RL")) p.rl = atof_f(value);
        else if (!strcmp(key, "SEED")) p.seed = atoi(value);
        else if (!strcmp(key, "BLOCK_SIZE")) p.block_size = atoi(value);
        else if (!strcmp(key, "LAST_STEP")) p.last_step = atoi(value);
        else if (!strcmp(key, "PK_FOLDS")) p.pk_folds = atoi(value);
        else if (!strcmp(key, "PK_BINS")) p.pk_bins = atoi(value);
        else if (!strcmp(key, "PK_LOG")) p.pk_log = atoi(value);
        else if (!strcmp(key, "REF_QUIRKS")) p.ref_quirks = atoi(value);
        else if (!strcmp(key, "PK_DUMP")) {
            int rc = mark_steps(p.pks, value, err, errlen, key);
            if (rc) return rc;
        } else if (!strcmp(key, "PARTICLE_DUMP")) {
            int rc = mark_steps(p.dumps, value, err, errlen, key);
            if (rc) return rc;
        } else if (!strcmp(key, "ANALYSIS_STEPS")) {
            int rc = mark_steps(p.analysis, value, err, errlen, key);
            if (rc) return rc;
        } else if (!strcmp(key, "ANALYSIS_DIR")) snprintf(p.analysis_dir, sizeof(p.analysis_dir), "%s", value);
        else if (!strcmp(key, "ANALYSIS_PY")) snprintf(p.analysis_py, sizeof(p.analysis_py), "%s", value);
        else if (!strcmp(key, "DO_ANALYSIS")) p.do_analysis = 1;
        else if (!strcmp(key, "DUMP_INIT")) p.dump_init = 1;
        else if (!strcmp(key, "DUMP_FINAL")) p.dump_final = 1;
        else if (!strcmp(key, "IPK")) snprintf(p.ipk, sizeof(p.ipk), "%s", value);
        else if (!strcmp(key, "OL")) p.ol = atof(value);
        else if (!strcmp(key, "NOISE")) {
            if (!strcmp(value, "CURAND")) p.noise = HGPM_NOISE_CURAND;
            else if (!strcmp(value, "PHILOX")) p.noise = HGPM_NOISE_PHILOX;
            else {
                set_err(err, errlen, "NOISE must be CURAND or PHILOX, not %s", value);
                return HGPM_ERR_ARG;
            }
        }
        // unknown keys are ignored, as in the reference
    }
    if (p.np == 0) {
        set_err(err, errlen, "NP missing or zero (params.cpp:228 asserts np != 0)");
        return HGPM_ERR_ARG;
    }
    if (p.last_step == -1) p.last_step = p.nsteps;
    hgpm_params_derive(&p);
    *out = p;
    return HGPM_OK;
}

extern "C" int hgpm_params_read(const char* path, hgpm_params* out, char* err, size_t errlen) {
    FILE* f = fopen(path, "rb");
    if (!f) {
        set_err(err, errlen, "file %s not found", path);
        return HGPM_ERR_IO;
    }
    std::string text;
    char buf[4096];
    size_t n;
    while ((n = fread(buf, 1, sizeof(buf), f)) > 0) text.append(buf, n);
    fclose(f);
    int rc = hgpm_params_parse(text.c_str(), out, err, errlen);
    if (rc == HGPM_OK) snprintf(out->fname, sizeof(out->fname), "%s", path);
    return rc;
}

extern "C" int hgpm_params_save(const hgpm_params* p) {
    char fname2[400];
    snprintf(fname2, sizeof(fname2), "%s.params", p->prefix);
    FILE* fp = fopen(fname2, "w+");
    if (!fp) return HGPM_ERR_IO;
    fprintf(fp, "OMEGA_CDM %g\n", p->omega_cdm);
    fprintf(fp, "DEUT %g\n", p->deut);
    fprintf(fp, "OMEGA_NU %g\n", p->omega_nu);
    fprintf(fp, "HUBBLE %g\n", p->hubble);
    fprintf(fp, "SS8 %g\n", p->ss8);
    fprintf(fp, "NS %g\n", p->ns);
    fprintf(fp, "W_DE %g\n", p->w_de);
    fprintf(fp, "WA_DE %g\n", p->wa_de);
    fprintf(fp, "T_CMB %g\n", p->t_cmb);
    fprintf(fp, "N_EFF_MASSLESS %g\n", p->neff_massless);
    fprintf(fp, "N_EFF_MASSIVE %g\n", p->neff_massive);
    fprintf(fp, "OMEGA_BARYON %g\n", p->omega_baryon);
    fprintf(fp, "OMEGA_CB %g\n", p->omega_cb);
    fprintf(fp, "OMEGA_MATTER %g\n", p->omega_matter);
    fprintf(fp, "OMEGA_RADIATION %g\n", p->omega_radiation);
    fprintf(fp, "M_F_NU_MASSLESS %g\n", p->f_nu_massless);
    fprintf(fp, "M_F_NU_MASSIVE %g\n", p->f_nu_massive);
    fprintf(fp, "OUTPUT_BASE_NAME %s\n", p->prefix);
    fprintf(fp, "Z_IN %g\n", p->z_ini);
    fprintf(fp, "Z_FIN %g\n", p->z_fin);
    fprintf(fp, "N_STEPS %d\n", p->nsteps);
    fprintf(fp, "NG %d\n", p->ng);
    fprintf(fp, "NP %d\n", p->np);
    fprintf(fp, "RL %g\n", p->rl);
    fprintf(fp, "SEED %d\n", p->seed);
    fprintf(fp, "BLOCK_SIZE %d\n", p->block_size);
    fprintf(fp, "PK_FOLDS %d\n", p->pk_folds);
    fclose(fp);
    return HGPM_OK;
}

// ===========================================================================
// time stepper (src/simulation/timestepper.cpp:7-68)
// ===========================================================================
static double omega_nu_massive(double a, const hgpm_params* p) {
    double mat = p->omega_nu / pow(a, 3.0);
    double rad = p->f_nu_massive * p->omega_radiation / pow(a, 4.0);
    return (mat >= rad) * mat + (rad > mat) * rad;
}

extern "C" double hgpm_get_adot(double aa, const hgpm_params* p) {
    double pp1 = pow(aa, -3.0 * (p->w_de + p->wa_de)) * exp(-3.0 * p->wa_de * (1.0 - aa));
    double tmp = p->omega_cb + (1.0 + p->f_nu_massless) * p->omega_radiation / aa +
                 omega_nu_massive(aa, p) * pow(aa, 3.0) +
                 (1.0 - p->omega_matter - (1.0 + p->f_nu_massless) * p->omega_radiation) * pp1;
    tmp /= aa;
    return sqrt(tmp);
}

extern "C" double hgpm_get_fscal(double aa, double adot, double omega_cb, int ref_quirks) {
    double dtdy = aa / (aa * adot);
    if (ref_quirks) dtdy = (double)(float)dtdy;  // timestepper.cpp:24 `float dtdy`
    double phiscal = 1.5 * omega_cb;
    return phiscal * dtdy * (1.0 / aa);
}

static void ts_update(hgpm_timestepper* ts) {
    ts->z = (1.0f / ts->aa) - 1;
    ts->adot = hgpm_get_adot(ts->aa, &ts->params);
    ts->fscal = hgpm_get_fscal(ts->aa, ts->adot, ts->params.omega_cb, ts->params.ref_quirks);
}

extern "C" void hgpm_ts_init(hgpm_timestepper* ts, const hgpm_params* p) {
    memset(ts, 0, sizeof(*ts));
    ts->params = *p;
    ts->deltaT = (((1 / (p->z_fin + 1)) - (1 / (p->z_ini + 1))) / (double)p->nsteps);
}
extern "C" void hgpm_ts_set_initial_z(hgpm_timestepper* ts, double z) {
    ts->aa = 1.0 / (z + 1.0);
    ts_update(ts);
}
extern "C" void hgpm_ts_advance_half(hgpm_timestepper* ts) {
    ts->aa += ts->deltaT * 0.5;
    ts_update(ts);
}
extern "C" void hgpm_ts_reverse_half(hgpm_timestepper* ts) {
    ts->aa -= ts->deltaT * 0.5;
    ts_update(ts);
}
extern "C" float hgpm_ts_drift_prefactor(const hgpm_timestepper* ts, float frac) {
    return (float)(((ts->deltaT) / (ts->aa * ts->aa * ts->adot)) * frac);
}

// ===========================================================================
// growth factor (src/initial_conditions/cosmo.cpp:81-139)
// ===========================================================================
template <class T>
static T g_da_dtau(T a, T om, T ol) {
    T d2 = (T)1 + om * (((T)1 / a) - (T)1) + ol * ((a * a) - (T)1);
    return std::sqrt(d2);
}
template <class T>
static T g_da_dtau3(T a, T om, T ol) {
    T d1 = g_da_dtau(a, om, ol);
    return (T)1 / (d1 * d1 * d1);
}
template <class T>
static T g_int(T a, T om, T ol, int bins) {
    T start = 0, end = a;
    T delta = (end - start) / ((T)bins);
    T sum = 0;
    for (int k = 1; k < bins; ++k) sum += g_da_dtau3(start + ((T)k) * delta, om, ol);
    sum += (g_da_dtau3(start, om, ol) + g_da_dtau3(end, om, ol)) / (T)2;
    sum *= delta;
    return sum;
}
template <class T>
static T g_delta(T a, T om, T ol, int bins) {
    T integral = g_int(a, om, ol, bins);
    T diff = g_da_dtau(a, om, ol);
    T mul = ((T)5 * om) / ((T)2 * a);
    return mul * diff * integral;
}

extern "C" void hgpm_growth(const hgpm_params* p, double z, double z_vel, double* delta, double* dot_delta) {
    if (p->ref_quirks) {
        // the reference's CosmoClass: float arithmetic, 100-bin trapezoid,
        // central difference with h = 1e-4 (cosmo.cpp:106-139)
        float om = (float)p->omega_matter;
        float ol = 1 - (om + (float)p->omega_nu);
        float a0 = 1.0f / (1.0f + (float)z);
        float a1 = 1.0f / (1.0f + (float)z_vel);
        float h = 0.0001f;
        *delta = g_delta<float>(a0, om, ol, 100);
        *dot_delta = (g_delta<float>(a1 + h, om, ol, 100) - g_delta<float>(a1 - h, om, ol, 100)) / (2.0f * h);
    } else {
        // FP64: the same integral with 20000 trapezoid bins and h = 1e-6
        double om = p->omega_matter;
        double ol = 1 - (om + p->omega_nu);
        double a0 = 1.0 / (1.0 + z), a1 = 1.0 / (1.0 + z_vel), h = 1e-6;
        *delta = g_delta<double>(a0, om, ol, 20000);
        *dot_delta = (g_delta<double>(a1 + h, om, ol, 20000) - g_delta<double>(a1 - h, om, ol, 20000)) / (2.0 * h);
    }
}

// ===========================================================================
// context (struct hgpm_ctx in hgpm_ctx.h)
// ===========================================================================

static std::vector<float2> twiddles(int n) {
    std::vector<float2> t(n);
    for (int m = 0; m < n; ++m) {
        double ang = -2.0 * M_PI * (double)m / (double)n;
        t[m] = make_float2((float)cos(ang), (float)sin(ang));
    }
    return t;
}

static int even_pad(int v) { return (v + 15) / 16 * 16; }

// Device bytes of one context: every buffer hgpm_create allocates (sized as
// it sizes them: spectra and the force grid cover the larger of the ng and
// np grids, which the ICs use), plus the ones made on first use (the float3
// staging of hgpm_load_state / hgpm_store_state, the P(k) partial sums, the
// RL and .ipk tables), each rounded up to the 2 MiB granularity of large
// device allocations.
extern "C" size_t hgpm_footprint_bytes(int ng, int np) {
    const size_t ncell = (size_t)ng * ng * ng, npart = (size_t)np * np * np;
    const size_t nspec = (size_t)ng * ng * even_pad(ng / 2 + 1);
    const size_t nspec_np = (size_t)np * np * even_pad(np / 2 + 1);
    const size_t spec_elems = std::max(nspec, nspec_np);
    const size_t force_elems = 4 * std::max(ncell, npart);
    const size_t nblocks = (size_t)window_records(np, ng) / 8;
    const size_t page = 2u << 20;
    auto r = [&](size_t b) { return (b + page - 1) / page * page; };
    size_t b = 0;
    b += r((npart * 4 + 255) / 256 * 256 * 7);          // particle SoA (one block)
    b += r(ncell * 8);                                  // int64 density
    b += r(spec_elems * 8);                             // spectrum
    b += r(spec_elems * 8 * 3);                         // potential / IC spectra
    b += r(force_elems * 4);                            // float4 force grid
    b += r((size_t)window_records(np, ng) * 4);         // per-block CIC windows
    b += r((4 + 2 * nblocks) * 4);                      // spill queues and counters
    b += r((size_t)ng * 8 * 2 + (size_t)np * 8 + (size_t)ng * 8 + (size_t)ng * 12 + (size_t)np * 4 + 8);  // tables
    b += r(npart * 6 * 4);                              // float3 staging (first host load/store)
    b += r((size_t)4 * 148 * pk_max_bins() * 16 + (size_t)pk_max_bins() * 16);  // P(k) partial sums
    b += r(20000 * 8);                                  // .ipk table (20000 bins)
    return b;
}

extern "C" int hgpm_create(const hgpm_params* p, int device, hgpm_ctx** out) {
    if (!p || !out) return HGPM_ERR_ARG;
    *out = nullptr;
    hgpm_ctx* c = new hgpm_ctx();
    c->p = *p;
    c->device = device;
    c->ng = p->ng;
    c->np = p->np;
    auto bad = [&](int code, const char* msg) {
        c->err = msg;
        *out = c;  // return the context so the caller can read the message
        return code;
    };
    if (!fft_size_supported(p->ng)) return bad(HGPM_ERR_ARG, "NG must be one of " HGPM_SIZES_TEXT);
    if (!fft_size_supported(p->np)) return bad(HGPM_ERR_ARG, "NP must be one of " HGPM_SIZES_TEXT);
    if (p->rl <= 0) return bad(HGPM_ERR_ARG, "RL must be positive");
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return bad(HGPM_ERR_CUDA, cudaGetErrorString(e));
    e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) return bad(HGPM_ERR_CUDA, cudaGetErrorString(e));
    c->ncell = (size_t)c->ng * c->ng * c->ng;
    {
        const char* nt = getenv("HGPM_NO_TMA");
        c->tma = !(nt && nt[0] == '1');
        const char* xt = getenv("HGPM_XTMA");
        if (xt && xt[0] >= '0' && xt[0] <= '2') c->xmode = xt[0] - '0';
        const char* pv = getenv("HGPM_PLANE");
        if (pv && (pv[0] == '0' || pv[0] == '1')) c->plane = pv[0] == '1';
        const char* kv = getenv("HGPM_KICK");
        c->kick_choice = kick_default(p->np, p->ng);
        if (kv && kv[0] >= '0' && kv[0] <= '9' && atoi(kv) < kick_candidates(p->np, p->ng)) c->kick_choice = atoi(kv);
        const char* dv = getenv("HGPM_DEPOSIT");
        if (dv && dv[0] >= '0' && dv[0] <= '9' && atoi(dv) < deposit_candidates(p->np, p->ng)) c->dep_choice = atoi(dv);
        ctx_apply_tuned(c);
    }
    c->blk = block_side(c->np, c->ng);
    c->npart = (size_t)c->np * c->np * c->np;
    c->zs = even_pad(c->ng / 2 + 1);
    c->zs_np = even_pad(c->np / 2 + 1);
    c->nspec = (size_t)c->ng * c->ng * c->zs;
    size_t nspec_np = (size_t)c->np * c->np * c->zs_np;
    size_t spec_elems = std::max(c->nspec, nspec_np);
    // float4 force grid (4 floats per cell); ICs use it as 3 planes of npart
    size_t force_elems = 4 * std::max(c->ncell, c->npart);
    int rc = HGPM_OK;
    do {
        // particles: one block, 7 arrays of npart 4-byte words (256-B aligned)
        size_t stride = (c->npart * 4 + 255) / 256 * 256;
        e = cudaMalloc(&c->part_block, stride * 7);
        if (e != cudaSuccess) break;
        char* b = (char*)c->part_block;
        c->part.cell = (uint32_t*)(b);
        c->part.ox = (float*)(b + stride);
        c->part.oy = (float*)(b + 2 * stride);
        c->part.oz = (float*)(b + 3 * stride);
        c->part.vx = (float*)(b + 4 * stride);
        c->part.vy = (float*)(b + 5 * stride);
        c->part.vz = (float*)(b + 6 * stride);
        if ((e = cudaMalloc(&c->rho64, c->ncell * 8)) != cudaSuccess) break;
        if ((e = cudaMemsetAsync(c->rho64, 0, c->ncell * 8, c->stream)) != cudaSuccess) break;
        if ((e = cudaMalloc(&c->spec, spec_elems * 8)) != cudaSuccess) break;
        if ((e = cudaMalloc(&c->fspec, 3 * spec_elems * 8)) != cudaSuccess) break;
        if ((e = cudaMalloc(&c->force, force_elems * 4)) != cudaSuccess) break;
        if ((e = cudaMalloc(&c->tw_ng, c->ng * 8)) != cudaSuccess) break;
        if ((e = cudaMalloc(&c->tw_np, c->np * 8)) != cudaSuccess) break;
        if ((e = cudaMalloc(&c->cosq, c->ng * 8)) != cudaSuccess) break;
        if ((e = cudaMalloc(&c->sk, c->ng * 4)) != cudaSuccess) break;
        if ((e = cudaMalloc(&c->pkw, c->ng * 4)) != cudaSuccess) break;
        // d_err[0]: IC table overrun; d_err[1]: a bounded TMA/mbarrier wait timed out
        if ((e = cudaMalloc(&c->d_err, 8)) != cudaSuccess) break;
        if ((e = cudaMalloc(&c->blkwin, (size_t)window_records(c->np, c->ng) * 4)) != cudaSuccess) break;
        {
            const int nblocks = window_records(c->np, c->ng) / 8;
            int* sp = nullptr;
            if ((e = cudaMalloc(&sp, (size_t)(4 + 2 * nblocks) * 4)) != cudaSuccess) break;
            // counters: deposit queue, kick queue, blocks over the kick's cap,
            // the kick's work counter
            c->dep_spill = SpillList{sp, sp + 4, nblocks, sp + 2, sp + 3};
            c->kick_spill = SpillList{sp + 1, sp + 4 + nblocks, nblocks, sp + 2, sp + 3};
        }
        if ((e = cudaMemsetAsync(c->d_err, 0, 8, c->stream)) != cudaSuccess) break;
        std::vector<float2> t1 = twiddles(c->ng), t2 = twiddles(c->np);
        if ((e = cudaMemcpy(c->tw_ng, t1.data(), c->ng * 8, cudaMemcpyHostToDevice)) != cudaSuccess) break;
        if ((e = cudaMemcpy(c->tw_np, t2.data(), c->np * 8, cudaMemcpyHostToDevice)) != cudaSuccess) break;
        if ((e = launch_ktables(c->ng, c->cosq, c->sk, c->pkw, c->stream)) != cudaSuccess) break;
        if (!p->ref_quirks) {
            std::vector<double> cq(c->ng);
            for (int i = 0; i < c->ng; ++i) {
                double s = sin(M_PI * (double)i / (double)c->ng);
                cq[i] = -2.0 * s * s;  // cos(2 pi i/ng) - 1
            }
            if ((e = cudaMemcpyAsync(c->cosq, cq.data(), c->ng * 8, cudaMemcpyHostToDevice, c->stream)) != cudaSuccess) break;
        }
        if ((e = cudaStreamSynchronize(c->stream)) != cudaSuccess) break;
    } while (0);
    if (e != cudaSuccess) {
        rc = e == cudaErrorMemoryAllocation ? HGPM_ERR_OOM : HGPM_ERR_CUDA;
        c->err = std::string("hgpm_create: ") + cudaGetErrorString(e);
        cudaGetLastError();
    } else {
        rc = ctx_set_rl_tables(c);
    }
    c->launches += 1;
    *out = c;
    return rc;
}

int ctx_set_rl_tables(hgpm_ctx* c) {
    if (!c->kf_pk) CK(cudaMalloc(&c->kf_pk, c->ng * 4));
    if (!c->kf_ic) CK(cudaMalloc(&c->kf_ic, c->np * 4));
    std::vector<float> kf(c->ng), kfi(c->np);
    const double dpk = 2.0 * M_PI / c->p.rl;
    for (int i = 0; i < c->ng; ++i) kf[i] = (float)((double)signed_mode(i, c->ng) * dpk);
    for (int i = 0; i < c->np; ++i) kfi[i] = (float)((double)signed_mode(i, c->np) * dpk);
    CK(cudaMemcpyAsync(c->kf_pk, kf.data(), c->ng * 4, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(c->kf_ic, kfi.data(), c->np * 4, cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return HGPM_OK;
}

extern "C" void hgpm_destroy(hgpm_ctx* c) {
    if (!c) return;
    if (c->stream) cudaStreamSynchronize(c->stream);
    // a view owns only its RL tables and its IC table
    void* own[] = {c->kf_pk, c->kf_ic, c->kf_fold, c->ic_table};
    for (void* q : own)
        if (q) cudaFree(q);
    if (!c->view) {
        void* ptrs[] = {c->part_block, c->rho64, c->spec, c->fspec, c->force, c->tw_ng, c->tw_np, c->cosq, c->sk,
                        c->pkw, c->d_err, c->stage, c->pk_part, c->pk_pcnt, c->pk_sum, c->pk_cnt, c->blkwin,
                        c->dep_spill.cnt};
        for (void* q : ptrs)
            if (q) cudaFree(q);
    }
    for (auto& r : c->recs) {
        cudaEventDestroy(r.a);
        cudaEventDestroy(r.b);
    }
    for (auto e : c->free_events) cudaEventDestroy(e);
    if (c->stream && !c->view) cudaStreamDestroy(c->stream);
    delete c;
}

extern "C" const char* hgpm_last_error(const hgpm_ctx* c) { return c ? c->err.c_str() : "null context"; }
extern "C" void* hgpm_stream(hgpm_ctx* c) { return c ? (void*)c->stream : nullptr; }
extern "C" int hgpm_ng(const hgpm_ctx* c) { return c ? c->ng : 0; }
extern "C" int hgpm_np(const hgpm_ctx* c) { return c ? c->np : 0; }

// Synchronise and report a timed-out bounded wait of a TMA pass, if any.
static int sync_check(hgpm_ctx* c) {
    int herr[2] = {0, 0};
    CK(cudaMemcpyAsync(herr, c->d_err, 8, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (herr[1]) {
        cudaMemsetAsync(c->d_err + 1, 0, 4, c->stream);
        return fail(c, HGPM_ERR_CUDA, "a TMA-fed FFT pass timed out waiting for its tile (results invalid)");
    }
    return HGPM_OK;
}

extern "C" int hgpm_sync(hgpm_ctx* c) {
    if (!c) return HGPM_ERR_ARG;
    return sync_check(c);
}

extern "C" int hgpm_test_wait_timeout(hgpm_ctx* c, unsigned polls) {
    if (!c || polls == 0 || polls > (1u << 20)) return HGPM_ERR_ARG;
    CK(launch_wait_timeout_probe(c->d_err + 1, polls, c->stream));
    return HGPM_OK;
}

// ===========================================================================
// state I/O
// ===========================================================================
static int ensure_stage(hgpm_ctx* c) {
    if (!c->stage) CK(cudaMalloc(&c->stage, c->npart * 6 * sizeof(float)));
    return HGPM_OK;
}

extern "C" int hgpm_load_state_device(hgpm_ctx* c, const float* x, const float* v) {
    if (!c || !x || !v) return HGPM_ERR_ARG;
    CK(launch_load_state(x, v, c->part, c->np, c->blk, c->ng, c->stream));
    count(c, PH_DRIFT, 1);
    c->have_state = true;
    c->win_valid = false;
    return HGPM_OK;
}

extern "C" int hgpm_store_state_device(hgpm_ctx* c, float* x, float* v) {
    if (!c || !x || !v) return HGPM_ERR_ARG;
    if (!c->have_state) return fail(c, HGPM_ERR_STATE, "no particle state loaded");
    CK(launch_store_state(c->part, x, v, c->np, c->blk, c->ng, c->stream));
    count(c, PH_DRIFT, 1);
    return HGPM_OK;
}

extern "C" int hgpm_load_state(hgpm_ctx* c, const float* x, const float* v) {
    if (!c || !x || !v) return HGPM_ERR_ARG;
    int rc = ensure_stage(c);
    if (rc) return rc;
    size_t bytes = c->npart * 3 * sizeof(float);
    CK(cudaMemcpyAsync(c->stage, x, bytes, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(c->stage + 3 * c->npart, v, bytes, cudaMemcpyHostToDevice, c->stream));
    rc = hgpm_load_state_device(c, c->stage, c->stage + 3 * c->npart);
    if (rc) return rc;
    CK(cudaStreamSynchronize(c->stream));
    return HGPM_OK;
}

extern "C" int hgpm_store_state(hgpm_ctx* c, float* x, float* v) {
    if (!c || !x || !v) return HGPM_ERR_ARG;
    int rc = ensure_stage(c);
    if (rc) return rc;
    rc = hgpm_store_state_device(c, c->stage, c->stage + 3 * c->npart);
    if (rc) return rc;
    size_t bytes = c->npart * 3 * sizeof(float);
    CK(cudaMemcpyAsync(x, c->stage, bytes, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(v, c->stage + 3 * c->npart, bytes, cudaMemcpyDeviceToHost, c->stream));
    return sync_check(c);
}

// ---- checkpoints: the exact device state (packed cells, offsets,
// velocities, in the context's internal order) plus the time stepper
namespace {
struct CkptHeader {
    char magic[8];  // "HGPMCK01"
    int32_t ng, np, blk, pad;
    double rl;
    int64_t npart;
    hgpm_timestepper ts;
};
}  // namespace

extern "C" size_t hgpm_checkpoint_bytes(const hgpm_ctx* c) {
    return c ? sizeof(CkptHeader) + c->npart * 7 * 4 : 0;
}

extern "C" int hgpm_checkpoint_save(hgpm_ctx* c, const hgpm_timestepper* ts, void* buf, size_t bytes) {
    if (!c || !ts || !buf) return HGPM_ERR_ARG;
    if (!c->have_state) return fail(c, HGPM_ERR_STATE, "no particle state loaded");
    if (bytes < hgpm_checkpoint_bytes(c)) return fail(c, HGPM_ERR_ARG, "checkpoint buffer too small");
    CkptHeader h;
    memset(&h, 0, sizeof(h));
    memcpy(h.magic, "HGPMCK01", 8);
    h.ng = c->ng;
    h.np = c->np;
    h.blk = c->blk;
    h.rl = c->p.rl;
    h.npart = (int64_t)c->npart;
    h.ts = *ts;
    memcpy(buf, &h, sizeof(h));
    char* d = (char*)buf + sizeof(h);
    const void* src[7] = {c->part.cell, c->part.ox, c->part.oy, c->part.oz, c->part.vx, c->part.vy, c->part.vz};
    for (int a = 0; a < 7; ++a)
        CK(cudaMemcpyAsync(d + (size_t)a * c->npart * 4, src[a], c->npart * 4, cudaMemcpyDeviceToHost, c->stream));
    return sync_check(c);
}

extern "C" int hgpm_checkpoint_load(hgpm_ctx* c, hgpm_timestepper* ts, const void* buf, size_t bytes) {
    if (!c || !buf) return HGPM_ERR_ARG;
    CkptHeader h;
    if (bytes < sizeof(h)) return fail(c, HGPM_ERR_ARG, "checkpoint truncated");
    memcpy(&h, buf, sizeof(h));
    if (memcmp(h.magic, "HGPMCK01", 8) != 0) return fail(c, HGPM_ERR_ARG, "not a checkpoint");
    if (h.ng != c->ng || h.np != c->np || h.blk != c->blk || h.npart != (int64_t)c->npart)
        return fail(c, HGPM_ERR_ARG, "checkpoint of NG %d NP %d does not fit this context (NG %d NP %d)", h.ng, h.np,
                    c->ng, c->np);
    if (bytes < hgpm_checkpoint_bytes(c)) return fail(c, HGPM_ERR_ARG, "checkpoint truncated");
    const char* s = (const char*)buf + sizeof(h);
    void* dst[7] = {c->part.cell, c->part.ox, c->part.oy, c->part.oz, c->part.vx, c->part.vy, c->part.vz};
    for (int a = 0; a < 7; ++a)
        CK(cudaMemcpyAsync(dst[a], s + (size_t)a * c->npart * 4, c->npart * 4, cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    c->have_state = true;
    c->win_valid = false;
    if (ts) *ts = h.ts;
    return HGPM_OK;
}

extern "C" int hgpm_analysis_rows(hgpm_ctx* c, float* rows) {
    if (!c || !rows) return HGPM_ERR_ARG;
    std::vector<float> x(c->npart * 3), v(c->npart * 3);
    int rc = hgpm_store_state(c, x.data(), v.data());
    if (rc) return rc;
    for (size_t i = 0; i < c->npart; ++i) {
        float* r = rows + 7 * i;
        r[0] = (float)i;
        for (int a = 0; a < 3; ++a) {
            r[1 + a] = x[3 * i + a];
            r[4 + a] = v[3 * i + a];
        }
    }
    return HGPM_OK;
}

extern "C" int hgpm_read_output(hgpm_ctx* c, const char* fname) {
    if (!c || !fname) return HGPM_ERR_ARG;
    FILE* fp = fopen(fname, "rb");
    if (!fp) return fail(c, HGPM_ERR_IO, "cannot open %s", fname);
    std::vector<float> x(c->npart * 3), v(c->npart * 3);
    const size_t nx = fread(x.data(), sizeof(float) * 3, c->npart, fp);
    const size_t nv = fread(v.data(), sizeof(float) * 3, c->npart, fp);
    fclose(fp);
    if (nx != c->npart || nv != c->npart)
        return fail(c, HGPM_ERR_IO, "%s holds fewer than 2 x %zu float3", fname, c->npart);
    return hgpm_load_state(c, x.data(), v.data());
}

extern "C" int hgpm_get_cells(hgpm_ctx* c, int32_t* cells) {
    if (!c || !cells) return HGPM_ERR_ARG;
    if (!c->have_state) return fail(c, HGPM_ERR_STATE, "no particle state loaded");
    std::vector<uint32_t> packed(c->npart);
    CK(cudaMemcpyAsync(packed.data(), c->part.cell, c->npart * 4, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    for (size_t i = 0; i < c->npart; ++i) {
        uint32_t q = packed[i];
        cells[lattice_of_internal(i, c->np, c->blk)] = (cell_x(q) * c->ng + cell_y(q)) * c->ng + cell_z(q);
    }
    return HGPM_OK;
}

// ===========================================================================
// phases
// ===========================================================================
extern "C" int hgpm_drift(hgpm_ctx* c, float prefactor) {
    if (!c) return HGPM_ERR_ARG;
    if (!c->have_state) return fail(c, HGPM_ERR_STATE, "no particle state loaded");
    PhaseScope ps(c, PH_DRIFT);
    CK(launch_drift(c->part, c->npart, c->ng, prefactor, c->stream));
    c->win_valid = false;
    count(c, PH_DRIFT, 1);
    return HGPM_OK;
}

float ctx_cic_mass(int ng, int np) {
    // pm_actions.cpp:229-230
    float gpscale = (((float)ng / (float)np));
    return gpscale * gpscale * gpscale;
}
static float cic_mass(int ng, int np) { return ctx_cic_mass(ng, np); }

static double mean_density(const hgpm_ctx* c) {
    return (double)cic_mass(c->ng, c->np) * (double)c->npart / (double)c->ncell;
}

static int deposit_impl(hgpm_ctx* c) {
    if (c->rho_dirty) CK(cudaMemsetAsync(c->rho64, 0, c->ncell * 8, c->stream));
    CK(launch_deposit(c->part, c->np, c->ng, cic_mass(c->ng, c->np), c->rho64, c->blkwin, c->dep_spill, c->stream,
                      Slots{}, 1, c->dep_choice));
    c->win_valid = true;
    count(c, PH_DEPOSIT, 2);  // windowed pass + spill pass
    c->rho_dirty = true;
    return HGPM_OK;
}

extern "C" int hgpm_deposit(hgpm_ctx* c) {
    if (!c) return HGPM_ERR_ARG;
    if (!c->have_state) return fail(c, HGPM_ERR_STATE, "no particle state loaded");
    PhaseScope ps(c, PH_DEPOSIT);
    return deposit_impl(c);
}

extern "C" int hgpm_get_density(hgpm_ctx* c, float* rho) {
    if (!c || !rho) return HGPM_ERR_ARG;
    if (!c->rho_dirty) return fail(c, HGPM_ERR_STATE, "no deposited density (call hgpm_deposit first)");
    std::vector<long long> h(c->ncell);
    CK(cudaMemcpyAsync(h.data(), c->rho64, c->ncell * 8, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    for (size_t i = 0; i < c->ncell; ++i) rho[i] = (float)((double)h[i] * kFixInv);
    return HGPM_OK;
}

// forward z + y passes of the fixed-point density into c->spec (consumes and
// zeroes the accumulator)
static int forward_zy(hgpm_ctx* c) {
    const int ng = c->ng, M = ng / 2;
    if (c->plane && plane_fft_supported(ng)) {
        PhaseScope ps(c, PH_ZFWD);
        CK(launch_zy_fwd(ng, c->rho64, c->spec, c->zs, mean_density(c), c->tw_ng, c->stream));
        c->rho_dirty = false;
        count(c, PH_ZFWD, 1);
        return HGPM_OK;
    }
    {
        PhaseScope ps(c, PH_ZFWD);
        CK(launch_zfwd(ng, c->rho64, true, c->spec, ng * ng, c->zs, mean_density(c), c->tw_ng, c->stream));
        c->rho_dirty = false;
        count(c, PH_ZFWD, 1);
    }
    {
        PhaseScope ps(c, PH_YFWD);
        if (c->tma)
            CK(launch_strided_tma(ng, false, false, c->spec, M + 1, c->zs, 0, 1, c->tw_ng, c->d_err + 1, c->stream));
        else
            CK(launch_strided(ng, false, c->spec, M + 1, (size_t)c->zs, (size_t)ng * c->zs, ng, 0, 1, c->tw_ng,
                              c->stream));
        count(c, PH_YFWD, 1);
    }
    return HGPM_OK;
}

extern "C" int hgpm_solve_gradient(hgpm_ctx* c) {
    if (!c) return HGPM_ERR_ARG;
    if (!c->rho_dirty) return fail(c, HGPM_ERR_STATE, "no deposited density (call hgpm_deposit first)");
    const int ng = c->ng, M = ng / 2;
    int rc = forward_zy(c);
    if (rc) return rc;
    const size_t cs = (size_t)ng * ng * c->zs;
    {
        PhaseScope ps(c, PH_POISSON);
        const double coeff = 0.5 / ((double)ng * ng * ng);
        if (c->xmode == 1)
            CK(launch_xpotential_tma(ng, c->spec, c->fspec, M + 1, c->zs, c->tw_ng, c->cosq, coeff, c->d_err + 1,
                                     c->stream));
        else if (c->xmode == 2)
            CK(launch_xpotential_wide(ng, c->spec, c->fspec, M + 1, (size_t)ng * c->zs, (size_t)c->zs, ng, c->tw_ng,
                                      c->cosq, coeff, c->stream));
        else
            CK(launch_xpotential(ng, c->spec, c->fspec, M + 1, (size_t)ng * c->zs, (size_t)c->zs, ng, c->tw_ng,
                                 c->cosq, coeff, c->stream));
        count(c, PH_POISSON, 1);
    }
    const bool plane_inv = c->plane && plane_fft_supported(ng) && kick_uses_phi2(c->kick_choice);
    if (!plane_inv) {
        PhaseScope ps(c, PH_YINV);
        if (c->tma)
            CK(launch_strided_tma(ng, true, false, c->fspec, M + 1, c->zs, 0, 1, c->tw_ng, c->d_err + 1, c->stream));
        else
            CK(launch_strided(ng, true, c->fspec, M + 1, (size_t)c->zs, (size_t)ng * c->zs, ng, 0, 1, c->tw_ng,
                              c->stream));
        count(c, PH_YINV, 1);
    }
    {
        // the real potential (in the space of the second force spectrum), then
        // the force grid by central differences, unless the kick gathers the
        // potential itself (hgpm_get_force then forms the grid on demand)
        PhaseScope ps(c, PH_ZINV);
        float* phi = reinterpret_cast<float*>(c->fspec + cs);
        c->force_valid = false;
        if (kick_uses_phi2(c->kick_choice)) {
            // the paired potential, in the force grid's space (with the
            // inverse y pass when the plane kernels run)
            if (plane_inv) CK(launch_yz_inv_pair(ng, c->fspec, c->force, c->zs, c->tw_ng, c->stream));
            else CK(launch_zinv_pair(ng, c->fspec, c->force, c->zs, c->tw_ng, c->stream));
            c->phi_valid = false;
            c->phi2_valid = true;
        } else {
            CK(launch_zinv(ng, c->fspec, phi, ng * ng, c->zs, 0, 0, 1, 1.0f, c->tw_ng, c->stream));
            c->phi_valid = true;
            c->phi2_valid = false;
            if (!kick_uses_phi(c->kick_choice)) {
                CK(launch_gradient(ng, phi, reinterpret_cast<float4*>(c->force), c->stream));
                c->force_valid = true;
            }
        }
        count(c, PH_ZINV, c->force_valid ? 2 : 1);
    }
    return HGPM_OK;
}

// The potential of the last solve in the form the context's kick gathers
// (the paired potential for the pair-gathering kick, else the real one), or
// null (the kick then gathers the force grid).
static const float* ctx_phi(const hgpm_ctx* c) {
    if (kick_uses_phi2(c->kick_choice)) return c->phi2_valid ? c->force : nullptr;
    return c->phi_valid ? reinterpret_cast<const float*>(c->fspec + (size_t)c->ng * c->ng * c->zs) : nullptr;
}

extern "C" int hgpm_get_force(hgpm_ctx* c, float* f) {
    if (!c || !f) return HGPM_ERR_ARG;
    if (!c->force_valid && !c->phi_valid && c->phi2_valid) {
        // the real potential from the potential's spectrum, which the solve
        // leaves in place (the grid below overwrites the paired potential)
        const int ng = c->ng;
        CK(launch_zinv(ng, c->fspec, reinterpret_cast<float*>(c->fspec + (size_t)ng * ng * c->zs), ng * ng, c->zs,
                       0, 0, 1, 1.0f, c->tw_ng, c->stream));
        count(c, PH_ZINV, 1);
        c->phi_valid = true;
    }
    if (!c->force_valid && c->phi_valid) {
        const float* phi = reinterpret_cast<const float*>(c->fspec + (size_t)c->ng * c->ng * c->zs);
        CK(launch_gradient(c->ng, phi, reinterpret_cast<float4*>(c->force), c->stream));
        count(c, PH_ZINV, 1);
        c->force_valid = true;
        c->phi2_valid = false;
    }
    // the device grid is float4 (F_x, F_y, F_z, 0) per cell; the ABI returns
    // three planes
    std::vector<float4> g(c->ncell);
    CK(cudaMemcpyAsync(g.data(), c->force, c->ncell * sizeof(float4), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    for (size_t i = 0; i < c->ncell; ++i) {
        f[i] = g[i].x;
        f[c->ncell + i] = g[i].y;
        f[2 * c->ncell + i] = g[i].z;
    }
    return HGPM_OK;
}

extern "C" int hgpm_kick_drift(hgpm_ctx* c, double deltaT, double fscal, float pf_a, float pf_b, int ndrift) {
    if (!c || ndrift < 0 || ndrift > 2) return HGPM_ERR_ARG;
    if (!c->have_state) return fail(c, HGPM_ERR_STATE, "no particle state loaded");
    PhaseScope ps(c, PH_KICK);
    CK(launch_kick_drift(c->part, c->np, c->ng, reinterpret_cast<const float4*>(c->force), deltaT, fscal, pf_a, pf_b,
                         ndrift, c->kick_choice, c->blkwin, c->win_valid, c->kick_spill, c->stream, Slots{},
                         KickSched{}, 1, ctx_phi(c)));
    if (ndrift > 0) c->win_valid = false;
    count(c, PH_KICK, kick_kernels(c->kick_choice, c->np, c->ng));
    return HGPM_OK;
}

extern "C" int hgpm_kick(hgpm_ctx* c, double deltaT, double fscal) {
    return hgpm_kick_drift(c, deltaT, fscal, 0.f, 0.f, 0);
}

extern "C" int hgpm_run_steps(hgpm_ctx* c, hgpm_timestepper* ts, int nsteps) {
    if (!c || !ts || nsteps < 0) return HGPM_ERR_ARG;
    if (!c->have_state) return fail(c, HGPM_ERR_STATE, "no particle state loaded");
    if (nsteps == 0) return HGPM_OK;
    int rc = hgpm_drift(c, hgpm_ts_drift_prefactor(ts, 0.5f));  // driver_pm.cpp:114
    if (rc) return rc;
    for (int step = 0; step < nsteps; ++step) {
        if ((rc = hgpm_deposit(c))) return rc;                   // :116
        if ((rc = hgpm_solve_gradient(c))) return rc;            // :117
        hgpm_ts_advance_half(ts);                                // :119
        const double dt = ts->deltaT, fs = ts->fscal;
        hgpm_ts_advance_half(ts);                                // :123
        const float pf = hgpm_ts_drift_prefactor(ts, 0.5f);      // :125 and the next step's :114
        if ((rc = hgpm_kick_drift(c, dt, fs, pf, pf, step + 1 < nsteps ? 2 : 1))) return rc;  // :121, :125
    }
    return HGPM_OK;
}

extern "C" int hgpm_step_host(hgpm_ctx* c, hgpm_timestepper* ts, float* x, float* v) {
    int rc = hgpm_load_state(c, x, v);
    if (rc) return rc;
    if ((rc = hgpm_run_steps(c, ts, 1))) return rc;
    return hgpm_store_state(c, x, v);
}

// ===========================================================================
// power spectrum
// ===========================================================================
// Bin edges of power.cu:174-187 for a box of side rl_bins: minK = 2pi/rl_bins,
// maxK = sqrt(3 (ng/2)^2 d^2).  (The reference sets them once per call from
// the most-folded box, rl / 2^PK_FOLDS, for every fold.)
static int pk_bins_setup(const hgpm_ctx* c, double rl_bins, int nbins, int log_bins, double* min_k,
                         double* bin_delta, std::vector<double>& centres) {
    double d = (2 * M_PI) / rl_bins;
    double mk = d;
    double maxk = sqrt(3 * ((c->ng / 2) * (c->ng / 2) * d * d));
    centres.resize(nbins);
    if (log_bins) {
        double dl = log(maxk / mk) / (double)nbins;
        for (int i = 0; i < nbins; ++i) centres[i] = mk * exp(dl * ((double)i + 0.5));
        *bin_delta = dl;
    } else {
        double bd = (maxk - mk) / ((double)nbins);
        for (int i = 0; i < nbins; ++i) centres[i] = mk + bd * (((float)i) + 0.5f);
        *bin_delta = bd;
    }
    *min_k = mk;
    return 0;
}

extern "C" int hgpm_power_spectrum(hgpm_ctx* c, int nbins, int log_bins, double* k_out, double* pk_out,
                                   int64_t* n_out) {
    return hgpm_power_spectrum_fold(c, 0, nbins, log_bins, k_out, pk_out, n_out);
}

// GetPowerSpectrum's fold loop body (power.cu:189-227) for one fold.
extern "C" int hgpm_power_spectrum_fold(hgpm_ctx* c, int fold, int nbins, int log_bins, double* k_out,
                                        double* pk_out, int64_t* n_out) {
    if (!c || !k_out || !pk_out || !n_out || nbins <= 0 || fold < 0) return HGPM_ERR_ARG;
    if (fold > 9) return fail(c, HGPM_ERR_ARG, "fold %d above 9", fold);
    if (nbins > pk_max_bins()) return fail(c, HGPM_ERR_ARG, "nbins %d above %d", nbins, pk_max_bins());
    if (!c->have_state) return fail(c, HGPM_ERR_STATE, "no particle state loaded");
    const int ng = c->ng, M = ng / 2;
    if (!c->pk_part) {
        c->pk_nparts = 4 * 148;
        CK(cudaMalloc(&c->pk_part, (size_t)c->pk_nparts * pk_max_bins() * 8));
        CK(cudaMalloc(&c->pk_pcnt, (size_t)c->pk_nparts * pk_max_bins() * 8));
        CK(cudaMalloc(&c->pk_sum, pk_max_bins() * 8));
        CK(cudaMalloc(&c->pk_cnt, pk_max_bins() * 8));
    }
    PhaseScope ps(c, PH_PK);
    // the fold's box: rl / 2^fold (power.cu:193); with ref_quirks the bins come
    // from rl / 2^max(PK_FOLDS, fold) and the power is scaled with the
    // unfolded rl, as the reference does for every fold (power.cu:174-187,
    // 215); without, both follow the fold's own box
    const double rl_f = c->p.rl / pow(2.0, fold);
    const int nf = c->p.pk_folds > fold ? c->p.pk_folds : fold;
    const double rl_bins = c->p.ref_quirks ? c->p.rl / pow(2.0, nf) : rl_f;
    const double rl_scale = c->p.ref_quirks ? c->p.rl : rl_f;
    int rc;
    if (fold == 0) {
        rc = deposit_impl(c);  // serial::CIC of the positions (power.cu:210)
        if (rc) return rc;
    } else {
        if (c->rho_dirty) CK(cudaMemsetAsync(c->rho64, 0, c->ncell * 8, c->stream));
        CK(launch_deposit_folded(c->part, c->npart, c->ng, fold, cic_mass(c->ng, c->np), c->rho64, c->stream));
        c->rho_dirty = true;
        count(c, PH_PK, 1);
        if (!c->kf_fold) CK(cudaMalloc(&c->kf_fold, c->ng * 4));
        std::vector<float> kf(c->ng);
        const double d = (2 * M_PI) / rl_f;
        for (int i = 0; i < c->ng; ++i) kf[i] = (float)((double)signed_mode(i, c->ng) * d);
        CK(cudaMemcpyAsync(c->kf_fold, kf.data(), c->ng * 4, cudaMemcpyHostToDevice, c->stream));
        CK(cudaStreamSynchronize(c->stream));
    }
    rc = forward_zy(c);
    if (rc) return rc;
    PkArgs a;
    std::vector<double> centres;
    pk_bins_setup(c, rl_bins, nbins, log_bins, &a.min_k, &a.bin_delta, centres);
    a.kf = fold == 0 ? c->kf_pk : c->kf_fold;
    a.filt = c->pkw;
    a.nbins = nbins;
    a.log_bins = log_bins;
    a.scale = (1.0f / ((double)ng * ng * ng)) * (rl_scale / ng);
    CK(launch_xpk(ng, c->spec, M + 1, (size_t)ng * c->zs, (size_t)c->zs, c->tw_ng, a, c->pk_part, c->pk_pcnt,
                  c->pk_nparts, c->pk_sum, c->pk_cnt, c->stream));
    count(c, PH_PK, 2);
    std::vector<double> sum(nbins);
    std::vector<unsigned long long> cnt(nbins);
    CK(cudaMemcpyAsync(sum.data(), c->pk_sum, nbins * 8, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(cnt.data(), c->pk_cnt, nbins * 8, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    for (int i = 0; i < nbins; ++i) {
        k_out[i] = centres[i];
        n_out[i] = (int64_t)cnt[i];
        pk_out[i] = cnt[i] ? sum[i] / (double)cnt[i] : 0.0;
    }
    return HGPM_OK;
}

extern "C" int hgpm_write_pk(const char* fname, int nbins, const double* k, const double* pk, const int64_t* count) {
    return hgpm_write_pk_fold(fname, 0, nbins, k, pk, count);
}

extern "C" int hgpm_write_pk_fold(const char* fname, int fold, int nbins, const double* k, const double* pk,
                                  const int64_t* count) {
    char fname2[400];
    snprintf(fname2, sizeof(fname2), "%s.fold.%d", fname, fold);
    FILE* fp = fopen(fname2, "w+");
    if (!fp) return HGPM_ERR_IO;
    for (int i = 0; i < nbins; ++i) {
        double o = pk[i];
        if ((o == o) && (count[i] != 0) && (o != 0)) fprintf(fp, "%g,%g,%d\n", k[i], o, (int)count[i]);
    }
    fclose(fp);
    return HGPM_OK;
}

extern "C" int hgpm_write_output(hgpm_ctx* c, const char* fname) {
    if (!c || !fname) return HGPM_ERR_ARG;
    std::vector<float> x(c->npart * 3), v(c->npart * 3);
    int rc = hgpm_store_state(c, x.data(), v.data());
    if (rc) return rc;
    FILE* fp = fopen(fname, "w+");
    if (!fp) return fail(c, HGPM_ERR_IO, "cannot open %s", fname);
    fwrite(x.data(), sizeof(float) * 3, c->npart, fp);
    fwrite(v.data(), sizeof(float) * 3, c->npart, fp);
    fclose(fp);
    return HGPM_OK;
}

// ===========================================================================
// initial conditions (src/initial_conditions/initializer.cpp:65-166)
// ===========================================================================
extern "C" int hgpm_read_ipk(const char* path, double* header20, double* table, int max_bins, int* nbins) {
    FILE* f = fopen(path, "rb");
    if (!f) return HGPM_ERR_IO;
    double header[20];
    if (fread(header, sizeof(header), 1, f) != 1) {
        fclose(f);
        return HGPM_ERR_IO;
    }
    int nb = (int)header[2];
    if (header20) memcpy(header20, header, sizeof(header));
    if (nbins) *nbins = nb;
    if (table) {
        if (nb > max_bins) {
            fclose(f);
            return HGPM_ERR_ARG;
        }
        if (fread(table, sizeof(double), nb, f) != (size_t)nb) {
            fclose(f);
            return HGPM_ERR_IO;
        }
    }
    fclose(f);
    return HGPM_OK;
}

static int ic_common(hgpm_ctx* c, const float* noise_host, const double* table, int nbins, double k_delta) {
    if (!c || !table || nbins < 2 || k_delta <= 0) return HGPM_ERR_ARG;
    const int n = c->np, M = n / 2;
    const size_t npart = c->npart;
    // time stepper state at the IC epoch (driver_pm.cpp:63-65)
    hgpm_timestepper ts;
    hgpm_ts_init(&ts, &c->p);
    hgpm_ts_set_initial_z(&ts, c->p.z_ini);
    hgpm_ts_reverse_half(&ts);
    // initializer.cpp:81-86
    double this_a = (1 / (c->p.z_ini + 1)) - (ts.deltaT / 2.0f);
    double velZ = (1.0f / this_a) - 1.0f;
    double delta, dot_delta;
    hgpm_growth(&c->p, c->p.z_ini, velZ, &delta, &dot_delta);
    // table range: the largest |k| on the n^3 grid must sit inside the table
    double kmax = sqrt(3.0) * (n / 2) * 2 * M_PI / c->p.rl;
    if ((int)(kmax / k_delta) + 1 >= nbins)
        return fail(c, HGPM_ERR_ARG, "input ipk only goes to k=%g, grid needs %g", k_delta * (nbins - 1), kmax);
    if (nbins > c->ic_table_cap) {
        if (c->ic_table) CK(cudaFree(c->ic_table));
        c->ic_table = nullptr;
        c->ic_table_cap = 0;
        CK(cudaMalloc(&c->ic_table, (size_t)nbins * 8));
        c->ic_table_cap = nbins;
    }
    double* d_table = c->ic_table;
    int rc = HGPM_OK;
    do {
        float* noise = c->force;  // scratch: the force grids are rebuilt every solve
        c->phi_valid = false;     // the IC spectra and displacements overwrite all three
        c->force_valid = false;
        c->phi2_valid = false;
        cudaError_t e;
        if (noise_host) {
            e = cudaMemcpyAsync(noise, noise_host, npart * 4, cudaMemcpyHostToDevice, c->stream);
        } else {
            e = launch_noise(noise, npart, c->p.seed, c->p.noise, c->stream);
            count(c, PH_PK, 1);
        }
        if (e != cudaSuccess) { rc = fail(c, HGPM_ERR_CUDA, "ic noise: %s", cudaGetErrorString(e)); break; }
        if ((e = cudaMemcpyAsync(d_table, table, (size_t)nbins * 8, cudaMemcpyHostToDevice, c->stream)) != cudaSuccess) {
            rc = fail(c, HGPM_ERR_CUDA, "ic table: %s", cudaGetErrorString(e)); break;
        }
        if ((e = cudaMemsetAsync(c->d_err, 0, 4, c->stream)) != cudaSuccess) { rc = fail(c, HGPM_ERR_CUDA, "%s", cudaGetErrorString(e)); break; }
        const size_t cs = (size_t)n * n * c->zs_np;
        e = launch_zfwd(n, noise, false, c->spec, n * n, c->zs_np, 0.0, c->tw_np, c->stream);
        if (e == cudaSuccess) e = launch_strided(n, false, c->spec, M + 1, (size_t)c->zs_np, (size_t)n * c->zs_np, n, 0, 1, c->tw_np, c->stream);
        if (e == cudaSuccess)
            e = launch_xic(n, c->spec, c->fspec, M + 1, (size_t)n * c->zs_np, (size_t)c->zs_np, n, cs, c->tw_np, d_table,
                           nbins, k_delta, ((double)n * n * n) / (c->p.rl * c->p.rl * c->p.rl), 1.0 / delta, c->kf_ic,
                           c->d_err, c->stream);
        if (e == cudaSuccess) e = launch_strided(n, true, c->fspec, M + 1, (size_t)c->zs_np, (size_t)n * c->zs_np, n, cs, 3, c->tw_np, c->stream);
        float scale = (float)(1.0f / ((double)npart));
        if (e == cudaSuccess) e = launch_zinv(n, c->fspec, c->force, n * n, c->zs_np, cs, npart, 3, scale, c->tw_np, c->stream);
        // placeParticles: velA = a - deltaT/2 (float), velMul in double then float
        double a = 1.0 / (1.0 + c->p.z_ini);
        float velA = a - (ts.deltaT * 0.5f);
        float velmul = (float)((double)(velA * velA) * dot_delta * ts.fscal);
        if (e == cudaSuccess) e = launch_place(c->force, npart, c->part, n, c->ng, (float)delta, velmul, c->stream);
        count(c, PH_PK, 6);
        if (e != cudaSuccess) { rc = fail(c, HGPM_ERR_CUDA, "ic kernels: %s", cudaGetErrorString(e)); break; }
        int herr = 0;
        if ((e = cudaMemcpyAsync(&herr, c->d_err, 4, cudaMemcpyDeviceToHost, c->stream)) != cudaSuccess ||
            (e = cudaStreamSynchronize(c->stream)) != cudaSuccess) {
            rc = fail(c, HGPM_ERR_CUDA, "ic sync: %s", cudaGetErrorString(e)); break;
        }
        if (herr) { rc = fail(c, HGPM_ERR_ARG, "ipk table too short for the grid's largest |k|"); break; }
        c->have_state = true;
        c->win_valid = false;
    } while (0);
    return rc;
}

extern "C" int hgpm_ic_generate(hgpm_ctx* c, const double* table, int nbins, double k_delta) {
    return ic_common(c, nullptr, table, nbins, k_delta);
}

extern "C" int hgpm_ic_from_noise(hgpm_ctx* c, const float* noise, const double* table, int nbins, double k_delta) {
    if (!noise) return HGPM_ERR_ARG;
    return ic_common(c, noise, table, nbins, k_delta);
}

extern "C" int hgpm_ic_noise(hgpm_ctx* c, float* out) {
    if (!c || !out) return HGPM_ERR_ARG;
    c->force_valid = false;  // the noise is drawn into the force grid's space
    c->phi2_valid = false;
    CK(launch_noise(c->force, c->npart, c->p.seed, c->p.noise, c->stream));
    count(c, PH_PK, 1);
    CK(cudaMemcpyAsync(out, c->force, c->npart * 4, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return HGPM_OK;
}

// ===========================================================================
// timing
// ===========================================================================
extern "C" int hgpm_enable_timing(hgpm_ctx* c, int on) {
    if (!c) return HGPM_ERR_ARG;
    c->timing = on != 0;
    return HGPM_OK;
}

extern "C" int hgpm_phase_times(hgpm_ctx* c, double* ms, int64_t* launches) {
    if (!c) return HGPM_ERR_ARG;
    CK(cudaStreamSynchronize(c->stream));
    for (auto& r : c->recs) {
        float t = 0.f;
        cudaEventElapsedTime(&t, r.a, r.b);
        c->phase_ms[r.phase] += t;
        c->free_events.push_back(r.a);
        c->free_events.push_back(r.b);
    }
    c->recs.clear();
    for (int i = 0; i < HGPM_NPHASE; ++i) {
        if (ms) ms[i] = c->phase_ms[i];
        if (launches) launches[i] = c->phase_launch[i];
        c->phase_ms[i] = 0.0;
        c->phase_launch[i] = 0;
    }
    return HGPM_OK;
}

extern "C" int64_t hgpm_kernel_launches(hgpm_ctx* c, int reset) {
    if (!c) return 0;
    int64_t n = c->launches;
    if (reset) c->launches = 0;
    return n;
}

extern "C" size_t hgpm_sizeof_params(void) { return sizeof(hgpm_params); }
extern "C" size_t hgpm_sizeof_timestepper(void) { return sizeof(hgpm_timestepper); }

// serial::forward_fft / backward_fft on a caller's cufftComplex grid
// (ffts.cu:244-294, 397-445).  Twiddle tables per (device, ng), made on first
// use and kept until exit.
extern "C" int hgpm_fft_c2c(void* data_dev, int ng, int inverse, void* stream) {
    if (!data_dev || !fft_size_supported(ng)) return HGPM_ERR_ARG;
    static std::mutex mu;
    static std::map<std::pair<int, int>, float2*> tables;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return HGPM_ERR_CUDA;
    float2* tw = nullptr;
    {
        std::lock_guard<std::mutex> g(mu);
        auto it = tables.find({dev, ng});
        if (it != tables.end()) {
            tw = it->second;
        } else {
            const std::vector<float2> t = twiddles(ng);
            if (cudaMalloc(&tw, ng * sizeof(float2)) != cudaSuccess) return HGPM_ERR_OOM;
            if (cudaMemcpy(tw, t.data(), ng * sizeof(float2), cudaMemcpyHostToDevice) != cudaSuccess) {
                cudaFree(tw);
                return HGPM_ERR_CUDA;
            }
            tables[{dev, ng}] = tw;
        }
    }
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    if (launch_fft_c2c(ng, reinterpret_cast<float2*>(data_dev), inverse != 0, tw, s) != cudaSuccess)
        return HGPM_ERR_CUDA;
    if (!stream && cudaStreamSynchronize(nullptr) != cudaSuccess) return HGPM_ERR_CUDA;
    return HGPM_OK;
}
