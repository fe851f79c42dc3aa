// haccgpm_serial.cpp — HACCGPM::serial:: over the C-ABI (see haccgpm.hpp).
#include "haccgpm.hpp"

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

CPUTimer_t CPUTimer() {
    using namespace std::chrono;
    return (CPUTimer_t)duration_cast<microseconds>(steady_clock::now().time_since_epoch()).count();
}

namespace HACCGPM {

static void die(const char* what, const char* msg) {
    fprintf(stderr, "HACCGPM: %s: %s\n", what, msg ? msg : "");
    exit(1);
}

static void check(hgpm_ctx* ctx, int rc, const char* what) {
    if (rc != HGPM_OK) die(what, ctx ? hgpm_last_error(ctx) : "invalid argument");
}

static void from_c(Params& p, const hgpm_params& c) {
    memset(&p, 0, sizeof(p));
    p.c = c;
    memcpy(p.fname, c.fname, sizeof(p.fname));
    memcpy(p.prefix, c.prefix, sizeof(p.prefix));
    memcpy(p.ipk, c.ipk, sizeof(p.ipk));
    p.ng = c.ng;
    p.np = c.np;
    p.rl = c.rl;
    p.blockSize = c.block_size;
    p.seed = c.seed;
    p.z_ini = c.z_ini;
    p.z_fin = c.z_fin;
    p.nsteps = c.nsteps;
    p.m_hubble = c.hubble;
    p.m_omega_cdm = c.omega_cdm;
    p.m_omega_nu = c.omega_nu;
    p.m_deut = c.deut;
    p.m_ss8 = c.ss8;
    p.m_ns = c.ns;
    p.m_w_de = c.w_de;
    p.m_wa_de = c.wa_de;
    p.m_Tcmb = c.t_cmb;
    p.m_neff_massless = c.neff_massless;
    p.m_neff_massive = c.neff_massive;
    p.m_omega_baryon = c.omega_baryon;
    p.m_omega_cb = c.omega_cb;
    p.m_omega_matter = c.omega_matter;
    p.m_omega_radiation = c.omega_radiation;
    p.m_f_nu_massless = c.f_nu_massless;
    p.m_f_nu_massive = c.f_nu_massive;
    for (int i = 0; i < HGPM_MAX_STEPS; ++i) {
        p.pks[i] = c.pks[i] != 0;
        p.dumps[i] = c.dumps[i] != 0;
    }
    p.lastStep = c.last_step;
    p.pkFolds = c.pk_folds;
    p.world_rank = 0;
    p.world_size = 1;
    for (int a = 0; a < 3; ++a) {
        p.local_grid_size[a] = p.ng;
        p.grid_dims[a] = 1;
        p.grid_coords[a] = 0;
    }
    p.dump_init = c.dump_init != 0;
    p.dump_final = c.dump_final != 0;
    p.ol = c.ol;
    p.overload = c.overload;
    p.pk_bins = c.pk_bins;
    p.pk_log = c.pk_log != 0;
    p.do_analysis = c.do_analysis != 0;
    for (int i = 0; i < HGPM_MAX_STEPS; ++i) p.analysis[i] = c.analysis[i] != 0;
    memcpy(p.analysis_dir, c.analysis_dir, sizeof(p.analysis_dir));
    memcpy(p.analysis_py, c.analysis_py, sizeof(p.analysis_py));
}

hgpm_params to_c(const Params& p) {
    hgpm_params c = p.c;
    memcpy(c.fname, p.fname, sizeof(c.fname));
    memcpy(c.prefix, p.prefix, sizeof(c.prefix));
    memcpy(c.ipk, p.ipk, sizeof(c.ipk));
    c.ng = p.ng;
    c.np = p.np;
    c.rl = p.rl;
    c.block_size = p.blockSize;
    c.seed = p.seed;
    c.z_ini = p.z_ini;
    c.z_fin = p.z_fin;
    c.nsteps = p.nsteps;
    c.hubble = p.m_hubble;
    c.omega_cdm = p.m_omega_cdm;
    c.omega_nu = p.m_omega_nu;
    c.deut = p.m_deut;
    c.ss8 = p.m_ss8;
    c.ns = p.m_ns;
    c.w_de = p.m_w_de;
    c.wa_de = p.m_wa_de;
    c.t_cmb = p.m_Tcmb;
    c.neff_massless = p.m_neff_massless;
    c.neff_massive = p.m_neff_massive;
    for (int i = 0; i < HGPM_MAX_STEPS; ++i) {
        c.pks[i] = p.pks[i] ? 1 : 0;
        c.dumps[i] = p.dumps[i] ? 1 : 0;
    }
    c.last_step = p.lastStep;
    c.pk_folds = p.pkFolds;
    c.dump_init = p.dump_init ? 1 : 0;
    c.dump_final = p.dump_final ? 1 : 0;
    c.ol = p.ol;
    c.pk_bins = p.pk_bins;
    c.pk_log = p.pk_log ? 1 : 0;
    c.do_analysis = p.do_analysis ? 1 : 0;
    for (int i = 0; i < HGPM_MAX_STEPS; ++i) c.analysis[i] = p.analysis[i] ? 1 : 0;
    memcpy(c.analysis_dir, p.analysis_dir, sizeof(c.analysis_dir));
    memcpy(c.analysis_py, p.analysis_py, sizeof(c.analysis_py));
    hgpm_params_derive(&c);
    return c;
}

static void print_params(const hgpm_params& p) {
    // params.cpp:41-70
    printf("Params:\n");
    printf("   OMEGA_CDM %g\n   DEUT %g\n   OMEGA_NU %g\n   HUBBLE %g\n", p.omega_cdm, p.deut, p.omega_nu, p.hubble);
    printf("   SS8 %g\n   NS %g\n   W_DE %g\n   WA_DE %g\n   T_CMB %g\n", p.ss8, p.ns, p.w_de, p.wa_de, p.t_cmb);
    printf("   N_EFF_MASSLESS %g\n   N_EFF_MASSIVE %g\n", p.neff_massless, p.neff_massive);
    printf("   OMEGA_BARYON %g\n   OMEGA_CB %g\n   OMEGA_MATTER %g\n   OMEGA_RADIATION %g\n", p.omega_baryon,
           p.omega_cb, p.omega_matter, p.omega_radiation);
    printf("   M_F_NU_MASSLESS %g\n   M_F_NU_MASSIVE %g\n", p.f_nu_massless, p.f_nu_massive);
    printf("   OUTPUT_BASE_NAME %s\n   Z_IN %g\n   Z_FIN %g\n   N_STEPS %d\n", p.prefix, p.z_ini, p.z_fin, p.nsteps);
    printf("   NG %d\n   NP %d\n   RL %g\n   SEED %d\n   BLOCK_SIZE %d\n   PK_FOLDS %d\n", p.ng, p.np, p.rl, p.seed,
           p.block_size, p.pk_folds);
}

Params read_params(const char* fname) {
    hgpm_params c;
    char err[512] = {0};
    if (hgpm_params_read(fname, &c, err, sizeof(err)) != HGPM_OK) die("read_params", err);
    print_params(c);
    if (hgpm_params_save(&c) != HGPM_OK) die("save_params", "cannot write <prefix>.params");
    Params p;
    from_c(p, c);
    return p;
}

// ---------------------------------------------------------------------------
Timestepper::Timestepper(Params iparams) : params(iparams), aa(0), z(0), deltaT(0), adot(0), fscal(0), world_rank(0) {
    hgpm_timestepper t;
    const hgpm_params c = HACCGPM::to_c(params);
    hgpm_ts_init(&t, &c);
    from_c(t);
}

hgpm_timestepper Timestepper::to_c() const {
    hgpm_timestepper t;
    const hgpm_params c = HACCGPM::to_c(params);
    hgpm_ts_init(&t, &c);
    t.aa = aa;
    t.z = z;
    t.deltaT = deltaT;
    t.adot = adot;
    t.fscal = fscal;
    return t;
}

void Timestepper::from_c(const hgpm_timestepper& t) {
    aa = t.aa;
    z = t.z;
    deltaT = t.deltaT;
    adot = t.adot;
    fscal = t.fscal;
}

void Timestepper::setInitialA(double a) { setInitialZ(1.0 / a - 1.0); }

void Timestepper::setInitialZ(double zz) {
    hgpm_timestepper t = to_c();
    hgpm_ts_set_initial_z(&t, zz);
    from_c(t);
}

void Timestepper::advanceHalfStep() {
    hgpm_timestepper t = to_c();
    hgpm_ts_advance_half(&t);
    from_c(t);
}

void Timestepper::reverseHalfStep() {
    hgpm_timestepper t = to_c();
    hgpm_ts_reverse_half(&t);
    from_c(t);
}

// ---------------------------------------------------------------------------
CosmoClass::CosmoClass(Params& params) {
    const hgpm_params c = to_c(params);
    Omega_m = c.omega_matter;
    Omega_cb = c.omega_cb;
    h = c.hubble;
    memcpy(ipk, c.ipk, sizeof(ipk));
}

void CosmoClass::read_ipk(double** out, int* nbins, double* k_delta, double* k_max, double* k_min, int) {
    double header[20];
    int nb = 0;
    if (hgpm_read_ipk(ipk, header, nullptr, 0, &nb) != HGPM_OK) die("read_ipk", ipk);
    double* t = new double[nb];
    if (hgpm_read_ipk(ipk, header, t, nb, &nb) != HGPM_OK) die("read_ipk", ipk);
    *out = t;
    *nbins = nb;
    // generate_ipk.py:192-202 header layout: [.., k_min, k_max, k_bins, k_delta, ..]
    *k_min = header[0];
    *k_max = header[1];
    *k_delta = header[3];
}

// ---------------------------------------------------------------------------
namespace serial {

MemoryManager::MemoryManager(Params params) {
    const hgpm_params c = to_c(params);
    const int rc = hgpm_create(&c, 0, &ctx);
    if (rc != HGPM_OK) die("MemoryManager", ctx ? hgpm_last_error(ctx) : "hgpm_create failed");
}

MemoryManager::~MemoryManager() { hgpm_destroy(ctx); }

void fft_cache_plan(int) {}

// on the legacy stream, returning when done (hgpm_fft_c2c with no stream)
static void fft_c2c(const char* name, floatFFT_t* d_grid, int ng, int inverse) {
    const int rc = hgpm_fft_c2c(d_grid, ng, inverse, nullptr);
    if (rc != HGPM_OK) die(name, rc == HGPM_ERR_ARG ? "unsupported grid size or null grid" : "CUDA error");
}

void forward_fft(floatFFT_t* d_grid, int ng, int) { fft_c2c("forward_fft", d_grid, ng, 0); }

void backward_fft(floatFFT_t* d_grid, int ng, int) { fft_c2c("backward_fft", d_grid, ng, 1); }

void InitGreens(Params&, MemoryManager&, int) {}

void GenerateDisplacementIC(MemoryManager& mem, CosmoClass& cosmo, Params&, Timestepper&, int) {
    double* table = nullptr;
    int nb = 0;
    double kd = 0, kmax = 0, kmin = 0;
    cosmo.read_ipk(&table, &nb, &kd, &kmax, &kmin);
    const int rc = hgpm_ic_generate(mem.ctx, table, nb, kd);
    delete[] table;
    check(mem.ctx, rc, "GenerateDisplacementIC");
}

void UpdatePositions(Params&, MemoryManager& mem, Timestepper ts, float frac, int) {
    const hgpm_timestepper t = ts.to_c();
    check(mem.ctx, hgpm_drift(mem.ctx, hgpm_ts_drift_prefactor(&t, frac)), "UpdatePositions");
}

void CIC(Params&, MemoryManager& mem, int) { check(mem.ctx, hgpm_deposit(mem.ctx), "CIC"); }

void SolveGradient(Params&, MemoryManager& mem, int) {
    check(mem.ctx, hgpm_solve_gradient(mem.ctx), "SolveGradient");
}

void UpdateVelocities(Params&, MemoryManager& mem, Timestepper ts, int) {
    check(mem.ctx, hgpm_kick(mem.ctx, ts.deltaT, ts.fscal), "UpdateVelocities");
}

void GetPowerSpectrum(Params& params, MemoryManager& mem, const char* fname, int) {
    const int nb = params.pk_bins > 0 ? params.pk_bins : 221;
    std::vector<double> k(nb), pk(nb);
    std::vector<int64_t> n(nb);
    // power.cu:189-227: one file per fold
    for (int fold = 0; fold <= params.pkFolds; ++fold) {
        check(mem.ctx,
              hgpm_power_spectrum_fold(mem.ctx, fold, nb, params.pk_log ? 1 : 0, k.data(), pk.data(), n.data()),
              "GetPowerSpectrum");
        if (hgpm_write_pk_fold(fname, fold, nb, k.data(), pk.data(), n.data()) != HGPM_OK)
            die("GetPowerSpectrum", fname);
    }
}

void writeOutput(Params&, MemoryManager& mem, char* fname, int) {
    check(mem.ctx, hgpm_write_output(mem.ctx, fname), "writeOutput");
}

double get_fscal(double m_aa, double m_adot, double m_omega_cb) { return hgpm_get_fscal(m_aa, m_adot, m_omega_cb, 1); }

void Analysis(Params& params, MemoryManager& mem, Timestepper& ts, int step, const AnalysisHook& hook) {
    if (!params.do_analysis || step < 0 || step >= HGPM_MAX_STEPS || !params.analysis[step] || !hook) return;
    printf("Doing Analysis Step\n");
    const int64_t n = (int64_t)params.np * params.np * params.np;
    std::vector<float> rows((size_t)n * 7);
    check(mem.ctx, hgpm_analysis_rows(mem.ctx, rows.data()), "Analysis");
    hook(rows.data(), n, 7, step, ts.aa, ts.z);
}

void WriteAnalysisRows(const char* dir, const float* rows, int64_t n, int ncols, int step) {
    char fname[2 * HGPM_PATH_MAX];
    snprintf(fname, sizeof(fname), "%s/analysis.%d", (dir && dir[0]) ? dir : ".", step);
    FILE* fp = fopen(fname, "wb");
    if (!fp) die("Analysis", fname);
    fwrite(rows, sizeof(float) * ncols, (size_t)n, fp);
    fclose(fp);
}

void RunSteps(Params&, MemoryManager& mem, Timestepper& ts, int nsteps) {
    hgpm_timestepper t = ts.to_c();
    check(mem.ctx, hgpm_run_steps(mem.ctx, &t, nsteps), "RunSteps");
    ts.aa = t.aa;
    ts.z = t.z;
    ts.deltaT = t.deltaT;
    ts.adot = t.adot;
    ts.fscal = t.fscal;
}

void printTimers(CPUTimer_t init, CPUTimer_t total) {
    // timers.cpp:52-61 prints per-phase totals; here the init and total wall
    // time (per-kernel device times come from hgpm_phase_times)
    printf("\n=========\nTIMERS\n");
    printf("   init: %g ms\n", (double)init * 1e-3);
    printf("   total: %g ms\n", (double)total * 1e-3);
}

}  // namespace serial
}  // namespace HACCGPM
