// harness.cu — drives the reference's own serial CUDA path (compiled from
// the HACC_GPM sources by oracle/Makefile) to produce parity fixtures.
// TEST INFRASTRUCTURE ONLY; never linked into the product.
//
// The sequence restates driver_pm.cpp:32-163 (serial()), which cannot be
// compiled here because it includes the absent SWFFT headers.
//
//   refpm run   <params>                    the serial() run loop as written
//   refpm load  <params> <ics> <n> <out>    x,v from <ics> (writeOutput layout),
//                                           writes <out>.rho (float ng^3, Re of
//                                           d_grid after serial::CIC),
//                                           <out>.force (float 3 x ng^3 from
//                                           d_grad after serial::SolveGradient),
//                                           <out>.pk.ini.fold.0, then n steps of
//                                           the loop and <out>.fin (x,v dump),
//                                           <out>.pk.fin.fold.0
//   refpm noise <params> <out>              the cuRAND white noise of
//                                           GenerateFourierAmplitudes (float np^3)
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

// ic_kernels.hpp includes haccgpm.hpp (which has no include guard)
#include "initial_conditions/ic_kernels.hpp"

using namespace HACCGPM;

static void die(const char* m) {
    fprintf(stderr, "refpm: %s\n", m);
    exit(2);
}

static void write_floats(const char* path, const float* p, size_t n) {
    FILE* f = fopen(path, "wb");
    if (!f) die("cannot write output");
    fwrite(p, sizeof(float), n, f);
    fclose(f);
}

static int run(const char* pfile) {
    Params params = read_params(pfile);
    serial::MemoryManager mem(params);
    serial::fft_cache_plan(params.ng);
    Timestepper ts(params);
    ts.setInitialZ(params.z_ini);
    ts.reverseHalfStep();
    CosmoClass cosmo(params);
    serial::GenerateDisplacementIC(mem, cosmo, params, ts);
    serial::InitGreens(params, mem);
    char buf[400];
    snprintf(buf, sizeof(buf), "%s.pk.ini", params.prefix);
    serial::GetPowerSpectrum(params, mem, buf);
    if (params.dump_init) {
        snprintf(buf, sizeof(buf), "%s.particles.ini", params.prefix);
        serial::writeOutput(params, mem, buf);
    }
    ts.advanceHalfStep();
    for (int step = 0; step < params.lastStep; step++) {
        serial::UpdatePositions(params, mem, ts, 0.5);
        serial::CIC(params, mem);
        serial::SolveGradient(params, mem);
        ts.advanceHalfStep();
        serial::UpdateVelocities(params, mem, ts);
        ts.advanceHalfStep();
        serial::UpdatePositions(params, mem, ts, 0.5);
        if (params.pks[step]) {
            snprintf(buf, sizeof(buf), "%s.pk.%d", params.prefix, step);
            serial::GetPowerSpectrum(params, mem, buf);
        }
        if (params.dumps[step]) {
            snprintf(buf, sizeof(buf), "%s.particles.%d", params.prefix, step);
            serial::writeOutput(params, mem, buf);
        }
    }
    snprintf(buf, sizeof(buf), "%s.pk.fin", params.prefix);
    serial::GetPowerSpectrum(params, mem, buf);
    if (params.dump_final) {
        snprintf(buf, sizeof(buf), "%s.particles.fin", params.prefix);
        serial::writeOutput(params, mem, buf);
    }
    return 0;
}

static int load(const char* pfile, const char* ics, int nsteps, const char* out) {
    Params params = read_params(pfile);
    serial::MemoryManager mem(params);
    serial::fft_cache_plan(params.ng);
    const size_t np3 = (size_t)params.np * params.np * params.np;
    const size_t ng3 = (size_t)params.ng * params.ng * params.ng;
    std::vector<float> xv(6 * np3);
    FILE* f = fopen(ics, "rb");
    if (!f || fread(xv.data(), sizeof(float), 6 * np3, f) != 6 * np3) die("cannot read ICs");
    fclose(f);
    cudaMemcpy(mem.d_pos, xv.data(), 12 * np3, cudaMemcpyHostToDevice);
    cudaMemcpy(mem.d_vel, xv.data() + 3 * np3, 12 * np3, cudaMemcpyHostToDevice);
    char buf[400];
    // step-0 fields from the loaded positions
    serial::CIC(params, mem);
    std::vector<float2> grid(ng3);
    cudaMemcpy(grid.data(), mem.d_grid, 8 * ng3, cudaMemcpyDeviceToHost);
    std::vector<float> rho(ng3);
    for (size_t i = 0; i < ng3; ++i) rho[i] = grid[i].x;
    snprintf(buf, sizeof(buf), "%s.rho", out);
    write_floats(buf, rho.data(), ng3);
    serial::SolveGradient(params, mem);
    std::vector<float4> grad(ng3);
    cudaMemcpy(grad.data(), mem.d_grad, 16 * ng3, cudaMemcpyDeviceToHost);
    std::vector<float> force(3 * ng3);
    for (size_t i = 0; i < ng3; ++i) {
        force[i] = grad[i].x;
        force[ng3 + i] = grad[i].y;
        force[2 * ng3 + i] = grad[i].z;
    }
    snprintf(buf, sizeof(buf), "%s.force", out);
    write_floats(buf, force.data(), 3 * ng3);
    snprintf(buf, sizeof(buf), "%s.pk.ini", out);
    serial::GetPowerSpectrum(params, mem, buf);
    // the run loop from the loaded state (driver_pm.cpp:63-65, 106-126)
    Timestepper ts(params);
    ts.setInitialZ(params.z_ini);
    ts.reverseHalfStep();
    ts.advanceHalfStep();
    for (int step = 0; step < nsteps; step++) {
        serial::UpdatePositions(params, mem, ts, 0.5);
        serial::CIC(params, mem);
        serial::SolveGradient(params, mem);
        ts.advanceHalfStep();
        serial::UpdateVelocities(params, mem, ts);
        ts.advanceHalfStep();
        serial::UpdatePositions(params, mem, ts, 0.5);
    }
    snprintf(buf, sizeof(buf), "%s.fin", out);
    serial::writeOutput(params, mem, buf);
    snprintf(buf, sizeof(buf), "%s.pk.fin", out);
    serial::GetPowerSpectrum(params, mem, buf);
    return 0;
}

static int noise(const char* pfile, const char* out) {
    Params params = read_params(pfile);
    serial::MemoryManager mem(params);
    const int np = params.np;
    const size_t np3 = (size_t)np * np * np;
    const int nb = (int)((np3 + params.blockSize - 1) / params.blockSize);
    launch_generate_rng(mem.d_grid, np, params.seed, nb, params.blockSize, 0);  // rng_initializer.cu:51-55
    std::vector<float2> g(np3);
    cudaMemcpy(g.data(), mem.d_grid, 8 * np3, cudaMemcpyDeviceToHost);
    std::vector<float> re(np3);
    for (size_t i = 0; i < np3; ++i) re[i] = g[i].x;
    write_floats(out, re.data(), np3);
    return 0;
}

// time: ICs as serial() makes them, then `warmup` + `nsteps` steps of the run
// loop; prints the CUDA-event time of the nsteps steps (the reference
// synchronises after every kernel, so events and wall clock agree).
static int time_steps(const char* pfile, int warmup, int nsteps) {
    Params params = read_params(pfile);
    serial::MemoryManager mem(params);
    serial::fft_cache_plan(params.ng);
    Timestepper ts(params);
    ts.setInitialZ(params.z_ini);
    ts.reverseHalfStep();
    CosmoClass cosmo(params);
    serial::GenerateDisplacementIC(mem, cosmo, params, ts);
    ts.advanceHalfStep();
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    for (int step = 0; step < warmup + nsteps; step++) {
        if (step == warmup) cudaEventRecord(a);
        serial::UpdatePositions(params, mem, ts, 0.5);
        serial::CIC(params, mem);
        serial::SolveGradient(params, mem);
        ts.advanceHalfStep();
        serial::UpdateVelocities(params, mem, ts);
        ts.advanceHalfStep();
        serial::UpdatePositions(params, mem, ts, 0.5);
    }
    cudaEventRecord(b);
    cudaEventSynchronize(b);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, b);
    fprintf(stderr, "REFPM_TIME ng=%d np=%d steps=%d ms_per_step=%.4f\n", params.ng, params.np, nsteps, ms / nsteps);
    return 0;
}

int main(int argc, char** argv) {
    if (argc >= 5 && !strcmp(argv[1], "time")) return time_steps(argv[2], atoi(argv[3]), atoi(argv[4]));
    if (argc >= 3 && !strcmp(argv[1], "run")) return run(argv[2]);
    if (argc >= 6 && !strcmp(argv[1], "load")) return load(argv[2], argv[3], atoi(argv[4]), argv[5]);
    if (argc >= 4 && !strcmp(argv[1], "noise")) return noise(argv[2], argv[3]);
    fprintf(stderr, "usage: refpm run <params> | load <params> <ics> <nsteps> <out> | noise <params> <out>\n");
    return 1;
}
