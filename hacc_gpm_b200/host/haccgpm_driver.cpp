// haccgpm_driver.cpp — the serial() run of HACC_GPM (src/driver_pm.cpp:32-163)
// on the B200 path, written against the drop-in header haccgpm.hpp.
//
//   haccgpm <params> [--fused]
//
// Writes what the reference's serial() writes: "<prefix>.params" (echo),
// "<prefix>.pk.ini.fold.0", "<prefix>.pk.<step>.fold.0" for PK_DUMP steps,
// "<prefix>.pk.fin.fold.0", and "<prefix>.particles.{ini,<step>,fin}" when
// DUMP_INIT / PARTICLE_DUMP / DUMP_FINAL ask for them (pk files for every
// fold up to PK_FOLDS), and with DO_ANALYSIS the analysis rows of the
// ANALYSIS_STEPS steps as "<ANALYSIS_DIR>/analysis.<step>".  The phase calls are
// the reference's, one per line of its loop; --fused runs the steps between
// two outputs through serial::RunSteps instead (same results, bit for bit:
// consecutive drifts fold into the kick kernel).
#include <cstdio>
#include <cstring>

#include "haccgpm.hpp"

static int serial(const char* params_file, bool fused) {
    using namespace HACCGPM;
    CPUTimer_t start = CPUTimer();
    Params params = read_params(params_file);
    serial::MemoryManager mem(params);
    serial::fft_cache_plan(params.ng);

    Timestepper ts(params);
    ts.setInitialZ(params.z_ini);
    ts.reverseHalfStep();
    CosmoClass cosmo(params);

    CPUTimer_t start_init = CPUTimer();
    serial::GenerateDisplacementIC(mem, cosmo, params, ts);
    CPUTimer_t init_time = CPUTimer() - start_init;

    serial::InitGreens(params, mem);
    char stepstr[400];
    snprintf(stepstr, sizeof(stepstr), "%s.pk.ini", params.prefix);
    serial::GetPowerSpectrum(params, mem, stepstr);
    if (params.dump_init) {
        snprintf(stepstr, sizeof(stepstr), "%s.particles.ini", params.prefix);
        serial::writeOutput(params, mem, stepstr);
    }
    ts.advanceHalfStep();

    for (int step = 0; step < params.lastStep;) {
        if (fused) {
            // run to the next step that writes something
            int end = step;
            while (end < params.lastStep - 1 && !params.pks[end] && !params.dumps[end] &&
                   !(params.do_analysis && params.analysis[end]))
                ++end;
            serial::RunSteps(params, mem, ts, end - step + 1);
            step = end;
        } else {
            serial::UpdatePositions(params, mem, ts, 0.5);
            serial::CIC(params, mem);
            serial::SolveGradient(params, mem);
            ts.advanceHalfStep();
            serial::UpdateVelocities(params, mem, ts);
            ts.advanceHalfStep();
            serial::UpdatePositions(params, mem, ts, 0.5);
        }
        if (params.pks[step]) {
            snprintf(stepstr, sizeof(stepstr), "%s.pk.%d", params.prefix, step);
            serial::GetPowerSpectrum(params, mem, stepstr);
        }
        if (params.dumps[step]) {
            snprintf(stepstr, sizeof(stepstr), "%s.particles.%d", params.prefix, step);
            serial::writeOutput(params, mem, stepstr);
        }
        // driver_pm.cpp:137-139: the analysis rows, here written for the
        // analysis code to read (ANALYSIS_DIR/analysis.<step>)
        serial::Analysis(params, mem, ts, step, [&](const float* rows, int64_t n, int ncols, int s, double, double) {
            serial::WriteAnalysisRows(params.analysis_dir, rows, n, ncols, s);
        });
        ++step;
    }

    snprintf(stepstr, sizeof(stepstr), "%s.pk.fin", params.prefix);
    serial::GetPowerSpectrum(params, mem, stepstr);
    if (params.dump_final) {
        snprintf(stepstr, sizeof(stepstr), "%s.particles.fin", params.prefix);
        serial::writeOutput(params, mem, stepstr);
    }
    serial::printTimers(init_time, CPUTimer() - start);
    return 0;
}

int main(int argc, char** argv) {
    const char* pfile = nullptr;
    bool fused = false;
    for (int i = 1; i < argc; ++i) {
        if (!strcmp(argv[i], "--fused")) fused = true;
        else if (argv[i][0] == '+') continue;  // the reference's +nXX rank flag; one GPU here
        else pfile = argv[i];
    }
    if (!pfile) {
        printf("USAGE: haccgpm <params> [--fused]\n");
        return 1;
    }
    printf("\n=========\nRUNNING IN SERIAL MODE\n=========\n");
    return serial(pfile, fused);
}
