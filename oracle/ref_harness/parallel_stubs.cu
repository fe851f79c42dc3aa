// parallel_stubs.cu — definitions of the multi-rank (MPI/SWFFT) symbols that
// the reference's serial translation units reference but its serial path
// never calls.  TEST INFRASTRUCTURE ONLY (reference harness).  Each aborts
// on the host if it is ever reached.
#include <cstdio>
#include <cstdlib>

#include "haccgpm.hpp"

static void not_built(const char* what) {
    fprintf(stderr, "refpm: %s is part of the multi-rank path, not built in this harness\n", what);
    abort();
}

namespace HACCGPM {
namespace parallel {
GridExchange::GridExchange(int3, int3, int3, int, int, int, int, int) { not_built("GridExchange"); }
void GridExchange::fill(float4*, int) { not_built("GridExchange::fill"); }
void GridExchange::resolve(float*, int) { not_built("GridExchange::resolve"); }
void TransferParticles(Params&, MemoryManager&, int) { not_built("TransferParticles"); }
void forward_fft(deviceFFT_t*, int, int) { not_built("parallel::forward_fft"); }
void backward_fft(deviceFFT_t*, int, int) { not_built("parallel::backward_fft"); }
void printTimingStats(const char*, double) { not_built("printTimingStats"); }
void sendPower(int*, double*, int, int, int, int) { not_built("sendPower"); }
void timing_stats(CPUTimer_t, CPUTimer_t*, CPUTimer_t*, CPUTimer_t*) { not_built("timing_stats"); }
}  // namespace parallel
}  // namespace HACCGPM
