// cpu_pm.cpp — OpenMP C++ transcription of HACC_GPM's serial PM step.
//
// TEST AND CPU-BASELINE INFRASTRUCTURE ONLY.  The reference has no CPU or FFTW
// path; this program restates its serial CUDA routines on the host, in the
// reference's own layout and precision (float3 positions and velocities, a
// float complex grid, float atomics), so that bench.py can time "the
// reference's algorithm on the host cores".  It is never linked into the
// product.  Each routine cites the reference file:line it transcribes; the
// FFT is a project-written mixed-radix (2/3/4) Stockham transform from the
// DFT definition (the reference calls cuFFT, ffts.cu:271/423).
//
// usage: cpu_pm --ng N --np N --rl L --steps K --warmup W [--threads T]
//               [--zini z] [--zfin z] [--nsteps-total S] [--seed s]
//               [--load FILE --start-step S]
//               [--omega-cb x --omega-m x --omega-r x --f-nu x]
// --load reads x then v (float3, lattice order: writeOutput's layout,
// io.cu:12-44) instead of the seeded perturbed lattice, and the time stepper
// starts S steps into the run (2S half steps of timestepper.cpp:49-57).
// Prints one JSON line: per-step seconds of the timed steps.
#include <omp.h>

#include <chrono>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>
#include <string>
#include <vector>

typedef std::complex<float> cf;

struct F3 {
    float x, y, z;
};

// ---------------------------------------------------------------------------
// 1D FFT (Stockham, radices 4/2/3/5), forward sign -1, unnormalised
// ---------------------------------------------------------------------------
struct Fft1 {
    int n;
    std::vector<int> radices;
    std::vector<cf> tw;  // exp(-2 pi i m / n)
    explicit Fft1(int n_) : n(n_) {
        int m = n;
        while (m % 4 == 0) { radices.push_back(4); m /= 4; }
        while (m % 2 == 0) { radices.push_back(2); m /= 2; }
        while (m % 3 == 0) { radices.push_back(3); m /= 3; }
        while (m % 5 == 0) { radices.push_back(5); m /= 5; }
        if (m != 1) { fprintf(stderr, "unsupported FFT size %d\n", n); exit(2); }
        tw.resize(n);
        for (int k = 0; k < n; ++k) tw[k] = cf((float)cos(-2 * M_PI * k / n), (float)sin(-2 * M_PI * k / n));
    }
    // in-place on a (buffer a, scratch b), sign = -1 forward, +1 inverse
    void run(cf* a, cf* b, int sign) const {
        int ns = 1;
        cf* src = a;
        cf* dst = b;
        for (int r : radices) {
            const int nb = n / r;
            for (int j = 0; j < nb; ++j) {
                const int k = j % ns;
                cf v[5];
                for (int q = 0; q < r; ++q) v[q] = src[j + q * nb];
                if (ns > 1)
                    for (int q = 1; q < r; ++q) {
                        cf w = tw[q * k * (n / (ns * r))];
                        v[q] *= (sign < 0 ? w : std::conj(w));
                    }
                cf y[5];
                if (r == 5) {
                    // the radix-5 DFT from its definition (sum over the five inputs)
                    for (int q = 0; q < 5; ++q) {
                        cf acc = 0;
                        for (int t = 0; t < 5; ++t) {
                            const double ang = sign * 2 * M_PI * (double)((q * t) % 5) / 5.0;
                            acc += v[t] * cf((float)cos(ang), (float)sin(ang));
                        }
                        y[q] = acc;
                    }
                } else if (r == 2) {
                    y[0] = v[0] + v[1];
                    y[1] = v[0] - v[1];
                } else if (r == 4) {
                    cf a0 = v[0] + v[2], a1 = v[0] - v[2], b0 = v[1] + v[3], d = v[1] - v[3];
                    cf b1 = sign < 0 ? cf(d.imag(), -d.real()) : cf(-d.imag(), d.real());
                    y[0] = a0 + b0;
                    y[2] = a0 - b0;
                    y[1] = a1 + b1;
                    y[3] = a1 - b1;
                } else {
                    const float s3 = 0.86602540378443864676f;
                    cf t1 = v[1] + v[2];
                    cf t2 = v[0] - 0.5f * t1;
                    cf d = (v[1] - v[2]) * s3;
                    cf rt = sign < 0 ? cf(d.imag(), -d.real()) : cf(-d.imag(), d.real());
                    y[0] = v[0] + t1;
                    y[1] = t2 + rt;
                    y[2] = t2 - rt;
                }
                const int base = (j / ns) * ns * r + k;
                for (int q = 0; q < r; ++q) dst[base + q * ns] = y[q];
            }
            std::swap(src, dst);
            ns *= r;
        }
        if (src != a) memcpy(a, src, sizeof(cf) * n);
    }
};

// 3D C2C in place, axis by axis, lines gathered into per-thread buffers
static void fft3(std::vector<cf>& g, int n, int sign, const Fft1& f) {
    const size_t n2 = (size_t)n * n;
    // z lines (contiguous)
#pragma omp parallel
    {
        std::vector<cf> scratch(n);
#pragma omp for schedule(static)
        for (long l = 0; l < (long)n2; ++l) f.run(&g[(size_t)l * n], scratch.data(), sign);
    }
    // y lines: for each x plane, blocks of z columns
    const int B = 16;
#pragma omp parallel
    {
        std::vector<cf> buf((size_t)n * B), scratch(n), line(n);
#pragma omp for schedule(static) collapse(2)
        for (int x = 0; x < n; ++x)
            for (int zb = 0; zb < n; zb += B) {
                const int w = std::min(B, n - zb);
                for (int y = 0; y < n; ++y)
                    for (int c = 0; c < w; ++c) buf[(size_t)c * n + y] = g[(size_t)x * n2 + (size_t)y * n + zb + c];
                for (int c = 0; c < w; ++c) f.run(&buf[(size_t)c * n], scratch.data(), sign);
                for (int y = 0; y < n; ++y)
                    for (int c = 0; c < w; ++c) g[(size_t)x * n2 + (size_t)y * n + zb + c] = buf[(size_t)c * n + y];
            }
    }
    // x lines
#pragma omp parallel
    {
        std::vector<cf> buf((size_t)n * B), scratch(n);
#pragma omp for schedule(static) collapse(2)
        for (int y = 0; y < n; ++y)
            for (int zb = 0; zb < n; zb += B) {
                const int w = std::min(B, n - zb);
                for (int x = 0; x < n; ++x)
                    for (int c = 0; c < w; ++c) buf[(size_t)c * n + x] = g[(size_t)x * n2 + (size_t)y * n + zb + c];
                for (int c = 0; c < w; ++c) f.run(&buf[(size_t)c * n], scratch.data(), sign);
                for (int x = 0; x < n; ++x)
                    for (int c = 0; c < w; ++c) g[(size_t)x * n2 + (size_t)y * n + zb + c] = buf[(size_t)c * n + x];
            }
    }
}

// ---------------------------------------------------------------------------
// PM routines
// ---------------------------------------------------------------------------
// UpdatePosKernel (update_positions_pm.cu:3-20)
static void update_positions(std::vector<F3>& x, const std::vector<F3>& v, float pf, float ng) {
#pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)x.size(); ++i) {
        F3 p = x[i];
        p.x += v[i].x * pf;
        p.y += v[i].y * pf;
        p.z += v[i].z * pf;
        p.x = fmodf(p.x + ng, ng);
        p.y = fmodf(p.y + ng, ng);
        p.z = fmodf(p.z + ng, ng);
        x[i] = p;
    }
}

// cudaMemset + CICKernel (cic_pm.cu:46-87, 142-147)
static void cic(std::vector<cf>& grid, const std::vector<F3>& x, int ng, float mass) {
    float* g = reinterpret_cast<float*>(grid.data());
    const size_t nc = (size_t)ng * ng * ng;
#pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)nc; ++i) grid[i] = cf(0.f, 0.f);
#pragma omp parallel for schedule(static)
    for (long p = 0; p < (long)x.size(); ++p) {
        const F3 q = x[p];
        int i = (int)q.x, j = (int)q.y, k = (int)q.z;
        float dfx = q.x - (float)i, dfy = q.y - (float)j, dfz = q.z - (float)k;
        for (int a = 0; a < 2; ++a)
            for (int b = 0; b < 2; ++b)
                for (int c = 0; c < 2; ++c) {
                    int nx = (i + a) % ng, ny = (j + b) % ng, nz = (k + c) % ng;
                    size_t idx = ((size_t)nx * ng + ny) * ng + nz;
                    float dx = a ? dfx : 1 - dfx, dy = b ? dfy : 1 - dfy, dz = c ? dfz : 1 - dfz;
                    float mul = dx * dy * dz * mass;
#pragma omp atomic
                    g[2 * idx] += mul;
                }
    }
}

static inline float kmode(int i, int ng, double d) {
    float l = (float)i;
    if (i > ng / 2 - 1) l = -(float)(ng - i);
    return (float)(l * d);
}

// SolveGradient one-grid (solver.cpp:144-170) with copyGridToFloat4
// (combine.cu:21-34), kspace_solve_gradient (kspace_solver.cu:55-90),
// calcGreens (calcGreens.hpp:11-25), getRealGrid
// (transform_density_field_initializer.cu:14-28).  grad is float4 per cell.
static void solve_gradient(std::vector<cf>& grid, std::vector<float>& grad, std::vector<cf>& rho, int ng,
                           const Fft1& f) {
    const size_t nc = (size_t)ng * ng * ng;
    fft3(grid, ng, -1, f);
#pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)nc; ++i) rho[i] = grid[i];
    std::vector<float> sk(ng);
    std::vector<double> cq(ng);
    const double d = 2 * M_PI / (double)ng;
    const float df = (float)((2 * M_PI) / ((float)ng));
    for (int i = 0; i < ng; ++i) {
        sk[i] = sinf(kmode(i, ng, d));
        cq[i] = (double)cosf((float)i * df);
    }
    const double coeff = 0.5 / ((double)ng * ng * ng);
    for (int dim = 0; dim < 3; ++dim) {
#pragma omp parallel for schedule(static)
        for (long idx = 0; idx < (long)nc; ++idx) {
            const int ix = (int)(idx / ((size_t)ng * ng)), iy = (int)((idx / ng) % ng), iz = (int)(idx % ng);
            double greens = 0.0;
            if (ix || iy || iz) greens = coeff / (cq[ix] + cq[iy] + cq[iz] - 3.0);
            const int id = dim == 0 ? ix : (dim == 1 ? iy : iz);
            const float c = (float)(-sk[id] * greens);
            const cf r = rho[idx];
            grid[idx] = cf(-c * r.imag(), c * r.real());
        }
        fft3(grid, ng, +1, f);
#pragma omp parallel for schedule(static)
        for (long idx = 0; idx < (long)nc; ++idx) grad[4 * idx + dim] = grid[idx].real();
    }
}

// ICICKernel (icic_pm.cu:72-127)
static void update_velocities(std::vector<F3>& v, const std::vector<float>& grad, const std::vector<F3>& x, int ng,
                              double deltaT, double fscal) {
#pragma omp parallel for schedule(static)
    for (long p = 0; p < (long)x.size(); ++p) {
        const F3 q = x[p];
        int i = (int)q.x, j = (int)q.y, k = (int)q.z;
        float dfx = q.x - (float)i, dfy = q.y - (float)j, dfz = q.z - (float)k;
        float dvx = 0, dvy = 0, dvz = 0;
        for (int a = 0; a < 2; ++a)
            for (int b = 0; b < 2; ++b)
                for (int c = 0; c < 2; ++c) {
                    int nx = (i + a) % ng, ny = (j + b) % ng, nz = (k + c) % ng;
                    size_t idx = ((size_t)nx * ng + ny) * ng + nz;
                    float dx = a ? dfx : 1 - dfx, dy = b ? dfy : 1 - dfy, dz = c ? dfz : 1 - dfz;
                    float mul = (float)((double)(dx * dy * dz) * deltaT * fscal);
                    dvx += mul * grad[4 * idx + 0];
                    dvy += mul * grad[4 * idx + 1];
                    dvz += mul * grad[4 * idx + 2];
                }
        v[p].x += dvx;
        v[p].y += dvy;
        v[p].z += dvz;
    }
}

// time stepper (timestepper.cpp:13-68) for flat LCDM with radiation
struct TS {
    double aa, deltaT, adot, fscal, om_cb, om_m, om_r, fnu;
    double get_adot(double a) const {
        double tmp = om_cb + (1.0 + fnu) * om_r / a + (1.0 - om_m - (1.0 + fnu) * om_r);
        return sqrt(tmp / a);
    }
    void upd() {
        adot = get_adot(aa);
        float dtdy = aa / (aa * adot);
        fscal = 1.5 * om_cb * dtdy * (1.0 / aa);
    }
    void half() { aa += deltaT * 0.5; upd(); }
    float pf(float frac) const { return (float)((deltaT / (aa * aa * adot)) * frac); }
};

static double arg_d(int argc, char** argv, const char* k, double def) {
    for (int i = 1; i + 1 < argc; ++i)
        if (!strcmp(argv[i], k)) return atof(argv[i + 1]);
    return def;
}

int main(int argc, char** argv) {
    const int ng = (int)arg_d(argc, argv, "--ng", 64);
    const int np = (int)arg_d(argc, argv, "--np", ng);
    const double rl = arg_d(argc, argv, "--rl", ng);
    const int steps = (int)arg_d(argc, argv, "--steps", 2);
    const int warmup = (int)arg_d(argc, argv, "--warmup", 0);
    const int threads = (int)arg_d(argc, argv, "--threads", 0);
    const double zini = arg_d(argc, argv, "--zini", 50.0);
    const double zfin = arg_d(argc, argv, "--zfin", 0.0);
    const int ntot = (int)arg_d(argc, argv, "--nsteps-total", 100);
    const int seed = (int)arg_d(argc, argv, "--seed", 21082001);
    const char* load = nullptr;
    for (int i = 1; i + 1 < argc; ++i)
        if (!strcmp(argv[i], "--load")) load = argv[i + 1];
    const int start_step = (int)arg_d(argc, argv, "--start-step", 0);
    if (threads > 0) omp_set_num_threads(threads);
    (void)rl;
    const size_t npart = (size_t)np * np * np, nc = (size_t)ng * ng * ng;
    std::vector<F3> x(npart), v(npart);
    if (load) {
        FILE* f = fopen(load, "rb");
        if (!f || fread(x.data(), sizeof(F3), npart, f) != npart || fread(v.data(), sizeof(F3), npart, f) != npart) {
            fprintf(stderr, "cpu_pm: cannot read %s\n", load);
            return 2;
        }
        fclose(f);
    } else
    // seeded perturbed lattice in Lagrangian order (synthetic ICs)
#pragma omp parallel
    {
        std::mt19937 gen(seed + omp_get_thread_num());
        std::normal_distribution<float> nd(0.f, 1.f);
#pragma omp for schedule(static)
        for (long i = 0; i < (long)npart; ++i) {
            int qx = (int)(i / ((size_t)np * np)), qy = (int)((i / np) % np), qz = (int)(i % np);
            float r = (float)ng / (float)np;
            x[i].x = fmodf(qx * r + 0.3f * nd(gen) + ng, ng);
            x[i].y = fmodf(qy * r + 0.3f * nd(gen) + ng, ng);
            x[i].z = fmodf(qz * r + 0.3f * nd(gen) + ng, ng);
            v[i].x = nd(gen);
            v[i].y = nd(gen);
            v[i].z = nd(gen);
        }
    }
    std::vector<cf> grid(nc), rho(nc);
    std::vector<float> grad(4 * nc);
    Fft1 f(ng);
    TS ts;
    ts.om_cb = arg_d(argc, argv, "--omega-cb", 0.31);
    ts.om_m = arg_d(argc, argv, "--omega-m", 0.31);
    ts.om_r = arg_d(argc, argv, "--omega-r", 5.3e-5);
    ts.fnu = arg_d(argc, argv, "--f-nu", 0.69);
    ts.deltaT = ((1 / (zfin + 1)) - (1 / (zini + 1))) / (double)ntot;
    ts.aa = 1.0 / (zini + 1.0);
    ts.upd();
    for (int s = 0; s < 2 * start_step; ++s) ts.half();
    const float gp = (float)ng / (float)np;
    const float mass = gp * gp * gp;
    std::vector<double> times;
    for (int s = 0; s < warmup + steps; ++s) {
        auto t0 = std::chrono::steady_clock::now();
        update_positions(x, v, ts.pf(0.5f), (float)ng);
        cic(grid, x, ng, mass);
        solve_gradient(grid, grad, rho, ng, f);
        ts.half();
        update_velocities(v, grad, x, ng, ts.deltaT, ts.fscal);
        ts.half();
        update_positions(x, v, ts.pf(0.5f), (float)ng);
        auto t1 = std::chrono::steady_clock::now();
        if (s >= warmup) times.push_back(std::chrono::duration<double>(t1 - t0).count());
    }
    double sum = 0;
    for (double t : times) sum += t;
    double chk = 0;
    for (size_t i = 0; i < npart; i += npart / 97 + 1) chk += x[i].x + x[i].y + x[i].z;
    printf("{\"ng\": %d, \"np\": %d, \"threads\": %d, \"steps\": %d, \"sec_per_step\": %.6f, \"checksum\": %.6f}\n", ng,
           np, omp_get_max_threads(), (int)times.size(), times.empty() ? 0.0 : sum / times.size(), chk);
    return 0;
}
