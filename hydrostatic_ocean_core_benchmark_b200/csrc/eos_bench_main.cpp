// eos_bench_b200 [n] [linear|seos|teos10] [n_repeat]
//
// Standalone equation-of-state bench over the C ABI (oc_density), with the
// command line, inputs, timing rule and output line of the reference's bench
// (libs/cuda/src/eos_bench.cu:131-180):
//   - n cells (default 3,000,000) with T = 5 + 15 (i mod 977) / 977,
//     S = 33 + 3 (i mod 733) / 733, z = 5000 (i mod 521) / 521, i = 1..n;
//   - 3 untimed runs, then n_repeat (default 20) timed runs of one launch plus
//     a device synchronisation: median and MAD of the wall times;
//   - checksum = sum of every max(1, n / 1000)-th result, in index order;
//   - "eos=... n=... wall=... mad=... checksum=..." as the reference prints it,
//     then the same runs timed with CUDA events and the achieved bandwidth at
//     32 B per cell (three reads, one write).
// The linear EOS uses the reference's defaults rho0 = 1025, alpha_T = 2e-4,
// beta_S = 7.4e-4, T0 = 10, S0 = 35.

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "ocean_b200.h"

namespace {

double median_of(std::vector<double> v) {
    std::sort(v.begin(), v.end());
    const size_t m = v.size();
    return m % 2 ? v[m / 2] : 0.5 * (v[m / 2 - 1] + v[m / 2]);
}

}  // namespace

int main(int argc, char** argv) {
    const long long n = argc > 1 ? std::atoll(argv[1]) : 3000000;
    const std::string kind = argc > 2 ? argv[2] : "teos10";
    const int n_repeat = argc > 3 ? std::atoi(argv[3]) : 20;
    int eos = -1;
    if (kind == "linear") eos = OC_EOS_LINEAR;
    else if (kind == "seos") eos = OC_EOS_SEOS;
    else if (kind == "teos10") eos = OC_EOS_TEOS10;
    if (eos < 0 || n < 1 || n_repeat < 1) {
        std::fprintf(stderr, "FATAL: unknown eos %s (or n, n_repeat < 1)\n", kind.c_str());
        return 1;
    }
    std::vector<double> ht(n), hs(n), hz(n), hrho(n);
    for (long long i = 1; i <= n; ++i) {
        ht[i - 1] = 5.0 + 15.0 * double(i % 977) / 977.0;
        hs[i - 1] = 33.0 + 3.0 * double(i % 733) / 733.0;
        hz[i - 1] = 5000.0 * double(i % 521) / 521.0;
    }
    const size_t bytes = size_t(n) * sizeof(double);
    double *dt = nullptr, *ds = nullptr, *dz = nullptr, *drho = nullptr;
    for (double** p : {&dt, &ds, &dz, &drho})
        if (cudaMalloc(p, bytes) != cudaSuccess) {
            std::fprintf(stderr, "FATAL: cudaMalloc failed\n");
            return 1;
        }
    cudaMemcpy(dt, ht.data(), bytes, cudaMemcpyHostToDevice);
    cudaMemcpy(ds, hs.data(), bytes, cudaMemcpyHostToDevice);
    cudaMemcpy(dz, hz.data(), bytes, cudaMemcpyHostToDevice);
    auto launch = [&]() {
        const int rc = oc_density(eos, 1025.0, 2.0e-4, 7.4e-4, 10.0, 35.0, dt, ds, dz, drho, n, nullptr);
        if (rc) {
            std::fprintf(stderr, "FATAL: oc_density failed (%d)\n", rc);
            std::exit(1);
        }
    };
    for (int w = 0; w < 3; ++w) {
        launch();
        cudaDeviceSynchronize();
    }
    std::vector<double> samples;
    for (int r = 0; r < n_repeat; ++r) {
        const auto t0 = std::chrono::steady_clock::now();
        launch();
        cudaDeviceSynchronize();
        const auto t1 = std::chrono::steady_clock::now();
        samples.push_back(std::chrono::duration<double>(t1 - t0).count());
    }
    const double wall = median_of(samples);
    std::vector<double> dev;
    for (double s : samples) dev.push_back(std::fabs(s - wall));
    const double wall_mad = median_of(dev);
    // device time of the same launches
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    std::vector<double> dev_ms;
    for (int r = 0; r < n_repeat; ++r) {
        cudaEventRecord(e0);
        launch();
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, e0, e1);
        dev_ms.push_back(ms);
    }
    const double kernel_s = median_of(dev_ms) * 1e-3;
    const cudaError_t err = cudaMemcpy(hrho.data(), drho, bytes, cudaMemcpyDeviceToHost);
    if (err != cudaSuccess) {
        std::fprintf(stderr, "FATAL: %s\n", cudaGetErrorString(err));
        return 1;
    }
    double chk = 0.0;
    const long long step = std::max(1LL, n / 1000);
    for (long long i = 0; i < n; i += step) chk += hrho[i];
    std::printf("eos=%10s n=%10lld wall=%13.6e mad=%13.6e checksum=%13.6e\n", kind.c_str(), n, wall, wall_mad, chk);
    std::printf("kernel=%13.6e s achieved=%.1f GB/s (32 B per cell)\n", kernel_s, 32.0 * double(n) / kernel_s / 1e9);
    for (double* p : {dt, ds, dz, drho}) cudaFree(p);
    return 0;
}
