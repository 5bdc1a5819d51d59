// Test harness (built by tests/test_gpu_parity.py): the FP64 reciprocal of the folded-division
// solver forms (rcp_ in pip_physics.cuh: a hardware seed refined by two Newton-Raphson steps)
// against the IEEE division 1.0 / x on the device, over seeded normal x whose reciprocal is
// normal: mantissas uniform, exponents uniform in [-1000, 1000], both signs, plus the powers
// of two and their neighbours.  Prints the largest difference in ulps of the IEEE quotient
// and how many reciprocals differ from it at all.
#include <cstdio>
#include <cstdlib>
#include <cstdint>
#include <cstring>
#include <cmath>
#include <vector>
#include <random>

#include "../pip_b200/csrc/pip_physics.cuh"

__global__ void run(int n, const double *x, double *r_nr, double *r_ieee) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  r_nr[i] = pip::rcp_(x[i]);
  r_ieee[i] = __drcp_rn(x[i]);
}

static int64_t ordered(double v) {
  int64_t b;
  std::memcpy(&b, &v, sizeof b);
  return b < 0 ? INT64_MIN - b : b;
}

int main(int argc, char **argv) {
  const int n = argc > 1 ? atoi(argv[1]) : 1 << 22;
  std::mt19937_64 g(2024);
  std::uniform_real_distribution<double> M(1.0, 2.0);
  std::uniform_int_distribution<int> E(-1000, 1000);
  std::vector<double> x(n);
  for (int i = 0; i < n; ++i) {
    double v;
    if (i < 6000) {                       // powers of two and their neighbours
      v = std::ldexp(1.0, (i / 3) % 2001 - 1000);
      if (i % 3 == 1) v = std::nextafter(v, 0.0);
      if (i % 3 == 2) v = std::nextafter(v, 1e308);
    } else {
      v = std::ldexp(M(g), E(g));
    }
    x[i] = (i & 1) ? -v : v;
  }
  double *dx, *dn, *di;
  cudaMalloc(&dx, sizeof(double) * n);
  cudaMalloc(&dn, sizeof(double) * n);
  cudaMalloc(&di, sizeof(double) * n);
  cudaMemcpy(dx, x.data(), sizeof(double) * n, cudaMemcpyHostToDevice);
  run<<<(n + 255) / 256, 256>>>(n, dx, dn, di);
  if (cudaDeviceSynchronize() != cudaSuccess) {
    printf("ERROR kernel\n");
    return 1;
  }
  std::vector<double> rn(n), ri(n);
  cudaMemcpy(rn.data(), dn, sizeof(double) * n, cudaMemcpyDeviceToHost);
  cudaMemcpy(ri.data(), di, sizeof(double) * n, cudaMemcpyDeviceToHost);
  int64_t worst = 0;
  long differ = 0, nonfinite = 0;
  for (int i = 0; i < n; ++i) {
    if (!std::isfinite(rn[i])) ++nonfinite;
    const int64_t d = std::llabs(ordered(rn[i]) - ordered(ri[i]));
    if (d) ++differ;
    if (d > worst) worst = d;
  }
  printf("values %d max_ulp %lld differ %ld nonfinite %ld\n", n, (long long)worst, differ, nonfinite);
  return 0;
}
