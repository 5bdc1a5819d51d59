// Test harness (built by tests/test_gpu_mixed.py): the paired FP32 Riemann solvers of
// pip_pair.cuh against the scalar reciprocal forms of pip_physics.cuh on the device, over
// seeded random face states of four kinds (unrelated states, including supersonic faces;
// nearby states; exact mirror pairs, a reflecting wall's face with vn and Bn negated; a
// near-zero Bn).  Prints, per kind, the largest difference relative to the face's flux
// scale (p + rho vn^2 + |B|^2 of the larger side: a wall's fluxes of mass and energy vanish,
// so the flux itself is no scale), the side counts, and the faces above 1e-4.
#include <cstdio>
#include <cstdlib>
#include <cmath>
#include <vector>
#include <random>

#include "../pip_b200/csrc/pip_pair.cuh"

using namespace pip;

// Which side of the HLLD fan a face lies in, as hlld_flux_rcp decides it from the fast
// speeds: 0 supersonic to the right (F_L), 1 to the left (F_R), 3 subsonic.
__device__ int hlld_side(const float (&v_l)[8], const float (&v_r)[8], float gm) {
  const float b2l = v_l[5] * v_l[5] + v_l[6] * v_l[6] + v_l[7] * v_l[7];
  const float b2r = v_r[5] * v_r[5] + v_r[6] * v_r[6] + v_r[7] * v_r[7];
  float f1 = gm * v_l[4];
  const float vfl = sqrtf(((f1 + b2l) + sqrtf(fmaxf((f1 + b2l) * (f1 + b2l) - 4.f * f1 * v_l[5] * v_l[5], 0.f))) / (2.f * v_l[0]));
  f1 = gm * v_r[4];
  const float vfr = sqrtf(((f1 + b2r) + sqrtf(fmaxf((f1 + b2r) * (f1 + b2r) - 4.f * f1 * v_r[5] * v_r[5], 0.f))) / (2.f * v_r[0]));
  const float sl = fminf(v_l[1], v_r[1]) - fmaxf(vfl, vfr);
  const float sr = fmaxf(v_l[1], v_r[1]) + fmaxf(vfl, vfr);
  if (sl >= 0.f) return 0;
  if (sr <= 0.f) return 1;
  return 3;
}

__global__ void run(int n, const float *vl, const float *vr, float gm, float igm1, float *fd_s,
                    float *fd_p, float *fc_s, float *fc_p, int *br) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float a[8], b[8], o[8], q[8];
  for (int k = 0; k < 8; ++k) {
    a[k] = vl[8 * i + k];
    b[k] = vr[8 * i + k];
  }
  hlld_flux_rcp<float, 8>(a, b, o, gm, igm1, 0.0f);
  pair::hlld_flux(a, b, q, gm, igm1);
  for (int k = 0; k < 8; ++k) {
    fd_s[8 * i + k] = o[k];
    fd_p[8 * i + k] = q[k];
  }
  br[i] = hlld_side(a, b, gm);
  float ha[5], hb[5], ho[5], hq[5];
  const int m[5] = {0, 1, 2, 3, 4};
  for (int k = 0; k < 5; ++k) {
    ha[k] = a[m[k]];
    hb[k] = b[m[k]];
  }
  hllc_flux_rcp<float>(ha, hb, ho, gm, igm1);
  pair::hllc_flux(ha, hb, hq, gm, igm1);
  for (int k = 0; k < 5; ++k) {
    fc_s[5 * i + k] = ho[k];
    fc_p[5 * i + k] = hq[k];
  }
}

int main(int argc, char **argv) {
  const int n = argc > 1 ? atoi(argv[1]) : 1 << 20;
  const float gm = 5.f / 3.f, igm1 = 1.f / (gm - 1.f);
  std::mt19937 g(12345);
  std::uniform_real_distribution<float> U(-1.f, 1.f);
  std::vector<float> vl(8 * (size_t)n), vr(8 * (size_t)n);
  for (int i = 0; i < n; ++i) {
    const int kind = i % 4;    // 0 random, 1 near states, 2 mirror pair, 3 weak Bn
    float *l = &vl[8 * (size_t)i], *r = &vr[8 * (size_t)i];
    l[0] = 1.f + 0.9f * U(g);
    l[4] = 0.5f + 0.45f * U(g);
    for (int k : {1, 2, 3}) l[k] = (kind == 0 ? 2.f : 0.5f) * U(g);
    for (int k : {5, 6, 7}) l[k] = U(g);
    if (kind == 0 && i % 8 == 0) l[1] += 6.f * U(g);     // supersonic faces
    for (int k = 0; k < 8; ++k) r[k] = l[k];
    if (kind == 0) {
      r[0] = 1.f + 0.9f * U(g);
      r[4] = 0.5f + 0.45f * U(g);
      for (int k : {1, 2, 3, 5, 6, 7}) r[k] = l[k] + U(g);
    } else if (kind == 1) {
      for (int k = 0; k < 8; ++k) r[k] = l[k] * (1.f + 0.05f * U(g));
    } else if (kind == 2) {
      r[1] = -l[1];
      r[5] = -l[5];
    } else {
      l[5] = 1e-4f * U(g);
      r[5] = l[5];
      for (int k : {0, 1, 2, 3, 4, 6, 7}) r[k] = l[k] * (1.f + 0.3f * U(g));
    }
  }
  float *d_vl, *d_vr, *fds, *fdp, *fcs, *fcp;
  int *d_br;
  cudaMalloc(&d_vl, sizeof(float) * vl.size());
  cudaMalloc(&d_vr, sizeof(float) * vr.size());
  cudaMalloc(&fds, sizeof(float) * 8 * (size_t)n);
  cudaMalloc(&fdp, sizeof(float) * 8 * (size_t)n);
  cudaMalloc(&fcs, sizeof(float) * 5 * (size_t)n);
  cudaMalloc(&fcp, sizeof(float) * 5 * (size_t)n);
  cudaMalloc(&d_br, sizeof(int) * (size_t)n);
  cudaMemcpy(d_vl, vl.data(), sizeof(float) * vl.size(), cudaMemcpyHostToDevice);
  cudaMemcpy(d_vr, vr.data(), sizeof(float) * vr.size(), cudaMemcpyHostToDevice);
  run<<<(n + 255) / 256, 256>>>(n, d_vl, d_vr, gm, igm1, fds, fdp, fcs, fcp, d_br);
  if (cudaDeviceSynchronize() != cudaSuccess) {
    printf("ERROR kernel\n");
    return 1;
  }
  std::vector<float> hs(8 * (size_t)n), hp(8 * (size_t)n), cs(5 * (size_t)n), cp(5 * (size_t)n);
  std::vector<int> br(n);
  cudaMemcpy(hs.data(), fds, sizeof(float) * hs.size(), cudaMemcpyDeviceToHost);
  cudaMemcpy(hp.data(), fdp, sizeof(float) * hp.size(), cudaMemcpyDeviceToHost);
  cudaMemcpy(cs.data(), fcs, sizeof(float) * cs.size(), cudaMemcpyDeviceToHost);
  cudaMemcpy(cp.data(), fcp, sizeof(float) * cp.size(), cudaMemcpyDeviceToHost);
  cudaMemcpy(br.data(), d_br, sizeof(int) * br.size(), cudaMemcpyDeviceToHost);
  // per face: largest |difference| / largest |flux| of the face
  double wd[4] = {0, 0, 0, 0}, wc[4] = {0, 0, 0, 0};
  long nd[4] = {0, 0, 0, 0}, above_d = 0, above_c = 0, nonfinite = 0;
  double mirror_d = 0.0, mirror_c = 0.0;
  for (int i = 0; i < n; ++i) {
    const int kind = i % 4;
    const float *l = &vl[8 * (size_t)i], *r = &vr[8 * (size_t)i];
    auto scale = [](const float *v, bool mag) {
      double s = std::fabs(v[4]) + std::fabs(v[0]) * v[1] * v[1];
      if (mag) s += (double)v[5] * v[5] + (double)v[6] * v[6] + (double)v[7] * v[7];
      return s;
    };
    const double sd = std::fmax(scale(l, true), scale(r, true));
    const double sh = std::fmax(scale(l, false), scale(r, false));
    double e = 0;
    for (int k = 0; k < 8; ++k) {
      if (!std::isfinite(hs[8 * (size_t)i + k]) || !std::isfinite(hp[8 * (size_t)i + k])) ++nonfinite;
      e = std::fmax(e, std::fabs((double)hs[8 * (size_t)i + k] - hp[8 * (size_t)i + k]));
    }
    const double rd = e / sd;
    double ec = 0;
    for (int k = 0; k < 5; ++k) {
      if (!std::isfinite(cs[5 * (size_t)i + k]) || !std::isfinite(cp[5 * (size_t)i + k])) ++nonfinite;
      ec = std::fmax(ec, std::fabs((double)cs[5 * (size_t)i + k] - cp[5 * (size_t)i + k]));
    }
    const double rc = ec / sh;
    wd[kind] = std::fmax(wd[kind], rd);
    wc[kind] = std::fmax(wc[kind], rc);
    nd[kind]++;
    if (rd > 1e-4) ++above_d;
    if (rc > 1e-4) ++above_c;
    if (kind == 2) {
      mirror_d = std::fmax(mirror_d, rd);
      mirror_c = std::fmax(mirror_c, rc);
    }
  }
  long nbr[6] = {0, 0, 0, 0, 0, 0};
  for (int i = 0; i < n; ++i) nbr[br[i]]++;
  printf("faces %d supersonic_left %ld supersonic_right %ld subsonic %ld\n", n, nbr[0], nbr[1], nbr[3]);
  for (int k = 0; k < 4; ++k) printf("kind %d faces %ld hlld_max %.3e hllc_max %.3e\n", k, nd[k], wd[k], wc[k]);
  printf("mirror hlld %.3e hllc %.3e\n", mirror_d, mirror_c);
  printf("above1e-4 hlld %ld hllc %ld nonfinite %ld\n", above_d, above_c, nonfinite);
  return 0;
}
