// pip_noalloc.cu -- pip_step_noalloc: run_solver on a caller-held device state with no
// allocation, for hosts that cannot call cudaMalloc (see include/pip_gpu.h).
//
// The stage buffer U1, the control block and the dx/dy tables live in one file-scope
// device array.  Its name is only a host-side stand-in in host code, so the first call on
// each device (with that device current) looks up its device address with
// cudaGetSymbolAddress and passes that address to the kernels.
#include <cuda_runtime.h>

#include <cmath>
#include <mutex>

#include "../../include/pip_gpu.h"
#include "pip_kernels.cuh"

namespace {

constexpr size_t kCtrlBytes = 256;
constexpr size_t kAxisBytes = sizeof(double) * PIP_NOALLOC_MAX_AXIS;
constexpr size_t kScratchBytes = (size_t)PIP_NOALLOC_SCRATCH_BYTES;
static_assert(sizeof(pip::DevCtrl) <= kCtrlBytes, "control block does not fit its slot");
static_assert(kScratchBytes == kCtrlBytes + 2 * kAxisBytes +
                                   sizeof(double) * pip::kMaxPlanes * PIP_NOALLOC_MAX_CELLS,
              "scratch layout");
constexpr int kMaxDevices = 64;

std::mutex g_setup_mutex;
void *g_scratch_addr[kMaxDevices];  // device address of the scratch array, per device

// A failed CUDA call: keep its code for pip_last_cuda_error, as the context calls do.
int cuda_fail(cudaError_t e) {
  pip::record_cuda_error((int)e);
  return PIP_ERR_CUDA;
}

// The whole control block starts from zero on every call, with this call's dt and cmax;
// both come in as launch arguments, so no host buffer has to outlive the call.
__global__ void noalloc_ctrl_kernel(pip::DevCtrl *ctrl, double dt, double cmax) {
  *ctrl = pip::DevCtrl{};
  ctrl->dt = dt;
  ctrl->cmax = cmax;
}

}  // namespace

// [control block | dx | dy | U1 (14 planes of up to PIP_NOALLOC_MAX_CELLS doubles)]
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

extern "C" int pip_step_noalloc(const pip_params *p, double *U_dev, double dt, double cmax,
                                void *stream) {
  if (!p || !U_dev) return PIP_ERR_NULL;
  pip::KParams k;
  const int st = pip::kparams_from_params(p, &k);
  if (st != PIP_OK) return st;
  // the FP64 kernels only; and no implicit conduction, whose BiCGstab needs buffers of
  // its own: pip_step runs HC after the two stages, which this entry point does not
  if (p->precision != PIP_FP64 || p->flag_heat != 0) return PIP_ERR_PARAM;
  if (k.nc > PIP_NOALLOC_MAX_CELLS || p->ix > PIP_NOALLOC_MAX_AXIS || p->jx > PIP_NOALLOC_MAX_AXIS)
    return PIP_ERR_PARAM;
  if (!(dt > 0.0) || !std::isfinite(dt) || !std::isfinite(cmax)) return PIP_ERR_PARAM;
  const pip::Launchers &L = p->fp_exact ? pip::launchers_exact() : pip::launchers_fast();

  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_fail(e);
  if (dev < 0 || dev >= kMaxDevices) return PIP_ERR_CUDA;
  void *base = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_addr[dev]) {
      void *ptr = nullptr;
      if ((e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch)) != cudaSuccess) return cuda_fail(e);
      if (!ptr) return PIP_ERR_CUDA;
      // both FP64 flavours, so a later call with the other fp_exact also finds its limit set
      if ((e = pip::launchers_fast().prepare()) != cudaSuccess) return cuda_fail(e);
      if ((e = pip::launchers_exact().prepare()) != cudaSuccess) return cuda_fail(e);
      g_scratch_addr[dev] = ptr;
    }
    base = g_scratch_addr[dev];
  }
  unsigned char *b = static_cast<unsigned char *>(base);
  pip::DevCtrl *ctrl = reinterpret_cast<pip::DevCtrl *>(b);
  double *ddx = reinterpret_cast<double *>(b + kCtrlBytes);
  double *ddy = reinterpret_cast<double *>(b + kCtrlBytes + kAxisBytes);
  double *U1 = reinterpret_cast<double *>(b + kCtrlBytes + 2 * kAxisBytes);
  k.dx = ddx;
  k.dy = ddy;

  cudaStream_t s = static_cast<cudaStream_t>(stream);
  noalloc_ctrl_kernel<<<1, 1, 0, s>>>(ctrl, dt, cmax);
  if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e);
  if ((e = cudaMemcpyAsync(ddx, p->dx, sizeof(double) * p->ix, cudaMemcpyHostToDevice, s)) != cudaSuccess)
    return cuda_fail(e);
  if ((e = cudaMemcpyAsync(ddy, p->dy, sizeof(double) * p->jx, cudaMemcpyHostToDevice, s)) != cudaSuccess)
    return cuda_fail(e);
  if ((e = L.stage(k, 1, U_dev, U_dev, U1, ctrl, 0, 0, s, nullptr, 0)) != cudaSuccess) return cuda_fail(e);
  if ((e = L.stage(k, 2, U1, U_dev, U_dev, ctrl, 0, 0, s, nullptr, 0)) != cudaSuccess) return cuda_fail(e);
  return PIP_OK;
}
