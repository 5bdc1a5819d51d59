// pip_halo.cu -- the two halves of mpi_bnd (MPI_rot.f90:128-339) as device copies between a
// context's state and a contiguous message buffer.
//
// A message of face f (0 x-, 1 x+, 2 y-, 3 y+) carries the `margin` interior layers next to
// that face, every plane of every array of the state the last RK stage wrote; the receiver
// writes it into the ghost layers of its opposite face.  Layer order is increasing index on
// both sides, so sender layer l (interior index m + l next to a lower face, n - 2m + l next
// to an upper face) lands in receiver ghost layer l (index l, or n - m + l), the pairing of
// mpi_bnd's sendx/recvx slices.  Buffer order: array, plane, layer, position along the face
// (x fastest within a y layer, so y messages copy whole rows).  Rows and columns include
// the ghost cells of the other direction, as the Fortran slices U(:, js:je, :, :) do.
#include <cuda_runtime.h>

#include "pip_kernels.cuh"

namespace pip {
namespace {

struct HaloGeom {
  int ix;          // row length
  int dir;         // 0 x, 1 y
  int m;           // layers
  int extent;      // positions along the face (jx for x faces, ix for y faces)
  int first;       // index of layer 0 (column for x faces, row for y faces)
  long long nc;    // cells per plane
  int nplanes;
  long long count; // elements per array
};

template <typename T>
__global__ void halo_pack_kernel(HaloGeom g, const T *__restrict__ a0, const T *__restrict__ a1,
                                 T *__restrict__ buf) {
  const int narr = a1 ? 2 : 1;
  const long long total = g.count * narr;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const long long a = t / g.count, r = t % g.count;
    const int k = (int)(r % g.extent);
    const long long nl = r / g.extent;
    const int l = (int)(nl % g.m), n = (int)(nl / g.m);
    const long long q = g.dir == 0 ? (long long)k * g.ix + g.first + l
                                   : (long long)(g.first + l) * g.ix + k;
    buf[t] = (a == 0 ? a0 : a1)[q + n * g.nc];
  }
}

template <typename T>
__global__ void halo_unpack_kernel(HaloGeom g, T *a0, T *a1, const T *__restrict__ buf) {
  const int narr = a1 ? 2 : 1;
  const long long total = g.count * narr;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const long long a = t / g.count, r = t % g.count;
    const int k = (int)(r % g.extent);
    const long long nl = r / g.extent;
    const int l = (int)(nl % g.m), n = (int)(nl / g.m);
    const long long q = g.dir == 0 ? (long long)k * g.ix + g.first + l
                                   : (long long)(g.first + l) * g.ix + k;
    (a == 0 ? a0 : a1)[q + n * g.nc] = buf[t];
  }
}

HaloGeom geom(const KParams &p, int face, bool pack) {
  HaloGeom g{};
  g.ix = p.ix;
  g.dir = face / 2;
  g.m = g.dir == 0 ? p.m0 : p.m1;
  g.extent = g.dir == 0 ? p.jx : p.ix;
  const int n = g.dir == 0 ? p.ix : p.jx;
  const bool lower = face % 2 == 0;
  if (pack) g.first = lower ? g.m : n - 2 * g.m;
  else g.first = lower ? 0 : n - g.m;
  g.nc = p.nc;
  g.nplanes = p.nvm + 5;
  g.count = (long long)g.nplanes * g.m * g.extent;
  return g;
}

int blocks_for(long long n) {
  long long b = (n + 255) / 256;
  return (int)(b < 148 * 16 ? (b < 1 ? 1 : b) : 148 * 16);
}

}  // namespace

long long halo_elems(const KParams &p, int face) { return geom(p, face, true).count; }

cudaError_t halo_pack(const KParams &p, int face, const void *a0, const void *a1, int elem_bytes,
                      void *buf, cudaStream_t s) {
  const HaloGeom g = geom(p, face, true);
  const int nb = blocks_for(g.count * (a1 ? 2 : 1));
  if (elem_bytes == 8)
    halo_pack_kernel<double><<<nb, 256, 0, s>>>(g, (const double *)a0, (const double *)a1, (double *)buf);
  else
    halo_pack_kernel<float><<<nb, 256, 0, s>>>(g, (const float *)a0, (const float *)a1, (float *)buf);
  return cudaGetLastError();
}

cudaError_t halo_unpack(const KParams &p, int face, void *a0, void *a1, int elem_bytes,
                        const void *buf, cudaStream_t s) {
  const HaloGeom g = geom(p, face, false);
  const int nb = blocks_for(g.count * (a1 ? 2 : 1));
  if (elem_bytes == 8)
    halo_unpack_kernel<double><<<nb, 256, 0, s>>>(g, (double *)a0, (double *)a1, (const double *)buf);
  else
    halo_unpack_kernel<float><<<nb, 256, 0, s>>>(g, (float *)a0, (float *)a1, (const float *)buf);
  return cudaGetLastError();
}

}  // namespace pip
