// The reference's "cuda" Diffusion (CUDADiffusion, elec/CUDADiffusion.cc:
// 30-160, kernel diff_6face_v1 in elec/CUDADiffusion_ker.cu:16-140) as a
// plugin: a 6-face flux stencil with its own conductivity rule, for users of
// `method = cuda` who compare against it.  Unlike FGR, each face carries the
// conductivity of the cell on its + side (not a face average):
//   S_ij(c) = sigma_c[i][j] area_i / h_j diffusionScale / volume
// on the - face of cell c along axis i, zero when that neighbour is absent;
// a tangential term (j != i) is kept only when the four nodes c -/+ e_j and
// c - e_i -/+ e_j all exist.  The flux through that face is
//   F_i(c) = sum_j S_ij(c) d_j,  d_i = V(c) - V(c - e_i),
//   d_j = 4-node average of the tangential difference across the face,
// and dVm(c) = sum_i F_i(c + e_i) - F_i(c).
//
// B200 layout: the padded Vm block (x fastest, one halo voxel) and nine
// SoA planes of face conductivities over the same block; one thread per
// cell reads its 19-point neighbourhood and 18 face terms.
#include <cuda_runtime.h>

#include <memory>
#include <vector>

#include "common.cuh"

namespace cdb {

struct D6Buf {
  void* p = nullptr;
  ~D6Buf() { if (p) cudaFree(p); }
  cudaError_t alloc(size_t b) { return b ? cudaMalloc(&p, b) : cudaSuccess; }
  template <typename T> T* as() const { return (T*)p; }
};

__global__ void d6_map_kernel(int64_t n, const int64_t* __restrict__ gid, int nx, int ny, int64_t bx, int64_t bxy,
                              int64_t* __restrict__ map, int64_t* __restrict__ voxel)
{
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int64_t g = gid[i];
  const int64_t x = g % nx, y = (g / nx) % ny, z = g / ((int64_t)nx * ny);
  const int64_t v = (x + 1) + bx * (y + 1) + bxy * (z + 1);
  map[v] = i;
  voxel[i] = v;
}

// Face conductivities of every cell (CUDADiffusion ctor, elec/CUDADiffusion.cc:73-122).
__global__ void d6_sigma_kernel(int64_t n, const int64_t* __restrict__ map, const int64_t* __restrict__ voxel,
                                const double* __restrict__ sigma6, int64_t bx, int64_t bxy, int64_t nvox, double hx,
                                double hy, double hz, double scale, double* __restrict__ face)
{
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int64_t v = voxel[i];
  const int64_t off[3] = {1, bx, bxy};
  const double* s = sigma6 + 6 * i;
  const double sig[3][3] = {{s[0], s[1], s[2]}, {s[1], s[3], s[4]}, {s[2], s[4], s[5]}};
  const double area[3] = {hy * hz, hx * hz, hx * hy};
  const double disc[3] = {hx, hy, hz};
  const double volume = hx * hy * hz;
  for (int a = 0; a < 3; ++a) {
    const bool left = map[v - off[a]] >= 0;
    for (int b = 0; b < 3; ++b) {
      double val = 0.0;
      if (left) {
        val = sig[a][b] * area[a] / disc[b] * scale / volume;
        if (a != b) {
          const bool grad = map[v - off[b]] >= 0 && map[v + off[b]] >= 0 && map[v - off[a] - off[b]] >= 0 &&
                            map[v - off[a] + off[b]] >= 0;
          if (!grad) val = 0.0;
        }
      }
      face[(int64_t)(3 * a + b) * nvox + v] = val;
    }
  }
}

__global__ void d6_scatter_kernel(int64_t n, const double* __restrict__ Vm, const int64_t* __restrict__ voxel,
                                  double* __restrict__ blk)
{
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) blk[voxel[i]] = Vm[i];
}

// Flux through the - face of voxel c along axis A (diff_6face_v1's x/y/z
// charges, in its term order).
template <int A>
__device__ __forceinline__ double d6_flux(const double* __restrict__ V, const double* __restrict__ face, int64_t nvox,
                                          int64_t c, int64_t ox, int64_t oy, int64_t oz)
{
  const int64_t o[3] = {ox, oy, oz};
  const int64_t b = c, a = c - o[A];
  double d[3];
  if (A == 0) {
    d[0] = -V[a] + V[b];
    d[1] = (-V[a - oy] + V[a + oy] - V[b - oy] + V[b + oy]) / 4.;
    d[2] = (-V[a - oz] + V[a + oz] - V[b - oz] + V[b + oz]) / 4.;
  } else if (A == 1) {
    d[0] = (-V[a - ox] - V[b - ox] + V[a + ox] + V[b + ox]) / 4.;
    d[1] = -V[a] + V[b];
    d[2] = (-V[a - oz] + V[a + oz] - V[b - oz] + V[b + oz]) / 4.;
  } else {
    d[0] = (-V[a - ox] - V[b - ox] + V[a + ox] + V[b + ox]) / 4.;
    d[1] = (-V[a - oy] - V[b - oy] + V[a + oy] + V[b + oy]) / 4.;
    d[2] = -V[a] + V[b];
  }
  const double* f = face + (int64_t)(3 * A) * nvox + c;
  return f[0] * d[0] + f[nvox] * d[1] + f[2 * nvox] * d[2];
}

// dVm(c) in diff_6face_v1's order: -F_x(c) + F_y(c+y) - F_y(c) + F_z(c+z) - F_z(c) + F_x(c+x).
__global__ void d6_calc_kernel(int64_t n, const int64_t* __restrict__ voxel, const double* __restrict__ V,
                               const double* __restrict__ face, int64_t bx, int64_t bxy, int64_t nvox,
                               double* __restrict__ dVm)
{
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int64_t c = voxel[i];
  double dV = -d6_flux<0>(V, face, nvox, c, 1, bx, bxy);
  dV += d6_flux<1>(V, face, nvox, c + bx, 1, bx, bxy);
  dV -= d6_flux<1>(V, face, nvox, c, 1, bx, bxy);
  dV += d6_flux<2>(V, face, nvox, c + bxy, 1, bx, bxy);
  dV -= d6_flux<2>(V, face, nvox, c, 1, bx, bxy);
  dV += d6_flux<0>(V, face, nvox, c + 1, 1, bx, bxy);
  dVm[i] = dV;
}

}  // namespace cdb

using namespace cdb;

struct cdb_diff6 {
  int device = 0;
  int64_t n = 0, bx = 0, bxy = 0, nvox = 0;
  D6Buf voxel, blk, face;
};

extern "C" {

cdb_status cdb_diff6_create(int device, int32_t nx, int32_t ny, int32_t nz, double dx, double dy, double dz,
                            int64_t nCells, const int64_t* gid, const double* sigma6, double diffusionScale,
                            cdb_diff6** out)
{
  CDB_CHECK(out && gid && sigma6, CDB_INVALID_ARG, "null argument");
  CDB_CHECK(nx > 0 && ny > 0 && nz > 0 && dx > 0 && dy > 0 && dz > 0, CDB_INVALID_ARG, "bad grid");
  const int64_t grid = (int64_t)nx * ny * nz;
  CDB_CHECK(nCells > 0 && nCells <= grid, CDB_INVALID_ARG, "nCells out of range");
  for (int64_t i = 0; i < nCells; ++i) CDB_CHECK(gid[i] >= 0 && gid[i] < grid, CDB_INVALID_ARG, "gid outside the grid");
  CDB_CUDA(cudaSetDevice(device));
  std::unique_ptr<cdb_diff6> d(new cdb_diff6);
  d->device = device;
  d->n = nCells;
  d->bx = nx + 2;
  d->bxy = d->bx * (ny + 2);
  d->nvox = d->bxy * (nz + 2);
  CDB_CUDA(d->voxel.alloc(nCells * 8));
  CDB_CUDA(d->blk.alloc(d->nvox * 8));
  CDB_CUDA(d->face.alloc(9 * d->nvox * 8));
  CDB_CUDA(cudaMemset(d->blk.p, 0, d->nvox * 8));
  CDB_CUDA(cudaMemset(d->face.p, 0, 9 * d->nvox * 8));
  D6Buf map, g, sig;
  CDB_CUDA(map.alloc(d->nvox * 8));
  CDB_CUDA(g.alloc(nCells * 8));
  CDB_CUDA(sig.alloc(nCells * 48));
  CDB_CUDA(cudaMemset(map.p, 0xff, d->nvox * 8));
  CDB_CUDA(cudaMemcpy(g.p, gid, nCells * 8, cudaMemcpyHostToDevice));
  CDB_CUDA(cudaMemcpy(sig.p, sigma6, nCells * 48, cudaMemcpyHostToDevice));
  const unsigned blocks = (unsigned)((nCells + 255) / 256);
  d6_map_kernel<<<blocks, 256>>>(nCells, g.as<int64_t>(), nx, ny, d->bx, d->bxy, map.as<int64_t>(),
                                 d->voxel.as<int64_t>());
  d6_sigma_kernel<<<blocks, 256>>>(nCells, map.as<int64_t>(), d->voxel.as<int64_t>(), sig.as<double>(), d->bx, d->bxy,
                                   d->nvox, dx, dy, dz, diffusionScale, d->face.as<double>());
  CDB_CUDA(cudaDeviceSynchronize());
  *out = d.release();
  return CDB_OK;
}

cdb_status cdb_diff6_update_local_voltage(cdb_diff6* d, const double* Vm, void* stream)
{
  CDB_CHECK(d && Vm, CDB_INVALID_ARG, "null argument");
  CDB_CUDA(cudaSetDevice(d->device));
  d6_scatter_kernel<<<(unsigned)((d->n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(d->n, Vm, d->voxel.as<int64_t>(),
                                                                                     d->blk.as<double>());
  CDB_CUDA(cudaGetLastError());
  return CDB_OK;
}

cdb_status cdb_diff6_calc(cdb_diff6* d, double* dVm, void* stream)
{
  CDB_CHECK(d && dVm, CDB_INVALID_ARG, "null argument");
  CDB_CUDA(cudaSetDevice(d->device));
  d6_calc_kernel<<<(unsigned)((d->n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(
      d->n, d->voxel.as<int64_t>(), d->blk.as<double>(), d->face.as<double>(), d->bx, d->bxy, d->nvox, dVm);
  CDB_CUDA(cudaGetLastError());
  return CDB_OK;
}

cdb_status cdb_diff6_get_face_sigma(cdb_diff6* d, double* host9)
{
  CDB_CHECK(d && host9, CDB_INVALID_ARG, "null argument");
  CDB_CUDA(cudaSetDevice(d->device));
  CDB_CUDA(cudaDeviceSynchronize());
  std::vector<double> face(9 * d->nvox);
  std::vector<int64_t> vox(d->n);
  CDB_CUDA(cudaMemcpy(face.data(), d->face.p, face.size() * 8, cudaMemcpyDeviceToHost));
  CDB_CUDA(cudaMemcpy(vox.data(), d->voxel.p, vox.size() * 8, cudaMemcpyDeviceToHost));
  for (int64_t i = 0; i < d->n; ++i)
    for (int k = 0; k < 9; ++k) host9[i * 9 + k] = face[(size_t)k * d->nvox + vox[i]];
  return CDB_OK;
}

cdb_status cdb_diff6_destroy(cdb_diff6* d)
{
  if (!d) return CDB_OK;
  cudaSetDevice(d->device);
  cudaDeviceSynchronize();
  delete d;
  return CDB_OK;
}

}  // extern "C"
