// FGR 19-point anisotropic diffusion on the device: node tables, the weight
// builder and the stencil.
//
// Reference: elec/FGRDiffusionOMP.cc:166-265 (precomputeCoefficients, f1),
// elec/FGRUtils.cc:10-148 (setGradientWeights, f2), elec/FGRDiffusionOMP.cc:109-131
// (calc).  For each tissue cell and each of its 6 faces whose neighbour is
// tissue:  sigma_face = (sigma_cell + sigma_nbr)/2,  sigmaTimesS = sigma_face S_face / V,
// and the face-normal gradient is the two-point difference across the face,
// while a tangential gradient is the four-node average difference (+1/4 on
// the two nodes one step along the axis, -1/4 on the two one step against it)
// and exists only when all four nodes are tissue.  A[k] += sigmaTimesS_j
// gradPhi_j[k] / h_j;  A0 = -sum_{k>=1} A[k];
// dVm_D = diffusionScale (A0 phi0 + sum_k A[k] phi_k).
//
// The weights are built with round-to-nearest intrinsics so no FMA
// contraction changes them: they equal the reference's bit for bit.
#pragma once
#include <cstdint>

namespace cdb {

// The 19 nodes in the reference's NodeLocation order (elec/FGRUtils.hh:22-24).
__host__ __device__ constexpr int node_dx(int k)
{
  return (k == 1 || k == 7 || k == 10 || k == 11 || k == 15) ? -1
       : (k == 3 || k == 8 || k == 9 || k == 13 || k == 17) ? 1 : 0;
}
__host__ __device__ constexpr int node_dy(int k)
{
  return (k == 2 || k == 7 || k == 8 || k == 12 || k == 16) ? -1
       : (k == 4 || k == 9 || k == 10 || k == 14 || k == 18) ? 1 : 0;
}
__host__ __device__ constexpr int node_dz(int k)
{
  return (k == 5 || k == 11 || k == 12 || k == 13 || k == 14) ? -1
       : (k == 6 || k == 15 || k == 16 || k == 17 || k == 18) ? 1 : 0;
}
__host__ __device__ constexpr int node_of(int dx, int dy, int dz)
{
  for (int k = 0; k < 19; ++k)
    if (node_dx(k) == dx && node_dy(k) == dy && node_dz(k) == dz) return k;
  return -1;
}

// Stencil classes: a tissue whose bounding box is one voxel thick in y and z
// (a cable along x) has non-zero weights only on x-neighbours, a sheet one
// voxel thick in z only on in-plane neighbours; every weight on a node that
// is not tissue is exactly zero, so dropping those nodes changes no bit.
enum StencilClass { kCable = 1, kSheet = 2, kVolume = 3 };
__host__ __device__ constexpr int class_rows(int cls) { return cls == kCable ? 3 : cls == kSheet ? 9 : 19; }
// Node of each row of a class.
__host__ __device__ constexpr int class_node(int cls, int row)
{
  return cls == kCable ? (row == 0 ? 0 : row == 1 ? 1 : 3)
       : cls == kSheet ? (row < 5 ? row : row + 2)
       : row;
}

// Faces in the reference's iFace order: -x, -y, +x, +y, -z, +z.
__host__ __device__ constexpr int face_axis(int f) { return (f == 0 || f == 2) ? 0 : (f == 1 || f == 3) ? 1 : 2; }
__host__ __device__ constexpr int face_sign(int f) { return (f == 0 || f == 1 || f == 4) ? -1 : 1; }

// Builds the weights of one cell.  tissue[k]: node k is tissue;
// sig(k, c): component c (a11 a12 a13 a22 a23 a33) of node k's tensor.
template <typename SigmaFn>
__host__ __device__ inline void fgr_cell_weights(const int tissue[19], SigmaFn sig, double hx, double hy, double hz,
                                                 double W[19])
{
#ifdef __CUDA_ARCH__
#define MUL(a, b) __dmul_rn((a), (b))
#define ADD(a, b) __dadd_rn((a), (b))
#define DIV(a, b) __ddiv_rn((a), (b))
#else
#define MUL(a, b) ((a) * (b))
#define ADD(a, b) ((a) + (b))
#define DIV(a, b) ((a) / (b))
#endif
  const double h[3] = {hx, hy, hz};
  const double hInv[3] = {DIV(1.0, hx), DIV(1.0, hy), DIV(1.0, hz)};
  const double vol = MUL(MUL(hx, hy), hz);
  for (int k = 0; k < 19; ++k) W[k] = 0.0;
  for (int face = 0; face < 6; ++face) {
    const int axis = face_axis(face), sign = face_sign(face);
    const int nbr = node_of(axis == 0 ? sign : 0, axis == 1 ? sign : 0, axis == 2 ? sign : 0);
    if (!tissue[nbr]) continue;
    double a[6];
    for (int c = 0; c < 6; ++c) a[c] = DIV(ADD(sig(0, c), sig(nbr, c)), 2.0);
    double S[3] = {0.0, 0.0, 0.0};
    const double area = axis == 0 ? MUL(h[1], h[2]) : axis == 1 ? MUL(h[0], h[2]) : MUL(h[0], h[1]);
    S[axis] = sign > 0 ? area : -area;
    double sts[3];
    sts[0] = DIV(ADD(ADD(MUL(a[0], S[0]), MUL(a[1], S[1])), MUL(a[2], S[2])), vol);
    sts[1] = DIV(ADD(ADD(MUL(a[1], S[0]), MUL(a[3], S[1])), MUL(a[4], S[2])), vol);
    sts[2] = DIV(ADD(ADD(MUL(a[2], S[0]), MUL(a[4], S[1])), MUL(a[5], S[2])), vol);
    double grad[3][19];
    for (int j = 0; j < 3; ++j)
      for (int k = 0; k < 19; ++k) grad[j][k] = 0.0;
    if (sign > 0) { grad[axis][nbr] = 1.0; grad[axis][0] = -1.0; }
    else { grad[axis][0] = 1.0; grad[axis][nbr] = -1.0; }
    for (int b = 0; b < 3; ++b) {
      if (b == axis) continue;
      const int u[3] = {b == 0, b == 1, b == 2};
      const int n3[3] = {axis == 0 ? sign : 0, axis == 1 ? sign : 0, axis == 2 ? sign : 0};
      const int kcp = node_of(u[0], u[1], u[2]), kcm = node_of(-u[0], -u[1], -u[2]);
      const int knp = node_of(n3[0] + u[0], n3[1] + u[1], n3[2] + u[2]);
      const int knm = node_of(n3[0] - u[0], n3[1] - u[1], n3[2] - u[2]);
      if (tissue[kcp] && tissue[kcm] && tissue[knp] && tissue[knm]) {
        grad[b][kcp] = 0.25; grad[b][knp] = 0.25;
        grad[b][kcm] = -0.25; grad[b][knm] = -0.25;
      }
    }
    for (int k = 0; k < 19; ++k)
      for (int j = 0; j < 3; ++j) W[k] = ADD(W[k], MUL(MUL(sts[j], grad[j][k]), hInv[j]));
  }
  double a0 = 0.0;
  for (int k = 1; k < 19; ++k) a0 = ADD(a0, -W[k]);
  W[0] = a0;
#undef MUL
#undef ADD
#undef DIV
}

}  // namespace cdb
