// Strategy kernels beyond the ghost-fluid pressure: the whole-domain magnetic
// potential solve of the 3D ferrofluid substep, and Galerkin coarsening of a
// stored-coefficient operator.
#pragma once
#include "mg_common.cuh"

namespace mg {

__device__ __forceinline__ bool is_pin(const int c[3], const int pin[3], int dim) {
  return c[0] == pin[0] && c[1] == pin[1] && (dim == 2 || c[2] == pin[2]);
}

// Harmonic mean of the permeabilities mu = 1 + chi of two cells.
__device__ __forceinline__ float mu_face(float chi_a, float chi_b) {
  const float ma = __fadd_rn(1.0f, chi_a), mb = __fadd_rn(1.0f, chi_b);
  return __fdiv_rn(__fmul_rn(2.0f, __fmul_rn(ma, mb)), __fadd_rn(ma, mb));
}

// Magnetic potential right-hand side on level 0:
//   b_I = -(1/dx) sum_k H_k (mu(I, I+e_k) - mu(I-e_k, I))
// over faces inside the domain (no flux through the boundary), b = 0 at the
// pinned cell.  H is constant (the external field).
__global__ void k_build_psi_b(Level L, float* b, const float* __restrict__ chi, float H0, float H1, float H2,
                              float dx, int p0, int p1, int p2) {
  const float Hk[3] = {H0, H1, H2};
  const int pin[3] = {p0, p1, p2};
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < L.g.count;
       i += (long long)gridDim.x * blockDim.x) {
    int c[3];
    L.g.coords(i, c);
    if (is_pin(c, pin, L.g.dim)) {
      b[i] = 0.0f;
      continue;
    }
    float acc = 0.0f;
    for (int k = 0; k < L.g.dim; ++k) {
      const long long s = L.g.stride(k);
      if (c[k] + 1 < L.g.n[k]) acc = __fadd_rn(acc, __fmul_rn(Hk[k], mu_face(chi[i], chi[i + s])));
      if (c[k] > 0) acc = __fsub_rn(acc, __fmul_rn(Hk[k], mu_face(chi[i - s], chi[i])));
    }
    b[i] = -__fdiv_rn(acc, dx);
  }
}

// Magnetic potential operator on level 0: face coefficient mu(I, J) / dx^2
// (symmetric positive definite), Neumann at the domain boundary, Dirichlet
// psi = 0 at the pinned cell (its couplings removed, its row the identity
// times 1/dx^2).
__global__ void k_build_psi_A(Level L, const float* __restrict__ chi, float dx, int p0, int p1, int p2) {
  const int pin[3] = {p0, p1, p2};
  const float dx2 = __fmul_rn(dx, dx);
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < L.g.count;
       i += (long long)gridDim.x * blockDim.x) {
    int c[3];
    L.g.coords(i, c);
    if (is_pin(c, pin, L.g.dim)) {
      L.Adiag[i] = __fdiv_rn(1.0f, dx2);
      for (int k = 0; k < L.g.dim; ++k) L.Ax[k][i] = 0.0f;
      continue;
    }
    float d = 0.0f;
    for (int k = 0; k < L.g.dim; ++k) {
      const long long s = L.g.stride(k);
      float up = 0.0f;
      if (c[k] > 0) d = __fadd_rn(d, __fdiv_rn(mu_face(chi[i - s], chi[i]), dx2));
      if (c[k] + 1 < L.g.n[k]) {
        const float cf = __fdiv_rn(mu_face(chi[i], chi[i + s]), dx2);
        d = __fadd_rn(d, cf);
        int cn[3] = {c[0], c[1], c[2]};
        cn[k] += 1;
        up = is_pin(cn, pin, L.g.dim) ? 0.0f : -cf;
      }
      L.Ax[k][i] = up;
    }
    L.Adiag[i] = d;
  }
}

// Galerkin coarse operator A_c = P^T A P for the reference's transfer pair
// (prolongation: piecewise constant, mgpcg.py:120-123; restriction: the
// unweighted sum of the 2^d children, mgpcg.py:111-118):
//   Ax_c[J][k] = sum of Ax[i][k] over the children i of J on its +k face
//   Adiag_c[J] = sum of Adiag[i] over the children + 2 * sum of the Ax of the
//                faces between two children of J
// Children are visited in lexicographic order.
__global__ void k_galerkin(Level F, Level C) {
  for (long long ic = (long long)blockIdx.x * blockDim.x + threadIdx.x; ic < C.g.count;
       ic += (long long)gridDim.x * blockDim.x) {
    int cc[3];
    C.g.coords(ic, cc);
    const int dim = C.g.dim;
    float d = 0.0f, ax[3] = {0.0f, 0.0f, 0.0f};
    for (int o0 = 0; o0 < 2; ++o0)
      for (int o1 = 0; o1 < 2; ++o1)
        for (int o2 = 0; o2 < (dim == 3 ? 2 : 1); ++o2) {
          const int o[3] = {o0, o1, o2};
          const long long i = F.g.index(2 * cc[0] + o0, 2 * cc[1] + o1, dim == 3 ? 2 * cc[2] + o2 : 0);
          d = __fadd_rn(d, F.Adiag[i]);
          for (int k = 0; k < dim; ++k) {
            const float a = F.Ax[k][i];
            if (o[k] == 0) d = __fadd_rn(d, __fmul_rn(2.0f, a));  // internal face
            else ax[k] = __fadd_rn(ax[k], a);                       // face to the next block
          }
        }
    C.Adiag[ic] = d;
    for (int k = 0; k < dim; ++k) C.Ax[k][ic] = (cc[k] + 1 < C.g.n[k]) ? ax[k] : 0.0f;
  }
}

}  // namespace mg
