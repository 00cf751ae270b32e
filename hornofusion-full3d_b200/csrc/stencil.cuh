// The 7-point pressure-correction operator applied at one compact cell,
// shared by the FP64 and FP32 kernels.
#pragma once

#include "cg_common.cuh"

namespace eaf {

template <typename T>
struct Coefs {
  const T* aP;
  const T* aE;
  const T* aN;
  const T* aT;
  const T* aW;  // general form only
  const T* aS;  // general form only
  const T* aB;  // general form only
};

// y = A x at compact cell c in the expression order of the reference matvec
// (x at c given as xc, at the neighbours produced by xv(cell))
// (src/mod_solver_3d.f90:597-603): aP*x - aW*xW - aE*xE - aS*xS - aN*xN
// - aB*xB - aT*xT. In the symmetric form aW(c) = aE(c-1), aS(c) =
// aN(south of c) and aB(c) = aT(c-plane); the wall links of a symmetric
// operator are zero and the reference's Krylov vectors are zero in their r/z
// halos, so the wall terms skipped here are exact zeros there too.
// apply_row_diag: the same row with the cell's own aP given by the caller.
template <bool SYM, typename T, typename XF>
__device__ __forceinline__ T apply_row_diag(const MeshDims& d, const Coefs<T>& A, T ap, T xc,
                                            XF xv, int c) {
  int i, j, k;
  cell_ijk(d, c, i, j, k);
  const int cs = j > 0 ? c - d.nr : c + (d.nth - 1) * d.nr;
  const int cn = j < d.nth - 1 ? c + d.nr : c - (d.nth - 1) * d.nr;
  T y = ap * xc;
  if (SYM) {
    if (i > 0) y = y - A.aE[c - 1] * xv(c - 1);
    if (i < d.nr - 1) y = y - A.aE[c] * xv(c + 1);
    y = y - A.aN[cs] * xv(cs);
    y = y - A.aN[c] * xv(cn);
    if (k > 0) y = y - A.aT[c - d.plane] * xv(c - d.plane);
    if (k < d.nz - 1) y = y - A.aT[c] * xv(c + d.plane);
  } else {
    const T xw = i > 0 ? xv(c - 1) : T(0);
    const T xe = i < d.nr - 1 ? xv(c + 1) : T(0);
    const T xb = k > 0 ? xv(c - d.plane) : T(0);
    const T xt = k < d.nz - 1 ? xv(c + d.plane) : T(0);
    y = y - A.aW[c] * xw;
    y = y - A.aE[c] * xe;
    y = y - A.aS[c] * xv(cs);
    y = y - A.aN[c] * xv(cn);
    y = y - A.aB[c] * xb;
    y = y - A.aT[c] * xt;
  }
  return y;
}

template <bool SYM, typename T, typename XF>
__device__ __forceinline__ T apply_row_with(const MeshDims& d, const Coefs<T>& A, T xc,
                                            XF xv, int c) {
  return apply_row_diag<SYM, T>(d, A, A.aP[c], xc, xv, c);
}

// The operator applied to a stored vector x.
template <bool SYM, typename T>
__device__ __forceinline__ T apply_row(const MeshDims& d, const Coefs<T>& A,
                                       const T* __restrict__ x, int c) {
  return apply_row_with<SYM, T>(d, A, x[c], [x](int cc) { return x[cc]; }, c);
}

template <typename T>
__device__ __forceinline__ Coefs<T> coefs_of(const T* aP, const T* aE, const T* aN,
                                             const T* aT, const T* aW, const T* aS,
                                             const T* aB) {
  Coefs<T> c;
  c.aP = aP; c.aE = aE; c.aN = aN; c.aT = aT; c.aW = aW; c.aS = aS; c.aB = aB;
  return c;
}

// Block-owned contiguous slice [begin, end) of n cells for block `bid` of `nb`.
struct Slice {
  int begin, end;
};
__device__ __forceinline__ Slice own_slice(int n, int nb, int bid) {
  const int chunk = (n + nb - 1) / nb;
  Slice s;
  s.begin = min(n, bid * chunk);
  s.end = min(n, s.begin + chunk);
  return s;
}

}  // namespace eaf

// Loop over the cells of slice S owned by this thread, unrolled by U with
// the loads of the U cells issued together; C names the cell index.
#define EAF_FOR_OWN(S, U, C, ...)                                           \
  for (int c0_ = (S).begin + (int)threadIdx.x; c0_ < (S).end;                \
       c0_ += (int)blockDim.x * (U)) {                                       \
    _Pragma("unroll") for (int u_ = 0; u_ < (U); ++u_) {                     \
      const int C = c0_ + u_ * (int)blockDim.x;                              \
      if (C < (S).end) { __VA_ARGS__ }                                       \
    }                                                                        \
  }
