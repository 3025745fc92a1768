// The 5-point operators of the external mode in face-coupling form.
//
// Both reference operators (make_coeff_streamfunction, solve_streamfct.f90:
// 123-148, and make_coeff_surf_press, solve_pressure.f90:87-131) are
//
//   (A p)(i,j) = ax(i) bx(j) [ FX(i+1,j) (p(i+1,j)-p(i,j)) + FX(i,j) (p(i-1,j)-p(i,j)) ]
//              +       by(j) [ FY(i,j+1) (p(i,j+1)-p(i,j)) + FY(i,j) (p(i,j-1)-p(i,j)) ]
//              + dcoef W(i,j) p(i,j)
//
// with FX(i,j) the coupling across the x-face between (i-1,j) and (i,j) and
// FY(i,j) across the y-face between (i,j-1) and (i,j):
//
//   streamfunction: FX = hvr(i,j)/dxt(i),  ax = 1/dxu(i), bx = 1/cosu(j)^2,
//                   FY = hur(i,j) cost(j)/dyt(j), by = 1/(dyu(j) cosu(j)), dcoef = 0
//   surf_press:     FX = m(i-1,j) m(i,j) hu(i-1,j)/dxu(i-1), ax = 1/dxt(i), bx = 1/cost(j)^2,
//                   FY = m(i,j-1) m(i,j) hv(i,j-1) cosu(j-1)/dyu(j-1), by = 1/(dyt(j) cost(j)),
//                   dcoef = -1/(grav dt^2) with free surface, W = m = maskT(:,:,nz)
//
// Expanding gives exactly the reference's cf(i,j,ii,jj) entries, with the
// centre cf(i,j,2,2) = -(E+W+N+S) (+ free-surface term).  Only two 2-D
// coefficient fields are stored (16 B/point in FP64) instead of the nine
// sweeps over cf(:,:,3,3) of apply_op (solve_pressure.f90:264-273); the
// difference form also avoids the cancellation of the sum form.
#pragma once
#include "common.cuh"

namespace pyomgpu {

template <typename T>
struct OpDev {
  const T* FX;       // padded layout
  const T* FY;       // padded layout
  const T* ax;       // [nx+4], index Fortran i + 1
  const T* bx;       // [ny+4], index Fortran j + 1
  const T* by;       // [ny+4]
  const T* W;        // Z (streamfunction) or maskT(:,:,nz) (surf_press), padded
  T dcoef;           // diagonal term dcoef*W
};

// (A p)(i,j) reading p from memory (valid halos required).
template <typename T>
__device__ __forceinline__ T apply_point(const OpDev<T>& op, const Geo& g, const T* __restrict__ p, int i, int j) {
  const T pc = p[g.at(i, j)];
  const T sx = op.ax[i + 1] * op.bx[j + 1];
  const T sy = op.by[j + 1];
  T r = sx * (op.FX[g.at(i + 1, j)] * (p[g.at(i + 1, j)] - pc) + op.FX[g.at(i, j)] * (p[g.at(i - 1, j)] - pc)) +
        sy * (op.FY[g.at(i, j + 1)] * (p[g.at(i, j + 1)] - pc) + op.FY[g.at(i, j)] * (p[g.at(i, j - 1)] - pc));
  if (op.dcoef != T(0)) r += op.dcoef * op.W[g.at(i, j)] * pc;
  return r;
}

}  // namespace pyomgpu
