// Non-hydrostatic pressure operator (non_hydrostatic.f90:70-138, 247-276) in
// compact device form.
//
// make_coeff_non_hydro stores a 3x3x3 stencil per cell (27 doubles), of which
// at most seven entries are nonzero: the six faces and the centre.  Every face
// coefficient is a 0/1 face mask times a metric factor that depends on one or
// two of (i, j, k) only:
//
//   east   maskU(i,j,k)   * tE(i,j) = ((1/dxu(i)  )/dxt(i))/cost(j)**2
//   west   maskU(i-1,j,k) * tW(i,j) = ((1/dxu(i-1))/dxt(i))/cost(j)**2
//   north  maskV(i,j,k)   * tN(j)   = (((1/dyu(j)  )/dyt(j))*cosu(j)  )/cost(j)
//   south  maskV(i,j-1,k) * tS(j)   = (((1/dyu(j-1))/dyt(j))*cosu(j-1))/cost(j)
//   top    maskW(i,j,k)   * tT(k)   = (1/dzw(k)  )/dzt(k)      (k < nz)
//   bottom maskW(i,j,k-1) * tB(k)   = (1/dzw(k-1))/dzt(k)      (k > 1)
//
// (mp/a/b/c with mp = 1 rounds exactly like 1/a/b/c, and with mp = 0 gives 0.)
// The device keeps one flag byte per cell (the six face masks and maskT) plus
// the 2-D tables tE, tW and the 1-D tables tN, tS, tT, tB, i.e. 1 byte per
// cell instead of 216.  The centre coefficient is rebuilt in the order the
// reference accumulates it (east, west, north, south, top, bottom), and the
// products are summed in apply_op_3D's (kk, jj, ii) order with separately
// rounded multiplies and adds, so A p is bit-identical to the reference's.
#pragma once
#include <cuda.h>
#include <stdint.h>

#include "common.cuh"

namespace pyomgpu {

constexpr int kNHThreads = 256;

enum : uint32_t { kNHE = 1u, kNHW = 2u, kNHN = 4u, kNHS = 8u, kNHT = 16u, kNHB = 32u, kNHMaskT = 64u };

// Padded 3-D layout: level k (1..nz) is a padded 2-D field of the Geo layout.
struct NHGeo {
  Geo g;
  int nz;
  size_t plane;  // g.size()
  __host__ __device__ __forceinline__ size_t at(int i, int j, int k) const {
    return (size_t)(k - 1) * plane + g.at(i, j);
  }
  __host__ __device__ __forceinline__ size_t size() const { return plane * (size_t)nz; }
};

struct NHOp {
  const uint8_t* flags;  // [nz][ny][fx], cell (i,j,k) at ((k-1)*ny + j-1)*fx + i-1
  const double* tE;      // padded 2-D
  const double* tW;      // padded 2-D
  const double* tN;      // [ny+4], index j+1
  const double* tS;      // [ny+4], index j+1
  const double* tT;      // [nz], index k-1
  const double* tB;      // [nz], index k-1
  int fx;                // flag row pitch, nx rounded up to 32
  __host__ __device__ __forceinline__ size_t fidx(int ny, int i, int j, int k) const {
    return ((size_t)(k - 1) * (size_t)ny + (size_t)(j - 1)) * (size_t)fx + (size_t)(i - 1);
  }
};

// Operator row with the seven field values given: bottom, south, west,
// centre, east, north, top; t* are the face factors (read only where the
// face flag is set).
__device__ __forceinline__ double nh_row(uint32_t f, double tE, double tW, double tN, double tS, double tT, double tB,
                                         double vb, double vs, double vw, double vc, double ve, double vn, double vt) {
  double c = 0.0;  // make_coeff_non_hydro's accumulation order
  if (f & kNHE) c = __dsub_rn(c, tE);
  if (f & kNHW) c = __dsub_rn(c, tW);
  if (f & kNHN) c = __dsub_rn(c, tN);
  if (f & kNHS) c = __dsub_rn(c, tS);
  if (f & kNHT) c = __dsub_rn(c, tT);
  if (f & kNHB) c = __dsub_rn(c, tB);
  // apply_op_3D: kk outermost, then jj, then ii; zero coefficients add nothing
  double a = 0.0;
  if (f & kNHB) a = __dadd_rn(a, __dmul_rn(tB, vb));
  if (f & kNHS) a = __dadd_rn(a, __dmul_rn(tS, vs));
  if (f & kNHW) a = __dadd_rn(a, __dmul_rn(tW, vw));
  a = __dadd_rn(a, __dmul_rn(c, vc));
  if (f & kNHE) a = __dadd_rn(a, __dmul_rn(tE, ve));
  if (f & kNHN) a = __dadd_rn(a, __dmul_rn(tN, vn));
  if (f & kNHT) a = __dadd_rn(a, __dmul_rn(tT, vt));
  return a;
}

// Operator row of cell (i,j,k) applied to a field given by fetch(di, dj, dk).
template <class Fetch>
__device__ __forceinline__ double nh_apply(const NHOp& op, const NHGeo& G, int i, int j, int k, uint32_t f,
                                           const Fetch& fetch) {
  const size_t q2 = G.g.at(i, j);  // the tables are read-only for the life of the operator
  const double tE = (f & kNHE) ? __ldg(op.tE + q2) : 0.0;
  const double tW = (f & kNHW) ? __ldg(op.tW + q2) : 0.0;
  const double tN = (f & kNHN) ? __ldg(op.tN + j + 1) : 0.0;
  const double tS = (f & kNHS) ? __ldg(op.tS + j + 1) : 0.0;
  const double tT = (f & kNHT) ? __ldg(op.tT + k - 1) : 0.0;
  const double tB = (f & kNHB) ? __ldg(op.tB + k - 1) : 0.0;
  return nh_row(f, tE, tW, tN, tS, tT, tB, (f & kNHB) ? fetch(0, 0, -1) : 0.0, (f & kNHS) ? fetch(0, -1, 0) : 0.0,
                (f & kNHW) ? fetch(-1, 0, 0) : 0.0, fetch(0, 0, 0), (f & kNHE) ? fetch(1, 0, 0) : 0.0,
                (f & kNHN) ? fetch(0, 1, 0) : 0.0, (f & kNHT) ? fetch(0, 0, 1) : 0.0);
}

// setcyclic_xyz (parallel_none.f90) applied per level: store v at (i,j,k) and
// at the halo copies of (i,j) on that level.
template <typename T>
__device__ __forceinline__ void nh_store_cyclic(T* __restrict__ a, const NHGeo& G, int i, int j, int k, T v) {
  store_cyclic(a + (size_t)(k - 1) * G.plane, G.g, i, j, v);
}
template <typename T>
__device__ __forceinline__ void nh_add_cyclic(T* __restrict__ a, const NHGeo& G, int i, int j, int k, T d) {
  add_cyclic(a + (size_t)(k - 1) * G.plane, G.g, i, j, d);
}

struct CGResult;

// Bricks of the CG sweeps: 32 cells in i (one per lane) x ty in j x kc in k,
// kc = (8/ty) * kw.  Warp w works on row jj = w % ty and marches over kw
// levels from (w / ty) * kw.  Per brick and pipeline stage, shared memory
// holds two boxes (brick + one-cell halo: i0-2..i0+33, i.e. 36 doubles
// starting on a 16-byte boundary of the padded layout, j0-1..j0+ty,
// k0-1..k0+kc) -- sweep A: res and s; sweep B: s and, in the second box's
// place, the brick's res and p -- and the brick's flag bytes.
constexpr int kNHBoxX = 36;
__host__ __device__ constexpr size_t nh_al(size_t b) { return (b + 127) / 128 * 128; }
__host__ __device__ constexpr size_t nh_rs_bytes(int ty, int kc) { return (size_t)kNHBoxX * (ty + 2) * (kc + 2) * 8; }
__host__ __device__ constexpr size_t nh_p_bytes(int ty, int kc) { return (size_t)32 * ty * kc * 8; }
__host__ __device__ constexpr size_t nh_f_bytes(int ty, int kc) { return (size_t)32 * ty * kc; }
// stage layout: [box 0][region 1: box 1, or the brick's res then p][flags]
__host__ __device__ constexpr size_t nh_region1_bytes(int ty, int kc) {
  return nh_al(nh_rs_bytes(ty, kc)) > 2 * nh_al(nh_p_bytes(ty, kc)) ? nh_al(nh_rs_bytes(ty, kc))
                                                                       : 2 * nh_al(nh_p_bytes(ty, kc));
}
__host__ __device__ constexpr size_t nh_flags_off(int ty, int kc) {
  return nh_al(nh_rs_bytes(ty, kc)) + nh_region1_bytes(ty, kc);
}
__host__ __device__ constexpr size_t nh_stage_bytes(int ty, int kc) {
  return nh_flags_off(ty, kc) + nh_al(nh_f_bytes(ty, kc));
}
// ns pipeline stages (2..4) + a full and an empty mbarrier per stage
constexpr int kNHMaxStages = 4;
__host__ __device__ constexpr size_t nh_smem_bytes(int ty, int kc, int ns) {
  return (size_t)ns * nh_stage_bytes(ty, kc) + 128;
}
constexpr size_t kNHSmemMax = 220 * 1024;

struct alignas(64) NHParams {
  CUtensorMap map_res, map_s[2];     // 3-D (pitch, ny+4, nz) maps, box 36 x (ty+2) x (kc+2)
  CUtensorMap map_res_brick;         // the same array as map_res, box 32 x ty x kc
  CUtensorMap map_p;                 // 3-D (pitch, ny+4, nz) map of p, box 32 x ty x kc
  CUtensorMap map_f;                 // 3-D (fx, ny, nz) map of the flags, box 32 x ty x kc
  NHGeo G;
  NHOp op;
  int ty, kw, kc;                    // brick shape
  int ns;                            // pipeline stages
  int small_chunk;                   // cluster variant: cells per block
  int nbx, nby, nbz;                 // bricks per dimension
  const double* forc;  // Fortran layout (nx+4, ny+4, nz), device
  double* p;           // padded p_non_hydro(:,:,:,taup1), in/out
  double* res;         // padded residual (halo = cyclic copies), updated in place
  double* s[2];        // padded search direction, double-buffered
  double eps;          // congr_epsilon_non_hydro
  int max_it;          // congr_max_itts_non_hydro
  double rtol;         // > 0: extra stop on the recursive residual, sqrt(sum r^2 maskT / sum forc^2 maskT)
  SyncCtl* ctl;
  double* slots;       // 2 * gridDim.x * 4 doubles
  unsigned long long timeout_ns;
  unsigned stall_extra;
  CGResult* out;
};

// Arrays of one solve_non_hydrostatic step (non_hydrostatic.f90:5-63), all
// device memory in Fortran layout; the u, v, w, p pointers are already offset
// to their time level.
struct NHStep {
  NHGeo G;
  const double *dxt, *dxu, *dyt, *dyu, *cost, *cosu;  // [nx+4] / [ny+4]
  const double *dzt, *dzw;                            // [nz]
  const uint8_t *maskU, *maskV, *maskW;               // (nx+4, ny+4, nz), 0/1
  double *u, *v, *w;                                  // taup1
  const double *w_tau, *dw_tau, *dw_taum1, *dw_mix;
  double *p1;                                         // p_non_hydro(:,:,:,taup1)
  const double *p0, *pm;                              // tau, taum1
  double* forc;                                       // (nx+4, ny+4, nz) scratch
  double dt_mom, AB_eps;
};
void launch_nh_step_pre(const NHStep& S, cudaStream_t st);
void launch_nh_step_post(const NHStep& S, cudaStream_t st);

const void* nh_cg_kernel_ptr(bool cyclic_x, bool cyclic_y);

// cluster variant for small grids: res, direction and flags distributed over
// the shared memory of up to kNHMaxCluster blocks
constexpr int kNHSmallThreads = 1024;
constexpr int kNHMaxCluster = 16;
constexpr size_t nh_small_smem_bytes(size_t chunk) { return (chunk * 33 + 15) / 16 * 16; }
constexpr size_t kNHSmallSmemMax = 223 * 1024;  // 227 KB per block less room for the static buffers
constexpr int kNHSmallMaxChunk = (int)(kNHSmallSmemMax / 33);
constexpr int kNHSmallMaxCells = kNHMaxCluster * kNHSmallMaxChunk;
constexpr int kNHClusterAuto = 32768;  // automatic choice: the cluster kernel up to this many cells
const void* nh_cg_small_kernel_ptr(bool cyclic_x, bool cyclic_y);
void launch_nh_apply(const NHGeo& G, const NHOp& op, const double* p, double* res, cudaStream_t st);
void launch_nh_pack(const NHGeo& G, const double* user, double* padded, cudaStream_t st);
void launch_nh_unpack(const NHGeo& G, const double* padded, double* user, cudaStream_t st);

}  // namespace pyomgpu
