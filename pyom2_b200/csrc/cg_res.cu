// On-chip-resident Jacobi-PCG kernel for congrad_streamfunction
// (solve_streamfct.f90:153-327): the control flow of cg_ref_kernel<false>,
// laid out so that an iteration moves no field through HBM and only the
// piece boundaries through L2.
//
// The grid is cut into npx x npy rectangular pieces, one per block and one
// block per SM (512 threads, cooperative launch).  For the whole solve a block
// keeps
//   shared memory: the search direction with a one-cell halo and the x- and
//                  y-face couplings FX, FY of its piece (~180 KB for a 160 x 45
//                  piece, i.e. 1440 x 720 over 144 SMs);
//   TMEM:          the residual, the solution and the preconditioner Z of the
//                  points a thread owns (tcgen05.ld/st of whole 32-bit columns
//                  of the thread's lane; no MMA), 96 of the 128 columns each
//                  thread of a 512-thread block can reach;
//   registers:     the direction and one more value per point: Z*res between
//                  the residual update and the next direction, As between the
//                  stencil and the residual update.
// Warps 1-15 own the points: a thread owns a column segment of P points, so
// the north and south neighbours of its stencil come from its own registers.
// Warp 0 runs the reductions across blocks and the control flow, so the
// registers of its exp/log arithmetic do not add to the workers' arrays.
//
// Reductions and halo exchange use no arrival counter:
//   * each block writes its partial sums into its own slot (the last word with
//     st.release); warp 0 of every block polls all slots (lane l: slots l,
//     l+32, ...) until no word is empty any more, and the sums are formed in a
//     fixed order, so all blocks obtain bit-identical scalars and take the
//     same decisions.  Slots rotate over three buffers; a block empties its
//     slot of epoch e+2 as soon as it completes epoch e, when every reader of
//     the slot's previous contents has finished.
//   * after the residual update a block stages (Z*res, s) of its boundary
//     points in shared memory and its workers copy them, one entry each, into
//     exchange records (4 words per padded position, with the setcyclic_xy
//     copies) before its slot is released, so once a block has acquired every slot
//     of that reduction the values of its halo are visible: it loads them
//     once (bypassing L1) and recomputes the neighbours' next direction on
//     the halo with the operation their owner uses.  A value is overwritten
//     only in the next sweep B, after the reader has published the next
//     reduction, which it does after its loads have returned.  Nothing polls
//     the exchange arrays (polling them from every thread swamped L2).
// Every wait is bounded by %globaltimer; on time-out the kernel records
// PYOMGPU_TIMEOUT in the control block, frees its TMEM and returns.
#include <math.h>

#include <type_traits>

#include "cg_res.cuh"
#include "tc.cuh"

namespace pyomgpu {
namespace {

__device__ __forceinline__ double ld_relaxed_f64(const double* p) {
  double v;
  asm volatile("ld.relaxed.gpu.global.f64 %0, [%1];" : "=d"(v) : "l"(p) : "memory");
  return v;
}
// Plain store, cached in L2 only (ordered before a later st.release of the
// same thread, or of thread 0 after a block barrier).
__device__ __forceinline__ void st_weak_f64(double* p, double v) { __stcg(p, v); }
// Relaxed (morally strong) store at GPU scope: a reader may observe it with a
// relaxed load and validate it on its own.
__device__ __forceinline__ void st_relaxed_f64(double* p, double v) {
  asm volatile("st.relaxed.gpu.global.f64 [%0], %1;" ::"l"(p), "d"(v) : "memory");
}
// Acquire side of the slot protocol: after relaxed loads have observed the
// released words of every slot, one fence makes everything released before
// them visible (the acquire pattern of the PTX memory model).
__device__ __forceinline__ void fence_acq_rel_gpu() { asm volatile("fence.acq_rel.gpu;" ::: "memory"); }

// ---- tagged words (two-reduction kernel) --------------------------------------
// A double travels as two 64-bit words, (tag << 32) | low half and (tag << 32) |
// high half, stored and loaded relaxed.  64-bit accesses are single-copy atomic,
// so a reader that sees the current tag in both words has both halves of the
// current value; a stale word carries an older tag.  No ordering between words
// is needed, hence no release, acquire or emptying.  The tag is the solve's
// generation (12 bits) and the epoch (20 bits; a stale word is at most two epochs
// old, so the wrap-around cannot confuse them).  Slots and records are filled
// with all-ones words before every solve, a tag no solve uses (generations stop
// at 4094), so no word left by an earlier solve or kernel can pass as current.
__device__ __forceinline__ unsigned res_tag(const CGResParams& P, unsigned ep) {
  return (P.tag_gen << 20) | (ep & 0xFFFFFu);
}
__device__ __forceinline__ void st_relaxed_u64(unsigned long long* p, unsigned long long v) {
  asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ unsigned long long tag_lo(unsigned tag, double v) {
  return ((unsigned long long)tag << 32) | (unsigned)__double2loint(v);
}
__device__ __forceinline__ unsigned long long tag_hi(unsigned tag, double v) {
  return ((unsigned long long)tag << 32) | (unsigned)__double2hiint(v);
}
__device__ __forceinline__ bool tag_ok(unsigned long long w, unsigned tag) { return (unsigned)(w >> 32) == tag; }
__device__ __forceinline__ double untag(unsigned long long lo, unsigned long long hi) {
  return __hiloint2double((int)(unsigned)hi, (int)(unsigned)lo);
}
__device__ __forceinline__ void st_release_f64(double* p, double v) {
  asm volatile("st.release.gpu.global.f64 [%0], %1;" ::"l"(p), "d"(v) : "memory");
}
__device__ __forceinline__ bool is_empty(double v) {
  return (unsigned long long)__double_as_longlong(v) == kResEmpty;
}
__device__ __forceinline__ double empty_word() { return __longlong_as_double((long long)kResEmpty); }
// A NaN that carries the empty pattern is sent as the canonical NaN.
__device__ __forceinline__ double sendable(double v) {
  return is_empty(v) ? __longlong_as_double(0x7fffffffffffffffll) : v;
}

// Writes v into the exchange record (4 words per padded position; a word
// offset is already added to a) of interior (i,j) and of the halo positions
// setcyclic_xy fills from it.
__device__ __forceinline__ void publish_cyclic(double* a, const Geo& g, int i, int j, double v) {
  st_weak_f64(a + 4 * g.at(i, j), v);
  int xc, yc;
  cyclic_copies(g, i, j, xc, yc);
  if (xc != 0x7fffffff) st_weak_f64(a + 4 * g.at(xc, j), v);
  if (yc != 0x7fffffff) {
    st_weak_f64(a + 4 * g.at(i, yc), v);
    if (xc != 0x7fffffff) st_weak_f64(a + 4 * g.at(xc, yc), v);
  }
}

// 32-byte relaxed accesses (four tagged words; each word is validated on its own,
// so the access need not be single-copy atomic as a whole).  The address is
// 32-byte aligned.
__device__ __forceinline__ void st_relaxed_v4_u64(unsigned long long* p, unsigned long long w0, unsigned long long w1,
                                                  unsigned long long w2, unsigned long long w3) {
  asm volatile("st.relaxed.gpu.global.v4.u64 [%0], {%1, %2, %3, %4};" ::"l"(p), "l"(w0), "l"(w1), "l"(w2), "l"(w3)
               : "memory");
}
__device__ __forceinline__ void ld_relaxed_v4_u64(const unsigned long long* p, unsigned long long& w0,
                                                  unsigned long long& w1, unsigned long long& w2,
                                                  unsigned long long& w3) {
  asm volatile("ld.relaxed.gpu.global.v4.u64 {%0, %1, %2, %3}, [%4];"
               : "=l"(w0), "=l"(w1), "=l"(w2), "=l"(w3)
               : "l"(p)
               : "memory");
}
// The same four words read by atomic no-op read-modify-writes (OR with 0).  An
// RMW is performed where the line is owned and reads the latest value; a gang
// whose blocks had polled one slot for microseconds with plain loads saw its
// new value ~2 us after the writer's fence, and with these reads mixed in it
// left a two-group lag (half the blocks ~2.5 us behind, alternating at the two
// reductions) less often.
__device__ __forceinline__ void rmw_read_v4_u64(const unsigned long long* p, unsigned long long& w0,
                                                unsigned long long& w1, unsigned long long& w2,
                                                unsigned long long& w3) {
  unsigned long long* q = const_cast<unsigned long long*>(p);
  asm volatile("atom.relaxed.gpu.global.or.b64 %0, [%1], 0;" : "=l"(w0) : "l"(q) : "memory");
  asm volatile("atom.relaxed.gpu.global.or.b64 %0, [%1], 0;" : "=l"(w1) : "l"(q + 1) : "memory");
  asm volatile("atom.relaxed.gpu.global.or.b64 %0, [%1], 0;" : "=l"(w2) : "l"(q + 2) : "memory");
  asm volatile("atom.relaxed.gpu.global.or.b64 %0, [%1], 0;" : "=l"(w3) : "l"(q + 3) : "memory");
}

__device__ __forceinline__ void st_relaxed_v2_u64(unsigned long long* p, unsigned long long w0, unsigned long long w1) {
  asm volatile("st.relaxed.gpu.global.v2.u64 [%0], {%1, %2};" ::"l"(p), "l"(w0), "l"(w1) : "memory");
}
__device__ __forceinline__ void ld_relaxed_v2_u64(const unsigned long long* p, unsigned long long& w0,
                                                  unsigned long long& w1) {
  asm volatile("ld.relaxed.gpu.global.v2.u64 {%0, %1}, [%2];" : "=l"(w0), "=l"(w1) : "l"(p) : "memory");
}

// FP32 fields: (q, s) as the tagged record at padded position pos -- 2 words
// at 2 * pos, (tag << 32) | the value's bits -- in one 16-byte store.
__device__ __forceinline__ void put_record_tagged(unsigned long long* a, long long pos, float q, float s,
                                                  unsigned tag) {
  st_relaxed_v2_u64(a + 2 * pos, ((unsigned long long)tag << 32) | __float_as_uint(q),
                    ((unsigned long long)tag << 32) | __float_as_uint(s));
}

// Writes (q, s) as the tagged record at padded position pos -- 4 words at
// 4 * pos: q low, q high, s low, s high -- in one 32-byte store.
__device__ __forceinline__ void put_record_tagged(unsigned long long* a, long long pos, double q, double s,
                                                  unsigned tag) {
  st_relaxed_v4_u64(a + 4 * pos, tag_lo(tag, q), tag_hi(tag, q), tag_lo(tag, s), tag_hi(tag, s));
}

__device__ __forceinline__ void st_release_cta_u32(unsigned* p, unsigned v) {
  asm volatile("st.release.cta.shared.u32 [%0], %1;" ::"r"((uint32_t)__cvta_generic_to_shared(p)), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned ld_relaxed_cta_u32(const unsigned* p) {
  unsigned v;
  asm volatile("ld.relaxed.cta.shared.u32 %0, [%1];" : "=r"(v) : "r"((uint32_t)__cvta_generic_to_shared(p)) : "memory");
  return v;
}

// 16 bytes global -> shared, asynchronous and not cached in L1 (both
// addresses 16-byte aligned); completed by cp_async_wait.
__device__ __forceinline__ void cp_async16(void* sdst, const void* gsrc) {
  const uint32_t d = (uint32_t)__cvta_generic_to_shared(sdst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.commit_group;\n\tcp.async.wait_all;" ::: "memory");
}

// An integer the compiler has to treat as produced here: index arithmetic
// derived from it is redone in each sweep instead of being hoisted out of the
// iteration loop and held in registers for the whole solve.
__device__ __forceinline__ int opaque(int v) {
  asm volatile("" : "+r"(v));
  return v;
}

// --------------------------------------------------------------------- TMEM
// 32x32b shape: thread t of warp w moves whole 32-bit columns of TMEM lane
// 32*(w%4) + t; a double occupies two adjacent columns (low word first).
__device__ __forceinline__ void tm_ld8(uint32_t taddr, uint32_t (&v)[8]) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
               : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7])
               : "r"(taddr)
               : "memory");
}
__device__ __forceinline__ void tm_st8(uint32_t taddr, const uint32_t (&v)[8]) {
  asm volatile("tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};" ::"r"(taddr), "r"(v[0]),
               "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]), "r"(v[7])
               : "memory");
}
__device__ __forceinline__ void tm_ld16(uint32_t taddr, uint32_t (&v)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]), "=r"(v[8]),
        "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
      : "r"(taddr)
      : "memory");
}
__device__ __forceinline__ void tm_st16(uint32_t taddr, const uint32_t (&v)[16]) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16};" ::"r"(
          taddr),
      "r"(v[0]), "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]), "r"(v[7]), "r"(v[8]), "r"(v[9]),
      "r"(v[10]), "r"(v[11]), "r"(v[12]), "r"(v[13]), "r"(v[14]), "r"(v[15])
      : "memory");
}
// N = 8 or 16 columns
template <int N>
__device__ __forceinline__ void tm_ld(uint32_t taddr, uint32_t (&v)[N]) {
  if constexpr (N == 8)
    tm_ld8(taddr, v);
  else
    tm_ld16(taddr, v);
}
template <int N>
__device__ __forceinline__ void tm_st(uint32_t taddr, const uint32_t (&v)[N]) {
  if constexpr (N == 8)
    tm_st8(taddr, v);
  else
    tm_st16(taddr, v);
}
__device__ __forceinline__ void tm_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void tm_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ double col_get(const uint32_t* v, int k) {
  return __hiloint2double((int)v[2 * k + 1], (int)v[2 * k]);
}
__device__ __forceinline__ void col_put(uint32_t* v, int k, double d) {
  v[2 * k] = (uint32_t)__double2loint(d);
  v[2 * k + 1] = (uint32_t)__double2hiint(d);
}
// FP32 fields: one column per value
__device__ __forceinline__ void col_put(uint32_t* v, int k, float f) { v[k] = __float_as_uint(f); }
template <typename T>
__device__ __forceinline__ T colT_get(const uint32_t* v, int k) {
  if constexpr (sizeof(T) == 8)
    return __hiloint2double((int)v[2 * k + 1], (int)v[2 * k]);
  else
    return __uint_as_float(v[k]);
}

// The operator and vectors of a solve in the field type T (FP64, or the FP32
// copies of the mixed-precision correction solve).
template <typename T>
__device__ __forceinline__ OpDev<T> res_op(const CGResParams& P) {
  if constexpr (sizeof(T) == 8) return P.op; else return P.op32;
}
template <typename T>
__device__ __forceinline__ const T* res_forc(const CGResParams& P) {
  if constexpr (sizeof(T) == 8) return P.forc; else return P.forc32;
}
template <typename T>
__device__ __forceinline__ T* res_solv(const CGResParams& P) {
  if constexpr (sizeof(T) == 8) return P.sol; else return P.sol32;
}
template <typename T>
__device__ __forceinline__ T* res_resv(const CGResParams& P) {
  if constexpr (sizeof(T) == 8) return P.res; else return P.res32;
}

// ------------------------------------------------------------ control flow
// Scalars of the solve in shared memory, advanced by thread 0 only (the
// reference's congrad_streamfunction variables).
struct ResCtl {
  double beta, bb, rtol2bb, betam1, betamin, step1, est, bq, alpha;
  int n, status, act, stop_after;
};
constexpr int kRun = 0, kDoneOk = 1, kDoneErr = 2, kNeedMaxp = 3;
constexpr int kStepInit = 0, kStepA = 1, kStepB = 2, kStepInitD = 3, kStepIter = 4, kStepMaxp = 5;

__device__ __forceinline__ void ctl_stop(ResCtl& C, int act, int status) {
  C.act = act;
  C.status = status;
}

// Start of iteration C.n: max_it, NaN and divergence tests, beta/betam1.
__device__ void ctl_begin(ResCtl& C, const CGResParams& P) {
  if (C.n > P.max_it) return ctl_stop(C, kDoneErr, PYOMGPU_MAXITER);  // solve_streamfct.f90:303-304
  if (C.beta != C.beta) {  // early NaN stop (the reference runs on and halts at the end)
    C.est = C.beta;
    return ctl_stop(C, kDoneErr, PYOMGPU_NAN);
  }
  if (C.n == 1) {  // :232-240
    C.betamin = fabs(C.beta);
  } else if (C.n > 2) {
    C.betamin = fmin(C.betamin, fabs(C.beta));
    if (fabs(C.beta) > 100.0 * C.betamin) return ctl_stop(C, kDoneErr, PYOMGPU_DIVERGED);
  }
  C.bq = C.beta / C.betam1;  // :244
}

// v = (Z res, res), sum f^2 and sum res^2 over the unknowns, max|Z res|
__device__ void ctl_init(ResCtl& C, const CGResParams& P, const double* v) {
  C.beta = v[0];
  C.bb = v[1] > 0.0 ? v[1] : v[2];  // the rtol stop relative to ||res_0|| for a zero forcing
  C.rtol2bb = P.rtol * P.rtol * C.bb;
  C.betam1 = 1.0;
  C.betamin = C.step1 = C.est = C.bq = C.alpha = 0.0;
  C.n = 0;
  C.status = PYOMGPU_OK;
  C.act = kRun;
  C.stop_after = 0;
  if (100.0 * v[3] < P.eps) {  // solve_streamfct.f90:210-213
    C.est = 100.0 * v[3];
    return ctl_stop(C, kDoneOk, PYOMGPU_OK);
  }
  C.n = 1;
  ctl_begin(C, P);
}

// v = (s, As), max|s|
__device__ void ctl_after_a(ResCtl& C, const CGResParams& P, const double* v) {
  const double F_1EM10 = (double)1.e-10f;  // solve_streamfct.f90:262, a default-real literal
  const double sAs = v[0], smax = v[1];
  C.stop_after = 0;
  if (fabs(sAs) < fabs(C.beta) * F_1EM10) {  // :262-266
    C.est = 100.0 * smax;
    return ctl_stop(C, kDoneOk, PYOMGPU_OK);
  }
  C.alpha = C.beta / sAs;
  const double step = fabs(C.alpha) * smax;  // :283-297, decided now, applied after the update
  if (C.n == 1) {
    C.step1 = step;
    C.est = step;
    C.stop_after = step < P.eps;
  } else if (step < P.eps) {
    const double rate = exp(log(step / C.step1) / (double)(C.n - 1));
    C.est = step * rate / (1.0 - rate);
    C.stop_after = C.est < P.eps;
  }
}

// v = (Z res, res) and sum res^2 over the unknowns of the updated residual
__device__ void ctl_after_b(ResCtl& C, const CGResParams& P, const double* v) {
  const double beta_next = v[0], rr_next = v[1];
  if (P.rtol > 0.0 && (C.bb > 0.0 ? rr_next <= C.rtol2bb : rr_next == 0.0)) {
    C.est = sqrt(rr_next);
    return ctl_stop(C, kDoneOk, PYOMGPU_OK);
  }
  C.betam1 = C.beta;
  C.beta = beta_next;
  C.n += 1;
  ctl_begin(C, P);
}

// Single-reduction form: with u = Z res, w = A u and the previous direction
// p' and s' = A p', the new direction p = u + bq p' has
//   (p, A p) = (u, w) + bq ((u, s') + (p', w)) + bq^2 (p', s'),
// the bilinear expansion of the reference's (p, Ap) (exact for any operator;
// this one is not symmetric, so the symmetric Chronopoulos-Gear shortcut
// (u, w) - bq beta / alpha' does not apply).  All four products come from the
// sweep before, so one reduction per iteration carries them with (Z res, res),
// the residual norm and max|p|.  Sets alpha, or C.act = kNeedMaxp when
// (p, Ap) is below the reference's breakdown threshold (its estimate then needs
// max|p| of the new direction: one more reduction).
__device__ void ctl1_direction(ResCtl& C, const CGResParams& P, const double* e) {
  const double F_1EM10 = (double)1.e-10f;  // solve_streamfct.f90:262, a default-real literal
  const double sAs = C.n == 1 ? e[0] : e[0] + C.bq * (e[1] + e[2]) + C.bq * C.bq * e[3];
  if (fabs(sAs) < fabs(C.beta) * F_1EM10) {  // :262-266
    C.act = kNeedMaxp;
    return;
  }
  C.alpha = C.beta / sAs;
}

// v = (Z res, res), (u, w), (u, s'), (p', w), (p', s'), sum res^2 over the
// unknowns of the updated residual and max|p| of iteration n, whose update is
// done (p', s' its direction and A-product): the reference's
// convergence test of iteration n (solve_streamfct.f90:283-297), the relative
// residual stop, then the start of iteration n+1.
__device__ void ctl1_iter(ResCtl& C, const CGResParams& P, const double* v) {
  const double step = fabs(C.alpha) * v[6];
  if (C.n == 1) {
    C.step1 = step;
    C.est = step;
    if (step < P.eps) return ctl_stop(C, kDoneOk, PYOMGPU_OK);
  } else if (step < P.eps) {
    const double rate = exp(log(step / C.step1) / (double)(C.n - 1));
    C.est = step * rate / (1.0 - rate);
    if (C.est < P.eps) return ctl_stop(C, kDoneOk, PYOMGPU_OK);
  }
  if (P.rtol > 0.0 && (C.bb > 0.0 ? v[5] <= C.rtol2bb : v[5] == 0.0)) {
    C.est = sqrt(v[5]);
    return ctl_stop(C, kDoneOk, PYOMGPU_OK);
  }
  C.betam1 = C.beta;
  C.beta = v[0];
  C.n += 1;
  ctl_begin(C, P);
  if (C.act == kRun) ctl1_direction(C, P, v + 1);
}

// ------------------------------------------------- reduction and exchange
template <typename T>
struct HaloT {
  int sidx;       // shared-memory index (-1: none)
  long long gidx; // padded position whose exchange record is received
  T q, s;         // received Z*res and direction
};
using Halo = HaloT<double>;


// Loads this thread's halo values from tagged records, polling (bounded) a
// record until both of its values carry `tag`.  False on time-out.
template <typename T>
__device__ __forceinline__ bool worker_halo_load_tagged(const CGResParams& P, HaloT<T> (&hl)[2], unsigned tag) {
  // parameters read once into registers (the polls' memory clobbers would reload them every spin)
  const unsigned long long* hx = reinterpret_cast<const unsigned long long*>(P.hx);
  int* const err = &P.ctl->error;
  const unsigned long long tmo = P.timeout_ns;
  const unsigned long long t0 = globaltimer_ns();
  // one record after the other (a worker rarely has two)
#pragma unroll 1
  for (int e = 0; e < 2; e++) {
    if (hl[e].sidx < 0) continue;
    for (unsigned spin = 1;; spin++) {
      bool ok;
      if constexpr (sizeof(T) == 8) {
        unsigned long long w0, w1, w2, w3;
        ld_relaxed_v4_u64(hx + 4 * hl[e].gidx, w0, w1, w2, w3);
        ok = tag_ok(w0, tag) && tag_ok(w1, tag) && tag_ok(w2, tag) && tag_ok(w3, tag);
        if (ok) {
          hl[e].q = untag(w0, w1);
          hl[e].s = untag(w2, w3);
        }
      } else {
        unsigned long long w0, w1;
        ld_relaxed_v2_u64(hx + 2 * hl[e].gidx, w0, w1);
        ok = tag_ok(w0, tag) && tag_ok(w1, tag);
        if (ok) {
          hl[e].q = __uint_as_float((unsigned)w0);
          hl[e].s = __uint_as_float((unsigned)w1);
        }
      }
      if (ok) break;
      if ((spin & 63u) == 0u && (ld_relaxed_i32(err) != 0 || globaltimer_ns() - t0 > tmo)) {
        atomicExch(err, PYOMGPU_TIMEOUT);
        return false;
      }
    }
  }
  return true;
}

// Boundary staging: the values of a piece's boundary points in shared memory,
// entries [0,ph) west column, [ph,2ph) east column, [2ph,2ph+pw) south row,
// [2ph+pw,2ph+2pw) north row (a corner point in two entries); quantity k of
// entry e at k*nent+e.  One quantity of one point:
template <typename T>
__device__ __forceinline__ void stage_one(T* spub, int pw, int ph, int lx, int ly, T v) {
  if (lx == 0) spub[ly] = v;
  if (lx == pw - 1) spub[ph + ly] = v;
  if (ly == 0) spub[2 * ph + lx] = v;
  if (ly == ph - 1) spub[2 * ph + pw + lx] = v;
}

// The staged boundary values (NQ quantities) to the exchange records (word k
// of a position's record, with the setcyclic_xy copies), one entry per worker
// thread; only the edges some block reads.
template <int NQ>
__device__ __forceinline__ void copy_out(const CGResParams& P, double* hx, const double* spub, int ilo, int ihi,
                                         int jlo, int jhi, int wt) {
  const Geo& g = P.g;
  const int pw = ihi - ilo + 1, ph = jhi - jlo + 1, nent = 2 * (pw + ph);
#pragma unroll 1
  for (int e = wt; e < nent; e += kResWorkers) {
    int i, j;
    bool need;
    if (e < ph) {
      i = ilo;
      j = jlo + e;
      need = ilo > 1 || g.cyclic_x;
    } else if (e < 2 * ph) {
      i = ihi;
      j = jlo + e - ph;
      need = ihi < g.nx || g.cyclic_x;
    } else if (e < 2 * ph + pw) {
      i = ilo + e - 2 * ph;
      j = jlo;
      need = jlo > 1 || g.cyclic_y;
    } else {
      i = ilo + e - 2 * ph - pw;
      j = jhi;
      need = jhi < g.ny || g.cyclic_y;
    }
    if (need) {
#pragma unroll
      for (int k = 0; k < NQ; k++) publish_cyclic(hx + k, g, i, j, spub[k * nent + e]);
    }
  }
}

// copy_out<2> for tagged records: (Z res, direction) of each staged boundary
// entry, written once, at the position the block across that edge polls: the
// point itself when the neighbour is an interior piece, its setcyclic_xy image
// in the domain halo (setcyclic_x: a(nx+1) = a(1), a(0) = a(nx); the same in y)
// when the edge is a cyclic domain edge; nothing at a closed domain edge.
template <typename T>
__device__ __forceinline__ void copy_out_tagged(const CGResParams& P, const T* spub, int ilo, int ihi, int jlo,
                                                int jhi, int wt, unsigned tag) {
  const Geo g = P.g;
  unsigned long long* hx = reinterpret_cast<unsigned long long*>(P.hx);
  const int pw = ihi - ilo + 1, ph = jhi - jlo + 1, nent = 2 * (pw + ph);
#pragma unroll 1
  for (int e = wt; e < nent; e += kResWorkers) {
    int i, j;
    bool own, img;
    if (e < ph) {  // west column
      i = ilo;
      j = jlo + e;
      own = ilo > 1;
      img = !own && g.cyclic_x;
    } else if (e < 2 * ph) {  // east column
      i = ihi;
      j = jlo + e - ph;
      own = ihi < g.nx;
      img = !own && g.cyclic_x;
    } else if (e < 2 * ph + pw) {  // south row
      i = ilo + e - 2 * ph;
      j = jlo;
      own = jlo > 1;
      img = !own && g.cyclic_y;
    } else {  // north row
      i = ilo + e - 2 * ph - pw;
      j = jhi;
      own = jhi < g.ny;
      img = !own && g.cyclic_y;
    }
    if (!own && !img) continue;
    int ti = i, tj = j;
    if (img) {
      if (e < ph)
        ti = g.nx + 1;
      else if (e < 2 * ph)
        ti = 0;
      else if (e < 2 * ph + pw)
        tj = g.ny + 1;
      else
        tj = 0;
    }
    put_record_tagged(hx, g.at(ti, tj), spub[e], spub[nent + e], tag);
  }
}

__device__ __forceinline__ double* res_slot(const CGResParams& P, unsigned ep, int b) {
  return P.slots + ((size_t)(ep % 3u) * P.nslot + b) * kResSlotWords;
}

// Worker side of a reduction: per-warp partials of the worker warps into wred.
template <int NV, int kMaxSlot>
__device__ __forceinline__ void worker_partials(const double (&v)[NV], double (*wred)[kResSlotWords]) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < NV; k++) {
    const double r = (k == kMaxSlot) ? warp_max(v[k]) : warp_sum(v[k]);
    if (lane == 0) wred[w][k] = r;
  }
}

// Controller side of epoch ep (warp 0, after the workers' partials are in
// wred): lane 0 sums them in warp order and publishes the block's slot (last
// word with st.release); lane l polls the slots l, l+32, ... of all npoll
// blocks until no word is empty; the totals are formed in a fixed order, so
// every block obtains the same bits, and lane 0 advances the control state.
// False on time-out.
// FRESH (tagged slots only): the pending slots are also read with
// rmw_read_v4_u64 instead of loads -- in a gang of at most kFreshEagerSlots - 1
// blocks on every pass after the second, in a larger one on every 8th pass
// once the poll has lasted kFreshPollNs (there the RMWs of all lanes of ~150
// blocks on every pass slowed each reduction).  On the 64 basins: 362 ms per
// batch with the eager reads in small gangs, 376-389 ms with the timed ones
// alone.
constexpr unsigned long long kFreshPollNs = 1500;
constexpr int kFreshEagerSlots = 97;
template <int NV, int kMaxSlot, int kStep, bool TAG = false, bool FRESH = false>
__device__ __forceinline__ bool controller_epoch(const CGResParams& P, unsigned ep, int bid, int npoll, ResCtl& C,
                                                 const double (*wred)[kResSlotWords], unsigned* hflag = nullptr,
                                                 unsigned long long* tr = nullptr) {
  const int lane = threadIdx.x;
  const unsigned tag = res_tag(P, ep);
  // parameters read once into registers (the polls' memory clobbers would reload them every spin)
  unsigned long long* const slot_base = reinterpret_cast<unsigned long long*>(P.slots);
  const int nslot = P.nslot;
  int* const err = &P.ctl->error;
  const unsigned long long tmo = P.timeout_ns;
  // tagged slots: 2 buffers x nslot x 2 kResSlotWords words; a block overwrites its
  // slot of epoch ep at ep+2, when every block has published ep+1, i.e. finished
  // reading epoch ep
  auto tslot = [&](unsigned e, int b) {
    return slot_base + ((size_t)(e & 1u) * nslot + b) * (2 * kResSlotWords);
  };
  if constexpr (TAG) {
    double t[NV];
#pragma unroll
    for (int k = 0; k < NV; k++) {
      const double x = (lane >= 1 && lane < kResThreads / 32) ? wred[lane][k] : 0.0;
      t[k] = (k == kMaxSlot) ? warp_max(x) : warp_sum(x);
    }
    double mv = 0.0;
#pragma unroll
    for (int k = 0; k < NV; k++)
      if ((lane >> 1) == k) mv = t[k];
    if (lane < 2 * NV) {
      st_relaxed_u64(tslot(ep, bid) + lane, (lane & 1) ? tag_hi(tag, mv) : tag_lo(tag, mv));
      // pushes the slot out before this block starts polling: without it a
      // relaxed store stayed invisible to the other blocks for ~2-3 us at times,
      // and dense gangs settled into two groups ~2.5 us apart (13-14 us per
      // iteration instead of ~9.5; no cost measured on the 1440x720 solve)
      asm volatile("fence.acq_rel.gpu;" ::: "memory");
    }
    if (tr != nullptr && lane == 0) tr[0] = globaltimer_ns();
  } else {
    double t[NV];  // lane w holds worker warp w's partials; fixed shuffle tree
#pragma unroll
    for (int k = 0; k < NV; k++) {
      const double x = (lane >= 1 && lane < kResThreads / 32) ? wred[lane][k] : 0.0;
      t[k] = (k == kMaxSlot) ? warp_max(x) : warp_sum(x);
    }
    // one word per lane (a lone lane's stores go out one after another); the
    // last word, released after a warp barrier, makes the others visible
    double* mine = res_slot(P, ep, bid);
    double mv = 0.0;
#pragma unroll
    for (int k = 0; k < NV; k++)
      if (lane == k) mv = t[k];
    if (lane < NV - 1) st_relaxed_f64(mine + lane, sendable(mv));
    __syncwarp();
    if (lane == NV - 1) st_release_f64(mine + NV - 1, sendable(mv));
    if (tr != nullptr && lane == 0) tr[0] = globaltimer_ns();
  }
  constexpr int kPer = kResMaxSlots / 32;
  double got[kPer][NV];
  unsigned want = 0, have = 0;
#pragma unroll
  for (int m = 0; m < kPer; m++) {
    if (lane + 32 * m < npoll) want |= 1u << m;
#pragma unroll
    for (int k = 0; k < NV; k++) got[m][k] = 0.0;
  }
  bool ok = true;
  const unsigned long long t0 = globaltimer_ns();
  if constexpr (TAG) {
    // every tagged word of every slot this lane polls in one pass of relaxed
    // loads (RMW reads: the FRESH passes)
    auto pass = [&](auto rmw) {
      const unsigned pend = want & ~have;
#pragma unroll
      for (int m = 0; m < kPer; m++) {
        if (!(pend >> m & 1u)) continue;
        const unsigned long long* sl = tslot(ep, lane + 32 * m);
        bool all = true;
#pragma unroll
        for (int k = 0; k < NV; k += 2) {  // two values (four words, 32 bytes) per load
          unsigned long long w0, w1, w2, w3;
          if constexpr (decltype(rmw)::value)
            rmw_read_v4_u64(sl + 2 * k, w0, w1, w2, w3);
          else
            ld_relaxed_v4_u64(sl + 2 * k, w0, w1, w2, w3);
          all = all && tag_ok(w0, tag) && tag_ok(w1, tag);
          got[m][k] = untag(w0, w1);  // kept only once every word of the slot is current
          if (k + 1 < NV) {
            all = all && tag_ok(w2, tag) && tag_ok(w3, tag);
            got[m][k + 1] = untag(w2, w3);
          }
        }
        if (all) have |= 1u << m;
      }
    };
    const bool eager = nslot <= kFreshEagerSlots;
    for (unsigned spin = 1; have != want; spin++) {
      if constexpr (FRESH) {
        if (eager ? spin > 2u : (spin & 7u) == 0u && globaltimer_ns() - t0 > kFreshPollNs)
          pass(std::true_type{});
        else
          pass(std::false_type{});
      } else {
        pass(std::false_type{});
      }
      if (have != want && (spin & 31u) == 0u && (ld_relaxed_i32(err) != 0 || globaltimer_ns() - t0 > tmo)) {
        atomicExch(err, PYOMGPU_TIMEOUT);
        ok = false;
        break;
      }
    }
  } else {
  // every word of every slot this lane polls is loaded relaxed in one pass (the
  // loads are independent: one L2 round trip per pass) and validated on its own:
  // a word is either empty or this epoch's value (a slot is emptied two epochs
  // ahead, and the fence below orders those stores before the next poll)
  for (unsigned spin = 1; have != want; spin++) {
#pragma unroll
    for (int m = 0; m < kPer; m++) {
      if (!((want & ~have) >> m & 1u)) continue;
      const double* sl = res_slot(P, ep, lane + 32 * m);
#pragma unroll
      for (int k = 0; k < NV; k++) got[m][k] = ld_relaxed_f64(sl + k);
    }
#pragma unroll
    for (int m = 0; m < kPer; m++) {
      if (!((want & ~have) >> m & 1u)) continue;
      bool all = true;
#pragma unroll
      for (int k = 0; k < NV; k++) all = all && !is_empty(got[m][k]);
      if (all) have |= 1u << m;
    }
    if (have != want && (spin & 31u) == 0u && (ld_relaxed_i32(err) != 0 || globaltimer_ns() - t0 > tmo)) {
      atomicExch(err, PYOMGPU_TIMEOUT);
      ok = false;
      break;
    }
  }
  fence_acq_rel_gpu();
  }
  if (tr != nullptr && lane == 0) tr[1] = globaltimer_ns();
  if (hflag != nullptr) {
    // every slot is acquired, so the exchange records written before them are
    // visible (released with them, or tagged and validated by the readers): let
    // the workers start loading their halo before the control step
    __syncwarp();
    if (lane == 0) st_release_cta_u32(hflag, ld_relaxed_cta_u32(hflag) + 1u);
  }
  if constexpr (!TAG) {
    // once every lane has seen its slots of epoch ep, every block has finished
    // reading epoch ep-1 (it published epoch ep), so this block's slot of that
    // buffer (= the one of epoch ep+2) is free; the next publication's release
    // orders these stores before it
    __syncwarp();
    if (lane < kResSlotWords) st_weak_f64(res_slot(P, ep + 2, bid) + lane, empty_word());
  }
  double out[NV];
#pragma unroll
  for (int k = 0; k < NV; k++) {
    double a = 0.0;
#pragma unroll
    for (int m = 0; m < kPer; m++)
      if (have >> m & 1u) a = (k == kMaxSlot) ? fmax(a, got[m][k]) : a + got[m][k];
    out[k] = (k == kMaxSlot) ? warp_max(a) : warp_sum(a);
  }
  if (lane == 0) {
    if (kStep == kStepInit)
      ctl_init(C, P, out);
    else if (kStep == kStepA)
      ctl_after_a(C, P, out);
    else if (kStep == kStepB)
      ctl_after_b(C, P, out);
    else if (kStep == kStepInitD)
      ctl1_direction(C, P, out);
    else if (kStep == kStepIter)
      ctl1_iter(C, P, out);
    else {  // kStepMaxp: the breakdown estimate, solve_streamfct.f90:262-266
      C.est = 100.0 * out[0];
      ctl_stop(C, kDoneOk, PYOMGPU_OK);
    }
    if (tr != nullptr) tr[2] = globaltimer_ns();
  }
  return ok;
}


__device__ __forceinline__ void workers_sync() {
  asm volatile("bar.sync 1, %0;" ::"r"(kResWorkers) : "memory");
}

}  // namespace

// Block layout: warp 0 is the controller (reductions across blocks, control
// flow), warps 1-15 are the workers that own the points.  Both sides pass the
// same sequence of block barriers: S1 (the workers' partials are in shared
// memory) and S2 (the controller's decision is in shared memory, or a wait
// timed out).  Work that overlaps the wait of the other blocks (the solution
// update) runs between S1 and S2.
//
// One solve by the blocks 0 .. npx*npy-1 of a group (bid: this block's index in
// it); the caller has allocated the block's 512 TMEM columns (address in
// *s_tmem) and provides the dynamic shared memory sm.  Every block of the
// group calls it for the same solve; a block returns once its share is done
// (all threads together, after a block barrier).
// WGT: the inner products (Z res, res) and (s, As) weighted by the cell area
// D = 1/(ax by), in which A = D^-1 S is self-adjoint (the work-queue kernel's
// option for the psin solves).
// FRESH: the reduction polls mix in atomic reads after a long wait
// (controller_epoch), for the gangs of the multi-solve kernel.
template <typename T, int P, bool TRACE, bool WGT = false, bool FRESH = false>
__device__ __forceinline__ void res_solve(const CGResParams& Pm, const int bid, double* sm, const uint32_t* s_tmem_p,
                                          ResCtl& C, double (*wred)[kResSlotWords]) {
  // points per TMEM chunk (FP64: tcgen05 .x16 / .x8, .x16 at P = 16 spills; FP32: .x8)
  constexpr int CH = sizeof(T) == 4 ? 8 : (P == 8 ? 8 : 4);
  constexpr int NC = P / CH;                     // chunks per field
  constexpr int CW = (int)(sizeof(T) / 4) * CH;  // TMEM columns per chunk
  static_assert(P % CH == 0 && NC * CW <= 32, "a field takes at most 32 TMEM columns per thread");
  const Geo g = Pm.g;
  const OpDev<T> op = res_op<T>(Pm);
  const int warp = threadIdx.x >> 5;
  // traced instantiation: this block's timestamps of loop trip t (nullptr outside the window)
  auto trace_row = [&](unsigned t) -> unsigned long long* {
    if (!TRACE) return nullptr;
    const int k = (int)t - Pm.trace_it0;
    if (k < 0 || k >= Pm.trace_nit) return nullptr;
    return Pm.trace + ((size_t)bid * Pm.trace_nit + k) * kResTracePhases;
  };

  const int nb = Pm.npx * Pm.npy;
  const int px = bid % Pm.npx, py = bid / Pm.npx;
  const int ilo = 1 + (int)(((long long)px * g.nx) / Pm.npx);
  const int ihi = (int)(((long long)(px + 1) * g.nx) / Pm.npx);
  const int jlo = 1 + (int)(((long long)py * g.ny) / Pm.npy);
  const int jhi = (int)(((long long)(py + 1) * g.ny) / Pm.npy);
  const int pw = ihi - ilo + 1, ph = jhi - jlo + 1, sp = pw + 2;
  const int pw_ = pw, ph_ = ph, jlo_ = jlo;
  T* ss = reinterpret_cast<T*>(sm);  // (pw+2) x (ph+2): direction, halo included
  T* sfx = ss + sp * (ph + 2);        // (pw+1) x ph: FX(ilo+lx, j), lx = 0..pw
  T* sfy = sfx + (pw + 1) * ph;       // pw x (ph+1): FY(i, jlo+ly), ly = 0..ph
  T* sbx = sfy + pw * (ph + 1);       // ph: bx(jlo+ly), then ph: by(jlo+ly)
  T* spub = sbx + 2 * ph;             // 2 x 2(pw+ph): staged boundary Z*res, direction
  const int nent = 2 * (pw + ph);

  for (int e = threadIdx.x; e < sp * (ph + 2); e += kResThreads) ss[e] = (T)0;
  for (int e = threadIdx.x; e < (pw + 1) * ph; e += kResThreads)
    sfx[e] = op.FX[g.at(ilo + e % (pw + 1), jlo + e / (pw + 1))];
  for (int e = threadIdx.x; e < pw * (ph + 1); e += kResThreads) sfy[e] = op.FY[g.at(ilo + e % pw, jlo + e / pw)];
  for (int e = threadIdx.x; e < ph; e += kResThreads) {
    sbx[e] = op.bx[jlo + e + 1];
    sbx[ph + e] = op.by[jlo + e + 1];
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();

  if (warp == 0) {
    // ============================================================ controller
    unsigned ep = 0;
    bool stopped_after_update = false;  // the stop decided before sweep B (C stays as the workers read it)
    __syncthreads();  // S1
    bool ok = controller_epoch<4, 3, kStepInit, true, FRESH>(Pm, ep, bid, nb + (Pm.stall_extra ? 1 : 0), C, wred);
    if (!__syncthreads_and(ok)) goto out;  // S2
    if (C.act == kRun) {
      for (unsigned trip = 0;; trip++) {
        unsigned long long* tr = threadIdx.x == 0 ? trace_row(trip) : nullptr;
        __syncthreads();  // S1: partials of sweep A
        if (TRACE && tr) tr[10] = globaltimer_ns();
        ok = controller_epoch<2, 1, kStepA, true, FRESH>(Pm, ++ep, bid, nb, C, wred, nullptr,
                                                        TRACE && tr ? tr + 11 : nullptr);
        if (!__syncthreads_and(ok)) goto out;  // S2
        if (C.act != kRun) break;
        if (C.stop_after) {  // the workers finish sweep B and stop
          stopped_after_update = true;
          break;
        }
        __syncthreads();  // S1: partials of sweep B
        if (TRACE && tr) tr[14] = globaltimer_ns();
        ok = controller_epoch<2, -1, kStepB, true, FRESH>(Pm, ++ep, bid, nb, C, wred, nullptr,
                                                   TRACE && tr ? tr + 15 : nullptr);
        if (!__syncthreads_and(ok)) goto out;  // S2
        if (C.act != kRun) break;
      }
    }
    if (bid == 0 && threadIdx.x == 0) {
      const int converged = stopped_after_update || C.act == kDoneOk;
      Pm.out->iterations = C.n;
      Pm.out->converged = converged;
      Pm.out->status = converged ? PYOMGPU_OK : (C.est != C.est ? PYOMGPU_NAN : C.status);
      Pm.out->est = C.est;
    }
  } else {
    // =============================================================== workers
    // this thread's column segment: column lx, rows ly0 .. ly0+nrow-1
    const int wt = (int)threadIdx.x - 32;
    const int lx_ = wt % Pm.wmax;
    const int ly0_ = (wt / Pm.wmax) * P;
    const int nrow_ = (lx_ < pw && ly0_ < ph) ? min(P, ph - ly0_) : 0;
    const int i_ = ilo + lx_;
    int lx = lx_, ly0 = ly0_, nrow = nrow_, i = i_;
    const T axi = nrow_ > 0 ? op.ax[i_ + 1] : (T)0;
    // TMEM of this thread: lane 32*(warp%4)+lane, 32 columns per field from 128*(warp/4)
    const uint32_t tm = *s_tmem_p + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)(128 * (warp >> 2));
    const uint32_t t_res = tm, t_sol = tm + 32, t_z = tm + 64;

    // halo positions received (west, east, south, north edges that have a
    // neighbour; a non-cyclic domain edge keeps the zero direction)
    HaloT<T> hl[2];
    {
      const int nW = (ilo > 1 || g.cyclic_x) ? ph : 0, nE = (ihi < g.nx || g.cyclic_x) ? ph : 0;
      const int nS = (jlo > 1 || g.cyclic_y) ? pw : 0, nN = (jhi < g.ny || g.cyclic_y) ? pw : 0;
#pragma unroll
      for (int e = 0; e < 2; e++) {
        const int h = wt + e * kResWorkers;
        hl[e].sidx = -1;
        hl[e].gidx = 0;
        hl[e].q = hl[e].s = (T)0;
        if (h >= nW + nE + nS + nN) continue;
        int hx, hy;
        if (h < nW) {
          hx = -1;
          hy = h;
        } else if (h < nW + nE) {
          hx = pw;
          hy = h - nW;
        } else if (h < nW + nE + nS) {
          hx = h - nW - nE;
          hy = -1;
        } else {
          hx = h - nW - nE - nS;
          hy = ph;
        }
        hl[e].sidx = (hy + 1) * sp + hx + 1;
        hl[e].gidx = (long long)g.at(ilo + hx, jlo + hy);
      }
    }

    T s[P], q[P];  // direction; q: Z*res before sweep A, As after it
    unsigned hready = 0;  // halo-carrying reductions completed

    // ---------------------------------------------------------------- init
    // res = forc - A sol, solve_streamfct.f90:196-201
    {
      double v[4] = {0.0, 0.0, 0.0, 0.0};  // beta, bb, rr, zresmax
#pragma unroll
      for (int c = 0; c < NC; c++) {
        uint32_t br[CW], bz[CW], bx[CW];
#pragma unroll
        for (int k = 0; k < CH; k++) {
          const int u = c * CH + k;
          T rv = 0, w = 0, x = 0;
          s[u] = 0;
          q[u] = 0;
          if (u < nrow) {  // partial sums in FP64 for either field type
            const int ly = ly0 + u, j = jlo + ly;
            const T f = res_forc<T>(Pm)[sizeof(T) == 8 ? fidx(g.nx, i, j) : g.at(i, j)];
            rv = f - apply_point(op, g, (const T*)res_solv<T>(Pm), i, j);
            w = op.W[g.at(i, j)];
            x = res_solv<T>(Pm)[g.at(i, j)];
            const T zr = w * rv;
            if constexpr (WGT)
              v[0] += (1.0 / ((double)axi * (double)sbx[ph + ly]) * zr) * rv;
            else
              v[0] += (double)zr * (double)rv;
            if (w != (T)0) {
              v[1] += (double)f * (double)f;
              v[2] += (double)rv * (double)rv;
            }
            v[3] = fmax(v[3], fabs((double)zr));
            q[u] = zr;
            stage_one(spub, pw, ph, lx, ly, zr);
            stage_one(spub + nent, pw, ph, lx, ly, (T)0);
          }
          col_put(br, k, rv);
          col_put(bz, k, w);
          col_put(bx, k, x);
        }
        tm_st<CW>(t_res + c * CW, br);
        tm_st<CW>(t_z + c * CW, bz);
        tm_st<CW>(t_sol + c * CW, bx);
      }
      tm_wait_st();
      worker_partials<4, 3>(v, wred);
    }
    workers_sync();
    copy_out_tagged(Pm, spub, ilo, ihi, jlo, jhi, wt, res_tag(Pm, 2u * hready));
    __syncthreads();  // S1
    // the neighbours' records of this exchange, polled until they carry its tag
    if (!__syncthreads_and(worker_halo_load_tagged(Pm, hl, res_tag(Pm, 2u * hready++)))) goto out;  // S2
    if (C.act != kRun) goto done;

    for (unsigned trip = 0;; trip++) {
      unsigned long long* tr = threadIdx.x == 32 ? trace_row(trip) : nullptr;
      if (TRACE && tr) tr[0] = globaltimer_ns();
      // ---------------------------------------------- sweep A: direction, As
      lx = opaque(lx_);
      ly0 = opaque(ly0_);
      nrow = opaque(nrow_);
      {
        const int sp = opaque(pw + 2);
        const T bq = (T)C.bq;
#pragma unroll
        for (int u = 0; u < P; u++)
          if (u < nrow) {
            s[u] = q[u] + bq * s[u];
            ss[(ly0 + u + 1) * sp + lx + 1] = s[u];
          }
#pragma unroll
        for (int e = 0; e < 2; e++)
          if (hl[e].sidx >= 0) ss[hl[e].sidx] = hl[e].q + bq * hl[e].s;
      }
      workers_sync();
      if (TRACE && tr) tr[1] = globaltimer_ns();
      lx = opaque(lx_);
      ly0 = opaque(ly0_);
      nrow = opaque(nrow_);
      {
        const int pw = opaque(pw_), sp = pw + 2, ph = opaque(ph_);
        double v[2] = {0.0, 0.0};  // (s, As), max|s|
        if (nrow > 0) {
          T fys = sfy[ly0 * pw + lx];
#pragma unroll
          for (int u = 0; u < P; u++)
            if (u < nrow) {
              const int ly = ly0 + u;
              const int k = (ly + 1) * sp + lx + 1;
              const T sc = s[u];
              const T se = ss[k + 1], sw = ss[k - 1];
              const T sn = (u + 1 < P && u + 1 < nrow) ? s[u + 1 < P ? u + 1 : u] : ss[k + sp];
              const T so = (u > 0) ? s[u > 0 ? u - 1 : 0] : ss[k - sp];
              const T fxw = sfx[ly * (pw + 1) + lx], fxe = sfx[ly * (pw + 1) + lx + 1];
              const T fyn = sfy[(ly + 1) * pw + lx];
              const T a = axi * sbx[ly] * (fxe * (se - sc) + fxw * (sw - sc)) +
                          sbx[ph + ly] * (fyn * (sn - sc) + fys * (so - sc));
              if constexpr (WGT)
                v[0] += (1.0 / ((double)axi * (double)sbx[ph + ly]) * sc) * a;
              else
                v[0] += (double)sc * (double)a;
              v[1] = fmax(v[1], fabs((double)sc));
              q[u] = a;
              fys = fyn;
            }
        }
        worker_partials<2, 1>(v, wred);
      }
      if (TRACE && tr) tr[2] = globaltimer_ns();
      __syncthreads();                           // S1
      if (TRACE && tr) tr[3] = globaltimer_ns();
      if (!__syncthreads_and(1)) goto out;      // S2
      if (TRACE && tr) tr[4] = globaltimer_ns();
      if (C.act != kRun) goto done;
      // ---------------------------------------------- sweep B: residual update
      lx = opaque(lx_);
      ly0 = opaque(ly0_);
      nrow = opaque(nrow_);
      i = opaque(i_);
      {
        const int pw = opaque(pw_), ph = opaque(ph_), jlo = opaque(jlo_);
        const T alpha = (T)C.alpha;
        const bool stop_after = C.stop_after != 0;
        double v[2] = {0.0, 0.0};  // (Z res, res), sum res^2 over the unknowns
#pragma unroll
        for (int c = 0; c < NC; c++) {
          uint32_t br[CW], bz[CW];
          tm_ld<CW>(t_res + c * CW, br);
          tm_ld<CW>(t_z + c * CW, bz);
          tm_wait_ld();
#pragma unroll
          for (int k = 0; k < CH; k++) {
            const int u = c * CH + k;
            if (u < nrow) {
              const T w = colT_get<T>(bz, k);
              const T rv = colT_get<T>(br, k) - alpha * q[u];
              const T zr = w * rv;
              if constexpr (WGT)
                v[0] += (1.0 / ((double)axi * (double)sbx[ph + ly0 + u]) * zr) * rv;
              else
                v[0] += (double)zr * (double)rv;
              if (w != (T)0) v[1] += (double)rv * (double)rv;
              q[u] = zr;
              col_put(br, k, rv);
            }
          }
          tm_st<CW>(t_res + c * CW, br);
        }
        // boundary points to the neighbours: (Z res, s) for their next direction
#pragma unroll
        for (int u = 0; u < P; u++)
          if (u < nrow) {
            stage_one(spub, pw, ph, lx, ly0 + u, q[u]);
            stage_one(spub + 2 * (pw + ph), pw, ph, lx, ly0 + u, s[u]);
          }
        if (TRACE && tr) tr[5] = globaltimer_ns();
        workers_sync();
        copy_out_tagged(Pm, spub, ilo, ihi, jlo, jhi, wt, res_tag(Pm, 2u * hready));
        if (TRACE && tr) tr[6] = globaltimer_ns();
        if (!stop_after) {
          worker_partials<2, -1>(v, wred);
          __syncthreads();  // S1
          if (TRACE && tr) tr[7] = globaltimer_ns();
        }
        // sol += alpha*s (solve_streamfct.f90:278), while the other blocks finish
#pragma unroll
        for (int c = 0; c < NC; c++) {
          uint32_t bx[CW];
          tm_ld<CW>(t_sol + c * CW, bx);
          tm_wait_ld();
#pragma unroll
          for (int k = 0; k < CH; k++) {
            const int u = c * CH + k;
            if (u < nrow) col_put(bx, k, colT_get<T>(bx, k) + alpha * s[u]);
          }
          tm_st<CW>(t_sol + c * CW, bx);
        }
        tm_wait_st();
        if (TRACE && tr) tr[8] = globaltimer_ns();
        if (stop_after) goto done;
      }
      // the halo of the next direction, while the controller completes reduction B
      if (!__syncthreads_and(worker_halo_load_tagged(Pm, hl, res_tag(Pm, 2u * hready++)))) goto out;  // S2
      if (TRACE && tr) tr[9] = globaltimer_ns();
      if (C.act != kRun) goto done;
    }

  done:
    // the residual and solution of the last iterate back to global memory
#pragma unroll
    for (int c = 0; c < NC; c++) {
      uint32_t br[CW], bx[CW];
      tm_ld<CW>(t_res + c * CW, br);
      tm_ld<CW>(t_sol + c * CW, bx);
      tm_wait_ld();
#pragma unroll
      for (int k = 0; k < CH; k++) {
        const int u = c * CH + k;
        if (u < nrow) {
          const int j = jlo + ly0 + u;
          store_cyclic(res_resv<T>(Pm), g, i, j, colT_get<T>(br, k));
          res_solv<T>(Pm)[g.at(i, j)] = colT_get<T>(bx, k);
        }
      }
    }
  }
out:
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
}

// Block layout: warp 0 is the controller, warps 1-15 the workers (res_solve).
template <int P, bool TRACE>
__global__ void __launch_bounds__(kResThreads, 1) cg_res_kernel(const __grid_constant__ CGResParams Pm) {
  extern __shared__ __align__(16) double sm[];
  __shared__ uint32_t s_tmem;
  __shared__ ResCtl C;
  __shared__ double wred[kResThreads / 32][kResSlotWords];
  if ((threadIdx.x >> 5) == 0) {
    tc::tmem_alloc(&s_tmem, 512);
    tc::tmem_relinquish();
  }
  res_solve<double, P, TRACE>(Pm, (int)blockIdx.x, sm, &s_tmem, C, wred);
  if ((threadIdx.x >> 5) == 0) tc::tmem_dealloc(s_tmem, 512);
}

// The same solve with FP32 fields (shared memory, TMEM, registers, exchange
// records) and FP64 partial sums and control: the correction solve of the
// mixed-precision path, on grids twice the size of the FP64 kernel's.
template <int P>
__global__ void __launch_bounds__(kResThreads, 1) cg_res32_kernel(const __grid_constant__ CGResParams Pm) {
  extern __shared__ __align__(16) double sm[];
  __shared__ uint32_t s_tmem;
  __shared__ ResCtl C;
  __shared__ double wred[kResThreads / 32][kResSlotWords];
  if ((threadIdx.x >> 5) == 0) {
    tc::tmem_alloc(&s_tmem, 512);
    tc::tmem_relinquish();
  }
  res_solve<float, P, false>(Pm, (int)blockIdx.x, sm, &s_tmem, C, wred);
  if ((threadIdx.x >> 5) == 0) tc::tmem_dealloc(s_tmem, 512);
}

// Many solves in one launch (ResMultiParams): block b runs list entries
// list_off[b] .. list_off[b+1]-1, each a piece of one job; before a job the
// block counts itself in at the job's join counter and waits (bounded) until
// the whole gang is there, so the solve's own waits start with every piece
// present.  A job has its own operator, vectors, slots, records, error flag
// and result, so different jobs never wait on one another.
template <int P, bool WGT>
__global__ void __launch_bounds__(kResThreads, 1) cg_res_multi_kernel(const __grid_constant__ ResMultiParams M) {
  extern __shared__ __align__(16) double sm[];
  __shared__ uint32_t s_tmem;
  __shared__ ResCtl C;
  __shared__ double wred[kResThreads / 32][kResSlotWords];
  __shared__ int s_ok;
  // the current job's parameters in shared memory: read there in the hot loop
  // (through a reference into global memory every global store would force
  // them to be reloaded, and the solve ran ~24 % slower per iteration)
  __shared__ CGResParams s_job;
  static_assert(sizeof(CGResParams) % 8 == 0, "copied as 8-byte words");
  if ((threadIdx.x >> 5) == 0) {
    tc::tmem_alloc(&s_tmem, 512);
    tc::tmem_relinquish();
  }
  for (int e = M.list_off[blockIdx.x]; e < M.list_off[blockIdx.x + 1]; e++) {
    const int2 ent = M.list[e];
    {
      const unsigned long long* src = reinterpret_cast<const unsigned long long*>(M.jobs + ent.x);
      unsigned long long* dst = reinterpret_cast<unsigned long long*>(&s_job);
      for (int w = threadIdx.x; w < (int)(sizeof(CGResParams) / 8); w += kResThreads) dst[w] = src[w];
    }
    __syncthreads();
    const CGResParams& Pm = s_job;
    if (threadIdx.x == 0) {
      const int nb = Pm.npx * Pm.npy;
      atomicAdd(M.join + ent.x, 1);
      int ok = 1;
      const unsigned long long t0 = globaltimer_ns();
      for (unsigned spin = 1; ld_relaxed_i32(M.join + ent.x) < nb; spin++)
        if ((spin & 63u) == 0u && (ld_relaxed_i32(M.error) != 0 || globaltimer_ns() - t0 > M.gang_timeout_ns)) {
          atomicExch(M.error, PYOMGPU_TIMEOUT);
          ok = 0;
          break;
        }
      s_ok = ok;
    }
    __syncthreads();
    const bool ok = s_ok != 0;
    __syncthreads();
    if (!ok) break;
    if (ent.y == 0 && threadIdx.x == 0) M.times[2 * ent.x] = globaltimer_ns();
    res_solve<double, P, false, WGT, true>(Pm, ent.y, sm, &s_tmem, C, wred);
    if (ent.y == 0 && threadIdx.x == 0) M.times[2 * ent.x + 1] = globaltimer_ns();
  }
  tc::fence_before_sync();
  __syncthreads();
  if ((threadIdx.x >> 5) == 0) tc::tmem_dealloc(s_tmem, 512);
}

template __global__ void cg_res_kernel<4, false>(const __grid_constant__ CGResParams);
template __global__ void cg_res_kernel<8, false>(const __grid_constant__ CGResParams);
template __global__ void cg_res_kernel<16, false>(const __grid_constant__ CGResParams);
template __global__ void cg_res_kernel<4, true>(const __grid_constant__ CGResParams);
template __global__ void cg_res_kernel<8, true>(const __grid_constant__ CGResParams);
template __global__ void cg_res_kernel<16, true>(const __grid_constant__ CGResParams);
template __global__ void cg_res_multi_kernel<16, false>(const __grid_constant__ ResMultiParams);
template __global__ void cg_res_multi_kernel<16, true>(const __grid_constant__ ResMultiParams);
template __global__ void cg_res32_kernel<16>(const __grid_constant__ CGResParams);
template __global__ void cg_res32_kernel<32>(const __grid_constant__ CGResParams);

// Single-reduction variant (one cross-block reduction per iteration) of the
// same Jacobi-PCG, in the style of Chronopoulos and Gear but with the exact
// expansion of (p, Ap) (ctl1_direction).  With u = Z res and w = A u, the
// sweep of iteration n does
//   p = u + bq p,  s = w + bq s  (= A p),  res -= alpha s,  u = Z res,
//   then w = A u (stencil),  sol += alpha p,
// and one reduction returns (u, res), (u, w), (u, s), (p, w), (p, s),
// |res|^2 over the unknowns and max|p|.  The reference's (p, Ap) and its
// convergence test of iteration n (which needs max|p| of that iteration) are
// evaluated at that reduction, so every stop leaves sol and res where the
// reference's control flow leaves them; in exact arithmetic the iterates are
// the reference's, in floating point they differ at rounding level (A p by
// recurrence, (p, Ap) by expansion).  Per point the block keeps res, sol, Z and w in TMEM (all 128
// columns of a thread) and p, s in registers; the exchange records carry
// (res, w, s) of the boundary points, from which the neighbour's next u on
// the halo is recomputed with its owner's operations (records double-buffered,
// as each sweep has only one reduction between a write and the next).
template <int P>
__global__ void __launch_bounds__(kResThreads, 1) cg_res1_kernel(const __grid_constant__ CGResParams Pm) {
  constexpr int CH = 4;       // points per TMEM chunk (tcgen05 .x8)
  constexpr int NC = P / CH;  // chunks per field
  constexpr int CW = 2 * CH;  // TMEM columns per chunk
  static_assert(P % CH == 0 && NC * CW <= 32, "a field takes at most 32 TMEM columns per thread");
  extern __shared__ __align__(16) double sm[];
  __shared__ uint32_t s_tmem;
  __shared__ ResCtl C;
  __shared__ double wred[kResThreads / 32][kResSlotWords];
  const Geo g = Pm.g;
  const OpDev<double> op = Pm.op;
  const int warp = threadIdx.x >> 5;
  if (warp == 0) {
    tc::tmem_alloc(&s_tmem, 512);
    tc::tmem_relinquish();
  }

  const int nb = gridDim.x;
  const int px = blockIdx.x % Pm.npx, py = blockIdx.x / Pm.npx;
  const int ilo = 1 + (int)(((long long)px * g.nx) / Pm.npx);
  const int ihi = (int)(((long long)(px + 1) * g.nx) / Pm.npx);
  const int jlo = 1 + (int)(((long long)py * g.ny) / Pm.npy);
  const int jhi = (int)(((long long)(py + 1) * g.ny) / Pm.npy);
  const int pw = ihi - ilo + 1, ph = jhi - jlo + 1, sp = pw + 2;
  const int pw_ = pw, ph_ = ph;
  double* ss = sm;                    // (pw+2) x (ph+2): u = Z res, halo included
  double* sfx = ss + sp * (ph + 2);   // (pw+1) x ph: FX(ilo+lx, j), lx = 0..pw
  double* sfy = sfx + (pw + 1) * ph;  // pw x (ph+1): FY(i, jlo+ly), ly = 0..ph
  double* sbx = sfy + pw * (ph + 1);  // ph: bx(jlo+ly), then ph: by(jlo+ly)
  double* spub = sbx + 2 * ph;        // 3 x 2(pw+ph): staged boundary res, w, s
  const int nent = 2 * (pw + ph);
  double* shalo = reinterpret_cast<double*>(  // 2(pw+ph) x 4: received exchange records, 16-byte aligned
      (reinterpret_cast<uintptr_t>(spub + 3 * nent) + 15) & ~(uintptr_t)15);

  for (int e = threadIdx.x; e < sp * (ph + 2); e += kResThreads) ss[e] = 0.0;
  for (int e = threadIdx.x; e < (pw + 1) * ph; e += kResThreads)
    sfx[e] = op.FX[g.at(ilo + e % (pw + 1), jlo + e / (pw + 1))];
  for (int e = threadIdx.x; e < pw * (ph + 1); e += kResThreads) sfy[e] = op.FY[g.at(ilo + e % pw, jlo + e / pw)];
  for (int e = threadIdx.x; e < ph; e += kResThreads) {
    sbx[e] = op.bx[jlo + e + 1];
    sbx[ph + e] = op.by[jlo + e + 1];
  }
  for (int e = threadIdx.x; e < 3 * nent; e += kResThreads) spub[e] = 0.0;
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();

  if (warp == 0) {
    // ============================================================ controller
    unsigned ep = 0;
    __syncthreads();  // S1: init partials
    bool ok = controller_epoch<4, 3, kStepInit>(Pm, ep, (int)blockIdx.x, nb + (Pm.stall_extra ? 1 : 0), C, wred);
    if (!__syncthreads_and(ok)) goto out;  // S2
    if (C.act == kRun) {
      __syncthreads();  // S1: delta of the first direction
      ok = controller_epoch<2, -1, kStepInitD>(Pm, ++ep, (int)blockIdx.x, nb, C, wred);
      if (!__syncthreads_and(ok)) goto out;  // S2
      while (C.act == kRun) {
        __syncthreads();  // S1: partials of one sweep
        ok = controller_epoch<7, 6, kStepIter>(Pm, ++ep, (int)blockIdx.x, nb, C, wred);
        if (!__syncthreads_and(ok)) goto out;  // S2
      }
      if (C.act == kNeedMaxp) {
        __syncthreads();  // S1: max|p| of the new direction
        ok = controller_epoch<2, 0, kStepMaxp>(Pm, ++ep, (int)blockIdx.x, nb, C, wred);
        if (!__syncthreads_and(ok)) goto out;  // S2
      }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      const int converged = C.act == kDoneOk;
      Pm.out->iterations = C.n;
      Pm.out->converged = converged;
      Pm.out->status = converged ? PYOMGPU_OK : (C.est != C.est ? PYOMGPU_NAN : C.status);
      Pm.out->est = C.est;
    }
  } else {
    // =============================================================== workers
    const int wt = (int)threadIdx.x - 32;
    const int lx_ = wt % Pm.wmax;
    const int ly0_ = (wt / Pm.wmax) * P;
    const int nrow_ = (lx_ < pw && ly0_ < ph) ? min(P, ph - ly0_) : 0;
    const int i_ = ilo + lx_;
    int lx = lx_, ly0 = ly0_, nrow = nrow_;
    const int i = i_;
    const double axi = nrow_ > 0 ? op.ax[i_ + 1] : 0.0;
    const uint32_t tm = s_tmem + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)(128 * (warp >> 2));
    const uint32_t t_res = tm, t_sol = tm + 32, t_z = tm + 64, t_w = tm + 96;

    // halo positions received (record wt + e*kResWorkers of shalo), with Z of the source point
    struct {
      int sidx, gidx;
      double z;
    } hl[2];
    {
      const int nW = (ilo > 1 || g.cyclic_x) ? ph : 0, nE = (ihi < g.nx || g.cyclic_x) ? ph : 0;
      const int nS = (jlo > 1 || g.cyclic_y) ? pw : 0, nN = (jhi < g.ny || g.cyclic_y) ? pw : 0;
#pragma unroll
      for (int e = 0; e < 2; e++) {
        const int h = wt + e * kResWorkers;
        hl[e].sidx = -1;
        hl[e].gidx = 0;
        hl[e].z = 0.0;
        if (h >= nW + nE + nS + nN) continue;
        int hx, hy;
        if (h < nW) {
          hx = -1;
          hy = h;
        } else if (h < nW + nE) {
          hx = pw;
          hy = h - nW;
        } else if (h < nW + nE + nS) {
          hx = h - nW - nE;
          hy = -1;
        } else {
          hx = h - nW - nE - nS;
          hy = ph;
        }
        hl[e].sidx = (hy + 1) * sp + hx + 1;
        hl[e].gidx = (int)g.at(ilo + hx, jlo + hy);
        int si = ilo + hx, sj = jlo + hy;  // the interior point the halo position copies
        if (si < 1) si += g.nx;
        if (si > g.nx) si -= g.nx;
        if (sj < 1) sj += g.ny;
        if (sj > g.ny) sj -= g.ny;
        hl[e].z = op.W[g.at(si, sj)];
      }
    }

    double p[P], s[P];  // direction and A p
    // Exchange records alternate between two buffers by reduction parity: a
    // record written before reduction e is rewritten only before e+2, which
    // needs every reader's slot of e+1, published after its loads returned.
    unsigned wep = 0;  // reduction the next copy-out precedes
    auto xbuf = [&](unsigned e) { return Pm.hx + (size_t)(e & 1u) * 4 * (size_t)Pm.hsize; };

    // w = A u on this thread's points (u = Z res in ss, halo included) into
    // TMEM and the boundary staging; adds the partials (w, u) and (p, w)
    auto stencil = [&](double& delta, double& pw_dot) {
      const int lx = opaque(lx_), ly0 = opaque(ly0_), nrow = opaque(nrow_);
      const int pw = opaque(pw_), ph = opaque(ph_), sp = pw + 2;
      double fys = 0.0, uc = 0.0, us = 0.0;
      if (nrow > 0) {
        fys = sfy[ly0 * pw + lx];
        uc = ss[(ly0 + 1) * sp + lx + 1];
        us = ss[ly0 * sp + lx + 1];
      }
#pragma unroll
      for (int c = 0; c < NC; c++) {
        uint32_t bw[CW];
#pragma unroll
        for (int k = 0; k < CH; k++) {
          const int u = c * CH + k;
          double a = 0.0;
          if (u < nrow) {
            const int ly = ly0 + u;
            const int kk = (ly + 1) * sp + lx + 1;
            const double ue = ss[kk + 1], uw = ss[kk - 1], un = ss[kk + sp];
            const double fxw = sfx[ly * (pw + 1) + lx], fxe = sfx[ly * (pw + 1) + lx + 1];
            const double fyn = sfy[(ly + 1) * pw + lx];
            a = axi * sbx[ly] * (fxe * (ue - uc) + fxw * (uw - uc)) +
                sbx[ph + ly] * (fyn * (un - uc) + fys * (us - uc));
            delta += a * uc;
            pw_dot += p[u] * a;
            stage_one(spub + 2 * (pw + ph), pw, ph, lx, ly, a);
            fys = fyn;
            us = uc;
            uc = un;
          }
          col_put(bw, k, a);
        }
        tm_st<CW>(t_w + c * CW, bw);
      }
      tm_wait_st();
    };

    // ---------------------------------------------------------------- init
    // res = forc - A sol, solve_streamfct.f90:196-201; u = Z res
    {
      double v[4] = {0.0, 0.0, 0.0, 0.0};  // (Z res, res), bb, rr, max|Z res|
#pragma unroll
      for (int c = 0; c < NC; c++) {
        uint32_t br[CW], bz[CW], bx[CW];
#pragma unroll
        for (int k = 0; k < CH; k++) {
          const int u = c * CH + k;
          double rv = 0.0, w = 0.0, x = 0.0;
          p[u] = 0.0;
          s[u] = 0.0;
          if (u < nrow) {
            const int ly = ly0 + u, j = jlo + ly;
            const double f = Pm.forc[fidx(g.nx, i, j)];
            rv = f - apply_point(op, g, Pm.sol, i, j);
            w = op.W[g.at(i, j)];
            x = Pm.sol[g.at(i, j)];
            const double zr = w * rv;
            v[0] += zr * rv;
            if (w != 0.0) {
              v[1] += f * f;
              v[2] += rv * rv;
            }
            v[3] = fmax(v[3], fabs(zr));
            ss[(ly + 1) * sp + lx + 1] = zr;
            stage_one(spub, pw, ph, lx, ly, rv);
          }
          col_put(br, k, rv);
          col_put(bz, k, w);
          col_put(bx, k, x);
        }
        tm_st<CW>(t_res + c * CW, br);
        tm_st<CW>(t_z + c * CW, bz);
        tm_st<CW>(t_sol + c * CW, bx);
      }
      tm_wait_st();
      worker_partials<4, 3>(v, wred);
    }
    workers_sync();
    copy_out<3>(Pm, xbuf(wep), spub, ilo, ihi, jlo, jhi, wt);
    __syncthreads();                       // S1
    if (!__syncthreads_and(1)) goto out;  // S2
    if (C.act != kRun) goto done;
    // u on the halo (Z res of the neighbours), then w = A u and delta of the first direction
#pragma unroll
    for (int e = 0; e < 2; e++)
      if (hl[e].sidx >= 0) ss[hl[e].sidx] = hl[e].z * __ldcg(xbuf(wep) + 4 * (long long)hl[e].gidx);
    ++wep;
    workers_sync();
    {
      double v[2] = {0.0, 0.0};
      double unused = 0.0;
      stencil(v[0], unused);
      worker_partials<2, -1>(v, wred);
    }
    workers_sync();
    copy_out<3>(Pm, xbuf(wep), spub, ilo, ihi, jlo, jhi, wt);
    __syncthreads();                       // S1
    if (!__syncthreads_and(1)) goto out;  // S2

    for (;;) {
      if (C.act == kNeedMaxp) {
        // the breakdown estimate needs max|p| of the direction that was to be used
        double v[2] = {0.0, 0.0};
        const double bq = C.bq;
        nrow = opaque(nrow_);
#pragma unroll
        for (int c = 0; c < NC; c++) {
          uint32_t br[CW], bz[CW];
          tm_ld<CW>(t_res + c * CW, br);
          tm_ld<CW>(t_z + c * CW, bz);
          tm_wait_ld();
#pragma unroll
          for (int k = 0; k < CH; k++) {
            const int u = c * CH + k;
            if (u < nrow) v[0] = fmax(v[0], fabs(col_get(bz, k) * col_get(br, k) + bq * p[u]));
          }
        }
        worker_partials<2, 0>(v, wred);
        __syncthreads();                       // S1
        if (!__syncthreads_and(1)) goto out;  // S2
        goto done;
      }
      if (C.act != kRun) goto done;
      // ------------------------------------------------- update and u = Z res
      lx = opaque(lx_);
      ly0 = opaque(ly0_);
      nrow = opaque(nrow_);
      const double alpha = C.alpha, bq = C.bq;
      // the neighbours' (res, w, s) records land in shared memory during the update
#pragma unroll
      for (int e = 0; e < 2; e++)
        if (hl[e].sidx >= 0) {
          const double* src = xbuf(wep) + 4 * (long long)hl[e].gidx;
          double* dst = shalo + 4 * (wt + e * kResWorkers);
          cp_async16(dst, src);
          cp_async16(dst + 2, src + 2);
        }
      // (u, res), (u, w), (u, s), (p, w), (p, s), rr, max|p| of the new u, w and this sweep's p, s
      double v[7] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
      {
        const int pw = opaque(pw_), ph = opaque(ph_), sp = pw + 2;
#pragma unroll
        for (int c = 0; c < NC; c++) {
          {
            uint32_t bw[CW];
            tm_ld<CW>(t_w + c * CW, bw);
            tm_wait_ld();
#pragma unroll
            for (int k = 0; k < CH; k++) s[c * CH + k] = col_get(bw, k) + bq * s[c * CH + k];
          }
          uint32_t br[CW], bz[CW];
          tm_ld<CW>(t_res + c * CW, br);
          tm_ld<CW>(t_z + c * CW, bz);
          tm_wait_ld();
#pragma unroll
          for (int k = 0; k < CH; k++) {
            const int u = c * CH + k;
            if (u < nrow) {
              const int ly = ly0 + u;
              const double z = col_get(bz, k);
              const double uo = z * col_get(br, k);
              p[u] = uo + bq * p[u];
              const double rv = col_get(br, k) - alpha * s[u];
              const double un = z * rv;
              ss[(ly + 1) * sp + lx + 1] = un;
              v[0] += un * rv;
              v[2] += un * s[u];
              v[4] += p[u] * s[u];
              if (z != 0.0) v[5] += rv * rv;
              v[6] = fmax(v[6], fabs(p[u]));
              col_put(br, k, rv);
              stage_one(spub, pw, ph, lx, ly, rv);
              stage_one(spub + 4 * (pw + ph), pw, ph, lx, ly, s[u]);
            }
          }
          tm_st<CW>(t_res + c * CW, br);
        }
      }
      cp_async_wait();
#pragma unroll
      for (int e = 0; e < 2; e++)
        if (hl[e].sidx >= 0) {
          const double* rec = shalo + 4 * (wt + e * kResWorkers);
          const double sh = rec[1] + bq * rec[2];
          ss[hl[e].sidx] = hl[e].z * (rec[0] - alpha * sh);
        }
      workers_sync();
      stencil(v[1], v[3]);
      worker_partials<7, 6>(v, wred);
      workers_sync();
      ++wep;
      copy_out<3>(Pm, xbuf(wep), spub, ilo, ihi, jlo, jhi, wt);
      __syncthreads();  // S1
      // sol += alpha p (solve_streamfct.f90:278), while the other blocks finish
#pragma unroll
      for (int c = 0; c < NC; c++) {
        uint32_t bx[CW];
        tm_ld<CW>(t_sol + c * CW, bx);
        tm_wait_ld();
#pragma unroll
        for (int k = 0; k < CH; k++) {
          const int u = c * CH + k;
          if (u < nrow) col_put(bx, k, col_get(bx, k) + alpha * p[u]);
        }
        tm_st<CW>(t_sol + c * CW, bx);
      }
      tm_wait_st();
      if (!__syncthreads_and(1)) goto out;  // S2
    }

  done:
    // the residual and solution of the last iterate back to global memory
    nrow = opaque(nrow_);
    ly0 = opaque(ly0_);
#pragma unroll
    for (int c = 0; c < NC; c++) {
      uint32_t br[CW], bx[CW];
      tm_ld<CW>(t_res + c * CW, br);
      tm_ld<CW>(t_sol + c * CW, bx);
      tm_wait_ld();
#pragma unroll
      for (int k = 0; k < CH; k++) {
        const int u = c * CH + k;
        if (u < nrow) {
          const int j = jlo + ly0 + u;
          store_cyclic(Pm.res, g, i, j, col_get(br, k));
          Pm.sol[g.at(i, j)] = col_get(bx, k);
        }
      }
    }
  }
out:
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(s_tmem, 512);
}

template __global__ void cg_res1_kernel<4>(const __grid_constant__ CGResParams);
template __global__ void cg_res1_kernel<8>(const __grid_constant__ CGResParams);
template __global__ void cg_res1_kernel<16>(const __grid_constant__ CGResParams);

const void* cg_res_multi_kernel_ptr(bool weighted) {
  return weighted ? (const void*)cg_res_multi_kernel<16, true> : (const void*)cg_res_multi_kernel<16, false>;
}
const void* cg_res32_kernel_ptr(int p) {
  return p == 16 ? (const void*)cg_res32_kernel<16> : p == 32 ? (const void*)cg_res32_kernel<32> : nullptr;
}

const void* cg_res_kernel_ptr(int p, bool single) {
  switch (p) {
    case 4: return single ? (const void*)cg_res1_kernel<4> : (const void*)cg_res_kernel<4, false>;
    case 8: return single ? (const void*)cg_res1_kernel<8> : (const void*)cg_res_kernel<8, false>;
    case 16: return single ? (const void*)cg_res1_kernel<16> : (const void*)cg_res_kernel<16, false>;
    default: return nullptr;
  }
}

const void* cg_res_trace_kernel_ptr(int p) {
  switch (p) {
    case 4: return (const void*)cg_res_kernel<4, true>;
    case 8: return (const void*)cg_res_kernel<8, true>;
    case 16: return (const void*)cg_res_kernel<16, true>;
    default: return nullptr;
  }
}

}  // namespace pyomgpu
