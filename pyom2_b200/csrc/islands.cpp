// Island labelling and perimeter tracing (host C++), run once per grid.
//
// Labelling restates the MOM flood fill of island_module.f90:7-419 (isleperim,
// expand, the bounded queue, and the cyclic neighbour rules) so that the land
// masses get the same numbers as in pyOM2: scan from the northern row down,
// west to east, 8-connected land, perimeter = ocean cells 8-adjacent to the
// mass.  Tracing restates streamfct_init.f90:95-267 (start point search, the
// right-hand walk along psi points, cyclic wrap).  The reference aborts on
// every failure; here each failure is a status code.
#include "islands.h"

#include <algorithm>
#include <cstring>
#include <vector>

namespace pyomgpu {

namespace {

constexpr int kOffmap = -1;

struct Queue {
  // Fixed-capacity FIFO that compacts to the front when the back reaches the
  // capacity (island_module.f90:291-317); overflow with a full queue is an error.
  std::vector<int> qi, qj;
  int front = 1, back = 0, cap;
  bool fault = false;
  explicit Queue(int capacity) : qi((size_t)capacity + 2), qj((size_t)capacity + 2), cap(capacity) {}
  void reset() {
    front = 1;
    back = 0;
  }
  bool empty() const { return front > back; }
  void push(int i, int j) {
    if (++back > cap) {
      if (front == 1) {
        fault = true;
        back = cap;
        return;
      }
      const int shift = front - 1;
      for (int p = front; p <= back - 1; ++p) {
        qi[p - shift] = qi[p];
        qj[p - shift] = qj[p];
      }
      front = 1;
      back -= shift;
    }
    qi[back] = i;
    qj[back] = j;
  }
  void pop(int& i, int& j) {
    i = qi[front];
    j = qj[front];
    ++front;
  }
};

struct Labeller {
  int imt, jmt;
  bool cyclic;
  int maxipp;
  int* map;  // (imt, jmt), 1-based access via at()
  std::vector<int> nippts, iofs;
  int& at(int i, int j) { return map[(size_t)(i - 1) + (size_t)(j - 1) * imt]; }
  int north(int j) const { return j < jmt ? j + 1 : kOffmap; }
  int south(int j) const { return j > 1 ? j - 1 : kOffmap; }
  int east(int i) const {
    if (cyclic) return i < imt - 1 ? i + 1 : i + 3 - imt;
    return i < imt ? i + 1 : kOffmap;
  }
  int west(int i) const {
    if (cyclic) return i > 2 ? i - 1 : i + imt - 3;
    return i > 1 ? i - 1 : kOffmap;
  }

  // Flood fill of one land mass from the queued seed (island_module.f90:134-273).
  int fill(int label, Queue& q) {
    long perimeter_total = 0;
    while (!q.empty()) {
      if (q.fault) return kIslQueue;
      int i, j;
      q.pop(i, j);
      if (i == kOffmap || j == kOffmap) continue;
      int& m = at(i, j);
      if (m == label || m == -label) continue;
      if (m == 1) {  // unassigned land: claim it and queue the 8 neighbours
        m = label;
        const int n = north(j), s = south(j), e = east(i), w = west(i);
        q.push(i, n);
        q.push(e, n);
        q.push(e, j);
        q.push(e, s);
        q.push(i, s);
        q.push(w, s);
        q.push(w, j);
        q.push(w, n);
        continue;
      }
      if (m == 0) {  // ocean next to this mass: perimeter point
        m = -label;
        nippts[label] += 1;
        if (iofs[label] + nippts[label] > maxipp) return kIslMaxipp;
        continue;
      }
      // m < 0: perimeter of an earlier mass (a "collision"); m > 1: another
      // mass's land.  Both are left untouched, as in the reference.
      (void)perimeter_total;
    }
    if (q.fault) return kIslQueue;
    q.reset();
    return 0;
  }
};

}  // namespace

int isleperim(const int* kmt, int imt, int jmt, bool cyclic, const IslandLimits& lim, int* map, int* nisle,
              std::vector<int>* nippts_out) {
  Labeller L;
  L.imt = imt;
  L.jmt = jmt;
  L.cyclic = cyclic;
  L.maxipp = lim.maxipp;
  L.map = map;
  L.nippts.assign((size_t)lim.mnisle + 2, 0);
  L.iofs.assign((size_t)lim.mnisle + 2, 0);
  for (int j = 1; j <= jmt; ++j)
    for (int i = 1; i <= imt; ++i) L.at(i, j) = kmt[(size_t)(i - 1) + (size_t)(j - 1) * imt] > 0 ? 0 : 1;
  Queue q(lim.maxq);
  int label = 2;
  const int iwest = cyclic ? 2 : 1, ieast = cyclic ? imt - 1 : imt;
  for (int j = jmt; j >= 1; --j)
    for (int i = iwest; i <= ieast; ++i) {
      if (L.at(i, j) != 1) continue;
      q.push(i, j);
      const int rc = L.fill(label, q);
      if (rc) return rc;
      ++label;
      if (label > lim.mnisle) return kIslMnisle;
      L.iofs[label] = L.iofs[label - 1] + L.nippts[label - 1];
      L.nippts[label] = 0;
    }
  // masses were numbered from 2; shift labels (and perimeter marks) down by one
  for (int i = iwest; i <= ieast; ++i)
    for (int j = 1; j <= jmt; ++j) {
      int& m = L.at(i, j);
      if (m > 0)
        m -= 1;
      else if (m < 0)
        m += 1;
    }
  const int n = label - 2;
  if (cyclic)
    for (int j = 1; j <= jmt; ++j) {
      L.at(1, j) = L.at(imt - 1, j);
      L.at(imt, j) = L.at(2, j);
    }
  *nisle = n;
  if (nippts_out) {
    nippts_out->assign((size_t)n, 0);
    for (int k = 1; k <= n; ++k) (*nippts_out)[k - 1] = L.nippts[k + 1];
  }
  return 0;
}

// Position helpers on the halo-extended grid: Fortran (i,j) with i in
// [-1, nx+2], j in [-1, ny+2]  <->  isleperim's 1-based (imt, jmt) indices.
namespace {
struct HaloGrid {
  int nx, ny;
  int X() const { return nx + 4; }
  size_t idx(int i, int j) const { return (size_t)(i + 1) + (size_t)(j + 1) * X(); }
  bool inside(int i, int j) const { return i >= -1 && i <= nx + 2 && j >= -1 && j <= ny + 2; }
};
}  // namespace

int island_map(int nx, int ny, bool cyclic_x, const int* kbot, const IslandLimits& lim, std::vector<int>& allmap,
               int* nisle, int* max_boundary) {
  HaloGrid H{nx, ny};
  const size_t n2 = (size_t)H.X() * (ny + 4);
  std::vector<int> kmt(n2, 0);
  // streamfct_init.f90:35-48: ocean columns become 5, the rest 0, cyclic copy
  for (int j = 1; j <= ny; ++j)
    for (int i = 1; i <= nx; ++i)
      if (kbot[H.idx(i, j)] > 0) kmt[H.idx(i, j)] = 5;
  if (cyclic_x)
    for (int j = -1; j <= ny + 2; ++j)
      for (int i = 1; i <= 2; ++i) {
        kmt[H.idx(nx + i, j)] = kmt[H.idx(i, j)];
        kmt[H.idx(1 - i, j)] = kmt[H.idx(nx - i + 1, j)];
      }
  allmap.assign(n2, 0);
  std::vector<int> nippts;
  int rc = isleperim(kmt.data(), H.X(), ny + 4, cyclic_x, lim, allmap.data(), nisle, &nippts);
  if (rc) return rc;
  if (cyclic_x)
    for (int j = -1; j <= ny + 2; ++j)
      for (int i = 1; i <= 2; ++i) {
        allmap[H.idx(nx + i, j)] = allmap[H.idx(i, j)];
        allmap[H.idx(1 - i, j)] = allmap[H.idx(nx - i + 1, j)];
      }
  // paranoia check (streamfct_init.f90:64-83)
  std::vector<char> seen((size_t)*nisle + 1, 0);
  for (int v : allmap)
    if (v >= 1 && v <= *nisle) seen[v] = 1;
  for (int k = 1; k <= *nisle; ++k)
    if (!seen[k]) return kIslMissing;
  int mx = 0;
  for (int v : nippts) mx = std::max(mx, v);
  *max_boundary = 20 * mx;
  return 0;
}

int island_trace(int nx, int ny, bool cyclic_x, const std::vector<int>& allmap, int nisle, int max_boundary,
                 const IslandLimits& lim, IslandSet& out) {
  HaloGrid H{nx, ny};
  const size_t n2 = (size_t)H.X() * (ny + 4);
  out.nisle = nisle;
  out.max_boundary = max_boundary;
  out.boundary.assign((size_t)nisle * max_boundary * 2, 0);
  out.line_dir.assign((size_t)nisle * max_boundary * 2, 0);
  out.nr_boundary.assign((size_t)nisle, 0);
  std::vector<int> kmt(n2), map(n2);
  auto B = [&](std::vector<int>& a, int isle, int n, int c) -> int& {
    return a[(size_t)(isle - 1) + (size_t)(n - 1) * nisle + (size_t)(c - 1) * nisle * max_boundary];
  };
  for (int isle = 1; isle <= nisle; ++isle) {
    // land map of this island alone: 1 land, -1 perimeter, 0 elsewhere (:106-108)
    for (size_t q = 0; q < n2; ++q) kmt[q] = allmap[q] == isle ? 0 : 1;
    int dummy = 0;
    int rc = isleperim(kmt.data(), H.X(), ny + 4, cyclic_x, lim, map.data(), &dummy, nullptr);
    if (rc) return rc;
    auto M = [&](int i, int j) -> int { return map[H.idx(i, j)]; };
    // start point: a horizontal coastline segment, searched from the middle
    // eastwards, then westwards (:116-165)
    int ij[2] = {0, 0}, dir[2] = {0, 0};
    bool found = false;
    auto probe = [&](int i) {
      for (int j = 0; j <= ny && !found; ++j) {
        if (M(i, j) == 1 && M(i, j + 1) == -1) {
          ij[0] = i;
          ij[1] = j;
          dir[0] = 1;
          dir[1] = 0;
          B(out.boundary, isle, 1, 1) = i - 1;
          B(out.boundary, isle, 1, 2) = j;
          found = true;
        } else if (M(i, j) == -1 && M(i, j + 1) == 1) {
          ij[0] = i - 1;
          ij[1] = j;
          dir[0] = -1;
          dir[1] = 0;
          B(out.boundary, isle, 1, 1) = i;
          B(out.boundary, isle, 1, 2) = j;
          found = true;
        }
      }
    };
    for (int i = nx / 2 + 1; i <= nx && !found; ++i) probe(i);
    for (int i = nx / 2; i >= 1 && !found; --i) probe(i);
    if (!found) return kIslNoStart;
    B(out.line_dir, isle, 1, 1) = dir[0];
    B(out.line_dir, isle, 1, 2) = dir[1];
    int n = 2;
    if (n > max_boundary) return kIslMaxBoundary;
    B(out.boundary, isle, n, 1) = ij[0];
    B(out.boundary, isle, n, 2) = ij[1];
    const int s0 = B(out.boundary, isle, 1, 1), s1 = B(out.boundary, isle, 1, 2);
    bool cont = true;
    while (cont) {
      // cells ahead-left (ijp) and ahead-right (ijr) of the walking direction (:184-191)
      int pi, pj, ri, rj;
      if (dir[0] == 0 && dir[1] == 1) {
        pi = ij[0]; pj = ij[1] + 1; ri = ij[0] + 1; rj = ij[1] + 1;
      } else if (dir[0] == -1 && dir[1] == 0) {
        pi = ij[0]; pj = ij[1]; ri = ij[0]; rj = ij[1] + 1;
      } else if (dir[0] == 0 && dir[1] == -1) {
        pi = ij[0] + 1; pj = ij[1]; ri = ij[0]; rj = ij[1];
      } else {
        pi = ij[0] + 1; pj = ij[1] + 1; ri = ij[0] + 1; rj = ij[1];
      }
      if (!H.inside(pi, pj) || !H.inside(ri, rj)) return kIslRange;
      const int a = M(pi, pj), b = M(ri, rj);
      if (a == -1 && b == 1) {
        // straight on
      } else if (a == -1 && b == -1) {  // turn right
        const int d0 = dir[1], d1 = -dir[0];
        dir[0] = d0;
        dir[1] = d1;
      } else if (a == 1 && (b == 1 || b == -1)) {  // turn left
        const int d0 = -dir[1], d1 = dir[0];
        dir[0] = d0;
        dir[1] = d1;
      } else {
        return kIslLostTrack;
      }
      B(out.line_dir, isle, n, 1) = dir[0];
      B(out.line_dir, isle, n, 2) = dir[1];
      ij[0] += dir[0];
      ij[1] += dir[1];
      if (ij[0] == s0 && ij[1] == s1) cont = false;
      if (cyclic_x && dir[0] == 1 && dir[1] == 0 && ij[0] > nx) ij[0] -= nx;
      if (cyclic_x && dir[0] == -1 && dir[1] == 0 && ij[0] < 1) ij[0] += nx;
      if (ij[0] == s0 && ij[1] == s1) cont = false;
      if (cont) {
        if (++n > max_boundary) return kIslMaxBoundary;
        B(out.boundary, isle, n, 1) = ij[0];
        B(out.boundary, isle, n, 2) = ij[1];
      }
    }
    out.nr_boundary[isle - 1] = n;
  }
  return 0;
}

// Dense LU with partial pivoting, LAPACK DGETF2 semantics (pivot = first
// largest |a| in the column, rows swapped in full, column scaled by the
// reciprocal pivot).  a is column-major n x n.  Returns info.
int lu_factor(int n, std::vector<double>& a, std::vector<int>& ipiv) {
  ipiv.assign((size_t)n, 0);
  int info = 0;
  auto A = [&](int i, int j) -> double& { return a[(size_t)i + (size_t)j * n]; };
  for (int k = 0; k < n; ++k) {
    int p = k;
    double mx = std::abs(A(k, k));
    for (int i = k + 1; i < n; ++i)
      if (std::abs(A(i, k)) > mx) {
        mx = std::abs(A(i, k));
        p = i;
      }
    ipiv[k] = p + 1;
    if (A(p, k) != 0.0) {
      if (p != k)
        for (int j = 0; j < n; ++j) std::swap(A(k, j), A(p, j));
      if (std::abs(A(k, k)) >= 2.2250738585072014e-308) {
        const double r = 1.0 / A(k, k);
        for (int i = k + 1; i < n; ++i) A(i, k) *= r;
      } else {
        for (int i = k + 1; i < n; ++i) A(i, k) /= A(k, k);
      }
    } else if (info == 0) {
      info = k + 1;
    }
    for (int j = k + 1; j < n; ++j) {
      const double t = A(k, j);
      if (t != 0.0)
        for (int i = k + 1; i < n; ++i) A(i, j) -= A(i, k) * t;
    }
  }
  return info;
}

}  // namespace pyomgpu
