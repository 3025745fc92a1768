// Island labelling and perimeter tracing on the GPU: the results of
// isleperim (island_module.f90:7-419) and of streamfct_init.f90:35-267, bit
// for bit those of the host restatement (islands.cpp), computed without the
// serial flood fill.
//
// Labelling.  isleperim scans the halo grid from the northern row down, west
// to east, and floods each unlabelled land mass (8-connected, cyclic in x
// through its east/west rules) with the next label; every ocean cell
// 8-adjacent to the mass gets minus that label unless an earlier mass already
// marked it.  So the masses are the 8-connected components of the land,
// numbered by the scan position of their first cell, and a perimeter cell
// carries minus the smallest label among its land neighbours.  Here:
//   1. union-find over the scanned cells (each cell starts under its
//      smallest-key land neighbour; lock-free compare-and-swap hooking of the
//      larger root under the smaller with the four forward neighbours;
//      pointer jumping in every find), every root the smallest scan key of
//      its component;
//   2. the roots, ranked in key order by a block scan, are the labels;
//   3. land cells take their root's label, ocean cells minus the smallest
//      label among their land neighbours (and are counted per label).
// Tracing.  streamfct_init re-runs isleperim on each island alone (its land
// only) and walks the coast of that map's first mass.  The per-island maps
// need no flood fill either: a second union-find joins neighbouring cells of
// equal island number, an island's first mass is the component of its
// smallest scan key, and the map value at a cell (1 own first mass, -1 next
// to it, else 0 or another mass) is evaluated where it is read.  The start
// points of all islands are searched at once (the first hit in the
// reference's search order per island), then one thread walks each island.
//
// Differences from the reference, both only in failure cases: there is no
// flood-fill queue, so its capacity limit maxq never applies; the perimeter
// limit maxipp is checked on the total after labelling.
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "islands.h"

namespace pyomgpu {

namespace {

constexpr int kIGThreads = 256;
constexpr int kUnionCap = 1 << 22;  // retries of one union before it reports failure

// The isleperim grid: imt = nx + 4 columns, jmt = ny + 4 rows, 1-based; the
// scanned columns are iwest..ieast and key(i,j) = (jmt - j) * W + (i - iwest)
// is the position in the scan order.
struct IGrid {
  int nx, ny, imt, jmt, iwest, ieast, W, cyclic;
  __host__ __device__ int key(int i, int j) const { return (jmt - j) * W + (i - iwest); }
  __host__ __device__ void cell(int k, int& i, int& j) const {
    j = jmt - k / W;
    i = iwest + k % W;
  }
  __host__ __device__ size_t at(int i, int j) const { return (size_t)(i - 1) + (size_t)(j - 1) * imt; }
  // island_module.f90:373-419; 0 = off the map
  __host__ __device__ int north(int j) const { return j < jmt ? j + 1 : 0; }
  __host__ __device__ int south(int j) const { return j > 1 ? j - 1 : 0; }
  __host__ __device__ int east(int i) const {
    if (cyclic) return i < imt - 1 ? i + 1 : i + 3 - imt;
    return i < imt ? i + 1 : 0;
  }
  __host__ __device__ int west(int i) const {
    if (cyclic) return i > 2 ? i - 1 : i + imt - 3;
    return i > 1 ? i - 1 : 0;
  }
  __host__ __device__ int K() const { return W * jmt; }
};

__device__ __forceinline__ int vload(const int* p) { return *(const volatile int*)p; }

// Root of x with intermediate pointer jumping: every visited node is pointed
// past its parent.  Parents only ever move to smaller keys of the same
// component, so concurrent jumps keep the forest valid.
__device__ __forceinline__ int find_root(int* parent, int x) {
  int curr = vload(parent + x);
  if (curr != x) {
    int prev = x, next;
    while (curr > (next = vload(parent + curr))) {
      parent[prev] = next;
      prev = curr;
      curr = next;
    }
  }
  return curr;
}

// Join the components of a and b: the larger root is hooked under the
// smaller one by compare-and-swap, retried from the value found when another
// thread got there first.  Each failed swap moves to a smaller key, so the
// retries are finite; the cap turns a pathological case into an error.
__device__ __forceinline__ bool unite(int* parent, int a, int b) {
  a = find_root(parent, a);
  b = find_root(parent, b);
  for (int it = 0; it < kUnionCap; ++it) {
    if (a == b) return true;
    if (a < b) {
      const int old = atomicCAS(parent + b, b, a);
      if (old == b) return true;
      b = old;
    } else {
      const int old = atomicCAS(parent + a, a, b);
      if (old == a) return true;
      a = old;
    }
  }
  return false;
}

// land of the labelling pass: kmt == 0 (streamfct_init.f90:35-48: ocean
// columns are 5, with the cyclic halo copies)
__device__ __forceinline__ bool is_land(const IGrid& G, const int* kbot, int i, int j) {
  // isleperim (i,j) -> Fortran (i-2, j-2); the halo columns of a cyclic grid copy the interior
  int fi = i - 2;
  const int fj = j - 2;
  if (G.cyclic) {
    if (fi > G.nx) fi -= G.nx;
    if (fi < 1) fi += G.nx;
  }
  if (fi < 1 || fi > G.nx || fj < 1 || fj > G.ny) return true;
  return kbot[(size_t)(fi + 1) + (size_t)(fj + 1) * (G.nx + 4)] <= 0;
}

// parent = the smallest key among the cell and its 8-adjacent land cells
// (shallow initial trees), -1 for ocean
__global__ void k_init_land(IGrid G, const int* kbot, int* parent) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= G.K()) return;
  int i, j;
  G.cell(k, i, j);
  if (!is_land(G, kbot, i, j)) {
    parent[k] = -1;
    return;
  }
  const int e = G.east(i), w = G.west(i), n = G.north(j), s = G.south(j);
  const int ni[8] = {i, e, e, e, i, w, w, w}, nj[8] = {n, n, j, s, s, s, j, n};
  int m = k;
  for (int q = 0; q < 8; ++q) {
    if (ni[q] == 0 || nj[q] == 0) continue;
    if (is_land(G, kbot, ni[q], nj[q])) m = min(m, G.key(ni[q], nj[q]));
  }
  parent[k] = m;
}

// union with the four forward neighbours (east, north-east, north, north-west):
// every 8-adjacent pair once
__global__ void k_union(IGrid G, int* parent, int* err) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= G.K() || parent[k] < 0) return;
  int i, j;
  G.cell(k, i, j);
  const int e = G.east(i), w = G.west(i), n = G.north(j);
  const int ni[4] = {e, e, i, w}, nj[4] = {j, n, n, n};
  for (int q = 0; q < 4; ++q) {
    if (ni[q] == 0 || nj[q] == 0) continue;
    const int kn = G.key(ni[q], nj[q]);
    if (parent[kn] < 0) continue;
    if (!unite(parent, k, kn)) atomicExch(err, 1);
  }
}

// union of 8-adjacent cells that carry the same island number (the per-island maps)
__global__ void k_init_isle(IGrid G, const int* allmap, int* parent, int* first_key) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= G.K()) return;
  int i, j;
  G.cell(k, i, j);
  const int v = allmap[G.at(i, j)];
  if (v <= 0) {
    parent[k] = -1;
    return;
  }
  atomicMin(first_key + v, k);
  const int e = G.east(i), w = G.west(i), n = G.north(j), s = G.south(j);
  const int ni[8] = {i, e, e, e, i, w, w, w}, nj[8] = {n, n, j, s, s, s, j, n};
  int m = k;
  for (int q = 0; q < 8; ++q) {
    if (ni[q] == 0 || nj[q] == 0) continue;
    if (allmap[G.at(ni[q], nj[q])] == v) m = min(m, G.key(ni[q], nj[q]));
  }
  parent[k] = m;
}

__global__ void k_union_isle(IGrid G, const int* allmap, int* parent, int* err) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= G.K() || parent[k] < 0) return;
  int i, j;
  G.cell(k, i, j);
  const int v = allmap[G.at(i, j)];
  const int e = G.east(i), w = G.west(i), n = G.north(j);
  const int ni[4] = {e, e, i, w}, nj[4] = {j, n, n, n};
  for (int q = 0; q < 4; ++q) {
    if (ni[q] == 0 || nj[q] == 0) continue;
    if (allmap[G.at(ni[q], nj[q])] != v) continue;
    if (!unite(parent, k, G.key(ni[q], nj[q]))) atomicExch(err, 1);
  }
}

__global__ void k_flatten(IGrid G, int* parent) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= G.K() || parent[k] < 0) return;
  parent[k] = find_root(parent, k);
}

// ---- ranks of the roots in key order: per-block counts, one-block scan of the
// counts, per-block exclusive scan
__global__ void k_root_count(IGrid G, const int* parent, int* block_count) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int r = (k < G.K() && parent[k] == k) ? 1 : 0;
  const int c = __syncthreads_count(r);
  if (threadIdx.x == 0) block_count[blockIdx.x] = c;
}

__global__ void k_scan_blocks(int* block_count, int nblocks, int* total) {
  // one block of kIGThreads threads, each scanning a contiguous run
  __shared__ int part[kIGThreads];
  const int per = (nblocks + kIGThreads - 1) / kIGThreads;
  const int b0 = threadIdx.x * per, b1 = min(nblocks, b0 + per);
  int sum = 0;
  for (int b = b0; b < b1; ++b) sum += block_count[b];
  part[threadIdx.x] = sum;
  __syncthreads();
  if (threadIdx.x == 0) {
    int run = 0;
    for (int t = 0; t < kIGThreads; ++t) {
      const int v = part[t];
      part[t] = run;
      run += v;
    }
    *total = run;
  }
  __syncthreads();
  int run = part[threadIdx.x];
  for (int b = b0; b < b1; ++b) {
    const int v = block_count[b];
    block_count[b] = run;
    run += v;
  }
}

__global__ void k_root_label(IGrid G, const int* parent, const int* block_offset, int* label) {
  __shared__ int warp_sum[kIGThreads / 32];
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int r = (k < G.K() && parent[k] == k) ? 1 : 0;
  const unsigned bal = __ballot_sync(0xffffffffu, r);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) warp_sum[w] = __popc(bal);
  __syncthreads();
  int before = 0;
  for (int q = 0; q < w; ++q) before += warp_sum[q];
  before += __popc(bal & ((1u << lane) - 1u));
  if (r) label[k] = block_offset[blockIdx.x] + before + 1;  // labels 1, 2, ... in scan order
}

// allmap over the scanned cells: land = its mass, ocean = minus the smallest
// adjacent mass (island_module.f90 "collisions" keep the first mass's mark)
__global__ void k_assign(IGrid G, const int* parent, const int* label, int* allmap, int* nippts) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= G.K()) return;
  int i, j;
  G.cell(k, i, j);
  if (parent[k] >= 0) {
    allmap[G.at(i, j)] = label[parent[k]];
    return;
  }
  const int e = G.east(i), w = G.west(i), n = G.north(j), s = G.south(j);
  const int ni[8] = {i, e, e, e, i, w, w, w}, nj[8] = {n, n, j, s, s, s, j, n};
  int best = 0x7fffffff;
  for (int q = 0; q < 8; ++q) {
    if (ni[q] == 0 || nj[q] == 0) continue;
    const int kn = G.key(ni[q], nj[q]);
    const int pr = parent[kn];
    if (pr >= 0) best = min(best, label[pr]);
  }
  if (best != 0x7fffffff) {
    allmap[G.at(i, j)] = -best;
    atomicAdd(nippts + best, 1);
  } else {
    allmap[G.at(i, j)] = 0;
  }
}

// halo columns of a cyclic grid: Fortran -1, 0 <- nx-1, nx and nx+1, nx+2 <- 1, 2
// (isleperim's own copy, island_module.f90:100-111, is overwritten by these,
// streamfct_init.f90:56-62)
__global__ void k_halo_copy(IGrid G, int* allmap) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x + 1;
  if (j > G.jmt) return;
  allmap[G.at(1, j)] = allmap[G.at(G.nx + 1, j)];
  allmap[G.at(2, j)] = allmap[G.at(G.nx + 2, j)];
  allmap[G.at(G.nx + 3, j)] = allmap[G.at(3, j)];
  allmap[G.at(G.nx + 4, j)] = allmap[G.at(4, j)];
}

// streamfct_init.f90:64-83: every label must still be in the map after the halo copies
__global__ void k_present(int n2, const int* allmap, int* present) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n2) return;
  const int v = allmap[q];
  if (v > 0) present[v] = 1;
}

// map value of island `isle`'s own isleperim call at isleperim (i,j), after its cyclic copy
__device__ int isle_map(const IGrid& G, const int* allmap, const int* parent, int root1, int isle, int i, int j) {
  if (G.cyclic) {
    if (i == 1) i = G.imt - 1;
    else if (i == G.imt) i = 2;
  }
  if (allmap[G.at(i, j)] == isle) {
    const int pr = parent[G.key(i, j)];
    return pr == root1 ? 1 : 2;  // 2: a further mass of this island's map
  }
  const int e = G.east(i), w = G.west(i), n = G.north(j), s = G.south(j);
  const int ni[8] = {i, e, e, e, i, w, w, w}, nj[8] = {n, n, j, s, s, s, j, n};
  for (int q = 0; q < 8; ++q) {
    if (ni[q] == 0 || nj[q] == 0) continue;
    if (allmap[G.at(ni[q], nj[q])] == isle && parent[G.key(ni[q], nj[q])] == root1) return -1;
  }
  return 0;
}

// Position of Fortran (i, j) in the start-point search order of
// streamfct_init.f90:116-165: columns nx/2+1 .. nx, then nx/2 .. 1; j = 0 .. ny.
__device__ __forceinline__ long long start_order(int nx, int ny, int i, int j) {
  const int h = nx / 2;
  const long long col = i >= h + 1 ? (long long)(i - (h + 1)) : (long long)(nx - h) + (h - i);
  return col * (ny + 1) + j;
}

// Start-point search of every island at once: (i, j) is a start of island v
// when v's map reads (1, -1) or (-1, 1) at (i, j), (i, j+1); each island keeps
// the first such point in the search order.
__global__ void k_start(IGrid G, const int* allmap, const int* parent, const int* first_key,
                        unsigned long long* start) {
  const int nx = G.nx, ny = G.ny;
  const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (e >= (long long)nx * (ny + 1)) return;
  const int i = 1 + (int)(e % nx), j = (int)(e / nx);
  const int c0 = allmap[G.at(i + 2, j + 2)], c1 = allmap[G.at(i + 2, j + 3)];
  for (int t = 0; t < 2; ++t) {
    const int v = t == 0 ? c0 : c1;
    if (v <= 0 || (t == 1 && v == c0)) continue;
    const int a = isle_map(G, allmap, parent, first_key[v], v, i + 2, j + 2);
    const int b = isle_map(G, allmap, parent, first_key[v], v, i + 2, j + 3);
    if ((a == 1 && b == -1) || (a == -1 && b == 1))
      atomicMin(start + v, (unsigned long long)start_order(nx, ny, i, j));
  }
}

// streamfct_init.f90:116-257: the coast walk, one thread per island, from the
// start point k_start found
__global__ void k_trace(IGrid G, const int* allmap, const int* parent, const int* first_key,
                        const unsigned long long* start, int nisle, int max_boundary, int* boundary, int* line_dir,
                        int* nr_boundary, int* status) {
  const int isle = blockIdx.x * blockDim.x + threadIdx.x + 1;
  if (isle > nisle) return;
  const int nx = G.nx, ny = G.ny;
  const int root1 = first_key[isle];
  auto M = [&](int fi, int fj) { return isle_map(G, allmap, parent, root1, isle, fi + 2, fj + 2); };
  auto B = [&](int* a, int n, int c) -> int& {
    return a[(size_t)(isle - 1) + (size_t)(n - 1) * nisle + (size_t)(c - 1) * nisle * max_boundary];
  };
  if (start[isle] == ~0ull) {
    status[isle - 1] = kIslNoStart;
    return;
  }
  int ij0 = 0, ij1 = 0, d0 = 0, d1 = 0;
  {
    const long long o = (long long)start[isle];
    const int h = nx / 2;
    const long long col = o / (ny + 1);
    const int j = (int)(o % (ny + 1));
    const int i = col < nx - h ? (int)(h + 1 + col) : (int)(h - (col - (nx - h)));
    if (M(i, j) == 1) {  // (1, -1): walk east
      ij0 = i;
      ij1 = j;
      d0 = 1;
      B(boundary, 1, 1) = i - 1;
      B(boundary, 1, 2) = j;
    } else {  // (-1, 1): walk west
      ij0 = i - 1;
      ij1 = j;
      d0 = -1;
      B(boundary, 1, 1) = i;
      B(boundary, 1, 2) = j;
    }
  }
  B(line_dir, 1, 1) = d0;
  B(line_dir, 1, 2) = d1;
  int n = 2;
  if (n > max_boundary) {
    status[isle - 1] = kIslMaxBoundary;
    return;
  }
  B(boundary, n, 1) = ij0;
  B(boundary, n, 2) = ij1;
  const int s0 = B(boundary, 1, 1), s1 = B(boundary, 1, 2);
  bool cont = true;
  while (cont) {  // ends at the start point, or after max_boundary points with an error
    int pi, pj, ri, rj;
    if (d0 == 0 && d1 == 1) {
      pi = ij0; pj = ij1 + 1; ri = ij0 + 1; rj = ij1 + 1;
    } else if (d0 == -1 && d1 == 0) {
      pi = ij0; pj = ij1; ri = ij0; rj = ij1 + 1;
    } else if (d0 == 0 && d1 == -1) {
      pi = ij0 + 1; pj = ij1; ri = ij0; rj = ij1;
    } else {
      pi = ij0 + 1; pj = ij1 + 1; ri = ij0 + 1; rj = ij1;
    }
    if (pi < -1 || pi > nx + 2 || pj < -1 || pj > ny + 2 || ri < -1 || ri > nx + 2 || rj < -1 || rj > ny + 2) {
      status[isle - 1] = kIslRange;
      return;
    }
    const int a = M(pi, pj), b = M(ri, rj);
    if (a == -1 && b == 1) {
    } else if (a == -1 && b == -1) {
      const int t0 = d1, t1 = -d0;
      d0 = t0;
      d1 = t1;
    } else if (a == 1 && (b == 1 || b == -1)) {
      const int t0 = -d1, t1 = d0;
      d0 = t0;
      d1 = t1;
    } else {
      status[isle - 1] = kIslLostTrack;
      return;
    }
    B(line_dir, n, 1) = d0;
    B(line_dir, n, 2) = d1;
    ij0 += d0;
    ij1 += d1;
    if (ij0 == s0 && ij1 == s1) cont = false;
    if (G.cyclic && d0 == 1 && d1 == 0 && ij0 > nx) ij0 -= nx;
    if (G.cyclic && d0 == -1 && d1 == 0 && ij0 < 1) ij0 += nx;
    if (ij0 == s0 && ij1 == s1) cont = false;
    if (cont) {
      if (++n > max_boundary) {
        status[isle - 1] = kIslMaxBoundary;
        return;
      }
      B(boundary, n, 1) = ij0;
      B(boundary, n, 2) = ij1;
    }
  }
  nr_boundary[isle - 1] = n;
  status[isle - 1] = 0;
}

int nblk(size_t n) { return (int)((n + kIGThreads - 1) / kIGThreads); }

struct DevBuf {
  std::vector<void*> owned;
  template <typename T>
  T* get(size_t n) {
    void* p = nullptr;
    if (cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T)) != cudaSuccess) return nullptr;
    owned.push_back(p);
    return (T*)p;
  }
  ~DevBuf() {
    for (void* p : owned) cudaFree(p);
  }
};

}  // namespace

int island_boundaries_gpu(int nx, int ny, bool cyclic_x, const int* kbot_dev, const IslandLimits& lim,
                          IslandSet& out, std::vector<int>* allmap_out, void* stream) {
  cudaStream_t st = (cudaStream_t)stream;
  IGrid G{};
  G.nx = nx;
  G.ny = ny;
  G.imt = nx + 4;
  G.jmt = ny + 4;
  G.cyclic = cyclic_x ? 1 : 0;
  G.iwest = cyclic_x ? 2 : 1;
  G.ieast = cyclic_x ? G.imt - 1 : G.imt;
  G.W = G.ieast - G.iwest + 1;
  const int K = G.K();
  const size_t n2 = (size_t)G.imt * G.jmt;
  const int nb = nblk((size_t)K);
  DevBuf D;
  int* parent = D.get<int>(K);
  int* label = D.get<int>(K);
  int* allmap = D.get<int>(n2);
  int* counts = D.get<int>(nb);
  int* scal = D.get<int>(4);  // total roots, union error
  if (!parent || !label || !allmap || !counts || !scal) return -100;
  if (cudaMemsetAsync(allmap, 0, n2 * sizeof(int), st) != cudaSuccess ||
      cudaMemsetAsync(scal, 0, 4 * sizeof(int), st) != cudaSuccess)
    return -101;
  k_init_land<<<nb, kIGThreads, 0, st>>>(G, kbot_dev, parent);
  k_union<<<nb, kIGThreads, 0, st>>>(G, parent, scal + 1);
  k_flatten<<<nb, kIGThreads, 0, st>>>(G, parent);
  k_root_count<<<nb, kIGThreads, 0, st>>>(G, parent, counts);
  k_scan_blocks<<<1, kIGThreads, 0, st>>>(counts, nb, scal);
  k_root_label<<<nb, kIGThreads, 0, st>>>(G, parent, counts, label);
  int h[2] = {0, 0};
  if (cudaMemcpyAsync(h, scal, 2 * sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return -102;
  if (h[1]) return -103;
  const int nisle = h[0];
  if (nisle + 2 > lim.mnisle) return kIslMnisle;  // island_module.f90:86-90
  int* nippts = D.get<int>((size_t)nisle + 2);
  if (!nippts) return -100;
  cudaMemsetAsync(nippts, 0, ((size_t)nisle + 2) * sizeof(int), st);
  k_assign<<<nb, kIGThreads, 0, st>>>(G, parent, label, allmap, nippts);
  if (cyclic_x) k_halo_copy<<<nblk(G.jmt), kIGThreads, 0, st>>>(G, allmap);
  int* present = D.get<int>((size_t)nisle + 2);
  if (!present) return -100;
  cudaMemsetAsync(present, 0, ((size_t)nisle + 2) * sizeof(int), st);
  k_present<<<nblk(n2), kIGThreads, 0, st>>>((int)n2, allmap, present);
  std::vector<int> hn((size_t)nisle + 2, 0), hp((size_t)nisle + 2, 0);
  if (cudaMemcpyAsync(hn.data(), nippts, hn.size() * sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaMemcpyAsync(hp.data(), present, hp.size() * sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return -102;
  long total = 0;
  int mx = 0;
  for (int k = 1; k <= nisle; ++k) {
    total += hn[k];
    mx = std::max(mx, hn[k]);
  }
  if (total > lim.maxipp) return kIslMaxipp;  // island_module.f90:256-258 (raised during the fill there)
  for (int k = 1; k <= nisle; ++k)
    if (!hp[k]) return kIslMissing;
  const int max_boundary = 20 * mx;           // streamfct_init.f90:87
  // per-island maps: components of equal island number, first mass = smallest key
  int* first_key = D.get<int>((size_t)nisle + 1);
  int* boundary = D.get<int>((size_t)std::max(1, nisle) * std::max(1, max_boundary) * 2);
  int* line_dir = D.get<int>((size_t)std::max(1, nisle) * std::max(1, max_boundary) * 2);
  int* nr = D.get<int>((size_t)std::max(1, nisle));
  int* status = D.get<int>((size_t)std::max(1, nisle));
  if (!first_key || !boundary || !line_dir || !nr || !status) return -100;
  cudaMemsetAsync(first_key, 0x7f, ((size_t)nisle + 1) * sizeof(int), st);
  cudaMemsetAsync(boundary, 0, (size_t)std::max(1, nisle) * std::max(1, max_boundary) * 2 * sizeof(int), st);
  cudaMemsetAsync(line_dir, 0, (size_t)std::max(1, nisle) * std::max(1, max_boundary) * 2 * sizeof(int), st);
  cudaMemsetAsync(nr, 0, (size_t)std::max(1, nisle) * sizeof(int), st);
  k_init_isle<<<nb, kIGThreads, 0, st>>>(G, allmap, parent, first_key);
  k_union_isle<<<nb, kIGThreads, 0, st>>>(G, allmap, parent, scal + 1);
  k_flatten<<<nb, kIGThreads, 0, st>>>(G, parent);
  unsigned long long* start = D.get<unsigned long long>((size_t)nisle + 1);
  if (!start) return -100;
  cudaMemsetAsync(start, 0xff, ((size_t)nisle + 1) * sizeof(unsigned long long), st);
  if (nisle > 0) {
    k_start<<<nblk((size_t)nx * (ny + 1)), kIGThreads, 0, st>>>(G, allmap, parent, first_key, start);
    k_trace<<<nblk(nisle), kIGThreads, 0, st>>>(G, allmap, parent, first_key, start, nisle, max_boundary, boundary,
                                                line_dir, nr, status);
  }
  out.nisle = nisle;
  out.max_boundary = max_boundary;
  out.boundary.assign((size_t)nisle * max_boundary * 2, 0);
  out.line_dir.assign((size_t)nisle * max_boundary * 2, 0);
  out.nr_boundary.assign((size_t)nisle, 0);
  std::vector<int> hs((size_t)std::max(1, nisle), 0);
  if (nisle > 0) {
    cudaMemcpyAsync(out.boundary.data(), boundary, out.boundary.size() * sizeof(int), cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(out.line_dir.data(), line_dir, out.line_dir.size() * sizeof(int), cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(out.nr_boundary.data(), nr, (size_t)nisle * sizeof(int), cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(hs.data(), status, (size_t)nisle * sizeof(int), cudaMemcpyDeviceToHost, st);
  }
  if (allmap_out) {
    allmap_out->assign(n2, 0);
    cudaMemcpyAsync(allmap_out->data(), allmap, n2 * sizeof(int), cudaMemcpyDeviceToHost, st);
  }
  cudaMemcpyAsync(h, scal, 2 * sizeof(int), cudaMemcpyDeviceToHost, st);
  if (cudaStreamSynchronize(st) != cudaSuccess || cudaGetLastError() != cudaSuccess) return -102;
  if (h[1]) return -103;
  for (int k = 0; k < nisle; ++k)
    if (hs[k]) return hs[k];
  return 0;
}

}  // namespace pyomgpu
