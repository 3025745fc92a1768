// Host island set-up (islands.cpp).
#pragma once
#include <cmath>
#include <vector>

namespace pyomgpu {

// Fixed sizes of the reference: mnisle, maxipp (streamfct_init.f90:16),
// maxq (island_module.f90:22).  Large grids need them raised.
struct IslandLimits {
  int mnisle = 1000;
  int maxipp = 20000;
  int maxq = 10000;
};

// failure codes of the island set-up (reference halt_stop sites)
constexpr int kIslMaxipp = -1;       // island_module.f90:256-258
constexpr int kIslQueue = -2;        // island_module.f90:310
constexpr int kIslMnisle = -3;       // island_module.f90:86-90
constexpr int kIslMissing = -5;      // streamfct_init.f90:72-82
constexpr int kIslNoStart = -6;      // streamfct_init.f90:159-163
constexpr int kIslLostTrack = -7;    // streamfct_init.f90:216-225
constexpr int kIslMaxBoundary = -8;  // streamfct_init.f90:249-253
constexpr int kIslRange = -9;        // map read outside the halo grid

struct IslandSet {
  int nisle = 0;
  int max_boundary = 0;
  std::vector<int> boundary;     // (nisle, max_boundary, 2) Fortran order
  std::vector<int> line_dir;     // (nisle, max_boundary, 2)
  std::vector<int> nr_boundary;  // (nisle)
};

int isleperim(const int* kmt, int imt, int jmt, bool cyclic, const IslandLimits& lim, int* map, int* nisle,
              std::vector<int>* nippts);
int island_map(int nx, int ny, bool cyclic_x, const int* kbot, const IslandLimits& lim, std::vector<int>& allmap,
               int* nisle, int* max_boundary);
int island_trace(int nx, int ny, bool cyclic_x, const std::vector<int>& allmap, int nisle, int max_boundary,
                 const IslandLimits& lim, IslandSet& out);
int lu_factor(int n, std::vector<double>& a, std::vector<int>& ipiv);

// The same labelling and tracing on the GPU (islands_gpu.cu), kbot (nx+4,
// ny+4) a device array; bit-identical results, no flood-fill queue (maxq
// unused).  Codes below -99 are CUDA failures.  stream is a cudaStream_t.
int island_boundaries_gpu(int nx, int ny, bool cyclic_x, const int* kbot_dev, const IslandLimits& lim,
                          IslandSet& out, std::vector<int>* allmap_out, void* stream);

}  // namespace pyomgpu
