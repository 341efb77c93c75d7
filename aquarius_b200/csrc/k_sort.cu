// Stable LSD radix sort of (u32 key, i32 value) pairs, 8 key bits per pass:
// the headless frame's (tile, primitive) lists and its longest-list-first
// tile order.  Each pass is three steps over tiles of 1024 pairs (256
// threads x 4 rounds): a per-tile digit histogram (shared-memory counts),
// an exclusive scan of the histograms in digit-major order (digit d of tile
// 0, 1, ... then digit d + 1: the same three-kernel scan as the particle
// sort), and a scatter in which every pair goes to its digit's base plus its
// rank among the tile's earlier pairs of that digit (warp ranks from
// match.any, per-warp counts summed in warp order).  A pair's destination is
// thus a function of the keys alone, so the output is deterministic and every
// pass keeps the order of equal digits: stable.
#include <algorithm>
#include <cstdint>

#include "aq_kernels.cuh"

namespace aqb {
namespace {

constexpr int kSortThreads = 256;
constexpr int kSortRounds = 4;
constexpr int kSortTile = kSortThreads * kSortRounds;
constexpr int kSortWarps = kSortThreads / 32;

__device__ __forceinline__ unsigned sort_digit(unsigned k, int shift, bool desc) {
  return ((desc ? ~k : k) >> shift) & 255u;
}

// hist[d * ntiles + tile] = pairs of the tile whose digit is d.
__global__ void __launch_bounds__(kSortThreads) k_sort_hist(const unsigned* __restrict__ keys, int n, int shift,
                                                           bool desc, int ntiles, int* __restrict__ hist) {
  __shared__ int h[256];
  const int tid = threadIdx.x;
  h[tid] = 0;
  __syncthreads();
#pragma unroll
  for (int r = 0; r < kSortRounds; ++r) {
    const int i = blockIdx.x * kSortTile + r * kSortThreads + tid;
    if (i < n) atomicAdd(&h[sort_digit(keys[i], shift, desc)], 1);
  }
  __syncthreads();
  hist[tid * ntiles + blockIdx.x] = h[tid];
}

// Pair i of the tile goes to off[d * ntiles + tile] + (pairs of digit d
// before it in the tile), d its digit.
__global__ void __launch_bounds__(kSortThreads) k_sort_scatter(const unsigned* __restrict__ kin,
                                                              const int* __restrict__ vin, unsigned* __restrict__ kout,
                                                              int* __restrict__ vout, int n, int shift, bool desc,
                                                              int ntiles, const int* __restrict__ off) {
  __shared__ int base[256];                // next destination of each digit
  __shared__ int wpos[kSortWarps][256];    // per round: pairs per warp and digit, then each warp's first slot
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  base[tid] = off[tid * ntiles + blockIdx.x];
#pragma unroll
  for (int w = 0; w < kSortWarps; ++w) wpos[w][tid] = 0;
  __syncthreads();
  for (int r = 0; r < kSortRounds; ++r) {
    const int i = blockIdx.x * kSortTile + r * kSortThreads + tid;
    const bool valid = i < n;
    const unsigned k = valid ? kin[i] : 0u;
    const int v = valid ? vin[i] : 0;
    const unsigned d = valid ? sort_digit(k, shift, desc) : 256u;  // 256: no digit
    const unsigned peers = __match_any_sync(0xffffffffu, d);
    const int rank = __popc(peers & ((1u << lane) - 1u));
    if (valid && rank == 0) wpos[warp][d] = __popc(peers);
    __syncthreads();
    int run = base[tid];
#pragma unroll
    for (int w = 0; w < kSortWarps; ++w) {
      const int c = wpos[w][tid];
      wpos[w][tid] = run;
      run += c;
    }
    base[tid] = run;
    __syncthreads();
    if (valid) {
      const int dst = wpos[warp][d] + rank;
      kout[dst] = k;
      vout[dst] = v;
    }
    __syncthreads();
#pragma unroll
    for (int w = 0; w < kSortWarps; ++w) wpos[w][tid] = 0;
    __syncthreads();
  }
}

int sort_tiles(int n) { return std::max(1, (n + kSortTile - 1) / kSortTile); }

}  // namespace

size_t radix_sort_temp_ints(int n) {
  const int nt = sort_tiles(n);
  const int C = 256 * nt - 1;
  return 2 * (size_t)std::max(n, 1) + 2 * (size_t)(256 * nt) + cell_scan_tiles(C) + 4;
}

cudaError_t radix_sort_pairs(cudaStream_t st, const unsigned* k0, const int* v0, unsigned* k1, int* v1, int n,
                             int bits, bool descending, int* tmp) {
  if (n <= 0) return cudaSuccess;
  const int nt = sort_tiles(n);
  const int C = 256 * nt - 1;  // the scan covers C + 1 = 256 * nt counts
  unsigned* kt = reinterpret_cast<unsigned*>(tmp);
  int* vt = tmp + std::max(n, 1);
  int* hist = vt + std::max(n, 1);
  int* hoff = hist + 256 * nt;
  int* tsum = hoff + 256 * nt;
  const int passes = std::max(1, (bits + 7) / 8);
  // the last pass writes (k1, v1): the passes alternate between (kt, vt) and
  // (k1, v1), the first reads (k0, v0)
  const unsigned* ks = k0;
  const int* vs = v0;
  for (int p = 0; p < passes; ++p) {
    const bool to_out = ((passes - 1 - p) % 2) == 0;
    unsigned* kd = to_out ? k1 : kt;
    int* vd = to_out ? v1 : vt;
    k_sort_hist<<<nt, kSortThreads, 0, st>>>(ks, n, 8 * p, descending, nt, hist);
    cudaError_t e = launch_cell_scan(st, C, hist, hoff, tsum);
    if (e != cudaSuccess) return e;
    k_sort_scatter<<<nt, kSortThreads, 0, st>>>(ks, vs, kd, vd, n, 8 * p, descending, nt, hoff);
    ks = kd;
    vs = vd;
  }
  return cudaGetLastError();
}

}  // namespace aqb
