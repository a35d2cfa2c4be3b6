// hfg_sort.cu -- reordering the particles by cell (no reference counterpart:
// the reference keeps its particles in seeding order for the whole run,
// EulerParticles.cpp:140-179).
//
// Particles seeded cell by cell start out ordered, so the lanes of a warp
// touch neighbouring corner-table entries in the substeps and neighbouring
// faces in the P2G scatter, where lane groups with equal corners merge their
// atomics.  A mixing flow spreads that order out.  This is a stable counting
// sort by the particle's cell (the binning of transPos2Index,
// EulerMathTool.cu:29-40), deterministic although its scatter uses atomics:
//   keys      key[p] = cell of particle p; count[cell] += 1
//   scan      exclusive prefix sums of the counts, in place (3 passes)
//   scatter   slot = atomicAdd(&off[key], 1); perm[slot] = p
//             (off[c] then holds the end of bucket c)
//   buckets   each cell's bucket sorted by original index: the order within a
//             cell is the previous order, whatever the atomics' order was
//   gather    out[j] = in[perm[j]] for each particle array
#include <algorithm>

#include "hfg_kernels.h"

namespace hfg {

namespace {

constexpr int kSortThreads = 256;
constexpr int kScanThreads = 1024;
constexpr int kScanPerThread = 4;
constexpr int kScanTile = kScanThreads * kScanPerThread;

inline int sortGrid(long long n, int threads = kSortThreads, int perSM = 16) {
  long long b = (n + threads - 1) / threads;
  long long cap = (long long)numSMs() * perSM;
  return (int)std::max(1LL, std::min(b, cap));
}

__global__ void kSortKeys(Geom g, const float* __restrict__ pos, long long P, unsigned int* __restrict__ key,
                          unsigned int* __restrict__ count) {
  for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < P; p += (long long)gridDim.x * blockDim.x) {
    unsigned int c = (unsigned int)binCell(g, pos[3 * p], pos[3 * p + 1], pos[3 * p + 2]);
    key[p] = c;
    atomicAdd(count + c, 1u);
  }
}

// Exclusive scan of a block-sized tile in place; the tile's total goes to
// sums[blockIdx.x].
__global__ void __launch_bounds__(kScanThreads) kScanTiles(unsigned int* __restrict__ a, long long n,
                                                           unsigned int* __restrict__ sums) {
  __shared__ unsigned int warpTot[kScanThreads / 32];
  const long long base = (long long)blockIdx.x * kScanTile + (long long)threadIdx.x * kScanPerThread;
  unsigned int v[kScanPerThread];
  unsigned int t = 0;
#pragma unroll
  for (int k = 0; k < kScanPerThread; ++k) {
    v[k] = base + k < n ? a[base + k] : 0u;
    t += v[k];
  }
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  unsigned int inc = t;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    unsigned int y = __shfl_up_sync(0xffffffffu, inc, d);
    if (lane >= d) inc += y;
  }
  if (lane == 31) warpTot[w] = inc;
  __syncthreads();
  if (w == 0) {
    unsigned int x = warpTot[lane];
    unsigned int xi = x;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      unsigned int y = __shfl_up_sync(0xffffffffu, xi, d);
      if (lane >= d) xi += y;
    }
    warpTot[lane] = xi - x;
    if (lane == 31) sums[blockIdx.x] = xi;
  }
  __syncthreads();
  unsigned int run = warpTot[w] + inc - t;
#pragma unroll
  for (int k = 0; k < kScanPerThread; ++k) {
    if (base + k < n) a[base + k] = run;
    run += v[k];
  }
}

// Exclusive scan of the tile totals by one block, chunk after chunk.
__global__ void __launch_bounds__(kScanThreads) kScanSums(unsigned int* __restrict__ sums, int nb) {
  __shared__ unsigned int warpTot[kScanThreads / 32];
  __shared__ unsigned int carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int c0 = 0; c0 < nb; c0 += kScanThreads) {
    int i = c0 + threadIdx.x;
    unsigned int x = i < nb ? sums[i] : 0u;
    unsigned int inc = x;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      unsigned int y = __shfl_up_sync(0xffffffffu, inc, d);
      if (lane >= d) inc += y;
    }
    if (lane == 31) warpTot[w] = inc;
    __syncthreads();
    if (w == 0) {
      unsigned int s = warpTot[lane], si = s;
#pragma unroll
      for (int d = 1; d < 32; d <<= 1) {
        unsigned int y = __shfl_up_sync(0xffffffffu, si, d);
        if (lane >= d) si += y;
      }
      warpTot[lane] = si - s;
    }
    __syncthreads();
    unsigned int base = carry;
    if (i < nb) sums[i] = base + warpTot[w] + inc - x;
    __syncthreads();
    if (threadIdx.x == kScanThreads - 1) carry = base + warpTot[w] + inc;
    __syncthreads();
  }
}

__global__ void kScanAdd(unsigned int* __restrict__ a, long long n, const unsigned int* __restrict__ sums) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    a[i] += sums[i / kScanTile];
}

__global__ void kSortScatter(const unsigned int* __restrict__ key, long long P, unsigned int* __restrict__ off,
                             unsigned int* __restrict__ perm) {
  for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < P; p += (long long)gridDim.x * blockDim.x)
    perm[atomicAdd(off + key[p], 1u)] = (unsigned int)p;
}

// Heap sort of a[0, n) ascending, in place: O(n log n) for the rare large
// bucket (particles crowded into one cell).
__device__ void heapSort(unsigned int* a, unsigned int n) {
  auto sift = [&](unsigned int i, unsigned int m) {
    unsigned int v = a[i];
    for (;;) {
      unsigned int ch = 2 * i + 1;
      if (ch >= m) break;
      if (ch + 1 < m && a[ch + 1] > a[ch]) ++ch;
      if (a[ch] <= v) break;
      a[i] = a[ch];
      i = ch;
    }
    a[i] = v;
  };
  for (unsigned int i = n / 2; i-- > 0;) sift(i, n);
  for (unsigned int m = n; m-- > 1;) {
    unsigned int t = a[0];
    a[0] = a[m];
    a[m] = t;
    sift(0, m);
  }
}

// After the scatter off[c] is the end of bucket c and off[c - 1] its start.
// Buckets hold a handful of particles (8 per fluid cell when seeded): an
// insertion sort per cell, or a heap sort for a bucket beyond 32.
__global__ void kSortBuckets(const unsigned int* __restrict__ off, long long n, unsigned int* __restrict__ perm) {
  for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
    unsigned int b = c ? off[c - 1] : 0u, e = off[c];
    if (e - b > 32) {
      heapSort(perm + b, e - b);
      continue;
    }
    for (unsigned int i = b + 1; i < e; ++i) {
      unsigned int v = perm[i];
      unsigned int j = i;
      while (j > b && perm[j - 1] > v) {
        perm[j] = perm[j - 1];
        --j;
      }
      perm[j] = v;
    }
  }
}

template <int W>
__global__ void kGather(const float* __restrict__ in, const unsigned int* __restrict__ perm, long long P,
                        float* __restrict__ out) {
  for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x; j < P; j += (long long)gridDim.x * blockDim.x) {
    const long long s = perm[j];
#pragma unroll
    for (int k = 0; k < W; ++k) out[W * j + k] = __ldg(in + W * s + k);
  }
}

}  // namespace

long long sortScanBlocks(long long nCells) { return (nCells + kScanTile - 1) / kScanTile; }

cudaError_t launchSortPermutation(const Geom& g, const float* pos, long long P, unsigned int* key, unsigned int* off,
                                  unsigned int* sums, unsigned int* perm, cudaStream_t s) {
  const long long n = g.r.size();
  if (n >= (1LL << 32) || P >= (1LL << 32)) return cudaErrorInvalidValue;
  cudaError_t e = cudaMemsetAsync(off, 0, sizeof(unsigned int) * n, s);
  if (e != cudaSuccess) return e;
  if (P > 0) kSortKeys<<<sortGrid(P), kSortThreads, 0, s>>>(g, pos, P, key, off);
  const long long nb = sortScanBlocks(n);
  kScanTiles<<<(unsigned)nb, kScanThreads, 0, s>>>(off, n, sums);
  kScanSums<<<1, kScanThreads, 0, s>>>(sums, (int)nb);
  kScanAdd<<<sortGrid(n), kSortThreads, 0, s>>>(off, n, sums);
  if (P > 0) {
    kSortScatter<<<sortGrid(P), kSortThreads, 0, s>>>(key, P, off, perm);
    kSortBuckets<<<sortGrid(n), kSortThreads, 0, s>>>(off, n, perm);
  }
  return cudaGetLastError();
}

cudaError_t launchGather(const float* in, int width, const unsigned int* perm, long long P, float* out,
                         cudaStream_t s) {
  if (P <= 0) return cudaSuccess;
  switch (width) {
    case 1: kGather<1><<<sortGrid(P), kSortThreads, 0, s>>>(in, perm, P, out); break;
    case 3: kGather<3><<<sortGrid(P), kSortThreads, 0, s>>>(in, perm, P, out); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

}  // namespace hfg
