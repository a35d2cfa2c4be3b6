// hfg_sort.cu -- reordering the particles by cell (no reference counterpart:
// the reference keeps its particles in seeding order for the whole run,
// EulerParticles.cpp:140-179).
//
// Particles seeded cell by cell start out ordered, so the lanes of a warp
// touch neighbouring corner-table entries in the substeps and neighbouring
// faces in the P2G scatter, where lane groups with equal corners merge their
// atomics.  A mixing flow spreads that order out.  This is a stable LSD radix
// sort of the particles by cell (the binning of transPos2Index,
// EulerMathTool.cu:29-40), 8 bits per pass, deterministic:
//   keys      key[p] = cell of particle p, value p; with a split, one more
//             bit above the cell for the particles from the split on, so the
//             particles below it stay the first ones (the boundary fix of the
//             reference's launch reaches exactly those, EulerParticlesTool.cu:880)
//   per pass  hist     per tile of 4096 particles, the count of each digit
//             scan     exclusive prefix sums of the counts, digit-major, so a
//                      digit's slots go to the tiles in particle order
//             scatter  each tile walks its particles in order, 256 at a time;
//                      a particle's slot is its digit's running base plus the
//                      particles before it with that digit (__match_any_sync
//                      within a warp, per-warp counts across warps)
//   gather    out[j] = in[perm[j]] for each particle array
// The cost does not depend on how the particles are spread over the cells
// (a cell can hold thousands where the flow presses particles onto a wall).
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

// key = cell, with groupBit added for the particles from `split` on, so each
// group stays together in its own index range
__global__ void kSortKeys(Geom g, const float* __restrict__ pos, long long P, long long split, unsigned int groupBit,
                          unsigned int* __restrict__ key) {
  for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < P; p += (long long)gridDim.x * blockDim.x)
    key[p] = (unsigned int)binCell(g, pos[3 * p], pos[3 * p + 1], pos[3 * p + 2]) | (p >= split ? groupBit : 0u);
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

constexpr int kRadixBits = 8, kRadixDigits = 1 << kRadixBits;
constexpr int kRadixThreads = 256, kRadixRounds = 16, kRadixTile = kRadixThreads * kRadixRounds;
constexpr int kRadixWarps = kRadixThreads / 32;
static_assert(kRadixThreads == kRadixDigits, "one thread per digit");

// counts[d * tiles + t] = particles of tile t whose digit (at shift) is d
__global__ void __launch_bounds__(kRadixThreads) kRadixHist(const unsigned int* __restrict__ key, long long P,
                                                            int shift, unsigned int* __restrict__ counts,
                                                            long long tiles) {
  __shared__ unsigned int h[kRadixDigits];
  h[threadIdx.x] = 0;
  __syncthreads();
  const long long base = (long long)blockIdx.x * kRadixTile;
  for (int r = 0; r < kRadixRounds; ++r) {
    long long i = base + r * kRadixThreads + threadIdx.x;
    if (i < P) atomicAdd(&h[(key[i] >> shift) & (kRadixDigits - 1)], 1u);
  }
  __syncthreads();
  counts[(long long)threadIdx.x * tiles + blockIdx.x] = h[threadIdx.x];
}

// Stable scatter of one tile, given the scanned counts.  valIn == nullptr:
// the values are the particle indices.
__global__ void __launch_bounds__(kRadixThreads) kRadixScatter(const unsigned int* __restrict__ keyIn,
                                                               const unsigned int* __restrict__ valIn, long long P,
                                                               int shift, const unsigned int* __restrict__ scanned,
                                                               long long tiles, unsigned int* __restrict__ keyOut,
                                                               unsigned int* __restrict__ valOut) {
  __shared__ unsigned int base[kRadixDigits];
  __shared__ unsigned int wcnt[kRadixWarps][kRadixDigits];
  const int t = threadIdx.x, lane = t & 31, w = t >> 5;
  base[t] = scanned[(long long)t * tiles + blockIdx.x];
#pragma unroll
  for (int k = 0; k < kRadixWarps; ++k) wcnt[k][t] = 0;
  __syncthreads();
  const long long tile0 = (long long)blockIdx.x * kRadixTile;
  for (int r = 0; r < kRadixRounds; ++r) {
    const long long i = tile0 + r * kRadixThreads + t;
    const bool valid = i < P;
    const unsigned int key = valid ? keyIn[i] : 0u;
    const unsigned int d = (key >> shift) & (kRadixDigits - 1);
    // invalid lanes get a tag no digit has, so they never join a group
    const unsigned int peers = __match_any_sync(0xffffffffu, valid ? d : (unsigned)kRadixDigits + lane);
    const unsigned int rankW = __popc(peers & ((1u << lane) - 1u));
    if (valid && rankW == 0) wcnt[w][d] = __popc(peers);
    __syncthreads();
    if (valid) {
      unsigned int slot = base[d] + rankW;
      for (int k = 0; k < w; ++k) slot += wcnt[k][d];
      keyOut[slot] = key;
      valOut[slot] = valIn ? valIn[i] : (unsigned int)i;
    }
    __syncthreads();
    unsigned int tot = 0;
#pragma unroll
    for (int k = 0; k < kRadixWarps; ++k) {
      tot += wcnt[k][t];
      wcnt[k][t] = 0;
    }
    base[t] += tot;
    __syncthreads();
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

long long sortTiles(long long P) { return (P + kRadixTile - 1) / kRadixTile; }
long long sortCountEntries(long long P) { return (long long)kRadixDigits * std::max(1LL, sortTiles(P)); }
long long sortScanBlocks(long long entries) { return (entries + kScanTile - 1) / kScanTile; }

int sortKeyBits(long long nCells, bool grouped) {
  int bits = 1;
  while (bits < 32 && ((nCells - 1) >> bits) != 0) ++bits;
  return bits + (grouped ? 1 : 0);
}

cudaError_t launchSortPermutation(const Geom& g, const float* pos, long long P, long long split, const SortScratch& sc,
                                  const unsigned int** perm, cudaStream_t s) {
  const long long n = g.r.size();
  if (n >= (1LL << 31) || P >= (1LL << 32)) return cudaErrorInvalidValue;
  *perm = sc.valA;
  if (P <= 0) return cudaSuccess;
  const bool grouped = split > 0 && split < P;
  const int bits = sortKeyBits(n, grouped);
  const unsigned int groupBit = grouped ? 1u << (bits - 1) : 0u;
  const int passes = (bits + kRadixBits - 1) / kRadixBits;
  const long long tiles = sortTiles(P), entries = sortCountEntries(P), nb = sortScanBlocks(entries);
  kSortKeys<<<sortGrid(P), kSortThreads, 0, s>>>(g, pos, P, grouped ? split : P, groupBit, sc.keyA);
  unsigned int *kIn = sc.keyA, *kOut = sc.keyB, *vIn = nullptr, *vOut = sc.valA;
  for (int pass = 0; pass < passes; ++pass) {
    const int shift = pass * kRadixBits;
    kRadixHist<<<(unsigned)tiles, kRadixThreads, 0, s>>>(kIn, P, shift, sc.counts, tiles);
    kScanTiles<<<(unsigned)nb, kScanThreads, 0, s>>>(sc.counts, entries, sc.sums);
    kScanSums<<<1, kScanThreads, 0, s>>>(sc.sums, (int)nb);
    kScanAdd<<<sortGrid(entries), kSortThreads, 0, s>>>(sc.counts, entries, sc.sums);
    kRadixScatter<<<(unsigned)tiles, kRadixThreads, 0, s>>>(kIn, vIn, P, shift, sc.counts, tiles, kOut, vOut);
    std::swap(kIn, kOut);
    vIn = vOut;
    vOut = (vOut == sc.valA) ? sc.valB : sc.valA;
  }
  *perm = vIn;
  return cudaGetLastError();
}

int sortPassesLaunches(long long nCells, bool grouped) {
  return 1 + 5 * ((sortKeyBits(nCells, grouped) + kRadixBits - 1) / kRadixBits);
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
