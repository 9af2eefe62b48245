// Device-wide exclusive scans over packed arrays (three passes: tile sums,
// scan of the tile sums in one block, tile scan with the tile's offset).
// In place: data[0..n) becomes the exclusive prefix and data[n] the total.
// The tile passes move every element with coalesced global loads and stores and
// hand each thread its kItems consecutive elements through shared memory padded
// by one word per 128 bytes, which keeps both access patterns free of bank
// conflicts for 32- and 64-bit elements.
#include "pxl_internal.cuh"

namespace pxl {

namespace {

constexpr int kTpb = 256;
constexpr int kItems = 8;
constexpr int kTile = kTpb * kItems;
constexpr int kSumItems = 4;  // tile sums per thread in the single-block pass

// shared-memory slot of tile element j: one padding element per 128 bytes
template <class T>
__device__ __forceinline__ int pad_idx(int j) {
  return j + j / (128 / int(sizeof(T)));
}
template <class T>
__host__ __device__ constexpr int tile_smem_elems() {
  return kTile + kTile / (128 / int(sizeof(T)));
}

// Loads tile elements base .. base + kTile (zero at and past n) with coalesced
// reads and returns this thread's kItems consecutive ones in v.
template <class T>
__device__ __forceinline__ void load_tile(const T* __restrict__ src, int64_t base, int64_t n, T* s,
                                          T (&v)[kItems]) {
#pragma unroll
  for (int k = 0; k < kItems; ++k) {
    const int j = k * kTpb + int(threadIdx.x);
    s[pad_idx<T>(j)] = base + j < n ? src[base + j] : T(0);
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < kItems; ++k) v[k] = s[pad_idx<T>(int(threadIdx.x) * kItems + k)];
}

// n_dev (optional) holds the live element count; tiles past it do nothing, so a
// launch sized for the buffer capacity costs only the live part.
__device__ __forceinline__ int64_t live_n(int64_t n, const uint32_t* n_dev) {
  return n_dev ? (int64_t(*n_dev) < n ? int64_t(*n_dev) : n) : n;
}

template <class T>
__global__ void k_tile_sums(const T* __restrict__ data, int64_t ncap, const uint32_t* n_dev, T* __restrict__ sums) {
  int64_t n = live_n(ncap, n_dev);
  int64_t base = int64_t(blockIdx.x) * kTile;
  if (base >= n && base > 0) return;
  T s = 0;
  for (int k = 0; k < kItems; ++k) {
    int64_t i = base + int64_t(k) * kTpb + threadIdx.x;
    if (i < n) s += data[i];
  }
  // block reduce
  __shared__ T sh[kTpb / 32];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    T v = threadIdx.x < kTpb / 32 ? sh[threadIdx.x] : T(0);
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (threadIdx.x == 0) sums[blockIdx.x] = v;
  }
}

template <class T>
__device__ T warp_incl(T v) {
  const unsigned lane = threadIdx.x & 31u;
  for (int o = 1; o < 32; o <<= 1) {
    T t = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= unsigned(o)) v += t;
  }
  return v;
}

// exclusive scan of the tile sums in one block of 1024 threads, kSumItems
// consecutive sums per thread
template <class T>
__global__ void __launch_bounds__(1024) k_scan_sums(T* __restrict__ sums, int64_t ncap, const uint32_t* n_dev) {
  int64_t n = live_n(ncap, n_dev);
  int64_t nt = (n + kTile - 1) / kTile;
  __shared__ T sh[33];
  __shared__ T carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  const unsigned lane = threadIdx.x & 31u, wid = threadIdx.x >> 5;
  for (int64_t b = 0; b < nt; b += int64_t(blockDim.x) * kSumItems) {
    const int64_t i0 = b + int64_t(threadIdx.x) * kSumItems;
    T v[kSumItems];
    T tsum = 0;
#pragma unroll
    for (int k = 0; k < kSumItems; ++k) {
      v[k] = i0 + k < nt ? sums[i0 + k] : T(0);
      tsum += v[k];
    }
    T inc = warp_incl(tsum);
    if (lane == 31) sh[wid] = inc;
    __syncthreads();
    if (wid == 0) {
      T s = sh[lane];
      T si = warp_incl(s);
      sh[lane] = si - s;
      if (lane == 31) sh[32] = si;
    }
    __syncthreads();
    T r = carry + sh[wid] + inc - tsum;
#pragma unroll
    for (int k = 0; k < kSumItems; ++k) {
      if (i0 + k < nt) sums[i0 + k] = r;
      r += v[k];
    }
    __syncthreads();
    if (threadIdx.x == 0) carry += sh[32];
    __syncthreads();
  }
  if (threadIdx.x == 0) sums[nt] = carry;
}

template <class T>
__global__ void k_tile_scan(T* __restrict__ data, int64_t ncap, const uint32_t* n_dev, const T* __restrict__ sums) {
  int64_t n = live_n(ncap, n_dev);
  int64_t nt = (n + kTile - 1) / kTile;
  int64_t base = int64_t(blockIdx.x) * kTile;
  if (n == 0) {
    if (blockIdx.x == 0 && threadIdx.x == 0) data[0] = 0;
    return;
  }
  if (int64_t(blockIdx.x) >= nt) return;
  __shared__ T s_tile[tile_smem_elems<T>()];
  // each thread owns kItems consecutive elements
  T v[kItems];
  load_tile<T>(data, base, n, s_tile, v);
  T tsum = 0;
#pragma unroll
  for (int k = 0; k < kItems; ++k) tsum += v[k];
  __shared__ T sh[33];
  const unsigned lane = threadIdx.x & 31u, wid = threadIdx.x >> 5;
  T inc = warp_incl(tsum);
  if (lane == 31) sh[wid] = inc;
  __syncthreads();
  if (wid == 0) {
    T s = lane < kTpb / 32 ? sh[lane] : T(0);
    T si = warp_incl(s);
    if (lane < kTpb / 32) sh[lane] = si - s;
  }
  __syncthreads();
  // a thread rewrites only the slots it read, so no barrier is needed before
  T run = sums[blockIdx.x] + sh[wid] + inc - tsum;
#pragma unroll
  for (int k = 0; k < kItems; ++k) {
    s_tile[pad_idx<T>(int(threadIdx.x) * kItems + k)] = run;
    run += v[k];
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < kItems; ++k) {
    const int j = k * kTpb + int(threadIdx.x);
    if (base + j < n) data[base + j] = s_tile[pad_idx<T>(j)];
  }
  if (int64_t(blockIdx.x) == nt - 1 && threadIdx.x == 0) data[n] = sums[nt];
}

// Shifted form for lists filled by atomic increments: out[0] = 0 and out[i + 1] = the
// exclusive prefix of in[i]. A fill that takes slot atomicAdd(&out[i + 1], 1) for each of
// the in[i] entries of key i leaves out[i] = start of key i and out[n] = total: the
// offsets of the filled lists, with no second counter array to clear.
template <class T>
__global__ void k_tile_scan_shift(const T* __restrict__ in, T* __restrict__ out, int64_t ncap, const uint32_t* n_dev,
                                  const T* __restrict__ sums) {
  int64_t n = live_n(ncap, n_dev);
  int64_t nt = (n + kTile - 1) / kTile;
  int64_t base = int64_t(blockIdx.x) * kTile;
  if (blockIdx.x == 0 && threadIdx.x == 0) out[0] = 0;
  if (int64_t(blockIdx.x) >= nt) return;
  __shared__ T s_tile[tile_smem_elems<T>()];
  T v[kItems];
  load_tile<T>(in, base, n, s_tile, v);
  T tsum = 0;
#pragma unroll
  for (int k = 0; k < kItems; ++k) tsum += v[k];
  __shared__ T sh[33];
  const unsigned lane = threadIdx.x & 31u, wid = threadIdx.x >> 5;
  T inc = warp_incl(tsum);
  if (lane == 31) sh[wid] = inc;
  __syncthreads();
  if (wid == 0) {
    T s = lane < kTpb / 32 ? sh[lane] : T(0);
    T si = warp_incl(s);
    if (lane < kTpb / 32) sh[lane] = si - s;
  }
  __syncthreads();
  T run = sums[blockIdx.x] + sh[wid] + inc - tsum;
#pragma unroll
  for (int k = 0; k < kItems; ++k) {
    s_tile[pad_idx<T>(int(threadIdx.x) * kItems + k)] = run;
    run += v[k];
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < kItems; ++k) {
    const int j = k * kTpb + int(threadIdx.x);
    if (base + j < n) out[base + j + 1] = s_tile[pad_idx<T>(j)];
  }
}

template <class T>
void excl_scan_shift(const T* in, T* out, int64_t ncap, const uint32_t* n_dev, T* tmp, cudaStream_t s) {
  int64_t nt = ncap > 0 ? (ncap + kTile - 1) / kTile : 1;
  k_tile_sums<T><<<unsigned(nt), kTpb, 0, s>>>(in, ncap, n_dev, tmp);
  k_scan_sums<T><<<1, 1024, 0, s>>>(tmp, ncap, n_dev);
  k_tile_scan_shift<T><<<unsigned(nt), kTpb, 0, s>>>(in, out, ncap, n_dev, tmp);
}

template <class T>
void excl_scan(T* data, int64_t ncap, const uint32_t* n_dev, T* tmp, cudaStream_t s) {
  int64_t nt = ncap > 0 ? (ncap + kTile - 1) / kTile : 1;
  k_tile_sums<T><<<unsigned(nt), kTpb, 0, s>>>(data, ncap, n_dev, tmp);
  k_scan_sums<T><<<1, 1024, 0, s>>>(tmp, ncap, n_dev);
  k_tile_scan<T><<<unsigned(nt), kTpb, 0, s>>>(data, ncap, n_dev, tmp);
}

}  // namespace

int64_t scan_tmp_elems(int64_t n) { return (n + kTile - 1) / kTile + 2; }

void excl_scan_u32(uint32_t* data, int64_t ncap, const uint32_t* n_dev, uint32_t* tmp, cudaStream_t s) {
  excl_scan<uint32_t>(data, ncap, n_dev, tmp, s);
}
void excl_scan_u64(uint64_t* data, int64_t ncap, const uint32_t* n_dev, uint64_t* tmp, cudaStream_t s) {
  excl_scan<uint64_t>(data, ncap, n_dev, tmp, s);
}
void excl_scan_shift_u32(const uint32_t* in, uint32_t* out, int64_t ncap, const uint32_t* n_dev, uint32_t* tmp,
                         cudaStream_t s) {
  excl_scan_shift<uint32_t>(in, out, ncap, n_dev, tmp, s);
}

}  // namespace pxl
