// Shot sampling (jq_sample_shots): inverse-CDF draws over the prefix sum of
// the probabilities, on the GPU.  Restates the distribution of the
// reference's jax.random.choice over the probabilities + histogram
// (jaqsi/simulation.py:860-917); the random stream is this library's own
// counter-based generator (splitmix64 of seed and shot index), not JAX's.
//
// Included by jqsim.cu inside namespace jq::(anonymous).

constexpr int kScanThreads = 256;
constexpr int kScanPer = 4;                        // elements per thread
constexpr int kScanTile = kScanThreads * kScanPer;  // elements per CTA

__device__ __forceinline__ uint64_t splitmix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

// Inclusive scan of one 1024-element tile of every row (blockIdx.y); the
// tile total goes to bsum[row * ntiles + tile].
__global__ void __launch_bounds__(kScanThreads) k_scan_tiles(const double* __restrict__ p, int64_t dim,
                                                             double* __restrict__ cdf, double* __restrict__ bsum,
                                                             int64_t ntiles, int64_t row0) {
  __shared__ double warp_tot[kScanThreads / 32];
  const int64_t row = row0 + blockIdx.y;
  const int64_t base = row * dim + static_cast<int64_t>(blockIdx.x) * kScanTile;
  const int64_t lim = dim - static_cast<int64_t>(blockIdx.x) * kScanTile;
  double v[kScanPer];
  double run = 0.0;
#pragma unroll
  for (int k = 0; k < kScanPer; ++k) {
    const int64_t i = static_cast<int64_t>(threadIdx.x) * kScanPer + k;
    const double x = i < lim ? fmax(p[base + i], 0.0) : 0.0;  // negative rounding noise counts as 0
    run += x;
    v[k] = run;
  }
  // exclusive scan of the per-thread totals across the CTA
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  double inc = run;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const double y = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += y;
  }
  if (lane == 31) warp_tot[warp] = inc;
  __syncthreads();
  double wbase = 0.0;
  for (int w = 0; w < warp; ++w) wbase += warp_tot[w];
  const double off = wbase + inc - run;
#pragma unroll
  for (int k = 0; k < kScanPer; ++k) {
    const int64_t i = static_cast<int64_t>(threadIdx.x) * kScanPer + k;
    if (i < lim) cdf[base + i] = v[k] + off;
  }
  if (threadIdx.x == kScanThreads - 1) bsum[row * ntiles + blockIdx.x] = off + run;
}

// Exclusive prefix of the tile totals of one row (one CTA per row, serial
// over chunks of the CTA's width).
__global__ void __launch_bounds__(kScanThreads) k_scan_totals(double* __restrict__ bsum, int64_t ntiles) {
  __shared__ double warp_tot[kScanThreads / 32];
  __shared__ double carry;
  double* b = bsum + static_cast<int64_t>(blockIdx.x) * ntiles;
  if (threadIdx.x == 0) carry = 0.0;
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int64_t c0 = 0; c0 < ntiles; c0 += kScanThreads) {
    const int64_t i = c0 + threadIdx.x;
    const double x = i < ntiles ? b[i] : 0.0;
    double inc = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const double y = __shfl_up_sync(0xffffffffu, inc, o);
      if (lane >= o) inc += y;
    }
    if (lane == 31) warp_tot[warp] = inc;
    __syncthreads();
    double wbase = 0.0;
    for (int w = 0; w < warp; ++w) wbase += warp_tot[w];
    const double excl = carry + wbase + inc - x;
    double chunk = 0.0;
    for (int w = 0; w < kScanThreads / 32; ++w) chunk += warp_tot[w];
    __syncthreads();
    if (i < ntiles) b[i] = excl;
    if (threadIdx.x == 0) carry += chunk;
    __syncthreads();
  }
}

__global__ void k_scan_add(double* __restrict__ cdf, int64_t dim, const double* __restrict__ bsum, int64_t ntiles,
                           int64_t row0) {
  const int64_t row = row0 + blockIdx.y;
  const double add = bsum[row * ntiles + blockIdx.x];
  const int64_t base = row * dim + static_cast<int64_t>(blockIdx.x) * kScanTile;
  const int64_t lim = dim - static_cast<int64_t>(blockIdx.x) * kScanTile;
  for (int64_t i = threadIdx.x; i < kScanTile && i < lim; i += blockDim.x) cdf[base + i] += add;
}

// One draw per shot: u uniform in [0, total), the smallest i with
// cdf[i] > u (a zero-probability index is never chosen).
__global__ void k_sample(const double* __restrict__ cdf, int64_t dim, int64_t shots, uint64_t seed,
                         uint32_t* __restrict__ counts, int64_t row0) {
  const int64_t row = row0 + blockIdx.y;
  const double* c = cdf + row * dim;
  const double total = c[dim - 1];
  if (!(total > 0.0)) return;
  const uint64_t rseed = splitmix64(seed ^ (0xD1B54A32D192ED03ull * static_cast<uint64_t>(row + 1)));
  for (int64_t s = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; s < shots;
       s += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const uint64_t r = splitmix64(rseed + static_cast<uint64_t>(s) * 0x9E3779B97F4A7C15ull);
    const double u = static_cast<double>(r >> 11) * 0x1.0p-53 * total;
    int64_t lo = 0, hi = dim - 1;
    while (lo < hi) {
      const int64_t mid = (lo + hi) >> 1;
      if (c[mid] > u) hi = mid;
      else lo = mid + 1;
    }
    atomicAdd(&counts[row * dim + lo], 1u);
  }
}

int sample_impl(const double* probs, int batch, int64_t dim, int64_t shots, uint64_t seed, void* ws,
                size_t ws_bytes, uint32_t* counts, cudaStream_t st) {
  const int64_t ntiles = (dim + kScanTile - 1) / kScanTile;
  const size_t need = sample_ws_bytes(batch, dim);
  if (!ws || ws_bytes < need) {
    set_error("jq_sample_shots: workspace too small: need " + std::to_string(need) + " bytes");
    return JQ_ENOMEM;
  }
  double* cdf = static_cast<double*>(ws);
  double* bsum = cdf + static_cast<int64_t>(batch) * dim;
  JQ_CUDA(cudaMemsetAsync(counts, 0, sizeof(uint32_t) * static_cast<size_t>(batch) * dim, st));
  // rows run along grid.y, at most kMaxGridY per launch (row0 keeps each
  // row's index, and so its random stream, whatever the slicing)
  for (int b0 = 0; b0 < batch; b0 += kMaxGridY) {
    const dim3 g(static_cast<unsigned>(ntiles), static_cast<unsigned>(std::min(batch - b0, kMaxGridY)));
    k_scan_tiles<<<g, kScanThreads, 0, st>>>(probs, dim, cdf, bsum, ntiles, b0);
  }
  k_scan_totals<<<batch, kScanThreads, 0, st>>>(bsum, ntiles);
  for (int b0 = 0; b0 < batch; b0 += kMaxGridY) {
    const dim3 g(static_cast<unsigned>(ntiles), static_cast<unsigned>(std::min(batch - b0, kMaxGridY)));
    k_scan_add<<<g, kScanThreads, 0, st>>>(cdf, dim, bsum, ntiles, b0);
  }
  if (shots > 0) {
    const int64_t gx = std::max<int64_t>(1, std::min<int64_t>((shots + 255) / 256, 4 * sm_count()));
    for (int b0 = 0; b0 < batch; b0 += kMaxGridY) {
      const dim3 g(static_cast<unsigned>(gx), static_cast<unsigned>(std::min(batch - b0, kMaxGridY)));
      k_sample<<<g, 256, 0, st>>>(cdf, dim, shots, seed, counts, b0);
    }
  }
  JQ_CUDA(cudaGetLastError());
  return JQ_OK;
}
