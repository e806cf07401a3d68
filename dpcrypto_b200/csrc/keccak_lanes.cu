// Keccak-f[1600] in each lanes-per-state layout, on independent states in device memory:
// one lane per state (keccak.cuh), a lane pair in bit-interleaved form (keccak_pair.cuh),
// five lanes per state (keccak5.cuh) and a warp per state (keccak25.cuh).  Used to check the layouts against each other and the
// oracle (dpkem_keccak_f1600_lanes) and to measure the latency of a dependent permutation
// chain per layout and batch size (dpkem_probe_keccak_chain), which is what picks the layout
// of each latency-bound sponge stage.
#include "common.cuh"
#include "keccak.cuh"
#include "keccak25.cuh"
#include "keccak5.cuh"
#include "keccak_pair.cuh"

namespace dpkem {
namespace {

// One warp per block.  in/out: n states of 25 little-endian 64-bit lanes.
template <int LANES>
__global__ void __launch_bounds__(32) lanes_kernel(const uint2 *in, uint2 *out, int n, int perms) {
  const int lane = threadIdx.x;
  if constexpr (LANES == 1) {
    const int s = blockIdx.x * 32 + lane;
    if (s >= n) return;
    uint2 a[25];
#pragma unroll
    for (int q = 0; q < 25; q++) a[q] = in[(size_t)s * 25 + q];
    for (int p = 0; p < perms; p++) keccak_f1600(a);
#pragma unroll
    for (int q = 0; q < 25; q++) out[(size_t)s * 25 + q] = a[q];
  } else if constexpr (LANES == 2) {
    const int s = blockIdx.x * 16 + (lane >> 1), p = lane & 1;
    const bool live = s < n;
    const int sc = live ? s : n - 1;
    uint32_t a[25];
#pragma unroll
    for (int q = 0; q < 25; q++) a[q] = kpair::to_slice(in[(size_t)sc * 25 + q], p);
    for (int r = 0; r < perms; r++) kpair::f1600(a, p);
#pragma unroll
    for (int q = 0; q < 25; q++) {
      const uint32_t h = kpair::from_slice(a[q], p);
      if (live) reinterpret_cast<uint32_t *>(out + (size_t)s * 25 + q)[p] = h;
    }
  } else if constexpr (LANES == 25) {
    const k25::Lane k = k25::make_lane();
    const int s = blockIdx.x;
    uint2 v = in[(size_t)s * 25 + k.i];
    for (int r = 0; r < perms; r++) k25::f1600(v, k);
    if (lane < 25) out[(size_t)s * 25 + k.i] = v;
  } else {
    __shared__ __align__(16) uint8_t xbuf[k5::kSmemPerWarp];
    const k5::Lanes k = k5::make_lanes(xbuf);
    const int g = lane / 5, s = blockIdx.x * 6 + g;
    const bool live = g < 6 && s < n;
    const int sc = live ? s : n - 1;
    uint2 a[5];
#pragma unroll
    for (int y = 0; y < 5; y++) a[y] = in[(size_t)sc * 25 + k.t + 5 * y];
    for (int r = 0; r < perms; r++) k5::f1600(a, k);
#pragma unroll
    for (int y = 0; y < 5; y++)
      if (live) out[(size_t)s * 25 + k.t + 5 * y] = a[y];
  }
}

template <int LANES>
constexpr int states_per_block() {
  return LANES == 1 ? 32 : LANES == 2 ? 16 : LANES == 25 ? 1 : 6;
}

template <int LANES>
void launch(const uint2 *in, uint2 *out, int n, int perms, cudaStream_t st) {
  constexpr int spb = states_per_block<LANES>();
  lanes_kernel<LANES><<<(n + spb - 1) / spb, 32, 0, st>>>(in, out, n, perms);
}

cudaError_t run(int lanes, const uint2 *in, uint2 *out, int n, int perms, cudaStream_t st) {
  switch (lanes) {
    case 1: launch<1>(in, out, n, perms, st); break;
    case 2: launch<2>(in, out, n, perms, st); break;
    case 5: launch<5>(in, out, n, perms, st); break;
    case 25: launch<25>(in, out, n, perms, st); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

}  // namespace

cudaError_t keccak_lanes(int lanes, const uint64_t *in, uint64_t *out, int n, int perms, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  return run(lanes, reinterpret_cast<const uint2 *>(in), reinterpret_cast<uint2 *>(out), n, perms, st);
}

cudaError_t probe_keccak_chain(int lanes, int n, int perms, cudaStream_t st, double *ms_out) {
  uint2 *buf = nullptr;
  const size_t bytes = (size_t)n * 25 * 8;
  cudaError_t e = cudaMalloc(&buf, 2 * bytes);
  if (e != cudaSuccess) return e;
  cudaMemsetAsync(buf, 0x5A, bytes, st);
  cudaEvent_t t0, t1;
  cudaEventCreate(&t0);
  cudaEventCreate(&t1);
  e = run(lanes, buf, buf + (size_t)n * 25, n, 2, st);  // warm-up
  float ms = 0.f;
  if (e == cudaSuccess) {
    cudaEventRecord(t0, st);
    e = run(lanes, buf, buf + (size_t)n * 25, n, perms, st);
    cudaEventRecord(t1, st);
  }
  if (e == cudaSuccess) e = cudaEventSynchronize(t1);
  if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, t0, t1);
  if (e == cudaSuccess) *ms_out = ms;
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  cudaFree(buf);
  return e;
}

}  // namespace dpkem
