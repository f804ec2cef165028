// Device-side potential builder: projected potentials of Gaussian atoms.
//
// V[s, y, x] = scale * sum_{atoms a of slice s} amp_a exp(-(dy^2 + dx^2) / (2 sigma^2)),
// dy, dx the periodic (minimum-image) distances of pixel (y ps_y, x ps_x) to
// the atom, wrapped as ((p - c + L/2) mod L) - L/2 over the box L = n ps.
// This is the potential model of the benchmark configurations (sums of
// isotropic Gaussians per slice); it replaces the host-side construction of
// V - and its host->device copy - that precedes simulate_fresnel_as /
// simulate_wpm in the reference's notebooks (get_abtem_transmit,
// propagation.py:286-299, builds abTEM potentials on the host instead).
//
// One CTA per 32 x 32 tile of one slice.  The slice's atoms stream through
// shared memory in chunks; each chunk is culled to the atoms within 7 sigma of
// the tile (a farther atom adds less than exp(-24.5) = 2.3e-11 of its peak),
// kept in input order so sums are reproducible, their 1D profiles along the
// tile's rows and columns evaluated in float64, and every pixel sums
// amp gy gx over the survivors.  Output is written once: the kernel is bound by
// the V store (4 B per pixel) for the lattices of the configurations.
#include <cuda_runtime.h>

#include "wap_internal.h"

namespace wap {

constexpr int kPotTile = 32;
constexpr int kPotThreads = 256;
constexpr int kPotChunk = 128;   // atoms culled per round (profiles: 2 x 16 KB of shared memory)

__device__ __forceinline__ double wrap_dist(double p, double c, double L) {
  const double t = p - c + 0.5 * L;
  return t - L * floor(t / L) - 0.5 * L;
}

__global__ void __launch_bounds__(kPotThreads) gaussian_potential_kernel(
    const double* __restrict__ atoms, const int32_t* __restrict__ slice_start, int ny, int nx, double ps_y,
    double ps_x, double sigma, double scale, float* __restrict__ V) {
  __shared__ float gy[kPotChunk][kPotTile];   // amp * exp(-dy^2 / 2 s^2) per survivor and tile row
  __shared__ float gx[kPotChunk][kPotTile];   // exp(-dx^2 / 2 s^2) per survivor and tile column
  __shared__ int keep[kPotChunk];
  __shared__ int warp_count[kPotThreads / 32];
  __shared__ int n_keep;
  const int s = blockIdx.z;
  const int y0 = blockIdx.y * kPotTile, x0 = blockIdx.x * kPotTile;
  const double Ly = ny * ps_y, Lx = nx * ps_x;
  const double cut = 7.0 * sigma;
  const double inv2s2 = 1.0 / (2.0 * sigma * sigma);
  // tile centre and half extents (the tile may be cut by the grid edge)
  const int ty = min(kPotTile, ny - y0), tx = min(kPotTile, nx - x0);
  const double cy = (y0 + 0.5 * (ty - 1)) * ps_y, cx = (x0 + 0.5 * (tx - 1)) * ps_x;
  const double hy = 0.5 * (ty - 1) * ps_y + cut, hx = 0.5 * (tx - 1) * ps_x + cut;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int col = threadIdx.x & (kPotTile - 1);
  const int row0 = threadIdx.x / kPotTile;   // rows row0 + 8 k
  float acc[kPotTile * kPotTile / kPotThreads] = {};

  const int a_begin = slice_start[s], a_end = slice_start[s + 1];
  for (int c0 = a_begin; c0 < a_end; c0 += kPotChunk) {
    // 1. cull this chunk to the atoms near the tile, keeping input order
    const int a = c0 + threadIdx.x;
    bool near = false;
    if (threadIdx.x < kPotChunk && a < a_end) {
      const double ya = atoms[3 * (long long)a], xa = atoms[3 * (long long)a + 1];
      near = fabs(wrap_dist(cy, ya, Ly)) <= hy && fabs(wrap_dist(cx, xa, Lx)) <= hx;
    }
    const unsigned ballot = __ballot_sync(0xffffffffu, near);
    if (lane == 0) warp_count[warp] = __popc(ballot);
    __syncthreads();
    int base = 0;
    for (int w = 0; w < warp; ++w) base += warp_count[w];
    if (near) keep[base + __popc(ballot & ((1u << lane) - 1u))] = a;
    if (threadIdx.x == 0) {
      int t = 0;
      for (int w = 0; w < kPotThreads / 32; ++w) t += warp_count[w];
      n_keep = t;
    }
    __syncthreads();
    const int nk = n_keep;
    // 2. 1D profiles of the survivors along the tile's rows and columns (float64)
    for (int i = threadIdx.x; i < nk * kPotTile; i += blockDim.x) {
      const int j = i / kPotTile, r = i - j * kPotTile;
      const long long ai = keep[j];
      const double ya = atoms[3 * ai], xa = atoms[3 * ai + 1], amp = atoms[3 * ai + 2];
      const double dy = wrap_dist((y0 + r) * ps_y, ya, Ly);
      const double dx = wrap_dist((x0 + r) * ps_x, xa, Lx);
      gy[j][r] = (float)(amp * exp(-dy * dy * inv2s2));
      gx[j][r] = (float)exp(-dx * dx * inv2s2);
    }
    __syncthreads();
    // 3. every pixel of the tile sums its survivors
    for (int j = 0; j < nk; ++j) {
      const float g = gx[j][col];
#pragma unroll
      for (int k = 0; k < kPotTile * kPotTile / kPotThreads; ++k) acc[k] = fmaf(gy[j][row0 + 8 * k], g, acc[k]);
    }
    __syncthreads();
  }
  const int x = x0 + col;
  if (x >= nx) return;
  float* out = V + (long long)s * ny * nx;
#pragma unroll
  for (int k = 0; k < kPotTile * kPotTile / kPotThreads; ++k) {
    const int y = y0 + row0 + 8 * k;
    if (y < ny) out[(long long)y * nx + x] = (float)(scale * (double)acc[k]);
  }
}

}  // namespace wap

using namespace wap;

extern "C" int wap_gaussian_potential(int n_slices, int ny, int nx, double ps_y, double ps_x, const double* atoms,
                                      const int32_t* slice_start, double sigma, double scale, float* V,
                                      void* stream) {
  clear_error();
  if (!atoms && n_slices > 0) return fail(WAP_ERR_ARG, "atoms must be a device pointer");
  if (!slice_start || !V) return fail(WAP_ERR_ARG, "slice_start and V must be non-NULL device pointers");
  if (n_slices < 1 || n_slices > 65535) return fail(WAP_ERR_ARG, "n_slices=%d out of range [1, 65535]", n_slices);
  if (ny < 1 || nx < 1 || ny > (1 << 16) || nx > (1 << 16)) return fail(WAP_ERR_ARG, "bad grid %d x %d", ny, nx);
  if (!(ps_y > 0) || !(ps_x > 0) || !(sigma > 0)) return fail(WAP_ERR_ARG, "sampling and sigma must be positive");
  const dim3 grid((nx + kPotTile - 1) / kPotTile, (ny + kPotTile - 1) / kPotTile, n_slices);
  count_launch();
  gaussian_potential_kernel<<<grid, kPotThreads, 0, (cudaStream_t)stream>>>(atoms, slice_start, ny, nx, ps_y, ps_x,
                                                                            sigma, scale, V);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? WAP_OK : cuda_fail(e, "gaussian_potential_kernel");
}
