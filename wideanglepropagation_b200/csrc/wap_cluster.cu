// One-launch multislice of single probes with the wave resident in the
// distributed shared memory of a thread-block cluster.
//
// A probe's wave (n x n complex64, 512 KB at 256^2) is spread over the 16 CTAs
// of one cluster.  CTA k owns rows [k R, (k+1) R) in its row slab and columns
// [k R, (k+1) R) in its column buffer (R = n / 16).  Every slice is
//   row pass     each CTA transforms its rows (inverse row FFT, [snapshot],
//                transmission, forward row FFT), exchanging through its own
//                slab, and stores every element straight into the column
//                buffer of the CTA that owns its column (st.shared::cluster)
//   barrier      barrier.cluster (release / acquire)
//   column pass  each CTA transforms its columns (column FFT, * H (hi + lo,
//                cached in shared memory for the launch), [pattern], inverse
//                column FFT) in its column buffer and stores every element
//                into the row slab of the CTA that owns its row
//   barrier
// so the wave never leaves the SMs between slices, and distributed shared
// memory is only ever written remotely, never read (stores are posted; the
// release barrier waits for them once per pass).  A buffer is rewritten by
// the other CTAs only in the pass after its owner read it, across a barrier,
// so one slab and one column buffer suffice.  The next slice's transmission
// row is fetched into registers during the column pass, hiding its L2
// latency.  The barriers are the hardware cluster barrier (all CTAs of a
// cluster are co-resident by construction); no CTA touches another's shared
// memory after the last one, so CTAs may exit independently.
//
// One cluster per probe.  Square grids of 128 points by default, 256 when
// asked for through WAP_KNOB_CLUSTER (there the 16 SMs of one cluster take
// longer than the cooperative chain on all SMs; a 512^2 wave would need
// 128 KB of slab and 128 KB of column buffer per CTA).  Falls back (-1) when
// the device cannot co-schedule a 16-CTA cluster of the kernel.
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "wap_internal.h"
#include "wap_passes.cuh"

namespace wap {

struct ClusterArgs {
  RowArgs r;
  ColArgs c;
  int n_slices;
  float2* stack;       // (B, n_slices, n, n) or null
  const float4* tw;    // stage twiddles of the (n, E) plan
};

__device__ __forceinline__ uint32_t cl_rank() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}
__device__ __forceinline__ uint32_t cl_id() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%clusterid.x;" : "=r"(r));
  return r;
}
__device__ __forceinline__ uint32_t cl_smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
// address of the same shared-memory offset in CTA `rank` of the cluster
__device__ __forceinline__ uint32_t cl_map(uint32_t addr, uint32_t rank) {
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(addr), "r"(rank));
  return r;
}
__device__ __forceinline__ void cl_st(uint32_t addr, float2 v) {
  asm volatile("st.shared::cluster.v2.f32 [%0], {%1, %2};" ::"r"(addr), "f"(v.x), "f"(v.y) : "memory");
}
// every thread of every CTA of the cluster; shared-memory writes before it
// are visible to the whole cluster after it
__device__ __forceinline__ void cl_sync() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}

template <int N, int E>
struct ClusterCfg {
  static constexpr int CS = 16;                 // CTAs per cluster
  static constexpr int T = N / E;               // threads per transform
  static constexpr int R = N / CS;              // rows (and columns) per CTA
  static constexpr int TPB = R * T;             // one row (column) transform per T threads
  static constexpr int PADN = RowExchange<true>::padded(N);
  static constexpr int TW = FFTPlan<N, E>::TW_SIZE;
  static constexpr size_t kTwBytes = (size_t)TW * sizeof(float4);
  static constexpr size_t kHBytes = (size_t)N * R * sizeof(float4);     // [N][R] (H, H_lo)
  static constexpr size_t kSlabBytes = (size_t)R * PADN * sizeof(float2);
  static constexpr size_t kColBytes = (size_t)N * R * sizeof(float2);   // column buffer [N][R]
  static constexpr size_t kBytes = kTwBytes + kHBytes + kSlabBytes + kColBytes;
  static_assert(T <= 32, "a row transform within one warp");
  static_assert(TPB % 32 == 0 && TPB <= 1024, "whole warps");
};

// slab index of row element x (one padding word per 16, as RowExchange)
__device__ __forceinline__ int cl_pad(int x) { return x + (x >> 4); }

template <int N, int E>
__global__ void __launch_bounds__(ClusterCfg<N, E>::TPB) cluster_kernel(const ClusterArgs a) {
  using K = ClusterCfg<N, E>;
  constexpr int T = K::T, R = K::R, PADN = K::PADN;
  extern __shared__ __align__(16) unsigned char cl_smem[];
  float4* tw = reinterpret_cast<float4*>(cl_smem);
  float4* hs = reinterpret_cast<float4*>(cl_smem + K::kTwBytes);
  float2* slab = reinterpret_cast<float2*>(cl_smem + K::kTwBytes + K::kHBytes);   // [R][PADN]
  float2* colb = slab + R * PADN;                                                 // [N][R]
  const RowArgs& r = a.r;
  const ColArgs& c = a.c;
  const int rank = (int)cl_rank();
  const int b = (int)cl_id();   // one probe per cluster
  const int tid = threadIdx.x;
  const long long plane = (long long)N * N;

  for (int i = tid; i < K::TW; i += K::TPB) tw[i] = __ldg(a.tw + i);
  for (int i = tid; i < N * R; i += K::TPB) {
    const long long o = (long long)(i / R) * N + rank * R + i % R;
    const float2 h = __ldg(c.H + o);
    const float2 l = c.H_lo ? __ldg(c.H_lo + o) : make_float2(0.f, 0.f);
    hs[i] = make_float4(h.x, h.y, l.x, l.y);
  }

  const int d = r.draw ? r.draw[b] : 0;
  // row roles: row rl of this CTA, lane t of its transform
  const int rl = tid / T, t = tid - rl * T;
  const int row = rank * R + rl;
  float2* srow = slab + rl * PADN;
  const RowExchange<true> xs{srow};
  // column roles: column cc of this CTA, lane tc of its transform
  const int cc = tid % R, tc = tid / R;
  const int col = rank * R + cc;
  const ColExchange<> cx{colb, R, cc};
  // remote targets: this thread's row elements in the column buffers
  // (element x goes to CTA x / R, [row][x % R]), its column elements in the
  // row slabs (row y to CTA y / R, [y % R][col])
  const uint32_t colb_row = cl_smem_u32(colb) + (uint32_t)(row * R) * sizeof(float2);
  const uint32_t slab_col = cl_smem_u32(slab) + (uint32_t)cl_pad(col) * sizeof(float2);
  // fftshift of the column for the pattern, and its place in the window
  const int sx = (col + (N >> 1)) & (N - 1);
  const int drx = sx - c.det.x0;
  const bool dcol = (unsigned)drx < (unsigned)c.det.nx;

  // the transmission row of the next row pass: exp(i phi) from the table, or
  // the potential, to be turned into exp(i phi) there
  float2 tn[E];
  auto fetch_t = [&](int s) {
    const long long vo = (long long)d * r.v_draw_stride + (long long)s * plane + (long long)row * N;
    if (r.ttab) {
#pragma unroll
      for (int e = 0; e < E; ++e) tn[e] = __ldg(r.ttab + vo + t + T * e);
    } else {
#pragma unroll
      for (int e = 0; e < E; ++e) tn[e].x = __ldg(r.V + vo + t + T * e);
    }
  };
  if (a.n_slices > 0) fetch_t(0);
  __syncthreads();

  for (int s = 0; s <= a.n_slices; ++s) {
    // ---- row pass: this CTA's rows
    float2 v[E];
    if (s == 0) {
      // move_probe (propagation.py:263-276): roll by position - (n//2, n//2)
      int sy = 0, sxp = 0;
      if (r.shifts) {
        sy = (r.shifts[2 * b] - (N >> 1)) & (N - 1);
        sxp = (r.shifts[2 * b + 1] - (N >> 1)) & (N - 1);
      }
      const float2* src = r.src + (long long)b * r.src_bstride + (long long)((row - sy) & (N - 1)) * N;
#pragma unroll
      for (int e = 0; e < E; ++e) v[e] = __ldg(src + ((t + T * e - sxp) & (N - 1)));
    } else {
#pragma unroll
      for (int e = 0; e < E; ++e) v[e] = srow[cl_pad(t + T * e)];
      fft<N, E, true>(v, t, xs, tw);
#pragma unroll
      for (int e = 0; e < E; ++e) v[e] = cscale(v[e], r.scale);
      // the wave after slice s - 1
      if (a.stack) {
        float2* sp = a.stack + ((long long)b * a.n_slices + (s - 1)) * plane + (long long)row * N;
#pragma unroll
        for (int e = 0; e < E; ++e) __stcs(sp + t + T * e, v[e]);
      }
      if (s == a.n_slices) {
        float2* pe = r.psi + (long long)b * r.psi_bstride + (long long)row * N;
#pragma unroll
        for (int e = 0; e < E; ++e) __stcg(pe + t + T * e, v[e]);
        break;
      }
    }
    if (r.ttab) {
#pragma unroll
      for (int e = 0; e < E; ++e) v[e] = cmul(v[e], tn[e]);
    } else {
#pragma unroll
      for (int e = 0; e < E; ++e) v[e] = cmul(v[e], transmission(tn[e].x, r.ri_a, r.ri_inv_den, r.kphase));
    }
    fft<N, E, false>(v, t, xs, tw);
#pragma unroll
    for (int e = 0; e < E; ++e) {
      const int x = t + T * e;
      cl_st(cl_map(colb_row + (uint32_t)(x % R) * sizeof(float2), (uint32_t)(x / R)), v[e]);
    }
    cl_sync();

    // ---- column pass: this CTA's columns, in its column buffer
    if (s + 1 < a.n_slices) fetch_t(s + 1);
#pragma unroll
    for (int e = 0; e < E; ++e) v[e] = colb[(tc + T * e) * R + cc];
    fft<N, E, false>(v, tc, cx, tw);
#pragma unroll
    for (int e = 0; e < E; ++e) {
      const float4 h = hs[(tc + T * e) * R + cc];
      v[e] = cmul_hl(v[e], make_float2(h.x, h.y), make_float2(h.z, h.w));
    }
    if (s == a.n_slices - 1 && c.dp) {
      float* dp = c.dp + (long long)b * c.det.plane() + drx;
#pragma unroll
      for (int e = 0; e < E; ++e) {
        const int ry = ((tc + T * e + (N >> 1)) & (N - 1)) - c.det.y0;
        if (dcol && (unsigned)ry < (unsigned)c.det.ny) __stcs(dp + ry * c.det.nx, fmaf(v[e].x, v[e].x, v[e].y * v[e].y));
      }
    }
    fft<N, E, true>(v, tc, cx, tw);
#pragma unroll
    for (int e = 0; e < E; ++e) {
      const int y = tc + T * e;
      cl_st(cl_map(slab_col + (uint32_t)((y % R) * PADN) * sizeof(float2), (uint32_t)(y / R)), v[e]);
    }
    cl_sync();
  }
}

// launch = false: only whether a cluster of this kernel can be co-scheduled
template <int N, int E>
static cudaError_t cluster_launch_t(const ClusterArgs& a, int n_probes, cudaStream_t st, bool launch, bool* fits) {
  using K = ClusterCfg<N, E>;
  auto kern = cluster_kernel<N, E>;
  cudaError_t e;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(K::CS * n_probes);
  cfg.blockDim = dim3(K::TPB);
  cfg.dynamicSmemBytes = K::kBytes;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = K::CS;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  if (!launch) {
    if ((e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)K::kBytes)) != cudaSuccess)
      return e;
    if ((e = cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1)) != cudaSuccess) return e;
    int clusters = 0;
    if ((e = cudaOccupancyMaxActiveClusters(&clusters, kern, &cfg)) != cudaSuccess) return e;
    *fits = clusters >= 1;
    return cudaSuccess;
  }
  const cudaError_t r = cudaLaunchKernelEx(&cfg, kern, a);
  if (r == cudaSuccess) count_launch();
  return r;
}

// elements per thread of the cluster kernel: 128 threads per CTA at 128^2
// (E = 8), 256 at 256^2 (E = 16, one exchange per transform)
static int cluster_elems(int n) { return n == 256 ? 16 : 8; }

static cudaError_t cluster_launch(int n, int e, const ClusterArgs& a, int n_probes, cudaStream_t st, bool launch,
                                  bool* fits) {
  switch (e * 10000 + n) {
    case 16 * 10000 + 256: return cluster_launch_t<256, 16>(a, n_probes, st, launch, fits);
    case 8 * 10000 + 256: return cluster_launch_t<256, 8>(a, n_probes, st, launch, fits);
    case 8 * 10000 + 128: return cluster_launch_t<128, 8>(a, n_probes, st, launch, fits);
    case 4 * 10000 + 128: return cluster_launch_t<128, 4>(a, n_probes, st, launch, fits);
    default: *fits = false; return cudaSuccess;
  }
}

constexpr int kClusterMaxProbes = 8;   // clusters that run at once on a B200 (16 SMs each)

int cluster_forward(wap_plan* p, const RowArgs& r, const ColArgs& c, int n_probes, int n_slices, float2* stack,
                    cudaStream_t st) {
  const int n = p->nx;
  const int kv = knob_value(WAP_KNOB_CLUSTER);
  if (kv == 0) return -1;
  if (p->generic || p->ny != n || n_probes > kClusterMaxProbes || n_slices < 1) return -1;
  // by default 128^2 only: at 256^2 the 16 SMs of a cluster take longer than
  // the cooperative chain on all SMs (B200, 20 slices: 164 vs 154 us)
  if (n != 128 && !(n == 256 && kv > 1)) return -1;
  int E = cluster_elems(n);
  if (kv == 4 || kv == 8 || kv == 16) E = kv;
  cudaError_t e;
  if (p->cl_e != E) {
    cudaFree(p->cl_tw);
    p->cl_tw = nullptr;
    p->cl_e = 0;
    const std::vector<float4> h = twiddle_table(n, E);
    if ((e = cudaMalloc(&p->cl_tw, h.size() * sizeof(float4))) != cudaSuccess ||
        (e = cudaMemcpy(p->cl_tw, h.data(), h.size() * sizeof(float4), cudaMemcpyHostToDevice)) != cudaSuccess)
      return cuda_fail(e, "cluster twiddle table");
    // whether this device co-schedules a 16-CTA cluster of the kernel (asked
    // once per plan and shape)
    bool fits = false;
    if ((e = cluster_launch(n, E, ClusterArgs{}, 1, st, false, &fits)) != cudaSuccess) {
      cudaGetLastError();
      fits = false;
    }
    p->cl_fits = fits ? 1 : 0;
    p->cl_e = E;
  }
  if (!p->cl_fits) return -1;
  ClusterArgs a{};
  a.r = r;
  a.c = c;
  a.r.probe0 = a.c.probe0 = 0;
  a.n_slices = n_slices;
  a.stack = stack;
  a.tw = p->cl_tw;
  bool fits = true;
  const ProfToken tok = prof_begin(WAP_KIND_ROW, st);
  // knob value 1: the launch counts as refused without being issued (a
  // host-side test of the fallback below)
  e = kv == 1 ? cudaErrorInvalidClusterSize : cluster_launch(n, E, a, n_probes, st, true, &fits);
  if (e != cudaSuccess) {
    prof_end(tok, st, 0.0);   // closes the trace token (a record of zero bytes)
    // a device shared with other work may refuse the 16-CTA cluster at launch
    // even where the occupancy query allowed it: the chain serves this plan
    // from now on (a refused launch leaves no error behind)
    if (e == cudaErrorInvalidClusterSize || e == cudaErrorLaunchOutOfResources) {
      if (kv != 1) cudaGetLastError();
      p->cl_fits = 0;
      return -1;
    }
    return cuda_fail(e, "cluster_kernel");
  }
  // one slice step: wave in / out twice, potential or table once
  prof_end(tok, st, (double)n_probes * n_slices * n * n * 20.0);
  return WAP_OK;
}

}  // namespace wap
