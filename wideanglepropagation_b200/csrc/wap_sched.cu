// Persistent batched multislice scheduler (Fresnel / angular spectrum).
//
// One launch advances every probe of every grid class of a scan through all of
// its slices.  The work is a ticket queue: the host lays out "pass descriptors"
// (class, probe group, pass), each expanding into probes x tiles tickets; CTAs
// claim tickets in increasing order with one atomicAdd and run the tile:
//
//   pass 2s     (row tile: ROWS consecutive rows of one probe)
//               s = 0: load psi0 rolled to the probe position (move_probe),
//               else inverse row FFT of slice s-1's column output, * 1/(n n);
//               then * t_s from the transmission table, forward row FFT
//   pass 2s+1   (column tile: n rows x W columns of one probe)
//               column FFT, * H (hi + lo), [dp on the last slice], inverse FFT
//   pass 2N     (row tile) inverse row FFT -> exit wave
//
// Dependencies are per probe: a tile of pass p needs every tile of passes
// 0..p-1 of the same probe, i.e. a per-probe completion counter >= the tile
// count of those passes.  Tickets are ordered (class, group, pass, probe,
// tile), so a tile only ever waits for smaller tickets, which were claimed by
// CTAs that are running or finished: the queue cannot deadlock.  Waits are
// bounded; on expiry the CTA records WAP_ERR_TIMEOUT, every CTA stops claiming,
// in-flight copies are drained (bounded) and the kernel returns.
//
// Probe groups are sized so that a group's waves stay L2-resident while the
// group walks through its slices; groups follow each other without a barrier.
//
// Tile loads use the Tensor Memory Accelerator: row tiles are contiguous
// (one cp.async.bulk), column tiles are 2D boxes of a tensor map over all
// probes' rows (cp.async.bulk.tensor.2d, no multicast).  A CTA copies the
// landed tile into registers, immediately issues the load of its next ticket
// into the same staging buffer, and computes the current tile meanwhile.
#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "wap_internal.h"
#include "wap_passes.cuh"

namespace wap {

constexpr int kSchedThreads = 256;
constexpr int kMaxClasses = 4;
// A tile is 256 compute threads x E elements (complex64): 32 KB for E = 16,
// 16 KB for E = 8; the exchange buffer holds rows x padded(n) of a row tile.
__host__ __device__ constexpr int kTileBytesFor(int e) { return 256 * e * 8; }
__host__ __device__ constexpr int kExchBytesFor(int e) { return 256 * e * 8 + 256 * e * 8 / 16; }
constexpr long long kSpinLimit = 1LL << 22;           // polls before a wait gives up

struct SchedClass {
  int n, log2n, n_slices, n_probes;
  int rows, cols_w;             // row-tile height, column-tile width
  int row_tiles, col_tiles;     // tiles per probe per pass
  int box_rows;                 // TMA box height for column tiles (<= 256)
  int done_off;                 // offset of this class's counters
  float2* psi;                  // (B, n, n) working buffer / exit
  const float2* psi0;           // (n, n) shared probe
  const int* positions;         // (B, 2) or null
  const int* draw;              // (B) or null
  const float2* ttab;           // (draws, N, n, n)
  long long ttab_draw_stride;   // N n n
  const float4* Hq;             // (n, n) interleaved (H_hi, H_lo)
  float* dp;                    // (B, n, n) or null
  const float4* tw;             // twiddles for (n, 16) in global memory
  int tw_off, tw_len;           // their place in the shared-memory copy
  float scale;                  // 1 / (n n)  (also folded into ttab)
  float inv_scale;              // n n
};

struct SchedDesc {
  long long base;   // first ticket
  int cls, pass, b0, nprobes, tiles;
};

struct alignas(64) SchedParams {
  CUtensorMap maps[kMaxClasses];   // column-tile tensor maps (one per class)
  SchedClass cls[kMaxClasses];
  const SchedDesc* desc;
  int n_desc;
  int n_classes;
  long long total;                 // number of tickets
  unsigned long long* ticket;      // claim counter
  int* done;                       // per-probe completed tiles
  int* status;                     // 0 or WAP_ERR_TIMEOUT
  long long spin_limit;            // polls before a wait gives up
  int stall_pass;                  // test hook: tiles of this pass wait forever (-1: off)
  int checks;                      // validate every task before use (debug)
  int tw_in_smem;                  // twiddles copied to shared memory (else read via L1)
  int* debug;                      // [code, cls, pass, b, tile, extra] of the first bad task
};

// ---------------------------------------------------------------------------
// PTX helpers: mbarrier, bulk / tensor copies, acquire loads
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t phase) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(phase)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
          smem_u32(dst)),
      "l"(map), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ int ld_acquire(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.global;" ::: "memory"); }

// ---------------------------------------------------------------------------
// tile bodies
// ---------------------------------------------------------------------------
struct Task {
  int cls, pass, b, tile, valid;
};

// tiles of passes 0..p-1 of one probe (row passes are the even ones)
__device__ __forceinline__ int tiles_before(const SchedClass& c, int p) {
  return ((p + 1) >> 1) * c.row_tiles + (p >> 1) * c.col_tiles;
}

// Debug validation of a decoded task (P.checks): record the first violation
// and report whether the task may be used.
__device__ __forceinline__ bool task_ok(const SchedParams& P, const Task& k, int where) {
  if (!P.checks) return true;
  bool ok = k.cls >= 0 && k.cls < P.n_classes;
  if (ok) {
    const SchedClass& c = P.cls[k.cls];
    ok = k.b >= 0 && k.b < c.n_probes && k.pass >= 0 && k.pass <= 2 * c.n_slices && k.tile >= 0 &&
         k.tile < ((k.pass & 1) ? c.col_tiles : c.row_tiles);
  }
  if (!ok && atomicCAS(P.debug, 0, where) == 0) {
    P.debug[1] = k.cls;
    P.debug[2] = k.pass;
    P.debug[3] = k.b;
    P.debug[4] = k.tile;
    P.debug[5] = k.valid;
  }
  return ok;
}

// Issue the TMA load of a task's input tile into `stage` (one thread).  This
// is the single arrival of the phase on `bar`: arrive.expect_tx(tile bytes),
// completed by the copy.  Returns false (no arrival) for tasks that load their
// input directly (first row pass).
__device__ __forceinline__ bool issue_load(const SchedParams& P, const Task& k, float2* stage, uint64_t* bar) {
  const SchedClass& c = P.cls[k.cls];
  const long long plane = (long long)c.n * c.n;
  if ((k.pass & 1) == 0) {
    if (k.pass == 0) return false;
    const float2* src = c.psi + (long long)k.b * plane + (long long)k.tile * c.rows * c.n;
    const uint32_t bytes = (uint32_t)(c.rows * c.n * sizeof(float2));
    mbar_expect_tx(bar, bytes);
    bulk_g2s(stage, src, bytes, bar);
  } else {
    const uint32_t bytes = (uint32_t)(c.n * c.cols_w * sizeof(float2));
    mbar_expect_tx(bar, bytes);
    for (int r0 = 0; r0 < c.n; r0 += c.box_rows)
      tma_load_2d(stage + r0 * c.cols_w, &P.maps[k.cls], k.tile * c.cols_w, k.b * c.n + r0, bar);
  }
  return true;
}

constexpr int kComputeWarps = kSchedThreads / 32;      // 8 compute warps
constexpr int kBlockThreads = kSchedThreads + 32;       // + 1 producer warp
constexpr int kFftBar = 2;                              // named barrier of the compute warps

// Row tile, phase 1: this thread's E input words into registers.
template <int N, int E>
__device__ __forceinline__ void row_load(const SchedClass& c, const Task& k, const float2* stage, float2 (&v)[E]) {
  constexpr int T = N / E;
  const int rl = threadIdx.x / T, t = threadIdx.x - rl * T;
  if (k.pass == 0) {
    // move_probe (propagation.py:263-276): roll psi0 by position - (n//2, n//2)
    const int row = k.tile * c.rows + rl;
    int sy = 0, sx = 0;
    if (c.positions) {
      sy = (c.positions[2 * k.b] - (N >> 1)) & (N - 1);
      sx = (c.positions[2 * k.b + 1] - (N >> 1)) & (N - 1);
    }
    const float2* s = c.psi0 + (long long)((row - sy) & (N - 1)) * N;
#pragma unroll
    for (int e = 0; e < E; ++e) v[e] = __ldg(s + ((t + T * e - sx) & (N - 1)));
  } else {
    const float2* s = stage + rl * N;
#pragma unroll
    for (int e = 0; e < E; ++e) v[e] = s[t + T * e];
  }
}

// Row tile, phase 2: [inverse row FFT, scale], [* t_s, forward row FFT], store.
template <int N, int E>
__device__ __forceinline__ void row_compute(const SchedClass& c, const Task& k, float2 (&v)[E], float2* exch,
                                            const float4* tw) {
  constexpr int T = N / E;
  constexpr int PADN = RowExchange<true>::padded(N);
  const int rl = threadIdx.x / T, t = threadIdx.x - rl * T;
  const int row = k.tile * c.rows + rl;
  const long long plane = (long long)N * N;
  const RowExchange<(T <= 32), kFftBar, kSchedThreads> xs{exch + rl * PADN};
  // ttab holds t / (n n): the inverse transform's normalisation rides on the
  // transmission multiply; the first pass (no inverse transform) undoes it
  // and the last pass (no transmission) applies it.  All factors are powers
  // of two, so this changes no rounding.
  if (k.pass != 0) {
    fft<N, E, true>(v, t, xs, tw);
  } else {
#pragma unroll
    for (int e = 0; e < E; ++e) v[e] = cscale(v[e], c.inv_scale);
  }
  if (k.pass == 2 * c.n_slices) {
#pragma unroll
    for (int e = 0; e < E; ++e) v[e] = cscale(v[e], c.scale);
  }
  if (k.pass < 2 * c.n_slices) {
    const int d = c.draw ? c.draw[k.b] : 0;
    const float2* trow =
        c.ttab + (long long)d * c.ttab_draw_stride + (long long)(k.pass >> 1) * plane + (long long)row * N;
#pragma unroll
    for (int e = 0; e < E; ++e) v[e] = cmul(v[e], __ldg(trow + t + T * e));
    fft<N, E, false>(v, t, xs, tw);
  }
  float2* prow = c.psi + (long long)k.b * plane + (long long)row * N;
#pragma unroll
  for (int e = 0; e < E; ++e) __stcg(prow + t + T * e, v[e]);
}

template <int N, int E>
__device__ __forceinline__ void col_load(const SchedClass& c, const float2* stage, float2 (&v)[E]) {
  constexpr int T = N / E;
  constexpr int W = kSchedThreads / T;
  const int cc = threadIdx.x % W, t = threadIdx.x / W;
#pragma unroll
  for (int e = 0; e < E; ++e) v[e] = stage[(t + T * e) * W + cc];
}

// Column tile: FFT, * H (hi + lo), [dp on the last slice], inverse FFT, store.
template <int N, int E>
__device__ __forceinline__ void col_compute(const SchedClass& c, const Task& k, float2 (&v)[E], float2* exch,
                                            const float4* tw) {
  constexpr int T = N / E;
  constexpr int W = kSchedThreads / T;
  const int cc = threadIdx.x % W, t = threadIdx.x / W;
  const int col = k.tile * W + cc;
  const long long plane = (long long)N * N;
  const ColExchange<kFftBar, kSchedThreads> xs{exch, W, cc};
  fft<N, E, false>(v, t, xs, tw);
  const float4* hcol = c.Hq + col;
#pragma unroll
  for (int e = 0; e < E; ++e) {
    const float4 h = __ldg(hcol + (t + T * e) * N);
    v[e] = cmul_hl(v[e], make_float2(h.x, h.y), make_float2(h.z, h.w));
  }
  if (c.dp && (k.pass >> 1) == c.n_slices - 1) {
    float* dp = c.dp + (long long)k.b * plane;
    const int sx = (col + (N >> 1)) & (N - 1);
#pragma unroll
    for (int e = 0; e < E; ++e) {
      const int sy = (t + T * e + (N >> 1)) & (N - 1);
      __stcs(dp + (long long)sy * N + sx, fmaf(v[e].x, v[e].x, v[e].y * v[e].y));
    }
  }
  fft<N, E, true>(v, t, xs, tw);
  float2* pcol = c.psi + (long long)k.b * plane + col;
#pragma unroll
  for (int e = 0; e < E; ++e) __stcg(pcol + (long long)(t + T * e) * N, v[e]);
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// bounded mbarrier wait; false if the limit expired
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t phase, long long limit) {
  long long spins = 0;
  while (!mbar_try_wait(bar, phase)) {
    if (++spins > limit) return false;
  }
  return true;
}

// Compute warps: take the published tile, pull it into registers, release the
// stage, run the transforms, store, report completion.
template <unsigned MASK, int E>
__device__ __forceinline__ void compute_loop(const SchedParams& P, float2* stage, float2* exch, const float4* tw_smem,
                                             uint64_t* full, uint64_t* empty, uint64_t* done_bar, const Task* s_task) {
  uint32_t fph = 0;
  uint32_t tiles_done = 0;   // selects the done barrier (two, alternating)
  const int lane = threadIdx.x & 31;
  while (true) {
    // Bounded wait for the next published item.  On expiry record the error
    // and keep waiting (bounded rounds): the producer's own waits are bounded
    // and it publishes the stop sentinel once an error is recorded, so every
    // compute warp reads the same item and runs the same barrier sequence.
    for (int round = 0; round < 4 && !mbar_wait(full, fph, P.spin_limit); ++round)
      atomicCAS(P.status, 0, WAP_ERR_TIMEOUT);
    fph ^= 1u;
    const Task k = *s_task;
    if (!k.valid) return;
    if (!task_ok(P, k, 1)) {
      __syncwarp();
      if (lane == 0) {
        mbar_arrive(empty);
        mbar_arrive(done_bar + (tiles_done & 1));
      }
      ++tiles_done;
      continue;
    }
    const SchedClass& c = P.cls[k.cls];
    const float4* tw = P.tw_in_smem ? tw_smem + c.tw_off : c.tw;
    float2 v[E];
#define WAP_SCHED_CASE(N, BIT)                                  \
    if constexpr ((MASK & BIT) != 0) {                            \
      if (c.n == N) {                                             \
        if (k.pass & 1) col_load<N, E>(c, stage, v);              \
        else row_load<N, E>(c, k, stage, v);                      \
        __syncwarp();                                             \
        if (lane == 0) mbar_arrive(empty);                        \
        if (k.pass & 1) col_compute<N, E>(c, k, v, exch, tw);     \
        else row_compute<N, E>(c, k, v, exch, tw);                \
      }                                                           \
    }
    WAP_SCHED_CASE(128, 1u)
    WAP_SCHED_CASE(256, 2u)
    WAP_SCHED_CASE(512, 4u)
    WAP_SCHED_CASE(1024, 8u)
#undef WAP_SCHED_CASE
    __syncwarp();
    if (lane == 0) mbar_arrive(done_bar + (tiles_done & 1));
    ++tiles_done;
  }
}

// ---------------------------------------------------------------------------
// the persistent kernel: 8 compute warps + 1 producer warp
// ---------------------------------------------------------------------------
template <unsigned MASK, int E>
__global__ void __launch_bounds__(kBlockThreads, E == 16 ? 3 : 4) scan_kernel(const __grid_constant__ SchedParams P) {
  extern __shared__ __align__(1024) unsigned char sched_smem[];
  float2* stage = reinterpret_cast<float2*>(sched_smem);
  constexpr int kTile = kTileBytesFor(E), kExch = kExchBytesFor(E);
  float2* exch = reinterpret_cast<float2*>(sched_smem + kTile);
  float4* tw_smem = reinterpret_cast<float4*>(sched_smem + kTile + kExch);
  __shared__ __align__(8) uint64_t full, empty, done_bar[2];
  __shared__ Task s_task;

  if (P.tw_in_smem) {
    for (int ci = 0; ci < P.n_classes; ++ci) {
      const SchedClass& c = P.cls[ci];
      for (int i = threadIdx.x; i < c.tw_len; i += blockDim.x) tw_smem[c.tw_off + i] = c.tw[i];
    }
  }
  if (threadIdx.x == 0) {
    mbar_init(&full, 1);
    mbar_init(&empty, kComputeWarps);
    mbar_init(&done_bar[0], kComputeWarps);
    mbar_init(&done_bar[1], kComputeWarps);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();

  if (threadIdx.x < kSchedThreads) {
    compute_loop<MASK, E>(P, stage, exch, tw_smem, &full, &empty, done_bar, &s_task);
    return;
  }

  // ---------------- producer warp (lane 0 does the work) ----------------
  const int lane = threadIdx.x & 31;
  if (lane != 0) return;
  int cursor = 0;
  auto claim = [&]() -> Task {
    Task out;
    out.valid = 0;
    out.cls = out.pass = out.b = out.tile = 0;
    if (*(volatile int*)P.status != 0) return out;
    const unsigned long long tk = atomicAdd(P.ticket, 1ULL);
    if ((long long)tk >= P.total) return out;
    while (cursor + 1 < P.n_desc && P.desc[cursor + 1].base <= (long long)tk) ++cursor;
    const SchedDesc d = P.desc[cursor];
    const long long local = (long long)tk - d.base;
    out.cls = d.cls;
    out.pass = d.pass;
    out.b = d.b0 + (int)(local / d.tiles);
    out.tile = (int)(local % d.tiles);
    out.valid = 1;
    return out;
  };
  auto need_of = [&](const Task& k) -> int {
    return k.pass == P.stall_pass ? 0x7fffffff : tiles_before(P.cls[k.cls], k.pass);
  };
  auto counter_of = [&](const Task& k) -> const int* { return P.done + P.cls[k.cls].done_off + k.b; };
  // Block until the task's inputs are complete (bounded).  Only called while
  // this CTA holds no unsignalled tile, so every task waited on has a smaller
  // ticket owned by a CTA that can finish it.
  auto wait_ready = [&](const Task& k) -> bool {
    const int need = need_of(k);
    const int* cnt = counter_of(k);
    long long spins = 0;
    unsigned ns = 32;
    while (ld_acquire(cnt) < need) {
      if (++spins > P.spin_limit || *(volatile int*)P.status != 0) {
        atomicCAS(P.status, 0, WAP_ERR_TIMEOUT);
        return false;
      }
      __nanosleep(ns);
      if (ns < 1024) ns <<= 1;
    }
    fence_proxy_async();
    return true;
  };
  auto tile_bytes = [&](const Task& k) -> uint32_t {
    const SchedClass& c = P.cls[k.cls];
    if (k.pass == 0) return 0;
    return (k.pass & 1) ? (uint32_t)(c.n * c.cols_w * 8) : (uint32_t)(c.rows * c.n * 8);
  };
  // publish a task (or the stop sentinel) to the compute warps
  auto publish = [&](const Task& k0) {
    Task k = k0;
    if (k.valid && !task_ok(P, k, 2)) k.valid = 0;
    s_task = k;
    // exactly one arrival per phase on `full` (count 1): issue_load's
    // arrive.expect_tx for tiles with a TMA load, a plain arrive otherwise
    const uint32_t bytes = k.valid ? tile_bytes(k) : 0;
    if (bytes) {
      issue_load(P, k, stage, &full);
    } else {
      mbar_arrive(&full);
    }
  };
  auto fail_wait = [&]() { atomicCAS(P.status, 0, WAP_ERR_TIMEOUT); };

  uint32_t eph = 0, dph[2] = {0, 0};
  uint32_t tiles_signalled = 0;
  uint32_t fph = 0;            // parity of the next full-barrier phase to complete
  bool load_out = false;       // the latest published item carried a TMA load
  auto publish_track = [&](const Task& kk) {
    load_out = kk.valid && tile_bytes(kk) != 0;
    publish(kk);
    fph ^= 1u;
  };
  Task k = claim();
  if (k.valid && !wait_ready(k)) k.valid = 0;
  publish_track(k);
  while (k.valid) {
    Task kn = claim();
    bool issued = false;
    if (kn.valid && ld_acquire(counter_of(kn)) >= need_of(kn)) {
      // inputs ready: stream the next tile in as soon as the stage is free
      if (!mbar_wait(&empty, eph, P.spin_limit)) fail_wait();
      eph ^= 1u;
      fence_proxy_async();
      publish_track(kn);
      issued = true;
    }
    // completion of k: every compute warp has stored its part.  The compute
    // warps may already have finished the prefetched tile too, so tiles
    // alternate between two barriers (a parity wait never sees two phases).
    {
      const int q = tiles_signalled & 1;
      if (!mbar_wait(&done_bar[q], dph[q], P.spin_limit)) fail_wait();
      dph[q] ^= 1u;
      ++tiles_signalled;
    }
    __threadfence();
    atomicAdd(P.done + P.cls[k.cls].done_off + k.b, 1);
    if (!issued) {
      // holding nothing unsignalled now: safe to block on kn's inputs
      if (kn.valid && !wait_ready(kn)) kn.valid = 0;
      if (!mbar_wait(&empty, eph, P.spin_limit)) fail_wait();
      eph ^= 1u;
      publish_track(kn);   // kn or the stop sentinel
    }
    k = kn;
  }
  // After an error the compute warps may have stopped without consuming the
  // last published tile: let its copy land (bounded) before the CTA exits.
  if (load_out && *(volatile int*)P.status != 0) mbar_wait(&full, fph ^ 1u, P.spin_limit);
}

}  // namespace wap

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
using namespace wap;

typedef void (*ScanKernel)(const SchedParams);

// kernel instances by elements per thread and the set of grid sizes they
// contain (bit 0: 128, 1: 256, 2: 512, 3: 1024); other sets use the
// all-sizes instance
template <int E>
static ScanKernel pick_scan_kernel_e(unsigned mask) {
  switch (mask) {
    case 1u: return scan_kernel<1u, E>;
    case 2u: return scan_kernel<2u, E>;
    case 4u: return scan_kernel<4u, E>;
    case 8u: return scan_kernel<8u, E>;
    case 6u: return scan_kernel<6u, E>;
    default: return scan_kernel<15u, E>;
  }
}
static ScanKernel pick_scan_kernel(unsigned mask, int e) {
  return e == 8 ? pick_scan_kernel_e<8>(mask) : pick_scan_kernel_e<16>(mask);
}

struct wap_scan {
  ScanKernel kernel = nullptr;
  int e = 16;
  int device = 0;
  int n_classes = 0;
  SchedParams params{};
  SchedDesc* d_desc = nullptr;
  unsigned long long* d_ticket = nullptr;
  int* d_done = nullptr;
  int* d_status = nullptr;
  int* d_debug = nullptr;
  int total_probes = 0;
  int grid = 0;
  size_t smem = 0;
  std::vector<float4*> d_tw;
  std::vector<float2*> d_ttab;
  std::vector<float4*> d_hq;
  std::vector<size_t> ttab_elems;
  std::vector<wap_scan_class> cls;
  std::vector<Physics> phys;
  long long n_tickets = 0;
};

static PFN_cuTensorMapEncodeTiled_v12000 get_encode() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }
  return fn;
}

static void scan_free(wap_scan* s) {
  if (!s) return;
  cudaFree(s->d_desc);
  cudaFree(s->d_ticket);
  cudaFree(s->d_done);
  cudaFree(s->d_status);
  cudaFree(s->d_debug);
  for (auto p : s->d_tw) cudaFree(p);
  for (auto p : s->d_ttab) cudaFree(p);
  for (auto p : s->d_hq) cudaFree(p);
  delete s;
}

static bool sched_size_ok(int n) { return n == 128 || n == 256 || n == 512 || n == 1024; }

extern "C" {

int wap_scan_create(wap_scan** out, int n_classes, const wap_scan_class* classes) {
  clear_error();
  if (!out) return fail(WAP_ERR_ARG, "scan pointer is NULL");
  *out = nullptr;
  if (n_classes < 1 || n_classes > kMaxClasses || !classes)
    return fail(WAP_ERR_ARG, "n_classes must be in [1, %d]", kMaxClasses);
  PFN_cuTensorMapEncodeTiled_v12000 encode = get_encode();
  if (!encode) return fail(WAP_ERR_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
  wap_scan* s = new wap_scan();
  cudaGetDevice(&s->device);
  s->n_classes = n_classes;
  s->cls.assign(classes, classes + n_classes);
  cudaError_t e;
  int sms = 0, per_sm = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, s->device);
  // elements per thread of the scheduler's transforms
  int E = 16;
  if (const char* ov = getenv("WAP_SCHED_E")) {   // debugging / A-B timing only
    if (!strcmp(ov, "8")) E = 8;
  }
  s->e = E;
  unsigned mask = 0;
  int tw_total = 0;
  for (int ci = 0; ci < n_classes; ++ci) {
    const int n = classes[ci].n;
    if (!sched_size_ok(n)) {
      scan_free(s);
      return fail(WAP_ERR_UNSUPPORTED, "scan grids must be 128, 256, 512 or 1024 (got %d)", n);
    }
    mask |= n == 128 ? 1u : n == 256 ? 2u : n == 512 ? 4u : 8u;
    tw_total += make_plan_shape(n, E).tw_size();
  }
  s->kernel = pick_scan_kernel(mask, E);
  // Keep the twiddles in shared memory only when they fit next to the stage
  // and exchange buffers without lowering the CTAs per SM (3 for E = 16,
  // 4 for E = 8).
  const size_t base_smem = kTileBytesFor(E) + kExchBytesFor(E);
  const int want_ctas = E == 16 ? 3 : 4;
  s->params.tw_in_smem = want_ctas * (base_smem + (size_t)tw_total * sizeof(float4) + 1024) <= 227 * 1024;
  if (const char* ov = getenv("WAP_SCHED_TWIDDLES")) {   // debugging / A-B timing only
    if (!strcmp(ov, "smem")) s->params.tw_in_smem = 1;
    if (!strcmp(ov, "global")) s->params.tw_in_smem = 0;
  }
  s->smem = base_smem + (s->params.tw_in_smem ? (size_t)tw_total * sizeof(float4) : 0);
  if ((e = cudaFuncSetAttribute(s->kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)s->smem)) != cudaSuccess) {
    scan_free(s);
    return cuda_fail(e, "cudaFuncSetAttribute(scan_kernel)");
  }
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, s->kernel, kBlockThreads, s->smem);
  if (per_sm < 1) {
    scan_free(s);
    return fail(WAP_ERR_CUDA, "scan_kernel does not fit on an SM");
  }
  s->grid = sms * per_sm;
  int tw_off = 0;

  std::vector<SchedDesc> desc;
  long long ticket = 0;
  int done_off = 0;
  for (int ci = 0; ci < n_classes; ++ci) {
    const wap_scan_class& c = classes[ci];
    if (c.n_slices < 1 || c.n_draws < 1 || c.n_probes < 1 || !c.V || !c.psi0 || !c.H || !c.exit) {
      scan_free(s);
      return fail(WAP_ERR_ARG, "scan class %d: bad sizes or NULL V/psi0/H/exit", ci);
    }
    const int n = c.n, T = n / E;
    SchedClass& sc = s->params.cls[ci];
    sc.n = n;
    sc.log2n = ilog2c(n);
    sc.n_slices = c.n_slices;
    sc.n_probes = c.n_probes;
    sc.rows = kSchedThreads / T;
    sc.cols_w = kSchedThreads / T;
    sc.row_tiles = n / sc.rows;
    sc.col_tiles = n / sc.cols_w;
    sc.box_rows = std::min(n, 256);
    sc.done_off = done_off;
    sc.psi = reinterpret_cast<float2*>(c.exit);
    sc.psi0 = reinterpret_cast<const float2*>(c.psi0);
    sc.positions = c.positions;
    sc.draw = c.draw;
    float4* dhq = nullptr;
    if ((e = cudaMalloc(&dhq, (size_t)n * n * sizeof(float4))) != cudaSuccess) {
      scan_free(s);
      return cuda_fail(e, "cudaMalloc(interleaved H)");
    }
    s->d_hq.push_back(dhq);
    sc.Hq = dhq;
    sc.dp = c.dp;
    sc.scale = (float)(1.0 / ((double)n * n));
    sc.inv_scale = (float)((double)n * n);
    sc.ttab_draw_stride = (long long)c.n_slices * n * n;
    // twiddles
    std::vector<float4> h = twiddle_table(n, E);
    float4* dtw = nullptr;
    if ((e = cudaMalloc(&dtw, h.size() * sizeof(float4))) != cudaSuccess ||
        (e = cudaMemcpy(dtw, h.data(), h.size() * sizeof(float4), cudaMemcpyHostToDevice)) != cudaSuccess) {
      cudaFree(dtw);
      scan_free(s);
      return cuda_fail(e, "twiddle upload");
    }
    s->d_tw.push_back(dtw);
    sc.tw = dtw;
    sc.tw_off = tw_off;
    sc.tw_len = (int)h.size();
    tw_off += sc.tw_len;
    // transmission table
    const size_t tt = (size_t)c.n_draws * c.n_slices * n * n;
    float2* dtt = nullptr;
    if ((e = cudaMalloc(&dtt, tt * sizeof(float2))) != cudaSuccess) {
      scan_free(s);
      return cuda_fail(e, "cudaMalloc(transmission table)");
    }
    s->d_ttab.push_back(dtt);
    s->ttab_elems.push_back(tt);
    sc.ttab = dtt;
    s->phys.push_back(physics(c.energy, c.dz));
    // column-tile tensor map: 2D (n columns x B n rows) of 8-byte elements
    cuuint64_t gdim[2] = {(cuuint64_t)n, (cuuint64_t)c.n_probes * n};
    cuuint64_t gstride[1] = {(cuuint64_t)n * 8};
    cuuint32_t box[2] = {(cuuint32_t)sc.cols_w, (cuuint32_t)sc.box_rows};
    cuuint32_t estride[2] = {1, 1};
    CUresult r = encode(&s->params.maps[ci], CU_TENSOR_MAP_DATA_TYPE_INT64, 2, c.exit, gdim, gstride, box, estride,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                        CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
      scan_free(s);
      return fail(WAP_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d) for class %d", (int)r, ci);
    }
    // pass descriptors: groups of G probes walk through all passes
    int G = c.group;
    if (G <= 0) {
      // enough tiles per pass to cover the resident CTAs twice, and a group
      // footprint of ~32 MB so that the group's waves stay in L2
      const int tiles = sc.row_tiles;
      G = std::max(1, (2 * s->grid + tiles - 1) / tiles);
      const int l2_cap = std::max(1, (int)((32ll << 20) / ((long long)n * n * 8)));
      G = std::min(std::max(G, 1), std::max(l2_cap, 1));
    }
    G = std::min(G, c.n_probes);
    for (int b0 = 0; b0 < c.n_probes; b0 += G) {
      const int nb = std::min(G, c.n_probes - b0);
      for (int p = 0; p <= 2 * c.n_slices; ++p) {
        SchedDesc d;
        d.base = ticket;
        d.cls = ci;
        d.pass = p;
        d.b0 = b0;
        d.nprobes = nb;
        d.tiles = (p & 1) ? sc.col_tiles : sc.row_tiles;
        desc.push_back(d);
        ticket += (long long)nb * d.tiles;
      }
    }
    done_off += c.n_probes;
  }
  s->n_tickets = ticket;
  s->total_probes = done_off;
  if ((e = cudaMalloc(&s->d_desc, desc.size() * sizeof(SchedDesc))) != cudaSuccess ||
      (e = cudaMemcpy(s->d_desc, desc.data(), desc.size() * sizeof(SchedDesc), cudaMemcpyHostToDevice)) != cudaSuccess ||
      (e = cudaMalloc(&s->d_ticket, sizeof(unsigned long long))) != cudaSuccess ||
      (e = cudaMalloc(&s->d_done, (size_t)done_off * sizeof(int))) != cudaSuccess ||
      (e = cudaMalloc(&s->d_status, sizeof(int))) != cudaSuccess) {
    scan_free(s);
    return cuda_fail(e, "scan allocation");
  }
  cudaMemset(s->d_status, 0, sizeof(int));
  s->params.desc = s->d_desc;
  s->params.n_desc = (int)desc.size();
  s->params.n_classes = n_classes;
  s->params.total = ticket;
  s->params.ticket = s->d_ticket;
  s->params.done = s->d_done;
  s->params.status = s->d_status;
  s->params.spin_limit = kSpinLimit;
  s->params.stall_pass = -1;
  s->params.checks = 0;
  if ((e = cudaMalloc(&s->d_debug, 8 * sizeof(int))) != cudaSuccess) {
    scan_free(s);
    return cuda_fail(e, "scan allocation");
  }
  cudaMemset(s->d_debug, 0, 8 * sizeof(int));
  s->params.debug = s->d_debug;
  *out = s;
  return WAP_OK;
}

int wap_scan_run(wap_scan* s, void* stream) {
  clear_error();
  if (!s) return fail(WAP_ERR_ARG, "scan is NULL");
  cudaStream_t st = (cudaStream_t)stream;
  cudaError_t e;
  if ((e = cudaMemsetAsync(s->d_ticket, 0, sizeof(unsigned long long), st)) != cudaSuccess ||
      (e = cudaMemsetAsync(s->d_done, 0, (size_t)s->total_probes * sizeof(int), st)) != cudaSuccess ||
      (e = cudaMemsetAsync(s->d_status, 0, sizeof(int), st)) != cudaSuccess)
    return cuda_fail(e, "scan reset");
  for (int ci = 0; ci < s->n_classes; ++ci) {
    const Physics& ph = s->phys[ci];
    const long long n4 = (long long)s->ttab_elems[ci] / 4;
    const ProfToken tok = prof_begin(WAP_KIND_TRANS, st);
    count_launch();
    trans_table_kernel<<<(unsigned)std::min<long long>((n4 + 255) / 256, 148LL * 16), 256, 0, st>>>(
        s->cls[ci].V, s->d_ttab[ci], n4, (float)ph.ri_a, (float)ph.ri_inv_den, (float)ph.kphase,
        s->params.cls[ci].scale);
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "trans_table_kernel");
    prof_end(tok, st, 12.0 * (double)s->ttab_elems[ci]);
    const long long nn = (long long)s->cls[ci].n * s->cls[ci].n;
    count_launch();
    interleave_h_kernel<<<(unsigned)std::min<long long>((nn + 255) / 256, 148LL * 8), 256, 0, st>>>(
        reinterpret_cast<const float2*>(s->cls[ci].H), reinterpret_cast<const float2*>(s->cls[ci].H_lo),
        s->d_hq[ci], nn);
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "interleave_h_kernel");
  }
  // algorithmic bytes of a slice step: wave in 8 + wave out 8 + potential 4
  // per pixel (the two passes' intermediate round trip is not counted)
  double bytes = 0;
  for (int ci = 0; ci < s->n_classes; ++ci) {
    const wap_scan_class& c = s->cls[ci];
    bytes += (double)c.n_probes * c.n_slices * c.n * c.n * 20.0;
  }
  const ProfToken tok = prof_begin(WAP_KIND_SCHED, st);
  count_launch();
  s->kernel<<<s->grid, kBlockThreads, s->smem, st>>>(s->params);
  if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "scan_kernel");
  prof_end(tok, st, bytes);
  return WAP_OK;
}

int wap_scan_status(wap_scan* s, int* status) {
  clear_error();
  if (!s || !status) return fail(WAP_ERR_ARG, "NULL argument");
  int h = 0;
  cudaError_t e = cudaMemcpy(&h, s->d_status, sizeof(int), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_fail(e, "scan status");
  *status = h;
  if (h != 0) return fail(h, "scan kernel reported status %d (a bounded wait expired)", h);
  return WAP_OK;
}

int wap_scan_info(const wap_scan* s, long long* tickets, int* grid, int* group0) {
  clear_error();
  if (!s || !tickets || !grid || !group0) return fail(WAP_ERR_ARG, "NULL argument");
  *tickets = s->n_tickets;
  *grid = s->grid;
  *group0 = 0;
  return WAP_OK;
}

int wap_scan_debug_stall(wap_scan* s, int pass, long long spin_limit) {
  clear_error();
  if (!s) return fail(WAP_ERR_ARG, "scan is NULL");
  s->params.stall_pass = pass;
  s->params.spin_limit = spin_limit > 0 ? spin_limit : kSpinLimit;
  return WAP_OK;
}

int wap_scan_debug_checks(wap_scan* s, int on, int* record) {
  clear_error();
  if (!s) return fail(WAP_ERR_ARG, "scan is NULL");
  s->params.checks = on;
  if (record) {
    cudaError_t e = cudaMemcpy(record, s->d_debug, 6 * sizeof(int), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(e, "scan debug record");
  }
  return WAP_OK;
}

int wap_scan_destroy(wap_scan* s) {
  clear_error();
  scan_free(s);
  return WAP_OK;
}

}  // extern "C"
