// Persistent batched multislice scheduler (Fresnel / angular spectrum), and
// the same machinery for the adjoint (gradient w.r.t. the potential).
//
// One launch advances every probe of every grid class of a scan through a
// per-probe chain of steps.  Each step is one pass over one probe's wave,
// split into tiles: row tiles (ROWS consecutive rows) or column tiles (n rows
// x W columns).  Forward chain (propagation.py:305-352), N slices:
//
//   FWD_ROW0   s = 0   psi0 rolled to the probe position (move_probe,
//                      propagation.py:263-276) -> * t_0 -> row FFT
//   FWD_ROW    s       inverse row FFT of slice s-1 -> * t_s -> row FFT
//   FWD_COL    s       column FFT -> * H (hi + lo) -> [dp = |.|^2 on the last
//                      slice] -> inverse column FFT
//   FWD_ROWN           inverse row FFT -> exit wave
//
// (t_s from a table shared by the probes of a potential draw.)  The gradient
// uses a forward that also stores the wave entering every k-th slice and the
// whole last k-slice segment, then a backward chain
//
//   SEED_ROW, SEED_COL          lambda = ifft2(conj(H) n^2 g fft2(exit))
//   per segment j (last first):
//     REC_ROW0, REC_COL, REC_ROW, ..., REC_ROWL   recompute psi_s of the
//                                                 segment from its checkpoint
//                                                 (skipped for the last one)
//     ADJ_ROW(s), ADJ_COL(s) for s = s1-1 .. s0   adjoint sweep: lambda_a =
//       ifft2 of the column output; dL/dV_s += 2 Re(conj(lambda_a) i t psi_s)
//       dphi/dV; lambda <- conj(t) lambda_a, row FFT; column FFT, * conj(H),
//       inverse column FFT.
//
// The work is a ticket queue: the host lays out descriptors (class, probe
// group, step), each expanding into probes x tiles tickets; a producer warp
// per CTA claims tickets in increasing order with one atomicAdd.  A tile of
// step p needs every tile of steps 0..p-1 of the same probe, i.e. a per-probe
// completion counter >= the prefix tile count of step p.  Tickets are ordered
// (class, group, step, probe, tile), so a tile only ever waits for smaller
// tickets, claimed by CTAs that are running or finished; a CTA never blocks
// while it holds an unsignalled tile, so the queue cannot deadlock.  Waits are
// bounded; on expiry the CTA records WAP_ERR_TIMEOUT, CTAs stop claiming,
// in-flight copies are drained (bounded) and the kernel returns.
//
// Probe groups are sized so that a group's waves stay L2-resident while the
// group walks through its chain; groups follow each other without a barrier.
//
// Tile loads use the Tensor Memory Accelerator: row tiles are contiguous (one
// cp.async.bulk), column tiles are 2D boxes of a tensor map over all probes'
// rows of a buffer (cp.async.bulk.tensor.2d, no multicast).  The producer warp
// issues the load of the next ticket as soon as the compute warps have pulled
// the current tile into registers, so loads overlap the transforms.
#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <type_traits>
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

enum StepType : int {
  ST_FWD_ROW0 = 0,
  ST_FWD_ROW,
  ST_FWD_ROWN,
  ST_FWD_COL,
  ST_SEED_ROW,
  ST_SEED_COL,
  ST_REC_ROW0,
  ST_REC_ROW,
  ST_REC_ROWL,
  ST_REC_COL,
  ST_ADJ_ROW,
  ST_ADJ_ROW0,
  ST_ADJ_COL,
};

__host__ __device__ constexpr bool step_is_col(int t) {
  return t == ST_FWD_COL || t == ST_SEED_COL || t == ST_REC_COL || t == ST_ADJ_COL;
}

// buffers a column tile reads: tensor-map index
enum BufferId : int { BUF_PSI = 0, BUF_LAM = 1, BUF_WORK = 2, BUF_COUNT = 3 };

struct Step {
  int type;
  int slice;
  int seg0;       // first slice of the step's checkpoint segment
  int ckpt_slot;  // forward rows: checkpoint slot written (-1: none); REC_ROW0 and the
                  // ADJ row of a segment's first slice: checkpoint slot read
  int seg_slot;   // forward/recompute rows: segment slot written; other ADJ rows: slot read
  int prefix;     // tiles of all earlier steps of the probe
};

struct SchedClass {
  int n, log2n, n_slices, n_probes;
  int rows, cols_w;             // row-tile height, column-tile width
  int row_tiles, col_tiles;     // tiles per probe per step
  int box_rows;                 // TMA box height for column tiles (<= 256)
  int done_off;                 // offset of this class's counters
  const Step* steps;            // the per-probe chain
  float2* psi;                  // (B, n, n) working buffer / exit
  const float2* psi0;           // (n, n) shared probe
  const int* positions;         // (B, 2) or null
  const int* draw;              // (B) or null
  const float* V;               // (draws, N, n, n) volts (adjoint only)
  const float2* ttab;           // (draws, N, n, n)  t / (n n)
  long long vstride;            // N n n (draw stride of V, ttab, grad)
  const float4* Hq;             // (n, n) interleaved (H_hi, H_lo)
  float* dp;                    // (B, n, n) or null (a windowed class: the scan's full-grid scratch)
  // gradient buffers
  float2* lam;                  // (B, n, n) adjoint state
  float2* work;                 // (B, n, n) recompute buffer
  float2* seg;                  // (B, k, n, n) waves of the current segment
  float2* ckpt;                 // (B, nck, n, n) checkpoints
  int ckpt_n, seg_n;            // slots per probe
  int ckpt_k;                   // gradient scans: checkpoint every ckpt_k slices (0: none)
  int seg_first;                // first slice of the trailing segments the forward keeps
  const float* g;               // (B, n, n) dL/d(dp), fftshifted like dp (full grid; zeros for an exit-only loss)
  const float2* seed_add;       // (B, n, n) spectrum added to the seed (exit-wave loss), or null
  float* grad;                  // (draws, N, n, n) probe sums of Re(conj(lambda_a) i a_s)
  float ri_a, ri_inv_den, kphase, e_plus_e0;
  const float4* tw;             // twiddles for (n, E) in global memory
  int tw_off, tw_len;           // their place in the shared-memory image
  float scale;                  // 1 / (n n)  (also folded into ttab)
  float inv_scale;              // n n
};

// Where adjoint rows read psi_s (the wave entering the slice) from:
constexpr int kPsiGlobal = 0;   // global loads inside the tile body
constexpr int kPsiStage2 = 1;   // a second staging buffer, loaded with lambda
constexpr int kPsiSplit = 2;    // the one stage, refilled once lambda is in registers

struct SchedDesc {
  long long base;   // first ticket
  int cls, pass, b0, nprobes, tiles;
};

struct alignas(64) SchedParams {
  CUtensorMap maps[kMaxClasses][BUF_COUNT];   // column-tile tensor maps
  SchedClass cls[kMaxClasses];
  const SchedDesc* desc;
  int n_desc;
  int n_classes;
  long long total;                 // number of tickets
  unsigned long long* ticket;      // claim counter
  int* done;                       // per-probe completed tiles
  int* status;                     // 0 or WAP_ERR_TIMEOUT
  long long spin_limit;            // polls before a wait gives up
  int stall_pass;                  // test hook: tiles of this step wait forever (-1: off)
  int checks;                      // validate every task before use (debug)
  int tw_in_smem;                  // twiddles copied to shared memory (else read via L1)
  const float4* tw_image;          // the shared-memory twiddle image of all classes
  int tw_image_len;                // its entries
  int stage2;                      // how adjoint rows get psi_s: kPsiGlobal / kPsiStage2 / kPsiSplit
  int* debug;                      // [code, cls, step, b, tile, extra] of the first bad task
  unsigned suspend_ns;             // mbarrier wait suspend-time hint (0: none)
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
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
// try_wait with a suspend-time hint (ns; 0: none): a waiting warp may sleep
// until the phase completes or the hint elapses instead of re-issuing the test
// (measured on the headline scan: 0, 200, 1000 and 4000 ns within 0.2 %)
constexpr uint32_t kMbarSuspendNs = 0;
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t phase, uint32_t hint_ns) {
  uint32_t ok;
  if (hint_ns) {
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(phase), "r"(hint_ns)
        : "memory");
  } else {
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(phase)
        : "memory");
  }
  return ok != 0;
}
// bounded mbarrier wait; false if the limit expired
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t phase, long long limit, uint32_t hint_ns) {
  long long spins = 0;
  while (!mbar_try_wait(bar, phase, hint_ns)) {
    if (++spins > limit) return false;
  }
  return true;
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
// tasks
// ---------------------------------------------------------------------------
struct Task {
  int cls, pass, b, tile, valid;
};

// Step of the plain forward chain, decoded from the pass index alone: rows on
// even passes (first one loads the probe, last one finishes the exit wave),
// columns on odd passes.
__device__ __forceinline__ Step forward_step(const SchedClass& c, int pass) {
  Step st;
  st.slice = pass >> 1;
  st.type = (pass & 1) ? ST_FWD_COL : pass == 0 ? ST_FWD_ROW0 : pass == 2 * c.n_slices ? ST_FWD_ROWN : ST_FWD_ROW;
  st.seg0 = 0;
  st.ckpt_slot = -1;
  st.seg_slot = -1;
  if (c.ckpt_k > 0 && !(pass & 1) && st.slice < c.n_slices) {
    // gradient scans: checkpoints every ckpt_k slices, the last segment whole
    if (st.slice % c.ckpt_k == 0) st.ckpt_slot = st.slice / c.ckpt_k;
    if (st.slice > c.seg_first) st.seg_slot = st.slice - c.seg_first;   // seg_first: its checkpoint
  }
  st.prefix = ((pass + 1) >> 1) * c.row_tiles + (pass >> 1) * c.col_tiles;
  return st;
}

template <bool GRAD>
__device__ __forceinline__ Step step_of(const SchedClass& c, int pass) {
  if constexpr (GRAD) return c.steps[pass];
  else return forward_step(c, pass);
}

// Debug validation of a decoded task (P.checks): record the first violation
// and report whether the task may be used.
template <bool GRAD>
__device__ __forceinline__ bool task_ok(const SchedParams& P, const Task& k, int where) {
  if (!(P.checks & 1)) return true;
  bool ok = k.cls >= 0 && k.cls < P.n_classes;
  if (ok) {
    const SchedClass& c = P.cls[k.cls];
    const int type = step_of<GRAD>(c, k.pass).type;
    ok = k.b >= 0 && k.b < c.n_probes && k.pass >= 0 && k.tile >= 0 &&
         k.tile < (step_is_col(type) ? c.col_tiles : c.row_tiles);
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

__device__ __forceinline__ uint32_t tile_bytes(const SchedClass& c, int type) {
  if (type == ST_FWD_ROW0) return 0;   // loaded directly (rolled probe)
  return step_is_col(type) ? (uint32_t)(c.n * c.cols_w * 8) : (uint32_t)(c.rows * c.n * 8);
}

// psi_s of an adjoint row (whole plane of probe b): the checkpoint for a
// segment's first slice, else the segment buffer
__device__ __forceinline__ const float2* adj_psi(const SchedClass& c, const Step& st, int b) {
  const long long plane = (long long)c.n * c.n;
  return st.ckpt_slot >= 0 ? c.ckpt + ((long long)b * c.ckpt_n + st.ckpt_slot) * plane
                           : c.seg + ((long long)b * c.seg_n + st.seg_slot) * plane;
}

// Issue the TMA load of a task's input tile into `stage` (one thread).  This
// is the single arrival of the phase on `bar`: arrive.expect_tx(tile bytes),
// completed by the copy.  Not called for tasks that load directly.
template <bool GRAD>
__device__ __forceinline__ void issue_load(const SchedParams& P, const Task& k, float2* stage, uint64_t* bar) {
  const SchedClass& c = P.cls[k.cls];
  const Step st = step_of<GRAD>(c, k.pass);
  const long long plane = (long long)c.n * c.n;
  const uint32_t bytes = tile_bytes(c, st.type);
  if (GRAD && P.stage2 == kPsiStage2 && (st.type == ST_ADJ_ROW || st.type == ST_ADJ_ROW0)) {
    // lambda rows into the stage, the same rows of psi_s into the second stage
    mbar_expect_tx(bar, 2 * bytes);
    const long long roff = (long long)k.tile * c.rows * c.n;
    bulk_g2s(stage, c.lam + (long long)k.b * plane + roff, bytes, bar);
    bulk_g2s(stage + bytes / sizeof(float2), adj_psi(c, st, k.b) + roff, bytes, bar);
    return;
  }
  mbar_expect_tx(bar, bytes);
  if (!step_is_col(st.type)) {
    const float2* base;
    switch (st.type) {
      case ST_REC_ROW0: base = c.ckpt + ((long long)k.b * c.ckpt_n + st.ckpt_slot) * plane; break;
      case ST_REC_ROW:
      case ST_REC_ROWL: base = c.work + (long long)k.b * plane; break;
      case ST_ADJ_ROW:
      case ST_ADJ_ROW0: base = c.lam + (long long)k.b * plane; break;
      default: base = c.psi + (long long)k.b * plane; break;   // FWD_ROW, FWD_ROWN, SEED_ROW
    }
    bulk_g2s(stage, base + (long long)k.tile * c.rows * c.n, bytes, bar);
  } else {
    const int buf = st.type == ST_FWD_COL ? BUF_PSI : st.type == ST_REC_COL ? BUF_WORK : BUF_LAM;
    for (int r0 = 0; r0 < c.n; r0 += c.box_rows)
      tma_load_2d(stage + r0 * c.cols_w, &P.maps[k.cls][buf], k.tile * c.cols_w, k.b * c.n + r0, bar);
  }
}

constexpr int kComputeWarps = kSchedThreads / 32;      // 8 compute warps
constexpr int kBlockThreads = kSchedThreads + 32;       // + 1 producer warp
// forward scans of at most this many slices use hi-only stage twiddles
constexpr int kHiTwiddleMaxSlices = 160;
constexpr int kFftBar = 2;                              // named barrier of the compute warps

// ---------------------------------------------------------------------------
// tile bodies
// ---------------------------------------------------------------------------
// Row tile, phase 1: this thread's E input words into registers.
template <int N, int E>
__device__ __forceinline__ void row_load(const SchedClass& c, const Task& k, int type, const float2* stage,
                                         float2 (&v)[E]) {
  constexpr int T = N / E;
  const int rl = threadIdx.x / T, t = threadIdx.x - rl * T;
  if (type == ST_FWD_ROW0) {
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

// Row tile, phase 2.  ttab holds t / (n n): the inverse transform's
// normalisation rides on the transmission multiply; steps without an inverse
// transform undo it, steps without a transmission apply it.  All these factors
// are powers of two, so no rounding changes.  The forward instance (!GRAD)
// runs the forward chain - with checkpoint / segment snapshots in gradient
// scans - and the gradient instance runs the backward chain.
template <int N, int E, bool GRAD, class TW, class Acquire, class Release>
__device__ __forceinline__ void row_compute(const SchedClass& c, const Task& k, const Step& st, float2 (&v)[E],
                                            float2* exch, const TW* tw, const float2* stage2,
                                            const Acquire& acquire, const Release& release) {
  constexpr int T = N / E;
  constexpr int PADN = RowExchange<true>::padded(N);
  const int rl = threadIdx.x / T, t = threadIdx.x - rl * T;
  const int row = k.tile * c.rows + rl;
  const long long plane = (long long)N * N;
  const RowExchange<(T <= 32), kFftBar, kSchedThreads> xs{exch + rl * PADN};
  const int type = st.type;
  // offset of this row in V / ttab / grad; evaluated after the inverse
  // transform so that it is not live across it
  auto row_off = [&]() -> long long {
    const int d = c.draw ? c.draw[k.b] : 0;
    return (long long)d * c.vstride + (long long)st.slice * plane + (long long)row * N;
  };
  // normalised wave entering slice st.slice into a snapshot slot
  auto snapshot = [&](float2* base, int slot, int slots, bool unnormalised) {
    float2* sp = base + ((long long)k.b * slots + slot) * plane + (long long)row * N;
    const float sc = unnormalised ? c.scale : 1.0f;
#pragma unroll
    for (int e = 0; e < E; ++e) __stcg(sp + t + T * e, cscale(v[e], sc));
  };

  if constexpr (!GRAD) {
    // forward: [inverse row FFT], then * t and row FFT, or the exit wave
    if (type != ST_FWD_ROW0) fft<N, E, true>(v, t, xs, tw);
    float2* prow = c.psi + (long long)k.b * plane + (long long)row * N;
    if (type == ST_FWD_ROWN) {
#pragma unroll
      for (int e = 0; e < E; ++e) __stcg(prow + t + T * e, cscale(v[e], c.scale));
      return;
    }
    if (st.ckpt_slot >= 0) snapshot(c.ckpt, st.ckpt_slot, c.ckpt_n, type != ST_FWD_ROW0);
    if (st.seg_slot >= 0) snapshot(c.seg, st.seg_slot, c.seg_n, type != ST_FWD_ROW0);
    if (type == ST_FWD_ROW0) {
#pragma unroll
      for (int e = 0; e < E; ++e) v[e] = cscale(v[e], c.inv_scale);
    }
    const float2* trow = c.ttab + row_off();
#pragma unroll
    for (int e = 0; e < E; ++e) v[e] = cmul(v[e], __ldg(trow + t + T * e));
    fft<N, E, false>(v, t, xs, tw);
#pragma unroll
    for (int e = 0; e < E; ++e) __stcg(prow + t + T * e, v[e]);
    return;
  } else {
    // --- inverse row transform (unnormalised) of the previous column output
    if (type != ST_REC_ROW0 && type != ST_SEED_ROW) fft<N, E, true>(v, t, xs, tw);
    // recompute rows keep the wave entering their slice for the adjoint sweep
    if (st.seg_slot >= 0 && (type == ST_REC_ROW0 || type == ST_REC_ROW || type == ST_REC_ROWL))
      snapshot(c.seg, st.seg_slot, c.seg_n, type != ST_REC_ROW0);
    if (type == ST_REC_ROWL) return;
    if (type == ST_ADJ_ROW || type == ST_ADJ_ROW0) {
      // v = n^2 lambda_a.  a_s = psi_s t_s; dL/dV = 2 Re(conj(lambda_a) i a_s) dphi/dV.
      // dphi/dV depends on V alone, so the probes' sum of Re(conj(lambda_a) i a_s)
      // is accumulated here and scaled by 2 dphi/dV once per voxel after the
      // sweep (grad_finalize_kernel).  lambda_psi = conj(t_s) lambda_a.
      // psi_s: from the stage (TMA) or straight from the segment buffer.
      const float2* prow = stage2 ? stage2 + rl * N : adj_psi(c, st, k.b) + (long long)row * N;
      const long long tro = row_off();
      const float2* trow = c.ttab + tro;
      float* grow = c.grad + tro;
      acquire();   // psi_s has landed in the stage (split mode)
#pragma unroll
      for (int e = 0; e < E; ++e) {
        const int x = t + T * e;
        const float2 lam = cscale(v[e], c.scale);
        const float2 tt = cscale(__ldg(trow + x), c.inv_scale);
        const float2 as = cmul(stage2 ? prow[x] : __ldcg(prow + x), tt);
        atomicAdd(grow + x, lam.y * as.x - lam.x * as.y);
        v[e] = cmulc(lam, tt);
      }
      release();   // psi_s consumed
      if (type == ST_ADJ_ROW0) return;
      fft<N, E, false>(v, t, xs, tw);
      float2* orow = c.lam + (long long)k.b * plane + (long long)row * N;
#pragma unroll
      for (int e = 0; e < E; ++e) __stcg(orow + t + T * e, v[e]);
      return;
    }
    // recompute rows: * t and forward row transform; the seed row: transform only
    if (type == ST_REC_ROW0) {
#pragma unroll
      for (int e = 0; e < E; ++e) v[e] = cscale(v[e], c.inv_scale);
    }
    if (type != ST_SEED_ROW) {
      const float2* trow = c.ttab + row_off();
#pragma unroll
      for (int e = 0; e < E; ++e) v[e] = cmul(v[e], __ldg(trow + t + T * e));
    }
    fft<N, E, false>(v, t, xs, tw);
    float2* dst = (type == ST_SEED_ROW) ? c.lam : c.work;
    float2* orow = dst + (long long)k.b * plane + (long long)row * N;
#pragma unroll
    for (int e = 0; e < E; ++e) __stcg(orow + t + T * e, v[e]);
  }
}

template <int N, int E>
__device__ __forceinline__ void col_load(const float2* stage, float2 (&v)[E]) {
  constexpr int T = N / E;
  constexpr int W = kSchedThreads / T;
  const int cc = threadIdx.x % W, t = threadIdx.x / W;
#pragma unroll
  for (int e = 0; e < E; ++e) v[e] = stage[(t + T * e) * W + cc];
}

// Column tile: FFT, * H or conj(H) (hi + lo), [dp / adjoint seed], inverse FFT.
template <int N, int E, bool GRAD, class TW>
__device__ __forceinline__ void col_compute(const SchedClass& c, const Task& k, const Step& st, float2 (&v)[E],
                                            float2* exch, const TW* tw) {
  constexpr int T = N / E;
  constexpr int W = kSchedThreads / T;
  const int cc = threadIdx.x % W, t = threadIdx.x / W;
  const int col = k.tile * W + cc;
  const long long plane = (long long)N * N;
  // 512-point columns (8 per tile) exchange through the padded tile: the
  // unpadded one costs the first stage's scatter a 2-way bank conflict
  // (B200, 512^2 scan: 14 % of its shared-memory wavefronts); its
  // (512 + 32) x 8 entries fill the exchange buffer exactly
  using XS = typename std::conditional<N == 512 && E == 16, ColExchangePad<kFftBar, kSchedThreads>,
                                       ColExchange<kFftBar, kSchedThreads>>::type;
  static_assert(N != 512 || E != 16 || (N + N / 16) * W * sizeof(float2) <= kExchBytesFor(16),
                "padded 512-point column tile fits the exchange buffer");
  const XS xs{exch, W, cc};
  const int type = st.type;
  fft<N, E, false>(v, t, xs, tw);
  const int sx = (col + (N >> 1)) & (N - 1);
  if constexpr (GRAD) {
    if (type == ST_SEED_COL) {
      // lambda seed: n^2 g Z with g = dL/d(dp) at the fftshifted position
      // (zero outside the detector window)
      // (+ the exit-wave loss's seed: fft2(dL/d(exit) / 2) at (ky, kx))
      const float* gp = c.g + (long long)k.b * plane;
#pragma unroll
      for (int e = 0; e < E; ++e) {
        const int sy = (t + T * e + (N >> 1)) & (N - 1);
        v[e] = cscale(v[e], c.inv_scale * __ldg(gp + (long long)sy * N + sx));
      }
      if (c.seed_add) {
        const float2* sp = c.seed_add + (long long)k.b * plane + col;
#pragma unroll
        for (int e = 0; e < E; ++e) v[e] = cadd(v[e], __ldcg(sp + (long long)(t + T * e) * N));
      }
    }
  }
  const bool conj = GRAD && (type == ST_SEED_COL || type == ST_ADJ_COL);
  const float4* hcol = c.Hq + col;
  if (conj) {
#pragma unroll
    for (int e = 0; e < E; ++e) {
      const float4 h = __ldg(hcol + (t + T * e) * N);
      v[e] = cmulc_hl(v[e], make_float2(h.x, h.y), make_float2(h.z, h.w));
    }
  } else {
#pragma unroll
    for (int e = 0; e < E; ++e) {
      const float4 h = __ldg(hcol + (t + T * e) * N);
      v[e] = cmul_hl(v[e], make_float2(h.x, h.y), make_float2(h.z, h.w));
    }
  }
  if (!GRAD && c.dp && st.slice == c.n_slices - 1) {
    float* dp = c.dp + (long long)k.b * plane;
#pragma unroll
    for (int e = 0; e < E; ++e) {
      const int sy = (t + T * e + (N >> 1)) & (N - 1);
      __stcs(dp + (long long)sy * N + sx, fmaf(v[e].x, v[e].x, v[e].y * v[e].y));
    }
  }
  fft<N, E, true>(v, t, xs, tw);
  float2* dst = !GRAD ? c.psi : type == ST_REC_COL ? c.work : c.lam;
  float2* pcol = dst + (long long)k.b * plane + col;
#pragma unroll
  for (int e = 0; e < E; ++e) __stcg(pcol + (long long)(t + T * e) * N, v[e]);
}

// Compute warps of an instance for one grid size: take the published tile,
// pull it into registers, release the stage, run the transforms, store,
// report completion.
// HI_TW: the stage twiddles are hi parts only (float2 entries; tw_off counts them)
template <unsigned MASK, int E, bool GRAD, bool HI_TW>
__device__ __forceinline__ void compute_loop_one(const SchedParams& P, float2* stage, float2* exch, const float4* tw_smem,
                                             uint64_t* full, uint64_t* empty, uint64_t* done_bar, const Task* s_task) {
  uint32_t fph = 0;
  uint32_t tiles_done = 0;   // selects the done barrier (two, alternating)
  const int lane = threadIdx.x & 31;
  while (true) {
    // Bounded wait for the next published item.  On expiry record the error
    // and keep waiting (bounded rounds): the producer's own waits are bounded
    // and it publishes the stop sentinel once an error is recorded, so every
    // compute warp reads the same item and runs the same barrier sequence.
    for (int round = 0; round < 4 && !mbar_wait(full, fph, P.spin_limit, P.suspend_ns); ++round)
      atomicCAS(P.status, 0, WAP_ERR_TIMEOUT);
    fph ^= 1u;
    const Task k = *s_task;
    if (!k.valid) return;
    if (!task_ok<GRAD>(P, k, 1)) {
      __syncwarp();
      if (lane == 0) {
        mbar_arrive(empty);
        mbar_arrive(done_bar + (tiles_done & 1));
      }
      ++tiles_done;
      continue;
    }
    const SchedClass& c = P.cls[k.cls];
    const Step st = step_of<GRAD>(c, k.pass);
    using TW = typename std::conditional<HI_TW, float2, float4>::type;
    // always the shared-memory image: a pointer that could be either space
    // would make every twiddle read a generic load
    const TW* tw = reinterpret_cast<const TW*>(tw_smem) + c.tw_off;
    const bool col = step_is_col(st.type);
    // Adjoint rows read psi_s next to lambda.  kPsiStage2: both arrive
    // together (second stage), released after psi_s is read.  kPsiSplit:
    // lambda is released as usual, then the producer refills the same stage
    // with psi_s - a second phase of `full` that lands during the inverse row
    // transform - released after psi_s is read.
    const bool adj = GRAD && (st.type == ST_ADJ_ROW || st.type == ST_ADJ_ROW0);
    const bool late = adj && P.stage2 == kPsiStage2;
    const bool split = adj && P.stage2 == kPsiSplit;
    const float2* st2 = late ? stage + kTileBytesFor(E) / sizeof(float2) : split ? stage : nullptr;
    auto acquire = [&]() {
      if (split) {
        for (int round = 0; round < 4 && !mbar_wait(full, fph, P.spin_limit, P.suspend_ns); ++round)
          atomicCAS(P.status, 0, WAP_ERR_TIMEOUT);
        fph ^= 1u;
      }
    };
    auto release = [&]() {
      if (late || split) {
        __syncwarp();
        if (lane == 0) mbar_arrive(empty);
      }
    };
    float2 v[E];
#define WAP_SCHED_CASE(N, BIT)                                            \
    if constexpr ((MASK & BIT) != 0) {                                      \
      if (c.n == N) {                                                       \
        if (col) col_load<N, E>(stage, v);                                  \
        else row_load<N, E>(c, k, st.type, stage, v);                       \
        if (!late) {                                                        \
          __syncwarp();                                                     \
          if (lane == 0) mbar_arrive(empty);                                \
        }                                                                   \
        if (col) col_compute<N, E, GRAD>(c, k, st, v, exch, tw);            \
        else row_compute<N, E, GRAD>(c, k, st, v, exch, tw, st2, acquire, release); \
      }                                                                     \
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

// Compute warps of an instance for several grid sizes: one loop per size.
// tile_loop<N> runs the tiles of n = N and hands a tile of another size back
// (pending) to the loop of that size.  Tickets are ordered class by class, so
// the hand-overs are rare, and each size's transforms sit in a region of
// their own: fewer spills than one loop over all sizes (256^2 + 512^2
// headline scan: 64.8 -> 63.5 ms).  Single-size instances keep the plain
// loop above, which is the faster of the two for them.
constexpr int kLoopStop = 0;    // the stop sentinel arrived
constexpr int kLoopOther = 1;   // tiles processed, then one of another size is pending
constexpr int kLoopIdle = 2;    // no tile processed: the pending tile is of another size

struct ComputeState {
  uint32_t fph;          // phase of the `full` barrier
  uint32_t tiles_done;   // selects the done barrier (two, alternating)
  Task k;                // the published tile taken last
  bool pending;          // k is taken but belongs to another size's loop
};

// HI_TW: the stage twiddles are hi parts only (float2 entries; tw_off counts them)
template <int N, int E, bool GRAD, bool HI_TW>
__device__ __forceinline__ int tile_loop(const SchedParams& P, float2* stage, float2* exch, const float4* tw_smem,
                                         uint64_t* full, uint64_t* empty, uint64_t* done_bar, const Task* s_task,
                                         ComputeState& cs) {
  const int lane = threadIdx.x & 31;
  int result = kLoopIdle;
  while (true) {
    if (!cs.pending) {
      // Bounded wait for the next published item.  On expiry record the error
      // and keep waiting (bounded rounds): the producer's own waits are bounded
      // and it publishes the stop sentinel once an error is recorded, so every
      // compute warp reads the same item and runs the same barrier sequence.
      for (int round = 0; round < 4 && !mbar_wait(full, cs.fph, P.spin_limit, P.suspend_ns); ++round)
        atomicCAS(P.status, 0, WAP_ERR_TIMEOUT);
      cs.fph ^= 1u;
      cs.k = *s_task;
    }
    cs.pending = false;
    const Task k = cs.k;
    if (!k.valid) return kLoopStop;
    if (!task_ok<GRAD>(P, k, 1)) {
      __syncwarp();
      if (lane == 0) {
        mbar_arrive(empty);
        mbar_arrive(done_bar + (cs.tiles_done & 1));
      }
      ++cs.tiles_done;
      result = kLoopOther;
      continue;
    }
    const SchedClass& c = P.cls[k.cls];
    if (c.n != N) {
      cs.pending = true;
      return result;
    }
    result = kLoopOther;
    const Step st = step_of<GRAD>(c, k.pass);
    using TW = typename std::conditional<HI_TW, float2, float4>::type;
    // always the shared-memory image: a pointer that could be either space
    // would make every twiddle read a generic load
    const TW* tw = reinterpret_cast<const TW*>(tw_smem) + c.tw_off;
    const bool col = step_is_col(st.type);
    // Adjoint rows read psi_s next to lambda.  kPsiStage2: both arrive
    // together (second stage), released after psi_s is read.  kPsiSplit:
    // lambda is released as usual, then the producer refills the same stage
    // with psi_s - a second phase of `full` that lands during the inverse row
    // transform - released after psi_s is read.
    const bool adj = GRAD && (st.type == ST_ADJ_ROW || st.type == ST_ADJ_ROW0);
    const bool late = adj && P.stage2 == kPsiStage2;
    const bool split = adj && P.stage2 == kPsiSplit;
    const float2* st2 = late ? stage + kTileBytesFor(E) / sizeof(float2) : split ? stage : nullptr;
    auto acquire = [&]() {
      if (split) {
        for (int round = 0; round < 4 && !mbar_wait(full, cs.fph, P.spin_limit, P.suspend_ns); ++round)
          atomicCAS(P.status, 0, WAP_ERR_TIMEOUT);
        cs.fph ^= 1u;
      }
    };
    auto release = [&]() {
      if (late || split) {
        __syncwarp();
        if (lane == 0) mbar_arrive(empty);
      }
    };
    float2 v[E];
    if (col) col_load<N, E>(stage, v);
    else row_load<N, E>(c, k, st.type, stage, v);
    if (!late) {
      __syncwarp();
      if (lane == 0) mbar_arrive(empty);
    }
    if (col) col_compute<N, E, GRAD>(c, k, st, v, exch, tw);
    else row_compute<N, E, GRAD>(c, k, st, v, exch, tw, st2, acquire, release);
    __syncwarp();
    if (lane == 0) mbar_arrive(done_bar + (cs.tiles_done & 1));
    ++cs.tiles_done;
  }
}

template <unsigned MASK, int E, bool GRAD, bool HI_TW>
__device__ __forceinline__ void compute_loop_split(const SchedParams& P, float2* stage, float2* exch,
                                                   const float4* tw_smem, uint64_t* full, uint64_t* empty,
                                                   uint64_t* done_bar, const Task* s_task) {
  ComputeState cs{0u, 0u, Task{}, false};
  const int lane = threadIdx.x & 31;
  while (true) {
    bool progress = false;
#define WAP_SCHED_LOOP(N, BIT)                                                                        \
    if constexpr ((MASK & BIT) != 0) {                                                                \
      const int r = tile_loop<N, E, GRAD, HI_TW>(P, stage, exch, tw_smem, full, empty, done_bar, s_task, cs); \
      if (r == kLoopStop) return;                                                                     \
      progress = progress || r == kLoopOther;                                                         \
    }
    WAP_SCHED_LOOP(128, 1u)
    WAP_SCHED_LOOP(256, 2u)
    WAP_SCHED_LOOP(512, 4u)
    WAP_SCHED_LOOP(1024, 8u)
#undef WAP_SCHED_LOOP
    if (!progress && cs.pending) {
      // a tile of a size this instance has no transforms for (the host builds
      // the instance from the classes' sizes, so this is a corrupted task):
      // record it and pass it through like an invalid one
      atomicCAS(P.status, 0, WAP_ERR_CUDA);
      __syncwarp();
      if (lane == 0) {
        mbar_arrive(empty);
        mbar_arrive(done_bar + (cs.tiles_done & 1));
      }
      ++cs.tiles_done;
      cs.pending = false;
    }
  }
}

// ---------------------------------------------------------------------------
// the persistent kernel: 8 compute warps + 1 producer warp
// ---------------------------------------------------------------------------
template <unsigned MASK, int E, bool GRAD, bool HI_TW = false>
__global__ void __launch_bounds__(kBlockThreads, E == 16 ? 3 : 4) scan_kernel(const __grid_constant__ SchedParams P) {
  extern __shared__ __align__(1024) unsigned char sched_smem[];
  float2* stage = reinterpret_cast<float2*>(sched_smem);
  constexpr int kTile = kTileBytesFor(E), kExch = kExchBytesFor(E);
  const int stages = (GRAD && P.stage2 == kPsiStage2) ? 2 : 1;
  float2* exch = reinterpret_cast<float2*>(sched_smem + stages * kTile);
  float4* tw_smem = reinterpret_cast<float4*>(sched_smem + stages * kTile + kExch);
  __shared__ __align__(8) uint64_t full, empty, done_bar[2];
  __shared__ Task s_task;

  for (int i = threadIdx.x; i < P.tw_image_len; i += blockDim.x) tw_smem[i] = P.tw_image[i];
  if (threadIdx.x == 0) {
    mbar_init(&full, 1);
    mbar_init(&empty, kComputeWarps);
    mbar_init(&done_bar[0], kComputeWarps);
    mbar_init(&done_bar[1], kComputeWarps);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();

  if (threadIdx.x < kSchedThreads) {
    if constexpr ((MASK & (MASK - 1)) == 0)
      compute_loop_one<MASK, E, GRAD, HI_TW>(P, stage, exch, tw_smem, &full, &empty, done_bar, &s_task);
    else
      compute_loop_split<MASK, E, GRAD, HI_TW>(P, stage, exch, tw_smem, &full, &empty, done_bar, &s_task);
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
    return k.pass == P.stall_pass ? 0x7fffffff : step_of<GRAD>(P.cls[k.cls], k.pass).prefix;
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
    if ((P.checks & 2) && spins) atomicAdd(reinterpret_cast<unsigned*>(P.debug) + 7, (unsigned)spins);
    fence_proxy_async();
    return true;
  };
  // publish a task (or the stop sentinel) to the compute warps: exactly one
  // arrival per phase on `full` (count 1) - issue_load's arrive.expect_tx for
  // tiles with a TMA load, a plain arrive otherwise
  auto fail_wait = [&]() { atomicCAS(P.status, 0, WAP_ERR_TIMEOUT); };
  uint32_t eph = 0, dph[2] = {0, 0};
  uint32_t fph = 0;            // parity of the next full-barrier phase to complete
  bool load_out = false;       // the latest published item carried a TMA load
  auto publish = [&](const Task& k0) {
    Task k = k0;
    if (k.valid && !task_ok<GRAD>(P, k, 2)) k.valid = 0;
    s_task = k;
    const SchedClass& c = P.cls[k.cls];
    const int type = k.valid ? step_of<GRAD>(c, k.pass).type : -1;
    const uint32_t bytes = k.valid ? tile_bytes(c, type) : 0u;
    load_out = bytes != 0;
    if (bytes) issue_load<GRAD>(P, k, stage, &full);
    else mbar_arrive(&full);
    fph ^= 1u;
    if (GRAD && P.stage2 == kPsiSplit && (type == ST_ADJ_ROW || type == ST_ADJ_ROW0)) {
      // second phase of the same tile: once every compute warp holds lambda,
      // refill the stage with the matching rows of psi_s
      if (!mbar_wait(&empty, eph, P.spin_limit, P.suspend_ns)) fail_wait();
      eph ^= 1u;
      fence_proxy_async();
      const Step st = step_of<GRAD>(c, k.pass);
      mbar_expect_tx(&full, bytes);
      bulk_g2s(stage, adj_psi(c, st, k.b) + (long long)k.tile * c.rows * c.n, bytes, &full);
      fph ^= 1u;
    }
  };

  uint32_t tiles_signalled = 0;
  Task k = claim();
  if (k.valid && !wait_ready(k)) k.valid = 0;
  publish(k);
  while (k.valid) {
    // the next ticket is claimed only now: claiming it while k still computes
    // (one tile earlier) found its inputs incomplete for a third of the tickets
    // of the headline scan and cost 4 % (56.8 against 54.5 ms)
    Task kn = claim();
    bool issued = false;
    const bool ready = kn.valid && ld_acquire(counter_of(kn)) >= need_of(kn);
    if ((P.checks & 2) && kn.valid && !ready) atomicAdd(P.debug + 6, 1);
    if (ready) {
      // inputs ready: stream the next tile in as soon as the stage is free
      if (!mbar_wait(&empty, eph, P.spin_limit, P.suspend_ns)) fail_wait();
      eph ^= 1u;
      fence_proxy_async();
      publish(kn);
      issued = true;
    }
    // completion of k: every compute warp has stored its part.  The compute
    // warps may already have finished the prefetched tile too, so tiles
    // alternate between two barriers (a parity wait never sees two phases).
    {
      const int q = tiles_signalled & 1;
      if (!mbar_wait(&done_bar[q], dph[q], P.spin_limit, P.suspend_ns)) fail_wait();
      dph[q] ^= 1u;
      ++tiles_signalled;
    }
    __threadfence();
    atomicAdd(P.done + P.cls[k.cls].done_off + k.b, 1);
    if (!issued) {
      // holding nothing unsignalled now: safe to block on kn's inputs
      if (kn.valid && !wait_ready(kn)) kn.valid = 0;
      if (!mbar_wait(&empty, eph, P.spin_limit, P.suspend_ns)) fail_wait();
      eph ^= 1u;
      publish(kn);   // kn or the stop sentinel
    }
    k = kn;
  }
  // After an error the compute warps may have stopped without consuming the
  // last published tile: let its copy land (bounded) before the CTA exits.
  if (load_out && *(volatile int*)P.status != 0) mbar_wait(&full, fph ^ 1u, P.spin_limit, P.suspend_ns);
}

// dL/dV += 2 dphi/dV(V) S for every voxel, S being the probes' sum of
// Re(conj(lambda_a) i a_s) from the adjoint sweep.  phi = kphase (n(V) - 1)
// with n(V) of propagation.py:66-81, so dphi/dV = kphase (E + E0 + V)
// inv_den / n(V).
static __global__ void __launch_bounds__(256) grad_finalize_kernel(const float* __restrict__ V,
                                                            const float* __restrict__ S, float* __restrict__ grad,
                                                            long long n4, float a, float inv_den, float kphase,
                                                            float e_plus_e0) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n4; i += (long long)gridDim.x * blockDim.x) {
    const float4 v = __ldg(reinterpret_cast<const float4*>(V) + i);
    const float4 sm = __ldcs(reinterpret_cast<const float4*>(S) + i);
    float4 g = reinterpret_cast<float4*>(grad)[i];
    auto term = [&](float vv, float ss) {
      const float dn = refr_minus_one(vv, a, inv_den);
      return 2.0f * ss * (kphase * (e_plus_e0 + vv) * inv_den / (1.0f + dn));
    };
    g.x += term(v.x, sm.x);
    g.y += term(v.y, sm.y);
    g.z += term(v.z, sm.z);
    g.w += term(v.w, sm.w);
    reinterpret_cast<float4*>(grad)[i] = g;
  }
}

// Detector windows of the scheduler.  An inlined window test in the persistent
// kernel's pattern store and adjoint seed raises the register pressure of
// every tile body (measured on B200: +1.2 % on the batched scan, +6 % on the
// adjoint sweep), so a windowed class runs on a full-grid scratch pattern and
// these two passes move the window in and out (about 0.1 % of a step).
static __global__ void __launch_bounds__(256) crop_window_kernel(const float* __restrict__ full,
                                                          float* __restrict__ dp, long long total, int n, Detector d) {
  const long long per = (long long)d.ny * d.nx;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
    const long long b = i / per;
    const int r = (int)(i - b * per), ry = r / d.nx, rx = r - ry * d.nx;
    dp[i] = __ldcs(full + (b * n + d.y0 + ry) * n + d.x0 + rx);
  }
}

static __global__ void __launch_bounds__(256) scatter_window_kernel(const float* __restrict__ g,
                                                             float* __restrict__ full, long long total, int n,
                                                             Detector d) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
    const long long b = i / ((long long)n * n);
    const int r = (int)(i - b * n * n), y = r / n - d.y0, x = r % n - d.x0;
    const bool in = (unsigned)y < (unsigned)d.ny && (unsigned)x < (unsigned)d.nx;
    full[i] = in ? __ldg(g + (b * d.ny + y) * d.nx + x) : 0.0f;
  }
}

}  // namespace wap

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
using namespace wap;

typedef void (*ScanKernel)(const SchedParams);

// kernel instances by elements per thread and the set of grid sizes they
// contain (bit 0: 128, 1: 256, 2: 512, 3: 1024); other sets use the
// all-sizes instance.  Gradient instances hold one size each.
template <int E>
static ScanKernel pick_fwd_e(unsigned mask) {
  switch (mask) {
    case 1u: return scan_kernel<1u, E, false>;
    case 2u: return scan_kernel<2u, E, false>;
    case 4u: return scan_kernel<4u, E, false>;
    case 8u: return scan_kernel<8u, E, false>;
    case 6u: return scan_kernel<6u, E, false>;
    default: return scan_kernel<15u, E, false>;
  }
}
static ScanKernel pick_fwd_hi(unsigned mask) {
  switch (mask) {
    case 1u: return scan_kernel<1u, 16, false, true>;
    case 2u: return scan_kernel<2u, 16, false, true>;
    case 4u: return scan_kernel<4u, 16, false, true>;
    case 8u: return scan_kernel<8u, 16, false, true>;
    case 6u: return scan_kernel<6u, 16, false, true>;
    default: return scan_kernel<15u, 16, false, true>;
  }
}
template <bool HI_TW>
static ScanKernel pick_grad(unsigned mask) {
  switch (mask) {
    case 1u: return scan_kernel<1u, 16, true, HI_TW>;
    case 2u: return scan_kernel<2u, 16, true, HI_TW>;
    case 4u: return scan_kernel<4u, 16, true, HI_TW>;
    default: return scan_kernel<8u, 16, true, HI_TW>;
  }
}

struct wap_scan {
  ScanKernel kernel = nullptr;       // forward chains (gradient scans: with snapshots)
  ScanKernel kernel_bwd = nullptr;   // backward chain of gradient scans
  bool grad = false;
  int e = 16;
  bool hi_tw = false;                // stage twiddles as hi parts only (forward scans of few slices)
  int device = 0;
  int n_classes = 0;
  SchedParams params{};
  SchedDesc* d_desc = nullptr;      // forward descriptors
  SchedDesc* d_desc_bwd = nullptr;  // backward descriptors (gradient scans)
  int n_desc = 0, n_desc_bwd = 0;
  long long n_tickets = 0, n_tickets_bwd = 0;
  Step* d_steps = nullptr;          // forward chains of all classes, back to back
  Step* d_steps_bwd = nullptr;      // backward chain (gradient scans: one class)
  unsigned long long* d_ticket = nullptr;
  int* d_done = nullptr;
  int* d_status = nullptr;
  int* d_debug = nullptr;
  int total_probes = 0;
  int grid = 0;
  size_t smem = 0;
  int grid_bwd = 0;                 // backward launch (two staging buffers with kPsiStage2)
  size_t smem_bwd = 0;
  int psi_mode = kPsiSplit;         // how the backward's adjoint rows get psi_s
  std::vector<Detector> det;        // per class: diffraction-pattern window (the whole grid: no window)
  std::vector<float*> d_dpfull;     // per windowed class: (B, n, n) full-grid pattern / seed scratch
  float* d_gsum = nullptr;          // (draws, N, n, n) probe sums of the adjoint sweep
  int ckpt_every = 0;
  std::vector<float4*> d_tw;
  float4* d_tw_seed = nullptr;      // gradient scans: the hi + lo (n, 16) table of the exit-wave seed passes
  std::vector<float2*> d_ttab;
  std::vector<float4*> d_hq;
  std::vector<void*> d_extra;       // gradient buffers
  std::vector<size_t> ttab_elems;
  std::vector<wap_scan_class> cls;
  std::vector<Physics> phys;
  std::vector<int> groups;          // per class: probes advanced together
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
  cudaFree(s->d_desc_bwd);
  cudaFree(s->d_steps);
  cudaFree(s->d_steps_bwd);
  cudaFree(s->d_ticket);
  cudaFree(s->d_done);
  cudaFree(s->d_status);
  cudaFree(s->d_debug);
  for (auto p : s->d_tw) cudaFree(p);
  cudaFree(s->d_tw_seed);
  for (auto p : s->d_ttab) cudaFree(p);
  for (auto p : s->d_hq) cudaFree(p);
  for (auto p : s->d_extra) cudaFree(p);
  for (auto p : s->d_dpfull) cudaFree(p);
  cudaFree(s->d_gsum);
  delete s;
}

static bool sched_size_ok(int n) { return n == 128 || n == 256 || n == 512 || n == 1024; }

// Scheduler overrides for A/B timing and tests (wap_scan_debug_override); -1:
// the library's own choice.  Set only by an explicit call, never from the
// environment, and read when a scan is created.
static int g_knob[WAP_KNOB_COUNT] = {-1, -1, -1, -1, -1, -1, -1, -1, -1};
static int knob(int k) { return g_knob[k]; }
namespace wap {
int knob_value(int k) { return (k >= 0 && k < WAP_KNOB_COUNT) ? g_knob[k] : -1; }
}  // namespace wap

static bool windowed(const Detector& d, int n) { return d.ny != n || d.nx != n; }

// detector window of a class's diffraction patterns (0 x 0: the whole grid)
static int class_detector(const wap_scan_class& c, int ci, Detector* d) {
  if (c.det_ny == 0 && c.det_nx == 0) {
    *d = Detector{0, 0, c.n, c.n};
    return WAP_OK;
  }
  if (c.det_ny < 1 || c.det_nx < 1 || c.det_y0 < 0 || c.det_x0 < 0 || c.det_y0 + c.det_ny > c.n ||
      c.det_x0 + c.det_nx > c.n)
    return fail(WAP_ERR_ARG, "scan class %d: detector window rows %d+%d, columns %d+%d outside the %d x %d grid", ci,
                c.det_y0, c.det_ny, c.det_x0, c.det_nx, c.n, c.n);
  *d = Detector{c.det_y0, c.det_x0, c.det_ny, c.det_nx};
  return WAP_OK;
}

// Record class ci's window and point its pattern at the user's buffer, or at
// the class's full-grid scratch (allocated the first time a window is set).
static int bind_detector(wap_scan* s, const wap_scan_class& c, int ci) {
  if ((int)s->det.size() < ci + 1) {
    s->det.resize(ci + 1);
    s->d_dpfull.resize(ci + 1, nullptr);
  }
  int rc = class_detector(c, ci, &s->det[ci]);
  if (rc) return rc;
  SchedClass& sc = s->params.cls[ci];
  sc.dp = c.dp;
  if (c.dp && windowed(s->det[ci], c.n)) {
    if (!s->d_dpfull[ci]) {
      cudaError_t e = cudaMalloc(&s->d_dpfull[ci], (size_t)c.n_probes * c.n * c.n * sizeof(float));
      if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc(full-grid pattern scratch)");
    }
    sc.dp = s->d_dpfull[ci];
  }
  return WAP_OK;
}

// column-tile tensor map over (B n rows) x (n columns) of 8-byte elements
static int encode_map(PFN_cuTensorMapEncodeTiled_v12000 encode, CUtensorMap* map, void* base, int n, int n_probes,
                      int cols_w, int box_rows) {
  cuuint64_t gdim[2] = {(cuuint64_t)n, (cuuint64_t)n_probes * n};
  cuuint64_t gstride[1] = {(cuuint64_t)n * 8};
  cuuint32_t box[2] = {(cuuint32_t)cols_w, (cuuint32_t)box_rows};
  cuuint32_t estride[2] = {1, 1};
  CUresult r = encode(map, CU_TENSOR_MAP_DATA_TYPE_INT64, 2, base, gdim, gstride, box, estride,
                      CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                      CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(WAP_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
  return WAP_OK;
}

// Trailing checkpoint segments whose waves the forward keeps, so that the
// backward recomputes none of them: memory stays O(sqrt N) - checkpoints every
// k slices plus 4k waves - and four segments' recompute (2k - 1 passes each)
// drop.  Two kept segments left the 512^2 x 64-slice gradient step at 3.03 x
// its forward after the forward scan itself had become faster, three at
// 2.93 - 2.98, four at 2.83 - 2.87 (B200, the same box).
constexpr int kKeptSegments = 4;

static int kept_first_slice(int n_slices, int k) {
  const int nck = (n_slices + k - 1) / k;
  return (nck - std::min(kKeptSegments, nck)) * k;
}

// Forward chain of one class: steps 0..2N (rows even, columns odd).  With
// ckpt_every > 0 the rows also store checkpoints (every k-th slice) and the
// waves of the kept trailing segments after their first slice (whose wave is
// a checkpoint).
static void forward_steps(const SchedClass& sc, int n_slices, int ckpt_every, std::vector<Step>& out) {
  const int N = n_slices;
  const int k = ckpt_every;
  const int last0 = k > 0 ? kept_first_slice(N, k) : N;
  int prefix = 0;
  for (int p = 0; p <= 2 * N; ++p) {
    Step st{};
    st.slice = p >> 1;
    st.ckpt_slot = -1;
    st.seg_slot = -1;
    if (p & 1) {
      st.type = ST_FWD_COL;
    } else if (p == 2 * N) {
      st.type = ST_FWD_ROWN;
    } else {
      st.type = p == 0 ? ST_FWD_ROW0 : ST_FWD_ROW;
      if (k > 0 && st.slice % k == 0) st.ckpt_slot = st.slice / k;
      if (k > 0 && st.slice > last0) st.seg_slot = st.slice - last0;
    }
    st.seg0 = k > 0 ? (st.slice / k) * k : 0;
    st.prefix = prefix;
    prefix += (p & 1) ? sc.col_tiles : sc.row_tiles;
    out.push_back(st);
  }
}

// Backward chain: seed, then per segment (last first) recompute + adjoint.
// The kept trailing segments need no recompute: their adjoint rows read the
// waves the forward stored (slot s - first kept slice).  Earlier segments are
// recomputed from their checkpoint, keeping the waves entering slices
// s0+1 .. s1-1; the adjoint row of slice s0 reads the checkpoint itself
// (one-slice segments need no recompute at all).
static void backward_steps(const SchedClass& sc, int n_slices, int k, std::vector<Step>& out) {
  const int N = n_slices;
  const int nck = (N + k - 1) / k;
  const int kept0 = kept_first_slice(N, k);
  int prefix = 0;
  auto push = [&](int type, int slice, int seg0, int ckpt_slot, int seg_slot) {
    Step st{type, slice, seg0, ckpt_slot, seg_slot, prefix};
    prefix += step_is_col(type) ? sc.col_tiles : sc.row_tiles;
    out.push_back(st);
  };
  push(ST_SEED_ROW, N - 1, 0, -1, -1);
  push(ST_SEED_COL, N - 1, 0, -1, -1);
  for (int j = nck - 1; j >= 0; --j) {
    const int s0 = j * k, s1 = std::min(s0 + k, N);
    if (s0 >= kept0) {
      for (int s = s1 - 1; s >= s0; --s) {
        const int type = s == 0 ? ST_ADJ_ROW0 : ST_ADJ_ROW;
        if (s == kept0) push(type, s, s0, j, -1);   // the first kept slice: checkpoint j
        else push(type, s, s0, -1, s - kept0);
        if (s > 0) push(ST_ADJ_COL, s, s0, -1, -1);
      }
      continue;
    }
    if (s1 - s0 > 1) {
      push(ST_REC_ROW0, s0, s0, j, -1);
      push(ST_REC_COL, s0, s0, -1, -1);
      for (int s = s0 + 1; s < s1 - 1; ++s) {
        push(ST_REC_ROW, s, s0, -1, s - s0);
        push(ST_REC_COL, s, s0, -1, -1);
      }
      push(ST_REC_ROWL, s1 - 1, s0, -1, s1 - 1 - s0);
    }
    for (int s = s1 - 1; s >= s0; --s) {
      const int type = s == 0 ? ST_ADJ_ROW0 : ST_ADJ_ROW;
      if (s == s0) push(type, s, s0, j, -1);   // psi_s0 is checkpoint j
      else push(type, s, s0, -1, s - s0);
      if (s > 0) push(ST_ADJ_COL, s, s0, -1, -1);
    }
  }
}

// Descriptors: groups of G probes walk through a class's chain.
static void build_desc(const std::vector<Step>& steps, int ci, int n_probes, int G, long long& ticket,
                       const SchedClass& sc, std::vector<SchedDesc>& out) {
  for (int b0 = 0; b0 < n_probes; b0 += G) {
    const int nb = std::min(G, n_probes - b0);
    for (size_t p = 0; p < steps.size(); ++p) {
      SchedDesc d;
      d.base = ticket;
      d.cls = ci;
      d.pass = (int)p;
      d.b0 = b0;
      d.nprobes = nb;
      d.tiles = step_is_col(steps[p].type) ? sc.col_tiles : sc.row_tiles;
      out.push_back(d);
      ticket += (long long)nb * d.tiles;
    }
  }
}

template <class T>
static int upload(T** dst, const std::vector<T>& src, const char* what) {
  cudaError_t e = cudaMalloc(dst, std::max<size_t>(1, src.size()) * sizeof(T));
  if (e == cudaSuccess && !src.empty()) e = cudaMemcpy(*dst, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice);
  return e == cudaSuccess ? WAP_OK : cuda_fail(e, what);
}

// Stage-twiddle table of the hi-only instance: the float2 hi parts packed two
// to a float4 entry (so the image and its prefix sharing work unchanged).
static std::vector<float4> pack_hi(const std::vector<float4>& t) {
  std::vector<float4> q((t.size() + 1) / 2, make_float4(0.f, 0.f, 0.f, 0.f));
  float2* qp = reinterpret_cast<float2*>(q.data());
  for (size_t i = 0; i < t.size(); ++i) qp[i] = make_float2(t[i].x, t[i].y);
  return q;
}

// Shared set-up of forward scans (ckpt_every = 0) and gradient scans.
static int scan_setup(wap_scan* s, int n_classes, const wap_scan_class* classes, int ckpt_every) {
  PFN_cuTensorMapEncodeTiled_v12000 encode = get_encode();
  if (!encode) return fail(WAP_ERR_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
  cudaGetDevice(&s->device);
  s->n_classes = n_classes;
  s->groups.clear();
  s->cls.assign(classes, classes + n_classes);
  s->grad = ckpt_every > 0;
  s->ckpt_every = ckpt_every;
  cudaError_t e;
  int rc0 = WAP_OK;
  int sms = 0, per_sm = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, s->device);
  // elements per thread of the scheduler's transforms (16; 8 for A/B timing)
  int E = 16;
  if (knob(WAP_KNOB_ELEMS) == 8 && !s->grad) E = 8;
  s->e = E;
  // Hi-only stage twiddles: each entry's float rounding repeats in every
  // transform, so its error grows linearly with the slices a wave crosses
  // (measured on one B200: 4.5e-6 exit-wave error against the float64 oracle
  // at 512^2 x 150 slices, 2.4e-6 with hi + lo; at most 4.9e-6 on 128^2 to
  // 1024^2 grids up to 160 slices); about 10 % faster.  Scans of at most
  // kHiTwiddleMaxSlices slices take them, in the forward and the backward
  // chain alike, so a gradient scan's recompute reproduces its forward waves.
  int max_slices = 0;
  for (int ci = 0; ci < n_classes; ++ci) max_slices = std::max(max_slices, classes[ci].n_slices);
  s->hi_tw = E == 16 && max_slices <= kHiTwiddleMaxSlices;
  if (knob(WAP_KNOB_TWIDDLES) == WAP_TW_FULL) s->hi_tw = false;
  if (knob(WAP_KNOB_TWIDDLES) == WAP_TW_HI) s->hi_tw = E == 16;
  unsigned mask = 0;
  for (int ci = 0; ci < n_classes; ++ci) {
    const int n = classes[ci].n;
    if (!sched_size_ok(n)) return fail(WAP_ERR_UNSUPPORTED, "scan grids must be 128, 256, 512 or 1024 (got %d)", n);
    mask |= n == 128 ? 1u : n == 256 ? 2u : n == 512 ? 4u : 8u;
  }
  // Shared-memory twiddle image: the tables of all classes, largest first; a
  // table equal to the start of one already placed (256 within 512 and 1024:
  // their first stages are the same radix-16 stage) reuses those entries.
  std::vector<std::vector<float4>> tables(n_classes);
  std::vector<int> image_off(n_classes, -1);
  std::vector<float4> image;
  {
    std::vector<int> order(n_classes);
    for (int ci = 0; ci < n_classes; ++ci) {
      tables[ci] = twiddle_table(classes[ci].n, E);
      if (s->hi_tw) tables[ci] = pack_hi(tables[ci]);
      order[ci] = ci;
    }
    std::stable_sort(order.begin(), order.end(),
                     [&](int a, int b) { return tables[a].size() > tables[b].size(); });
    for (int ci : order) {
      const std::vector<float4>& t = tables[ci];
      for (int cj : order) {
        if (image_off[cj] < 0 || tables[cj].size() < t.size()) continue;
        if (!memcmp(tables[cj].data(), t.data(), t.size() * sizeof(float4))) {
          image_off[ci] = image_off[cj];
          break;
        }
      }
      if (image_off[ci] < 0) {
        image_off[ci] = (int)image.size();
        image.insert(image.end(), t.begin(), t.end());
      }
    }
  }
  const int tw_total = (int)image.size();
  s->kernel = s->hi_tw ? pick_fwd_hi(mask) : E == 8 ? pick_fwd_e<8>(mask) : pick_fwd_e<16>(mask);
  if (s->grad) s->kernel_bwd = s->hi_tw ? pick_grad<true>(mask) : pick_grad<false>(mask);
  // Keep the twiddles in shared memory only when they fit next to the stage
  // and exchange buffers without lowering the CTAs per SM.
  const size_t base_smem = kTileBytesFor(E) + kExchBytesFor(E);
  const size_t tw_smem_bytes = (size_t)tw_total * sizeof(float4);
  auto ctas_per_sm = [&](ScanKernel k, size_t bytes, int* out) -> int {
    cudaError_t err = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (err != cudaSuccess) return cuda_fail(err, "cudaFuncSetAttribute(scan_kernel)");
    *out = 0;
    err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(out, k, kBlockThreads, bytes);
    if (err != cudaSuccess) return cuda_fail(err, "cudaOccupancyMaxActiveBlocksPerMultiprocessor(scan_kernel)");
    return WAP_OK;
  };
  int per_sm_tw = 0;
  if ((rc0 = ctas_per_sm(s->kernel, base_smem, &per_sm)) || (rc0 = ctas_per_sm(s->kernel, base_smem + tw_smem_bytes, &per_sm_tw)))
    return rc0;
  // the twiddle image always goes to shared memory (when it costs CTAs per
  // SM, the launch simply has fewer)
  s->params.tw_in_smem = 1;
  (void)per_sm_tw;
  s->smem = base_smem + tw_smem_bytes;
  if ((rc0 = ctas_per_sm(s->kernel, s->smem, &per_sm))) return rc0;
  if (per_sm < 1) return fail(WAP_ERR_CUDA, "scan_kernel does not fit on an SM");
  s->grid = sms * per_sm;
  if (s->grad) {
    // kPsiStage2 stages psi_s next to lambda: one more tile of shared memory
    const int m = knob(WAP_KNOB_PSI);
    if (m >= kPsiGlobal && m <= kPsiSplit) s->psi_mode = m;
    s->smem_bwd = s->smem + (s->psi_mode == kPsiStage2 ? kTileBytesFor(E) : 0);
    int per_sm_bwd = 0;
    if ((rc0 = ctas_per_sm(s->kernel_bwd, s->smem_bwd, &per_sm_bwd))) return rc0;
    if (per_sm_bwd < 1) return fail(WAP_ERR_CUDA, "scan_kernel (backward) does not fit on an SM");
    s->grid_bwd = sms * per_sm_bwd;
  }
  {
    float4* dimg = nullptr;
    if ((rc0 = upload(&dimg, image, "twiddle image upload")) != WAP_OK) return rc0;
    s->d_tw.push_back(dimg);
    s->params.tw_image = dimg;
    s->params.tw_image_len = tw_total;
  }

  std::vector<SchedDesc> desc, desc_bwd;
  std::vector<Step> steps_all, steps_bwd_all;
  std::vector<size_t> step_off;
  long long ticket = 0, ticket_bwd = 0;
  int done_off = 0;
  int rc;
  for (int ci = 0; ci < n_classes; ++ci) {
    const wap_scan_class& c = classes[ci];
    if (c.n_slices < 1 || c.n_draws < 1 || c.n_probes < 1 || !c.V || !c.psi0 || !c.H || !c.exit)
      return fail(WAP_ERR_ARG, "scan class %d: bad sizes or NULL V/psi0/H/exit", ci);
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
    sc.V = c.V;
    sc.dp = c.dp;
    if ((rc0 = bind_detector(s, c, ci))) return rc0;
    sc.vstride = (long long)c.n_slices * n * n;
    sc.scale = (float)(1.0 / ((double)n * n));
    sc.inv_scale = (float)((double)n * n);
    const Physics ph = physics(c.energy, c.dz);
    s->phys.push_back(ph);
    sc.ri_a = (float)ph.ri_a;
    sc.ri_inv_den = (float)ph.ri_inv_den;
    sc.kphase = (float)ph.kphase;
    sc.e_plus_e0 = (float)ph.e_plus_e0;
    float4* dhq = nullptr;
    if ((e = cudaMalloc(&dhq, (size_t)n * n * sizeof(float4))) != cudaSuccess)
      return cuda_fail(e, "cudaMalloc(interleaved H)");
    s->d_hq.push_back(dhq);
    sc.Hq = dhq;
    const std::vector<float4>& h = tables[ci];
    float4* dtw = nullptr;
    if ((rc = upload(&dtw, h, "twiddle upload")) != WAP_OK) return rc;
    s->d_tw.push_back(dtw);
    sc.tw = dtw;
    // the pass kernels that form an exit-wave seed read float4 hi + lo entries,
    // whichever table format the scan itself uses
    if (s->grad && ci == 0 && (rc = upload(&s->d_tw_seed, twiddle_table(n, E), "twiddle upload")) != WAP_OK)
      return rc;
    sc.tw_off = image_off[ci] * (s->hi_tw ? 2 : 1);   // in table entries (float2 for hi-only)
    sc.tw_len = (int)h.size();
    const size_t tt = (size_t)c.n_draws * c.n_slices * n * n;
    float2* dtt = nullptr;
    if ((e = cudaMalloc(&dtt, tt * sizeof(float2))) != cudaSuccess) return cuda_fail(e, "cudaMalloc(transmission table)");
    s->d_ttab.push_back(dtt);
    s->ttab_elems.push_back(tt);
    sc.ttab = dtt;
    if (s->grad) {
      const int k = ckpt_every;
      sc.ckpt_n = (c.n_slices + k - 1) / k;
      sc.seg_first = kept_first_slice(c.n_slices, k);
      sc.seg_n = std::max(k, c.n_slices - sc.seg_first);   // kept waves, or one recomputed segment
      sc.ckpt_k = k;
      const size_t plane = (size_t)n * n, B = (size_t)c.n_probes;
      const size_t sizes[4] = {B * plane * 8, B * plane * 8, B * (size_t)sc.seg_n * plane * 8,
                               B * sc.ckpt_n * plane * 8};
      float2** dsts[4] = {&sc.lam, &sc.work, &sc.seg, &sc.ckpt};
      for (int i = 0; i < 4; ++i) {
        void* p = nullptr;
        if ((e = cudaMalloc(&p, sizes[i])) != cudaSuccess) return cuda_fail(e, "cudaMalloc(gradient buffers)");
        s->d_extra.push_back(p);
        *dsts[i] = reinterpret_cast<float2*>(p);
      }
      if ((e = cudaMalloc(&s->d_gsum, tt * sizeof(float))) != cudaSuccess)
        return cuda_fail(e, "cudaMalloc(gradient sums)");
    }
    if ((rc = encode_map(encode, &s->params.maps[ci][BUF_PSI], c.exit, n, c.n_probes, sc.cols_w, sc.box_rows)))
      return rc;
    if (s->grad) {
      if ((rc = encode_map(encode, &s->params.maps[ci][BUF_LAM], sc.lam, n, c.n_probes, sc.cols_w, sc.box_rows)))
        return rc;
      if ((rc = encode_map(encode, &s->params.maps[ci][BUF_WORK], sc.work, n, c.n_probes, sc.cols_w, sc.box_rows)))
        return rc;
    }
    // chains and descriptors: groups of G probes walk through all steps
    std::vector<Step> steps, steps_bwd;
    forward_steps(sc, c.n_slices, ckpt_every, steps);
    if (s->grad) backward_steps(sc, c.n_slices, ckpt_every, steps_bwd);
    int G = c.group;
    if (G <= 0 && knob(WAP_KNOB_GROUP) > 0) G = knob(WAP_KNOB_GROUP);
    if (G <= 0) {
      // enough tiles per step to cover the resident CTAs four times (a
      // group's steps are a dependency chain, so this is the parallelism
      // available), and no more, so that the group's waves stay in L2: about
      // 4 x 444 tiles x 32 KB = 56 MB for every grid size on a 148-SM part
      G = std::max(1, (4 * s->grid + sc.row_tiles - 1) / sc.row_tiles);
      // then even groups: the batch in round(B / G) groups of equal size, so
      // that no small last group runs its chain with the SMs half idle
      const int ng = std::max(1, (c.n_probes + G / 2) / G);
      G = (c.n_probes + ng - 1) / ng;
    }
    G = std::min(G, c.n_probes);
    s->groups.push_back(G);
    build_desc(steps, ci, c.n_probes, G, ticket, sc, desc);
    if (s->grad) build_desc(steps_bwd, ci, c.n_probes, G, ticket_bwd, sc, desc_bwd);
    step_off.push_back(steps_all.size());
    steps_all.insert(steps_all.end(), steps.begin(), steps.end());
    steps_bwd_all.insert(steps_bwd_all.end(), steps_bwd.begin(), steps_bwd.end());
    done_off += c.n_probes;
  }
  s->n_tickets = ticket;
  s->n_tickets_bwd = ticket_bwd;
  s->total_probes = done_off;
  s->n_desc = (int)desc.size();
  s->n_desc_bwd = (int)desc_bwd.size();
  if ((rc = upload(&s->d_desc, desc, "scan descriptors")) || (rc = upload(&s->d_steps, steps_all, "scan steps")))
    return rc;
  if (s->grad && ((rc = upload(&s->d_desc_bwd, desc_bwd, "scan descriptors")) ||
                  (rc = upload(&s->d_steps_bwd, steps_bwd_all, "scan steps"))))
    return rc;
  for (int ci = 0; ci < n_classes; ++ci) s->params.cls[ci].steps = s->d_steps + step_off[ci];
  if ((e = cudaMalloc(&s->d_ticket, sizeof(unsigned long long))) != cudaSuccess ||
      (e = cudaMalloc(&s->d_done, (size_t)done_off * sizeof(int))) != cudaSuccess ||
      (e = cudaMalloc(&s->d_status, sizeof(int))) != cudaSuccess ||
      (e = cudaMalloc(&s->d_debug, 8 * sizeof(int))) != cudaSuccess)
    return cuda_fail(e, "scan allocation");
  cudaMemset(s->d_status, 0, sizeof(int));
  cudaMemset(s->d_debug, 0, 8 * sizeof(int));
  s->params.desc = s->d_desc;
  s->params.n_desc = s->n_desc;
  s->params.n_classes = n_classes;
  s->params.total = ticket;
  s->params.ticket = s->d_ticket;
  s->params.done = s->d_done;
  s->params.status = s->d_status;
  s->params.spin_limit = kSpinLimit;
  s->params.suspend_ns = knob(WAP_KNOB_SUSPEND) >= 0 ? (unsigned)knob(WAP_KNOB_SUSPEND) : kMbarSuspendNs;
  s->params.stall_pass = -1;
  s->params.checks = 0;
  s->params.debug = s->d_debug;
  return WAP_OK;
}

// issue resets, per-class tables and the persistent kernel for one chain
static int scan_launch(wap_scan* s, bool backward, cudaStream_t st) {
  cudaError_t e;
  if ((e = cudaMemsetAsync(s->d_ticket, 0, sizeof(unsigned long long), st)) != cudaSuccess ||
      (e = cudaMemsetAsync(s->d_done, 0, (size_t)s->total_probes * sizeof(int), st)) != cudaSuccess ||
      (e = cudaMemsetAsync(s->d_status, 0, sizeof(int), st)) != cudaSuccess)
    return cuda_fail(e, "scan reset");
  SchedParams params = s->params;
  params.stage2 = 0;
  int grid = s->grid;
  size_t smem = s->smem;
  if (backward) {
    params.stage2 = s->psi_mode;
    params.cls[0].grad = s->d_gsum;
    const wap_scan_class& c = s->cls[0];
    const long long total = (long long)c.n_probes * c.n * c.n;
    const bool no_dp = !s->params.cls[0].g;   // a loss on the exit wave alone: the seed reads g = 0
    if (no_dp || windowed(s->det[0], c.n)) {
      if (s->d_dpfull.empty()) s->d_dpfull.resize(1, nullptr);
      if (!s->d_dpfull[0] && (e = cudaMalloc(&s->d_dpfull[0], total * sizeof(float))) != cudaSuccess)
        return cuda_fail(e, "cudaMalloc(full-grid seed scratch)");
      if (no_dp) {
        if ((e = cudaMemsetAsync(s->d_dpfull[0], 0, total * sizeof(float), st)) != cudaSuccess)
          return cuda_fail(e, "seed scratch reset");
      } else {
        // the seed reads a full-grid dL/d(dp): zero outside the window
        count_launch();
        scatter_window_kernel<<<(unsigned)std::min<long long>((total + 255) / 256, 148LL * 16), 256, 0, st>>>(
            s->params.cls[0].g, s->d_dpfull[0], total, c.n, s->det[0]);
        if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "scatter_window_kernel");
      }
      params.cls[0].g = s->d_dpfull[0];
    }
    if ((e = cudaMemsetAsync(s->d_gsum, 0, s->ttab_elems[0] * sizeof(float), st)) != cudaSuccess)
      return cuda_fail(e, "gradient sums reset");
    grid = s->grid_bwd;
    smem = s->smem_bwd;
    params.desc = s->d_desc_bwd;
    params.n_desc = s->n_desc_bwd;
    params.total = s->n_tickets_bwd;
    params.cls[0].steps = s->d_steps_bwd;   // gradient scans hold one class
  } else {
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
  (backward ? s->kernel_bwd : s->kernel)<<<grid, kBlockThreads, smem, st>>>(params);
  if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "scan_kernel");
  prof_end(tok, st, bytes);
  if (!backward) {
    for (int ci = 0; ci < s->n_classes; ++ci) {
      const wap_scan_class& c = s->cls[ci];
      if (!c.dp || !windowed(s->det[ci], c.n)) continue;
      const long long total = (long long)c.n_probes * s->det[ci].ny * s->det[ci].nx;
      count_launch();
      crop_window_kernel<<<(unsigned)std::min<long long>((total + 255) / 256, 148LL * 16), 256, 0, st>>>(
          s->d_dpfull[ci], c.dp, total, c.n, s->det[ci]);
      if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "crop_window_kernel");
    }
  }
  if (backward) {
    const Physics& ph = s->phys[0];
    const long long n4 = (long long)s->ttab_elems[0] / 4;
    count_launch();
    grad_finalize_kernel<<<(unsigned)std::min<long long>((n4 + 255) / 256, 148LL * 16), 256, 0, st>>>(
        s->cls[0].V, s->d_gsum, s->params.cls[0].grad, n4, (float)ph.ri_a, (float)ph.ri_inv_den, (float)ph.kphase,
        (float)ph.e_plus_e0);
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "grad_finalize_kernel");
  }
  return WAP_OK;
}

extern "C" {

int wap_scan_create(wap_scan** out, int n_classes, const wap_scan_class* classes) {
  clear_error();
  if (!out) return fail(WAP_ERR_ARG, "scan pointer is NULL");
  *out = nullptr;
  if (n_classes < 1 || n_classes > kMaxClasses || !classes)
    return fail(WAP_ERR_ARG, "n_classes must be in [1, %d]", kMaxClasses);
  wap_scan* s = new wap_scan();
  const int rc = scan_setup(s, n_classes, classes, 0);
  if (rc != WAP_OK) {
    scan_free(s);
    return rc;
  }
  *out = s;
  return WAP_OK;
}

int wap_scan_grad_create(wap_scan** out, const wap_scan_class* cls, int ckpt_every) {
  clear_error();
  if (!out || !cls) return fail(WAP_ERR_ARG, "NULL argument");
  *out = nullptr;
  if (ckpt_every < 1) return fail(WAP_ERR_ARG, "ckpt_every must be >= 1");
  if (!cls->dp) return fail(WAP_ERR_ARG, "the gradient scan needs a dp buffer");
  wap_scan* s = new wap_scan();
  const int rc = scan_setup(s, 1, cls, std::min(ckpt_every, cls->n_slices));
  if (rc != WAP_OK) {
    scan_free(s);
    return rc;
  }
  *out = s;
  return WAP_OK;
}

// Re-point a scan at new buffers with the same shapes (no device allocation):
// pointers of every class and the wave's column-tile tensor map are replaced.
int wap_scan_bind(wap_scan* s, int n_classes, const wap_scan_class* classes) {
  clear_error();
  if (!s || !classes) return fail(WAP_ERR_ARG, "NULL argument");
  if (n_classes != s->n_classes) return fail(WAP_ERR_ARG, "scan has %d classes, got %d", s->n_classes, n_classes);
  PFN_cuTensorMapEncodeTiled_v12000 encode = get_encode();
  if (!encode) return fail(WAP_ERR_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
  for (int ci = 0; ci < n_classes; ++ci) {
    const wap_scan_class& c = classes[ci];
    const wap_scan_class& o = s->cls[ci];
    if (c.n != o.n || c.n_slices != o.n_slices || c.n_draws != o.n_draws || c.n_probes != o.n_probes)
      return fail(WAP_ERR_ARG, "scan class %d: shapes differ from the ones the scan was created for", ci);
    if (!c.V || !c.psi0 || !c.H || !c.exit) return fail(WAP_ERR_ARG, "scan class %d: NULL V/psi0/H/exit", ci);
    if (s->grad && !c.dp) return fail(WAP_ERR_ARG, "the gradient scan needs a dp buffer");
    SchedClass& sc = s->params.cls[ci];
    CUtensorMap map;
    int rc = encode_map(encode, &map, c.exit, c.n, c.n_probes, sc.cols_w, sc.box_rows);
    if (rc) return rc;
    s->params.maps[ci][BUF_PSI] = map;
    sc.psi = reinterpret_cast<float2*>(c.exit);
    sc.psi0 = reinterpret_cast<const float2*>(c.psi0);
    sc.positions = c.positions;
    sc.draw = c.draw;
    sc.V = c.V;
    sc.dp = c.dp;
    if ((rc = bind_detector(s, c, ci))) return rc;
    s->cls[ci] = c;
    s->phys[ci] = physics(c.energy, c.dz);
    const Physics& ph = s->phys[ci];
    sc.ri_a = (float)ph.ri_a;
    sc.ri_inv_den = (float)ph.ri_inv_den;
    sc.kphase = (float)ph.kphase;
    sc.e_plus_e0 = (float)ph.e_plus_e0;
  }
  return WAP_OK;
}

int wap_scan_run(wap_scan* s, void* stream) {
  clear_error();
  if (!s) return fail(WAP_ERR_ARG, "scan is NULL");
  return scan_launch(s, false, (cudaStream_t)stream);
}

int wap_scan_grad_backward(wap_scan* s, const float* grad_dp, float* grad_V, void* stream) {
  clear_error();
  if (!s || !grad_dp || !grad_V) return fail(WAP_ERR_ARG, "NULL argument");
  return wap_scan_grad_backward_ex(s, grad_dp, nullptr, grad_V, stream);
}

int wap_scan_grad_backward_ex(wap_scan* s, const float* grad_dp, const float* grad_exit, float* grad_V,
                              void* stream) {
  clear_error();
  if (!s || !grad_V || (!grad_dp && !grad_exit)) return fail(WAP_ERR_ARG, "need grad_V and grad_dp or grad_exit");
  if (!s->grad) return fail(WAP_ERR_ARG, "scan was not created for gradients");
  cudaStream_t st = (cudaStream_t)stream;
  SchedClass& sc = s->params.cls[0];
  const wap_scan_class& c = s->cls[0];
  sc.g = grad_dp;
  sc.grad = grad_V;
  sc.seed_add = nullptr;
  if (grad_exit) {
    // fft2(grad_exit / 2) into the recompute buffer (free until the first
    // recompute, which the seed precedes in every probe's chain), with the
    // pass kernels and the scan's twiddles; the seed column step adds it
    const int n = c.n, E = 16, T = n / E;
    const long long plane = (long long)n * n;
    RowArgs r{};
    r.psi = sc.work;
    r.psi_bstride = plane;
    r.src = reinterpret_cast<const float2*>(grad_exit);
    r.src_bstride = plane;
    r.tw = s->d_tw_seed;
    r.ny = n;
    r.nx = n;
    r.flags = ROW_LOAD_SRC | ROW_FFT | ROW_SCALE_SRC;
    r.scale = 1.0f;
    r.src_scale = 0.5f;
    ColArgs cc{};
    cc.psi = sc.work;
    cc.psi_bstride = plane;
    cc.tw = s->d_tw_seed;
    cc.ny = n;
    cc.nx = n;
    cc.flags = COL_NO_H | COL_FWD_ONLY;
    cc.det = Detector{0, 0, n, n};
    const int col_w = std::max(2, std::min(16, kColThreads / T));
    cudaError_t e;
    for (int b0 = 0; b0 < c.n_probes; b0 += 65535) {
      const int nb = std::min(65535, c.n_probes - b0);
      r.probe0 = b0;
      cc.probe0 = b0;
      if ((e = launch_row(n, E, r, nb, rows_per_cta(n, E, n), st)) != cudaSuccess) return cuda_fail(e, "exit seed rows");
      if ((e = launch_col(n, E, cc, nb, col_w, st)) != cudaSuccess) return cuda_fail(e, "exit seed columns");
    }
    sc.seed_add = sc.work;
  }
  return scan_launch(s, true, st);
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

int wap_scan_status_async(wap_scan* s, int* host_status, void* stream) {
  clear_error();
  if (!s || !host_status) return fail(WAP_ERR_ARG, "NULL argument");
  cudaError_t e = cudaMemcpyAsync(host_status, s->d_status, sizeof(int), cudaMemcpyDeviceToHost, (cudaStream_t)stream);
  if (e != cudaSuccess) return cuda_fail(e, "scan status copy");
  return WAP_OK;
}

int wap_scan_debug_override(int which, int value) {
  clear_error();
  if (which < 0 || which >= WAP_KNOB_COUNT) return fail(WAP_ERR_ARG, "unknown scheduler override %d", which);
  g_knob[which] = value < 0 ? -1 : value;
  return WAP_OK;
}

int wap_scan_info(const wap_scan* s, long long* tickets, int* grid, int* group0) {
  clear_error();
  if (!s || !tickets || !grid || !group0) return fail(WAP_ERR_ARG, "NULL argument");
  *tickets = s->n_tickets;
  *grid = s->grid;
  *group0 = s->groups.empty() ? 0 : s->groups[0];
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
    cudaError_t e = cudaMemcpy(record, s->d_debug, 8 * sizeof(int), cudaMemcpyDeviceToHost);
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
