// Well-separated proxy interactions of the decoupled-degree treecode
// (q = (n+1)^2 proxies, n = 5..10) over chunks of the interaction list.
//
// The reference evaluates each (target panel, source panel) pair of its
// interaction list with a loop over the proxies
// (src/fmm_interactions/bve_vel.cpp:35-150).  Here the treecode's
// well-separated list (CSR by target panel) is cut into chunks of at most C
// consecutive entries of one target panel (near-equal lengths), and a block
// evaluates S chunks side by side.  One block of four warps per target panel
// (k_interact_wide) runs a target's whole list in one block and leaves
// (32 - q mod 32) lanes of its last warp idle; chunks spread long lists over
// the GPU, and the slots fill the warps (81 proxies: 3 slots in 256
// threads).  Each slot writes the raw sums a = sum g d of its chunk (float64)
// to its own row; k_cc_reduce adds a target's chunks in list order and
// applies the cross product.  The result depends on C (the order of the
// float64 additions), not on S.
#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "../../include/sbslpm.h"
#include "bve_kernels.cuh"
#include "cc_tcgen05.cuh"
#include "device_common.cuh"

namespace sbslpm {
namespace {

using dev::blocks_for;
using dev::pair32x2;
using dev::pair64;

// A block holds S chunk slots of Q target proxies each: thread k works on
// target node k % Q of slot k / Q (threads past S*Q idle), so that a block
// of a multiple of 32 threads leaves few lanes idle for any Q.  Every slot
// walks its own chunk, staging one source panel at a time in its own part of
// the shared tile.  (Loading the next panel into registers during the
// current one, with a double-buffered tile, measured slower: the extra
// registers cost more occupancy than the barrier it saves.)
template <int Q, int S>
struct CcShape {
  static constexpr int NT = (S * Q + 31) / 32 * 32;
  static constexpr bool ok = NT <= 512 && 5 * S * Q >= 4 * NT;  // at most a fifth of the lanes idle
};

__device__ __forceinline__ int chunk_entries_max(const int4* __restrict__ chunks, int nchunks, int first, int S) {
  int m = 0;
  for (int h = 0; h < S && first + h < nchunks; h++) {
    const int4 c = chunks[first + h];
    m = max(m, c.z - c.y);
  }
  return m;
}

// Mixed precision: proxies relative to panel centres (kPackScale), float32
// pairs two at a time (FADD2 / FFMA2 / FMUL2), per-source-panel float32 sums
// added into float64.
template <int Q, int S, bool GUARD>
__global__ void __launch_bounds__(CcShape<Q, S>::NT)
    k_cc32(StepGeom g, const int4* __restrict__ chunks, int nchunks, double* __restrict__ partial) {
  constexpr int Q2 = (Q + 1) / 2;
  __shared__ float4 tile[S][2 * Q2];  // (x0,x1,y0,y1),(z0,z1,w0,w1); odd q: zero-strength partner
  const int h = threadIdx.x / Q, j = threadIdx.x - h * Q;
  const int c = blockIdx.x * S + h;
  const bool live = h < S && c < nchunks;
  const int nmax = chunk_entries_max(chunks, nchunks, blockIdx.x * S, S);
  int4 ch = make_int4(0, 0, 0, 0);
  if (live) ch = chunks[c];
  const int n = ch.z - ch.y;
  const long pn = (long)g.panels * Q;
  double cx = 0, cy = 0, cz = 0;
  float dtx = 0, dty = 0, dtz = 0;
  if (live) {
    const double* ct = g.pd_centre + 4 * (long)ch.x;
    cx = ct[0];
    cy = ct[1];
    cz = ct[2];
    const long o = (long)ch.x * Q + j;
    dtx = (float)((g.px[o] - cx) * kPackScale);
    dty = (float)((g.px[pn + o] - cy) * kPackScale);
    dtz = (float)((g.px[2 * pn + o] - cz) * kPackScale);
  }
  const float feps = (float)g.eps;
  const float2 eps2 = make_float2(feps, feps);
  double ax = 0, ay = 0, az = 0;
  for (int e = 0; e < nmax; e++) {
    const bool act = live && e < n;
    int sp = 0;
    if (act) sp = __ldg(g.src_panel + ch.y + e);
    __syncthreads();
    if (act && j < Q2) {
      const long sb = (long)sp * Q + 2 * j;
      const float4 s0 = g.srcf[sb];
      const float4 s1 = (2 * j + 1 < Q) ? g.srcf[sb + 1] : make_float4(0.f, 0.f, 0.f, 0.f);
      tile[h][2 * j] = make_float4(s0.x, s1.x, s0.y, s1.y);
      tile[h][2 * j + 1] = make_float4(s0.z, s1.z, s0.w, s1.w);
    }
    __syncthreads();
    if (act) {
      const double* cs = g.pd_centre + 4 * (long)sp;
      const float b0 = (float)((cs[0] - cx) * kPackScale) - dtx, b1 = (float)((cs[1] - cy) * kPackScale) - dty,
                  b2 = (float)((cs[2] - cz) * kPackScale) - dtz;
      const float2 bx = make_float2(b0, b0), by = make_float2(b1, b1), bz = make_float2(b2, b2);
      float2 fx = make_float2(0.f, 0.f), fy = fx, fz = fx;
      const float4* tb = tile[h];
#pragma unroll 8
      for (int k2 = 0; k2 < Q2; k2++) {
        const float4 A = tb[2 * k2], B = tb[2 * k2 + 1];
        pair32x2<GUARD>(bx, by, bz, make_float2(A.x, A.y), make_float2(A.z, A.w), make_float2(B.x, B.y),
                        make_float2(B.z, B.w), eps2, fx, fy, fz);
      }
      ax += (double)fx.x + (double)fx.y;
      ay += (double)fy.x + (double)fy.y;
      az += (double)fz.x + (double)fz.y;
    }
  }
  if (live) {
    double* p = partial + (long)c * 3 * Q;
    p[j] = ax;
    p[Q + j] = ay;
    p[2 * Q + j] = az;
  }
}

// Mixed precision without shared-memory staging: the source proxies are read
// straight from a pair-transposed copy (srcp: per panel, proxies (2k, 2k+1)
// as (x0,x1,y0,y1),(z0,z1,w0,w1), a zero-strength partner after an odd
// count) through the L1 cache, where a warp's lanes share every 16-byte
// load, so a slot walks its chunk with no barrier at all.  A thread holds TPT
// target proxies (j, j + QT, ...), so each pair of source loads feeds TPT
// targets.
template <int Q, int S, int TPT>
struct CcDirectShape {
  static constexpr int QT = (Q + TPT - 1) / TPT;  // threads per slot
  static constexpr int NT = (S * QT + 31) / 32 * 32;
  static constexpr bool ok = NT <= 512 && 5 * S * QT >= 4 * NT;  // at most a fifth of the lanes idle
};

template <int Q, int S, int TPT, bool GUARD>
__global__ void __launch_bounds__(CcDirectShape<Q, S, TPT>::NT)
    k_cc32d(StepGeom g, const int4* __restrict__ chunks, int nchunks, const float4* __restrict__ srcp,
            double* __restrict__ partial) {
  constexpr int Q2 = (Q + 1) / 2, QT = CcDirectShape<Q, S, TPT>::QT;
  const int h = threadIdx.x / QT, jt = threadIdx.x - h * QT;
  const int c = blockIdx.x * S + h;
  if (h >= S || c >= nchunks) return;  // no barrier below: idle lanes leave
  const int4 ch = chunks[c];
  const long pn = (long)g.panels * Q;
  const double* ct = g.pd_centre + 4 * (long)ch.x;
  const double cx = ct[0], cy = ct[1], cz = ct[2];
  float dtx[TPT], dty[TPT], dtz[TPT];
  double ax[TPT], ay[TPT], az[TPT];
#pragma unroll
  for (int r = 0; r < TPT; r++) {
    const int j = jt + r * QT;
    const long o = (long)ch.x * Q + (j < Q ? j : 0);
    dtx[r] = (float)((g.px[o] - cx) * kPackScale);
    dty[r] = (float)((g.px[pn + o] - cy) * kPackScale);
    dtz[r] = (float)((g.px[2 * pn + o] - cz) * kPackScale);
    ax[r] = ay[r] = az[r] = 0;
  }
  const float feps = (float)g.eps;
  const float2 eps2 = make_float2(feps, feps);
  for (int e = ch.y; e < ch.z; e++) {
    const int sp = __ldg(g.src_panel + e);
    const double* cs = g.pd_centre + 4 * (long)sp;
    const float bx0 = (float)((cs[0] - cx) * kPackScale), by0 = (float)((cs[1] - cy) * kPackScale),
                bz0 = (float)((cs[2] - cz) * kPackScale);
    float2 bx[TPT], by[TPT], bz[TPT], fx[TPT], fy[TPT], fz[TPT];
#pragma unroll
    for (int r = 0; r < TPT; r++) {
      const float b0 = bx0 - dtx[r], b1 = by0 - dty[r], b2 = bz0 - dtz[r];
      bx[r] = make_float2(b0, b0);
      by[r] = make_float2(b1, b1);
      bz[r] = make_float2(b2, b2);
      fx[r] = fy[r] = fz[r] = make_float2(0.f, 0.f);
    }
    const float4* sb = srcp + (long)sp * 2 * Q2;
#pragma unroll 8
    for (int k2 = 0; k2 < Q2; k2++) {
      const float4 A = __ldg(sb + 2 * k2), B = __ldg(sb + 2 * k2 + 1);
      const float2 sx = make_float2(A.x, A.y), sy = make_float2(A.z, A.w), sz = make_float2(B.x, B.y),
                   sw = make_float2(B.z, B.w);
#pragma unroll
      for (int r = 0; r < TPT; r++) pair32x2<GUARD>(bx[r], by[r], bz[r], sx, sy, sz, sw, eps2, fx[r], fy[r], fz[r]);
    }
#pragma unroll
    for (int r = 0; r < TPT; r++) {
      ax[r] += (double)fx[r].x + (double)fx[r].y;
      ay[r] += (double)fy[r].x + (double)fy[r].y;
      az[r] += (double)fz[r].x + (double)fz[r].y;
    }
  }
  double* p = partial + (long)c * 3 * Q;
#pragma unroll
  for (int r = 0; r < TPT; r++) {
    const int j = jt + r * QT;
    if (j >= Q) continue;
    p[j] = ax[r];
    p[Q + j] = ay[r];
    p[2 * Q + j] = az[r];
  }
}

// Mixed precision with the source proxies brought into shared memory by the
// bulk-copy engine (TMA, cp.async.bulk): each slot owns two buffers of one
// source panel's pair-transposed proxies (Q2 x 32 bytes, contiguous in srcp)
// and two pairs of mbarriers.  The slot's first thread issues the copies of
// its chunk's first two entries at once and each later one as soon as all
// the slot's threads have released the buffer (empty barrier), so the next
// panel arrives while the current one is evaluated, and no barrier spans the
// block.  Every wait is bounded (0.2 s of %globaltimer): one that runs out
// sets kErrTimeout and the slot stops.
__device__ __forceinline__ unsigned long long cc_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ bool cc_mbar_wait(uint32_t bar, uint32_t parity) {
  const unsigned long long t0 = cc_ns();
  while (true) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
    if (cc_ns() - t0 > 200000000ull) return false;
  }
}

__device__ __forceinline__ void cc_bulk_load(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" : : "r"(bar), "r"(bytes) : "memory");
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
               :
               : "r"(dst), "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}

template <int Q, int S, bool GUARD>
__global__ void __launch_bounds__(CcShape<Q, S>::NT)
    k_cc32t(StepGeom g, const int4* __restrict__ chunks, int nchunks, const float4* __restrict__ srcp,
            double* __restrict__ partial) {
  constexpr int Q2 = (Q + 1) / 2;
  constexpr uint32_t kBytes = Q2 * 32;
  __shared__ __align__(128) float4 buf[S][2][2 * Q2];
  __shared__ __align__(8) unsigned long long full[S][2], empty[S][2];
  const int h = threadIdx.x / Q, j = threadIdx.x - h * Q;
  const int c = blockIdx.x * S + h;
  if (threadIdx.x == 0) {
    for (int k = 0; k < S; k++)
      for (int b = 0; b < 2; b++) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" : : "r"((uint32_t)__cvta_generic_to_shared(&full[k][b]))
                     : "memory");
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;"
                     :
                     : "r"((uint32_t)__cvta_generic_to_shared(&empty[k][b])), "r"(Q)
                     : "memory");
      }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (h >= S || c >= nchunks) return;  // no block-wide barrier below
  const int4 ch = chunks[c];
  const int n = ch.z - ch.y;
  const bool producer = j == 0;
  // shared-memory addresses of buffer / barrier b of this slot: base + b * stride
  const uint32_t f0 = (uint32_t)__cvta_generic_to_shared(&full[h][0]);
  const uint32_t e0 = (uint32_t)__cvta_generic_to_shared(&empty[h][0]);
  const uint32_t d0 = (uint32_t)__cvta_generic_to_shared(&buf[h][0][0]);
  auto fb = [&](int b) { return f0 + 8u * (uint32_t)b; };
  auto eb = [&](int b) { return e0 + 8u * (uint32_t)b; };
  auto db = [&](int b) { return d0 + kBytes * (uint32_t)b; };
  if (producer) {
    for (int e = 0; e < n && e < 2; e++)
      cc_bulk_load(db(e), srcp + (long)__ldg(g.src_panel + ch.y + e) * 2 * Q2, kBytes, fb(e));
  }
  const long pn = (long)g.panels * Q;
  const double* ct = g.pd_centre + 4 * (long)ch.x;
  const double cx = ct[0], cy = ct[1], cz = ct[2];
  const long o = (long)ch.x * Q + j;
  const float dtx = (float)((g.px[o] - cx) * kPackScale), dty = (float)((g.px[pn + o] - cy) * kPackScale),
              dtz = (float)((g.px[2 * pn + o] - cz) * kPackScale);
  const float feps = (float)g.eps;
  const float2 eps2 = make_float2(feps, feps);
  double ax = 0, ay = 0, az = 0;
  bool ok = true;
  for (int e = 0; e < n; e++) {
    const int b = e & 1;
    const uint32_t par = (uint32_t)((e >> 1) & 1);
    if (!cc_mbar_wait(fb(b), par)) {
      ok = false;
      break;
    }
    const int sp = __ldg(g.src_panel + ch.y + e);
    const double* cs = g.pd_centre + 4 * (long)sp;
    const float b0 = (float)((cs[0] - cx) * kPackScale) - dtx, b1 = (float)((cs[1] - cy) * kPackScale) - dty,
                b2 = (float)((cs[2] - cz) * kPackScale) - dtz;
    const float2 bx = make_float2(b0, b0), by = make_float2(b1, b1), bz = make_float2(b2, b2);
    float2 fx = make_float2(0.f, 0.f), fy = fx, fz = fx;
    const float4* tb = buf[h][b];
#pragma unroll 8
    for (int k2 = 0; k2 < Q2; k2++) {
      const float4 A = tb[2 * k2], B = tb[2 * k2 + 1];
      pair32x2<GUARD>(bx, by, bz, make_float2(A.x, A.y), make_float2(A.z, A.w), make_float2(B.x, B.y),
                      make_float2(B.z, B.w), eps2, fx, fy, fz);
    }
    ax += (double)fx.x + (double)fx.y;
    ay += (double)fy.x + (double)fy.y;
    az += (double)fz.x + (double)fz.y;
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" : : "r"(eb(b)) : "memory");
    if (producer && e + 2 < n) {  // refill this buffer once the slot has released it
      if (!cc_mbar_wait(eb(b), par)) {
        // the copy of entry e + 1 may still be in flight: let it land (bounded) before leaving
        cc_mbar_wait(fb(b ^ 1), (uint32_t)(((e + 1) >> 1) & 1));
        ok = false;
        break;
      }
      cc_bulk_load(db(b), srcp + (long)__ldg(g.src_panel + ch.y + e + 2) * 2 * Q2, kBytes, fb(b));
    }
  }
  if (!ok) {
    dev::flag(g.err, kErrTimeout);
    return;
  }
  double* p = partial + (long)c * 3 * Q;
  p[j] = ax;
  p[Q + j] = ay;
  p[2 * Q + j] = az;
}

// Mixed precision, one warp per chunk: the warp's lanes hold the target
// panel's Q proxies, TPT = ceil(Q / 32) per lane (j = lane + 32 r), so that
// every staged source pair feeds TPT targets; each warp stages its chunk's
// source panels in its own two shared-memory buffers with cp.async (16 bytes
// per lane, the next entry's panel in flight while the current one is
// evaluated) and synchronises with __syncwarp only -- no barrier spans the
// block, and warps of a block never wait for each other.  The pair
// arithmetic and the order of every target's sums are those of k_cc32, so
// the result is bit-identical to the staged form's.
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;"
               :
               : "r"((uint32_t)__cvta_generic_to_shared(smem)), "l"(gmem)
               : "memory");
}

template <int Q>
struct CcWarpShape {
  static constexpr int TPT = (Q + 31) / 32;  // target proxies per lane
  static constexpr int Q2 = (Q + 1) / 2;
  static constexpr int NF4 = 2 * Q2;  // float4 per staged source panel
};

template <int Q, int WPB, bool GUARD>
__global__ void __launch_bounds__(32 * WPB)
    k_cc32w(StepGeom g, const int4* __restrict__ chunks, int nchunks, const float4* __restrict__ srcp,
            double* __restrict__ partial) {
  using Sh = CcWarpShape<Q>;
  constexpr int TPT = Sh::TPT, Q2 = Sh::Q2, NF4 = Sh::NF4;
  __shared__ __align__(16) float4 buf[WPB][2][NF4];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int c = blockIdx.x * WPB + warp;
  if (c >= nchunks) return;  // the whole warp: nothing below waits on other warps
  const int4 ch = chunks[c];
  const int n = ch.z - ch.y;
  const long pn = (long)g.panels * Q;
  const double* ct = g.pd_centre + 4 * (long)ch.x;
  const double cx = ct[0], cy = ct[1], cz = ct[2];
  float dtx[TPT], dty[TPT], dtz[TPT];
  double ax[TPT], ay[TPT], az[TPT];
#pragma unroll
  for (int r = 0; r < TPT; r++) {
    const int j = lane + 32 * r;
    const long o = (long)ch.x * Q + (j < Q ? j : 0);
    dtx[r] = (float)((g.px[o] - cx) * kPackScale);
    dty[r] = (float)((g.px[pn + o] - cy) * kPackScale);
    dtz[r] = (float)((g.px[2 * pn + o] - cz) * kPackScale);
    ax[r] = ay[r] = az[r] = 0;
  }
  auto stage = [&](int e) {  // entry e's source panel into buffer e & 1 (one cp.async group per call)
    if (e < n) {
      const float4* s = srcp + (long)__ldg(g.src_panel + ch.y + e) * NF4;
      float4* d = buf[warp][e & 1];
      for (int k = lane; k < NF4; k += 32) cp_async16(d + k, s + k);
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
  };
  stage(0);
  const float feps = (float)g.eps;
  const float2 eps2 = make_float2(feps, feps);
  for (int e = 0; e < n; e++) {
    stage(e + 1);  // the next panel flies while this one is evaluated
    asm volatile("cp.async.wait_group 1;" ::: "memory");
    __syncwarp();
    const int sp = __ldg(g.src_panel + ch.y + e);
    const double* cs = g.pd_centre + 4 * (long)sp;
    const float bx0 = (float)((cs[0] - cx) * kPackScale), by0 = (float)((cs[1] - cy) * kPackScale),
                bz0 = (float)((cs[2] - cz) * kPackScale);
    float2 bx[TPT], by[TPT], bz[TPT], fx[TPT], fy[TPT], fz[TPT];
#pragma unroll
    for (int r = 0; r < TPT; r++) {
      const float b0 = bx0 - dtx[r], b1 = by0 - dty[r], b2 = bz0 - dtz[r];
      bx[r] = make_float2(b0, b0);
      by[r] = make_float2(b1, b1);
      bz[r] = make_float2(b2, b2);
      fx[r] = fy[r] = fz[r] = make_float2(0.f, 0.f);
    }
    const float4* tb = buf[warp][e & 1];
#pragma unroll 4
    for (int k2 = 0; k2 < Q2; k2++) {
      const float4 A = tb[2 * k2], B = tb[2 * k2 + 1];
      const float2 sx = make_float2(A.x, A.y), sy = make_float2(A.z, A.w), sz = make_float2(B.x, B.y),
                   sw = make_float2(B.z, B.w);
#pragma unroll
      for (int r = 0; r < TPT; r++) pair32x2<GUARD>(bx[r], by[r], bz[r], sx, sy, sz, sw, eps2, fx[r], fy[r], fz[r]);
    }
#pragma unroll
    for (int r = 0; r < TPT; r++) {
      ax[r] += (double)fx[r].x + (double)fx[r].y;
      ay[r] += (double)fy[r].x + (double)fy[r].y;
      az[r] += (double)fz[r].x + (double)fz[r].y;
    }
    __syncwarp();  // every lane is done with this buffer before stage(e + 2) refills it
  }
  asm volatile("cp.async.wait_group 0;" ::: "memory");
  double* p = partial + (long)c * 3 * Q;
#pragma unroll
  for (int r = 0; r < TPT; r++) {
    const int j = lane + 32 * r;
    if (j >= Q) continue;
    p[j] = ax[r];
    p[Q + j] = ay[r];
    p[2 * Q + j] = az[r];
  }
}

// The pair-transposed copy of the packed proxy sources that k_cc32d reads.
__global__ void k_cc_pair_sources(const float4* __restrict__ srcf, int q, long pairs, float4* __restrict__ srcp) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= pairs) return;
  const int q2 = (q + 1) / 2;
  const long p = i / q2;
  const int k = (int)(i - p * q2);
  const float4 s0 = srcf[p * q + 2 * k];
  const float4 s1 = 2 * k + 1 < q ? srcf[p * q + 2 * k + 1] : make_float4(0.f, 0.f, 0.f, 0.f);
  srcp[2 * i] = make_float4(s0.x, s1.x, s0.y, s1.y);
  srcp[2 * i + 1] = make_float4(s0.z, s1.z, s0.w, s1.w);
}

// Float64: the same slots and chunks with absolute proxy positions (pair64).
template <int Q, int S, bool GUARD>
__global__ void __launch_bounds__(CcShape<Q, S>::NT)
    k_cc64(StepGeom g, const int4* __restrict__ chunks, int nchunks, const double4* __restrict__ src,
           double* __restrict__ partial) {
  __shared__ double4 tile[S][Q];
  const int h = threadIdx.x / Q, j = threadIdx.x - h * Q;
  const int c = blockIdx.x * S + h;
  const bool live = h < S && c < nchunks;
  const int nmax = chunk_entries_max(chunks, nchunks, blockIdx.x * S, S);
  int4 ch = make_int4(0, 0, 0, 0);
  if (live) ch = chunks[c];
  const int n = ch.z - ch.y;
  const long pn = (long)g.panels * Q;
  double tx = 0, ty = 0, tz = 0;
  if (live) {
    const long o = (long)ch.x * Q + j;
    tx = g.px[o];
    ty = g.px[pn + o];
    tz = g.px[2 * pn + o];
  }
  double ax = 0, ay = 0, az = 0;
  for (int e = 0; e < nmax; e++) {
    const bool act = live && e < n;
    __syncthreads();
    if (act) tile[h][j] = src[(long)__ldg(g.src_panel + ch.y + e) * Q + j];
    __syncthreads();
    if (act) {
      const double4* tb = tile[h];
#pragma unroll 3
      for (int k = 0; k < Q; k++) pair64<GUARD>(tx, ty, tz, tb[k], g.eps, ax, ay, az);
    }
  }
  if (live) {
    double* p = partial + (long)c * 3 * Q;
    p[j] = ax;
    p[Q + j] = ay;
    p[2 * Q + j] = az;
  }
}

// Target proxy velocities: a target's chunk sums added in list order, then
// u = cb * x cross a.  Panels with no entries get zeros.
__global__ void k_cc_reduce(StepGeom g, const int* __restrict__ cstart, const double* __restrict__ partial, double cb,
                            double* __restrict__ out) {
  const int q = g.q;
  const long pn = (long)g.panels * q;
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= pn) return;
  const int t = (int)(i / q), j = (int)(i - (long)t * q);
  double sx = 0, sy = 0, sz = 0;
  for (int c = cstart[t]; c < cstart[t + 1]; c++) {
    const double* p = partial + (long)c * 3 * q;
    sx += p[j];
    sy += p[q + j];
    sz += p[2 * q + j];
  }
  const double px = g.px[i], py = g.px[pn + i], pz = g.px[2 * pn + i];
  out[i] = cb * (py * sz - pz * sy);
  out[pn + i] = cb * (pz * sx - px * sz);
  out[2 * pn + i] = cb * (px * sy - py * sx);
}

// Batched ensembles: the well-separated interactions of a proxy-degree group
// for MB members at once.  Treecode proxies never move, so a cluster pair's
// differences, distances and reciprocals are the same for every member; they
// are evaluated once per pair of the group's union list and applied to the MB
// members' strengths with the paired float32 instructions across members.
// One block per (target cluster, member group of MB consecutive group bits,
// the members being theta-sorted), a thread per target proxy; a member
// outside an entry's bits takes zero strength there.  Per member and source
// cluster: float32 sums added into float64; every (target, member) of the
// group is written (zeros without entries).
// members per group of the shared well-separated kernel (4 measured faster
// than 8 there: fewer registers, more resident blocks)
constexpr int kCcGroup = 4;

template <int Q, int MB, bool GUARD>
__global__ void __launch_bounds__((Q + 31) / 32 * 32) k_cc_multi(CcTcGroup g) {
  constexpr int Q2 = (Q + 1) / 2;
  __shared__ float4 tq[2 * Q2];   // (x0,x1,y0,y1),(z0,z1,0,0)
  __shared__ float wt[2 * Q2][MB];
  const int T = blockIdx.x, grp = blockIdx.y, j = threadIdx.x;
  const bool tgt = j < Q;
  const float4* sf[MB];
  int valid = 0;
#pragma unroll
  for (int m = 0; m < MB; m++) {
    const int jg = grp * MB + m;
    sf[m] = jg < g.nmem ? g.mem[g.idx[jg]].fg.srcf : nullptr;
    if (jg < g.nmem) valid |= 1 << m;
  }
  const double* ct = g.centre + 4 * (long)T;
  const float4 self = tgt ? g.pxf[(long)T * Q + j] : make_float4(0.f, 0.f, 0.f, 0.f);
  double ax[MB], ay[MB], az[MB];
#pragma unroll
  for (int m = 0; m < MB; m++) ax[m] = ay[m] = az[m] = 0;
  const float feps = (float)g.eps;
  const float2 eps2 = make_float2(feps, feps);
  const int word = (grp * MB) >> 5, shift = (grp * MB) & 31;
  for (int e = g.ustart[T]; e < g.ustart[T + 1]; e++) {
    const int bits = (int)((__ldg(g.umask + (long)e * g.mw + word) >> shift) & ((1u << MB) - 1)) & valid;
    if (!bits) continue;
    const int S = __ldg(g.usrc + e);
    const double* cs = g.centre + 4 * (long)S;
    const float bx0 = (float)((cs[0] - ct[0]) * kPackScale), by0 = (float)((cs[1] - ct[1]) * kPackScale),
                bz0 = (float)((cs[2] - ct[2]) * kPackScale);
    __syncthreads();
    if (j < Q2) {
      const float4 s0 = g.pxf[(long)S * Q + 2 * j];
      const float4 s1 = 2 * j + 1 < Q ? g.pxf[(long)S * Q + 2 * j + 1] : make_float4(0.f, 0.f, 0.f, 0.f);
      tq[2 * j] = make_float4(s0.x, s1.x, s0.y, s1.y);
      tq[2 * j + 1] = make_float4(s0.z, s1.z, 0.f, 0.f);
    }
    if (j < 2 * Q2) {
#pragma unroll
      for (int m = 0; m < MB; m++)
        wt[j][m] = (j < Q && ((bits >> m) & 1)) ? sf[m][(long)S * Q + j].w : 0.f;
    }
    __syncthreads();
    if (tgt) {
      const float b0 = bx0 - self.x, b1 = by0 - self.y, b2 = bz0 - self.z;
      const float2 bx = make_float2(b0, b0), by = make_float2(b1, b1), bz = make_float2(b2, b2);
      float2 fx[MB / 2], fy[MB / 2], fz[MB / 2];
#pragma unroll
      for (int p = 0; p < MB / 2; p++) fx[p] = fy[p] = fz[p] = make_float2(0.f, 0.f);
#pragma unroll 6
      for (int k2 = 0; k2 < Q2; k2++) {
        const float4 A = tq[2 * k2], B = tq[2 * k2 + 1];
        const float2 dx = __fadd2_rn(bx, make_float2(A.x, A.y)), dy = __fadd2_rn(by, make_float2(A.z, A.w)),
                     dz = __fadd2_rn(bz, make_float2(B.x, B.y));
        const float2 den = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __ffma2_rn(dz, dz, eps2)));
        float r0 = dev::recip_f32(den.x), r1 = dev::recip_f32(den.y);
        if (GUARD) {
          r0 = den.x > 0.0f ? r0 : 0.0f;
          r1 = den.y > 0.0f ? r1 : 0.0f;
        }
        const float2* w0 = reinterpret_cast<const float2*>(&wt[2 * k2][0]);
        const float2* w1 = reinterpret_cast<const float2*>(&wt[2 * k2 + 1][0]);
#pragma unroll
        for (int p = 0; p < MB / 2; p++) {
          const float2 g0 = __fmul2_rn(w0[p], make_float2(r0, r0)), g1 = __fmul2_rn(w1[p], make_float2(r1, r1));
          fx[p] = __ffma2_rn(g0, make_float2(dx.x, dx.x), fx[p]);
          fy[p] = __ffma2_rn(g0, make_float2(dy.x, dy.x), fy[p]);
          fz[p] = __ffma2_rn(g0, make_float2(dz.x, dz.x), fz[p]);
          fx[p] = __ffma2_rn(g1, make_float2(dx.y, dx.y), fx[p]);
          fy[p] = __ffma2_rn(g1, make_float2(dy.y, dy.y), fy[p]);
          fz[p] = __ffma2_rn(g1, make_float2(dz.y, dz.y), fz[p]);
        }
      }
#pragma unroll
      for (int p = 0; p < MB / 2; p++) {
        ax[2 * p] += (double)fx[p].x;
        ay[2 * p] += (double)fy[p].x;
        az[2 * p] += (double)fz[p].x;
        ax[2 * p + 1] += (double)fx[p].y;
        ay[2 * p + 1] += (double)fy[p].y;
        az[2 * p + 1] += (double)fz[p].y;
      }
    }
  }
  if (!tgt) return;
  const long pn = (long)g.Pf * Q, o = (long)T * Q + j;
  const double px = g.px[o], py = g.px[pn + o], pz = g.px[2 * pn + o];
#pragma unroll
  for (int m = 0; m < MB; m++) {
    if (!((valid >> m) & 1)) continue;
    double* out = g.mem[g.idx[grp * MB + m]].ftgt;
    out[o] = kBiotSavartPacked * (py * az[m] - pz * ay[m]);
    out[pn + o] = kBiotSavartPacked * (pz * ax[m] - px * az[m]);
    out[2 * pn + o] = kBiotSavartPacked * (px * ay[m] - py * ax[m]);
  }
}

template <int Q>
void launch_multi_q(const CcTcGroup& g, cudaStream_t st) {
  constexpr int MB = kCcGroup, NT = (Q + 31) / 32 * 32;
  const dim3 grid((unsigned)g.Pf, (unsigned)((g.nmem + MB - 1) / MB));
  if (!(g.eps > 0)) SB_LAUNCH((k_cc_multi<Q, MB, true>), grid, NT, 0, st, g);
  else SB_LAUNCH((k_cc_multi<Q, MB, false>), grid, NT, 0, st, g);
}

template <int Q, int S>
void launch_q_s(const StepGeom& g, bool mixed, const int4* chunks, int nchunks, const double4* src, double* partial,
                cudaStream_t st) {
  if constexpr (CcShape<Q, S>::ok) {
    constexpr int NT = CcShape<Q, S>::NT;
    const unsigned grid = (unsigned)((nchunks + S - 1) / S);
    const bool guard = !(g.eps > 0);
    if (mixed) {
      if (guard) SB_LAUNCH((k_cc32<Q, S, true>), grid, NT, 0, st, g, chunks, nchunks, partial);
      else SB_LAUNCH((k_cc32<Q, S, false>), grid, NT, 0, st, g, chunks, nchunks, partial);
    } else {
      if (guard) SB_LAUNCH((k_cc64<Q, S, true>), grid, NT, 0, st, g, chunks, nchunks, src, partial);
      else SB_LAUNCH((k_cc64<Q, S, false>), grid, NT, 0, st, g, chunks, nchunks, src, partial);
    }
  }
}

template <int Q, int S, int TPT>
void launch_direct_s(const StepGeom& g, const int4* chunks, int nchunks, const float4* srcp, double* partial,
                     cudaStream_t st) {
  if constexpr (CcDirectShape<Q, S, TPT>::ok) {
    constexpr int NT = CcDirectShape<Q, S, TPT>::NT;
    const unsigned grid = (unsigned)((nchunks + S - 1) / S);
    if (!(g.eps > 0)) SB_LAUNCH((k_cc32d<Q, S, TPT, true>), grid, NT, 0, st, g, chunks, nchunks, srcp, partial);
    else SB_LAUNCH((k_cc32d<Q, S, TPT, false>), grid, NT, 0, st, g, chunks, nchunks, srcp, partial);
  }
}

template <int Q, int TPT>
void launch_direct_t(const StepGeom& g, int slots, const int4* chunks, int nchunks, const float4* srcp,
                     double* partial, cudaStream_t st) {
  switch (slots) {
    case 1: launch_direct_s<Q, 1, TPT>(g, chunks, nchunks, srcp, partial, st); break;
    case 2: launch_direct_s<Q, 2, TPT>(g, chunks, nchunks, srcp, partial, st); break;
    case 3: launch_direct_s<Q, 3, TPT>(g, chunks, nchunks, srcp, partial, st); break;
    case 4: launch_direct_s<Q, 4, TPT>(g, chunks, nchunks, srcp, partial, st); break;
    case 6: launch_direct_s<Q, 6, TPT>(g, chunks, nchunks, srcp, partial, st); break;
    default: launch_direct_s<Q, 8, TPT>(g, chunks, nchunks, srcp, partial, st); break;
  }
}

template <int Q, int S>
void launch_bulk_s(const StepGeom& g, const int4* chunks, int nchunks, const float4* srcp, double* partial,
                   cudaStream_t st) {
  if constexpr (CcShape<Q, S>::ok) {
    constexpr int NT = CcShape<Q, S>::NT;
    const unsigned grid = (unsigned)((nchunks + S - 1) / S);
    if (!(g.eps > 0)) SB_LAUNCH((k_cc32t<Q, S, true>), grid, NT, 0, st, g, chunks, nchunks, srcp, partial);
    else SB_LAUNCH((k_cc32t<Q, S, false>), grid, NT, 0, st, g, chunks, nchunks, srcp, partial);
  }
}

template <int Q>
void launch_warp_q(const StepGeom& g, int warps, const int4* chunks, int nchunks, const float4* srcp,
                   double* partial, cudaStream_t st) {
  const bool guard = !(g.eps > 0);
#define SB_WQ(W)                                                                                          \
  case W: {                                                                                               \
    const unsigned grid = (unsigned)((nchunks + W - 1) / W);                                              \
    if (guard) SB_LAUNCH((k_cc32w<Q, W, true>), grid, 32 * W, 0, st, g, chunks, nchunks, srcp, partial);  \
    else SB_LAUNCH((k_cc32w<Q, W, false>), grid, 32 * W, 0, st, g, chunks, nchunks, srcp, partial);       \
    break;                                                                                                \
  }
  switch (warps) { SB_WQ(1) SB_WQ(2) SB_WQ(4) default: SB_WQ(8) }
#undef SB_WQ
}

template <int Q>
void launch_bulk_q(const StepGeom& g, int slots, const int4* chunks, int nchunks, const float4* srcp,
                   double* partial, cudaStream_t st) {
  switch (slots) {
    case 1: launch_bulk_s<Q, 1>(g, chunks, nchunks, srcp, partial, st); break;
    case 2: launch_bulk_s<Q, 2>(g, chunks, nchunks, srcp, partial, st); break;
    case 3: launch_bulk_s<Q, 3>(g, chunks, nchunks, srcp, partial, st); break;
    case 4: launch_bulk_s<Q, 4>(g, chunks, nchunks, srcp, partial, st); break;
    case 6: launch_bulk_s<Q, 6>(g, chunks, nchunks, srcp, partial, st); break;
    default: launch_bulk_s<Q, 8>(g, chunks, nchunks, srcp, partial, st); break;
  }
}

template <int Q, int TPT>
bool direct_ok_t(int slots) {
  switch (slots) {
    case 1: return CcDirectShape<Q, 1, TPT>::ok;
    case 2: return CcDirectShape<Q, 2, TPT>::ok;
    case 3: return CcDirectShape<Q, 3, TPT>::ok;
    case 4: return CcDirectShape<Q, 4, TPT>::ok;
    case 6: return CcDirectShape<Q, 6, TPT>::ok;
    case 8: return CcDirectShape<Q, 8, TPT>::ok;
    default: return false;
  }
}

template <int Q>
void launch_q(const StepGeom& g, bool mixed, int slots, const int4* chunks, int nchunks, const double4* src,
              double* partial, cudaStream_t st) {
  switch (slots) {
    case 1: launch_q_s<Q, 1>(g, mixed, chunks, nchunks, src, partial, st); break;
    case 2: launch_q_s<Q, 2>(g, mixed, chunks, nchunks, src, partial, st); break;
    case 3: launch_q_s<Q, 3>(g, mixed, chunks, nchunks, src, partial, st); break;
    case 4: launch_q_s<Q, 4>(g, mixed, chunks, nchunks, src, partial, st); break;
    case 6: launch_q_s<Q, 6>(g, mixed, chunks, nchunks, src, partial, st); break;
    default: launch_q_s<Q, 8>(g, mixed, chunks, nchunks, src, partial, st); break;
  }
}

template <int Q>
bool shape_ok_q(int slots) {
  switch (slots) {
    case 1: return CcShape<Q, 1>::ok;
    case 2: return CcShape<Q, 2>::ok;
    case 3: return CcShape<Q, 3>::ok;
    case 4: return CcShape<Q, 4>::ok;
    case 6: return CcShape<Q, 6>::ok;
    case 8: return CcShape<Q, 8>::ok;
    default: return false;
  }
}

}  // namespace

bool cc_chunk_supported(int q) { return q == 36 || q == 49 || q == 64 || q == 81 || q == 100 || q == 121; }

bool cc_chunk_shape_ok(int q, int slots) {
  switch (q) {
    case 36: return shape_ok_q<36>(slots);
    case 49: return shape_ok_q<49>(slots);
    case 64: return shape_ok_q<64>(slots);
    case 81: return shape_ok_q<81>(slots);
    case 100: return shape_ok_q<100>(slots);
    case 121: return shape_ok_q<121>(slots);
    default: return false;
  }
}

bool cc_warp_shape_ok(int q, int warps) {
  return cc_chunk_supported(q) && (warps == 1 || warps == 2 || warps == 4 || warps == 8);
}

int cc_chunk_threads(int q, int slots, int direct_tpt) {
  if (direct_tpt == kCcWarpForm) return 32 * slots;
  const int qt = direct_tpt > 0 && direct_tpt != kCcBulkForm ? (q + direct_tpt - 1) / direct_tpt : q;
  return (slots * qt + 31) / 32 * 32;
}

bool cc_direct_shape_ok(int q, int slots, int tpt) {
  if (tpt != 1 && tpt != 2) return false;
#define SB_DOK(Q)                                                         \
  case Q:                                                                 \
    return tpt == 1 ? direct_ok_t<Q, 1>(slots) : direct_ok_t<Q, 2>(slots);
  switch (q) { SB_DOK(36) SB_DOK(49) SB_DOK(64) SB_DOK(81) SB_DOK(100) SB_DOK(121) default: return false; }
#undef SB_DOK
}

void launch_cc_pair_sources(const float4* srcf, int q, int panels, float4* srcp, cudaStream_t st) {
  const long pairs = (long)panels * ((q + 1) / 2);
  SB_LAUNCH(k_cc_pair_sources, blocks_for(pairs, 256), 256, 0, st, srcf, q, pairs, srcp);
}

void launch_cc_chunks(const StepGeom& g, int precision, int slots, const int4* chunks, int nchunks, const int* cstart,
                      const double4* src, double* partial, double* out, cudaStream_t st, int direct_tpt,
                      const float4* srcp) {
  const bool mixed = precision == SBSLPM_MIXED;
  if (nchunks > 0 && mixed && direct_tpt == kCcWarpForm) {
#define SB_WQQ(Q) \
  case Q: launch_warp_q<Q>(g, slots, chunks, nchunks, srcp, partial, st); break;
    switch (g.q) { SB_WQQ(36) SB_WQQ(49) SB_WQQ(64) SB_WQQ(81) SB_WQQ(100) SB_WQQ(121) default: break; }
#undef SB_WQQ
  } else if (nchunks > 0 && mixed && direct_tpt == kCcBulkForm) {
#define SB_BQ(Q) \
  case Q: launch_bulk_q<Q>(g, slots, chunks, nchunks, srcp, partial, st); break;
    switch (g.q) { SB_BQ(36) SB_BQ(49) SB_BQ(64) SB_BQ(81) SB_BQ(100) SB_BQ(121) default: break; }
#undef SB_BQ
  } else if (nchunks > 0 && mixed && direct_tpt > 0) {
#define SB_DQ(Q)                                                                          \
  case Q:                                                                                 \
    if (direct_tpt == 1) launch_direct_t<Q, 1>(g, slots, chunks, nchunks, srcp, partial, st); \
    else launch_direct_t<Q, 2>(g, slots, chunks, nchunks, srcp, partial, st);                 \
    break;
    switch (g.q) { SB_DQ(36) SB_DQ(49) SB_DQ(64) SB_DQ(81) SB_DQ(100) SB_DQ(121) default: break; }
#undef SB_DQ
  } else if (nchunks > 0) {
    switch (g.q) {
      case 36: launch_q<36>(g, mixed, slots, chunks, nchunks, src, partial, st); break;
      case 49: launch_q<49>(g, mixed, slots, chunks, nchunks, src, partial, st); break;
      case 64: launch_q<64>(g, mixed, slots, chunks, nchunks, src, partial, st); break;
      case 81: launch_q<81>(g, mixed, slots, chunks, nchunks, src, partial, st); break;
      case 100: launch_q<100>(g, mixed, slots, chunks, nchunks, src, partial, st); break;
      default: launch_q<121>(g, mixed, slots, chunks, nchunks, src, partial, st); break;
    }
  }
  const long pn = (long)g.panels * g.q;
  SB_LAUNCH(k_cc_reduce, blocks_for(pn, 256), 256, 0, st, g, cstart, partial,
            mixed ? kBiotSavartPacked : kBiotSavart, out);
}

void launch_cc_multi(const CcTcGroup& g, cudaStream_t st) {
  if (g.nmem <= 0 || !g.usrc) return;
  switch (g.Q) {
    case 36: launch_multi_q<36>(g, st); break;
    case 49: launch_multi_q<49>(g, st); break;
    case 64: launch_multi_q<64>(g, st); break;
    case 81: launch_multi_q<81>(g, st); break;
    case 100: launch_multi_q<100>(g, st); break;
    default: launch_multi_q<121>(g, st); break;
  }
}

void build_cc_chunks(const std::vector<int>& start, int chunk_len, std::vector<int4>& chunks,
                     std::vector<int>& cstart) {
  const int panels = (int)start.size() - 1;
  chunks.clear();
  cstart.assign(panels + 1, 0);
  for (int t = 0; t < panels; t++) {
    cstart[t] = (int)chunks.size();
    const int len = start[t + 1] - start[t];
    const int nc = (len + chunk_len - 1) / chunk_len;
    for (int k = 0; k < nc; k++)  // near-equal chunks: entries [len k / nc, len (k+1) / nc)
      chunks.push_back(make_int4(t, start[t] + (int)((long)len * k / nc), start[t] + (int)((long)len * (k + 1) / nc), 0));
  }
  cstart[panels] = (int)chunks.size();
}

}  // namespace sbslpm
