// Well-separated proxy interactions of a batched ensemble on the tensor cores
// (tcgen05.mma kind::tf32, accumulators in tensor memory).  The problem is
// stated in cc_tcgen05.cuh; this file holds the kernels and their launchers.
//
// One CTA owns one target cluster T and one tile of members: 16 producer
// warps and one MMA warp.  For each source cluster S of T's union list and
// each KC-wide chunk of S's proxies (KC = 16, or 8 when A has 384 rows)
//   1. the producers build the A chunk (rows (c, a) = c Q + a, the three
//      components of the packed pair term for target proxy a) on the CUDA
//      cores, split into TF32 high and low parts,
//   2. they copy the members' strengths for the chunk two chunks ahead with
//      cp.async (B, one row per member, zero-filled for members whose list
//      lacks (T, S)),
//   3. the MMA warp issues the MMAs (per 128-row tile of A and 8-wide K
//      step; three passes for 3xTF32) and commits them to the chunk slot's
//      mbarrier,
// with two A slots and four B slots, handed over by full / empty mbarriers,
// so that building one chunk overlaps the MMAs of the previous one.  Each source cluster accumulates in its own tensor-memory set
// (two sets, alternating), and once its MMAs are complete (the slot wait of
// two chunks later proves it) the set is read with tcgen05.ld and added into
// float64 sums in shared memory: float32 accumulation across the hundreds of
// source clusters of a target would cost an order of magnitude in accuracy
// (about 1,600 accumulator roundings per output), per-cluster sums keep the
// float32 pair kernel's accuracy.  The epilogue writes
// u = -1/(4 pi) sqrt(2) t x D for every member.
//
// Shared-memory operands use the no-swizzle K-major canonical layout: 8-row x
// 16-byte core matrices, element (r, k) of a chunk at byte
//     (r / 8) * (KC * 32) + (k / 4) * 128 + (r % 8) * 16 + (k % 4) * 4,
// i.e. leading-dimension byte offset 128 (the two 16-byte K halves of an
// 8-wide K step) and stride byte offset KC * 32 (consecutive 8-row groups).
// Every operand address the MMAs can form stays inside its chunk image.
//
// Every wait is bounded (one second of %globaltimer, CcTcGroup::wait_ns); a
// wait that runs out sets kErrTimeout, waits (bounded) for the MMAs already
// issued, frees the tensor memory and returns.
#include <cuda_runtime.h>

#include <cstdint>

#include "cc_tcgen05.cuh"
#include "device_common.cuh"

namespace sbslpm {
namespace {

constexpr int kCcThreads = 512;  // producer threads; one more warp issues the MMAs

__host__ __device__ constexpr int cc_rows(int Q) { return (3 * Q + 127) / 128 * 128; }

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Shared-memory matrix descriptor: start, leading / stride byte offsets (all
// >> 4), descriptor version 1, no swizzle.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return static_cast<uint64_t>((addr >> 4) & 0x3FFFu) | (static_cast<uint64_t>((lbo >> 4) & 0x3FFFu) << 16) |
         (static_cast<uint64_t>((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}"
      :
      : "r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" : : "r"(bar) : "memory");
}

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, unsigned long long bound_ns) {
  const unsigned long long t0 = global_ns();
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
    if (global_ns() - t0 > bound_ns) return false;
  }
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

__host__ __device__ constexpr int tmem_cols_for(int need) {
  int c = 32;
  while (c < need) c <<= 1;
  return c;
}

// K per chunk: two 8-wide K steps, or one where 384 A rows would not leave
// room for the float64 accumulators.
__host__ __device__ constexpr int cc_kc(int Q) { return cc_rows(Q) > 256 ? 8 : 16; }

constexpr int kDepth = 2;  // chunks of B and source proxies in flight ahead of the one being built
constexpr int kRing = kDepth + 2;

// Byte offset of element (r, k4 * 4) of a chunk image (see the file comment;
// the stride byte offset is KC * 32).
template <int KC>
__device__ __forceinline__ int chunk_off(int r, int k4) {
  return (r >> 3) * (KC * 32) + k4 * 128 + (r & 7) * 16;
}

// TF32 split of a float: hi rounded to 10 mantissa bits (ties away from
// zero, as cvt.rna.tf32), lo = x - hi exactly; the MMA reads lo's top 19 bits.
__device__ __forceinline__ float tf32_hi(float x) {
  return __uint_as_float((__float_as_uint(x) + 0x1000u) & 0xFFFFE000u);
}

__device__ __forceinline__ void cp_async16(uint32_t saddr, const void* g, bool on) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" : : "r"(saddr), "l"(g), "r"(on ? 16 : 0) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared::cta.b64 st, [%0];\n\t}" : : "r"(bar) : "memory");
}

// Waits for the phase of the given parity, or until the CTA's abort flag is
// set (by another thread's expired wait) or bound_ns pass (sets it).
__device__ __forceinline__ bool mbar_wait_abortable(uint32_t bar, uint32_t parity, volatile int* abort_flag,
                                                    unsigned long long bound_ns) {
  const unsigned long long t0 = global_ns();
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
    if (*abort_flag) return false;
    if (global_ns() - t0 > bound_ns) {
      *abort_flag = 1;
      return false;
    }
    __nanosleep(32);  // back off: the spinning warp's issue slots go to the producers
  }
}

// Warp roles: warps 0..15 build the operands and fold the accumulators into
// float64 (producers, 512 threads), warp 16 issues the MMAs.  Per chunk i the
// producers wait until the MMAs of chunk i - 2 are complete (empty[i & 1]),
// fold a finished source cluster in, start the copies of chunk i + 2, build
// A(i), wait for their own copies of chunk i and arrive on full[i & 1]; the
// MMA warp waits on full[i & 1], issues chunk i and commits to empty[i & 1].
template <int Q, int PASSES, bool GUARD>
__global__ void __launch_bounds__(kCcThreads + 32, 1) k_cc_tc(CcTcGroup g) {
  constexpr int ROWS = cc_rows(Q), TILES = ROWS / 128, KP8 = (Q + 7) / 8 * 8, IMG = PASSES == 3 ? 2 : 1;
  constexpr int KC = cc_kc(Q), V = KC / 4, SBO = KC * 32, R3 = 3 * Q, kch = (KP8 + KC - 1) / KC;
  extern __shared__ __align__(128) unsigned char sm[];
  __shared__ __align__(8) unsigned long long full[2], empty[2];
  __shared__ uint32_t s_tmem;
  __shared__ int s_abort, s_last;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const bool producer = tid < kCcThreads;
  const int T = blockIdx.x, ty = blockIdx.y, N = g.ntile, mw = g.mw;
  const int ncols = tmem_cols_for(2 * TILES * N);
  const int a_bytes = ROWS * KC * 4, b_bytes = N * KC * 4;
  // shared memory: A slots | B ring | per-warp source ring | float64 sums | union list cache
  unsigned char* const a_base = sm;
  unsigned char* const b_base = a_base + 2 * IMG * a_bytes;
  // warp w's source proxies (V) and source-cluster centre (2 x 16 bytes) per ring slot
  float4* const wsrc = reinterpret_cast<float4*>(b_base + kRing * IMG * b_bytes);
  double* const acc = reinterpret_cast<double*>(wsrc + (kCcThreads / 32) * kRing * 8);  // [member column][row c Q + a]
  int* const lsrc = reinterpret_cast<int*>(acc + (long)R3 * N);
  unsigned* const lmask = reinterpret_cast<unsigned*>(lsrc + g.maxlist);
  auto A_img = [&](int slot, int lo) { return a_base + (slot * IMG + lo) * a_bytes; };
  auto B_img = [&](int ring, int lo) { return b_base + (ring * IMG + lo) * b_bytes; };
  volatile int* abort_flag = &s_abort;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" : : "r"(smem_u32(&s_tmem)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    for (int k = 0; k < 2; k++) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" : : "r"(smem_u32(&full[k])), "r"(kCcThreads) : "memory");
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" : : "r"(smem_u32(&empty[k])) : "memory");
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    s_abort = 0;
    s_last = -1;
  }
  const int e0 = g.ustart[T], e1 = g.ustart[T + 1], ns = e1 - e0;
  const int total = ns * kch;
  // A rows at or beyond 3Q are never written below: zero both slots once
  for (int f = tid; f < 2 * IMG * a_bytes / 16; f += blockDim.x)
    reinterpret_cast<float4*>(a_base)[f] = make_float4(0.f, 0.f, 0.f, 0.f);
  for (int f = tid; f < R3 * N; f += blockDim.x) acc[f] = 0.0;
  for (int f = tid; f < ns; f += blockDim.x) lsrc[f] = __ldg(g.usrc + e0 + f);
  for (int f = tid; f < ns * mw; f += blockDim.x) lmask[f] = __ldg(g.umask + (long)e0 * mw + f);
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = s_tmem;
  const long pn = (long)g.Pf * Q;
  const double* ct = g.centre + 4 * (long)T;

  // Add source cluster s's accumulators (tensor-memory set s & 1) into the
  // float64 sums: warp w reads lane quarter w & 3, the four warps of a
  // quarter take every fourth 16-column block.
  const int quarter = warp & 3, wq = warp >> 2, nblk = N / 16;
  auto flush = [&](int s) {
    __syncwarp();
    const uint32_t set = (uint32_t)((s & 1) * TILES * N);
#pragma unroll
    for (int t = 0; t < TILES; t++) {
      const int row = 128 * t + 32 * quarter + lane;
      for (int blk = wq; blk < nblk; blk += 4) {
        uint32_t r[16];
        tmem_ld16(tmem + ((uint32_t)(32 * quarter) << 16) + set + (uint32_t)(t * N + 16 * blk), r);
        if (row < R3) {
#pragma unroll
          for (int k = 0; k < 16; k++) acc[(long)(16 * blk + k) * R3 + row] += (double)__uint_as_float(r[k]);
        }
      }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  };

  if (!producer) {
    // ---- MMA warp ----
    const uint32_t idesc = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(N >> 3) << 17) | ((128u >> 4) << 24);
    int c = 0;
    for (; c < total; c++) {
      // warp-uniform decision, so that the warp stays converged for the exit path
      if (!__all_sync(0xffffffffu, mbar_wait_abortable(smem_u32(&full[c & 1]), (uint32_t)((c >> 1) & 1), abort_flag,
                                                       g.wait_ns)))
        break;
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      if (lane == 0) {
        const int kc = c % kch, slot = c & 1, ring = c % kRing;
        const int ksteps = min(KC / 8, (KP8 - kc * KC) / 8);
        const uint32_t ah = smem_u32(A_img(slot, 0)), bh = smem_u32(B_img(ring, 0));
        const uint32_t al = smem_u32(A_img(slot, IMG - 1)), bl = smem_u32(B_img(ring, IMG - 1));
        const uint32_t set = (uint32_t)(((c / kch) & 1) * TILES * N);
#pragma unroll
        for (int t = 0; t < TILES; t++) {
          for (int ks = 0; ks < ksteps; ks++) {
            const uint32_t d = tmem + set + (uint32_t)(t * N);
            const uint64_t adh = smem_desc(ah + t * 16 * SBO + ks * 256, 128, SBO);
            const uint64_t bdh = smem_desc(bh + ks * 256, 128, SBO);
            mma_tf32(d, adh, bdh, idesc, (kc > 0 || ks > 0) ? 1u : 0u);
            if (PASSES == 3) {
              mma_tf32(d, adh, smem_desc(bl + ks * 256, 128, SBO), idesc, 1u);
              mma_tf32(d, smem_desc(al + t * 16 * SBO + ks * 256, 128, SBO), bdh, idesc, 1u);
            }
          }
        }
        mma_commit(smem_u32(&empty[slot]));
      }
      __syncwarp();
    }
    if (lane == 0) s_last = c - 1;  // the last chunk committed (its commit tracks all earlier MMAs)
  } else {
    // ---- producers ----
    // Asynchronous copies of chunk c's B rows (zero-filled for members
    // without the pair) into ring slot c % kRing; one commit group per chunk
    // (empty past the end).
    const int a = tid & 127, part = tid >> 7;  // this thread's A row and its V K columns of each chunk
    auto issue = [&](int c) {
      if (c < total) {
        const int el = c / kch, kc = c % kch, S = lsrc[el], ring = c % kRing;
        const long base4 = ((long)S * kch + kc) * ((long)g.npad * (KC / 4)) + (long)ty * N * (KC / 4);
        const float4* wh = reinterpret_cast<const float4*>(g.whi) + base4;
        const float4* wl = reinterpret_cast<const float4*>(g.wlo) + base4;
        const unsigned* mk = lmask + el * mw;
        for (int f = tid; f < N * (KC / 4); f += kCcThreads) {
          const int jg = ty * N + (f / (2 * KC)) * 8 + (f & 7);
          const bool on = (mk[jg >> 5] >> (jg & 31)) & 1u;
          cp_async16(smem_u32(B_img(ring, 0)) + 16 * f, wh + f, on);
          if (PASSES == 3) cp_async16(smem_u32(B_img(ring, 1)) + 16 * f, wl + f, on);
        }
        // the warp's source proxies (zero beyond Q) and the source-cluster centre
        float4* ws = wsrc + (warp * kRing + ring) * 8;
        const int b = kc * KC + part * V + lane;
        if (lane < V) cp_async16(smem_u32(ws + lane), g.pxf + (long)S * Q + (b < Q ? b : 0), b < Q);
        else if (lane < V + 2)
          cp_async16(smem_u32(ws + 4 + (lane - V)), g.centre + 4 * (long)S + 2 * (lane - V), true);
      }
      asm volatile("cp.async.commit_group;" ::: "memory");
    };
    float dtx = 0.f, dty = 0.f, dtz = 0.f;
    if (a < Q) {
      const long o = (long)T * Q + a;
      dtx = (float)((g.px[o] - ct[0]) * kPackScale);
      dty = (float)((g.px[pn + o] - ct[1]) * kPackScale);
      dtz = (float)((g.px[2 * pn + o] - ct[2]) * kPackScale);
    }
    const float feps = (float)g.eps;

    for (int d = 0; d < kDepth; d++) issue(d);
    const float2 eps2 = make_float2(feps, feps);
    float2 bx2 = make_float2(0.f, 0.f), by2 = bx2, bz2 = bx2;
    int flushed = 0;
    for (int i = 0; i < total; i++) {
      const int slot = i & 1, ring = i % kRing;
      if (i >= 2) {
        // warp-uniform decision: the flush below needs the whole warp
        if (!__all_sync(0xffffffffu, mbar_wait_abortable(smem_u32(&empty[slot]), (uint32_t)(((i >> 1) - 1) & 1),
                                                         abort_flag, g.wait_ns)))
          break;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        // chunk i - 2 is complete: if it closed a source cluster, fold that cluster in
        if ((i - 2) % kch == kch - 1) flush(flushed++);
      }
      asm volatile("cp.async.wait_group %0;" : : "n"(kDepth - 1) : "memory");  // this thread's copies of chunk i
      __syncwarp();
      issue(i + kDepth);  // ring slot of chunk i - 2, whose MMAs are complete
      const float4* ws = wsrc + (warp * kRing + ring) * 8;
      const int kc = i % kch;
      if (kc == 0) {
        const double2 c01 = *reinterpret_cast<const double2*>(ws + 4), c23 = *reinterpret_cast<const double2*>(ws + 5);
        const float bx = (float)((c01.x - ct[0]) * kPackScale) - dtx;
        const float by = (float)((c01.y - ct[1]) * kPackScale) - dty;
        const float bz = (float)((c23.x - ct[2]) * kPackScale) - dtz;
        bx2 = make_float2(bx, bx);
        by2 = make_float2(by, by);
        bz2 = make_float2(bz, bz);
      }
      // A chunk: rows c Q + a, columns kc*KC + part*V .. +V-1, two sources per paired-FP32 step
      if (a < Q) {
        float2 v[3][V / 2];
#pragma unroll
        for (int p = 0; p < V / 2; p++) {
          const float4 s0 = ws[2 * p], s1 = ws[2 * p + 1];
          const float2 dx = __fadd2_rn(bx2, make_float2(s0.x, s1.x)), dy = __fadd2_rn(by2, make_float2(s0.y, s1.y)),
                       dz = __fadd2_rn(bz2, make_float2(s0.z, s1.z));
          const float2 den = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __ffma2_rn(dz, dz, eps2)));
          float r0 = dev::recip_f32(den.x), r1 = dev::recip_f32(den.y);
          if (GUARD) {
            r0 = den.x > 0.f ? r0 : 0.f;
            r1 = den.y > 0.f ? r1 : 0.f;
          }
          const int b = kc * KC + part * V + 2 * p;
          if (b >= Q) r0 = 0.f;
          if (b + 1 >= Q) r1 = 0.f;
          const float2 r = make_float2(r0, r1);
          v[0][p] = __fmul2_rn(r, dx);
          v[1][p] = __fmul2_rn(r, dy);
          v[2][p] = __fmul2_rn(r, dz);
        }
        const float2 neg1 = make_float2(-1.f, -1.f);
#pragma unroll
        for (int c = 0; c < 3; c++) {
          const int off = chunk_off<KC>(c * Q + a, (part * V) >> 2) + ((part * V) & 3) * 4;
          float2 hi[V / 2], lo[V / 2];
#pragma unroll
          for (int p = 0; p < V / 2; p++) {
            hi[p] = make_float2(tf32_hi(v[c][p].x), tf32_hi(v[c][p].y));
            lo[p] = __ffma2_rn(hi[p], neg1, v[c][p]);  // exact: v - hi
          }
          if constexpr (V == 4) {
            *reinterpret_cast<float4*>(A_img(slot, 0) + off) = make_float4(hi[0].x, hi[0].y, hi[1].x, hi[1].y);
            if (PASSES == 3)
              *reinterpret_cast<float4*>(A_img(slot, 1) + off) = make_float4(lo[0].x, lo[0].y, lo[1].x, lo[1].y);
          } else {
            *reinterpret_cast<float2*>(A_img(slot, 0) + off) = hi[0];
            if (PASSES == 3) *reinterpret_cast<float2*>(A_img(slot, 1) + off) = lo[0];
          }
        }
      }
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      if (!(g.withhold && i == 0 && tid == 0)) mbar_arrive(smem_u32(&full[slot]));
    }
    asm volatile("cp.async.wait_all;" ::: "memory");
  }
  __syncthreads();
  // every MMA committed is complete before the sums are read and the memory freed
  int good = 1;
  if (tid == 0 && s_last >= 0)
    good = mbar_wait(smem_u32(&empty[s_last & 1]), (uint32_t)((s_last >> 1) & 1), g.wait_ns);
  const bool ok = __syncthreads_and(good && !s_abort && s_last == total - 1);
  if (!ok && tid == 0) dev::flag(g.err, kErrTimeout);
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");

  if (ok && producer) {
    // the clusters not folded in by the loop: those whose last chunk is
    // within two of the end ((s + 1) kch - 1 + 2 >= total)
    for (int s = 0; s < ns; s++)
      if ((s + 1) * kch + 1 >= total) flush(s);
  }
  __syncthreads();
  if (ok && producer) {
    for (int qq = tid; qq < Q * N; qq += kCcThreads) {
      const int j = qq / Q, ta = qq - j * Q, jg = ty * N + j;
      if (jg >= g.nmem) continue;
      const double sx = acc[(long)j * R3 + ta], sy = acc[(long)j * R3 + Q + ta], sz = acc[(long)j * R3 + 2 * Q + ta];
      const long o = (long)T * Q + ta;
      const double px = g.px[o], py = g.px[pn + o], pz = g.px[2 * pn + o];
      double* out = g.mem[g.idx[jg]].ftgt;
      out[o] = kBiotSavartPacked * (py * sz - pz * sy);
      out[pn + o] = kBiotSavartPacked * (pz * sx - px * sz);
      out[2 * pn + o] = kBiotSavartPacked * (px * sy - py * sx);
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" : : "r"(tmem), "r"(ncols) : "memory");
}

// Strength image: per source cluster S and K chunk kc (KC = cc_kc(Q) wide), a
// block of npad * KC/4 float4 laid out as the B chunk in shared memory,
// [member / 8][k4][member % 8]: the TF32 split of w_b(member) for
// b = kc*KC + k4*4 .. +3 (zero beyond Q and for padding members).
__global__ void k_cc_tc_pack(CcTcGroup g, int KC) {
  const long per = (long)g.npad * (KC / 4);
  const long n4 = (long)g.Pf * g.kch * per;
  const long f = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (f >= n4) return;
  const long blk = f / per;
  const int loc = (int)(f % per);
  const int kc = (int)(blk % g.kch);
  const long S = blk / g.kch;
  const int r8 = loc & 7, k4 = (loc >> 3) % (KC / 4), jg = (loc / (2 * KC)) * 8 + r8;
  const float4* sf = jg < g.nmem ? g.mem[g.idx[jg]].fg.srcf : nullptr;
  float h[4], l[4];
#pragma unroll
  for (int e = 0; e < 4; e++) {
    const int k = kc * KC + k4 * 4 + e;
    const float w = (sf && k < g.Q) ? sf[S * g.Q + k].w : 0.f;
    h[e] = tf32_hi(w);
    l[e] = w - h[e];
  }
  reinterpret_cast<float4*>(g.whi)[f] = make_float4(h[0], h[1], h[2], h[3]);
  reinterpret_cast<float4*>(g.wlo)[f] = make_float4(l[0], l[1], l[2], l[3]);
}

// At most 512 tensor-memory columns per SM over the CTAs resident on it:
// the dynamic shared memory is raised until the occupancy guarantees that.
template <int Q, int PASSES, bool GUARD>
cudaError_t prepare_q(const CcTcGroup& g, size_t& use) {
  int dev = 0, optin = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  cudaFuncAttributes fa{};
  if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, k_cc_tc<Q, PASSES, GUARD>);
  if (e != cudaSuccess) return e;
  const size_t maxdyn = (size_t)optin - fa.sharedSizeBytes;
  use = cc_tc_smem_bytes(Q, g.ntile, PASSES, g.maxlist, g.mw);
  if (use > maxdyn) return cudaErrorInvalidValue;
  e = cudaFuncSetAttribute(k_cc_tc<Q, PASSES, GUARD>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)maxdyn);
  if (e != cudaSuccess) return e;
  const int cols = cc_tc_tmem_cols(Q, g.ntile);
  for (int guard = 0; guard < 64; guard++) {
    int occ = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_cc_tc<Q, PASSES, GUARD>, kCcThreads + 32, use);
    if (e != cudaSuccess) return e;
    if (occ * cols <= 512) return cudaSuccess;
    if (use >= maxdyn) break;
    use = use + 8 * 1024 > maxdyn ? maxdyn : use + 8 * 1024;
  }
  return cudaErrorInvalidValue;  // the tensor-memory budget cannot be guaranteed
}

template <int Q>
cudaError_t prepare_q(CcTcGroup& g) {
  const bool guard = !(g.eps > 0);
  cudaError_t e = guard ? prepare_q<Q, 3, true>(g, g.smem3) : prepare_q<Q, 3, false>(g, g.smem3);
  if (e != cudaSuccess) return e;
  return guard ? prepare_q<Q, 1, true>(g, g.smem1) : prepare_q<Q, 1, false>(g, g.smem1);
}

template <int Q>
void launch_q(const CcTcGroup& g, int passes, cudaStream_t st) {
  const bool guard = !(g.eps > 0);
  const dim3 grid((unsigned)g.Pf, (unsigned)(g.npad / g.ntile));
  if (passes == 3) {
    if (guard) SB_LAUNCH((k_cc_tc<Q, 3, true>), grid, kCcThreads + 32, g.smem3, st, g);
    else SB_LAUNCH((k_cc_tc<Q, 3, false>), grid, kCcThreads + 32, g.smem3, st, g);
  } else {
    if (guard) SB_LAUNCH((k_cc_tc<Q, 1, true>), grid, kCcThreads + 32, g.smem1, st, g);
    else SB_LAUNCH((k_cc_tc<Q, 1, false>), grid, kCcThreads + 32, g.smem1, st, g);
  }
}

}  // namespace

size_t cc_tc_smem_bytes(int Q, int ntile, int passes, int maxlist, int mw) {
  const int rows = cc_rows(Q), kc = cc_kc(Q), img = passes == 3 ? 2 : 1;
  const size_t a = 2 * (size_t)img * rows * kc * 4, b = (size_t)kRing * img * ntile * kc * 4;
  const size_t ws = (size_t)(kCcThreads / 32) * kRing * 8 * 16, acc = (size_t)3 * Q * ntile * 8;
  return a + b + ws + acc + (size_t)maxlist * 4 * (1 + mw);
}

int cc_tc_tmem_cols(int Q, int ntile) { return tmem_cols_for(2 * (cc_rows(Q) / 128) * ntile); }

int cc_tc_kc(int Q) { return cc_kc(Q); }

int cc_tc_max_tile(int Q) {
  // two accumulator sets within 512 tensor-memory columns, and the 3xTF32
  // kernel's shared memory within 208 KB (the rest of the 227 KB opt-in
  // limit holds the target's cached union list)
  const int tiles = cc_rows(Q) / 128;
  int n = 16;
  while (n + 16 <= 256 && 2 * tiles * (n + 16) <= 512 && cc_tc_smem_bytes(Q, n + 16, 3, 0, 0) <= 208 * 1024) n += 16;
  return n;
}

void launch_cc_tc_pack(const CcTcGroup& g, cudaStream_t st) {
  const int kc = cc_kc(g.Q);
  const long n4 = (long)g.Pf * g.kch * g.npad * (kc / 4);
  SB_LAUNCH(k_cc_tc_pack, (unsigned)((n4 + 255) / 256), 256, 0, st, g, kc);
}

cudaError_t cc_tc_prepare(CcTcGroup& g) {
  switch (g.Q) {
    case 16: return prepare_q<16>(g);
    case 25: return prepare_q<25>(g);
    case 36: return prepare_q<36>(g);
    case 49: return prepare_q<49>(g);
    case 64: return prepare_q<64>(g);
    case 81: return prepare_q<81>(g);
    case 100: return prepare_q<100>(g);
    case 121: return prepare_q<121>(g);
    default: return cudaErrorInvalidValue;
  }
}

void launch_cc_tc(const CcTcGroup& g, int passes, cudaStream_t st) {
  switch (g.Q) {
    case 16: launch_q<16>(g, passes, st); break;
    case 25: launch_q<25>(g, passes, st); break;
    case 36: launch_q<36>(g, passes, st); break;
    case 49: launch_q<49>(g, passes, st); break;
    case 64: launch_q<64>(g, passes, st); break;
    case 81: launch_q<81>(g, passes, st); break;
    case 100: launch_q<100>(g, passes, st); break;
    case 121: launch_q<121>(g, passes, st); break;
    default: break;
  }
}

}  // namespace sbslpm
