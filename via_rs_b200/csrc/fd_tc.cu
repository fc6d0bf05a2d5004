// The FirstDim scan as a tcgen05 integer GEMM (crates/via-server/src/first_dim.rs:94-184).
//
// One persistent CTA per SM walks work units (t, c-tile): for every database
// column tile jt it streams the (t, jt) byte planes chunk by chunk (64 rows of
// the reduction at a time) together with the matching chunk of the split
// selection, issues the byte-product MMAs into a TMEM accumulator, and an
// epilogue folds the accumulator columns into residues mod q2.
//
// Warp roles (64 + 32 EPI + 32 threads): warp 0 lane 0 issues the bulk copies,
// warp 1 allocates TMEM and its lane 0 issues the MMAs, the EPI warps 2 ..
// EPI + 1 read TMEM and write the outputs (8 for one query, 16 for grouped
// tiles), and the last warp expands the two-bit top byte plane of packed
// chunks (fd_tc.cuh) in shared memory before the MMAs read it. Every wait is
// bounded in time; when one runs out the CTA raises an error word and leaves
// its loops instead of waiting on.
//
// Accumulator placement. The selection chunk stacks the five byte limbs of the
// N columns of a c-tile as rows l*N + c of the MMA's N dimension. The MMA of
// database limb k writes TMEM columns starting at k*S:
//  * grouped tiles (S = N, N a multiple of 16): column k*N + l*N + c collects
//    every product with k + l = g in column g*N + c, nine groups per output;
//  * the single-query tile (N = 2, S = 16): five disjoint regions of 16
//    columns, product (k, l, c) in column 16k + 2l + c.
#include <algorithm>

#include "fd_tc.cuh"
#include "ntt_fp.cuh"

namespace via {
namespace {

// Epilogue warps: 8 for the single-query tile, 16 for grouped tiles, whose
// epilogue (nine TMEM groups folded per output) sets the pace of a batch.
constexpr int EPI_ONE = 8, EPI_GROUPED = 16;
constexpr int fd_threads(int epi) { return 64 + 32 * epi + 32; }
constexpr int ZERO_TILE = 256 * 32;  // zero operand for clearing grouped accumulators
constexpr unsigned long long WAIT_NS = 2000000000ull;  // 2 s per wait
constexpr unsigned WAIT_SPINS = 1u << 26;

struct KParams {
  const uint8_t* db;
  const uint8_t* sel;
  u64* out;
  int* err;
  int n, J, n_jt, n_kc, n_ct, N, Np, nq;
  int stages, grouped, acc_stride, nacc, tmem_cols, order;
  int packed4, chunk, stage_bytes, sel_off, unp_off;  // chunk layout (FD_CHUNK or FD_CHUNK_P4) and stage offsets
  unsigned fault_ns;  // test hook: > 0 makes the epilogue's first wait run out after this long
  double qd, qinv, c24, c48;  // q2, its rounded inverse, 2^24 and 2^48 mod q2, as doubles
};

__device__ __forceinline__ u32 smem_addr(const void* p) { return (u32)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(u64* bar, u32 count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(u64* bar, u32 bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(u64* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(u64* bar, u32 parity) {
  u32 ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
// Waits for the phase of `parity` to complete. Gives up (false) after WAIT_NS,
// after WAIT_SPINS polls, or, when `honor_abort`, once another role of the CTA
// has aborted.
__device__ bool mbar_wait(u64* bar, u32 parity, volatile int* abort_flag, bool honor_abort = true) {
  if (mbar_try_wait(bar, parity)) return true;
  const unsigned long long t0 = global_ns();
  for (unsigned it = 1; it < WAIT_SPINS; ++it) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((it & 31) == 0) {
      if (honor_abort && *abort_flag) return false;
      if (global_ns() - t0 > WAIT_NS) return false;
    }
  }
  return false;
}

// The test hook's wait: polls a barrier that no thread or copy ever completes
// until `limit_ns` has passed (or WAIT_SPINS polls), then reports failure.
__device__ bool mbar_wait_never(u64* bar, unsigned limit_ns) {
  const unsigned long long t0 = global_ns();
  for (unsigned it = 0; it < WAIT_SPINS; ++it) {
    if (mbar_try_wait(bar, 0)) return true;
    if ((it & 31) == 0 && global_ns() - t0 > limit_ns) return false;
  }
  return false;
}

__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, u32 bytes, u64* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Shared-memory matrix descriptor, K-major without swizzle: 8-row x 16-byte
// core matrices, `lbo` bytes between the two core matrices of a 32-byte K
// slice, `sbo` bytes between 8-row groups.
__device__ __forceinline__ u64 smem_desc(u32 addr, u32 lbo, u32 sbo) {
  return (u64)((addr >> 4) & 0x3FFF) | ((u64)((lbo >> 4) & 0x3FFF) << 16) | ((u64)((sbo >> 4) & 0x3FFF) << 32) |
         (1ull << 46);
}

// kind::i8 instruction descriptor: unsigned A and B, K-major, S32 accumulator, M = 128.
__device__ __forceinline__ u32 idesc_u8(int n) { return (2u << 4) | ((u32)(n >> 3) << 17) | ((u32)(128 >> 4) << 24); }

__device__ __forceinline__ void mma_u8(u32 d_tmem, u64 adesc, u64 bdesc, u32 idesc, u32 accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}
__device__ __forceinline__ void mma_commit(u64* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_addr(bar))
               : "memory");
}

__device__ __forceinline__ void tmem_ld4(u32 taddr, u32 (&r)[4]) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0, %1, %2, %3}, [%4];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(taddr));
}
__device__ __forceinline__ void tmem_ld8(u32 taddr, u32 (&r)[8]) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
               : "r"(taddr));
}
__device__ __forceinline__ void tmem_ld16(u32 taddr, u32 (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, "
      "[%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
template <int W>
__device__ __forceinline__ void tmem_ld(u32 taddr, u32 (&r)[W]) {
  if constexpr (W == 4)
    tmem_ld4(taddr, r);
  else
    tmem_ld8(taddr, r);
}
// Orders later uses of r after the wait above (the loads' results are only
// defined once tcgen05.wait::ld has returned).
template <int K>
__device__ __forceinline__ void pin(u32 (&r)[K]) {
#pragma unroll
  for (int x = 0; x < K; ++x) asm volatile("" : "+r"(r[x]));
}

// Work unit u -> (slot t, c-tile ct) in the tile's order.
__device__ __forceinline__ void unit_coords(const KParams& P, int u, int& t, int& ct) {
  if (P.order) {
    t = u % P.n;
    ct = u / P.n;
  } else {
    t = u / P.n_ct;
    ct = u % P.n_ct;
  }
}

// Integers below 2^52 to and from doubles, exactly: the double 2^52 + x has the
// bit pattern 0x4330000000000000 | x.
__device__ __forceinline__ double u52_to_double(u64 x) {
  return __dadd_rn(__longlong_as_double((long long)(x | 0x4330000000000000ull)), -4503599627370496.0);
}
__device__ __forceinline__ u64 double_to_u52(double x) {
  return (u64)__double_as_longlong(__dadd_rn(x, 4503599627370496.0)) & 0xFFFFFFFFFFFFFull;
}

// sum_g v_g 2^{8g} mod q for nine group sums v_g < 2^31 and q < 2^40, on the
// FP64 pipe: with lo, m1, m2 the sums of groups 0-2, 3-5 and 6-8 at their own
// scale (each below 2^31 (1 + 2^8 + 2^16) < 2^48), the value is
// lo + m1 2^24 + m2 2^48, and lo + fp_mulmod(m1, 2^24 mod q) + fp_mulmod(m2,
// 2^48 mod q) is an integer of magnitude below 2^48 + 1.125 q (ntt_fp.cuh
// bounds), which fp_canonical brings into [0, q).
__device__ __forceinline__ u64 fold9(const u32 (&v)[9], const KParams& P) {
  const u64 lo = (u64)v[0] + ((u64)v[1] << 8) + ((u64)v[2] << 16);
  const u64 m1 = (u64)v[3] + ((u64)v[4] << 8) + ((u64)v[5] << 16);
  const u64 m2 = (u64)v[6] + ((u64)v[7] << 8) + ((u64)v[8] << 16);
  const double r1 = fp_mulmod(u52_to_double(m1), P.c24, P.qd, P.qinv);
  const double r2 = fp_mulmod(u52_to_double(m2), P.c48, P.qd, P.qinv);
  const double s = __dadd_rn(__dadd_rn(u52_to_double(lo), r1), r2);
  return double_to_u52(fp_canonical(s, P.qd, P.qinv));
}

template <int EPI>
__global__ void __launch_bounds__(fd_threads(EPI), 1) k_fd_tc(KParams P) {
  constexpr int UNPACK_WARP = 2 + EPI;
  extern __shared__ __align__(1024) uint8_t smem[];
  const int stage_bytes = P.stage_bytes;
  uint8_t* zero_tile = smem + (size_t)P.stages * stage_bytes;
  u64* full = reinterpret_cast<u64*>(zero_tile + ZERO_TILE);
  u64* empty = full + P.stages;
  u64* unp = empty + P.stages;  // packed chunks: the stage's top byte plane is expanded
  u64* acc_full = unp + P.stages;
  u64* acc_empty = acc_full + 2;
  u64* drain = acc_empty + 2;
  u64* never = drain + 1;  // the test hook's barrier: initialised, never arrived on
  u32* tmem_slot = reinterpret_cast<u32*>(never + 1);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < P.stages; ++s) {
      mbar_init(full + s, 1);
      mbar_init(empty + s, 1);
      mbar_init(unp + s, 1);
    }
    for (int a = 0; a < 2; ++a) {
      mbar_init(acc_full + a, 1);
      mbar_init(acc_empty + a, EPI * 32);
    }
    mbar_init(drain, 1);
    mbar_init(never, 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  for (int x = threadIdx.x; x < ZERO_TILE / 16; x += blockDim.x)
    reinterpret_cast<uint4*>(zero_tile)[x] = make_uint4(0, 0, 0, 0);
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(tmem_slot)),
                 "r"((u32)P.tmem_cols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const u32 tmem = *tmem_slot;

  const int units = P.n * P.n_ct;
  const u32 sel_chunk = (u32)P.Np * FD_KC;

  if (warp == 0) {
    if (lane == 0) {
      // ---- Producer: bulk copies of (database chunk, selection chunk) per stage.
      int s = 0;
      u32 ph = 0;
      u32 armed = 0, armed_par = 0;  // per stage: armed at least once; parity of its last armed phase
      bool ok = true;
      for (int u = blockIdx.x; ok && u < units; u += gridDim.x) {
        int t, ct;
        unit_coords(P, u, t, ct);
        const uint8_t* selu = P.sel + ((size_t)t * P.n_ct + ct) * P.n_kc * sel_chunk;
        const uint8_t* dbt = P.db + (size_t)t * P.n_jt * P.n_kc * P.chunk;
        for (int jt = 0; ok && jt < P.n_jt; ++jt)
          for (int kc = 0; kc < P.n_kc; ++kc) {
            if (!mbar_wait(empty + s, ph ^ 1, abort_flag)) {
              ok = false;
              break;
            }
            uint8_t* dst = smem + (size_t)s * stage_bytes;
            mbar_expect_tx(full + s, (u32)P.chunk + sel_chunk);
            bulk_g2s(dst, dbt + ((size_t)jt * P.n_kc + kc) * P.chunk, (u32)P.chunk, full + s);
            bulk_g2s(dst + P.sel_off, selu + (size_t)kc * sel_chunk, sel_chunk, full + s);
            armed |= 1u << s;
            armed_par = (armed_par & ~(1u << s)) | (ph << s);
            if (++s == P.stages) {
              s = 0;
              ph ^= 1;
            }
          }
      }
      if (!ok) {
        atomicOr(P.err, 1);
        *abort_flag = 1;
      }
      // Every copy this CTA started lands before the CTA can exit: the last
      // phase armed on each stage completes (at once on the normal path).
      for (int k = 0; k < P.stages; ++k)
        if ((armed >> k) & 1)
          if (!mbar_wait(full + k, (armed_par >> k) & 1, abort_flag, false)) atomicOr(P.err, 1);
    }
  } else if (warp == 1) {
    if (lane == 0) {
      // ---- MMA issuer.
      int s = 0, a = 0;
      u32 ph = 0, aph = 0;
      bool ok = true;
      const u32 lbo_a = (FD_MT / 8) * 128, lbo_b = (u32)(P.Np / 8) * 128;
      const u32 idesc = idesc_u8(P.Np);
      const u32 zero_addr = smem_addr(zero_tile);
      for (int u = blockIdx.x; ok && u < units; u += gridDim.x) {
        for (int jt = 0; ok && jt < P.n_jt; ++jt) {
          if (!mbar_wait(acc_empty + a, aph ^ 1, abort_flag)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const u32 dacc = tmem + (u32)(a * P.acc_stride);
          if (P.grouped)  // columns [4N, 9N) start at zero; [0, 5N) are set by the first limb-0 product.
            mma_u8(dacc + 4 * P.N, smem_desc(zero_addr, lbo_a, 128), smem_desc(zero_addr, lbo_b, 128), idesc, 0);
          for (int kc = 0; kc < P.n_kc; ++kc) {
            // Packed chunks: the stage's copies have landed and its top plane is expanded.
            if (!mbar_wait(full + s, ph, abort_flag) || (P.packed4 && !mbar_wait(unp + s, ph, abort_flag))) {
              ok = false;
              break;
            }
            tc_fence_after();
            const u32 sa = smem_addr(smem + (size_t)s * stage_bytes);
            const u32 sb = sa + (u32)P.sel_off;
            const u32 a4 = P.packed4 ? sa + (u32)P.unp_off : sa + 4 * FD_PLANE;  // the top byte plane
#pragma unroll
            for (int ks = 0; ks < FD_KC / 32; ++ks) {
#pragma unroll
              for (int k = 0; k < FD_LIMBS; ++k) {
                const u64 ad = smem_desc((k == 4 ? a4 : sa + k * FD_PLANE) + ks * 2 * lbo_a, lbo_a, 128);
                const u64 bd = smem_desc(sb + ks * 2 * lbo_b, lbo_b, 128);
                const u32 col = P.grouped ? (u32)(k * P.N) : (u32)(16 * k);
                const u32 accum = (kc == 0 && ks == 0) ? (P.grouped ? (k > 0) : 0u) : 1u;
                mma_u8(dacc + col, ad, bd, idesc, accum);
              }
            }
            mma_commit(empty + s);  // frees the stage once these MMAs have read it
            if (++s == P.stages) {
              s = 0;
              ph ^= 1;
            }
          }
          if (!ok) break;
          mma_commit(acc_full + a);
          if (++a == P.nacc) {
            a = 0;
            aph ^= 1;
          }
        }
      }
      if (!ok) {
        atomicOr(P.err, 2);
        *abort_flag = 1;
      }
      // Every MMA issued above completes before TMEM is released.
      mma_commit(drain);
      if (!mbar_wait(drain, 0, abort_flag, false)) atomicOr(P.err, 2);
    }
  } else if (warp == UNPACK_WARP) {
    // ---- Packed chunks: expand the top byte plane of each landed stage
    // (fd_tc.cuh layout) into the stage's unpacked area, then release it to
    // the MMAs. The same walk over units, column tiles and row chunks as the
    // MMA issuer; a wait that runs out aborts the CTA.
    if (P.packed4) {
      int s = 0;
      u32 ph = 0;
      bool ok = true;
      for (int u = blockIdx.x; ok && u < units; u += gridDim.x)
        for (int jt = 0; ok && jt < P.n_jt; ++jt)
          for (int kc = 0; kc < P.n_kc; ++kc) {
            if (!__all_sync(0xffffffffu, mbar_wait(full + s, ph, abort_flag))) {
              ok = false;
              break;
            }
            uint8_t* stg = smem + (size_t)s * stage_bytes;
            const uint4* pk = reinterpret_cast<const uint4*>(stg + 4 * FD_PLANE);
            uint4* up = reinterpret_cast<uint4*>(stg + P.unp_off);
#pragma unroll
            for (int i = 0; i < FD_PACK4 / 16 / 32; ++i) {  // four quads per lane
              const int Q = lane + 32 * i;
              const uint4 w = pk[Q];
#pragma unroll
              for (int k = 0; k < 4; ++k)
                up[4 * Q + k] = make_uint4((w.x >> (2 * k)) & 0x03030303u, (w.y >> (2 * k)) & 0x03030303u,
                                           (w.z >> (2 * k)) & 0x03030303u, (w.w >> (2 * k)) & 0x03030303u);
            }
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // visible to the MMAs' async proxy
            __syncwarp();
            if (lane == 0) mbar_arrive(unp + s);
            if (++s == P.stages) {
              s = 0;
              ph ^= 1;
            }
          }
      if (!ok && lane == 0) {
        atomicOr(P.err, 8);
        *abort_flag = 1;
      }
    }
  } else {
    // ---- Epilogue: TMEM -> residues mod q2 -> out[b][j][mb][t]. Warp w
    // reads TMEM lanes 32 (w % 4) .. + 31 (its lane quadrant: database rows of
    // the tile); the EPI / 4 warps of a quadrant split the columns.
    const int ew = warp - 2, quad = warp & 3, part = ew >> 2;
    const int row = quad * 32 + lane;
    int a = 0;
    u32 aph = 0;
    // The test hook: a wait that runs out before any accumulator is read.
    bool ok = P.fault_ns == 0 || mbar_wait_never(never, P.fault_ns);
    for (int u = blockIdx.x; ok && u < units; u += gridDim.x) {
      int t, ct;
      unit_coords(P, u, t, ct);
      for (int jt = 0; jt < P.n_jt; ++jt) {
        // Warp-uniform: the TMEM loads below are .sync.aligned.
        if (!__all_sync(0xffffffffu, mbar_wait(acc_full + a, aph, abort_flag))) {
          ok = false;
          break;
        }
        tc_fence_after();
        const u32 tb = tmem + (u32)(a * P.acc_stride) + ((u32)(quad * 32) << 16);
        const int j = jt * FD_MT + row;
        const bool jok = j < P.J;
        bool released = false;
        if (P.grouped) {
          // CW-column chunks of the tile, dealt round-robin to the quadrant's
          // warps (N is a multiple of 8). A warp frees the accumulator once its
          // last chunk is in registers, so the next tile's MMAs overlap the
          // folding and stores of that chunk.
          constexpr int CW = EPI >= 16 ? 4 : 8, STEP = (EPI / 4) * CW;
          const size_t qs = (size_t)2 * P.J * P.n;  // between queries
          u64* orow = P.out + (size_t)j * 2 * P.n + t;
          for (int c0 = part * CW; c0 < P.N; c0 += STEP) {
            u32 v[9][CW];
#pragma unroll
            for (int g = 0; g < 9; ++g) tmem_ld<CW>(tb + (u32)(g * P.N + c0), v[g]);
            tmem_wait_ld();
#pragma unroll
            for (int g = 0; g < 9; ++g) pin(v[g]);
            if (c0 + STEP >= P.N) {
              tc_fence_before();
              mbar_arrive(acc_empty + a);
              released = true;
            }
#pragma unroll
            for (int x = 0; x < CW; ++x) {
              const int cg = ct * P.N + c0 + x;
              if (jok && cg < 2 * P.nq) {
                u32 w[9];
#pragma unroll
                for (int g = 0; g < 9; ++g) w[g] = v[g][x];
                orow[(size_t)(cg >> 1) * qs + (size_t)(cg & 1) * P.n] = fold9(w, P);
              }
            }
          }
        } else if (part < 2) {
          u32 r[FD_LIMBS][16];
#pragma unroll
          for (int k = 0; k < FD_LIMBS; ++k) tmem_ld16(tb + (u32)(16 * k), r[k]);
          tmem_wait_ld();
#pragma unroll
          for (int k = 0; k < FD_LIMBS; ++k) pin(r[k]);
          // N = 2: part 0 writes the mask column, part 1 the body.
          u32 w0[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, w1[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
          for (int k = 0; k < FD_LIMBS; ++k)
#pragma unroll
            for (int l = 0; l < FD_LIMBS; ++l) {
              w0[k + l] += r[k][2 * l];
              w1[k + l] += r[k][2 * l + 1];
            }
          u32 w[9];
#pragma unroll
          for (int g = 0; g < 9; ++g) w[g] = part ? w1[g] : w0[g];
          if (jok) P.out[((size_t)j * 2 + part) * P.n + t] = fold9(w, P);
        }
        if (!released) {
          tc_fence_before();
          mbar_arrive(acc_empty + a);
        }
        if (++a == P.nacc) {
          a = 0;
          aph ^= 1;
        }
      }
    }
    if (!ok) {
      atomicOr(P.err, 4);
      *abort_flag = 1;
    }
  }

  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((u32)P.tmem_cols)
                 : "memory");
  }
}

// Split selection: [t][ct][kc][Np x 64 bytes, core-matrix order], row l*N + c
// holding byte l of column c (query b = cg/2, mask or body = cg%2) of the
// c-tile. One thread per (t, ct, c, 16 consecutive rows i). Grouped tiles whose
// 5N is not a multiple of 16 pad the operand to Np rows: rows 5N .. Np-1 are
// written as zeros (they reach accumulator columns that are read), one thread
// per padding row as the virtual columns c = N .. N + Np - 5N - 1.
__global__ void k_fd_split(const u64* __restrict__ sel, int nq, int I, int n, int n_k16, int n_kc, int n_ct, int N,
                           int Np, int pad, uint8_t* __restrict__ out) {
  const int NC = N + pad;  // pad: zero rows of a grouped tile
  const long total = (long)n * n_ct * NC * n_k16;
  const long gid = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= total) return;
  const int t = (int)(gid % n);
  long r = gid / n;
  const int k16 = (int)(r % n_k16);
  r /= n_k16;
  const int c = (int)(r % NC);
  const int ct = (int)(r / NC);
  if (c >= N) {
    const int kc = k16 / (FD_KC / 16), kk = k16 % (FD_KC / 16);
    uint8_t* base = out + (((size_t)t * n_ct + ct) * n_kc + kc) * ((size_t)Np * FD_KC);
    const int rr = FD_LIMBS * N + (c - N);
    *reinterpret_cast<uint4*>(base + ((size_t)kk * (Np / 8) + rr / 8) * 128 + (rr % 8) * 16) = make_uint4(0, 0, 0, 0);
    return;
  }
  const int cg = ct * N + c;
  const bool valid = cg < 2 * nq;
  const int b = cg >> 1, mb = cg & 1;
  u32 w[FD_LIMBS][4];
#pragma unroll
  for (int l = 0; l < FD_LIMBS; ++l) w[l][0] = w[l][1] = w[l][2] = w[l][3] = 0;
#pragma unroll
  for (int x = 0; x < 16; ++x) {
    const int i = k16 * 16 + x;
    if (valid && i < I) {
      const u64 v = sel[(((size_t)b * I + i) * 2 + mb) * n + t];
#pragma unroll
      for (int l = 0; l < FD_LIMBS; ++l) w[l][x >> 2] |= (u32)((v >> (8 * l)) & 0xFF) << (8 * (x & 3));
    }
  }
  const int kc = k16 / (FD_KC / 16), kk = k16 % (FD_KC / 16);
  uint8_t* base = out + (((size_t)t * n_ct + ct) * n_kc + kc) * ((size_t)Np * FD_KC);
#pragma unroll
  for (int l = 0; l < FD_LIMBS; ++l) {
    const int rr = l * N + c;
    *reinterpret_cast<uint4*>(base + ((size_t)kk * (Np / 8) + rr / 8) * 128 + (rr % 8) * 16) =
        make_uint4(w[l][0], w[l][1], w[l][2], w[l][3]);
  }
}

// Database rows [i0, i0 + 16) (u64 [16][J][n]) -> byte planes. One thread per (t, j).
// Packed chunks (packed4): the top byte goes to the two-bit plane, OR-ed into
// the quad words the four threads of a group quad share (the planes start zeroed).
__global__ void k_fd_planes(const u64* __restrict__ stage, int i0, int I, int J, int n, int n_jt, int n_kc,
                            int packed4, uint8_t* __restrict__ planes) {
  const long gid = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= (long)J * n) return;
  const int t = (int)(gid % n), j = (int)(gid / n);
  u32 w[FD_LIMBS][4];
#pragma unroll
  for (int l = 0; l < FD_LIMBS; ++l) w[l][0] = w[l][1] = w[l][2] = w[l][3] = 0;
#pragma unroll
  for (int x = 0; x < 16; ++x) {
    if (i0 + x < I) {
      const u64 v = stage[((size_t)x * J + j) * n + t];
#pragma unroll
      for (int l = 0; l < FD_LIMBS; ++l) w[l][x >> 2] |= (u32)((v >> (8 * l)) & 0xFF) << (8 * (x & 3));
    }
  }
  const int kc = i0 / FD_KC, kk = (i0 % FD_KC) / 16;
  const int jt = j / FD_MT, r = j % FD_MT;
  const int chunk = packed4 ? FD_CHUNK_P4 : FD_CHUNK;
  uint8_t* base = planes + (((size_t)t * n_jt + jt) * n_kc + kc) * chunk;
  const int G = (kk * (FD_MT / 8) + r / 8) * 8 + r % 8;  // this thread's 16-byte group in every plane
  const int planes_full = packed4 ? 4 : FD_LIMBS;
#pragma unroll
  for (int l = 0; l < FD_LIMBS; ++l)
    if (l < planes_full)
      *reinterpret_cast<uint4*>(base + (size_t)l * FD_PLANE + (size_t)G * 16) =
          make_uint4(w[l][0], w[l][1], w[l][2], w[l][3]);
  if (packed4) {
    // Byte 4w + b of group 4Q + k -> bits 8b + 2k of word w of quad Q; the top
    // bytes are below 4.
    unsigned int* pq = reinterpret_cast<unsigned int*>(base + 4 * FD_PLANE) + (G >> 2) * 4;
    const int k = G & 3;
#pragma unroll
    for (int ww = 0; ww < 4; ++ww) {
      const u32 bits = (w[4][ww] & 0x03030303u) << (2 * k);
      if (bits) atomicOr(pq + ww, bits);
    }
  }
}

// Bytes of one shared-memory stage ahead of its selection chunk: the planes,
// and for packed chunks the expanded top plane after them.
constexpr int fd_stage_planes(bool packed4) { return packed4 ? FD_CHUNK_P4 + FD_PLANE : FD_CHUNK; }

struct Tiling {
  int grouped, N, Np, n_ct, stages, acc_stride, nacc, tmem_cols, order;
  size_t smem;
};

// packed4: stages hold FD_CHUNK_P4 bytes of planes, then the expanded top plane.
Tiling tiling(int nq, const FdTile& tile, bool packed4) {
  Tiling T{};
  int acc_cols;
  if (nq == 1) {
    T.grouped = 0;
    T.N = 2;
    T.Np = 16;
    T.n_ct = 1;
    T.stages = tile.stages ? tile.stages : 4;
    T.order = 0;
    acc_cols = 16 * FD_LIMBS;
  } else {
    const int cap = tile.n_max ? tile.n_max : 48;
    T.grouped = 1;
    T.n_ct = (2 * nq + cap - 1) / cap;
    // n_max = 24 tiles round N to 8 and pad the MMA operand to a multiple of 16
    // rows, so that two accumulator sets (up to 224 columns each) fit in TMEM.
    T.N = fd_round_up((2 * nq + T.n_ct - 1) / T.n_ct, cap == 24 ? 8 : 16);
    T.Np = fd_round_up(FD_LIMBS * T.N, 16);
    T.stages = tile.stages ? tile.stages : 3;
    T.order = tile.order;
    // Limb k's MMA writes columns [k N, k N + Np); the epilogue reads [0, 9 N).
    acc_cols = std::max(9 * T.N, 4 * T.N + T.Np);
  }
  T.acc_stride = fd_round_up(acc_cols, 32);
  T.nacc = 2 * T.acc_stride <= 512 ? 2 : 1;
  int cols = T.nacc * T.acc_stride, p2 = 32;
  while (p2 < cols) p2 <<= 1;
  T.tmem_cols = p2;
  T.smem = (size_t)T.stages * (fd_stage_planes(packed4) + (size_t)T.Np * FD_KC) + ZERO_TILE + 256;
  return T;
}

// The built-in shared-memory limit the kernel was first tuned under.
constexpr int SMEM_DEFAULT = 200 * 1024;

}  // namespace

size_t fd_planes_bytes(int I, int J, int n, bool packed4) {
  return (size_t)(fd_round_up(I, FD_KC) / FD_KC) * (fd_round_up(J, FD_MT) / FD_MT) * n *
         (packed4 ? FD_CHUNK_P4 : FD_CHUNK);
}

bool fd_supported(int I, int n, u64 q) { return I >= 1 && I <= 4096 && n >= 1 && q < (1ull << 40); }

bool fd_tile_valid(const FdPlan& p, int nq, const FdTile& t) {
  if (nq < 1) return false;
  if (t.n_max != 0 && t.n_max != 16 && t.n_max != 24 && t.n_max != 32 && t.n_max != 48) return false;
  if (t.stages != 0 && (t.stages < 2 || t.stages > 6)) return false;
  if (t.order != 0 && t.order != 1) return false;
  if (nq == 1 && (t.n_max != 0 || t.order != 0)) return false;
  const Tiling T = tiling(nq, t, p.packed4);
  const size_t limit = p.smem_max > 0 ? (size_t)p.smem_max : (size_t)SMEM_DEFAULT;
  return T.Np <= 256 && T.nacc * T.acc_stride <= 512 && T.smem <= limit;
}

FdTile fd_tile_for(const FdPlan& p, int nq) {
  const FdTile* below = nullptr;
  for (const auto& e : p.tuned) {
    if ((e.first == 1) != (nq == 1)) continue;  // one-query and batch tiles do not mix
    if (e.first >= nq) return fd_tile_valid(p, nq, e.second) ? e.second : FdTile{};
    below = &e.second;
  }
  return below && fd_tile_valid(p, nq, *below) ? *below : FdTile{};
}

void fd_set_tile(FdPlan& p, int nq, const FdTile& t) {
  for (auto& e : p.tuned)
    if (e.first == nq) {
      e.second = t;
      return;
    }
  p.tuned.push_back({nq, t});
  std::sort(p.tuned.begin(), p.tuned.end(),
            [](const std::pair<int, FdTile>& a, const std::pair<int, FdTile>& b) { return a.first < b.first; });
}

std::vector<FdTile> fd_tile_candidates(const FdPlan& p, int nq) {
  std::vector<FdTile> out;
  out.push_back(FdTile{});  // the default first
  auto add = [&](FdTile t) {
    const Tiling a = tiling(nq, t, p.packed4);
    if (!fd_tile_valid(p, nq, t)) return;
    for (const FdTile& o : out) {  // skip tiles that launch the same kernel configuration
      const Tiling b = tiling(nq, o, p.packed4);
      if (a.N == b.N && a.n_ct == b.n_ct && a.stages == b.stages && a.order == b.order) return;
    }
    out.push_back(t);
  };
  if (nq == 1) {
    for (int st = 2; st <= 6; ++st) add(FdTile{0, st, 0});
  } else {
    for (int nm : {16, 24, 32, 48})
      for (int st = 2; st <= 5; ++st)
        for (int od = 0; od <= 1; ++od) add(FdTile{nm, st, od});
  }
  return out;
}

void fd_rows_to_planes(const u64* stage, int i0, const FdPlan& p, uint8_t* planes, cudaStream_t st) {
  const long total = (long)p.J * p.n;
  k_fd_planes<<<(unsigned)((total + 255) / 256), 256, 0, st>>>(stage, i0, p.I, p.J, p.n, p.J_pad / FD_MT,
                                                              p.I_pad / FD_KC, p.packed4 ? 1 : 0, planes);
  VIA_LAUNCHED();
}

size_t fd_sel_bytes(const FdPlan& p, int nq) {
  // Every candidate's split selection: n * n_ct * Np * I_pad bytes.
  size_t bytes = 0;
  for (const FdTile& t : fd_tile_candidates(p, nq)) {
    const Tiling T = tiling(nq, t, p.packed4);
    bytes = std::max(bytes, (size_t)p.n * T.n_ct * (size_t)T.Np * p.I_pad);
  }
  return bytes;
}

int fd_prepare_device() {
  int dev = 0, optin = 0;
  VIA_CUDA(cudaGetDevice(&dev));
  VIA_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  const int limit = std::max(optin, SMEM_DEFAULT);
  VIA_CUDA(cudaFuncSetAttribute(k_fd_tc<EPI_ONE>, cudaFuncAttributeMaxDynamicSharedMemorySize, limit));
  VIA_CUDA(cudaFuncSetAttribute(k_fd_tc<EPI_GROUPED>, cudaFuncAttributeMaxDynamicSharedMemorySize, limit));
  return limit;
}

void fd_scan(const FdPlan& p, const u64* sel_eval, u64* out_eval, int nq, uint8_t* scratch, cudaStream_t st,
             const FdTile* force) {
  const FdTile tile = force ? *force : fd_tile_for(p, nq);
  if (force && !fd_tile_valid(p, nq, tile)) throw CudaError(100, "scan tile not valid for this batch");
  const Tiling T = tiling(nq, tile, p.packed4);
  const int n_k16 = p.I_pad / 16, n_kc = p.I_pad / FD_KC;
  const int pad = T.grouped ? T.Np - FD_LIMBS * T.N : 0;
  const long total = (long)p.n * T.n_ct * (T.N + pad) * n_k16;
  k_fd_split<<<(unsigned)((total + 255) / 256), 256, 0, st>>>(sel_eval, nq, p.I, p.n, n_k16, n_kc, T.n_ct, T.N, T.Np, pad,
                                                              scratch);
  VIA_LAUNCHED();
  KParams K;
  K.db = p.planes;
  K.sel = scratch;
  K.out = out_eval;
  K.err = p.err;
  K.n = p.n;
  K.J = p.J;
  K.n_jt = p.J_pad / FD_MT;
  K.n_kc = n_kc;
  K.n_ct = T.n_ct;
  K.N = T.N;
  K.Np = T.Np;
  K.nq = nq;
  K.stages = T.stages;
  K.grouped = T.grouped;
  K.acc_stride = T.acc_stride;
  K.nacc = T.nacc;
  K.tmem_cols = T.tmem_cols;
  K.order = T.order;
  K.packed4 = p.packed4 ? 1 : 0;
  K.chunk = p.packed4 ? FD_CHUNK_P4 : FD_CHUNK;
  K.stage_bytes = fd_stage_planes(p.packed4) + T.Np * FD_KC;
  K.sel_off = fd_stage_planes(p.packed4);
  K.unp_off = FD_CHUNK_P4;
  K.fault_ns = p.fault_wait_ns;
  K.qd = (double)p.m.q;
  K.qinv = 1.0 / K.qd;
  K.c24 = (double)(((u64)1 << 24) % p.m.q);
  K.c48 = (double)(((u64)1 << 48) % p.m.q);
  const int units = p.n * T.n_ct;
  const int grid = std::min(units, p.grid);
  if (T.grouped)
    k_fd_tc<EPI_GROUPED><<<grid, fd_threads(EPI_GROUPED), T.smem, st>>>(K);
  else
    k_fd_tc<EPI_ONE><<<grid, fd_threads(EPI_ONE), T.smem, st>>>(K);
  VIA_LAUNCHED();
}

std::vector<FdTuneResult> fd_measure_tiles(const FdPlan& p, int nq, const u64* sel_eval, u64* out_eval,
                                           uint8_t* scratch, cudaStream_t st, int reps) {
  std::vector<FdTuneResult> out;
  cudaEvent_t e0, e1;
  VIA_CUDA(cudaEventCreate(&e0));
  VIA_CUDA(cudaEventCreate(&e1));
  try {
    for (const FdTile& t : fd_tile_candidates(p, nq)) {
      fd_scan(p, sel_eval, out_eval, nq, scratch, st, &t);  // warm-up
      VIA_CUDA(cudaEventRecord(e0, st));
      for (int r = 0; r < reps; ++r) fd_scan(p, sel_eval, out_eval, nq, scratch, st, &t);
      VIA_CUDA(cudaEventRecord(e1, st));
      VIA_CUDA(cudaEventSynchronize(e1));
      float ms = 0.f;
      VIA_CUDA(cudaEventElapsedTime(&ms, e0, e1));
      out.push_back(FdTuneResult{t, ms / (float)std::max(1, reps)});
    }
  } catch (...) {
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    throw;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return out;
}

}  // namespace via
