// Tensor-core products of the FP32 LU on the 5th-generation tensor cores (tcgen05):
//
//   C (m x n, FP32, column-major, ldc) -= A (m x K) * B (K x n)   (the trailing update)
//   C = A * B                                                     (the block TRSMs)
//
// FP32 operands are split once per call into BF16 hi (+ lo) parts (split_a_kernel /
// split_b_kernel), stored K-major so the Tensor Memory Accelerator can bring 64-wide
// K chunks into 128-byte-swizzled shared memory.  One thread issues, per K chunk and
// per 16-wide K step, one product hi*hi or the three products hi*hi + hi*lo + lo*hi as
// tcgen05.mma (kind::f16, BF16 inputs, FP32 accumulation in tensor memory, M = 128,
// N = 256); a tcgen05.commit signals an mbarrier when they are done, and eight warps
// drain the 128 x 256 accumulator with tcgen05.ld (one TMEM lane = one row of C): they
// stage 128 x 32 boxes in shared memory and either add each box into C with a bulk
// tensor reduction (cp.reduce.async.bulk.tensor .add.f32, staging -acc), so the L2
// performs the read-modify-write of C and the SM never waits on a load of C, or store
// it (cp.async.bulk.tensor).  Every element of C receives exactly one addition per call,
// C + (-acc), the same IEEE operation as C - acc: the result is deterministic.  With a
// triangular operand a tile runs only the K chunks that meet its nonzero part.
//
// Every mbarrier wait is bounded (the context's wait limit, 2 s by default): on timeout
// the kernel records an error word, the other roles stop at their next wait, the
// producer waits (bounded) for its own copies and the MMA warp for its own MMAs, and the
// tensor memory is freed.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <atomic>
#include <cstdint>
#include <cstdio>
#include <cstdlib>

#include "lu.cuh"

namespace bem {

namespace {

constexpr int UM = 128;                 // tile rows (UMMA M)
constexpr int UN = 256;                 // tile columns (UMMA N)
constexpr int UK = 64;                  // K chunk per TMA box (128 bytes of BF16)
constexpr int kMaxK = 1024;             // largest panel width
constexpr int kRasterW = 16;            // column tiles per raster group
constexpr int A_TILE = UM * UK * 2;     // 16 KB
constexpr int B_TILE = UN * UK * 2;     // 32 KB
// Shared memory: a ring of K chunks, then the barriers, then the epilogue's staging
// boxes (128 x 32 FP32 each, NSTG per epilogue half).  Three products stage hi + lo of
// A and B (96 KB a chunk); one product only the hi parts (48 KB).
template <int NPROD, int STAGES, int NSTG>
struct Cfg {
  static constexpr int stage = NPROD == 3 ? 2 * A_TILE + 2 * B_TILE : A_TILE + B_TILE;
  static constexpr int ring = STAGES * stage;
  static constexpr int box = 32 * UM * 4;
  static constexpr int smem = ring + 1024 + 256 + 2 * NSTG * box;
  static_assert(smem <= 227 * 1024, "shared memory");
  static_assert((2 * STAGES + 5) * 8 <= 128, "barrier block");
};
constexpr unsigned kTmemCols = 512;     // two 128 x 256 FP32 accumulators
constexpr int kEpiThreads = 256;        // 8 epilogue warps
constexpr int kThreads = 64 + kEpiThreads;

__device__ __forceinline__ unsigned smem_u32(const void* p) {
  return (unsigned)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ unsigned long long globaltimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// bounded wait on an mbarrier phase; gives up early when another role aborted
__device__ __forceinline__ bool mbar_wait(unsigned bar, unsigned parity, volatile int* abort_flag,
                                          unsigned long long wait_ns) {
  const unsigned long long t0 = globaltimer();
  while (true) {
    unsigned done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
    if (abort_flag && *abort_flag) return false;
    if (globaltimer() - t0 > wait_ns) return false;
  }
}

__device__ __forceinline__ uint64_t sw128_desc(unsigned saddr) {
  // K-major, 128-byte swizzle: SBO = 1024 B between 8-row groups, LBO = 16 B,
  // descriptor version 1, layout type 2
  return (uint64_t)((saddr >> 4) & 0x3FFF) | (1ull << 16) | (64ull << 32) | (1ull << 46) | (2ull << 61);
}

__device__ __forceinline__ void umma_commit(unsigned bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

// Persistent, warp-specialised: warp 0 (one lane) streams K chunks with TMA through a
// ring of stages, warp 1 (one lane) issues the MMAs into one of two TMEM accumulators,
// warps 2-9 drain the other accumulator into C, so the update of C by one tile
// overlaps the loads and MMAs of the next.
template <int NPROD, int STAGES, int NSTG, bool STORE>
__global__ void __launch_bounds__(kThreads, 1)
    umma_update_kernel(const __grid_constant__ CUtensorMap tAh, const __grid_constant__ CUtensorMap tAl,
                       const __grid_constant__ CUtensorMap tBh, const __grid_constant__ CUtensorMap tBl,
                       const __grid_constant__ CUtensorMap tC, int M, int N, int K, int kmode, int* err,
                       unsigned long long wait_ns) {
  using C_ = Cfg<NPROD, STAGES, NSTG>;
  constexpr int kStages = STAGES, STAGE = C_::stage, kRing = C_::ring;
  extern __shared__ __align__(16) unsigned char umma_smem[];
  const unsigned raw = smem_u32(umma_smem);
  const unsigned base = (raw + 1023u) & ~1023u;  // 1024-byte aligned operand tiles
  unsigned char* gbase = umma_smem + (base - raw);
  uint64_t* bars = reinterpret_cast<uint64_t*>(gbase + kRing);
  uint64_t* full = bars;                      // [kStages] TMA -> MMA
  uint64_t* empty = bars + kStages;           // [kStages] MMA -> TMA
  uint64_t* tfull = bars + 2 * kStages;       // [2] MMA -> epilogue
  uint64_t* tempty = bars + 2 * kStages + 2;  // [2] epilogue -> MMA
  uint64_t* drain = bars + 2 * kStages + 4;   // MMA completion before teardown
  unsigned* tmem_slot = reinterpret_cast<unsigned*>(gbase + kRing + 128);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(gbase + kRing + 136);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int tiles_m = (M + UM - 1) / UM, tiles_n = (N + UN - 1) / UN, total = tiles_m * tiles_n;
  // Tile order: groups of kRasterW column tiles, row tiles within a group, the group's
  // column tiles innermost, so that the CTAs of a wave share a few A row tiles and B
  // column tiles and A is streamed from DRAM once per group instead of once per column
  // tile (A of a 72,710-row update is 149 MB, more than the L2)
  auto coords = [&](int t, int& m0, int& n0) {
    const int g = t / (kRasterW * tiles_m), r = t - g * kRasterW * tiles_m;
    const int nb0 = g * kRasterW, wg = min(kRasterW, tiles_n - nb0);
    m0 = (r / wg) * UM;
    n0 = (nb0 + r % wg) * UN;
  };
  // K chunks of the tile at (m0, n0): all, or with a triangular operand only those that
  // meet its nonzero part (kmode 1: A lower triangular, kmode 2: B upper triangular)
  auto chunks = [&](int m0, int n0) {
    const int ke = kmode == 1 ? min(K, m0 + UM) : (kmode == 2 ? min(K, n0 + UN) : K);
    return (ke + UK - 1) / UK;
  };

  if (threadIdx.x == 0) {
    *abort_flag = 0;
    for (int s = 0; s < kStages; ++s) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&full[s])), "r"(1) : "memory");
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&empty[s])), "r"(1) : "memory");
    }
    for (int b = 0; b < 2; ++b) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&tfull[b])), "r"(1) : "memory");
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&tempty[b])), "r"(kEpiThreads) : "memory");
    }
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(drain)), "r"(1) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const unsigned tmem = *tmem_slot;

  auto fail = [&]() {
    *abort_flag = 1;
    atomicCAS(err, 0, BEM_ERR_TIMEOUT);
  };

  if (warp == 0) {
    if (lane == 0) {
      int stage = 0;
      unsigned phase = 0;
      int last[kStages];
#pragma unroll
      for (int s = 0; s < kStages; ++s) last[s] = -1;
      const CUtensorMap* maps[4] = {&tAh, &tAl, &tBh, &tBl};
      for (int t = blockIdx.x; t < total && !*abort_flag; t += gridDim.x) {
        int m0, n0;
        coords(t, m0, n0);
        const int row[4] = {m0, m0, n0, n0};
        const int nchunk = chunks(m0, n0);
        for (int c = 0; c < nchunk; ++c) {
          if (!mbar_wait(smem_u32(&empty[stage]), phase ^ 1u, abort_flag, wait_ns)) {
            fail();
            break;
          }
          const unsigned st = base + stage * STAGE;
          const unsigned bar = smem_u32(&full[stage]);
          // three products need hi and lo of both operands, one product only hi
          constexpr unsigned kBytes = NPROD == 3 ? (unsigned)STAGE : (unsigned)(A_TILE + B_TILE);
          asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(kBytes)
                       : "memory");
          // stage layout: three products [A hi | A lo | B hi | B lo], one [A hi | B hi]
          const unsigned dst[4] = {st, st + A_TILE, NPROD == 3 ? st + 2 * A_TILE : st + A_TILE,
                                   st + 2 * A_TILE + B_TILE};
#pragma unroll
          for (int q = 0; q < 4; ++q)
            if (NPROD == 3 || q == 0 || q == 2)
              asm volatile(
                "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
                "[%4];" ::"r"(dst[q]),
                "l"(reinterpret_cast<uint64_t>(maps[q])), "r"(c * UK), "r"(row[q]), "r"(bar)
                : "memory");
          last[stage] = (int)phase;
          if (++stage == kStages) {
            stage = 0;
            phase ^= 1u;
          }
        }
      }
      // this CTA's own copies must have landed before its shared memory goes away
      for (int s = 0; s < kStages; ++s)
        if (last[s] >= 0) mbar_wait(smem_u32(&full[s]), (unsigned)last[s], nullptr, wait_ns);
    }
  } else if (warp == 1) {
    if (lane == 0) {
      // F32 accumulate, BF16 A and B, both K-major, N = 256, M = 128
      const unsigned idesc =
          (1u << 4) | (1u << 7) | (1u << 10) | ((unsigned)(UN >> 3) << 17) | ((unsigned)(UM >> 4) << 24);
      int stage = 0, ab = 0;
      unsigned phase = 0, aphase = 0;
      for (int t = blockIdx.x; t < total && !*abort_flag; t += gridDim.x) {
        if (!mbar_wait(smem_u32(&tempty[ab]), aphase ^ 1u, abort_flag, wait_ns)) {
          fail();
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const unsigned d = tmem + (unsigned)(ab * UN);
        int tm0, tn0;
        coords(t, tm0, tn0);
        const int nchunk = chunks(tm0, tn0);
        bool ok = true;
        for (int c = 0; c < nchunk; ++c) {
          if (!mbar_wait(smem_u32(&full[stage]), phase, abort_flag, wait_ns)) {
            ok = false;
            break;
          }
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          const unsigned st = base + stage * STAGE;
          const unsigned ah = st, al = st + A_TILE, bh = NPROD == 3 ? st + 2 * A_TILE : st + A_TILE,
                         bl = st + 2 * A_TILE + B_TILE;
#pragma unroll
          for (int kk = 0; kk < UK / 16; ++kk) {
            const unsigned off = kk * 32;  // 16 BF16 = 32 bytes along K inside the swizzle atom
            const uint64_t a_h = sw128_desc(ah + off), a_l = sw128_desc(al + off);
            const uint64_t b_h = sw128_desc(bh + off), b_l = sw128_desc(bl + off);
            const uint64_t pa[3] = {a_h, a_h, a_l}, pb[3] = {b_h, b_l, b_h};
#pragma unroll
            for (int q = 0; q < NPROD; ++q) {
              const int acc = (c | kk | q) != 0;
              asm volatile(
                  "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                  "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d),
                  "l"(pa[q]), "l"(pb[q]), "r"(idesc), "r"(acc)
                  : "memory");
            }
          }
          umma_commit(smem_u32(&empty[stage]));  // frees the stage once these MMAs are done
          if (++stage == kStages) {
            stage = 0;
            phase ^= 1u;
          }
        }
        if (!ok) {
          fail();
          break;
        }
        umma_commit(smem_u32(&tfull[ab]));  // accumulator ready for the epilogue
        if (++ab == 2) {
          ab = 0;
          aphase ^= 1u;
        }
      }
      umma_commit(smem_u32(drain));
      mbar_wait(smem_u32(drain), 0, nullptr, wait_ns);
    }
    __syncwarp();
  } else {
    // 8 epilogue warps: warp w reads TMEM lane quarter (w % 4) of one half (128
    // columns) of the accumulator, 32 columns at a time; the 4 warps of a half fill
    // that half's staging box and its leader thread issues the box's reduction
    const int lq = warp & 3;
    const int half = (warp - 2) >> 2;  // 0 or 1
    float* stg0 = reinterpret_cast<float*>(gbase + kRing + 256) + half * NSTG * (32 * UM);
    int bx = 0;  // boxes this half has staged: box bx uses buffer bx % NSTG
    const bool leader = (lq == 0 && lane == 0);
    int ab = 0;
    unsigned aphase = 0;
    bool pending = false;
    for (int t = blockIdx.x; t < total; t += gridDim.x) {  // leaves only through the barrier below
      int m0, n0;
      coords(t, m0, n0);
      // the four warps of a half leave together: an abort ends every warp's wait, and
      // the barrier's AND makes the decision the same for all four (a warp that left
      // on its own would leave the others waiting at the named barriers)
      const int ok = mbar_wait(smem_u32(&tfull[ab]), aphase, abort_flag, wait_ns) ? 1 : 0;
      int all_ok;
      asm volatile(
          "{\n\t.reg .pred p, q;\n\tsetp.ne.b32 p, %1, 0;\n\t"
          "bar.red.and.pred q, %2, 128, p;\n\tselp.b32 %0, 1, 0, q;\n\t}\n"
          : "=r"(all_ok)
          : "r"(ok), "r"(1 + half)
          : "memory");
      if (!all_ok) {
        fail();
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll 1
      for (int q = 0; q < UN / 64; ++q) {
        const int j0 = half * (UN / 2) + 32 * q;
        unsigned r[32];
        const unsigned taddr = tmem + ((unsigned)(lq * 32) << 16) + (unsigned)(ab * UN + j0);
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
            "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
            : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
              "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
              "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]),
              "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]),
              "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
            : "r"(taddr)
            : "memory");
        // the box that last used this buffer must have been read out of shared memory
        // (bulk groups complete in order: at most NSTG - 1 newer ones may still read)
        float* stg = stg0 + (bx % NSTG) * (32 * UM);
        const unsigned stg_s = smem_u32(stg);
        ++bx;
        if (leader && pending) asm volatile("cp.async.bulk.wait_group.read %0;" ::"n"(NSTG - 1) : "memory");
        asm volatile("bar.sync %0, 128;" ::"r"(1 + half) : "memory");
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        const int rr = lq * 32 + lane;
#pragma unroll
        for (int j = 0; j < 32; ++j) stg[j * UM + rr] = STORE ? __uint_as_float(r[j]) : -__uint_as_float(r[j]);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("bar.sync %0, 128;" ::"r"(1 + half) : "memory");
        if (leader) {
          // rows m0.. (128-aligned, never negative), columns n0 + j0..; the tensor map
          // clips the box at M and N
          if (STORE)
            asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.bulk_group [%0, {%1, %2}], [%3];" ::"l"(
                             reinterpret_cast<uint64_t>(&tC)),
                         "r"(m0), "r"(n0 + j0), "r"(stg_s)
                         : "memory");
          else
            asm volatile(
                "cp.reduce.async.bulk.tensor.2d.global.shared::cta.add.tile.bulk_group [%0, {%1, %2}], [%3];" ::"l"(
                    reinterpret_cast<uint64_t>(&tC)),
                "r"(m0), "r"(n0 + j0), "r"(stg_s)
                : "memory");
          asm volatile("cp.async.bulk.commit_group;" ::: "memory");
          pending = true;
        }
      }
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(&tempty[ab])) : "memory");
      if (++ab == 2) {
        ab = 0;
        aphase ^= 1u;
      }
    }
    // the reductions this CTA issued complete before it ends
    if (leader && pending) asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 1) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
  }
}

// ---- CTA pairs (cta_group::2) -----------------------------------------------------
// A pair of CTAs (a cluster of two) computes a 256 x 256 tile of C with
// tcgen05.mma.cta_group::2 (M = 256, N = 256), issued by one thread of the pair's
// first CTA.  Each CTA stages its own 128 rows of A and its own 128 columns of B per K
// chunk (hi, or hi and lo for three products): 32 KB instead of the single CTA's 48 KB
// for the same 128 x 256 share of C with one product, 64 KB instead of 96 KB with
// three, so each SM's operand stream falls by a third; the tensor cores read the
// partner's half of B from its shared memory.  Each CTA holds its 128 rows of the
// accumulator in its own tensor memory and drains them with its own eight epilogue
// warps, as above (reductions into C, or stores with STORE).  With a triangular
// operand (kmode) a tile runs the K chunks that meet the nonzero part of its 256 rows
// or columns.
//   * Both CTAs' copies complete on the first CTA's `full` barrier (a .cta_group::2
//     copy may signal the partner's barrier); the first CTA arms it with the pair's
//     bytes and its MMA thread waits on it alone.
//   * The MMA commits arrive on both CTAs' `empty` and `tfull` barriers (multicast
//     commit), so each producer and each epilogue waits on its own shared memory.
//   * Both epilogues release an accumulator on the first CTA's `tempty` barrier, one
//     arrival per warp (16).
// Every wait is bounded as in umma_update_kernel; a CTA also gives up a wait when the
// error word is set (after the first millisecond of a wait), so that a failure in one
// CTA of the pair ends the other's waits too.
constexpr int PK = 128;  // rows of A and columns of B staged per CTA of a pair
constexpr int B_HALF = PK * UK * 2;  // 16 KB

template <int NPROD, int STAGES>
struct PairCfg {
  static constexpr int stage = NPROD == 3 ? 2 * A_TILE + 2 * B_HALF : A_TILE + B_HALF;  // 64 or 32 KB
  static constexpr int ring = STAGES * stage;
  static constexpr int box = 32 * UM * 4;
  static constexpr int bar_bytes = 256;  // barriers, then the TMEM address and the abort flag
  static constexpr int smem = ring + 1024 + bar_bytes + 2 * box;  // one staging box per epilogue half
  static_assert(smem <= 227 * 1024, "shared memory");
  static_assert((2 * STAGES + 5) * 8 <= 192, "barrier block");
};

__device__ __forceinline__ unsigned cluster_ctarank() {
  unsigned r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}

// shared::cluster address of the first CTA's copy of this CTA's shared location a
__device__ __forceinline__ unsigned map_first(unsigned a) {
  unsigned r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(0));
  return r;
}

// arrives on the barrier at shared offset bar in both CTAs of the pair once the MMAs
// this thread issued are done
__device__ __forceinline__ void umma_commit_pair(unsigned bar) {
  asm volatile(
      "tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64 [%0], %1;" ::"r"(bar),
      "h"((unsigned short)3)
      : "memory");
}

__device__ __forceinline__ void cluster_sync() {
  asm volatile("barrier.cluster.arrive.release.aligned;" ::: "memory");
  asm volatile("barrier.cluster.wait.acquire.aligned;" ::: "memory");
}

// bounded wait with cluster-scope acquire (arrivals from the partner CTA); gives up
// early when this CTA aborted or, after 1 ms, when the error word is set
__device__ __forceinline__ bool mbar_wait_pair(unsigned bar, unsigned parity, volatile int* abort_flag,
                                               const volatile int* err, unsigned long long wait_ns) {
  const unsigned long long t0 = globaltimer();
  while (true) {
    unsigned done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
    if (abort_flag && *abort_flag) return false;
    const unsigned long long dt = globaltimer() - t0;
    if (dt > wait_ns || (dt > 1000000ull && *err != 0)) return false;
  }
}

template <int NPROD, int STAGES, bool STORE>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(kThreads, 1)
    umma_pair_kernel(const __grid_constant__ CUtensorMap tAh, const __grid_constant__ CUtensorMap tAl,
                     const __grid_constant__ CUtensorMap tBh, const __grid_constant__ CUtensorMap tBl,
                     const __grid_constant__ CUtensorMap tC, int M, int N, int K, int kmode, int* err,
                     unsigned long long wait_ns) {
  constexpr int NSTG = 1;
  using C_ = PairCfg<NPROD, STAGES>;
  constexpr int STAGE = C_::stage, kRing = C_::ring;
  extern __shared__ __align__(16) unsigned char umma_smem[];
  const unsigned raw = smem_u32(umma_smem);
  const unsigned base = (raw + 1023u) & ~1023u;  // 1024-byte aligned operand tiles
  unsigned char* gbase = umma_smem + (base - raw);
  uint64_t* bars = reinterpret_cast<uint64_t*>(gbase + kRing);
  uint64_t* full = bars;                    // [STAGES] copies -> MMA (the first CTA's are used)
  uint64_t* empty = bars + STAGES;          // [STAGES] MMA -> this CTA's producer
  uint64_t* tfull = bars + 2 * STAGES;      // [2] MMA -> this CTA's epilogue
  uint64_t* tempty = bars + 2 * STAGES + 2; // [2] both epilogues -> MMA (the first CTA's)
  uint64_t* drain = bars + 2 * STAGES + 4;  // MMA completion before teardown
  unsigned* tmem_slot = reinterpret_cast<unsigned*>(gbase + kRing + 192);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(gbase + kRing + 200);
  const volatile int* gerr = err;

  const unsigned rank = cluster_ctarank();
  const bool first = rank == 0;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int pair = (int)(blockIdx.x >> 1), npairs = (int)(gridDim.x >> 1);
  const int tiles_m = (M + 2 * UM - 1) / (2 * UM), tiles_n = (N + UN - 1) / UN, total = tiles_m * tiles_n;
  // the grouped tile order of umma_update_kernel, with 256-row tiles
  auto coords = [&](int t, int& m0, int& n0) {
    const int g = t / (kRasterW * tiles_m), r = t - g * kRasterW * tiles_m;
    const int nb0 = g * kRasterW, wg = min(kRasterW, tiles_n - nb0);
    m0 = (r / wg) * (2 * UM);
    n0 = (nb0 + r % wg) * UN;
  };
  // K chunks of the pair's tile (kmode 1: A lower triangular, 2: B upper triangular)
  auto chunks = [&](int m0, int n0) {
    const int ke = kmode == 1 ? min(K, m0 + 2 * UM) : (kmode == 2 ? min(K, n0 + UN) : K);
    return (ke + UK - 1) / UK;
  };

  if (threadIdx.x == 0) {
    *abort_flag = 0;
    for (int s = 0; s < STAGES; ++s) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&full[s])), "r"(1) : "memory");
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&empty[s])), "r"(1) : "memory");
    }
    for (int b = 0; b < 2; ++b) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&tfull[b])), "r"(1) : "memory");
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&tempty[b])), "r"(2 * kEpiThreads / 32)
                   : "memory");
    }
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(drain)), "r"(1) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  if (warp == 1) {  // one warp of each CTA of the pair allocates, collectively
    asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  cluster_sync();  // both CTAs' barriers are initialised before any copy or arrival
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const unsigned tmem = *tmem_slot;

  auto fail = [&]() {
    *abort_flag = 1;
    atomicCAS(err, 0, BEM_ERR_TIMEOUT);
  };

  if (warp == 0) {
    if (lane == 0) {
      int stage = 0;
      unsigned phase = 0;
      int last[STAGES];
#pragma unroll
      for (int s = 0; s < STAGES; ++s) last[s] = -1;
      const unsigned full_first = map_first(smem_u32(&full[0]));
      for (int t = pair; t < total && !*abort_flag; t += npairs) {
        int m0, n0;
        coords(t, m0, n0);
        // this CTA's rows of A and columns of B; a half wholly outside the matrix loads
        // the first half again (its products fall outside C and are not stored)
        const int ar = (m0 + PK * (int)rank < M) ? m0 + PK * (int)rank : m0;
        const int br = (n0 + PK * (int)rank < N) ? n0 + PK * (int)rank : n0;
        const int nchunk = chunks(m0, n0);
        bool ok = true;
        for (int c = 0; c < nchunk; ++c) {
          if (!mbar_wait_pair(smem_u32(&empty[stage]), phase ^ 1u, abort_flag, gerr, wait_ns)) {
            ok = false;
            break;
          }
          const unsigned st = base + stage * STAGE;
          const unsigned bar = full_first + 8u * (unsigned)stage;
          if (first)  // the pair's bytes: both CTAs' copies complete on this barrier
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(&full[stage])),
                         "r"(2 * STAGE)
                         : "memory");
          // stage layout: three products [A hi | A lo | B hi | B lo], one [A hi | B hi]
          const CUtensorMap* maps[4] = {&tAh, &tAl, &tBh, &tBl};
          const int row[4] = {ar, ar, br, br};
          const unsigned dst[4] = {st, st + A_TILE, NPROD == 3 ? st + 2 * A_TILE : st + A_TILE,
                                   st + 2 * A_TILE + B_HALF};
#pragma unroll
          for (int q = 0; q < 4; ++q)
            if (NPROD == 3 || q == 0 || q == 2)
              asm volatile(
                  "cp.async.bulk.tensor.2d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes [%0], "
                  "[%1, {%2, %3}], [%4];" ::"r"(dst[q]),
                  "l"(reinterpret_cast<uint64_t>(maps[q])), "r"(c * UK), "r"(row[q]), "r"(bar)
                  : "memory");
          last[stage] = (int)phase;
          if (++stage == STAGES) {
            stage = 0;
            phase ^= 1u;
          }
        }
        if (!ok) {
          fail();
          break;
        }
      }
      // the first CTA's barrier counts the pair's copies: the phases it armed complete
      // once both CTAs' copies have landed
      if (first)
        for (int s = 0; s < STAGES; ++s)
          if (last[s] >= 0) mbar_wait(smem_u32(&full[s]), (unsigned)last[s], nullptr, wait_ns);
    }
  } else if (warp == 1) {
    if (lane == 0 && first) {
      // F32 accumulate, BF16 A and B, both K-major, N = 256, M = 256 (the pair)
      const unsigned idesc =
          (1u << 4) | (1u << 7) | (1u << 10) | ((unsigned)(UN >> 3) << 17) | ((unsigned)((2 * UM) >> 4) << 24);
      int stage = 0, ab = 0;
      unsigned phase = 0, aphase = 0;
      for (int t = pair; t < total && !*abort_flag; t += npairs) {
        if (!mbar_wait_pair(smem_u32(&tempty[ab]), aphase ^ 1u, abort_flag, gerr, wait_ns)) {
          fail();
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const unsigned d = tmem + (unsigned)(ab * UN);
        int tm0, tn0;
        coords(t, tm0, tn0);
        const int nchunk = chunks(tm0, tn0);
        bool ok = true;
        for (int c = 0; c < nchunk; ++c) {
          if (!mbar_wait_pair(smem_u32(&full[stage]), phase, abort_flag, gerr, wait_ns)) {
            ok = false;
            break;
          }
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          const unsigned st = base + stage * STAGE;
          const unsigned ah = st, al = st + A_TILE, bh = NPROD == 3 ? st + 2 * A_TILE : st + A_TILE,
                         bl = st + 2 * A_TILE + B_HALF;
#pragma unroll
          for (int kk = 0; kk < UK / 16; ++kk) {
            const unsigned off = kk * 32;  // 16 BF16 = 32 bytes along K inside the swizzle atom
            const uint64_t a_h = sw128_desc(ah + off), a_l = sw128_desc(al + off);
            const uint64_t b_h = sw128_desc(bh + off), b_l = sw128_desc(bl + off);
            const uint64_t pa[3] = {a_h, a_h, a_l}, pb[3] = {b_h, b_l, b_h};
#pragma unroll
            for (int q = 0; q < NPROD; ++q) {
              const int acc = (c | kk | q) != 0;
              asm volatile(
                  "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                  "tcgen05.mma.cta_group::2.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d),
                  "l"(pa[q]), "l"(pb[q]), "r"(idesc), "r"(acc)
                  : "memory");
            }
          }
          umma_commit_pair(smem_u32(&empty[stage]));  // frees the stage in both CTAs
          if (++stage == STAGES) {
            stage = 0;
            phase ^= 1u;
          }
        }
        if (!ok) {
          fail();
          break;
        }
        umma_commit_pair(smem_u32(&tfull[ab]));  // the accumulator is ready for both epilogues
        if (++ab == 2) {
          ab = 0;
          aphase ^= 1u;
        }
      }
      asm volatile("tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(drain))
                   : "memory");
      mbar_wait(smem_u32(drain), 0, nullptr, wait_ns);
    }
    __syncwarp();
  } else {
    // 8 epilogue warps, as in umma_update_kernel, on this CTA's 128 rows of the tile
    const int lq = warp & 3;
    const int half = (warp - 2) >> 2;  // 0 or 1
    float* stg0 = reinterpret_cast<float*>(gbase + kRing + C_::bar_bytes) + half * NSTG * (32 * UM);
    int bx = 0;
    const bool leader = (lq == 0 && lane == 0);
    const unsigned tempty_first = map_first(smem_u32(&tempty[0]));
    int ab = 0;
    unsigned aphase = 0;
    bool pending = false;
    for (int t = pair; t < total; t += npairs) {  // leaves only through the barrier below
      int m0, n0;
      coords(t, m0, n0);
      const int rm0 = m0 + PK * (int)rank;  // this CTA's rows
      const int ok = mbar_wait_pair(smem_u32(&tfull[ab]), aphase, abort_flag, gerr, wait_ns) ? 1 : 0;
      int all_ok;
      asm volatile(
          "{\n\t.reg .pred p, q;\n\tsetp.ne.b32 p, %1, 0;\n\t"
          "bar.red.and.pred q, %2, 128, p;\n\tselp.b32 %0, 1, 0, q;\n\t}\n"
          : "=r"(all_ok)
          : "r"(ok), "r"(1 + half)
          : "memory");
      if (!all_ok) {
        fail();
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      if (rm0 < M) {
#pragma unroll 1
        for (int q = 0; q < UN / 64; ++q) {
          const int j0 = half * (UN / 2) + 32 * q;
          if (n0 + j0 >= N) break;  // boxes wholly right of C (uniform over the half)
          unsigned r[32];
          const unsigned taddr = tmem + ((unsigned)(lq * 32) << 16) + (unsigned)(ab * UN + j0);
          asm volatile(
              "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
              "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
              : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
                "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]),
                "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]),
                "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
              : "r"(taddr)
              : "memory");
          float* stg = stg0 + (bx % NSTG) * (32 * UM);
          const unsigned stg_s = smem_u32(stg);
          ++bx;
          if (leader && pending) asm volatile("cp.async.bulk.wait_group.read %0;" ::"n"(NSTG - 1) : "memory");
          asm volatile("bar.sync %0, 128;" ::"r"(1 + half) : "memory");
          asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
          const int rr = lq * 32 + lane;
#pragma unroll
          for (int j = 0; j < 32; ++j) stg[j * UM + rr] = STORE ? __uint_as_float(r[j]) : -__uint_as_float(r[j]);
          asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
          asm volatile("bar.sync %0, 128;" ::"r"(1 + half) : "memory");
          if (leader) {
            if (STORE)
              asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.bulk_group [%0, {%1, %2}], [%3];" ::"l"(
                               reinterpret_cast<uint64_t>(&tC)),
                           "r"(rm0), "r"(n0 + j0), "r"(stg_s)
                           : "memory");
            else
              asm volatile(
                  "cp.reduce.async.bulk.tensor.2d.global.shared::cta.add.tile.bulk_group [%0, {%1, %2}], [%3];" ::"l"(
                      reinterpret_cast<uint64_t>(&tC)),
                  "r"(rm0), "r"(n0 + j0), "r"(stg_s)
                  : "memory");
            asm volatile("cp.async.bulk.commit_group;" ::: "memory");
            pending = true;
          }
        }
      }
      // this warp's reads of the accumulator are done: one arrival on the first CTA's
      // barrier
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      __syncwarp();
      if (lane == 0)
        asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(tempty_first +
                                                                                           8u * (unsigned)ab)
                     : "memory");
      if (++ab == 2) {
        ab = 0;
        aphase ^= 1u;
      }
    }
    if (leader && pending) asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  // the first CTA's MMAs (which read this CTA's shared memory and write its tensor
  // memory) are complete, and no copy of either CTA signals the other's barriers
  cluster_sync();
  if (*gerr != 0) {
    // after a failure a copy that the partner issued may still be in flight to this
    // CTA's shared memory: give it time to land before the memory goes away
    const unsigned long long t0 = globaltimer();
    while (globaltimer() - t0 < 100000ull) __nanosleep(1000);
  }
  if (warp == 1) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
  }
}

// A (m x K, FP32, column-major lda) -> hi/lo BF16 [m][K] (K contiguous); lo nullable
__global__ void split_a_kernel(int m, int K, const float* __restrict__ A, int64_t lda, __nv_bfloat16* hi,
                               __nv_bfloat16* lo) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int groups = K / 8;
  if (t >= (int64_t)m * groups) return;
  const int r = (int)(t % m), g = (int)(t / m);
  __align__(16) __nv_bfloat16 h[8], l[8];
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    const float v = A[r + (int64_t)(8 * g + q) * lda];
    h[q] = __float2bfloat16_rn(v);
    l[q] = __float2bfloat16_rn(v - __bfloat162float(h[q]));
  }
  *reinterpret_cast<uint4*>(hi + (int64_t)r * K + 8 * g) = *reinterpret_cast<uint4*>(h);
  if (lo) *reinterpret_cast<uint4*>(lo + (int64_t)r * K + 8 * g) = *reinterpret_cast<uint4*>(l);
}

// B (K x n, FP32, column-major ldb) -> hi/lo BF16 [n][K]; lo nullable
__global__ void split_b_kernel(int n, int K, const float* __restrict__ B, int64_t ldb, __nv_bfloat16* hi,
                               __nv_bfloat16* lo) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int groups = K / 8;
  if (t >= (int64_t)n * groups) return;
  const int g = (int)(t % groups), col = (int)(t / groups);
  __align__(16) __nv_bfloat16 h[8], l[8];
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    const float v = B[8 * g + q + (int64_t)col * ldb];
    h[q] = __float2bfloat16_rn(v);
    l[q] = __float2bfloat16_rn(v - __bfloat162float(h[q]));
  }
  *reinterpret_cast<uint4*>(hi + (int64_t)col * K + 8 * g) = *reinterpret_cast<uint4*>(h);
  if (lo) *reinterpret_cast<uint4*>(lo + (int64_t)col * K + 8 * g) = *reinterpret_cast<uint4*>(l);
}

PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;

bool make_map(CUtensorMap* map, const void* ptr, int rows, int K, int box_rows) {
  cuuint64_t dims[2] = {(cuuint64_t)K, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)K * 2};
  cuuint32_t box[2] = {(cuuint32_t)UK, (cuuint32_t)box_rows};
  cuuint32_t estr[2] = {1, 1};
  return g_encode(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(ptr), dims, strides, box, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// single CTAs: four ring stages of 48 KB for one product, two of 96 KB for three; one
// staging box per epilogue half (two measured no faster)
using K1 = Cfg<1, 4, 1>;
using K3 = Cfg<3, 2, 1>;
// CTA pairs: six 32 KB stages for one product, three 64 KB stages for three (the ring
// depth measured best: five or four stages of one product were slower)
using KP1 = PairCfg<1, 6>;
using KP3 = PairCfg<3, 3>;
std::atomic<int> g_pair_clusters[64];  // co-resident CTA pairs per device (-1: none)

// the most clusters of two of `fn` (smem bytes each) the device holds at once, or -1
template <typename F>
int pair_capacity(bem_ctx* c, F* fn, int smem) {
  if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) != cudaSuccess) return -1;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(2 * (unsigned)c->sm_count);
  cfg.blockDim = dim3(kThreads);
  cfg.dynamicSmemBytes = smem;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = 2;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  int n = 0;
  if (cudaOccupancyMaxActiveClusters(&n, fn, &cfg) != cudaSuccess || n <= 0) return -1;
  return n;
}

// Kernel attributes (per device), and how many CTA pairs the device holds at once;
// called before a factorisation is captured into a graph.
int umma_setup(bem_ctx* c) {
  static DeviceOnce attr;  // the kernel attribute is per device
  if (attr.pending()) {
    int pc = pair_capacity(c, umma_pair_kernel<1, 6, false>, KP1::smem);
    const int p3 = pair_capacity(c, umma_pair_kernel<3, 3, false>, KP3::smem);
    const int p3s = pair_capacity(c, umma_pair_kernel<3, 3, true>, KP3::smem);
    pc = std::min(pc, std::min(p3, p3s));
    cudaGetLastError();  // a device without room for the pair kernels keeps the single-CTA kernel
    g_pair_clusters[current_device()].store(pc);
    if (std::getenv("BEM_LU_PROFILE"))
      std::fprintf(stderr, "umma: %d CTA pairs resident per launch (-1: single CTAs)\n", pc);
    BEM_CUDA(c, cudaFuncSetAttribute(umma_update_kernel<1, 4, 1, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     K1::smem));
    BEM_CUDA(c, cudaFuncSetAttribute(umma_update_kernel<3, 2, 1, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     K3::smem));
    BEM_CUDA(c, cudaFuncSetAttribute(umma_update_kernel<3, 2, 1, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     K3::smem));
    attr.mark();
  }
  return BEM_OK;
}

}  // namespace

bool umma_supported(int K) { return K > 0 && K <= kMaxK && K % UK == 0; }

// Grows the BF16 operand buffer to what an M x N x K update needs (before a captured
// factorisation, whose first trailing update is its largest).
int umma_reserve(bem_ctx* c, int M, int N, int K) {
  if (int rc = umma_setup(c)) return rc;
  const size_t need = 2 * ((size_t)M * K + (size_t)N * K) * sizeof(__nv_bfloat16) + 256;
  if (c->umma_buf.count < need) {
    c->umma_buf.release();
    BEM_CUDA(c, c->umma_buf.alloc(need));
  }
  if (c->umma_err.count < 1) BEM_CUDA(c, c->umma_err.alloc(1));
  return BEM_OK;
}

// C (M x N) -= A (M x K) * B (K x N) on tcgen05: nprod = 3, the three-term BF16 split
// (FP32-grade products); nprod = 1, one BF16 product (hi * hi).  store: C = A B
// instead (three products only; the epilogue's boxes are stored, not added).  kmode 1
// (A lower triangular) or 2 (B upper triangular): each tile runs only the K chunks that
// meet the operand's nonzero part.
int gemm_umma_bf16(bem_ctx* c, int M, int N, int K, const float* A, int64_t lda, const float* B, int64_t ldb,
                   float* C, int64_t ldc, int nprod, bool store, int kmode) {
  if (kmode < 0 || kmode > 2) return bem_fail(c, BEM_ERR_ARG, "umma: kmode must be 0, 1 or 2");
  if (nprod != 1 && nprod != 3) return bem_fail(c, BEM_ERR_ARG, "umma: nprod must be 1 or 3");
  if (store && nprod != 3) return bem_fail(c, BEM_ERR_ARG, "umma: the storing form takes three products");
  if (!umma_supported(K)) return bem_fail(c, BEM_ERR_ARG, "umma: K must be a multiple of 64 up to 1024");
  if (!g_encode) {
    cudaDriverEntryPointQueryResult q;
    void* fn = nullptr;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess || !fn)
      return bem_fail(c, BEM_ERR_CUDA, "cuTensorMapEncodeTiled not available");
    g_encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
  }
  if (int rc = umma_setup(c)) return rc;
  const size_t na = (size_t)M * K, nb_ = (size_t)N * K;
  const size_t need = 2 * (na + nb_) * sizeof(__nv_bfloat16) + 256;
  if (c->umma_buf.count < need) {
    c->umma_buf.release();
    BEM_CUDA(c, c->umma_buf.alloc(need));
  }
  if (c->umma_err.count < 1) BEM_CUDA(c, c->umma_err.alloc(1));
  __nv_bfloat16* ah = reinterpret_cast<__nv_bfloat16*>(c->umma_buf.p);
  __nv_bfloat16* al = ah + na;
  __nv_bfloat16* bh = al + na;
  __nv_bfloat16* bl = bh + nb_;
  const int64_t ta = (int64_t)M * (K / 8), tb = (int64_t)N * (K / 8);
  split_a_kernel<<<(unsigned)((ta + 255) / 256), 256, 0, c->stream>>>(M, K, A, lda, ah, nprod == 3 ? al : nullptr);
  BEM_LAUNCH_CHECK(c);
  split_b_kernel<<<(unsigned)((tb + 255) / 256), 256, 0, c->stream>>>(N, K, B, ldb, bh, nprod == 3 ? bl : nullptr);
  BEM_LAUNCH_CHECK(c);
  CUtensorMap mAh, mAl, mBh, mBl;
  if (!make_map(&mAh, ah, M, K, UM) || !make_map(&mAl, al, M, K, UM) || !make_map(&mBh, bh, N, K, UN) ||
      !make_map(&mBl, bl, N, K, UN))
    return bem_fail(c, BEM_ERR_CUDA, "umma: tensor map encoding failed");
  const int64_t tiles = (int64_t)((M + UM - 1) / UM) * ((N + UN - 1) / UN);
  if (tiles > INT32_MAX) return bem_fail(c, BEM_ERR_ARG, "umma: too many tiles");
  // C: FP32, column-major; box 128 rows x 32 columns.  The base is 16-byte aligned
  // (the trailing block of an lda-multiple-of-32 matrix at a 256-multiple offset) and
  // ldc * 4 is a multiple of 16 bytes.
  if ((reinterpret_cast<uintptr_t>(C) & 15) != 0 || (ldc * 4) % 16 != 0)
    return bem_fail(c, BEM_ERR_ARG, "umma: C must be 16-byte aligned with ldc a multiple of 4");
  CUtensorMap mC;
  {
    cuuint64_t dims[2] = {(cuuint64_t)M, (cuuint64_t)N};
    cuuint64_t strides[1] = {(cuuint64_t)ldc * 4};
    cuuint32_t box[2] = {(cuuint32_t)UM, 32u};
    cuuint32_t estr[2] = {1, 1};
    if (g_encode(&mC, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, C, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                 CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_NONE,
                 CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
      return bem_fail(c, BEM_ERR_CUDA, "umma: tensor map encoding of C failed");
  }
  // CTA pairs for tiles of more than 128 rows (BEM_UMMA_PAIR=0: single CTAs)
  const int pairs = g_pair_clusters[current_device()].load();
  static const bool pair_env = [] {
    const char* e = std::getenv("BEM_UMMA_PAIR");
    return !(e && std::atoi(e) == 0);
  }();
  if (M > UM && pairs > 0 && pair_env) {
    CUtensorMap mBph, mBpl;  // B halves of 128 columns per CTA
    if (!make_map(&mBph, bh, N, K, PK) || !make_map(&mBpl, bl, N, K, PK))
      return bem_fail(c, BEM_ERR_CUDA, "umma: tensor map encoding failed");
    const int64_t ptiles = (int64_t)((M + 2 * UM - 1) / (2 * UM)) * ((N + UN - 1) / UN);
    const int pgrid = 2 * (int)std::min<int64_t>(ptiles, pairs);
    if (store)
      umma_pair_kernel<3, 3, true><<<pgrid, kThreads, KP3::smem, c->stream>>>(mAh, mAl, mBph, mBpl, mC, M, N, K,
                                                                              kmode, c->umma_err.p, c->wait_ns);
    else if (nprod == 3)
      umma_pair_kernel<3, 3, false><<<pgrid, kThreads, KP3::smem, c->stream>>>(mAh, mAl, mBph, mBpl, mC, M, N, K,
                                                                               kmode, c->umma_err.p, c->wait_ns);
    else
      umma_pair_kernel<1, 6, false><<<pgrid, kThreads, KP1::smem, c->stream>>>(mAh, mAl, mBph, mBpl, mC, M, N, K,
                                                                               kmode, c->umma_err.p, c->wait_ns);
    BEM_LAUNCH_CHECK(c);
    return BEM_OK;
  }
  const int grid = (int)std::min<int64_t>(tiles, c->sm_count);
  if (store)
    umma_update_kernel<3, 2, 1, true><<<grid, kThreads, K3::smem, c->stream>>>(mAh, mAl, mBh, mBl, mC, M, N, K,
                                                                               kmode, c->umma_err.p, c->wait_ns);
  else if (nprod == 3)
    umma_update_kernel<3, 2, 1, false><<<grid, kThreads, K3::smem, c->stream>>>(mAh, mAl, mBh, mBl, mC, M, N, K,
                                                                                kmode, c->umma_err.p, c->wait_ns);
  else
    umma_update_kernel<1, 4, 1, false><<<grid, kThreads, K1::smem, c->stream>>>(mAh, mAl, mBh, mBl, mC, M, N, K,
                                                                                kmode, c->umma_err.p, c->wait_ns);
  BEM_LAUNCH_CHECK(c);
  return BEM_OK;
}

}  // namespace bem
