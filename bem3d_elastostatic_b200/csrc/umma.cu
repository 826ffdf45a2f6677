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
#include <cstdint>

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
    for (int t = blockIdx.x; t < total && !*abort_flag; t += gridDim.x) {
      int m0, n0;
      coords(t, m0, n0);
      // the four warps of a half leave together (they meet at named barriers below)
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

}  // namespace

bool umma_supported(int K) { return K > 0 && K <= kMaxK && K % UK == 0; }

// Grows the BF16 operand buffer to what an M x N x K update needs (before a captured
// factorisation, whose first trailing update is its largest).
int umma_reserve(bem_ctx* c, int M, int N, int K) {
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
  // one product: four ring stages (48 KB each); three products: two (96 KB each); one
  // staging box per epilogue half (two measured no faster)
  using K1 = Cfg<1, 4, 1>;
  using K3 = Cfg<3, 2, 1>;
  static DeviceOnce attr;  // the kernel attribute is per device
  if (attr.pending()) {
    BEM_CUDA(c, cudaFuncSetAttribute(umma_update_kernel<1, 4, 1, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     K1::smem));
    BEM_CUDA(c, cudaFuncSetAttribute(umma_update_kernel<3, 2, 1, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     K3::smem));
    BEM_CUDA(c, cudaFuncSetAttribute(umma_update_kernel<3, 2, 1, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     K3::smem));
    attr.mark();
  }
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
