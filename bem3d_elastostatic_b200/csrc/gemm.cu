// Tensor-core GEMMs for the LU trailing update, column-major C (M x N) op= A (M x K) B (K x N).
//
//   dgemm_dmma_kernel   FP64 operands and accumulators on the FP64 tensor path
//                       (mma.sync m8n8k4 .f64).  CTA tile 128x128x16, 8 warps of
//                       64x32, cp.async double-buffered shared-memory tiles with
//                       conflict-free pitches.
//   sgemm_bf16_kernel   FP32 operands rounded to BF16 on the way into shared memory,
//                       FP32 accumulation (mma.sync m16n8k16 .bf16, ldmatrix fragments).
//                       SPLIT = 3 carries each operand as hi + lo BF16 parts and sums
//                       hi*hi + hi*lo + lo*hi, which keeps ~16 mantissa bits of every
//                       product (an FP32-grade factorisation); SPLIT = 1 is plain BF16.
// Both require 16-byte aligned bases and leading dimensions that keep every column
// 16-byte aligned; gemm() falls back to the SIMT kernel otherwise.
#include <cuda_bf16.h>

#include "lu.cuh"

namespace bem {

// ---------------------------------------------------------------------------------
// FP64: DMMA
// ---------------------------------------------------------------------------------
namespace {
constexpr int DBM = 128, DBN = 128, DBK = 16;
constexpr int DPA = DBM + 4;  // As[k][m] pitch (doubles)
constexpr int DPB = DBK + 4;  // Bs[n][k] pitch (doubles)
constexpr size_t kDmmaSmem = 2 * (DBK * DPA + DBN * DPB) * sizeof(double);

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, int src_bytes) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b) {
  asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}
}  // namespace

template <int MODE>
__global__ void __launch_bounds__(256, 1)
    dgemm_dmma_kernel(int M, int N, int K, const double* __restrict__ A, int64_t lda, const double* __restrict__ B,
                      int64_t ldb, double* C, int64_t ldc) {
  extern __shared__ __align__(16) double dsm[];
  double* As = dsm;                      // [2][DBK][DPA]
  double* Bs = dsm + 2 * DBK * DPA;      // [2][DBN][DPB]
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = (warp >> 2) * 64;  // 2 warps along M
  const int wn = (warp & 3) * 32;   // 4 warps along N
  const int m0 = blockIdx.y * DBM, n0 = blockIdx.x * DBN;

  auto load_tile = [&](int buf, int k0) {
    double* as = As + buf * DBK * DPA;
    double* bs = Bs + buf * DBN * DPB;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int idx = tid + 256 * i;
      {  // A: 16 k x 64 m-pairs
        const int k = idx >> 6, m = (idx & 63) * 2;
        const int gm = m0 + m, gk = k0 + k;
        int bytes = 0;
        if (gk < K && gm < M) bytes = (gm + 1 < M) ? 16 : 8;
        const double* src = bytes ? A + gm + (int64_t)gk * lda : A;
        cp_async16(as + k * DPA + m, src, bytes);
      }
      {  // B: 128 n x 8 k-pairs
        const int n = idx >> 3, k = (idx & 7) * 2;
        const int gn = n0 + n, gk = k0 + k;
        int bytes = 0;
        if (gn < N && gk < K) bytes = (gk + 1 < K) ? 16 : 8;
        const double* src = bytes ? B + gk + (int64_t)gn * ldb : B;
        cp_async16(bs + n * DPB + k, src, bytes);
      }
    }
    cp_async_commit();
  };

  double acc[8][4][2];
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;

  const int nk = (K + DBK - 1) / DBK;
  load_tile(0, 0);
  for (int kt = 0; kt < nk; ++kt) {
    const int buf = kt & 1;
    cp_async_wait_all();
    __syncthreads();
    if (kt + 1 < nk) load_tile(buf ^ 1, (kt + 1) * DBK);
    const double* as = As + buf * DBK * DPA;
    const double* bs = Bs + buf * DBN * DPB;
#pragma unroll
    for (int kk = 0; kk < DBK; kk += 4) {
      double a[8], b[4];
#pragma unroll
      for (int i = 0; i < 8; ++i) a[i] = as[(kk + (lane & 3)) * DPA + wm + 8 * i + (lane >> 2)];
#pragma unroll
      for (int j = 0; j < 4; ++j) b[j] = bs[(wn + 8 * j + (lane >> 2)) * DPB + kk + (lane & 3)];
#pragma unroll
      for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) dmma(acc[i][j][0], acc[i][j][1], a[i], b[j]);
    }
  }
  // epilogue: two row-tiles at a time, every load of C issued before any store so the
  // read-modify-write costs one memory round trip per chunk, not one per element
#pragma unroll
  for (int i0 = 0; i0 < 8; i0 += 2) {
    double old[2][4][2];
#pragma unroll
    for (int di = 0; di < 2; ++di) {
      const int gm = m0 + wm + 8 * (i0 + di) + (lane >> 2);
#pragma unroll
      for (int j = 0; j < 4; ++j)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int gn = n0 + wn + 8 * j + 2 * (lane & 3) + h;
          old[di][j][h] = (MODE == 0 && gm < M && gn < N) ? C[gm + (int64_t)gn * ldc] : 0.0;
        }
    }
#pragma unroll
    for (int di = 0; di < 2; ++di) {
      const int gm = m0 + wm + 8 * (i0 + di) + (lane >> 2);
#pragma unroll
      for (int j = 0; j < 4; ++j)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int gn = n0 + wn + 8 * j + 2 * (lane & 3) + h;
          if (gm < M && gn < N)
            C[gm + (int64_t)gn * ldc] = (MODE == 0) ? old[di][j][h] - acc[i0 + di][j][h] : acc[i0 + di][j][h];
        }
    }
  }
}

// ---------------------------------------------------------------------------------
// FP32 data, BF16 tensor cores
// ---------------------------------------------------------------------------------
namespace {
constexpr int HBM_ = 128, HBN = 128, HBK = 32;
constexpr int HPA = HBM_ + 8;  // As[k][m] pitch (bf16): 272 B rows
constexpr int HPB = HBK + 8;   // Bs[n][k] pitch (bf16): 80 B rows

__device__ __forceinline__ void ldsm_x4(unsigned& r0, unsigned& r1, unsigned& r2, unsigned& r3, const void* p) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(p);
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
               : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
               : "r"(s));
}
__device__ __forceinline__ void ldsm_x4_t(unsigned& r0, unsigned& r1, unsigned& r2, unsigned& r3, const void* p) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(p);
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];\n"
               : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
               : "r"(s));
}
__device__ __forceinline__ void hmma(float* c, const unsigned* a, const unsigned* b) {
  asm(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}
__device__ __forceinline__ void split_bf16(float v, __nv_bfloat16& hi, __nv_bfloat16& lo) {
  hi = __float2bfloat16_rn(v);
  lo = __float2bfloat16_rn(v - __bfloat162float(hi));
}
}  // namespace

template <int MODE, int SPLIT>
__global__ void __launch_bounds__(256, 1)
    sgemm_bf16_kernel(int M, int N, int K, const float* __restrict__ A, int64_t lda, const float* __restrict__ B,
                      int64_t ldb, float* C, int64_t ldc) {
  constexpr int NP = (SPLIT == 3) ? 2 : 1;  // hi (+ lo) planes
  extern __shared__ __align__(16) unsigned char hsm[];
  __nv_bfloat16* As = reinterpret_cast<__nv_bfloat16*>(hsm);  // [NP][HBK][HPA]
  __nv_bfloat16* Bs = As + NP * HBK * HPA;                     // [NP][HBN][HPB]
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = (warp >> 2) * 64, wn = (warp & 3) * 32;
  const int m0 = blockIdx.y * HBM_, n0 = blockIdx.x * HBN;

  float4 ra[4], rb[4];
  auto gload = [&](int k0) {
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int idx = tid + 256 * i;
      {  // A: 32 k x 32 m-quads
        const int k = idx >> 5, m = (idx & 31) * 4;
        const int gm = m0 + m, gk = k0 + k;
        float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
        if (gk < K) {
          const float* p = A + gm + (int64_t)gk * lda;
          if (gm + 3 < M)
            v = *reinterpret_cast<const float4*>(p);
          else {
            if (gm < M) v.x = p[0];
            if (gm + 1 < M) v.y = p[1];
            if (gm + 2 < M) v.z = p[2];
          }
        }
        ra[i] = v;
      }
      {  // B: 128 n x 8 k-quads
        const int n = idx >> 3, k = (idx & 7) * 4;
        const int gn = n0 + n, gk = k0 + k;
        float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
        if (gn < N) {
          const float* p = B + gk + (int64_t)gn * ldb;
          if (gk + 3 < K)
            v = *reinterpret_cast<const float4*>(p);
          else {
            if (gk < K) v.x = p[0];
            if (gk + 1 < K) v.y = p[1];
            if (gk + 2 < K) v.z = p[2];
          }
        }
        rb[i] = v;
      }
    }
  };
  auto sstore = [&]() {
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int idx = tid + 256 * i;
      {
        const int k = idx >> 5, m = (idx & 31) * 4;
        const float f[4] = {ra[i].x, ra[i].y, ra[i].z, ra[i].w};
        __align__(8) __nv_bfloat16 h[4], l[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) split_bf16(f[q], h[q], l[q]);
        *reinterpret_cast<uint2*>(As + k * HPA + m) = *reinterpret_cast<uint2*>(h);
        if (NP == 2) *reinterpret_cast<uint2*>(As + HBK * HPA + k * HPA + m) = *reinterpret_cast<uint2*>(l);
      }
      {
        const int n = idx >> 3, k = (idx & 7) * 4;
        const float f[4] = {rb[i].x, rb[i].y, rb[i].z, rb[i].w};
        __align__(8) __nv_bfloat16 h[4], l[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) split_bf16(f[q], h[q], l[q]);
        *reinterpret_cast<uint2*>(Bs + n * HPB + k) = *reinterpret_cast<uint2*>(h);
        if (NP == 2) *reinterpret_cast<uint2*>(Bs + HBN * HPB + n * HPB + k) = *reinterpret_cast<uint2*>(l);
      }
    }
  };

  float acc[4][4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[i][j][q] = 0.f;

  const int nk = (K + HBK - 1) / HBK;
  gload(0);
  for (int kt = 0; kt < nk; ++kt) {
    __syncthreads();
    sstore();
    __syncthreads();
    if (kt + 1 < nk) gload((kt + 1) * HBK);
#pragma unroll
    for (int kk = 0; kk < HBK; kk += 16) {
      unsigned a[NP][4][4], b[NP][4][2];
#pragma unroll
      for (int p = 0; p < NP; ++p) {
        const __nv_bfloat16* as = As + p * HBK * HPA;
        const __nv_bfloat16* bs = Bs + p * HBN * HPB;
        const int q = lane >> 3, r = lane & 7;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          const int kb = (q & 2) ? 8 : 0, mb = (q & 1) ? 8 : 0;
          ldsm_x4_t(a[p][i][0], a[p][i][1], a[p][i][2], a[p][i][3],
                    as + (kk + kb + r) * HPA + wm + 16 * i + mb);
        }
#pragma unroll
        for (int j = 0; j < 4; j += 2) {
          const int nb = (q & 2) ? 8 : 0, kb = (q & 1) ? 8 : 0;
          ldsm_x4(b[p][j][0], b[p][j][1], b[p][j + 1][0], b[p][j + 1][1],
                  bs + (wn + 8 * j + nb + r) * HPB + kk + kb);
        }
      }
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          if (SPLIT == 3) {
            hmma(acc[i][j], a[1][i], b[0][j]);
            hmma(acc[i][j], a[0][i], b[1][j]);
          }
          hmma(acc[i][j], a[0][i], b[0][j]);
        }
    }
  }
  // epilogue: one 16-row tile at a time, loads before stores (see the FP64 kernel)
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    float old[4][4];
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int gm = m0 + wm + 16 * i + (lane >> 2) + ((q & 2) ? 8 : 0);
        const int gn = n0 + wn + 8 * j + 2 * (lane & 3) + (q & 1);
        old[j][q] = (MODE == 0 && gm < M && gn < N) ? C[gm + (int64_t)gn * ldc] : 0.f;
      }
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int gm = m0 + wm + 16 * i + (lane >> 2) + ((q & 2) ? 8 : 0);
        const int gn = n0 + wn + 8 * j + 2 * (lane & 3) + (q & 1);
        if (gm < M && gn < N) C[gm + (int64_t)gn * ldc] = (MODE == 0) ? old[j][q] - acc[i][j][q] : acc[i][j][q];
      }
  }
}

// ---------------------------------------------------------------------------------
// dispatch
// ---------------------------------------------------------------------------------
static bool aligned16(const void* p) { return ((uintptr_t)p & 15) == 0; }

int gemm_dmma(bem_ctx* c, int M, int N, int K, const double* A, int64_t lda, const double* B, int64_t ldb, double* C,
              int64_t ldc, int mode) {
  static DeviceOnce attr;
  if (attr.pending()) {
    cudaFuncSetAttribute(dgemm_dmma_kernel<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kDmmaSmem);
    cudaFuncSetAttribute(dgemm_dmma_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kDmmaSmem);
    attr.mark();
  }
  dim3 grid((N + DBN - 1) / DBN, (M + DBM - 1) / DBM);
  if (mode == 0)
    dgemm_dmma_kernel<0><<<grid, 256, kDmmaSmem, c->stream>>>(M, N, K, A, lda, B, ldb, C, ldc);
  else
    dgemm_dmma_kernel<1><<<grid, 256, kDmmaSmem, c->stream>>>(M, N, K, A, lda, B, ldb, C, ldc);
  BEM_LAUNCH_CHECK(c);
  return BEM_OK;
}

int gemm_bf16(bem_ctx* c, int M, int N, int K, const float* A, int64_t lda, const float* B, int64_t ldb, float* C,
              int64_t ldc, int mode, int split) {
  static DeviceOnce attr;
  const size_t smem1 = (size_t)(HBK * HPA + HBN * HPB) * sizeof(__nv_bfloat16);
  const size_t smem3 = 2 * smem1;
  if (attr.pending()) {
    cudaFuncSetAttribute(sgemm_bf16_kernel<0, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem1);
    cudaFuncSetAttribute(sgemm_bf16_kernel<1, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem1);
    cudaFuncSetAttribute(sgemm_bf16_kernel<0, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem3);
    cudaFuncSetAttribute(sgemm_bf16_kernel<1, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem3);
    attr.mark();
  }
  dim3 grid((N + HBN - 1) / HBN, (M + HBM_ - 1) / HBM_);
  if (split == 3) {
    if (mode == 0)
      sgemm_bf16_kernel<0, 3><<<grid, 256, smem3, c->stream>>>(M, N, K, A, lda, B, ldb, C, ldc);
    else
      sgemm_bf16_kernel<1, 3><<<grid, 256, smem3, c->stream>>>(M, N, K, A, lda, B, ldb, C, ldc);
  } else {
    if (mode == 0)
      sgemm_bf16_kernel<0, 1><<<grid, 256, smem1, c->stream>>>(M, N, K, A, lda, B, ldb, C, ldc);
    else
      sgemm_bf16_kernel<1, 1><<<grid, 256, smem1, c->stream>>>(M, N, K, A, lda, B, ldb, C, ldc);
  }
  BEM_LAUNCH_CHECK(c);
  return BEM_OK;
}

bool gemm_tc_ok(const void* A, int64_t lda, const void* B, int64_t ldb, int elem) {
  const int q = 16 / elem;  // elements per 16 bytes
  return aligned16(A) && aligned16(B) && (lda % q) == 0 && (ldb % q) == 0;
}

}  // namespace bem
