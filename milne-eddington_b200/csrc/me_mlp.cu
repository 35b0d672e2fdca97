// me_mlp.cu -- the learned initialiser: a small MLP that maps a normalised
// Stokes profile to the nine ME parameters, trained on the GPU on profiles the
// GPU forward model synthesises from seeded parameter draws plus noise.
//
//   features (4 nl)  ->  256 GELU  ->  256 GELU  ->  256 GELU  ->  10 outputs
//   outputs: B, cos(theta), sin(2 phi), cos(2 phi), v, Doppler width, a, eta0,
//            beta, S / I_max, each standardised with the training-set moments.
//
// Everything is hand-written here: the data synthesis, BF16 tensor-core GEMMs
// (mma.sync m16n8k16, FP32 accumulation) with fused bias / GELU epilogues,
// the backward pass, Adam with FP32 master weights, and the inference that
// turns a map into per-pixel starting parameters for the LM.  The reference
// has no learned part; the plain LM with its restarts stays the fallback.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/me_b200.h"
#include "me_kernels.h"
#include "me_umma.cuh"

namespace me {
namespace mlp {

constexpr int kHidden = 256;
constexpr int kOut = 10;
constexpr int kLayers = 4;
typedef __nv_bfloat16 bf16;

// ---------------------------------------------------------------------------
// GEMM: C[M x N] = A[M x R] * Bt[N x R]^T, A and Bt row-major BF16 with R
// contiguous (R % 32 == 0), FP32 accumulation on the tensor cores
// (mma.sync.m16n8k16.row.col.f32.bf16.bf16.f32).  Epilogue: + bias[n] (if
// given), store FP32 pre-activation Z (if given), then GELU (if gelu) into
// BF16 Y (if given) and/or FP32 Yf (if given).  CTA tile 64 x 64, 4 warps of
// 32 x 32, K steps of 32 through shared memory.
// ---------------------------------------------------------------------------
constexpr int kTM = 64, kTN = 64, kTK = 32;

__device__ __forceinline__ void mma_bf16(float c[4], const unsigned a[4], const unsigned b[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
      "{%8,%9}, {%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

__device__ __forceinline__ float gelu_f(float z) {
  return 0.5f * z * (1.f + erff(z * 0.70710678118654752f));
}
__device__ __forceinline__ float gelu_grad(float z) {
  const float cdf = 0.5f * (1.f + erff(z * 0.70710678118654752f));
  const float pdf = 0.3989422804014327f * __expf(-0.5f * z * z);
  return cdf + z * pdf;
}

__global__ void __launch_bounds__(128) gemm_kernel(const bf16 *__restrict__ A,
                                                   const bf16 *__restrict__ Bt, int M, int N,
                                                   int R, const float *__restrict__ bias,
                                                   float *__restrict__ Z, int gelu,
                                                   bf16 *__restrict__ Y, float *__restrict__ Yf) {
  __shared__ __align__(16) bf16 sA[kTM][kTK + 8];
  __shared__ __align__(16) bf16 sB[kTN][kTK + 8];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int m0 = blockIdx.y * kTM, n0 = blockIdx.x * kTN;
  const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
  const int g = lane >> 2, t4 = lane & 3;
  float acc[2][4][4];
#pragma unroll
  for (int i = 0; i < 2; i++)
#pragma unroll
    for (int j = 0; j < 4; j++)
#pragma unroll
      for (int k = 0; k < 4; k++) acc[i][j][k] = 0.f;
  // split-K: blockIdx.z takes R / gridDim.z of the reduction (a multiple of
  // kTK); partial sums are added into Yf, which the caller zeroes
  const int rz = R / (int)gridDim.z;
  const int kbeg = blockIdx.z * rz, kend = kbeg + rz;
  for (int k0 = kbeg; k0 < kend; k0 += kTK) {
    // 64 x 32 BF16 tiles: 128 threads x 16 elements (two 16-byte chunks) each
#pragma unroll
    for (int c = 0; c < 2; c++) {
      const int chunk = tid + c * 128;  // 256 chunks of 8 elements
      const int r = chunk >> 2, col = (chunk & 3) * 8;
      uint4 va = make_uint4(0, 0, 0, 0), vb = make_uint4(0, 0, 0, 0);
      if (m0 + r < M) va = *reinterpret_cast<const uint4 *>(A + (size_t)(m0 + r) * R + k0 + col);
      if (n0 + r < N) vb = *reinterpret_cast<const uint4 *>(Bt + (size_t)(n0 + r) * R + k0 + col);
      *reinterpret_cast<uint4 *>(&sA[r][col]) = va;
      *reinterpret_cast<uint4 *>(&sB[r][col]) = vb;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < kTK; kk += 16) {
      unsigned af[2][4], bfr[4][2];
#pragma unroll
      for (int i = 0; i < 2; i++) {
        const int r = wm + i * 16 + g;
        af[i][0] = *reinterpret_cast<const unsigned *>(&sA[r][kk + t4 * 2]);
        af[i][1] = *reinterpret_cast<const unsigned *>(&sA[r + 8][kk + t4 * 2]);
        af[i][2] = *reinterpret_cast<const unsigned *>(&sA[r][kk + 8 + t4 * 2]);
        af[i][3] = *reinterpret_cast<const unsigned *>(&sA[r + 8][kk + 8 + t4 * 2]);
      }
#pragma unroll
      for (int j = 0; j < 4; j++) {
        const int n = wn + j * 8 + g;
        bfr[j][0] = *reinterpret_cast<const unsigned *>(&sB[n][kk + t4 * 2]);
        bfr[j][1] = *reinterpret_cast<const unsigned *>(&sB[n][kk + 8 + t4 * 2]);
      }
#pragma unroll
      for (int i = 0; i < 2; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) mma_bf16(acc[i][j], af[i], bfr[j]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 2; i++) {
#pragma unroll
    for (int j = 0; j < 4; j++) {
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const int m = m0 + wm + i * 16 + g + h * 8;
        if (m >= M) continue;
#pragma unroll
        for (int e = 0; e < 2; e++) {
          const int n = n0 + wn + j * 8 + t4 * 2 + e;
          if (n >= N) continue;
          float z = acc[i][j][h * 2 + e];
          if (gridDim.z > 1) {
            atomicAdd(Yf + (size_t)m * N + n, z);
            continue;
          }
          if (bias) z += bias[n];
          if (Z) Z[(size_t)m * N + n] = z;
          const float y = gelu ? gelu_f(z) : z;
          if (Y) Y[(size_t)m * N + n] = __float2bfloat16(y);
          if (Yf) Yf[(size_t)m * N + n] = y;
        }
      }
    }
  }
}

// ---------------------------------------------------------------------------
// The same GEMM and epilogue on the sm_100a tensor cores.  A CTA owns a
// 128 x bn tile of C (bn = N up to 256, N % 16 == 0); TMA brings 128 x 64 and
// bn x 64 BF16 tiles of A and Bt into a two-stage ring of 128-byte-swizzled
// shared memory; thread 0 issues four tcgen05.mma (K = 16 each) per stage into
// an FP32 accumulator of bn tensor-memory columns and commits each stage to
// the mbarrier that frees it for the next load; after the last commit every
// warp reads its 32 accumulator rows with tcgen05.ld and applies the epilogue
// (bias, Z, GELU, Y, Yf, or split-K atomics) on 16-column chunks.  Waits are
// bounded: on expiry the CTA writes a code to *err (1: operand load, 2: stage
// release, 3: accumulator), drains what it issued, frees its tensor memory
// and leaves C unwritten.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(128, 1)
    umma_gemm_kernel(const __grid_constant__ CUtensorMap tmA,
                     const __grid_constant__ CUtensorMap tmB, int M, int N, int R, int bn,
                     const float *__restrict__ bias, float *__restrict__ Z, int gelu,
                     bf16 *__restrict__ Y, float *__restrict__ Yf, int *__restrict__ err) {
  using namespace me::umma;
  extern __shared__ uint8_t smem_raw[];
  const uint32_t raw = smem_u32(smem_raw);
  const uint32_t base = (raw + 1023u) & ~1023u;
  const uint32_t stB = (uint32_t)bn * kBK * 2;  // a multiple of 2048: bn % 16 == 0
  const uint32_t sA = base, sB = base + kStages * kStageA;
  const uint32_t bars = sB + kStages * stB;
  // full[s] = bars + 8 s, empty[s] = bars + 8 (kStages + s), done after them
  const uint32_t done = bars + 8 * 2 * kStages;
  uint32_t *misc = reinterpret_cast<uint32_t *>(smem_raw + (done + 8 - raw));
  volatile uint32_t *abort_flag = misc + 1;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t ncols = tmem_cols(bn);

  if (warp == 0) {
    tmem_alloc(smem_u32(misc), ncols);
    tmem_relinquish();
  }
  if (threadIdx.x == 32) {
    for (int s = 0; s < kStages; s++) {
      mbar_init(bars + 8 * s, 1);
      mbar_init(bars + 8 * (kStages + s), 1);
    }
    mbar_init(done, 1);
    *abort_flag = 0;
    mbar_fence_init();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = misc[0];

  const int m0 = blockIdx.y * kBM, n0 = blockIdx.x * bn;
  const int rz = R / (int)gridDim.z, kbeg = blockIdx.z * rz;
  const int nk = (rz + kBK - 1) / kBK;
  const uint32_t tx = (uint32_t)(kBM + bn) * kBK * 2;

  if (warp == 0) {
    if (lane == 0) {
      const uint32_t idesc = idesc_bf16_f32(kBM, bn);
      int code = 0, loaded = 0, kb = 0;
      for (; loaded < nk && loaded < kStages; loaded++) {
        const uint32_t full = bars + 8 * loaded;
        mbar_expect_tx(full, tx);
        tma_load_2d(sA + loaded * kStageA, &tmA, full, kbeg + loaded * kBK, m0);
        tma_load_2d(sB + loaded * stB, &tmB, full, kbeg + loaded * kBK, n0);
      }
      for (; kb < nk; kb++) {
        const int s = kb % kStages;
        if (!mbar_wait(bars + 8 * s, (uint32_t)(kb / kStages) & 1u)) {
          code = 1;
          break;
        }
        tc_fence_after();
#pragma unroll
        for (int k = 0; k < kBK / 16; k++)
          umma_bf16(tmem, sw128_kmajor_desc(sA + s * kStageA + 32 * k),
                   sw128_kmajor_desc(sB + s * stB + 32 * k), idesc, (kb | k) != 0);
        mma_commit(bars + 8 * (kStages + s));
        // refill the stage of the previous k block once its MMAs have read it
        if (kb >= 1 && loaded < nk) {
          const int ls = loaded % kStages;  // == (kb - 1) % kStages
          if (!mbar_wait(bars + 8 * (kStages + ls), (uint32_t)(loaded / kStages - 1) & 1u)) {
            code = 2;
            break;
          }
          const uint32_t full = bars + 8 * ls;
          mbar_expect_tx(full, tx);
          tma_load_2d(sA + ls * kStageA, &tmA, full, kbeg + loaded * kBK, m0);
          tma_load_2d(sB + ls * stB, &tmB, full, kbeg + loaded * kBK, n0);
          loaded++;
        }
      }
      mma_commit(done);  // tracks every MMA issued above
      if (code) {
        // loads issued and not consumed: let them land before the CTA exits
        for (int j = kb; j < loaded; j++) mbar_wait(bars + 8 * (j % kStages), (uint32_t)(j / kStages) & 1u);
        *abort_flag = 1;
        atomicExch(err, code);
      }
    }
    __syncwarp();
  }
  if (!mbar_wait(done, 0)) {
    *abort_flag = 1;
    atomicExch(err, 3);
  }
  __syncthreads();
  tc_fence_after();
  if (!*abort_flag) {
    const int row = m0 + warp * 32 + lane;
    const uint32_t trow = tmem + ((uint32_t)(warp * 32) << 16);
    for (int c = 0; c < bn; c += 16) {
      const int n = n0 + c;
      if (n >= N) break;  // the same for the whole warp
      float v[16];
      tmem_ld16(trow + (uint32_t)c, v);
      if (row >= M) continue;
      const size_t o = (size_t)row * N + n;
      if (gridDim.z > 1) {
#pragma unroll
        for (int j = 0; j < 16; j++) atomicAdd(Yf + o + j, v[j]);
        continue;
      }
      if (bias) {
#pragma unroll
        for (int j = 0; j < 16; j++) v[j] += __ldg(bias + n + j);
      }
      if (Z) {
#pragma unroll
        for (int j = 0; j < 16; j += 4)
          *reinterpret_cast<float4 *>(Z + o + j) = make_float4(v[j], v[j + 1], v[j + 2], v[j + 3]);
      }
      if (gelu) {
#pragma unroll
        for (int j = 0; j < 16; j++) v[j] = gelu_f(v[j]);
      }
      if (Y) {
        uint32_t pk[8];
#pragma unroll
        for (int j = 0; j < 8; j++) {
          const __nv_bfloat162 h = __floats2bfloat162_rn(v[2 * j], v[2 * j + 1]);
          pk[j] = *reinterpret_cast<const uint32_t *>(&h);
        }
        *reinterpret_cast<uint4 *>(Y + o) = make_uint4(pk[0], pk[1], pk[2], pk[3]);
        *reinterpret_cast<uint4 *>(Y + o + 8) = make_uint4(pk[4], pk[5], pk[6], pk[7]);
      }
      if (Yf) {
#pragma unroll
        for (int j = 0; j < 16; j += 4)
          *reinterpret_cast<float4 *>(Yf + o + j) =
              make_float4(v[j], v[j + 1], v[j + 2], v[j + 3]);
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, ncols);
}

// cuTensorMapEncodeTiled from the driver, looked up once through the runtime
// (the library does not link libcuda)
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static const PFN_cuTensorMapEncodeTiled_v12000 fn = []() {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault,
                                         &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      p = nullptr;
    return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }();
  return fn;
}

// Tensor map of a row-major BF16 matrix [rows][cols] read in boxes of
// box_rows x 64 with the 128-byte swizzle; boxes reaching past the matrix
// read zeros
bool tile_map(CUtensorMap *map, const bf16 *p, int rows, int cols, int box_rows) {
  const PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
  if (!enc || (reinterpret_cast<uintptr_t>(p) & 15) || (cols * 2) % 16 || box_rows < 1 ||
      box_rows > 256)
    return false;
  const cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)cols * 2};
  const cuuint32_t box[2] = {(cuuint32_t)me::umma::kBK, (cuuint32_t)box_rows};
  const cuuint32_t estr[2] = {1, 1};
  return enc(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<bf16 *>(p), dims, strides, box,
             estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
             CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Which GEMM runs: the tcgen05 kernel wherever its shape rules hold (N % 16 ==
// 0, each split-K share a multiple of 64, tensor maps encodable), else the
// mma.sync kernel; GemmPath::mma_sync forces the latter.
enum class GemmPath { tcgen05 = 0, mma_sync = 1 };

// Tensor maps already encoded for a model's buffers: a map is a function of
// (address, rows, columns, box rows) alone, so a hit is always valid.
struct TileMapCache {
  struct Entry {
    const void *p;
    int rows, cols, box_rows;
    CUtensorMap map;
  };
  std::vector<Entry> entries;
};

struct GemmCtx {
  GemmPath path = GemmPath::tcgen05;
  int *err = nullptr;             // device flag of the tcgen05 kernel's bounded waits
  long long *launches = nullptr;  // [2]: launches of each kernel, indexed by GemmPath
  TileMapCache *maps = nullptr;   // may be null (no caching)
};

bool cached_tile_map(TileMapCache *c, CUtensorMap *map, const bf16 *p, int rows, int cols,
                     int box_rows) {
  if (c)
    for (const TileMapCache::Entry &e : c->entries)
      if (e.p == p && e.rows == rows && e.cols == cols && e.box_rows == box_rows) {
        *map = e.map;
        return true;
      }
  if (!tile_map(map, p, rows, cols, box_rows)) return false;
  if (c) {
    if (c->entries.size() >= 256) c->entries.clear();
    c->entries.push_back({p, rows, cols, box_rows, *map});
  }
  return true;
}

// Per-device facts the launch needs, looked up once per device: the SM count
// and whether the kernel's shared-memory limit has been raised.
struct DeviceFacts {
  int sms = 0;
  bool smem_ok = false;
};

const DeviceFacts &device_facts() {
  static DeviceFacts facts[64];
  static std::once_flag once[64];
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
    static const DeviceFacts none;
    return none;
  }
  std::call_once(once[dev], [dev]() {
    DeviceFacts f;
    if (cudaDeviceGetAttribute(&f.sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
      f.sms = 0;
    f.smem_ok = cudaFuncSetAttribute(umma_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     me::umma::kSmemMax) == cudaSuccess;
    facts[dev] = f;
  });
  return facts[dev];
}

// split > 1: R % (split * kTK) == 0, only Yf (zeroed by the caller), no
// epilogue.  Returns the kernel that ran.
GemmPath gemm(const GemmCtx &g, const bf16 *A, const bf16 *Bt, int M, int N, int R,
              const float *bias, float *Z, int gelu, bf16 *Y, float *Yf, cudaStream_t st,
              int split = 1) {
  if (g.path == GemmPath::tcgen05 && g.err && N % 16 == 0 && R % split == 0 &&
      (split == 1 || (R / split) % me::umma::kBK == 0)) {
    // column tile: all of N up to 256, halved (in multiples of 16, down to
    // 32) while the grid has fewer than two CTAs per SM, so that small
    // batches still spread over the GPU
    const DeviceFacts &dv = device_facts();
    int bn = N <= me::umma::kMaxBN ? N : me::umma::kMaxBN;
    const long long tiles_m = (M + me::umma::kBM - 1) / me::umma::kBM;
    while (bn > 32 && bn % 32 == 0 &&
           (long long)((N + bn - 1) / bn) * tiles_m * split < 2LL * dv.sms)
      bn /= 2;
    CUtensorMap ma, mb;
    if (dv.smem_ok && cached_tile_map(g.maps, &ma, A, M, R, me::umma::kBM) &&
        cached_tile_map(g.maps, &mb, Bt, N, R, bn)) {
      dim3 grid((N + bn - 1) / bn, (M + me::umma::kBM - 1) / me::umma::kBM, split);
      umma_gemm_kernel<<<grid, 128, me::umma::smem_bytes(bn), st>>>(ma, mb, M, N, R, bn, bias, Z,
                                                                    gelu, Y, Yf, g.err);
      if (g.launches) g.launches[(int)GemmPath::tcgen05]++;
      return GemmPath::tcgen05;
    }
  }
  dim3 grid((N + kTN - 1) / kTN, (M + kTM - 1) / kTM, split);
  gemm_kernel<<<grid, 128, 0, st>>>(A, Bt, M, N, R, bias, Z, gelu, Y, Yf);
  if (g.launches) g.launches[(int)GemmPath::mma_sync]++;
  return GemmPath::mma_sync;
}

// out[c][r] = in[r][c] (BF16), rows x cols
__global__ void transpose_kernel(const bf16 *in, int rows, int cols, bf16 *out) {
  __shared__ bf16 tile[32][33];
  const int bx = blockIdx.x * 32, by = blockIdx.y * 32;
  for (int i = threadIdx.y; i < 32; i += 8) {
    const int r = by + i, c = bx + threadIdx.x;
    if (r < rows && c < cols) tile[i][threadIdx.x] = in[(size_t)r * cols + c];
  }
  __syncthreads();
  for (int i = threadIdx.y; i < 32; i += 8) {
    const int c = bx + i, r = by + threadIdx.x;
    if (r < rows && c < cols) out[(size_t)c * rows + r] = tile[threadIdx.x][i];
  }
}

void transpose(const bf16 *in, int rows, int cols, bf16 *out, cudaStream_t st) {
  dim3 grid((cols + 31) / 32, (rows + 31) / 32), block(32, 8);
  transpose_kernel<<<grid, block, 0, st>>>(in, rows, cols, out);
}

// ---------------------------------------------------------------------------
// Training data: parameter draws (Philox per sample) -> FP32 synthesis at the
// plan's grid -> noise -> normalised features (BF16) and encoded targets.
// ---------------------------------------------------------------------------
struct Prior {  // the training distribution
  float b_lo, b_hi, cost_lo, cost_hi, phi_lo, phi_hi, v_sigma, w_lo, w_hi, a_lo, a_hi, eta_lo,
      eta_hi, s, beta_lo, beta_hi, noise;
  // second population (B and eta0 ranges) drawn with probability mix
  float mix, mb_lo, mb_hi, meta_lo, meta_hi;
};

__device__ __forceinline__ void draws16(unsigned long long seed, long long i, float u[16]) {
#pragma unroll
  for (int blk = 0; blk < 4; blk++) {
    uint32_t c[4] = {(uint32_t)((unsigned long long)i & 0xffffffffu),
                     (uint32_t)((unsigned long long)i >> 32), 0x4D4C5000u, (uint32_t)blk};
    philox10(c, (uint32_t)(seed & 0xffffffffu), (uint32_t)(seed >> 32));
#pragma unroll
    for (int k = 0; k < 4; k++) u[blk * 4 + k] = ((float)c[k] + 0.5f) * 2.3283064365386963e-10f;
  }
}

// features of one profile: I / I_max - 1, Q, U, V / I_max (x 10), then the
// training-set standardisation (mean, inv_std); also returns I_max
__device__ __forceinline__ float feature_value(int s, float v, float imax_inv) {
  return s == 0 ? v * imax_inv - 1.f : 10.f * v * imax_inv;
}

__global__ void synth_train_kernel(const __grid_constant__ DevPlan P, Prior pr,
                                   unsigned long long seed, long long n, int ld, float *Xraw,
                                   float *Tgt) {
  __shared__ float s_tab[100];
  __shared__ float s_rden[kRden * 128];
  VoigtK<float> K;
  voigt_block_setup<float>(K, P, s_tab);
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  float u[16];
  draws16(seed, i, u);
  double par[9];
  const bool second = u[9] < pr.mix;  // u[9]: the population
  par[0] = second ? pr.mb_lo + (pr.mb_hi - pr.mb_lo) * u[0] : pr.b_lo + (pr.b_hi - pr.b_lo) * u[0];
  const double cost = pr.cost_lo + (pr.cost_hi - pr.cost_lo) * u[1];
  par[1] = acos(cost);
  par[2] = pr.phi_lo + (pr.phi_hi - pr.phi_lo) * u[2];
  // Box-Muller for v
  par[3] = pr.v_sigma * sqrt(-2.0 * log((double)u[3])) * cos(6.283185307179586 * u[4]);
  par[4] = pr.w_lo + (pr.w_hi - pr.w_lo) * u[5];
  par[5] = pr.a_lo + (pr.a_hi - pr.a_lo) * u[6];
  par[6] = second ? pr.meta_lo + (pr.meta_hi - pr.meta_lo) * u[7]
                  : pr.eta_lo + (pr.eta_hi - pr.eta_lo) * u[7];
  par[7] = pr.s;
  par[8] = pr.beta_lo + (pr.beta_hi - pr.beta_lo) * u[8];
  SynthCall<float> c;
  synth_setup<float>(c, par, P, P.step);
  voigt_prepare<float>(K, c.p5, s_rden + threadIdx.x, blockDim.x);
  const float ones[4] = {1.f, 1.f, 1.f, 1.f};
  const int nl = P.nl;
  float *xr = Xraw + (size_t)i * ld;  // row of this sample: the profile, then features
  float imax = 0.f;
  unsigned long long nseed = seed ^ 0x9E3779B97F4A7C15ull;
  for (int iw = 0; iw < nl; iw++) {
    float syn[4];
    if (P.nsub > 1)
      channel_point<float, false, true>(c, P, K, ones, iw, syn, nullptr);
    else
      channel_point<float, false, false>(c, P, K, ones, iw, syn, nullptr);
    // noise: 4 normals per wavelength from one Philox call
    uint32_t cc[4] = {(uint32_t)((unsigned long long)i & 0xffffffffu),
                      (uint32_t)((unsigned long long)i >> 32), (uint32_t)iw, 0x4E4F4953u};
    philox10(cc, (uint32_t)(nseed & 0xffffffffu), (uint32_t)(nseed >> 32));
#pragma unroll
    for (int s = 0; s < 4; s += 2) {
      const float u1 = ((float)cc[s] + 0.5f) * 2.3283064365386963e-10f;
      const float u2 = ((float)cc[s + 1] + 0.5f) * 2.3283064365386963e-10f;
      const float r = sqrtf(-2.f * logf(u1));
      float sn, cs;
      sincosf(6.2831853f * u2, &sn, &cs);
      syn[s] += pr.noise * r * cs;
      syn[s + 1] += pr.noise * r * sn;
    }
#pragma unroll
    for (int s = 0; s < 4; s++) xr[s * nl + iw] = syn[s];
    imax = fmaxf(imax, syn[0]);
  }
  const float inv = 1.f / imax;
  for (int k = 0; k < 4 * nl; k++) xr[k] = feature_value(k / nl, xr[k], inv);
  for (int k = 4 * nl; k < ld; k++) xr[k] = 0.f;
  float *t = Tgt + (size_t)i * kOut;
  t[0] = (float)par[0];
  t[1] = (float)cost;
  t[2] = (float)sin(2.0 * par[2]);
  t[3] = (float)cos(2.0 * par[2]);
  t[4] = (float)par[3];
  t[5] = (float)par[4];
  t[6] = (float)par[5];
  t[7] = (float)par[6];
  t[8] = (float)par[8];
  t[9] = (float)(par[7] * inv);
}

// per-column mean and 1/std over n rows of an FP32 [n][cols] array
__global__ void moments_kernel(const float *x, long long n, int cols, double *sum, double *sum2) {
  const int col = blockIdx.x;
  double s = 0, s2 = 0;
  for (long long r = threadIdx.x; r < n; r += blockDim.x) {
    const double v = x[(size_t)r * cols + col];
    s += v;
    s2 += v * v;
  }
  __shared__ double a[256], b[256];
  a[threadIdx.x] = s;
  b[threadIdx.x] = s2;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) {
      a[threadIdx.x] += a[threadIdx.x + w];
      b[threadIdx.x] += b[threadIdx.x + w];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    sum[col] = a[0];
    sum2[col] = b[0];
  }
}

// x <- (x - mean) * istd, written to BF16 X (and in place to the FP32 copy)
__global__ void standardise_kernel(float *xf, long long n, int cols, const float *mean,
                                   const float *istd, bf16 *X) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n * cols) return;
  const int c = (int)(i % cols);
  const float v = (xf[i] - mean[c]) * istd[c];
  xf[i] = v;
  if (X) X[i] = __float2bfloat16(v);
}

// features of map profiles (FP64 [n][4][nl]) for inference, standardised:
// one warp per profile, each lane on pairs of consecutive features, so that a
// warp reads 512 contiguous bytes (16-byte loads when the profiles are 16-byte
// aligned, VEC) and writes 128 contiguous bytes per step.  Every value is the
// same expression of the same inputs as in the training features.
template <bool VEC>
__global__ void __launch_bounds__(256)
    map_features_kernel(const double *__restrict__ prof, long long n, int nl, int ld,
                        const float *__restrict__ mean, const float *__restrict__ istd, bf16 *X,
                        float *imax_out) {
  const long long i = blockIdx.x * (long long)(blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (i >= n) return;  // the same for the whole warp
  const double *p = prof + (size_t)i * 4 * nl;
  double imax = 0.0;
  for (int iw = lane; iw < nl; iw += 32) imax = fmax(imax, p[iw]);
#pragma unroll
  for (int o = 16; o; o >>= 1) imax = fmax(imax, __shfl_xor_sync(0xffffffffu, imax, o));
  const float inv = imax > 0 ? (float)(1.0 / imax) : 0.f;
  __nv_bfloat162 *x = reinterpret_cast<__nv_bfloat162 *>(X + (size_t)i * ld);
  const int nf = 4 * nl;  // even, so a pair starting below nf ends below it
  for (int k = 2 * lane; k < ld; k += 64) {
    float v0 = 0.f, v1 = 0.f;  // the padding columns stay zero
    if (k < nf) {
      double q0, q1;
      if (VEC) {
        const double2 q = *reinterpret_cast<const double2 *>(p + k);
        q0 = q.x;
        q1 = q.y;
      } else {
        q0 = p[k];
        q1 = p[k + 1];
      }
      v0 = (feature_value(k / nl, (float)q0, inv) - mean[k]) * istd[k];
      v1 = (feature_value((k + 1) / nl, (float)q1, inv) - mean[k + 1]) * istd[k + 1];
    }
    x[k >> 1] = __floats2bfloat162_rn(v0, v1);
  }
  if (lane == 0) imax_out[i] = (float)imax;
}

// network outputs (standardised) -> the nine ME parameters [n][9] (FP64)
__global__ void decode_kernel(const float *Y, long long n, int ld, const float *tmean,
                              const float *tstd, const float *imax, double *par) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  float t[kOut];
#pragma unroll
  for (int k = 0; k < kOut; k++) t[k] = Y[(size_t)i * ld + k] * tstd[k] + tmean[k];
  double *p = par + (size_t)i * 9;
  p[0] = fmax((double)t[0], 0.0);
  p[1] = acos(fmin(fmax((double)t[1], -1.0), 1.0));
  double phi = 0.5 * atan2((double)t[2], (double)t[3]);
  if (phi < 0) phi += kPi;
  p[2] = phi;
  p[3] = t[4];
  p[4] = t[5];
  p[5] = t[6];
  p[6] = t[7];
  p[7] = (double)t[9] * imax[i];
  p[8] = t[8];
}

// ---------------------------------------------------------------------------
// loss and optimiser
// ---------------------------------------------------------------------------
// dY = 2 (Y - T) / (rows * kOut) for the batch rows idx[0..rows) (T standardised,
// [n][kOut]); Y and dY have row stride ld, the columns past kOut get zero.
// loss += mean squared error of the batch.
__global__ void mse_grad_kernel(const float *Yf, int ld, const float *Tstd, const long long *idx,
                                int rows, bf16 *dYb, double *loss) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  float sq = 0.f;
  if (i < rows * ld) {
    const int r = i / ld, k = i % ld;
    float gr = 0.f;
    if (k < kOut) {
      const float d = Yf[i] - Tstd[(size_t)idx[r] * kOut + k];
      gr = 2.f * d / (float)(rows * kOut);
      sq = d * d;
    }
    dYb[i] = __float2bfloat16(gr);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) sq += __shfl_xor_sync(0xffffffffu, sq, o);
  __shared__ float part[32];
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = sq;
  __syncthreads();
  if (threadIdx.x == 0) {
    float t = 0.f;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += part[w];
    atomicAdd(loss, (double)t / (double)(rows * kOut));
  }
}

// dA_prev = dH * gelu'(Z): BF16 out
__global__ void gelu_back_kernel(const float *dH, const float *Z, long long n, bf16 *dZb) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  dZb[i] = __float2bfloat16(dH[i] * gelu_grad(Z[i]));
}

// db[c] += sum over a chunk of rows of dZ[r][c] (db zeroed before); grid
// (cols / 32, row chunks), block (32, 8)
__global__ void bias_grad_kernel(const bf16 *dZ, int rows, int cols, int rows_per_chunk,
                                 float *db) {
  const int c = blockIdx.x * 32 + threadIdx.x;
  const int r0 = blockIdx.y * rows_per_chunk;
  const int r1 = min(rows, r0 + rows_per_chunk);
  float s = 0.f;
  if (c < cols)
    for (int r = r0 + threadIdx.y; r < r1; r += 8) s += __bfloat162float(dZ[(size_t)r * cols + c]);
  __shared__ float part[8][33];
  part[threadIdx.y][threadIdx.x] = s;
  __syncthreads();
  if (threadIdx.y == 0 && c < cols) {
    float t = 0.f;
#pragma unroll
    for (int k = 0; k < 8; k++) t += part[k][threadIdx.x];
    atomicAdd(db + c, t);
  }
}

// Adam (Kingma & Ba 2015) on FP32 master weights, refreshing the BF16 copy
// and its transpose.  w is [rows][cols].
__global__ void adam_kernel(float *w, float *m, float *v, const float *g, long long n, int cols,
                            float lr, float b1, float b2, float eps, float c1, float c2,
                            bf16 *wb, bf16 *wbt, int rows) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.f - b1) * gi;
  const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  const float wi = w[i] - lr * (mi * c1) / (sqrtf(vi * c2) + eps);
  w[i] = wi;
  if (wb) {
    wb[i] = __float2bfloat16(wi);
    const long long r = i / cols, c = i % cols;
    wbt[(size_t)c * rows + r] = __float2bfloat16(wi);
  }
}

// gather rows idx[] of X [n][cols] into Xb [rows][cols]
__global__ void gather_kernel(const bf16 *X, const long long *idx, int rows, int cols, bf16 *Xb) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= (long long)rows * cols) return;
  const int r = (int)(i / cols), c = (int)(i % cols);
  Xb[i] = X[(size_t)idx[r] * cols + c];
}

// a random permutation of [0, n) per epoch: Feistel network on the index
// space (cycle-walking), keyed per epoch
__device__ __forceinline__ unsigned long long feistel(unsigned long long x, int bits, uint32_t k0,
                                                      uint32_t k1) {
  const int half = (bits + 1) / 2;
  const unsigned long long mask = (1ull << half) - 1;
  unsigned long long l = x >> half, r = x & mask;
  for (int round = 0; round < 4; round++) {
    uint32_t c[4] = {(uint32_t)r, (uint32_t)round, 0x46454953u, 0};
    philox10(c, k0, k1);
    const unsigned long long f = c[0] & mask;
    const unsigned long long nl = r, nr = (l ^ f) & mask;
    l = nl;
    r = nr;
  }
  return (l << half) | r;
}

__global__ void permute_kernel(long long n, int bits, uint32_t k0, uint32_t k1, long long *perm) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  unsigned long long x = (unsigned long long)i;
  do {
    x = feistel(x, bits, k0, k1);
  } while (x >= (unsigned long long)n);
  perm[i] = (long long)x;
}

}  // namespace mlp
}  // namespace me

// ---------------------------------------------------------------------------
// Host side: model, training, inference, files (C ABI in include/me_b200.h).
// ---------------------------------------------------------------------------
namespace {

using namespace me::mlp;

constexpr int kOutPad = 32;      // output rows of the last layer (10 used, zero weights past)

struct DBuf {
  void *p = nullptr;
  size_t n = 0;
  DBuf() = default;
  DBuf(const DBuf &) = delete;
  DBuf &operator=(const DBuf &) = delete;
  ~DBuf() { release(); }
  cudaError_t ensure(size_t bytes) {
    if (bytes <= n) return cudaSuccess;
    release();
    cudaError_t e = cudaMalloc(&p, bytes);
    if (e == cudaSuccess)
      n = bytes;
    else
      p = nullptr;
    return e;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  template <class T>
  T *as() const {
    return static_cast<T *>(p);
  }
};

int fail(int code, const std::string &m) { return me::record_error(code, m.c_str()); }

#define MCK(call)                                                               \
  do {                                                                          \
    cudaError_t e_ = (call);                                                    \
    if (e_ != cudaSuccess)                                                      \
      return fail(ME_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

inline unsigned nblk(long long n, int b = 256) { return (unsigned)((n + b - 1) / b); }

}  // namespace

struct me_mlp {
  int device = 0;
  int nl = 0, nin = 0, nip = 0;  // grid size, features, padded input width
  int din[kLayers], dout[kLayers];
  // per layer: FP32 master W [dout][din] and b, BF16 W and W^T, Adam moments, gradients
  DBuf w[kLayers], b[kLayers], wb[kLayers], wbt[kLayers], mw[kLayers], vw[kLayers], mb[kLayers],
      vb[kLayers], gw[kLayers], gb[kLayers];
  DBuf fmean, fistd, tmean, tstd;  // feature and target standardisation (device)
  std::vector<float> h_fmean, h_fistd, h_tmean, h_tstd;
  long long adam_t = 0;
  // batch work buffers
  int cap = 0;
  DBuf xb, xbt, z[kLayers], a[kLayers], at[kLayers], yf, dyb, dybt, dh, dz, dzt, loss;
  DBuf imax;
  // GEMM kernel choice and the tcgen05 kernel's error flag (device int)
  GemmPath gemm_path = GemmPath::tcgen05;
  DBuf gerr;
  long long gemm_launches[2] = {0, 0};
  TileMapCache maps;
};

namespace {

size_t wcount(const me_mlp *m, int l) { return (size_t)m->dout[l] * m->din[l]; }

GemmCtx ctx(me_mlp *m) {
  GemmCtx g;
  g.path = m->gemm_path;
  g.err = m->gerr.as<int>();
  g.launches = m->gemm_launches;
  g.maps = &m->maps;
  return g;
}

// reads and clears the tcgen05 GEMM's error flag (synchronises the device)
int gemm_status(me_mlp *m) {
  if (!m->gerr.p) return ME_OK;
  int e = 0;
  MCK(cudaMemcpy(&e, m->gerr.p, sizeof(int), cudaMemcpyDeviceToHost));
  if (!e) return ME_OK;
  MCK(cudaMemset(m->gerr.p, 0, sizeof(int)));
  static const char *what[] = {"", "operand load", "stage release", "accumulator"};
  return fail(ME_ERR_CUDA, std::string("tensor-core GEMM: wait for the ") +
                               what[e >= 1 && e <= 3 ? e : 0] + " timed out");
}

long long param_count(const me_mlp *m) {
  long long n = 0;
  for (int l = 0; l < kLayers; l++) n += (long long)wcount(m, l) + m->dout[l];
  return n;
}

int ensure_batch(me_mlp *m, int B) {
  if (B <= m->cap) return ME_OK;
  const size_t r = (size_t)B;
  MCK(m->xb.ensure(r * m->nip * 2));
  MCK(m->xbt.ensure(r * m->nip * 2));
  for (int l = 0; l < kLayers; l++) {
    MCK(m->z[l].ensure(r * m->dout[l] * 4));
    MCK(m->a[l].ensure(r * m->dout[l] * 2));
    MCK(m->at[l].ensure(r * m->dout[l] * 2));
  }
  MCK(m->yf.ensure(r * kOutPad * 4));
  MCK(m->dyb.ensure(r * kOutPad * 2));
  MCK(m->dybt.ensure(r * kOutPad * 2));
  MCK(m->dh.ensure(r * kHidden * 4));
  MCK(m->dz.ensure(r * kHidden * 2));
  MCK(m->dzt.ensure(r * kHidden * 2));
  MCK(m->loss.ensure(sizeof(double)));
  MCK(m->imax.ensure(r * 4));
  m->cap = B;
  return ME_OK;
}

__global__ void init_weights_kernel(float *w, long long n, int din, int din_used, int dout_used,
                                    unsigned long long seed, float scale) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int c = (int)(i % din);
  const long long r = i / din;
  uint32_t cc[4] = {(uint32_t)i, (uint32_t)(i >> 32), 0x494E4954u, 0};
  me::philox10(cc, (uint32_t)seed, (uint32_t)(seed >> 32));
  const float u1 = ((float)cc[0] + 0.5f) * 2.3283064365386963e-10f;
  const float u2 = ((float)cc[1] + 0.5f) * 2.3283064365386963e-10f;
  const float g = sqrtf(-2.f * logf(u1)) * cosf(6.2831853f * u2);
  w[i] = (c < din_used && r < dout_used) ? scale * g : 0.f;
}

// BF16 copy of W [rows][cols] and of its transpose
__global__ void to_bf16_kernel(const float *w, long long n, int cols, int rows, bf16 *wb,
                               bf16 *wbt) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const bf16 v = __float2bfloat16(w[i]);
  wb[i] = v;
  const long long r = i / cols, c = i % cols;
  wbt[(size_t)c * rows + r] = v;
}

__global__ void f32_to_bf16_kernel(const float *x, long long n, bf16 *y) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i < n) y[i] = __float2bfloat16(x[i]);
}

__global__ void iota_kernel(long long *idx, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) idx[i] = i;
}

int refresh_bf16(me_mlp *m, cudaStream_t st) {
  for (int l = 0; l < kLayers; l++) {
    const long long nw = (long long)wcount(m, l);
    to_bf16_kernel<<<nblk(nw), 256, 0, st>>>(m->w[l].as<float>(), nw, m->din[l], m->dout[l],
                                              m->wb[l].as<bf16>(), m->wbt[l].as<bf16>());
  }
  MCK(cudaGetLastError());
  return ME_OK;
}

int alloc_model(me_mlp *m, int nl) {
  m->nl = nl;
  m->nin = 4 * nl;
  m->nip = (m->nin + 31) / 32 * 32;
  MCK(m->gerr.ensure(sizeof(int)));
  MCK(cudaMemset(m->gerr.p, 0, sizeof(int)));
  const int din[kLayers] = {m->nip, kHidden, kHidden, kHidden};
  const int dout[kLayers] = {kHidden, kHidden, kHidden, kOutPad};
  for (int l = 0; l < kLayers; l++) {
    m->din[l] = din[l];
    m->dout[l] = dout[l];
    const size_t nw = wcount(m, l);
    for (DBuf *d : {&m->w[l], &m->mw[l], &m->vw[l], &m->gw[l]}) MCK(d->ensure(nw * 4));
    for (DBuf *d : {&m->wb[l], &m->wbt[l]}) MCK(d->ensure(nw * 2));
    for (DBuf *d : {&m->b[l], &m->mb[l], &m->vb[l], &m->gb[l]}) MCK(d->ensure(dout[l] * 4));
    MCK(cudaMemset(m->mw[l].p, 0, nw * 4));
    MCK(cudaMemset(m->vw[l].p, 0, nw * 4));
    MCK(cudaMemset(m->b[l].p, 0, dout[l] * 4));
    MCK(cudaMemset(m->mb[l].p, 0, dout[l] * 4));
    MCK(cudaMemset(m->vb[l].p, 0, dout[l] * 4));
  }
  MCK(m->fmean.ensure(m->nip * 4));
  MCK(m->fistd.ensure(m->nip * 4));
  MCK(m->tmean.ensure(kOut * 4));
  MCK(m->tstd.ensure(kOut * 4));
  m->h_fmean.assign(m->nip, 0.f);
  m->h_fistd.assign(m->nip, 1.f);
  m->h_tmean.assign(kOut, 0.f);
  m->h_tstd.assign(kOut, 1.f);
  return ME_OK;
}

int upload_standardisation(me_mlp *m) {
  MCK(cudaMemcpy(m->fmean.p, m->h_fmean.data(), m->nip * 4, cudaMemcpyHostToDevice));
  MCK(cudaMemcpy(m->fistd.p, m->h_fistd.data(), m->nip * 4, cudaMemcpyHostToDevice));
  MCK(cudaMemcpy(m->tmean.p, m->h_tmean.data(), kOut * 4, cudaMemcpyHostToDevice));
  MCK(cudaMemcpy(m->tstd.p, m->h_tstd.data(), kOut * 4, cudaMemcpyHostToDevice));
  return ME_OK;
}

// He initialisation (sqrt(2 / fan_in)) for the GELU layers, sqrt(1 / fan_in)
// for the output layer; zero biases; zero weights on the padding
int init_model(me_mlp *m, unsigned long long seed) {
  for (int l = 0; l < kLayers; l++) {
    const long long nw = (long long)wcount(m, l);
    const int din_used = l == 0 ? m->nin : m->din[l];
    const int dout_used = l == kLayers - 1 ? kOut : m->dout[l];
    const float scale = (l == kLayers - 1 ? 1.f : 1.41421356f) / sqrtf((float)din_used);
    init_weights_kernel<<<nblk(nw), 256>>>(m->w[l].as<float>(), nw, m->din[l], din_used,
                                           dout_used, seed * 131 + l, scale);
  }
  MCK(cudaGetLastError());
  return refresh_bf16(m, nullptr);
}

// forward pass of B rows of m->xb -> m->yf [B][32] FP32 (pre-activations
// kept in m->z when `keep`)
void forward(me_mlp *m, int B, bool keep, cudaStream_t st) {
  const bf16 *in = m->xb.as<bf16>();
  for (int l = 0; l < kLayers; l++) {
    const bool last = l == kLayers - 1;
    gemm(ctx(m), in, m->wb[l].as<bf16>(), B, m->dout[l], m->din[l], m->b[l].as<float>(),
         (!last && keep) ? m->z[l].as<float>() : nullptr, last ? 0 : 1,
         last ? nullptr : m->a[l].as<bf16>(), last ? m->yf.as<float>() : nullptr, st);
    in = m->a[l].as<bf16>();
  }
}

// backward from dY (m->dyb, BF16 [B][32]) into m->gw / m->gb
void backward(me_mlp *m, int B, cudaStream_t st) {
  const bf16 *dcur = m->dyb.as<bf16>();  // dZ of layer l, BF16 [B][dout]
  for (int l = kLayers - 1; l >= 0; l--) {
    const int dout = m->dout[l], din = m->din[l];
    // dW [dout][din] = dZ^T A_prev: GEMM of dZ^T [dout][B] and A_prev^T [din][B]
    bf16 *dzt = l == kLayers - 1 ? m->dybt.as<bf16>() : m->dzt.as<bf16>();
    transpose(dcur, B, dout, dzt, st);
    const bf16 *aprev = l == 0 ? m->xb.as<bf16>() : m->a[l - 1].as<bf16>();
    bf16 *aprevt = l == 0 ? m->xbt.as<bf16>() : m->at[l - 1].as<bf16>();
    transpose(aprev, B, din, aprevt, st);
    int split = 1;
    while (split < 16 && B % (2 * split * kTK) == 0 && B / (2 * split) >= 256) split *= 2;
    cudaMemsetAsync(m->gw[l].p, 0, wcount(m, l) * 4, st);
    gemm(ctx(m), dzt, aprevt, dout, din, B, nullptr, nullptr, 0, nullptr, m->gw[l].as<float>(), st, split);
    cudaMemsetAsync(m->gb[l].p, 0, dout * 4, st);
    const int chunk = 256;
    bias_grad_kernel<<<dim3((dout + 31) / 32, (B + chunk - 1) / chunk), dim3(32, 8), 0, st>>>(
        dcur, B, dout, chunk, m->gb[l].as<float>());
    if (l == 0) break;
    // dA_prev [B][din] = dZ W: GEMM of dZ [B][dout] and W^T [din][dout]
    gemm(ctx(m), dcur, m->wbt[l].as<bf16>(), B, din, dout, nullptr, nullptr, 0, nullptr,
         m->dh.as<float>(), st);
    gelu_back_kernel<<<nblk((long long)B * din), 256, 0, st>>>(
        m->dh.as<float>(), m->z[l - 1].as<float>(), (long long)B * din, m->dz.as<bf16>());
    dcur = m->dz.as<bf16>();
  }
}

void adam_step(me_mlp *m, float lr, cudaStream_t st) {
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  m->adam_t++;
  const float c1 = (float)(1.0 / (1.0 - pow((double)b1, (double)m->adam_t)));
  const float c2 = (float)(1.0 / (1.0 - pow((double)b2, (double)m->adam_t)));
  for (int l = 0; l < kLayers; l++) {
    const long long nw = (long long)wcount(m, l);
    adam_kernel<<<nblk(nw), 256, 0, st>>>(m->w[l].as<float>(), m->mw[l].as<float>(),
                                           m->vw[l].as<float>(), m->gw[l].as<float>(), nw,
                                           m->din[l], lr, b1, b2, eps, c1, c2,
                                           m->wb[l].as<bf16>(), m->wbt[l].as<bf16>(), m->dout[l]);
    adam_kernel<<<nblk(m->dout[l]), 256, 0, st>>>(m->b[l].as<float>(), m->mb[l].as<float>(),
                                                   m->vb[l].as<float>(), m->gb[l].as<float>(),
                                                   m->dout[l], m->dout[l], lr, b1, b2, eps, c1,
                                                   c2, nullptr, nullptr, 1);
  }
}

// loss and gradients of the rows idx[0..B) of the standardised targets T
// (the batch features already in m->xb); loss accumulated into m->loss
void loss_grad(me_mlp *m, int B, const float *T, const long long *idx, cudaStream_t st) {
  forward(m, B, true, st);
  mse_grad_kernel<<<nblk((long long)B * kOutPad), 256, 0, st>>>(
      m->yf.as<float>(), kOutPad, T, idx, B, m->dyb.as<bf16>(), m->loss.as<double>());
  backward(m, B, st);
}

void prior_from(const me_mlp_train_params *tp, Prior &pr) {
  pr.b_lo = (float)tp->b_range[0];
  pr.b_hi = (float)tp->b_range[1];
  pr.cost_lo = (float)tp->cos_theta_range[0];
  pr.cost_hi = (float)tp->cos_theta_range[1];
  pr.phi_lo = (float)tp->phi_range[0];
  pr.phi_hi = (float)tp->phi_range[1];
  pr.v_sigma = (float)tp->v_sigma;
  pr.w_lo = (float)tp->doppler_range[0];
  pr.w_hi = (float)tp->doppler_range[1];
  pr.a_lo = (float)tp->damping_range[0];
  pr.a_hi = (float)tp->damping_range[1];
  pr.eta_lo = (float)tp->eta_range[0];
  pr.eta_hi = (float)tp->eta_range[1];
  pr.s = (float)tp->s;
  pr.beta_lo = (float)tp->beta_range[0];
  pr.beta_hi = (float)tp->beta_range[1];
  pr.noise = (float)tp->noise;
  pr.mix = (float)tp->mix_weight;
  pr.mb_lo = (float)tp->mix_b_range[0];
  pr.mb_hi = (float)tp->mix_b_range[1];
  pr.meta_lo = (float)tp->mix_eta_range[0];
  pr.meta_hi = (float)tp->mix_eta_range[1];
}

}  // namespace

namespace me {
// plan constants with device grid pointers, and the plan's device (me_api.cu)
int plan_devplan(const me_plan *p, DevPlan *out, int *device);

int mlp_gemm_status(me_mlp *m) { return gemm_status(m); }
}  // namespace me

extern "C" int me_mlp_train_params_default(me_mlp_train_params *tp) {
  if (!tp) return fail(ME_ERR_ARG, "null argument");
  memset(tp, 0, sizeof(*tp));
  tp->samples = 1LL << 22;
  tp->epochs = 16;
  tp->batch = 4096;
  tp->lr = 1e-3;
  tp->seed = 20240607ULL;
  tp->b_range[0] = 0;
  tp->b_range[1] = 3000;
  tp->cos_theta_range[0] = -1;
  tp->cos_theta_range[1] = 1;
  tp->phi_range[0] = 0;
  tp->phi_range[1] = me::kPi;
  tp->v_sigma = 1.5;
  tp->doppler_range[0] = 150;
  tp->doppler_range[1] = 350;
  tp->damping_range[0] = 0.1;
  tp->damping_range[1] = 0.8;
  tp->eta_range[0] = 2;
  tp->eta_range[1] = 30;
  tp->s = 1.0;
  tp->beta_range[0] = 0.1;
  tp->beta_range[1] = 0.6;
  tp->noise = 1e-3;
  return ME_OK;
}

extern "C" void me_mlp_destroy(me_mlp *m) {
  if (!m) return;
  int cur = 0;
  cudaGetDevice(&cur);
  cudaSetDevice(m->device);
  delete m;
  cudaSetDevice(cur);
}

extern "C" int me_mlp_train(me_plan *plan, const me_mlp_train_params *tp, me_mlp **out,
                            double *final_loss) {
  if (!plan || !tp || !out) return fail(ME_ERR_ARG, "null argument");
  *out = nullptr;
  if (tp->batch < 256 || tp->batch % 256 || tp->samples < tp->batch || tp->epochs < 0 ||
      tp->samples > (1LL << 31) || !(tp->lr > 0))
    return fail(ME_ERR_ARG,
                "batch a multiple of 256, batch <= samples <= 2^31, epochs >= 0, lr > 0");
  if (tp->gemm != ME_GEMM_TCGEN05 && tp->gemm != ME_GEMM_MMA_SYNC)
    return fail(ME_ERR_ARG, "gemm must be ME_GEMM_TCGEN05 or ME_GEMM_MMA_SYNC");
  if (!(tp->mix_weight >= 0.0 && tp->mix_weight <= 1.0))
    return fail(ME_ERR_ARG, "mix_weight must lie in [0, 1]");
  me::DevPlan P;
  int device = 0;
  int rc = me::plan_devplan(plan, &P, &device);
  if (rc) return rc;
  MCK(cudaSetDevice(device));
  me_mlp *m = new me_mlp();
  m->device = device;
  m->gemm_path = tp->gemm == ME_GEMM_TCGEN05 ? GemmPath::tcgen05 : GemmPath::mma_sync;
  rc = alloc_model(m, P.nl);
  if (!rc) rc = init_model(m, tp->seed);
  if (rc) {
    delete m;
    return rc;
  }
  std::unique_ptr<me_mlp, void (*)(me_mlp *)> guard(m, me_mlp_destroy);
  cudaStream_t st = nullptr;
  const long long n = tp->samples;
  const int nip = m->nip;
  // ---- training set: FP32 synthesis on the plan's grid, then standardisation ----
  DBuf Xf, X, T;
  MCK(Xf.ensure((size_t)n * nip * 4));
  MCK(T.ensure((size_t)n * kOut * 4));
  Prior pr;
  prior_from(tp, pr);
  synth_train_kernel<<<nblk(n, 128), 128, 0, st>>>(P, pr, tp->seed, n, nip, Xf.as<float>(),
                                                    T.as<float>());
  MCK(cudaGetLastError());
  {
    DBuf s1, s2;
    MCK(s1.ensure(nip * 8));
    MCK(s2.ensure(nip * 8));
    std::vector<double> a(nip), b(nip);
    moments_kernel<<<nip, 256, 0, st>>>(Xf.as<float>(), n, nip, s1.as<double>(), s2.as<double>());
    MCK(cudaMemcpy(a.data(), s1.p, nip * 8, cudaMemcpyDeviceToHost));
    MCK(cudaMemcpy(b.data(), s2.p, nip * 8, cudaMemcpyDeviceToHost));
    for (int c = 0; c < nip; c++) {
      const double mu = a[c] / n, var = b[c] / n - mu * mu;
      m->h_fmean[c] = c < m->nin ? (float)mu : 0.f;
      m->h_fistd[c] = (c < m->nin && var > 1e-20) ? (float)(1.0 / sqrt(var)) : 0.f;
    }
    moments_kernel<<<kOut, 256, 0, st>>>(T.as<float>(), n, kOut, s1.as<double>(), s2.as<double>());
    MCK(cudaMemcpy(a.data(), s1.p, kOut * 8, cudaMemcpyDeviceToHost));
    MCK(cudaMemcpy(b.data(), s2.p, kOut * 8, cudaMemcpyDeviceToHost));
    std::vector<float> tinv(kOut);
    for (int c = 0; c < kOut; c++) {
      const double mu = a[c] / n, var = b[c] / n - mu * mu;
      m->h_tmean[c] = (float)mu;
      m->h_tstd[c] = var > 1e-20 ? (float)sqrt(var) : 1.f;
      tinv[c] = 1.f / m->h_tstd[c];
    }
    rc = upload_standardisation(m);
    if (rc) return rc;
    DBuf tiv;
    MCK(tiv.ensure(kOut * 4));
    MCK(cudaMemcpy(tiv.p, tinv.data(), kOut * 4, cudaMemcpyHostToDevice));
    MCK(X.ensure((size_t)n * nip * 2));
    standardise_kernel<<<nblk((long long)n * nip), 256, 0, st>>>(
        Xf.as<float>(), n, nip, m->fmean.as<float>(), m->fistd.as<float>(), X.as<bf16>());
    standardise_kernel<<<nblk((long long)n * kOut), 256, 0, st>>>(
        T.as<float>(), n, kOut, m->tmean.as<float>(), tiv.as<float>(), nullptr);
    MCK(cudaStreamSynchronize(st));
  }
  Xf.release();
  // ---- Adam on shuffled batches ----
  const int B = tp->batch;
  rc = ensure_batch(m, B);
  if (rc) return rc;
  DBuf perm;
  MCK(perm.ensure((size_t)n * sizeof(long long)));
  int bits = 1;
  while ((1LL << bits) < n) bits++;
  const long long steps = n / B;
  double last = 0.0;
  for (int ep = 0; ep < tp->epochs; ep++) {
    const unsigned long long k = tp->seed * 0x9E3779B97F4A7C15ull + 0x51ull * (ep + 1);
    permute_kernel<<<nblk(n), 256, 0, st>>>(n, bits, (uint32_t)k, (uint32_t)(k >> 32),
                                            perm.as<long long>());
    MCK(cudaMemsetAsync(m->loss.p, 0, sizeof(double), st));
    for (long long s = 0; s < steps; s++) {
      const long long *idx = perm.as<long long>() + s * B;
      gather_kernel<<<nblk((long long)B * nip), 256, 0, st>>>(X.as<bf16>(), idx, B, nip,
                                                              m->xb.as<bf16>());
      loss_grad(m, B, T.as<float>(), idx, st);
      adam_step(m, (float)tp->lr, st);
    }
    MCK(cudaGetLastError());
    double l = 0;
    MCK(cudaMemcpyAsync(&l, m->loss.p, sizeof(double), cudaMemcpyDeviceToHost, st));
    MCK(cudaStreamSynchronize(st));
    rc = gemm_status(m);
    if (rc) return rc;
    last = l / (double)steps;
  }
  if (final_loss) *final_loss = last;
  *out = guard.release();
  return ME_OK;
}

extern "C" int me_mlp_predict_device(me_mlp *m, const double *d_prof, long npix, double *d_par,
                                     void *stream) {
  if (!m || (npix > 0 && (!d_prof || !d_par)) || npix < 0)
    return fail(ME_ERR_ARG, "null argument");
  if (npix == 0) return ME_OK;
  MCK(cudaSetDevice(m->device));
  cudaStream_t st = (cudaStream_t)stream;
  const int chunk = (int)(npix < me::kMlpPredChunk ? (npix + 255) / 256 * 256 : me::kMlpPredChunk);
  int rc = ensure_batch(m, chunk);
  if (rc) return rc;
  for (long long r0 = 0; r0 < npix; r0 += chunk) {
    const int rows = (int)((npix - r0) < chunk ? (npix - r0) : chunk);
    // a chunk starts 32 nl r0 bytes in, so its alignment is the base's
    if ((reinterpret_cast<uintptr_t>(d_prof) & 15) == 0)
      map_features_kernel<true><<<nblk(rows, 8), 256, 0, st>>>(
          d_prof + (size_t)r0 * 4 * m->nl, rows, m->nl, m->nip, m->fmean.as<float>(),
          m->fistd.as<float>(), m->xb.as<bf16>(), m->imax.as<float>());
    else
      map_features_kernel<false><<<nblk(rows, 8), 256, 0, st>>>(
          d_prof + (size_t)r0 * 4 * m->nl, rows, m->nl, m->nip, m->fmean.as<float>(),
          m->fistd.as<float>(), m->xb.as<bf16>(), m->imax.as<float>());
    forward(m, rows, false, st);
    decode_kernel<<<nblk(rows, 128), 128, 0, st>>>(m->yf.as<float>(), rows, kOutPad,
                                                   m->tmean.as<float>(), m->tstd.as<float>(),
                                                   m->imax.as<float>(), d_par + (size_t)r0 * 9);
  }
  MCK(cudaGetLastError());
  if (!stream) {
    MCK(cudaStreamSynchronize(st));
    return gemm_status(m);
  }
  return ME_OK;
}

extern "C" int me_mlp_predict(me_mlp *m, const double *prof, long npix, double *par) {
  if (!m || (npix > 0 && (!prof || !par)) || npix < 0) return fail(ME_ERR_ARG, "null argument");
  if (npix == 0) return ME_OK;
  MCK(cudaSetDevice(m->device));
  DBuf dp, dq;
  MCK(dp.ensure((size_t)npix * 4 * m->nl * 8));
  MCK(dq.ensure((size_t)npix * 9 * 8));
  MCK(cudaMemcpy(dp.p, prof, (size_t)npix * 4 * m->nl * 8, cudaMemcpyHostToDevice));
  int rc = me_mlp_predict_device(m, dp.as<double>(), npix, dq.as<double>(), nullptr);
  if (rc) return rc;
  MCK(cudaMemcpy(par, dq.p, (size_t)npix * 9 * 8, cudaMemcpyDeviceToHost));
  return ME_OK;
}

extern "C" int me_mlp_shape(const me_mlp *m, int *nl, int *nin_pad, long long *nparams) {
  if (!m) return fail(ME_ERR_ARG, "null argument");
  if (nl) *nl = m->nl;
  if (nin_pad) *nin_pad = m->nip;
  if (nparams) *nparams = param_count(m);
  return ME_OK;
}

namespace {
// copies the parameters (or gradients) between a flat host array and the device
int copy_flat(const me_mlp *m, bool grads, float *host, bool to_host) {
  size_t off = 0;
  for (int l = 0; l < kLayers; l++) {
    const DBuf &W = grads ? m->gw[l] : m->w[l];
    const DBuf &Bv = grads ? m->gb[l] : m->b[l];
    const size_t nw = wcount(m, l);
    if (to_host) {
      MCK(cudaMemcpy(host + off, W.p, nw * 4, cudaMemcpyDeviceToHost));
      MCK(cudaMemcpy(host + off + nw, Bv.p, m->dout[l] * 4, cudaMemcpyDeviceToHost));
    } else {
      MCK(cudaMemcpy(W.p, host + off, nw * 4, cudaMemcpyHostToDevice));
      MCK(cudaMemcpy(Bv.p, host + off + nw, m->dout[l] * 4, cudaMemcpyHostToDevice));
    }
    off += nw + m->dout[l];
  }
  return ME_OK;
}
}  // namespace

extern "C" int me_mlp_get_params(const me_mlp *m, float *params) {
  if (!m || !params) return fail(ME_ERR_ARG, "null argument");
  MCK(cudaSetDevice(m->device));
  return copy_flat(m, false, params, true);
}

extern "C" int me_mlp_set_params(me_mlp *m, const float *params) {
  if (!m || !params) return fail(ME_ERR_ARG, "null argument");
  MCK(cudaSetDevice(m->device));
  int rc = copy_flat(m, false, const_cast<float *>(params), false);
  if (rc) return rc;
  rc = refresh_bf16(m, nullptr);
  if (rc) return rc;
  MCK(cudaDeviceSynchronize());
  return ME_OK;
}

extern "C" int me_mlp_loss_grad(me_mlp *m, const float *x, const float *t, int rows, double *loss,
                                float *grad) {
  if (!m || !x || !t || !loss || !grad) return fail(ME_ERR_ARG, "null argument");
  if (rows < 256 || rows % 256) return fail(ME_ERR_ARG, "rows must be a positive multiple of 256");
  MCK(cudaSetDevice(m->device));
  int rc = ensure_batch(m, rows);
  if (rc) return rc;
  DBuf xf, tf, idx;
  MCK(xf.ensure((size_t)rows * m->nip * 4));
  MCK(tf.ensure((size_t)rows * kOut * 4));
  MCK(idx.ensure((size_t)rows * 8));
  MCK(cudaMemcpy(xf.p, x, (size_t)rows * m->nip * 4, cudaMemcpyHostToDevice));
  MCK(cudaMemcpy(tf.p, t, (size_t)rows * kOut * 4, cudaMemcpyHostToDevice));
  f32_to_bf16_kernel<<<nblk((long long)rows * m->nip), 256>>>(xf.as<float>(),
                                                               (long long)rows * m->nip,
                                                               m->xb.as<bf16>());
  iota_kernel<<<nblk(rows), 256>>>(idx.as<long long>(), rows);
  MCK(cudaMemset(m->loss.p, 0, sizeof(double)));
  loss_grad(m, rows, tf.as<float>(), idx.as<long long>(), nullptr);
  MCK(cudaGetLastError());
  MCK(cudaDeviceSynchronize());
  rc = gemm_status(m);
  if (rc) return rc;
  MCK(cudaMemcpy(loss, m->loss.p, sizeof(double), cudaMemcpyDeviceToHost));
  return copy_flat(m, true, grad, true);
}

extern "C" int me_mlp_set_gemm(me_mlp *m, int path) {
  if (!m) return fail(ME_ERR_ARG, "null argument");
  if (path != ME_GEMM_TCGEN05 && path != ME_GEMM_MMA_SYNC)
    return fail(ME_ERR_ARG, "path must be ME_GEMM_TCGEN05 or ME_GEMM_MMA_SYNC");
  m->gemm_path = path == ME_GEMM_TCGEN05 ? GemmPath::tcgen05 : GemmPath::mma_sync;
  return ME_OK;
}

extern "C" int me_mlp_gemm_launches(const me_mlp *m, long long *tcgen05, long long *mma_sync) {
  if (!m) return fail(ME_ERR_ARG, "null argument");
  if (tcgen05) *tcgen05 = m->gemm_launches[(int)GemmPath::tcgen05];
  if (mma_sync) *mma_sync = m->gemm_launches[(int)GemmPath::mma_sync];
  return ME_OK;
}

extern "C" int me_gemm_bf16(int device, int path, const uint16_t *a, const uint16_t *bt, int m,
                            int n, int r, int split, const float *bias, int gelu, float *z,
                            float *y, int *ran) {
  if (!a || !bt || !y) return fail(ME_ERR_ARG, "null argument");
  if (path != ME_GEMM_TCGEN05 && path != ME_GEMM_MMA_SYNC)
    return fail(ME_ERR_ARG, "path must be ME_GEMM_TCGEN05 or ME_GEMM_MMA_SYNC");
  if (m < 1 || n < 1 || r < 32 || split < 1 || r % (32 * split))
    return fail(ME_ERR_ARG, "need m, n >= 1, r >= 32 and r % (32 split) == 0");
  if (split > 1 && (bias || gelu || z))
    return fail(ME_ERR_ARG, "a split reduction has no bias, GELU or z");
  int nd = 0;
  if (cudaGetDeviceCount(&nd) != cudaSuccess || nd == 0)
    return fail(ME_ERR_NODEVICE, "no CUDA device");
  if (device < 0 || device >= nd) return fail(ME_ERR_ARG, "device out of range");
  MCK(cudaSetDevice(device));
  DBuf da, db, dbias, dz, dy, derr;
  const size_t mr = (size_t)m * r, nr = (size_t)n * r, mn = (size_t)m * n;
  MCK(da.ensure(mr * 2));
  MCK(db.ensure(nr * 2));
  MCK(dy.ensure(mn * 4));
  MCK(derr.ensure(sizeof(int)));
  MCK(cudaMemcpy(da.p, a, mr * 2, cudaMemcpyHostToDevice));
  MCK(cudaMemcpy(db.p, bt, nr * 2, cudaMemcpyHostToDevice));
  MCK(cudaMemset(dy.p, 0, mn * 4));
  MCK(cudaMemset(derr.p, 0, sizeof(int)));
  if (bias) {
    MCK(dbias.ensure((size_t)n * 4));
    MCK(cudaMemcpy(dbias.p, bias, (size_t)n * 4, cudaMemcpyHostToDevice));
  }
  if (z) MCK(dz.ensure(mn * 4));
  GemmCtx g;
  g.path = path == ME_GEMM_TCGEN05 ? GemmPath::tcgen05 : GemmPath::mma_sync;
  g.err = derr.as<int>();
  const GemmPath used = gemm(g, da.as<bf16>(), db.as<bf16>(), m, n, r, dbias.as<float>(),
                             dz.as<float>(), gelu, nullptr, dy.as<float>(), nullptr, split);
  if (ran) *ran = used == GemmPath::tcgen05 ? ME_GEMM_TCGEN05 : ME_GEMM_MMA_SYNC;
  MCK(cudaGetLastError());
  MCK(cudaDeviceSynchronize());
  int e = 0;
  MCK(cudaMemcpy(&e, derr.p, sizeof(int), cudaMemcpyDeviceToHost));
  if (e) return fail(ME_ERR_CUDA, "tensor-core GEMM: a bounded wait timed out");
  MCK(cudaMemcpy(y, dy.p, mn * 4, cudaMemcpyDeviceToHost));
  if (z) MCK(cudaMemcpy(z, dz.p, mn * 4, cudaMemcpyDeviceToHost));
  return ME_OK;
}

// File: "MEMLP001", int32 nl, int32 nin_pad, float fmean[nin_pad],
// fistd[nin_pad], tmean[10], tstd[10], then the parameters as
// me_mlp_get_params lays them out (little-endian).
static const char kMagic[8] = {'M', 'E', 'M', 'L', 'P', '0', '0', '1'};

extern "C" int me_mlp_save(const me_mlp *m, const char *path) {
  if (!m || !path) return fail(ME_ERR_ARG, "null argument");
  MCK(cudaSetDevice(m->device));
  std::vector<float> prm((size_t)param_count(m));
  int rc = copy_flat(m, false, prm.data(), true);
  if (rc) return rc;
  FILE *f = fopen(path, "wb");
  if (!f) return fail(ME_ERR_IO, std::string("cannot write ") + path);
  const int32_t hdr[2] = {m->nl, m->nip};
  bool ok = fwrite(kMagic, 1, 8, f) == 8 && fwrite(hdr, 4, 2, f) == 2 &&
            fwrite(m->h_fmean.data(), 4, m->nip, f) == (size_t)m->nip &&
            fwrite(m->h_fistd.data(), 4, m->nip, f) == (size_t)m->nip &&
            fwrite(m->h_tmean.data(), 4, kOut, f) == (size_t)kOut &&
            fwrite(m->h_tstd.data(), 4, kOut, f) == (size_t)kOut &&
            fwrite(prm.data(), 4, prm.size(), f) == prm.size();
  ok = (fclose(f) == 0) && ok;
  if (!ok) return fail(ME_ERR_IO, std::string("short write to ") + path);
  return ME_OK;
}

extern "C" int me_mlp_load(const char *path, int device, me_mlp **out) {
  if (!path || !out) return fail(ME_ERR_ARG, "null argument");
  *out = nullptr;
  FILE *f = fopen(path, "rb");
  if (!f) return fail(ME_ERR_IO, std::string("cannot read ") + path);
  char magic[8];
  int32_t hdr[2];
  bool ok = fread(magic, 1, 8, f) == 8 && memcmp(magic, kMagic, 8) == 0 &&
            fread(hdr, 4, 2, f) == 2 && hdr[0] > 0 && hdr[0] <= ME_MAX_NL &&
            hdr[1] == (4 * hdr[0] + 31) / 32 * 32;
  if (!ok) {
    fclose(f);
    return fail(ME_ERR_FORMAT, std::string("not an initialiser file: ") + path);
  }
  int nd = 0;
  if (cudaGetDeviceCount(&nd) != cudaSuccess || nd == 0) {
    fclose(f);
    return fail(ME_ERR_NODEVICE, "no CUDA device");
  }
  if (device < 0 || device >= nd) {
    fclose(f);
    return fail(ME_ERR_ARG, "device out of range");
  }
  cudaSetDevice(device);
  me_mlp *m = new me_mlp();
  m->device = device;
  std::unique_ptr<me_mlp, void (*)(me_mlp *)> guard(m, me_mlp_destroy);
  int rc = alloc_model(m, hdr[0]);
  if (rc) {
    fclose(f);
    return rc;
  }
  std::vector<float> prm((size_t)param_count(m));
  ok = fread(m->h_fmean.data(), 4, m->nip, f) == (size_t)m->nip &&
       fread(m->h_fistd.data(), 4, m->nip, f) == (size_t)m->nip &&
       fread(m->h_tmean.data(), 4, kOut, f) == (size_t)kOut &&
       fread(m->h_tstd.data(), 4, kOut, f) == (size_t)kOut &&
       fread(prm.data(), 4, prm.size(), f) == prm.size();
  fclose(f);
  if (!ok) return fail(ME_ERR_FORMAT, std::string("truncated initialiser file: ") + path);
  rc = upload_standardisation(m);
  if (!rc) rc = me_mlp_set_params(m, prm.data());
  if (rc) return rc;
  *out = guard.release();
  return ME_OK;
}
