// Surrogate pricer on the B200 tensor cores (include/fpe_surrogate.h).
//
// Every dense product of the MLP -- forward, input gradient and weight
// gradient -- is one shape of kernel: C[M x N] = A[M x K] B[N x K]^T with both
// operands BF16 and K-contiguous ("K-major"), FP32 accumulation in tensor
// memory.  The backward pass keeps feature-major (transposed) copies of the
// activations and gradients, written by the producing epilogues, so that the
// weight gradients are K-major products over the batch as well.
//
// Products with K a multiple of 64 run in a persistent kernel (k_gemm_bf16_tma,
// one CTA per SM): TMA loads 64-wide K chunks of A and B in the 128-byte
// swizzled layout into a four-stage mbarrier pipeline, one thread issues
// tcgen05.mma (M = 128, N <= 256, K = 16) into one of two TMEM accumulators,
// and four epilogue warps drain the other accumulator (tcgen05.ld, bias /
// SiLU / SiLU', stores) under the next tile's MMAs.  The remaining products
// (K = 16 input layers, split-K weight gradients) use k_gemm_bf16_tc: one CTA
// per 128 x N tile, K staged by cp.async into two buffers in the canonical
// no-swizzle K-major layout, the next chunk loading while the MMAs run.  In
// both, warp w reads TMEM lanes 32 (w % 4) .. + 31, the tile's rows.
//
// Adam follows the reference update rule (src/nn/adam.mojo:31-64).

#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <vector>

#include "../../include/fpe_surrogate.h"
#include "bulk_pipe.cuh"

namespace fpe {
namespace mlp {

using bf16 = __nv_bfloat16;

constexpr int kTileM = 128;
constexpr int kTileN = 256;
constexpr int kChunkK = 64;
constexpr int kThreads = 256;  // two warpgroups: both stage operands and split the epilogue's columns
constexpr int kBufBytes = (kTileM + kTileN) * kChunkK * 2;  // one A + B chunk
constexpr int kSmemBytes = 2 * kBufBytes;                    // double buffered (96 KB: <= 2 CTAs per SM)

// ---- tcgen05 helpers ---------------------------------------------------------
// Shared-memory matrix descriptor: start address, leading-dimension byte
// offset (between the two 8-element K halves of an MMA step) and stride byte
// offset (between 8-row groups), all >> 4; descriptor version 1; no swizzle.
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= uint64_t((saddr >> 4) & 0x3FFFu);
  d |= uint64_t((lbo >> 4) & 0x3FFFu) << 16;
  d |= uint64_t((sbo >> 4) & 0x3FFFu) << 32;
  d |= uint64_t(1) << 46;
  return d;
}

// Instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B, both
// K-major, N >> 3 at bit 17, M >> 4 at bit 24.
__host__ __device__ constexpr uint32_t umma_idesc_bf16(int m, int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | (uint32_t(n >> 3) << 17) | (uint32_t(m >> 4) << 24);
}

__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
// Warp-wide: allocate ncols TMEM columns, address written to *slot (shared).
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)),
               "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate) {
  const uint32_t z = 0;
  asm volatile(
      "{\n\t"
      ".reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t"
      "}\n" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(z), "r"(z), "r"(z), "r"(z)
      : "memory");
}
__device__ __forceinline__ void umma_commit(unsigned long long* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   smem_u32(bar))
               : "memory");
}
// 16 consecutive FP32 columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int j = 0; j < 16; ++j) v[j] = __uint_as_float(r[j]);
}

// The same load without its completion wait (several loads, then one
// tmem_wait_ld, before the registers are read).
__device__ __forceinline__ void tmem_ld16_async(uint32_t taddr, uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// 1 / (1 + e^-z) with the hardware exponential and reciprocal (a few ulp; the
// network's activations are rounded to BF16 anyway), branch-free so that the
// epilogues' elements interleave.  z is clamped at -80 so that 1 + e^-z stays
// below 2^126, where the fast division is exact to its stated error.
__device__ __forceinline__ float sigmoidf_(float z) { return __fdividef(1.0f, 1.0f + __expf(-fmaxf(z, -80.0f))); }

// ---- the product kernel --------------------------------------------------------
enum Epi : int {
  EPI_F32 = 0,        // Cf = A B^T (+ bias) (optionally SiLU)
  EPI_BIAS_SILU = 1,  // z = A B^T + bias: Cf = z (optional), Cb / CbT = bf16(silu(z))
  EPI_DSILU = 2,      // g = (A B^T) .* silu'(zin): Cf = g (optional), Cb / CbT = bf16(g)
};

struct GemmParams {
  const bf16* A;
  int lda;
  const bf16* B;
  int ldb;
  int M, N, K;
  int epi;
  int act;           // EPI_F32: 1 applies SiLU
  const float* bias;  // N, or null
  const float* zin;   // EPI_DSILU: M x N pre-activations (ldz)
  int ldz;
  float* Cf;
  int ldcf;
  bf16* Cb;
  int ldcb;
  bf16* CbT;  // transposed (N x M)
  int ldcbt;
  int tn;      // N tile width (16..256, a multiple of 16)
  int ksplit;  // K slices (grid z); > 1 only with EPI_F32 + atomic
  int atomic;  // EPI_F32: accumulate into Cf with atomicAdd (Cf zeroed by the caller)
  int* err;
};

// Epilogue of 16 accumulator columns gn .. gn + 15 of output row gm.
// b: the 16 columns' biases (zeros without a bias).
__device__ __forceinline__ void epilogue16(const GemmParams& P, const float (&b)[16], int gm, int gn, float (&v)[16]) {
  if (P.epi == EPI_F32) {
#pragma unroll
    for (int j = 0; j < 16; ++j) {
      float z = v[j] + b[j];
      if (P.act) z = z * sigmoidf_(z);
      v[j] = z;
    }
  } else if (P.epi == EPI_BIAS_SILU) {
#pragma unroll
    for (int j = 0; j < 16; ++j) v[j] += b[j];
  } else {
    const float* zr = P.zin + size_t(gm) * P.ldz + gn;
#pragma unroll
    for (int j = 0; j < 16; ++j) {
      const float z = zr[j], s = sigmoidf_(z);
      v[j] *= s * (1.0f + z * (1.0f - s));
    }
  }
  if (P.Cf && P.atomic) {
    float* d = P.Cf + size_t(gm) * P.ldcf + gn;
#pragma unroll
    for (int j = 0; j < 16; ++j) atomicAdd(d + j, v[j]);
  } else if (P.Cf) {
    float4* d = reinterpret_cast<float4*>(P.Cf + size_t(gm) * P.ldcf + gn);
#pragma unroll
    for (int q = 0; q < 4; ++q) d[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
  }
  if (P.Cb || P.CbT) {
    __align__(16) __nv_bfloat162 h2[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      float x0 = v[2 * j], x1 = v[2 * j + 1];
      if (P.epi == EPI_BIAS_SILU) {
        x0 *= sigmoidf_(x0);
        x1 *= sigmoidf_(x1);
      }
      h2[j] = __floats2bfloat162_rn(x0, x1);  // one packed conversion per pair
    }
    const bf16* h = reinterpret_cast<const bf16*>(h2);
    if (P.Cb) {
      uint4* d = reinterpret_cast<uint4*>(P.Cb + size_t(gm) * P.ldcb + gn);
      d[0] = *reinterpret_cast<const uint4*>(&h[0]);
      d[1] = *reinterpret_cast<const uint4*>(&h[8]);
    }
    if (P.CbT) {
#pragma unroll
      for (int j = 0; j < 16; ++j) P.CbT[size_t(gn + j) * P.ldcbt + gm] = h[j];
    }
  }
}

// Stage rows [row0, row0 + rows) x K [k0, k0 + kc) of a K-contiguous BF16
// matrix into the canonical layout: core matrix (row / 8, k / 8) at
// ((row / 8) * (kc / 8) + k / 8) * 128 bytes, row % 8 at 16 bytes each.  Each
// 16-byte piece moves by an asynchronous copy, so all of a thread's pieces are
// in flight together (completed by cp_async_wait_all).  Consecutive threads
// fill consecutive 16-byte rows of one core matrix (bank-conflict free).
__device__ __forceinline__ void stage_kmajor(unsigned char* dst, const bf16* src, int ld, int row0, int rows,
                                             int k0, int kc) {
  const int k8n = kc >> 3;
  for (int v = threadIdx.x; v < rows * k8n; v += blockDim.x) {
    const int q = v >> 3, rr = v & 7;     // core matrix q = (row group, k group)
    const int rg = q / k8n, j = q - rg * k8n;
    const int r = rg * 8 + rr;
    cp_async_elem<16>(dst + size_t(q) * 128 + rr * 16, src + size_t(row0 + r) * ld + k0 + 8 * j);
  }
}

__global__ void __launch_bounds__(kThreads, 1) k_gemm_bf16_tc(GemmParams P) {
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ unsigned long long bar[2];
  __shared__ uint32_t tmem_slot;
  const int m0 = blockIdx.x * kTileM, n0 = blockIdx.y * P.tn;
  const int Nt = min(P.tn, P.N - n0);
  // K slice of this CTA (split-K): whole 64-wide chunks
  const int kslice = ((P.K + P.ksplit - 1) / P.ksplit + kChunkK - 1) / kChunkK * kChunkK;
  const int kbeg = blockIdx.z * kslice, kend = min(P.K, kbeg + kslice);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  uint32_t ncols = 32;
  while (int(ncols) < Nt) ncols <<= 1;
  unsigned char* bufA[2] = {smem, smem + kBufBytes};
  unsigned char* bufB[2] = {smem + kTileM * kChunkK * 2, smem + kBufBytes + kTileM * kChunkK * 2};

  if (warp == 0) tmem_alloc(&tmem_slot, ncols);
  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    mbar_init_fence();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_slot;

  const int nchunk = kend > kbeg ? (kend - kbeg + kChunkK - 1) / kChunkK : 0;
  const uint32_t idesc = umma_idesc_bf16(kTileM, Nt);
  uint32_t phase = 0;
  bool ok = true;
  auto load = [&](int c, int b) {
    const int k0 = kbeg + c * kChunkK, kc = min(kChunkK, kend - k0);
    stage_kmajor(bufA[b], P.A, P.lda, m0, kTileM, k0, kc);
    stage_kmajor(bufB[b], P.B, P.ldb, n0, Nt, k0, kc);
  };
  if (nchunk > 0) load(0, 0);
  cp_async_wait_all();
  fence_proxy_async_smem();
  __syncthreads();
  for (int c = 0; c < nchunk; ++c) {
    const int b = c & 1;
    if (c >= 1) {  // the MMAs of chunk c - 1 are done: buffer b ^ 1 is free
      const int bp = b ^ 1;
      if (mbar_wait_bounded(&bar[bp], (phase >> bp) & 1u, kBulkWaitLimit)) {
        phase ^= 1u << bp;
      } else {
        ok = false;
      }
      tc_fence_after();
    }
    if (tid == 0 && ok) {
      tc_fence_after();
      const int k0 = kbeg + c * kChunkK, kc = min(kChunkK, kend - k0), k8n = kc >> 3;
      const uint32_t sa = smem_u32(bufA[b]), sb = smem_u32(bufB[b]);
      for (int s = 0; s < (kc >> 4); ++s) {
        const uint64_t ad = umma_desc(sa + 256u * s, 128u, uint32_t(k8n) * 128u);
        const uint64_t bd = umma_desc(sb + 256u * s, 128u, uint32_t(k8n) * 128u);
        umma_bf16(tmem, ad, bd, idesc, (c > 0 || s > 0) ? 1u : 0u);
      }
      umma_commit(&bar[b]);
    }
    if (c + 1 < nchunk) load(c + 1, b ^ 1);
    cp_async_wait_all();
    fence_proxy_async_smem();
    __syncthreads();
  }
  if (nchunk > 0) {
    const int bl = (nchunk - 1) & 1;
    if (mbar_wait_bounded(&bar[bl], (phase >> bl) & 1u, kBulkWaitLimit)) {
      phase ^= 1u << bl;
    } else {
      ok = false;
    }
    tc_fence_after();
  }
  ok = __syncthreads_and(ok ? 1 : 0) != 0;
  if (ok && nchunk > 0) {
    // warp w reads TMEM lanes 32 (w % 4) .. + 31 (tile rows); the two
    // warpgroups take alternate 16-column chunks of the accumulator
    const int quarter = warp & 3, half = warp >> 2;
    const int r = 32 * quarter + lane;
    const int gm = m0 + r;
    const uint32_t trow = tmem + (uint32_t(32 * quarter) << 16);
    for (int c = 16 * half; c < Nt; c += 32) {
      float v[16];
      tmem_ld16(trow + uint32_t(c), v);
      float b[16];
#pragma unroll
      for (int j = 0; j < 16; ++j) b[j] = P.bias ? P.bias[n0 + c + j] : 0.0f;
      epilogue16(P, b, gm, n0 + c, v);
    }
  } else if (!ok && tid == 0 && P.err) {
    atomicExch(P.err, 1);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    tmem_dealloc(tmem, ncols);
  }
}

// ---- persistent product with TMA staging ------------------------------------------
// C = A B^T for M a multiple of 128, K a multiple of 64 and N-tiles of up to
// 256 columns (a multiple of 16): one CTA per SM loops over the 128 x tn
// output tiles, with three roles:
//   warp 0 (one lane): TMA loads of the A and B K-chunks (64 BF16 = one
//     128-byte swizzle row per matrix row) into kPStages shared-memory
//     stages, each completing on its "full" mbarrier; a stage is refilled
//     once its "empty" barrier says that the MMAs reading it are done;
//   warp 1 (one lane): tcgen05.mma of each chunk into one of two TMEM
//     accumulators, tcgen05.commit to the stage's "empty" barrier, and after a
//     tile's last chunk to the accumulator's "full" barrier;
//   warps 2..9: the epilogue of a finished accumulator (warp w reads TMEM
//     lanes 32 (w % 4) .. + 31, the two warps of a lane quarter split the
//     columns; BF16 outputs leave through a per-warp shared staging tile as
//     whole 128-byte row segments), then an arrival on its "empty" barrier;
// so the loads of later chunks, the MMAs of tile i + 1 and the epilogue of
// tile i overlap.  Every wait is bounded: a wait that gives up sets *P.err and
// ends the CTA's loop, and the copies and MMAs already issued are waited out
// before the TMEM is released.  The tensor maps describe this GPU's own
// operands only, and no load is multicast.
constexpr int kPStages = 3;
constexpr int kPEpiWarps = 8;                    // two per TMEM lane quarter
constexpr int kPThreads = 64 + 32 * kPEpiWarps;  // TMA warp, MMA warp, epilogue warps
constexpr int kPStageA = kTileM * 128;           // 128 rows x 64 BF16
// Dynamic shared memory (offsets from the 1024-byte aligned base): a resident
// B of up to 128 KB then the A stages, or A + B stages; then one 4 KB staging
// tile (32 rows x 128 bytes) per epilogue warp for the coalesced BF16 stores.
constexpr int kPBres = 4 * kTileN * 128;  // 128 KB: K <= 256 at N = 256
constexpr int kPStagingOff =
    (kPBres + kPStages * kPStageA) > kPStages * (kPStageA + kTileN * 128) ? kPBres + kPStages * kPStageA
                                                                           : kPStages * (kPStageA + kTileN * 128);
constexpr int kPSmemBytes = kPStagingOff + kPEpiWarps * 4096 + 1024;  // + alignment of the swizzle atoms

// Shared-memory matrix descriptor of a K-major operand in the 128-byte
// swizzled layout that TMA writes (rows of 128 bytes, 8-row groups 1024 bytes
// apart): start address >> 4, stride byte offset 1024 >> 4, version 1,
// layout type 2 (128-byte swizzle).  The leading byte offset is unused for
// this layout.  An MMA step of K = 16 advances the start address by 32 bytes
// inside the swizzle row.
__device__ __forceinline__ uint64_t umma_desc_sw128(uint32_t saddr) {
  uint64_t d = 0;
  d |= uint64_t((saddr >> 4) & 0x3FFFu);
  d |= uint64_t(1) << 16;
  d |= uint64_t(1024 >> 4) << 32;
  d |= uint64_t(1) << 46;
  d |= uint64_t(2) << 61;
  return d;
}

// Tile (x = K offset in elements, y = row) of a 2-D tensor map into shared
// memory, completing on bar.  x is a multiple of 64: 128 bytes.
__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, int x, int y, uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
      "[%4];" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar)
      : "memory");
}

__global__ void __launch_bounds__(kPThreads, 1)
    k_gemm_bf16_tma(const __grid_constant__ CUtensorMap mapA, const __grid_constant__ CUtensorMap mapB,
                    GemmParams P) {
  extern __shared__ __align__(1024) unsigned char psmem[];
  __shared__ unsigned long long full[kPStages], empty[kPStages], accf[2], acce[2], done, bfull;
  __shared__ uint32_t tmem_slot;
  __shared__ volatile int give_up;  // a bounded wait gave up: every role leaves its loop
  __shared__ float sbias[kTileN * 4];  // the biases of up to four N-tiles
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t base = (smem_u32(psmem) + 1023u) & ~1023u;  // swizzle atoms are 1024-byte aligned
  const int BN = P.tn;
  const int tiles_m = P.M / kTileM, tiles_n = (P.N + BN - 1) / BN, ntiles = tiles_m * tiles_n;
  const int nk = P.K / kChunkK;
  uint32_t acc_cols = 32;
  while (int(acc_cols) < BN) acc_cols <<= 1;
  const uint32_t ncols = 2 * acc_cols;  // two accumulators
  // With one N-tile whose B fits the stages' B area (K <= 256 at N = 256), B
  // stays resident: its nk chunks are loaded once, at the start, and the
  // stages carry A alone (a sixth of the bytes per tile at K = N = 256).
  // When every N-tile's B fits the resident area (N x K <= 256 x 256), all of B
  // stays in shared memory: chunk kc of the nb = tiles_n x BN rows at
  // base + kc nb 128, loaded once at the start, and the stages carry A alone.
  const uint32_t bchunk = uint32_t(BN) * 128u;                    // bytes of one B chunk of one N-tile
  const uint32_t brow = uint32_t(tiles_n) * bchunk;               // bytes of one B chunk of all N-tiles
  const bool bres = uint32_t(nk) * brow <= uint32_t(kPBres);
  const uint32_t stage_bytes = bres ? uint32_t(kPStageA) : uint32_t(kPStageA) + bchunk;
  const uint32_t abase = bres ? base + uint32_t(kPBres) : base;  // stage 0
  if (warp == 1) tmem_alloc(&tmem_slot, ncols);
  if (tid == 0) {
    for (int s = 0; s < kPStages; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int a = 0; a < 2; ++a) {
      mbar_init(&accf[a], 1);
      mbar_init(&acce[a], kPThreads - 64);
    }
    mbar_init(&done, 1);
    mbar_init(&bfull, 1);
    give_up = 0;
    mbar_init_fence();
  }
  const bool bias_sh = P.bias && P.N <= kTileN * 4;
  if (bias_sh)
    for (int j = tid; j < P.N; j += blockDim.x) sbias[j] = P.bias[j];
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_slot;
  // the 16 biases of columns n .. n + 15 (shared-memory loads when the copy exists)
  auto bias16 = [&](int n, float (&b)[16]) {
    if (bias_sh) {
#pragma unroll
      for (int j = 0; j < 16; ++j) b[j] = sbias[n + j];
    } else {
#pragma unroll
      for (int j = 0; j < 16; ++j) b[j] = P.bias ? P.bias[n + j] : 0.0f;
    }
  };
  auto fail = [&]() {
    give_up = 1;
    if (P.err) atomicExch(P.err, 1);
  };
  if (warp == 0) {
    if (lane == 0) {
      int stage = 0;
      uint32_t ph = 0, pend = 0, pend_ph = 0;  // stages with a load in flight, and its phase parity
      const bool any = int(blockIdx.x) < ntiles;
      if (bres && any) {
        mbar_arrive_expect_tx(&bfull, uint32_t(nk) * brow);
        for (int kc = 0; kc < nk; ++kc)
          for (int nt = 0; nt < tiles_n; ++nt)
            tma_load_2d(base + uint32_t(kc) * brow + uint32_t(nt) * bchunk, &mapB, kc * kChunkK, nt * BN,
                        smem_u32(&bfull));
      }
      for (int t = blockIdx.x; t < ntiles && !give_up; t += gridDim.x) {
        const int m0 = (t / tiles_n) * kTileM, n0 = (t % tiles_n) * BN;
        for (int kc = 0; kc < nk; ++kc) {
          // a fresh barrier counts as having completed the phase before its first
          if (!mbar_wait_bounded(&empty[stage], ph ^ 1u, kBulkWaitLimit)) {
            fail();
            break;
          }
          const uint32_t sa = abase + uint32_t(stage) * stage_bytes;
          mbar_arrive_expect_tx(&full[stage], stage_bytes);
          tma_load_2d(sa, &mapA, kc * kChunkK, m0, smem_u32(&full[stage]));
          if (!bres) tma_load_2d(sa + kPStageA, &mapB, kc * kChunkK, n0, smem_u32(&full[stage]));
          pend |= 1u << stage;
          pend_ph = (pend_ph & ~(1u << stage)) | (ph << stage);
          if (++stage == kPStages) {
            stage = 0;
            ph ^= 1u;
          }
        }
      }
      // the loads this thread issued have all landed before the CTA ends
      for (int s = 0; s < kPStages; ++s)
        if ((pend >> s) & 1u) mbar_wait_bounded(&full[s], (pend_ph >> s) & 1u, kBulkWaitLimit);
      if (bres && any) mbar_wait_bounded(&bfull, 0, kBulkWaitLimit);
    }
  } else if (warp == 1) {
    if (lane == 0) {
      int stage = 0, acc = 0;
      uint32_t ph = 0, aph = 0;
      const uint32_t idesc = umma_idesc_bf16(kTileM, BN);
      if (bres && int(blockIdx.x) < ntiles && !mbar_wait_bounded(&bfull, 0, kBulkWaitLimit)) fail();
      for (int t = blockIdx.x; t < ntiles && !give_up; t += gridDim.x) {
        if (!mbar_wait_bounded(&acce[acc], aph ^ 1u, kBulkWaitLimit)) {
          fail();
          break;
        }
        tc_fence_after();
        const uint32_t d = tmem + uint32_t(acc) * acc_cols;
        bool ok = true;
        for (int kc = 0; kc < nk; ++kc) {
          if (!mbar_wait_bounded(&full[stage], ph, kBulkWaitLimit)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t sa = abase + uint32_t(stage) * stage_bytes;
          const uint32_t sb = bres ? base + uint32_t(kc) * brow + uint32_t(t % tiles_n) * bchunk : sa + kPStageA;
#pragma unroll
          for (int s = 0; s < kChunkK / 16; ++s)
            umma_bf16(d, umma_desc_sw128(sa + 32u * s), umma_desc_sw128(sb + 32u * s), idesc,
                      (kc > 0 || s > 0) ? 1u : 0u);
          umma_commit(&empty[stage]);  // the stage is free once these MMAs are done
          if (++stage == kPStages) {
            stage = 0;
            ph ^= 1u;
          }
        }
        if (!ok) {
          fail();
          break;
        }
        umma_commit(&accf[acc]);  // the accumulator is complete once every MMA above is
        acc ^= 1;
        if (acc == 0) aph ^= 1u;
      }
      // every MMA this thread issued has finished before the TMEM is released
      umma_commit(&done);
      mbar_wait_bounded(&done, 0, kBulkWaitLimit);
    }
  } else {
    // epilogue: warp w reads TMEM lanes 32 (w % 4) .. + 31, the tile's rows;
    // the two warps of a lane quarter (h = (w - 2) / 4) split the columns
    const int quarter = warp & 3, row = 32 * quarter + lane, h = (warp - 2) >> 2;
    // bias + SiLU to BF16 only (the inference layers): 64-column spans 64 h,
    // 64 h + 128, ... go through this warp's 4 KB staging tile, rows written
    // with their 16-byte chunks rotated by row (conflict-free), then read back
    // so that each store instruction writes four whole 128-byte row segments
    const bool staged = P.epi == EPI_BIAS_SILU && P.Cb && !P.Cf && !P.CbT;
    unsigned char* const stile = psmem + (base - smem_u32(psmem)) + kPStagingOff + (warp - 2) * 4096;
    int acc = 0;
    uint32_t aph = 0;
    // the warp's decisions are uniform: tcgen05.ld is warp-collective
    for (int t = blockIdx.x; t < ntiles && !__any_sync(0xffffffffu, give_up != 0); t += gridDim.x) {
      const int m0 = (t / tiles_n) * kTileM, n0 = (t % tiles_n) * BN;
      const int Nt = min(BN, P.N - n0);
      if (!__all_sync(0xffffffffu, mbar_wait_bounded(&accf[acc], aph, kBulkWaitLimit))) {
        fail();
        break;
      }
      tc_fence_after();
      const uint32_t trow = tmem + (uint32_t(32 * quarter) << 16) + uint32_t(acc) * acc_cols;
      if (staged && (Nt & 63) == 0) {
        for (int c = 64 * h; c < Nt; c += 128) {
          uint32_t r[4][16];
#pragma unroll
          for (int k = 0; k < 4; ++k) tmem_ld16_async(trow + uint32_t(c + 16 * k), r[k]);
          tmem_wait_ld();
#pragma unroll
          for (int k = 0; k < 4; ++k) {
            float b[16];
            bias16(n0 + c + 16 * k, b);
            uint32_t pk[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) {
              float x0 = __uint_as_float(r[k][2 * j]) + b[2 * j];
              float x1 = __uint_as_float(r[k][2 * j + 1]) + b[2 * j + 1];
              x0 *= sigmoidf_(x0);
              x1 *= sigmoidf_(x1);
              const __nv_bfloat162 h2 = __floats2bfloat162_rn(x0, x1);
              pk[j] = *reinterpret_cast<const uint32_t*>(&h2);
            }
            // chunks 2k and 2k + 1 of this lane's row
#pragma unroll
            for (int u = 0; u < 2; ++u) {
              const int ch = 2 * k + u;
              *reinterpret_cast<uint4*>(stile + lane * 128 + ((ch ^ (lane & 7)) << 4)) =
                  make_uint4(pk[4 * u], pk[4 * u + 1], pk[4 * u + 2], pk[4 * u + 3]);
            }
          }
          __syncwarp();
#pragma unroll
          for (int it = 0; it < 8; ++it) {
            const int rr = 4 * it + (lane >> 3), ch = lane & 7;
            const uint4 v = *reinterpret_cast<const uint4*>(stile + rr * 128 + ((ch ^ (rr & 7)) << 4));
            *reinterpret_cast<uint4*>(P.Cb + size_t(m0 + 32 * quarter + rr) * P.ldcb + n0 + c + 8 * ch) = v;
          }
          __syncwarp();  // the tile is rewritten by the next span
        }
      } else {
        // 16-column chunks 16 h, 16 h + 64, ... and the chunk 32 columns on
        // from each, two per completion wait
        for (int c = 16 * h; c < Nt; c += 64) {
          uint32_t r0[16], r1[16];
          const bool two = c + 32 < Nt;  // uniform in the warp
          tmem_ld16_async(trow + uint32_t(c), r0);
          if (two) tmem_ld16_async(trow + uint32_t(c + 32), r1);
          tmem_wait_ld();
          float v[16], b[16];
#pragma unroll
          for (int j = 0; j < 16; ++j) v[j] = __uint_as_float(r0[j]);
          bias16(n0 + c, b);
          epilogue16(P, b, m0 + row, n0 + c, v);
          if (two) {
#pragma unroll
            for (int j = 0; j < 16; ++j) v[j] = __uint_as_float(r1[j]);
            bias16(n0 + c + 32, b);
            epilogue16(P, b, m0 + row, n0 + c + 32, v);
          }
        }
      }
      tc_fence_before();
      mbar_arrive(&acce[acc]);
      acc ^= 1;
      if (acc == 0) aph ^= 1u;
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    tmem_dealloc(tmem, ncols);
  }
}

// ---- small kernels of the MLP -----------------------------------------------------
// X fp32 (n x n_in) -> BF16 (rows x in_pad) and its transpose; rows >= n and
// columns >= n_in are zero.
__global__ void k_pack_input(const float* __restrict__ x, int n, int n_in, int in_pad, int rows,
                             bf16* __restrict__ X, bf16* __restrict__ XT) {
  const int total = rows * in_pad;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < total; e += gridDim.x * blockDim.x) {
    const int r = e / in_pad, c = e - r * in_pad;
    const float v = (r < n && c < n_in) ? x[size_t(r) * n_in + c] : 0.0f;
    const bf16 b = __float2bfloat16_rn(v);
    X[e] = b;
    if (XT) XT[size_t(c) * rows + r] = b;
  }
}

// y_hat[r] = sum_j H[r][j] w[j] + b, one warp per row.
__global__ void k_out_forward(const bf16* __restrict__ H, int hidden, int rows, const float* __restrict__ w,
                              const float* __restrict__ b, float* __restrict__ y) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (warp >= rows) return;
  const bf16* h = H + size_t(warp) * hidden;
  float acc = 0.0f;
  for (int j = lane; j < hidden; j += 32) acc = fmaf(__bfloat162float(h[j]), w[j], acc);
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if (lane == 0) y[warp] = acc + b[0];
}

// dy[r] = 2 w_r (y_hat - y) / n (zero for padded rows); loss += w_r (y_hat - y)^2 / n.
__global__ void k_loss_grad(const float* __restrict__ yhat, const float* __restrict__ y,
                            const float* __restrict__ wt, int n, int rows, float* __restrict__ dy,
                            float* __restrict__ loss) {
  float part = 0.0f;
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < rows; r += gridDim.x * blockDim.x) {
    float g = 0.0f;
    if (r < n) {
      const float e = yhat[r] - y[r], w = wt ? wt[r] : 1.0f;
      g = 2.0f * w * e / float(n);
      part += w * e * e / float(n);
    }
    dy[r] = g;
  }
  for (int o = 16; o > 0; o >>= 1) part += __shfl_down_sync(0xffffffffu, part, o);
  if ((threadIdx.x & 31) == 0 && loss) atomicAdd(loss, part);
}

// Output layer backward: dZ[r][j] = dy[r] w[j] silu'(Z[r][j]) (fp32, bf16, bf16^T).
__global__ void k_out_backward(const float* __restrict__ dy, const float* __restrict__ w,
                               const float* __restrict__ Z, int rows, int hidden, float* __restrict__ dZ,
                               bf16* __restrict__ dZb, bf16* __restrict__ dZbT) {
  const int total = rows * hidden;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < total; e += gridDim.x * blockDim.x) {
    const int r = e / hidden, j = e - r * hidden;
    const float z = Z[e], s = sigmoidf_(z);
    const float g = dy[r] * w[j] * s * (1.0f + z * (1.0f - s));
    dZ[e] = g;
    const bf16 b = __float2bfloat16_rn(g);
    dZb[e] = b;
    dZbT[size_t(j) * rows + r] = b;
  }
}

// out[j] = sum_r X[r][j] (* s[r]) over rows, one block of 256 threads per 32
// columns: 8 row-slices x 32 columns, then a shared-memory reduction.
template <typename T>
__global__ void k_colsum(const T* __restrict__ X, int ld, int rows, int cols, const float* __restrict__ s,
                         float* __restrict__ out) {
  __shared__ float red[8][33];
  const int c = blockIdx.x * 32 + (threadIdx.x & 31), slice = threadIdx.x >> 5;
  float acc = 0.0f;
  if (c < cols) {
    for (int r = slice; r < rows; r += 8) {
      float x;
      if constexpr (sizeof(T) == 2) {
        x = __bfloat162float(X[size_t(r) * ld + c]);
      } else {
        x = X[size_t(r) * ld + c];
      }
      acc = fmaf(x, s ? s[r] : 1.0f, acc);
    }
  }
  red[slice][threadIdx.x & 31] = acc;
  __syncthreads();
  if (slice == 0 && c < cols) {
    float t = 0.0f;
    for (int k = 0; k < 8; ++k) t += red[k][threadIdx.x & 31];
    out[c] = t;
  }
}

__global__ void k_sum(const float* __restrict__ x, int n, float* __restrict__ out) {
  __shared__ float red[32];
  float acc = 0.0f;
  for (int i = threadIdx.x; i < n; i += blockDim.x) acc += x[i];
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    float t = 0.0f;
    for (int k = 0; k < int(blockDim.x >> 5); ++k) t += red[k];
    out[0] = t;
  }
}

// Step counter and hyper-parameters of one Adam step, on the device so that
// a captured training step replays correctly: t = ++step, lr = lr_arg, or
// (lr_arg < 0) the schedule entry of step t; hyper = {lr, 1 - b1^t, 1 - b2^t}.
__global__ void k_adam_prologue(int* __restrict__ step, const float* __restrict__ table, int len, float lr_arg,
                                float b1, float b2, float* __restrict__ hyper) {
  const int t = ++step[0];
  float lr = lr_arg;
  if (lr_arg < 0.0f) lr = (table && len > 0) ? table[min(t - 1, len - 1)] : 0.0f;
  hyper[0] = lr;
  hyper[1] = 1.0f - powf(b1, float(t));
  hyper[2] = 1.0f - powf(b2, float(t));
}

// Adam (reference src/nn/adam.mojo:31-64): m = b1 m + (1-b1) g, v = b2 v + (1-b2) g^2,
// theta -= lr * (m / (1 - b1^t)) / (sqrt(v / (1 - b2^t)) + eps).
__global__ void k_adam(float* __restrict__ theta, const float* __restrict__ g, float* __restrict__ m,
                       float* __restrict__ v, int64_t n, const float* __restrict__ hyper, float b1, float b2,
                       float eps) {
  const float lr = hyper[0], c1 = hyper[1], c2 = hyper[2];
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    theta[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  }
}

// BF16 copies of a weight matrix W (out x in, row-major) and of its transpose.
__global__ void k_cast_weights(const float* __restrict__ W, int out, int in, bf16* __restrict__ Wb,
                               bf16* __restrict__ WbT) {
  const int total = out * in;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < total; e += gridDim.x * blockDim.x) {
    const int o = e / in, i = e - o * in;
    const bf16 b = __float2bfloat16_rn(W[e]);
    Wb[e] = b;
    WbT[size_t(i) * out + o] = b;
  }
}

}  // namespace mlp
}  // namespace fpe

// =====================================================================================
// Host side
// =====================================================================================
namespace {

using fpe::mlp::bf16;

#define MK(x)                                                                       \
  do {                                                                              \
    cudaError_t e_ = (x);                                                           \
    if (e_ != cudaSuccess) {                                                        \
      if (std::getenv("FPE_DEBUG"))                                                 \
        std::fprintf(stderr, "fpe_mlp: %s failed: %s (%s:%d)\n", #x, cudaGetErrorString(e_), \
                     __FILE__, __LINE__);                                           \
      return -1;                                                                    \
    }                                                                               \
  } while (0)

struct MlpCtx {
  bool ok = false;
  cudaStream_t stream = nullptr;
  int sms = 0;  // SMs of the device: the persistent product's grid
  // the driver's tensor-map encoder (through the runtime's entry-point query,
  // so that the library needs no link against the driver library); null: the
  // persistent TMA product is unavailable and every product takes the
  // per-tile kernel
  PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
};

MlpCtx& mctx() {
  static MlpCtx c;
  static std::once_flag once;
  std::call_once(once, [] {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n <= 0) return;
    if (cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking) != cudaSuccess) return;
    if (cudaFuncSetAttribute(fpe::mlp::k_gemm_bf16_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             fpe::mlp::kSmemBytes) != cudaSuccess)
      return;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&c.sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
      return;
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess && fn &&
        cudaFuncSetAttribute(fpe::mlp::k_gemm_bf16_tma, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             fpe::mlp::kPSmemBytes) == cudaSuccess)
      c.encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    c.ok = true;
  });
  return c;
}

// Tensor map of a K-contiguous BF16 matrix (rows x K, row stride ld
// elements): boxes of 64 K-elements (128 bytes) x box_rows rows in the
// 128-byte swizzled layout; rows past the end read as zeros.
int make_map(CUtensorMap* m, const bf16* base, int rows, int K, int ld, int box_rows) {
  const cuuint64_t dims[2] = {cuuint64_t(K), cuuint64_t(rows)};
  const cuuint64_t strides[1] = {cuuint64_t(ld) * sizeof(bf16)};
  const cuuint32_t box[2] = {cuuint32_t(fpe::mlp::kChunkK), cuuint32_t(box_rows)};
  const cuuint32_t estr[2] = {1, 1};
  const CUresult r = mctx().encode(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<bf16*>(base), dims, strides,
                                   box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                                   CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? 0 : -1;
}

int launch_gemm(const fpe::mlp::GemmParams& P, cudaStream_t s) {
  using namespace fpe::mlp;
  if (P.M <= 0 || P.N <= 0 || P.K <= 0 || P.M % kTileM || P.N % 16 || P.K % 16 || P.lda % 8 || P.ldb % 8)
    return -1;
  if ((reinterpret_cast<uintptr_t>(P.A) | reinterpret_cast<uintptr_t>(P.B)) & 15) return -1;
  if (P.Cf && (P.ldcf % 4 || (reinterpret_cast<uintptr_t>(P.Cf) & 15))) return -1;
  if (P.Cb && (P.ldcb % 8 || (reinterpret_cast<uintptr_t>(P.Cb) & 15))) return -1;
  if (P.tn < 16 || P.tn > kTileN || P.tn % 16 || P.ksplit < 1) return -1;
  if (P.ksplit > 1 && !(P.epi == EPI_F32 && P.atomic && !P.bias && !P.act && !P.Cb && !P.CbT)) return -1;
  if (P.ksplit == 1 && P.K % kChunkK == 0 && mctx().encode) {
    // persistent product, one CTA per SM, N-tiles as wide as N allows (128-wide
    // tiles at N = 256, for a shorter last wave, measured no faster)
    GemmParams Q = P;
    Q.tn = std::min(P.N, kTileN);
    CUtensorMap ma, mb;
    if (make_map(&ma, P.A, P.M, P.K, P.lda, kTileM) == 0 && make_map(&mb, P.B, P.N, P.K, P.ldb, Q.tn) == 0) {
      const int tiles = (P.M / kTileM) * ((P.N + Q.tn - 1) / Q.tn);
      k_gemm_bf16_tma<<<std::min(tiles, mctx().sms), kPThreads, kPSmemBytes, s>>>(ma, mb, Q);
      MK(cudaGetLastError());
      return 0;
    }
  }
  const dim3 grid(P.M / kTileM, (P.N + P.tn - 1) / P.tn, P.ksplit);
  k_gemm_bf16_tc<<<grid, kThreads, kSmemBytes, s>>>(P);
  MK(cudaGetLastError());
  return 0;
}

fpe::mlp::GemmParams gp(const bf16* A, int lda, const bf16* B, int ldb, int M, int N, int K, int epi, int* err) {
  fpe::mlp::GemmParams P{};
  P.A = A;
  P.lda = lda;
  P.B = B;
  P.ldb = ldb;
  P.M = M;
  P.N = N;
  P.K = K;
  P.epi = epi;
  P.err = err;
  // narrower N tiles when the row tiles alone would leave most SMs idle
  P.tn = (M / fpe::mlp::kTileM < 74 && N >= 256) ? 128 : std::min(N, fpe::mlp::kTileN);
  if (P.tn % 16) P.tn = fpe::mlp::kTileN;
  P.ksplit = 1;
  return P;
}

inline int grid_for(int64_t n, int block = 256) {
  const int64_t g = (n + block - 1) / block;
  return int(g < 1 ? 1 : (g > 148 * 32 ? 148 * 32 : g));
}

uint64_t splitmix(uint64_t& s) {
  uint64_t z = (s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

}  // namespace

struct FpeMlp {
  int n_in = 0, in_pad = 0, hidden = 0, layers = 0, rows = 0;  // rows: max rows per call (multiple of 128)
  int64_t n_params = 0;
  std::vector<int64_t> off_w, off_b;  // per hidden layer
  int64_t off_wo = 0, off_bo = 0;
  float *theta = nullptr, *grad = nullptr, *m = nullptr, *v = nullptr;
  std::vector<bf16*> Wb, WbT;
  bf16 *X = nullptr, *XT = nullptr;
  std::vector<float*> Z;
  std::vector<bf16*> H, HT;
  float *dZ[2] = {nullptr, nullptr};
  bf16 *dZb[2] = {nullptr, nullptr}, *dZbT[2] = {nullptr, nullptr};
  float *yhat = nullptr, *dy = nullptr, *loss = nullptr;
  int* err = nullptr;
  // inference: rows per launch sequence and its own buffers
  int irows = 0;
  bf16* Xi = nullptr;
  bf16* Hi[2] = {nullptr, nullptr};
  float* yi = nullptr;
  int* step = nullptr;          // Adam step counter (device)
  float* hyper = nullptr;       // {lr, 1 - b1^t, 1 - b2^t} of the current step (device)
  float* lr_table = nullptr;    // learning-rate schedule (device), lr_len entries
  int lr_len = 0;
  std::vector<void*> allocs;

  int in_of(int l) const { return l == 0 ? in_pad : hidden; }
  template <typename T>
  int alloc(T** p, size_t count) {
    void* q = nullptr;
    MK(cudaMalloc(&q, std::max<size_t>(count, 1) * sizeof(T)));
    MK(cudaMemset(q, 0, std::max<size_t>(count, 1) * sizeof(T)));
    allocs.push_back(q);
    *p = static_cast<T*>(q);
    return 0;
  }
  ~FpeMlp() {
    for (void* p : allocs) cudaFree(p);
  }
};

namespace {

int mlp_cast_all(FpeMlp* M, cudaStream_t s) {
  for (int l = 0; l < M->layers; ++l) {
    const int in = M->in_of(l);
    fpe::mlp::k_cast_weights<<<grid_for(int64_t(M->hidden) * in), 256, 0, s>>>(
        M->theta + M->off_w[l], M->hidden, in, M->Wb[l], M->WbT[l]);
  }
  MK(cudaGetLastError());
  return 0;
}

// Forward over rows [0, rows) of the packed input; keep = 1 stores Z and H^T
// (training buffers), otherwise only H (inference buffers Xi, Hi, yi).
int mlp_forward_packed(FpeMlp* M, int rows, bool keep, cudaStream_t s) {
  using namespace fpe::mlp;
  const bf16* in = keep ? M->X : M->Xi;
  int ld_in = M->in_pad;
  for (int l = 0; l < M->layers; ++l) {
    GemmParams P = gp(in, ld_in, M->Wb[l], M->in_of(l), rows, M->hidden, M->in_of(l), EPI_BIAS_SILU, M->err);
    P.bias = M->theta + M->off_b[l];
    P.Cb = keep ? M->H[l] : M->Hi[l & 1];
    P.ldcb = M->hidden;
    if (keep) {
      P.Cf = M->Z[l];
      P.ldcf = M->hidden;
      P.CbT = M->HT[l];
      P.ldcbt = M->rows;
    }
    if (launch_gemm(P, s)) return -1;
    in = P.Cb;
    ld_in = M->hidden;
  }
  const bf16* last = keep ? M->H[M->layers - 1] : M->Hi[(M->layers - 1) & 1];
  k_out_forward<<<(rows * 32 + 255) / 256, 256, 0, s>>>(last, M->hidden, rows, M->theta + M->off_wo,
                                                         M->theta + M->off_bo, keep ? M->yhat : M->yi);
  MK(cudaGetLastError());
  return 0;
}

// Forward + backward: gradient of sum_i w_i (y_hat_i - y_i)^2 / n into M->grad,
// loss into M->loss.
int mlp_backward(FpeMlp* M, const float* x, const float* y, const float* w, int n, cudaStream_t s) {
  using namespace fpe::mlp;
  const int R = M->rows, Hd = M->hidden;
  k_pack_input<<<grid_for(int64_t(R) * M->in_pad), 256, 0, s>>>(x, n, M->n_in, M->in_pad, R, M->X, M->XT);
  MK(cudaGetLastError());
  if (mlp_forward_packed(M, R, true, s)) return -1;
  MK(cudaMemsetAsync(M->loss, 0, sizeof(float), s));
  k_loss_grad<<<grid_for(R), 256, 0, s>>>(M->yhat, y, w, n, R, M->dy, M->loss);
  const int L = M->layers;
  // output layer
  k_colsum<bf16><<<(Hd + 31) / 32, 256, 0, s>>>(M->H[L - 1], Hd, R, Hd, M->dy, M->grad + M->off_wo);
  k_sum<<<1, 256, 0, s>>>(M->dy, R, M->grad + M->off_bo);
  int cur = 0;
  k_out_backward<<<grid_for(int64_t(R) * Hd), 256, 0, s>>>(M->dy, M->theta + M->off_wo, M->Z[L - 1], R, Hd,
                                                             M->dZ[cur], M->dZb[cur], M->dZbT[cur]);
  MK(cudaGetLastError());
  for (int l = L - 1; l >= 0; --l) {
    const int in = M->in_of(l);
    // dW_l = dZ_l^T H_{l-1}: A = dZ_l^T (hidden x R), B = H_{l-1}^T (in x R)
    const bf16* Bt = l == 0 ? M->XT : M->HT[l - 1];
    GemmParams P = gp(M->dZbT[cur], R, Bt, R, Hd, in, R, EPI_F32, M->err);
    P.Cf = M->grad + M->off_w[l];
    P.ldcf = in;
    // the batch is the reduction dimension: split it so that the few row
    // tiles (hidden / 128) still spread over the SMs, accumulating atomically
    P.tn = std::min(in, fpe::mlp::kTileN);
    P.ksplit = std::max(1, std::min(64, R / 128));
    P.atomic = 1;
    MK(cudaMemsetAsync(P.Cf, 0, size_t(Hd) * in * sizeof(float), s));
    if (launch_gemm(P, s)) return -1;
    k_colsum<float><<<(Hd + 31) / 32, 256, 0, s>>>(M->dZ[cur], Hd, R, Hd, nullptr, M->grad + M->off_b[l]);
    if (l > 0) {
      // dZ_{l-1} = (dZ_l W_l) .* silu'(Z_{l-1}): A = dZ_l (R x hidden), B = W_l^T (hidden x hidden)
      GemmParams Q = gp(M->dZb[cur], Hd, M->WbT[l], Hd, R, Hd, Hd, EPI_DSILU, M->err);
      Q.zin = M->Z[l - 1];
      Q.ldz = Hd;
      Q.Cf = M->dZ[cur ^ 1];
      Q.ldcf = Hd;
      Q.Cb = M->dZb[cur ^ 1];
      Q.ldcb = Hd;
      Q.CbT = M->dZbT[cur ^ 1];
      Q.ldcbt = R;
      if (launch_gemm(Q, s)) return -1;
      cur ^= 1;
    }
  }
  MK(cudaGetLastError());
  return 0;
}

int check_err(FpeMlp* M, cudaStream_t s) {
  int h = 0;
  MK(cudaMemcpyAsync(&h, M->err, sizeof(int), cudaMemcpyDeviceToHost, s));
  MK(cudaStreamSynchronize(s));
  return h ? -2 : 0;
}

}  // namespace

extern "C" {

FpeMlp* fpe_mlp_create(int32_t n_in, int32_t hidden, int32_t layers, int32_t max_rows, uint64_t seed) {
  if (n_in <= 0 || n_in > 256 || (hidden != 128 && hidden != 256) || layers < 1 || layers > 16 ||
      max_rows <= 0)
    return nullptr;
  if (!mctx().ok) return nullptr;
  auto* M = new FpeMlp();
  M->n_in = n_in;
  M->in_pad = (n_in + 15) & ~15;
  M->hidden = hidden;
  M->layers = layers;
  M->rows = (max_rows + 127) & ~127;
  int64_t o = 0;
  for (int l = 0; l < layers; ++l) {
    M->off_w.push_back(o);
    o += int64_t(hidden) * M->in_of(l);
    M->off_b.push_back(o);
    o += hidden;
  }
  M->off_wo = o;
  o += hidden;
  M->off_bo = o;
  o += 1;
  M->n_params = o;
  // host init: U(-1/sqrt(fan_in), 1/sqrt(fan_in)), padded input columns zero
  std::vector<float> h(size_t(o), 0.0f);
  uint64_t st = seed * 0x2545F4914F6CDD1Dull + 1;
  auto uni = [&](float a) { return float((double(splitmix(st) >> 11) * 0x1.0p-53 * 2.0 - 1.0) * a); };
  for (int l = 0; l < layers; ++l) {
    const int fan = l == 0 ? n_in : hidden, in = M->in_of(l);
    const float a = 1.0f / std::sqrt(float(fan));
    for (int r = 0; r < hidden; ++r)
      for (int c = 0; c < fan; ++c) h[size_t(M->off_w[l] + int64_t(r) * in + c)] = uni(a);
    for (int r = 0; r < hidden; ++r) h[size_t(M->off_b[l] + r)] = uni(a);
  }
  {
    const float a = 1.0f / std::sqrt(float(hidden));
    for (int r = 0; r < hidden; ++r) h[size_t(M->off_wo + r)] = uni(a);
    h[size_t(M->off_bo)] = uni(a);
  }
  bool bad = M->alloc(&M->theta, o) || M->alloc(&M->grad, o) || M->alloc(&M->m, o) || M->alloc(&M->v, o);
  M->Wb.resize(layers);
  M->WbT.resize(layers);
  M->Z.resize(layers);
  M->H.resize(layers);
  M->HT.resize(layers);
  const size_t R = size_t(M->rows);
  for (int l = 0; l < layers && !bad; ++l) {
    const size_t wsz = size_t(hidden) * M->in_of(l);
    bad = M->alloc(&M->Wb[l], wsz) || M->alloc(&M->WbT[l], wsz) || M->alloc(&M->Z[l], R * hidden) ||
          M->alloc(&M->H[l], R * hidden) || M->alloc(&M->HT[l], R * hidden);
  }
  for (int k = 0; k < 2 && !bad; ++k)
    bad = M->alloc(&M->dZ[k], R * hidden) || M->alloc(&M->dZb[k], R * hidden) || M->alloc(&M->dZbT[k], R * hidden);
  bad = bad || M->alloc(&M->X, R * M->in_pad) || M->alloc(&M->XT, R * M->in_pad) || M->alloc(&M->yhat, R) ||
        M->alloc(&M->dy, R) || M->alloc(&M->loss, 1) || M->alloc(&M->err, 1) || M->alloc(&M->step, 1) ||
        M->alloc(&M->hyper, 4);
  M->irows = std::max(M->rows, 65536);
  bad = bad || M->alloc(&M->Xi, size_t(M->irows) * M->in_pad) || M->alloc(&M->Hi[0], size_t(M->irows) * hidden) ||
        M->alloc(&M->Hi[1], size_t(M->irows) * hidden) || M->alloc(&M->yi, size_t(M->irows));
  if (bad || cudaMemcpy(M->theta, h.data(), size_t(o) * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess ||
      mlp_cast_all(M, mctx().stream) || cudaStreamSynchronize(mctx().stream) != cudaSuccess) {
    delete M;
    return nullptr;
  }
  return M;
}

void fpe_mlp_destroy(FpeMlp* M) {
  if (!M) return;
  cudaDeviceSynchronize();
  delete M;
}

int64_t fpe_mlp_layout(const FpeMlp* M, int32_t* layout) {
  if (!M) return -1;
  if (layout) {
    layout[0] = M->n_in;
    layout[1] = M->in_pad;
    layout[2] = M->hidden;
    layout[3] = M->layers;
  }
  return M->n_params;
}

int32_t fpe_mlp_get_params(FpeMlp* M, float* out, int64_t n) {
  if (!M || !out || n != M->n_params) return -1;
  MK(cudaStreamSynchronize(mctx().stream));
  MK(cudaMemcpy(out, M->theta, size_t(n) * sizeof(float), cudaMemcpyDeviceToHost));
  return 0;
}

int32_t fpe_mlp_set_params(FpeMlp* M, const float* in, int64_t n) {
  if (!M || !in || n != M->n_params) return -1;
  cudaStream_t s = mctx().stream;
  MK(cudaStreamSynchronize(s));
  MK(cudaMemcpy(M->theta, in, size_t(n) * sizeof(float), cudaMemcpyHostToDevice));
  MK(cudaMemset(M->m, 0, size_t(n) * sizeof(float)));
  MK(cudaMemset(M->v, 0, size_t(n) * sizeof(float)));
  MK(cudaMemset(M->step, 0, sizeof(int)));
  if (mlp_cast_all(M, s)) return -1;
  MK(cudaStreamSynchronize(s));
  return 0;
}

int32_t fpe_mlp_forward(FpeMlp* M, const float* x, int32_t n, float* y, void* stream) {
  if (!M || !x || !y || n < 0) return -1;
  cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : mctx().stream;
  for (int32_t r0 = 0; r0 < n; r0 += M->irows) {
    const int cnt = std::min(M->irows, n - r0);
    const int rows = (cnt + 127) & ~127;
    fpe::mlp::k_pack_input<<<grid_for(int64_t(rows) * M->in_pad), 256, 0, s>>>(
        x + size_t(r0) * M->n_in, cnt, M->n_in, M->in_pad, rows, M->Xi, nullptr);
    if (mlp_forward_packed(M, rows, false, s)) return -1;
    MK(cudaMemcpyAsync(y + r0, M->yi, size_t(cnt) * sizeof(float), cudaMemcpyDeviceToDevice, s));
  }
  MK(cudaGetLastError());
  return 0;
}

int32_t fpe_mlp_train_step(FpeMlp* M, const float* x, const float* y, const float* w, int32_t n, float lr,
                           float* loss_dev, void* stream) {
  if (!M || !x || !y || n <= 0 || n > M->rows) return -1;
  cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : mctx().stream;
  if (mlp_backward(M, x, y, w, n, s)) return -1;
  if (loss_dev) MK(cudaMemcpyAsync(loss_dev, M->loss, sizeof(float), cudaMemcpyDeviceToDevice, s));
  const float b1 = 0.9f, b2 = 0.999f;
  fpe::mlp::k_adam_prologue<<<1, 1, 0, s>>>(M->step, M->lr_table, M->lr_len, lr, b1, b2, M->hyper);
  fpe::mlp::k_adam<<<grid_for(M->n_params), 256, 0, s>>>(M->theta, M->grad, M->m, M->v, M->n_params, M->hyper,
                                                          b1, b2, 1e-8f);
  MK(cudaGetLastError());
  return mlp_cast_all(M, s);
}

int32_t fpe_mlp_set_lr_schedule(FpeMlp* M, const float* host_table, int32_t n) {
  if (!M || n < 0 || (n > 0 && !host_table)) return -1;
  MK(cudaStreamSynchronize(mctx().stream));
  if (M->lr_table) {
    cudaFree(M->lr_table);
    for (auto& p : M->allocs)
      if (p == M->lr_table) p = nullptr;
    M->lr_table = nullptr;
    M->lr_len = 0;
  }
  if (n > 0) {
    if (M->alloc(&M->lr_table, size_t(n))) return -1;
    MK(cudaMemcpy(M->lr_table, host_table, size_t(n) * sizeof(float), cudaMemcpyHostToDevice));
    M->lr_len = n;
  }
  return 0;
}

int32_t fpe_mlp_gradient(FpeMlp* M, const float* x, const float* y, const float* w, int32_t n, float* grad_host,
                         float* loss_host) {
  if (!M || !x || !y || n <= 0 || n > M->rows || !grad_host) return -1;
  cudaStream_t s = mctx().stream;
  MK(cudaMemsetAsync(M->err, 0, sizeof(int), s));
  if (mlp_backward(M, x, y, w, n, s)) return -1;
  MK(cudaMemcpyAsync(grad_host, M->grad, size_t(M->n_params) * sizeof(float), cudaMemcpyDeviceToHost, s));
  if (loss_host) MK(cudaMemcpyAsync(loss_host, M->loss, sizeof(float), cudaMemcpyDeviceToHost, s));
  return check_err(M, s);
}

int32_t fpe_gemm_bf16(const void* a, int32_t lda, const void* b, int32_t ldb, int32_t M, int32_t N, int32_t K,
                      const float* bias, int32_t act, float* c, int32_t ldc, void* stream) {
  if (!a || !b || !c) return -1;
  if (!mctx().ok) return -1;
  cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : mctx().stream;
  static int* d_err = nullptr;
  static std::mutex mu;
  {
    std::lock_guard<std::mutex> lock(mu);
    if (!d_err) MK(cudaMalloc(&d_err, sizeof(int)));
  }
  MK(cudaMemsetAsync(d_err, 0, sizeof(int), s));
  fpe::mlp::GemmParams P = gp(static_cast<const bf16*>(a), lda, static_cast<const bf16*>(b), ldb, M, N, K,
                              fpe::mlp::EPI_F32, d_err);
  P.bias = bias;
  P.act = act;
  P.Cf = c;
  P.ldcf = ldc;
  if (launch_gemm(P, s)) return -1;
  int h = 0;
  MK(cudaMemcpyAsync(&h, d_err, sizeof(int), cudaMemcpyDeviceToHost, s));
  MK(cudaStreamSynchronize(s));
  return h ? -2 : 0;
}

}  // extern "C"
