// K4 Schur complement on the 5th-generation tensor cores (tcgen05, sm_100a):
//     C -= L * U   (complex, FP32 planes Cr/Ci, FP32 accuracy through 3xTF32 products)
//
// Operands are pre-split (k_split_a / k_split_b) into four K-major planes each:
// hi(real), lo(real), hi(imag), lo(imag), hi = x rounded to TF32, lo = (x - hi) rounded
// to TF32.  With a = ah + al, b = bh + bl the complex product accumulates
//     Dr += ah_r bh_r + ah_r bl_r + al_r bh_r - (ah_i bh_i + ah_i bl_i + al_i bh_i)
//     Di += ah_r bh_i + ah_r bl_i + al_r bh_i + ah_i bh_r + ah_i bl_r + al_i bh_r
// (12 MMAs per 8-deep K slice; the minus sign is the MMA's negate-A bit).
//
// Persistent kernel, one CTA per SM, 192 threads:
//   warp 0  TMA producer: 3-stage ring of {4 A tiles 128x16, 4 B tiles 128x16} fp32,
//           64-byte swizzle, one mbarrier pair per stage;
//   warp 1  MMA issuer (one thread): tcgen05.mma.cta_group::1.kind::tf32, M=N=128, K=8,
//           accumulators in TMEM (2 buffers x {Dr, Di} x 128 columns = 512 columns);
//   warps 2-5 epilogue: tcgen05.ld of the accumulators, C -= D with 16-byte loads/stores,
//           overlapped with the next tile's MMAs.
// Every wait is bounded; a timeout sets *err and the kernel drains and returns.
#include <cuda.h>
#include <cudaTypedefs.h>

#include "pss_internal.cuh"

namespace {

constexpr int BM = 128, BN = 128, BK = 16, KSUB = 8;
constexpr int STAGES = 3;
constexpr int TILE_BYTES = BM * BK * 4;          // 8 KB per plane tile
constexpr int STAGE_BYTES = 8 * TILE_BYTES;      // 4 A + 4 B planes
constexpr int EPI_BYTES = 2 * BM * 32 * 4;  // epilogue staging: 32 columns of the tile, both planes
constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + EPI_BYTES + 1024 + 256;
static_assert(SMEM_BYTES <= 232448, "dynamic shared memory of one CTA");
constexpr uint32_t TMEM_COLS = 512;
constexpr long long kWaitCap = 1LL << 24;
// Written to *err when a bounded wait gives up: negative, like LAPACK's argument errors, so an
// LU's info keeps its positive values for zero pivots.
constexpr int kErrTimeout = -1;

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
// Bounded wait for the phase with parity `par` to complete: at most `cap` polls.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t par, long long cap = kWaitCap) {
  const uint32_t a = smem_u32(bar);
  for (long long it = 0; it < cap; ++it) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(a), "r"(par)
        : "memory");
    if (ok) return true;
  }
  return false;
}

__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, uint64_t *bar, int c0, int c1,
                                            int c2) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5}], "
      "[%2];" ::"r"(smem_u32(dst)),
      "l"(map), "r"(smem_u32(bar)), "r"(c0), "r"(c1), "r"(c2)
      : "memory");
}

// Shared-memory matrix descriptor: K-major, 64-byte swizzle, 8-row core groups 512 B apart.
__device__ __forceinline__ uint64_t sdesc(const void *p) {
  const uint64_t addr = smem_u32(p);
  uint64_t d = 0;
  d |= (addr >> 4) & 0x3FFFull;                 // start address
  d |= (uint64_t)1 << 16;                       // leading byte offset (unused for swizzled K-major)
  d |= (uint64_t)(512 >> 4) << 32;              // stride byte offset: 8 rows x 64 B
  d |= (uint64_t)1 << 46;                       // descriptor version (sm_100)
  d |= (uint64_t)4 << 61;                       // swizzle mode: 64-byte
  return d;
}

// Instruction descriptor, kind::tf32: D f32, A/B tf32, K-major A and B, M = N = 128.
__host__ __device__ constexpr uint32_t idesc_tf32(bool negA) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((negA ? 1u : 0u) << 13) | ((uint32_t)(BN >> 3) << 17) |
         ((uint32_t)(BM >> 4) << 24);
}

__device__ __forceinline__ void mma_tf32(uint32_t dtmem, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(dtmem),
      "l"(da), "l"(db), "r"(idesc), "r"(acc)
      : "memory");
}

__device__ __forceinline__ void mma_commit(uint64_t *bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float *v) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

struct GemmArgs {
  float *Cr, *Ci;
  long long ldc, ms;  // leading dimension; elements between the matrices of the batch
  int m0, n0;         // C offset of the update (rows, columns)
  int M, N;           // extent of the update
  int nk;             // number of BK slices (K / 16, K padded with zeros)
  int nb;             // matrices in the batch
  int *err;           // one error word per matrix
  int tma_epi;        // C -= D by TMA reduce-add (mapCr / mapCi), else by loads and stores
  long long wait_cap; // polls of a pipeline hand-off wait (the final drain waits use kWaitCap)
};

// OR / AND of a predicate over the 128 epilogue threads (named barrier 1).
__device__ __forceinline__ bool epi_any(bool v) {
  uint32_t r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\tsetp.ne.u32 q, %1, 0;\n\tbar.red.or.pred p, 1, 128, q;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(r)
      : "r"((uint32_t)v)
      : "memory");
  return r != 0;
}
__device__ __forceinline__ bool epi_all(bool v) {
  uint32_t r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\tsetp.ne.u32 q, %1, 0;\n\tbar.red.and.pred p, 1, 128, q;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(r)
      : "r"((uint32_t)v)
      : "memory");
  return r != 0;
}

// A bounded wait gave up: every matrix of the batch is marked (its update is incomplete).
__device__ __forceinline__ void fail_all(const GemmArgs &g) {
  for (int b = 0; b < g.nb; ++b) atomicExch(g.err + b, kErrTimeout);
}

__global__ void __launch_bounds__(192, 1) k_cgemm_tf32x3(const __grid_constant__ CUtensorMap mapA,
                                                         const __grid_constant__ CUtensorMap mapB,
                                                         const __grid_constant__ CUtensorMap mapCr,
                                                         const __grid_constant__ CUtensorMap mapCi, GemmArgs g) {
  extern __shared__ __align__(1024) unsigned char smraw[];
  unsigned char *base = (unsigned char *)(((uintptr_t)smraw + 1023) & ~(uintptr_t)1023);
  unsigned char *epi = base + STAGES * STAGE_BYTES;  // [2 planes][128 rows][32 floats], 128-byte swizzle
  uint64_t *full = (uint64_t *)(epi + EPI_BYTES);
  uint64_t *empty = full + STAGES;
  uint64_t *accf = empty + STAGES;  // [2]
  uint64_t *acce = accf + 2;        // [2]
  uint64_t *drain = acce + 2;       // MMA issuer's final commit
  uint32_t *tmem_slot = (uint32_t *)(drain + 1);
  int *abort_flag = (int *)(tmem_slot + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int tiles_m = (g.M + BM - 1) / BM, tiles_n = (g.N + BN - 1) / BN;
  const int per = tiles_m * tiles_n;  // tiles per matrix
  const int ntiles = per * g.nb;

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) { mbar_init(&full[s], 1); mbar_init(&empty[s], 1); }
    for (int a = 0; a < 2; ++a) { mbar_init(&accf[a], 1); mbar_init(&acce[a], 4); }
    mbar_init(drain, 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;

  if (warp == 0) {
    if (lane == 0) {  // ---------------- TMA producer ----------------
      int s = 0;
      uint32_t ph = 0;
      int last_ph[STAGES];  // parity of the last phase each stage was loaded for (-1: never)
      for (int q = 0; q < STAGES; ++q) last_ph[q] = -1;
      for (int t = blockIdx.x; t < ntiles && !*(volatile int *)abort_flag; t += gridDim.x) {
        const int b = t / per, tt = t % per;
        const int mt = tt / tiles_n, nt = tt % tiles_n;
        for (int kb = 0; kb < g.nk; ++kb) {
          if (!mbar_wait(&empty[s], ph ^ 1, g.wait_cap)) { fail_all(g); *(volatile int *)abort_flag = 1; break; }
          mbar_expect_tx(&full[s], STAGE_BYTES);
          unsigned char *st = base + s * STAGE_BYTES;
          for (int p = 0; p < 4; ++p) tma_load_3d(st + p * TILE_BYTES, &mapA, &full[s], kb * BK, mt * BM, 4 * b + p);
          for (int p = 0; p < 4; ++p)
            tma_load_3d(st + (4 + p) * TILE_BYTES, &mapB, &full[s], kb * BK, nt * BN, 4 * b + p);
          last_ph[s] = (int)ph;
          if (++s == STAGES) { s = 0; ph ^= 1; }
        }
      }
      // Copies still in flight land before the shared memory is released (bounded).
      for (int q = 0; q < STAGES; ++q)
        if (last_ph[q] >= 0 && !mbar_wait(&full[q], (uint32_t)last_ph[q])) fail_all(g);
    }
  } else if (warp == 1) {
    if (lane == 0) {  // ---------------- MMA issuer ----------------
      int s = 0;
      uint32_t ph = 0;
      int local = 0;
      const uint32_t id_pos = idesc_tf32(false), id_neg = idesc_tf32(true);
      for (int t = blockIdx.x; t < ntiles && !*(volatile int *)abort_flag; t += gridDim.x, ++local) {
        const int ab = local & 1;
        const uint32_t aph = (local >> 1) & 1;
        if (!mbar_wait(&acce[ab], aph ^ 1, g.wait_cap)) { fail_all(g); *(volatile int *)abort_flag = 1; break; }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t dr = tmem + ab * 256, di = dr + 128;
        bool ok = true;
        for (int kb = 0; kb < g.nk; ++kb) {
          if (!mbar_wait(&full[s], ph, g.wait_cap)) { ok = false; break; }
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          unsigned char *st = base + s * STAGE_BYTES;
          for (int ks = 0; ks < BK / KSUB; ++ks) {
            const int off = ks * KSUB * 4;  // 32 bytes per 8-deep slice inside the 64-byte row
            const uint64_t ahr = sdesc(st + 0 * TILE_BYTES + off), alr = sdesc(st + 1 * TILE_BYTES + off);
            const uint64_t ahi = sdesc(st + 2 * TILE_BYTES + off), ali = sdesc(st + 3 * TILE_BYTES + off);
            const uint64_t bhr = sdesc(st + 4 * TILE_BYTES + off), blr = sdesc(st + 5 * TILE_BYTES + off);
            const uint64_t bhi = sdesc(st + 6 * TILE_BYTES + off), bli = sdesc(st + 7 * TILE_BYTES + off);
            const uint32_t first = (kb == 0 && ks == 0) ? 0u : 1u;
            mma_tf32(dr, ahr, bhr, id_pos, first);
            mma_tf32(dr, ahr, blr, id_pos, 1);
            mma_tf32(dr, alr, bhr, id_pos, 1);
            mma_tf32(dr, ahi, bhi, id_neg, 1);
            mma_tf32(dr, ahi, bli, id_neg, 1);
            mma_tf32(dr, ali, bhi, id_neg, 1);
            mma_tf32(di, ahr, bhi, id_pos, first);
            mma_tf32(di, ahr, bli, id_pos, 1);
            mma_tf32(di, alr, bhi, id_pos, 1);
            mma_tf32(di, ahi, bhr, id_pos, 1);
            mma_tf32(di, ahi, blr, id_pos, 1);
            mma_tf32(di, ali, bhr, id_pos, 1);
          }
          mma_commit(&empty[s]);  // stage s free once these MMAs have read it
          if (++s == STAGES) { s = 0; ph ^= 1; }
        }
        if (!ok) { fail_all(g); *(volatile int *)abort_flag = 1; break; }
        mma_commit(&accf[ab]);    // accumulators ready for the epilogue
      }
      // Every MMA this thread issued completes before the accumulators are freed (bounded).
      mma_commit(drain);
      if (!mbar_wait(drain, 0)) fail_all(g);
    }
  } else {  // ---------------- epilogue: warps 2..5 ----------------
    const int lg = warp & 3;             // TMEM lane group this warp may access
    const int row_in_tile = lg * 32 + lane;
    int local = 0;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x, ++local) {
      const int ab = local & 1;
      const uint32_t aph = (local >> 1) & 1;
      // decisions uniform over the 4 epilogue warps: tcgen05.ld needs whole warps and the
      // staging tile's named barrier needs all 128 threads
      if (epi_any(*(volatile int *)abort_flag != 0)) break;
      if (!epi_all(mbar_wait(&accf[ab], aph, g.wait_cap))) {
        if (threadIdx.x == 64) { fail_all(g); *(volatile int *)abort_flag = 1; }
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const int b = t / per, tt = t % per;
      const int mt = tt / tiles_n, nt = tt % tiles_n;
      const int r = mt * BM + row_in_tile;
      float *Cr = g.Cr + b * g.ms, *Ci = g.Ci + b * g.ms;
      const uint32_t trow = tmem + ((uint32_t)(lg * 32) << 16) + ab * 256;
      for (int ch = 0; ch < BN / 32; ++ch) {
        float vr[32], vi[32];
        tmem_ld32(trow + ch * 32, vr);
        tmem_ld32(trow + 128 + ch * 32, vi);
        const int c = nt * BN + ch * 32;
        if (g.tma_epi) {
          // -D into the staging tile (128-byte swizzle: 16-byte chunk q of row r at q ^ (r & 7)),
          // then one thread adds it to C in L2 with a TMA reduce per plane.
          if (threadIdx.x == 64) asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
          asm volatile("bar.sync 1, 128;" ::: "memory");  // staging free (previous reduce has read it)
          float4 *sr = reinterpret_cast<float4 *>(epi + row_in_tile * 128);
          float4 *si = reinterpret_cast<float4 *>(epi + BM * 128 + row_in_tile * 128);
#pragma unroll
          for (int q = 0; q < 8; ++q) {
            const int pq = q ^ (row_in_tile & 7);
            sr[pq] = make_float4(-vr[4 * q], -vr[4 * q + 1], -vr[4 * q + 2], -vr[4 * q + 3]);
            si[pq] = make_float4(-vi[4 * q], -vi[4 * q + 1], -vi[4 * q + 2], -vi[4 * q + 3]);
          }
          asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
          asm volatile("bar.sync 1, 128;" ::: "memory");
          if (threadIdx.x == 64) {
            const int x = g.n0 + c, y = g.m0 + mt * BM;
            asm volatile(
                "cp.reduce.async.bulk.tensor.3d.global.shared::cta.add.tile.bulk_group [%0, {%2, %3, %4}], [%1];" ::"l"(
                    &mapCr),
                "r"(smem_u32(epi)), "r"(x), "r"(y), "r"(b)
                : "memory");
            asm volatile(
                "cp.reduce.async.bulk.tensor.3d.global.shared::cta.add.tile.bulk_group [%0, {%2, %3, %4}], [%1];" ::"l"(
                    &mapCi),
                "r"(smem_u32(epi + BM * 128)), "r"(x), "r"(y), "r"(b)
                : "memory");
            asm volatile("cp.async.bulk.commit_group;" ::: "memory");
          }
        } else if (r < g.M) {
          float *pr = Cr + (long long)(g.m0 + r) * g.ldc + g.n0 + c;
          float *pi = Ci + (long long)(g.m0 + r) * g.ldc + g.n0 + c;
          if (c + 32 <= g.N && (((uintptr_t)pr | (uintptr_t)pi) & 15) == 0) {
#pragma unroll
            for (int q = 0; q < 8; ++q) {
              float4 a = reinterpret_cast<float4 *>(pr)[q], b = reinterpret_cast<float4 *>(pi)[q];
              a.x -= vr[4 * q]; a.y -= vr[4 * q + 1]; a.z -= vr[4 * q + 2]; a.w -= vr[4 * q + 3];
              b.x -= vi[4 * q]; b.y -= vi[4 * q + 1]; b.z -= vi[4 * q + 2]; b.w -= vi[4 * q + 3];
              reinterpret_cast<float4 *>(pr)[q] = a;
              reinterpret_cast<float4 *>(pi)[q] = b;
            }
          } else {
            for (int q = 0; q < 32; ++q)
              if (c + q < g.N) { pr[q] -= vr[q]; pi[q] -= vi[q]; }
          }
        }
      }
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      __syncwarp();
      if (lane == 0) mbar_arrive(&acce[ab]);
    }
    // the reduces complete (and stop reading the staging tile) before the CTA exits
    if (threadIdx.x == 64) asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 1) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS));
  }
}

__device__ __forceinline__ float tf32_rna(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

// A planes [nb][4][M][KP]: rows r of L21 (matrix rows m0 + r, columns k0 .. k0+K-1).
__global__ void k_split_a(const float *__restrict__ Ar0, const float *__restrict__ Ai0, long long ld, long long ms,
                          int m0, int M, int k0, int K, int KP, float *__restrict__ out0) {
  const float *Ar = Ar0 + blockIdx.y * ms, *Ai = Ai0 + blockIdx.y * ms;
  float *out = out0 + (long long)blockIdx.y * 4 * M * KP;
  const long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (idx >= (long long)M * KP) return;
  const int r = (int)(idx / KP), k = (int)(idx % KP);
  float xr = 0.f, xi = 0.f;
  if (k < K) {
    xr = Ar[(long long)(m0 + r) * ld + k0 + k];
    xi = Ai[(long long)(m0 + r) * ld + k0 + k];
  }
  const float hr = tf32_rna(xr), hi = tf32_rna(xi);
  const long long pl = (long long)M * KP;
  out[idx] = hr;
  out[pl + idx] = tf32_rna(xr - hr);
  out[2 * pl + idx] = hi;
  out[3 * pl + idx] = tf32_rna(xi - hi);
}

// B planes [nb][4][N][KP]: B[n][k] = U12[k][n] (matrix rows k0 + k, columns n0 + n).
__global__ void k_split_b(const float *__restrict__ Ar0, const float *__restrict__ Ai0, long long ld, long long ms,
                          int k0, int K, int n0, int N, int KP, float *__restrict__ out0) {
  __shared__ float tr[32][33], ti[32][33];
  const float *Ar = Ar0 + blockIdx.z * ms, *Ai = Ai0 + blockIdx.z * ms;
  float *out = out0 + (long long)blockIdx.z * 4 * N * KP;
  const int nb = blockIdx.x * 32, kb = blockIdx.y * 32;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 32 x 8
  for (int y = ty; y < 32; y += 8) {
    const int k = kb + y, n = nb + tx;
    const bool v = k < K && n < N;
    tr[y][tx] = v ? Ar[(long long)(k0 + k) * ld + n0 + n] : 0.f;
    ti[y][tx] = v ? Ai[(long long)(k0 + k) * ld + n0 + n] : 0.f;
  }
  __syncthreads();
  const long long pl = (long long)N * KP;
  for (int y = ty; y < 32; y += 8) {
    const int n = nb + y, k = kb + tx;
    if (n >= N || k >= KP) continue;
    const float xr = tr[tx][y], xi = ti[tx][y];
    const float hr = tf32_rna(xr), hi = tf32_rna(xi);
    const long long o = (long long)n * KP + k;
    out[o] = hr;
    out[pl + o] = tf32_rna(xr - hr);
    out[2 * pl + o] = hi;
    out[3 * pl + o] = tf32_rna(xi - hi);
  }
}

std::atomic<PFN_cuTensorMapEncodeTiled_v12000> g_encode{nullptr};

int get_encoder() {
  if (g_encode.load(std::memory_order_acquire)) return 0;
  cudaDriverEntryPointQueryResult q;
  void *fn = nullptr;
  if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
      q != cudaDriverEntryPointSuccess || !fn) {
    pss_set_error("cuTensorMapEncodeTiled unavailable");
    return -3;
  }
  g_encode.store((PFN_cuTensorMapEncodeTiled_v12000)fn, std::memory_order_release);
  return 0;
}

// C plane of every matrix of the batch for the reduce-add epilogue: columns [0, cols),
// rows [0, rows), matrix z; 32 x 128 boxes with the 128-byte swizzle of the staging tile.
int make_cmap(CUtensorMap *m, const float *c, long long ld, long long ms, int rows, int cols, int nb) {
  cuuint64_t dims[3] = {(cuuint64_t)cols, (cuuint64_t)rows, (cuuint64_t)nb};
  cuuint64_t strides[2] = {(cuuint64_t)ld * 4, (cuuint64_t)(nb > 1 ? ms : ld * rows) * 4};
  cuuint32_t box[3] = {32, BM, 1};
  cuuint32_t es[3] = {1, 1, 1};
  CUresult r = g_encode.load(std::memory_order_acquire)(
      m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, (void *)c, dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
      CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    pss_set_error("cuTensorMapEncodeTiled (C) failed (%d)", (int)r);
    return -3;
  }
  return 0;
}

int make_map(CUtensorMap *m, const float *planes, int rows, int KP, int nplanes) {
  cuuint64_t dims[3] = {(cuuint64_t)KP, (cuuint64_t)rows, (cuuint64_t)nplanes};
  cuuint64_t strides[2] = {(cuuint64_t)KP * 4, (cuuint64_t)rows * KP * 4};
  cuuint32_t box[3] = {BK, BM, 1};
  cuuint32_t es[3] = {1, 1, 1};
  CUresult r = g_encode.load(std::memory_order_acquire)(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, (void *)planes, dims, strides, box, es,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    pss_set_error("cuTensorMapEncodeTiled failed (%d)", (int)r);
    return -3;
  }
  return 0;
}

constexpr int kMaxDevices = 64;
int g_num_sms[kMaxDevices] = {};  // per device, written once under g_setup
DeviceOnce g_setup;
std::atomic<long long> g_wait_cap{kWaitCap};  // pss_set_wait_limit

}  // namespace

extern "C" int pss_set_wait_limit(int64_t iterations) {
  if (iterations < 0) { pss_set_error("wait limit must be >= 0"); return -1; }
  g_wait_cap.store(iterations == 0 ? kWaitCap : (long long)iterations, std::memory_order_relaxed);
  return 0;
}

// Workspace for the split operands of a batch of nb updates with up to Mmax rows / Nmax
// columns, K <= KP.
size_t pss_tc_ws_bytes(int Mmax, int Nmax, int KP, int nb) {
  return 4 * sizeof(float) * ((size_t)Mmax * KP + (size_t)Nmax * KP) * nb + 1024;
}

// For each matrix b < nb (at Ar/Ai + b*ms):
// C[m0:m0+M, n0:n0+N] -= A[m0:m0+M, k0:k0+K] * A[k0:k0+K, n0:n0+N] on FP32 planes.
int pss_cgemm_tc(float *Ar, float *Ai, long long ld, long long ms, int nb, int m0, int M, int n0, int N, int k0,
                 int K, void *ws, size_t ws_bytes, int *err, cudaStream_t st) {
  if (M <= 0 || N <= 0 || K <= 0 || nb <= 0) return 0;
  const int KP = ((K + BK - 1) / BK) * BK;
  if (ws_bytes < pss_tc_ws_bytes(M, N, KP, nb)) { pss_set_error("tensor-core GEMM workspace too small"); return -4; }
  if (get_encoder()) return -3;
  int dev = 0;
  PSS_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) { pss_set_error("device %d out of range", dev); return -3; }
  if (int rc = device_once(g_setup, [dev] {
        int nsm = 0;
        PSS_CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
        PSS_CUDA_TRY(cudaFuncSetAttribute(k_cgemm_tf32x3, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES));
        g_num_sms[dev] = nsm;
        return 0;
      }))
    return rc;
  float *pa = (float *)(((uintptr_t)ws + 255) & ~(uintptr_t)255);
  float *pb = pa + 4 * (size_t)M * KP * nb;
  pb = (float *)(((uintptr_t)pb + 255) & ~(uintptr_t)255);
  pss_count_launch();
  k_split_a<<<dim3(cdiv_u((long long)M * KP, 256), nb), 256, 0, st>>>(Ar, Ai, ld, ms, m0, M, k0, K, KP, pa);
  pss_count_launch();
  k_split_b<<<dim3(cdiv_u(N, 32), cdiv_u(KP, 32), nb), 256, 0, st>>>(Ar, Ai, ld, ms, k0, K, n0, N, KP, pb);
  CUtensorMap ma, mb, mcr, mci;
  if (make_map(&ma, pa, M, KP, 4 * nb) || make_map(&mb, pb, N, KP, 4 * nb)) return -3;
  // TMA reduce-add epilogue when every box start and stride is 16-byte aligned
  const bool tma_epi = ld % 4 == 0 && (nb == 1 || ms % 4 == 0) && n0 % 4 == 0 &&
                       (((uintptr_t)Ar | (uintptr_t)Ai) & 15) == 0;
  if (tma_epi) {
    if (make_cmap(&mcr, Ar, ld, ms, m0 + M, n0 + N, nb) || make_cmap(&mci, Ai, ld, ms, m0 + M, n0 + N, nb)) return -3;
  } else {
    mcr = mci = ma;  // not read
  }
  GemmArgs g{Ar, Ai, ld, ms, m0, n0, M, N, KP / BK, nb, err, tma_epi ? 1 : 0,
             g_wait_cap.load(std::memory_order_relaxed)};
  const int tiles = ((M + BM - 1) / BM) * ((N + BN - 1) / BN) * nb;
  const int grid = std::min(tiles, g_num_sms[dev]);
  const int tok = pss_prof_begin(st);
  pss_count_launch();
  k_cgemm_tf32x3<<<grid, 192, SMEM_BYTES, st>>>(ma, mb, mcr, mci, g);
  pss_prof_end(tok, st, PSS_PROF_TC_UPDATE, 8.0 * nb * M * (double)N * K);
  PSS_CUDA_TRY(cudaGetLastError());
  return 0;
}
