// Unique face-pair classes of a sheet on the device: the O(nface^2) classing of setup_rwg
// (src/RWG.jl:287-319).  Pair (match face m, source face n) is keyed by the source face's
// shape class and the offset of the match centroid from the source's first vertex, both
// quantised on the grid g the host chooses (the reference's KD-tree radius, 1e-6 of the
// distance between the first two centroids); equal keys are translation-equivalent pairs.
// Classes are numbered in the order of their first member in column-major (match fastest)
// order, as the reference numbers them.
//
//   k_ufp_insert  one thread per pair: the key into an open-addressing hash table (slot state
//                 claimed by atomicCAS, key words written, then published), the pair's index
//                 folded into the slot's first member with atomicMin; each pair's slot kept;
//   k_ufp_flag    1 where a pair is its class's first member;
//   k_scan_*      exclusive prefix sum of the flags (block sums, one pass over them, block scan
//                 plus offset): the class number of every first member;
//   k_ufp_assign  every pair's class = the number of its class's first member; the
//                 representatives' indices.
// Every wait is bounded (an insertion that would wait on a slot too long, or a table that
// fills, reports an error and the host grows the table or gives up).
#include <climits>
#include <vector>

#include "pss_internal.cuh"

namespace {

constexpr int kScanBlock = 1024;  // flags per CTA of the scan (256 threads x 4)
constexpr int kSpin = 1 << 20;
constexpr int kMaxProbe = 4096;  // a longer probe sequence means the table is (nearly) full

__device__ __forceinline__ unsigned long long mix64(unsigned long long x) {
  x ^= x >> 33;
  x *= 0xff51afd7ed558ccdULL;
  x ^= x >> 33;
  x *= 0xc4ceb9fe1a85ec53ULL;
  x ^= x >> 33;
  return x;
}

struct UfpTable {
  unsigned long long *w0, *w1;  // key words: dx, and (shape << 32) | (uint32) dy
  int *state;                   // 0 empty, 1 being written, 2 published
  long long *first;             // smallest column-major pair index of the class
  unsigned long long mask;      // capacity - 1 (a power of two)
};

__global__ void k_ufp_insert(long long nface, const double *__restrict__ cen, const double *__restrict__ r1,
                             const long long *__restrict__ shape, double g, UfpTable T, int *__restrict__ slot_of,
                             int *__restrict__ err) {
  const long long npairs = nface * nface;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < npairs;
       p += (long long)gridDim.x * blockDim.x) {
    const long long m = p % nface, n = p / nface;
    const long long dx = (long long)rint((cen[2 * m] - r1[2 * n]) / g);
    const long long dy = (long long)rint((cen[2 * m + 1] - r1[2 * n + 1]) / g);
    const unsigned long long k0 = (unsigned long long)dx;
    const unsigned long long k1 = ((unsigned long long)(unsigned int)shape[n] << 32) | (unsigned int)dy;
    unsigned long long s = mix64(k0 ^ mix64(k1)) & T.mask;
    bool done = false;
    for (int probe = 0; probe < kMaxProbe && !done; ++probe, s = (s + 1) & T.mask) {
      const int st = atomicCAS(&T.state[s], 0, 1);
      if (st == 0) {  // claimed an empty slot: write the key, then publish it
        T.w0[s] = k0;
        T.w1[s] = k1;
        __threadfence();
        atomicExch(&T.state[s], 2);
        atomicMin(&T.first[s], p);
        slot_of[p] = (int)s;
        done = true;
        break;
      }
      int spins = 0;
      while (atomicAdd(&T.state[s], 0) == 1 && ++spins < kSpin) {
      }
      if (spins >= kSpin) { atomicExch(err, 2); return; }
      __threadfence();
      if (((volatile unsigned long long *)T.w0)[s] == k0 && ((volatile unsigned long long *)T.w1)[s] == k1) {
        atomicMin(&T.first[s], p);
        slot_of[p] = (int)s;
        done = true;
      }
    }
    if (!done) { atomicExch(err, 1); return; }  // table full
  }
}

__global__ void k_ufp_flag(long long npairs, const int *__restrict__ slot_of, const long long *__restrict__ first,
                           int *__restrict__ flag) {
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < npairs;
       p += (long long)gridDim.x * blockDim.x)
    flag[p] = first[slot_of[p]] == p;
}

// exclusive scan, phase 1: the sum of each block of kScanBlock flags
__global__ void __launch_bounds__(256) k_scan_sums(long long n, const int *__restrict__ in, long long *__restrict__ bsum) {
  __shared__ long long red[256];
  const long long base = (long long)blockIdx.x * kScanBlock;
  long long s = 0;
  for (int q = 0; q < 4; ++q) {
    const long long i = base + threadIdx.x * 4 + q;
    if (i < n) s += in[i];
  }
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) bsum[blockIdx.x] = red[0];
}

// phase 2: exclusive scan of the block sums in one CTA (chunks of 256, carried), and the total
__global__ void __launch_bounds__(256) k_scan_blocks(long long nb, long long *__restrict__ bsum, long long *__restrict__ total) {
  __shared__ long long buf[256];
  __shared__ long long carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (long long c0 = 0; c0 < nb; c0 += 256) {
    const long long i = c0 + threadIdx.x;
    const long long v = i < nb ? bsum[i] : 0;
    buf[threadIdx.x] = v;
    __syncthreads();
    for (int o = 1; o < 256; o <<= 1) {  // inclusive Hillis-Steele scan
      const long long t = threadIdx.x >= o ? buf[threadIdx.x - o] : 0;
      __syncthreads();
      buf[threadIdx.x] += t;
      __syncthreads();
    }
    if (i < nb) bsum[i] = carry + buf[threadIdx.x] - v;
    __syncthreads();
    if (threadIdx.x == 255) carry += buf[255];
    __syncthreads();
  }
  if (threadIdx.x == 0) *total = carry;
}

// phase 3: exclusive scan inside each block plus the block's offset
__global__ void __launch_bounds__(256) k_scan_apply(long long n, const int *__restrict__ in, const long long *__restrict__ bsum,
                                                    long long *__restrict__ out) {
  __shared__ long long buf[256];
  const long long base = (long long)blockIdx.x * kScanBlock;
  int v[4];
  long long s = 0;
  for (int q = 0; q < 4; ++q) {
    const long long i = base + threadIdx.x * 4 + q;
    v[q] = i < n ? in[i] : 0;
    s += v[q];
  }
  buf[threadIdx.x] = s;
  __syncthreads();
  for (int o = 1; o < 256; o <<= 1) {
    const long long t = threadIdx.x >= o ? buf[threadIdx.x - o] : 0;
    __syncthreads();
    buf[threadIdx.x] += t;
    __syncthreads();
  }
  long long run = bsum[blockIdx.x] + buf[threadIdx.x] - s;
  for (int q = 0; q < 4; ++q) {
    const long long i = base + threadIdx.x * 4 + q;
    if (i < n) out[i] = run;
    run += v[q];
  }
}

__global__ void k_ufp_assign(long long npairs, const int *__restrict__ slot_of, const long long *__restrict__ first,
                             const int *__restrict__ flag, const long long *__restrict__ rank, int *__restrict__ ufpm,
                             long long *__restrict__ rep, long long rep_cap) {
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < npairs;
       p += (long long)gridDim.x * blockDim.x) {
    ufpm[p] = (int)(rank[first[slot_of[p]]] + 1);
    if (flag[p] && rank[p] < rep_cap) rep[rank[p]] = p + 1;
  }
}

struct Buf {
  void *p = nullptr;
  ~Buf() {
    if (p) cudaFree(p);
  }
};

}  // namespace

extern "C" int pss_face_pair_classes(pss_ctx *ctx, int64_t nface, const double *cen, const double *r1,
                                     const int64_t *shape, double g, int32_t *ufpm, int64_t *rep, int64_t rep_cap,
                                     int64_t *nufp_out) {
  if (!ctx || !cen || !r1 || !shape || !ufpm || !rep || !nufp_out || nface <= 0 || !(g > 0) || rep_cap <= 0) {
    pss_set_error("invalid argument");
    return -1;
  }
  if (nface > 16384) {
    pss_set_error("face-pair classing on the device takes at most 16384 faces (%lld given)", (long long)nface);
    return -1;
  }
  for (int64_t f = 0; f < nface; ++f)
    if (shape[f] < 0 || shape[f] > INT_MAX) { pss_set_error("shape class out of range"); return -1; }
  int dev = 0;
  if (pss_ctx_device(ctx, &dev)) return -1;
  PSS_CUDA_TRY(cudaSetDevice(dev));
  const long long npairs = (long long)nface * nface;
  const long long nblk = (npairs + kScanBlock - 1) / kScanBlock;
  Buf dcen, dr1, dshape, dslot, dflag, drank, dbsum, dtot, dufpm, drep, derr;
  PSS_CUDA_TRY(cudaMalloc(&dcen.p, 2 * nface * sizeof(double)));
  PSS_CUDA_TRY(cudaMalloc(&dr1.p, 2 * nface * sizeof(double)));
  PSS_CUDA_TRY(cudaMalloc(&dshape.p, nface * sizeof(long long)));
  PSS_CUDA_TRY(cudaMalloc(&dslot.p, npairs * sizeof(int)));
  PSS_CUDA_TRY(cudaMalloc(&dflag.p, npairs * sizeof(int)));
  PSS_CUDA_TRY(cudaMalloc(&drank.p, npairs * sizeof(long long)));
  PSS_CUDA_TRY(cudaMalloc(&dbsum.p, nblk * sizeof(long long)));
  PSS_CUDA_TRY(cudaMalloc(&dtot.p, sizeof(long long)));
  PSS_CUDA_TRY(cudaMalloc(&dufpm.p, npairs * sizeof(int)));
  PSS_CUDA_TRY(cudaMalloc(&drep.p, rep_cap * sizeof(long long)));
  PSS_CUDA_TRY(cudaMalloc(&derr.p, sizeof(int)));
  PSS_CUDA_TRY(cudaMemcpy(dcen.p, cen, 2 * nface * sizeof(double), cudaMemcpyHostToDevice));
  PSS_CUDA_TRY(cudaMemcpy(dr1.p, r1, 2 * nface * sizeof(double), cudaMemcpyHostToDevice));
  PSS_CUDA_TRY(cudaMemcpy(dshape.p, shape, nface * sizeof(long long), cudaMemcpyHostToDevice));
  // the table: the power of two at or above twice the pairs (every key fits at a load of at
  // most one half, whatever the sheet's symmetry: a structured meander has a class for
  // every 2.5 pairs, a perturbed one nearly one per pair), at most 2^28 slots (7.5 GB)
  unsigned long long cap = 1ull << 20;
  while (cap < 2ull * (unsigned long long)npairs && cap < (1ull << 28)) cap <<= 1;
  {
    Buf w0, w1, state, first;
    PSS_CUDA_TRY(cudaMalloc(&w0.p, cap * sizeof(unsigned long long)));
    PSS_CUDA_TRY(cudaMalloc(&w1.p, cap * sizeof(unsigned long long)));
    PSS_CUDA_TRY(cudaMalloc(&state.p, cap * sizeof(int)));
    PSS_CUDA_TRY(cudaMalloc(&first.p, cap * sizeof(long long)));
    PSS_CUDA_TRY(cudaMemset(state.p, 0, cap * sizeof(int)));
    PSS_CUDA_TRY(cudaMemset(first.p, 0x7f, cap * sizeof(long long)));  // 0x7f7f...: above any pair index
    PSS_CUDA_TRY(cudaMemset(derr.p, 0, sizeof(int)));
    UfpTable T{(unsigned long long *)w0.p, (unsigned long long *)w1.p, (int *)state.p, (long long *)first.p, cap - 1};
    const int grid = (int)std::min<long long>((npairs + 255) / 256, 148LL * 16);
    pss_count_launch();
    k_ufp_insert<<<grid, 256>>>(nface, (const double *)dcen.p, (const double *)dr1.p, (const long long *)dshape.p, g,
                                T, (int *)dslot.p, (int *)derr.p);
    int herr = 0;
    PSS_CUDA_TRY(cudaMemcpy(&herr, derr.p, sizeof(int), cudaMemcpyDeviceToHost));
    if (herr) {
      pss_set_error("face-pair class table %s", herr == 1 ? "overflowed" : "insertion did not settle");
      return -3;
    }
    pss_count_launch();
    k_ufp_flag<<<grid, 256>>>(npairs, (const int *)dslot.p, (const long long *)first.p, (int *)dflag.p);
    pss_count_launch();
    k_scan_sums<<<(unsigned)nblk, 256>>>(npairs, (const int *)dflag.p, (long long *)dbsum.p);
    pss_count_launch();
    k_scan_blocks<<<1, 256>>>(nblk, (long long *)dbsum.p, (long long *)dtot.p);
    pss_count_launch();
    k_scan_apply<<<(unsigned)nblk, 256>>>(npairs, (const int *)dflag.p, (const long long *)dbsum.p,
                                          (long long *)drank.p);
    pss_count_launch();
    k_ufp_assign<<<grid, 256>>>(npairs, (const int *)dslot.p, (const long long *)first.p, (const int *)dflag.p,
                                (const long long *)drank.p, (int *)dufpm.p, (long long *)drep.p, rep_cap);
    PSS_CUDA_TRY(cudaGetLastError());
    long long nufp = 0;
    PSS_CUDA_TRY(cudaMemcpy(&nufp, dtot.p, sizeof(long long), cudaMemcpyDeviceToHost));
    *nufp_out = nufp;
    if (nufp > rep_cap) {
      pss_set_error("%lld classes, more than the %lld representatives the caller has room for", nufp,
                    (long long)rep_cap);
      return -5;
    }
    PSS_CUDA_TRY(cudaMemcpy(ufpm, dufpm.p, npairs * sizeof(int), cudaMemcpyDeviceToHost));
    PSS_CUDA_TRY(cudaMemcpy(rep, drep.p, nufp * sizeof(long long), cudaMemcpyDeviceToHost));
    return 0;
  }
}
