// Singlet Gram of the batched Krylov basis on the 5th-generation tensor cores
// (tcgen05, accumulators in tensor memory): the projected Gram V^H P_S V that
// the reference forms per basis (rpm_statevector_engine.py:521-529) and the
// batched step uses for the populations at the observation points.
//
// G_kl = sum_q conj(a_k(q)) a_l(q), a_k(q) = (V_k[Q + q] - V_k[2Q + q]) / sqrt 2
// (Q = n / 4: the two singlet-carrying electron blocks), as a real product:
// X is 128 x K with row k = Re d_k and row 64 + k = Im d_k (d = V_k[Q + .] -
// V_k[2Q + .], rows >= M zero); C = X X^T; G = (C_rr + C_ii, C_ri - C_ir) / 2.
// Precision: X = Xh + Xl with Xh the TF32 rounding of X; C ~ Xh Xh^T + Xh Xl^T
// + Xl Xh^T (three TF32 MMAs per K step: products to about 2^-22).  The
// tensor cores' FP32 accumulation rounds towards zero, a bias that grows with
// the number of accumulating MMAs (about 1e-6 relative after 48 of them), so
// the large term Xh Xh^T and the two small ones go to separate accumulators
// that are drained into FP64 sums after every 32-row chunk (four accumulating
// MMAs on the large term).
//
// One CTA per (trajectory, row range), the same grid and partial-sum layout as
// the CUDA-core kernel k_b_gram (batched.cu).  Roles (12 warps):
//   warp 11      loader: two 2-D tensor copies per chunk (the 32-row segments
//                of both singlet-carrying electron blocks of every basis
//                vector) into a raw stage (3 stages, mbarrier tx counts)
//   warps 6-9    transform: d = p1 - p2, TF32 split, stores into the K-major
//                no-swizzle operand tiles (2 stages of hi + lo)
//   warp 10      MMA: three tcgen05.mma (M = N = 128, K = 8) per K step, four
//                K steps per 32-row chunk; per chunk a pair of accumulators
//                (large, small terms), double-buffered in TMEM (512 columns)
//   warps 0-5    epilogue: tcgen05.ld of the finished accumulator, FP64 sums;
//                warps 0/1 C_rr rows, 2/3 C_ii rows, 4/5 C_ri rows
// Every wait is bounded; on a timeout the kernel raises the sticky status word
// and every role leaves its loop.
#pragma once
// Included by batched.cu after the definitions of TrajState and BatchDev.
#include "common.cuh"
#include "ptx.cuh"

namespace rpm {

namespace gramtc {

using namespace ptx;

constexpr int kGC = 32;          // rows (q) per chunk
constexpr int kRawStages = 3;
constexpr int kTileStages = 2;
constexpr int kMaxBasis = 64;    // basis vectors (rows of X per real part)
constexpr int kRawBytes = kMaxBasis * 2 * kGC * 8;       // 32 KiB: [half][k][32 q] float2
constexpr int kTileBytes = 128 * kGC * 4;                // 16 KiB: one 128 x 32 TF32 operand
constexpr int kSbo = (kGC / 4) * 128;                    // 1024: next group of 8 rows
constexpr int kLbo = 128;                                // next 4-column (16-byte) core matrix
constexpr int kSmemBytes = kRawStages * kRawBytes + kTileStages * 2 * kTileBytes + 1024;
constexpr int kThreads = 12 * 32;
constexpr int kTmemCols = 512;   // two buffers of two 128-column FP32 accumulators
constexpr int kCombLd = 65;      // padded rows of the final combine buffers

// Instruction descriptor of tcgen05.mma kind::tf32: D F32, A and B TF32,
// both K-major, N = 128 (bits 17-22: N / 8), M = 128 (bits 24-28: M / 16).
constexpr unsigned kIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((128u >> 3) << 17) | ((128u >> 4) << 24);

// Shared-memory matrix descriptor: K-major, no swizzle, version 1.
__device__ __forceinline__ unsigned long long smem_desc(unsigned addr) {
  return (unsigned long long)((addr & 0x3FFFFu) >> 4) | ((unsigned long long)(kLbo >> 4) << 16) |
         ((unsigned long long)(kSbo >> 4) << 32) | (1ull << 46);
}

// Byte offset of element (row r, column kk) of a 128 x 32 TF32 operand tile.
__host__ __device__ constexpr int tile_offset(int r, int kk) {
  return (r >> 3) * kSbo + (kk >> 2) * kLbo + (r & 7) * 16 + (kk & 3) * 4;
}

__device__ __forceinline__ unsigned tf32_rna(float x) {
  unsigned r;
  asm("cvt.rna.tf32.f32 %0, %1;\n" : "=r"(r) : "f"(x));
  return r;
}

__device__ __forceinline__ void tma_2d(void* dst, const CUtensorMap* map, int x, int y, unsigned long long* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];\n"
      ::"r"(smem_u32(dst)), "l"(map), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }

__device__ __forceinline__ void tc_mma(unsigned d_tmem, unsigned long long a, unsigned long long b, bool accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}\n" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(kIdesc), "r"(accumulate ? 1 : 0)
      : "memory");
}
// The mbarrier completes once every tcgen05 operation this thread issued before has completed.
__device__ __forceinline__ void tc_commit(unsigned long long* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(smem_u32(bar))
               : "memory");
}
// Two 16-column loads of this warp's lanes, then one wait for both.
__device__ __forceinline__ void tc_ld16x2(unsigned ta, unsigned tb, float (&va)[16], float (&vb)[16]) {
  unsigned r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(ta)
      : "memory");
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];\n"
      : "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(tb)
      : "memory");
  asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) {
    va[i] = __uint_as_float(r[i]);
    vb[i] = __uint_as_float(r[16 + i]);
  }
}

// Bounded wait shared by the roles; false once the status word is raised.
__device__ __forceinline__ bool wait(unsigned long long* bar, unsigned parity, int* status) {
  return mbar_wait(bar, parity, status);
}
// Bounded wait that ignores the status word: copies and MMAs already issued
// complete before shared or tensor memory is released.
__device__ __forceinline__ void wait_quiet(unsigned long long* bar, unsigned parity) {
  const long long t0 = clock64();
  while (!mbar_test(bar, parity))
    if (clock64() - t0 > kWaitCycles) return;
}

// vmap: basis_rows_map of the basis buffer with a box of kGC elements x
// (m + 1) slots.
__global__ void __launch_bounds__(kThreads, 1) k_b_gram_tc(const __grid_constant__ CUtensorMap vmap, BatchDev B) {
  extern __shared__ unsigned char smem_raw[];
  unsigned char* base =
      reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
  unsigned char* raw = base;                              // [kRawStages][half][slot][32] float2
  unsigned char* tiles = base + kRawStages * kRawBytes;   // [kTileStages][hi, lo] operand tiles
  __shared__ __align__(8) unsigned long long raw_full[kRawStages], raw_empty[kRawStages], tile_full[kTileStages],
      tile_empty[kTileStages], acc_full[2], acc_empty[2], mma_done;
  __shared__ unsigned tmem_slot;
  const int b = blockIdx.y;
  const TrajState& s = B.st[b];
  if (s.done) return;
  const int M = s.msize;
  const long long q4 = s.n / 4;
  const long long rows_per = ((q4 + B.gblk - 1) / B.gblk + kGC - 1) / kGC * kGC;
  const long long r_begin = (long long)blockIdx.x * rows_per;
  const long long r_end = min(q4, r_begin + rows_per);
  double2* out = B.gpart + ((size_t)b * B.gblk + blockIdx.x) * kBMaxK * kBMaxK;  // compact M x M
  if (r_begin >= r_end) {
    for (int idx = threadIdx.x; idx < M * M; idx += blockDim.x) out[idx] = make_double2(0.0, 0.0);
    return;
  }
  const int nchunks = (int)((r_end - r_begin + kGC - 1) / kGC);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int* status = B.kstatus;
  if (threadIdx.x == 0) {
    for (int i = 0; i < kRawStages; ++i) {
      mbar_init(&raw_full[i], 1);
      mbar_init(&raw_empty[i], 4);
    }
    for (int i = 0; i < kTileStages; ++i) {
      mbar_init(&tile_full[i], 4);
      mbar_init(&tile_empty[i], 1);
    }
    for (int i = 0; i < 2; ++i) {
      mbar_init(&acc_full[i], 1);
      mbar_init(&acc_empty[i], 6);
    }
    mbar_init(&mma_done, 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  // operand rows >= M (real and imaginary) stay zero for the whole launch
  for (int idx = threadIdx.x; idx < kTileStages * 2 * kTileBytes / 16; idx += blockDim.x)
    reinterpret_cast<uint4*>(tiles)[idx] = make_uint4(0u, 0u, 0u, 0u);
  fence_async_smem();
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(&tmem_slot)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const unsigned tmem = tmem_slot;
  const int nslot = B.m + 1;  // basis slots per trajectory (the copy box)
  double acc[64];
#pragma unroll
  for (int i = 0; i < 64; ++i) acc[i] = 0.0;

  if (warp == 11) {
    // ------------------------------ loader ------------------------------
    int armed[kRawStages];
#pragma unroll
    for (int i = 0; i < kRawStages; ++i) armed[i] = -1;
    for (int c = 0; c < nchunks; ++c) {
      const int rs = c % kRawStages;
      if (c >= kRawStages) {
        bool ok = wait(&raw_empty[rs], (unsigned)(((c - kRawStages) / kRawStages) & 1), status);
        if (!__all_sync(0xffffffffu, ok)) break;
      }
      const long long r0 = r_begin + (long long)c * kGC;
      if (lane == 0) {
        // rows (1 + h) Q + r0 .. + 31 of slots b (m + 1) .. b (m + 1) + m, for h = 0, 1
        mbar_arrive_expect_tx(&raw_full[rs], (unsigned)(2 * nslot * kGC * 8));
        for (int h = 0; h < 2; ++h)
          tma_2d(raw + rs * kRawBytes + h * nslot * kGC * 8, &vmap, (int)((1 + h) * q4 + r0), b * nslot, &raw_full[rs]);
      }
      __syncwarp();
      armed[rs] = c;
    }
    // copies still in flight land before the CTA may exit (normally the
    // transform warps have consumed every stage already)
#pragma unroll
    for (int i = 0; i < kRawStages; ++i)
      if (armed[i] >= 0) wait_quiet(&raw_full[i], (unsigned)((armed[i] / kRawStages) & 1));
  } else if (warp >= 6 && warp <= 9) {
    // ---------------------------- transform -----------------------------
    const int tt = threadIdx.x - 6 * 32;
    for (int c = 0; c < nchunks; ++c) {
      const int rs = c % kRawStages, ts = c % kTileStages;
      bool ok = wait(&raw_full[rs], (unsigned)((c / kRawStages) & 1), status);
      if (ok && c >= kTileStages) ok = wait(&tile_empty[ts], (unsigned)(((c - kTileStages) / kTileStages) & 1), status);
      if (!__all_sync(0xffffffffu, ok)) break;
      const long long r0 = r_begin + (long long)c * kGC;
      const unsigned char* rw = raw + rs * kRawBytes;
      unsigned char* th = tiles + ts * 2 * kTileBytes;
#pragma unroll
      for (int u = 0; u < 8 * kMaxBasis / 128; ++u) {  // at most four items per thread
        const int it = tt + 128 * u;
        if (it >= 8 * M) break;
        const int k = it >> 3, g = it & 7;
        const float4* p1 = reinterpret_cast<const float4*>(rw + k * kGC * 8 + g * 32);
        const float4* p2 = reinterpret_cast<const float4*>(rw + (nslot + k) * kGC * 8 + g * 32);
        const float4 a0 = p1[0], a1 = p1[1], b0 = p2[0], b1 = p2[1];
        float re[4] = {a0.x - b0.x, a0.z - b0.z, a1.x - b1.x, a1.z - b1.z};
        float im[4] = {a0.y - b0.y, a0.w - b0.w, a1.y - b1.y, a1.w - b1.w};
        const long long qq = r0 + 4 * g;
        unsigned rh[4], rl[4], ih[4], il[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          if (qq + j >= r_end) re[j] = im[j] = 0.f;  // rows of the next range or past the vector
          rh[j] = tf32_rna(re[j]);
          ih[j] = tf32_rna(im[j]);
          rl[j] = __float_as_uint(re[j] - __uint_as_float(rh[j]));
          il[j] = __float_as_uint(im[j] - __uint_as_float(ih[j]));
        }
        *reinterpret_cast<uint4*>(th + tile_offset(k, 4 * g)) = make_uint4(rh[0], rh[1], rh[2], rh[3]);
        *reinterpret_cast<uint4*>(th + kTileBytes + tile_offset(k, 4 * g)) = make_uint4(rl[0], rl[1], rl[2], rl[3]);
        *reinterpret_cast<uint4*>(th + tile_offset(64 + k, 4 * g)) = make_uint4(ih[0], ih[1], ih[2], ih[3]);
        *reinterpret_cast<uint4*>(th + kTileBytes + tile_offset(64 + k, 4 * g)) =
            make_uint4(il[0], il[1], il[2], il[3]);
      }
      // generic-proxy stores become visible to the tensor cores' reads
      fence_async_smem();
      __syncwarp();
      if (lane == 0) {
        mbar_arrive(&raw_empty[rs]);
        mbar_arrive(&tile_full[ts]);
      }
    }
  } else if (warp == 10) {
    // -------------------------------- MMA -------------------------------
    if (lane == 0) {
      for (int c = 0; c < nchunks; ++c) {
        const int ts = c % kTileStages, a = c & 1;
        bool ok = true;
        if (c >= 2) ok = wait(&acc_empty[a], (unsigned)(((c - 2) >> 1) & 1), status);
        if (ok) ok = wait(&tile_full[ts], (unsigned)((c / kTileStages) & 1), status);
        if (!ok) break;
        tc_fence_after();
        const unsigned big = tmem + (unsigned)(a * 256), small = big + 128;
        const unsigned hi = smem_u32(tiles + ts * 2 * kTileBytes), lo = hi + kTileBytes;
#pragma unroll
        for (int ks = 0; ks < kGC / 8; ++ks) {
          const unsigned long long ah = smem_desc(hi + ks * 2 * kLbo), al = smem_desc(lo + ks * 2 * kLbo);
          tc_mma(big, ah, ah, ks > 0);
          tc_mma(small, ah, al, ks > 0);
          tc_mma(small, al, ah, true);
        }
        tc_commit(&tile_empty[ts]);
        tc_commit(&acc_full[a]);
      }
      // every MMA issued has completed before tensor memory is freed
      tc_commit(&mma_done);
      wait_quiet(&mma_done, 0u);
    }
    __syncwarp();
  } else {
    // ------------------------------ epilogue ----------------------------
    const int qd = warp & 3;
    const int col0 = warp < 2 ? 0 : 64;
    for (int c = 0; c < nchunks; ++c) {
      const int a = c & 1;
      const bool ok = wait(&acc_full[a], (unsigned)((c >> 1) & 1), status);
      if (!__all_sync(0xffffffffu, ok)) break;
      tc_fence_after();
      const unsigned row = tmem + ((unsigned)(32 * qd) << 16) + (unsigned)(a * 256 + col0);
#pragma unroll
      for (int g = 0; g < 4; ++g) {  // 16 columns of the large term and the same of the small terms
        if (16 * g < M) {            // columns >= M of each half are zero
          float vb[16], vs[16];
          tc_ld16x2(row + 16 * g, row + 128 + 16 * g, vb, vs);
          // the small terms are 2^-11 of the large one: their FP32 sum keeps both
#pragma unroll
          for (int i = 0; i < 16; ++i) acc[16 * g + i] += (double)(vb[i] + vs[i]);
        }
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&acc_empty[a]);
    }
  }

  // ------------------------- free TMEM, combine -------------------------
  __shared__ int failed;
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(kTmemCols) : "memory");
  }
  if (threadIdx.x == 0) failed = *reinterpret_cast<volatile int*>(status);
  __syncthreads();
  if (failed) return;
  // C_rr, C_ii and C_ri rows of the FP64 sums, in the (now idle) stage memory
  double* rr = reinterpret_cast<double*>(base);
  double* ii = rr + kMaxBasis * kCombLd;
  double* ri = ii + kMaxBasis * kCombLd;
  if (warp < 6) {
    const int row = 32 * (warp & 3) + lane;  // row of C
    double* dst = warp < 2 ? rr + row * kCombLd : warp < 4 ? ii + (row - 64) * kCombLd : ri + row * kCombLd;
#pragma unroll
    for (int i = 0; i < 64; ++i) dst[i] = acc[i];
  }
  __syncthreads();
  // G = (C_rr + C_ii, C_ri - C_ir) / 2 with C_ir = C_ri^T (C is symmetric)
  for (int idx = threadIdx.x; idx < M * M; idx += blockDim.x) {
    const int k = idx / M, l = idx - k * M;
    out[idx] = make_double2(0.5 * (rr[k * kCombLd + l] + ii[k * kCombLd + l]),
                            0.5 * (ri[k * kCombLd + l] - ri[l * kCombLd + k]));
  }
}

}  // namespace gramtc
}  // namespace rpm
