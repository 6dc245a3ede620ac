// Persistent Lanczos kernel: the iterations of one Krylov step for every
// trajectory of a shape group in ONE launch (the batched path's dominant
// work; the reference's per-vector loop is rpm_statevector_engine.py:651-688,
// its H psi :221-253).
//
// Work items are tiles of the two shape-specialised passes (hpsi_fast.cuh):
//   R(j, b, t): rows 16t .. 16t+15 of vector b, iteration j -- forms
//               v_j = (w'_j - alpha_{j-1} v_{j-1}) / beta_{j-1} (j > 0),
//               writes it back and writes the right-radical partial;
//   L(j, b, t): columns 8t .. 8t+7 of both electron-B halves -- applies the
//               left radical and the pair operator, adds the partial, writes
//               w'_{j+1} and reduces <v_j, w'>, |w'|^2, |v_j|^2; the last L
//               tile of (j, b) sets alpha_j, beta_j and the breakdown flags.
// One CTA per SM dequeues items from a global counter in a fixed order:
// vectors in wavefront groups of gv, each group through all iterations of
// the launch (all m, or a segment between two reorthogonalisations), every
// iteration as R tiles of the group's vectors, then their L tiles.  A phase
// of vector b starts only after the phase before it has completed on every
// CTA (per-vector progress counters); in this order an item only ever depends
// on items dequeued before it, so every wait ends, and the vectors of one
// group stay in L2 between the phases.  Every wait has a time limit, after
// which the kernel sets a sticky status word and drains.
//
// Inside a CTA one producer warp dequeues, waits for the item's dependencies
// and stages it with the Tensor Memory Accelerator into one of two shared-
// memory stages (mbarrier transaction counts): pass-R rows by bulk copies into
// padded rows, pass-L columns by 5-D tensor copies, the coefficient table and
// the outer-index records by bulk copies.  Eight consumer warps (10
// selectable) compute the other stage meanwhile, and a finisher warp does the
// device-scope bookkeeping of finished tiles.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <atomic>
#include <mutex>
#include <string>
#include <vector>

#include "common.cuh"
#include "hpsi.cuh"
#include "hpsi_fast.cuh"
#include "ptx.cuh"

namespace rpm {
namespace {

using namespace fastpass;
using namespace ptx;

constexpr int kTabCache = 256;                   // vectors whose table pointers are cached in shared memory

constexpr int align128c(int b) { return (b + 127) & ~127; }
constexpr int cmax(int a, int b) { return a > b ? a : b; }

__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// ---------------------------------------------------------------------------
// PTX helpers: tensor copies, acquire / release (mbarriers and bulk copies: ptx.cuh)
// ---------------------------------------------------------------------------
__device__ __forceinline__ void tma_5d(void* dst, const CUtensorMap* map, int c0, int c1, int c2, int c3, int c4,
                                       unsigned long long* bar) {
  asm volatile(
      "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5, "
      "%6}], [%7];\n" ::"r"(smem_u32(dst)),
      "l"(map), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4), "r"(smem_u32(bar))
      : "memory");
}
// Order this thread's generic-proxy global accesses with async-proxy (TMA)
// accesses.
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async;\n" ::: "memory"); }
__device__ __forceinline__ int ld_acquire(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];\n" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release(int* p, int v) {
  asm volatile("st.release.gpu.global.b32 [%0], %1;\n" ::"l"(p), "r"(v) : "memory");
}
// Device-scope acquire-release fetch-and-add: earlier writes this thread
// performed or observed become visible before the update, and later reads see
// what the other updaters published before theirs.
__device__ __forceinline__ unsigned atom_add_acq_rel(unsigned* p, unsigned v) {
  unsigned old;
  asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], %2;\n" : "=r"(old) : "l"(p), "r"(v) : "memory");
  return old;
}
// Wait until *p >= need (acquire); false after the time limit or a raised status.
__device__ bool wait_progress(const int* p, int need, int* status) {
  const long long t0 = clock64();
  while (true) {
    if (ld_acquire(p) >= need) return true;
    if (*reinterpret_cast<volatile int*>(status)) return false;
    if (clock64() - t0 > kWaitCycles) {
      atomicExch(status, 1);
      return false;
    }
    __nanosleep(128);
  }
}

// ---------------------------------------------------------------------------
// Shape constants
// ---------------------------------------------------------------------------
// Left radical (N1L spin-1, NHL spin-1/2 digits) -> pass L; right radical -> pass R.
template <int N1L, int NHL, int N1R, int NHR>
struct PShape {
  using PR = PassR<float2, N1R, NHR>;
  using PL = PassL<float2, N1L, NHL>;
  using SR = typename PR::S;
  using SL = typename PL::S;
  static constexpr int HL = PL::HL, HR = PR::HR;
  static constexpr int TR = PR::TR;                  // rows per R tile
  static constexpr int RT = (2 * HL + TR - 1) / TR;  // R tiles per vector
  static constexpr int LT = HR / 8;                  // L tiles per vector
  static constexpr int PT = RT + LT;
  // l extent of one tensor-copy box (<= 256 rows, dividing HL)
  static constexpr int LSPLIT = (HL + 255) / 256;
  static constexpr int BL = HL / LSPLIT;
  static_assert(HL % LSPLIT == 0, "l extent must split into equal tensor boxes");
  static_assert(HR % 8 == 0, "pass L tiles need 8 | HR");
  static constexpr int TAB_BYTES = align128c(cmax(SR::NTAB, SL::NTAB) * 8);
  // outer records (pass R), or outer records + the 128-byte pair operator (pass L)
  static constexpr int OREC_BYTES =
      align128c(cmax((PR::NO * 24 + 15) / 16 * 16, (PL::NO * 24 + 15) / 16 * 16 + 128));
  static constexpr int R_TILE_BYTES = TR * PR::RS * 8;  // one padded R tile
  static constexpr int L_TILE_BYTES = 2 * HL * 16 * 8;
  // an L stage also holds one 2 KiB pass-R partial buffer per consumer warp
  static constexpr int kMaxConsumerWarps = 10;
  static constexpr int PBUF_BYTES = 2048;
  static constexpr int TILE_BYTES =
      align128c(cmax(2 * R_TILE_BYTES, L_TILE_BYTES + kMaxConsumerWarps * PBUF_BYTES));
  static constexpr int STAGE = TAB_BYTES + OREC_BYTES + TILE_BYTES;
  static constexpr int SMEM = 2 * STAGE + 1024;  // + alignment slack
};

struct Item {
  int kind;  // 0: R, 1: L, -1: end
  int j, b, tile, skip;
  float al, sc, bp;  // R with j > 0: alpha_{j-1}, 1 / beta_{j-1}, beta_{j-1}
};

// Item index -> (phase, iteration within the launch, vector, tile) in the
// wavefront order over `mseg` iterations.
template <class PS>
__device__ __forceinline__ Item decode(long long idx, int mseg, int nb, int gv) {
  Item it{};
  const long long full_groups = nb / gv;
  const long long per_group = (long long)mseg * gv * PS::PT;
  long long vg, r;
  int g;
  if (idx < full_groups * per_group) {
    vg = idx / per_group;
    r = idx - vg * per_group;
    g = gv;
  } else {
    vg = full_groups;
    r = idx - full_groups * per_group;
    g = nb - (int)full_groups * gv;
  }
  it.j = (int)(r / ((long long)g * PS::PT));
  int q = (int)(r - (long long)it.j * g * PS::PT);
  if (q < g * PS::RT) {
    it.kind = 0;
    it.b = (int)vg * gv + q / PS::RT;
    it.tile = q % PS::RT;
  } else {
    q -= g * PS::RT;
    it.kind = 1;
    it.b = (int)vg * gv + q / PS::LT;
    it.tile = q % PS::LT;
  }
  return it;
}

// CW consumer warps, one producer warp and one finisher warp per CTA, one
// CTA per SM.  Registers are allocated per SM sub-partition (4 per SM,
// 16,384 registers each, warps assigned round-robin), so the cap is the
// largest multiple of 8 that fits ceil((CW + 2) / 4) warps into one
// sub-partition.
template <int CW>
struct PRegs {
  static constexpr int per_part = (CW + 2 + 3) / 4;
  static constexpr int raw = 16384 / (per_part * 32) / 8 * 8;
  static constexpr int value = raw > 255 ? 255 : raw;
};

// An item moves through three roles:
//   producer  -- dequeues, waits for the item's dependency, stages tiles,
//                table and outer records by TMA into stage s (two stages),
//                completes full[s];
//   consumers -- wait full[s], compute their warp tasks (the pass-R combine
//                of v_j is shared by all consumer warps and joined by the
//                bounded barrier comb[s]), leave the item record and their
//                L sums in slot q of a ring (kRing slots) and arrive on
//                empty[s] and cdone[q];
//   finisher  -- waits cdone[q], takes the record, frees the slot (ffree[q])
//                and does the device-scope bookkeeping: the tile count, the
//                alpha/beta finalisation of the last L tile and the progress
//                release.
// No CTA-wide barrier is used after set-up, warps that finish a tile early
// move on to the next one, and the finisher may lag kRing items behind.
template <int N1L, int NHL, int N1R, int NHR, int CW>
__global__ void __maxnreg__(PRegs<CW>::value)
    k_lanczos_persistent(const __grid_constant__ CUtensorMap vmap, PersistentLanczos p) {
  constexpr int kConsumers = CW * 32;
  using PS = PShape<N1L, NHL, N1R, NHR>;
  using PR = typename PS::PR;
  using PL = typename PS::PL;
  constexpr int HL = PS::HL, HR = PS::HR, TR = PS::TR, RS = PR::RS;
  constexpr long long QUARTER = (long long)HL * HR;
  constexpr int OREC_R = ((PR::NO * 24) + 15) / 16 * 16;
  constexpr int OREC_L = ((PL::NO * 24) + 15) / 16 * 16 + 128;  // + the pair operator
  static_assert(OREC_R <= PS::OREC_BYTES && OREC_L <= PS::OREC_BYTES, "outer records exceed their stage slot");
  static_assert(CW <= PS::kMaxConsumerWarps, "an L stage holds the partial buffers of at most kMaxConsumerWarps warps");
  extern __shared__ unsigned char smem_raw[];
  unsigned char* base =
      reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
  constexpr int kRing = 4;
  __shared__ __align__(8) unsigned long long full_bar[2], empty_bar[2], comb_bar[2], cdone_bar[kRing],
      ffree_bar[kRing];
  __shared__ Item meta[2];
  __shared__ Item fmeta[kRing];
  __shared__ double red[kRing][CW][3];
  __shared__ const void* tab_ptr[4][kTabCache];  // per vector: tabR, tabL, orecR, orecL
  auto stage_tab = [&](int s) { return reinterpret_cast<float2*>(base + s * PS::STAGE); };
  auto stage_orec = [&](int s) { return reinterpret_cast<ORec<float2>*>(base + s * PS::STAGE + PS::TAB_BYTES); };
  auto stage_tile = [&](int s) {
    return reinterpret_cast<float2*>(base + s * PS::STAGE + PS::TAB_BYTES + PS::OREC_BYTES);
  };
  auto view_ptrs = [&](int b, const void*(&out)[4]) {
    if (b < kTabCache) {
      for (int k = 0; k < 4; ++k) out[k] = tab_ptr[k][b];
    } else {
      const CubeView<float2>* v = p.views + (p.sys_of ? p.sys_of[b] : 0);
      out[0] = v->tabR;
      out[1] = v->tabL;
      out[2] = v->orecR;
      out[3] = v->orecL;
    }
  };
  if (threadIdx.x == 0) {
    for (int s = 0; s < 2; ++s) {
      mbar_init(&full_bar[s], 1);
      mbar_init(&empty_bar[s], CW);
      mbar_init(&comb_bar[s], CW);
    }
    for (int q = 0; q < kRing; ++q) {
      mbar_init(&cdone_bar[q], CW);
      mbar_init(&ffree_bar[q], 1);
    }
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  for (int b = threadIdx.x; b < min(p.nb, kTabCache); b += blockDim.x) {
    const CubeView<float2>* v = p.views + (p.sys_of ? p.sys_of[b] : 0);
    tab_ptr[0][b] = v->tabR;
    tab_ptr[1][b] = v->tabL;
    tab_ptr[2][b] = v->orecR;
    tab_ptr[3][b] = v->orecL;
  }
  __syncthreads();
  const int mseg = p.j1 - p.j0;
  const long long total = (long long)mseg * p.nb * PS::PT;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  if (warp == CW) {
    // ----------------------------- producer -----------------------------
    // per stage: the last use armed (copies or end) and whether it got copies
    long long armed_use[2] = {-1, -1};
    bool armed_copies[2] = {false, false};
    // the dequeue runs one item ahead, so its latency overlaps the wait for a free stage
    long long next_idx = 0;
    if (lane == 0) next_idx = atomicAdd(p.work, 1u);
    for (long long it = 0;; ++it) {
      const int s = (int)(it & 1);
      const long long use = it >> 1;
      bool ok = true;
      long long idx = 0;
      if (lane == 0) {
        idx = next_idx;
        if (use >= 1) ok = mbar_wait(&empty_bar[s], (unsigned)((use - 1) & 1), p.status);
        if (ok && idx < total) next_idx = atomicAdd(p.work, 1u);
      }
      ok = __shfl_sync(0xffffffffu, ok, 0);
      idx = __shfl_sync(0xffffffffu, idx, 0);
      Item m{};
      m.kind = -1;
      if (ok && idx < total) {
        m = decode<PS>(idx, mseg, p.nb, p.gv);
        m.j += p.j0;
        if (lane == 0) {
          const int need = m.kind == 0 ? 2 * m.j : 2 * m.j + 1;
          if (need > 0) ok = wait_progress(p.prog + m.b, need, p.status);
          if (ok) {
            // per-vector scalars published with the progress this item waited
            // for: the consumers take them from the item record
            m.skip = *reinterpret_cast<volatile int*>(p.skip + (long long)m.b * p.istride) != 0;
            if (m.kind == 0 && m.j > 0) {
              const long long d = (long long)m.b * p.dstride;
              m.al = (float)__ldcg(p.alpha + d + m.j - 1);
              m.sc = (float)__ldcg(p.scale + d);
              m.bp = (float)__ldcg(p.beta + d + m.j - 1);
            }
          }
        }
        ok = __shfl_sync(0xffffffffu, ok, 0);
        m.skip = __shfl_sync(0xffffffffu, m.skip, 0);
        if (!ok) m.kind = -1;
      }
      armed_use[s] = use;
      armed_copies[s] = m.kind >= 0 && !m.skip;
      if (m.kind < 0 || m.skip) {
        // the end, or a vector that stopped: no data, the record only
        if (lane == 0) {
          meta[s] = m;
          mbar_arrive(&full_bar[s]);
        }
        __syncwarp();
        if (m.kind < 0) break;
        continue;
      }
      fence_proxy_async();
      const void* ptrs[4];
      view_ptrs(m.b, ptrs);
      const float2* vj = p.V + (long long)m.b * p.vstride + (long long)m.j * p.ld;
      float2* tile = stage_tile(s);
      if (m.kind == 0) {
        const int row0 = m.tile * TR;
        const int rows = min(TR, 2 * HL - row0);
        const bool prev = m.j > 0;
        const unsigned bytes = (unsigned)(rows * 2 * HR * 8 * (prev ? 2 : 1) + PS::SR::NTAB * 8 + OREC_R);
        if (lane == 0) {
          meta[s] = m;
          mbar_arrive_expect_tx(&full_bar[s], bytes);
        }
        __syncwarp();
        if (lane == 0) bulk_g2s(stage_tab(s), ptrs[0], PS::SR::NTAB * 8, &full_bar[s]);
        if (lane == 1) bulk_g2s(stage_orec(s), ptrs[2], OREC_R, &full_bar[s]);
        const int rr = lane & 15, which = lane >> 4;
        if (rr < rows && (which == 0 || prev)) {
          const float2* src = which == 0 ? vj : vj - p.ld;
          float2* dst = tile + which * TR * RS + rr * RS;
          const int rho = row0 + rr;
          const int ea = rho >= HL ? 1 : 0;
          const long long g = 2 * ea * QUARTER + (long long)(rho - ea * HL) * HR;
          bulk_g2s(dst, src + g, HR * 8, &full_bar[s]);
          bulk_g2s(dst + HR, src + g + QUARTER, HR * 8, &full_bar[s]);
        }
      } else {
        const unsigned bytes = (unsigned)(PS::L_TILE_BYTES + PS::SL::NTAB * 8 + OREC_L);
        if (lane == 0) {
          meta[s] = m;
          mbar_arrive_expect_tx(&full_bar[s], bytes);
        }
        __syncwarp();
        if (lane == 0) bulk_g2s(stage_tab(s), ptrs[1], PS::SL::NTAB * 8, &full_bar[s]);
        if (lane == 1) bulk_g2s(stage_orec(s), ptrs[3], OREC_L, &full_bar[s]);
        if (lane >= 2 && lane < 2 + 2 * PS::LSPLIT) {
          const int q = lane - 2;
          const int ea = q / PS::LSPLIT, part = q % PS::LSPLIT;
          const long long slot = p.slot0 + (long long)m.b * (p.m + 1) + m.j;
          tma_5d(tile + (ea * HL + part * PS::BL) * 16, &vmap, m.tile * 8, 0, part * PS::BL, ea, (int)slot,
                 &full_bar[s]);
        }
      }
      __syncwarp();
    }
    // drain: copies this warp issued complete before the CTA may exit (a
    // stage armed again later was consumed, so its copies completed)
    if (lane == 0) {
      for (int s = 0; s < 2; ++s)
        if (armed_copies[s]) mbar_wait(&full_bar[s], (unsigned)(armed_use[s] & 1), p.status);
    }
    return;
  }

  if (warp == CW + 1) {
    // ----------------------------- finisher -----------------------------
    for (long long it = 0;; ++it) {
      const int q = (int)(it % kRing);
      bool ok = true;
      if (lane == 0) ok = mbar_wait(&cdone_bar[q], (unsigned)((it / kRing) & 1), p.status);
      ok = __shfl_sync(0xffffffffu, ok, 0);
      if (!ok) break;
      const Item m = fmeta[q];
      if (m.kind < 0) break;
      if (lane == 0) {
        const int b = m.b;
        double t0 = 0.0, t1 = 0.0, t2 = 0.0;
        if (m.kind == 1 && !m.skip)
          for (int w = 0; w < CW; ++w) {
            t0 += red[q][w][0];
            t1 += red[q][w][1];
            t2 += red[q][w][2];
          }
        mbar_arrive(&ffree_bar[q]);  // the slot's record and sums are taken
        if (m.kind == 1 && !m.skip) {
          double* part = p.part + (long long)b * p.part_stride + m.tile * 3;
          part[0] = t0;
          part[1] = t1;
          part[2] = t2;
        }
        // the consumers' global writes (ordered before this thread by cdone)
        // and the sums become visible device-wide with the count; the last
        // tile of a phase sees every other tile's sums
        fence_proxy_async();
        const int ntiles = m.kind == 0 ? PS::RT : PS::LT;
        const unsigned done = atom_add_acq_rel(p.cnt + b, 1u);
        if (done == (unsigned)ntiles - 1) {
          p.cnt[b] = 0;
          if (m.kind == 1 && !m.skip) {
            // alpha_j, beta_j and the breakdown test from the tiles' sums, in tile order
            double s0 = 0.0, s1 = 0.0, s2 = 0.0;
            const double* pt = p.part + (long long)b * p.part_stride;
            for (int k = 0; k < PS::LT; ++k) {
              s0 += __ldcg(pt + 3 * k);
              s1 += __ldcg(pt + 3 * k + 1);
              s2 += __ldcg(pt + 3 * k + 2);
            }
            const double alpha = s2 > 0.0 ? s0 / s2 : 0.0;
            p.alpha[(long long)b * p.dstride + m.j] = alpha;
            if (m.j < p.m - 1) {
              const double beta = sqrt(fmax(s1 - s0 * alpha, 0.0));  // |w' - alpha v_j|
              p.beta[(long long)b * p.dstride + m.j] = beta;
              p.scale[(long long)b * p.dstride] = beta > 0.0 ? 1.0 / beta : 0.0;
              const double ref = fabs(alpha) + (m.j == 0 ? 0.0 : p.beta[(long long)b * p.dstride + m.j - 1]);
              const int cap = p.mcap ? p.mcap[(long long)b * p.istride] : p.m;
              if (m.j + 1 >= cap) {  // this vector's Krylov cap: its basis ends here
                p.skip[(long long)b * p.istride] = 1;
                p.msize[(long long)b * p.istride] = cap;
              } else if (!(beta > p.breakdown_rel * ref)) {
                p.stop[(long long)b * p.istride] = 1;
                p.skip[(long long)b * p.istride] = 1;
                p.msize[(long long)b * p.istride] = m.j + 1;
              }
            }
          }
          st_release(p.prog + b, m.kind == 0 ? 2 * m.j + 1 : 2 * m.j + 2);
        }
      }
      __syncwarp();
    }
    return;
  }

  // ----------------------------- consumers -----------------------------
  const int tid = threadIdx.x;  // 0 .. kConsumers - 1
  unsigned comb_use[2] = {0u, 0u};
  for (long long it = 0;; ++it) {
    const int s = (int)(it & 1);
    if (!mbar_wait(&full_bar[s], (unsigned)((it >> 1) & 1), p.status)) break;
    Item m = meta[s];
    const int q = (int)(it % kRing);
    // the ring slot of this item is free once the finisher took item it - kRing
    if (it >= kRing && !mbar_wait(&ffree_bar[q], (unsigned)((it / kRing - 1) & 1), p.status)) break;
    if (m.kind < 0) {
      if (warp == 0 && lane == 0) fmeta[q] = m;
      __syncwarp();
      if (lane == 0) mbar_arrive(&cdone_bar[q]);  // lets the finisher see the end
      break;
    }
    // a vector stopped by a breakdown (or finished before this Krylov step)
    // keeps its counters moving but does no arithmetic (the producer read the
    // flag after the progress this item waited for)
    const bool skip = m.skip != 0;
    bool ok = true;
    if (!skip) {
      float2* tab = stage_tab(s);
      const ORec<float2>* orec = stage_orec(s);
      float2* tile = stage_tile(s);
      const int b = m.b;
      float2* vj = p.V + (long long)b * p.vstride + (long long)m.j * p.ld;
      float2* yb = p.ya + (long long)b * p.ld;
      if (m.kind == 0) {
        const int row0 = m.tile * TR;
        const int rows = min(TR, 2 * HL - row0);
        float2* ptile = tile + TR * RS;
        const bool prev = m.j > 0;
        float bprev = 0.0f;
        if (prev) {
          // v_j = (w'_j - alpha_{j-1} v_{j-1}) / beta_{j-1}: into the tile and the basis
          const float al = m.al, sc = m.sc;
          bprev = m.bp;
          constexpr int CH = HR / 2;  // 16-byte units per half row
          for (int u = tid; u < rows * 2 * CH; u += kConsumers) {
            const int rr = u / (2 * CH), rem = u - rr * (2 * CH);
            const int e = rem / CH, c = rem - e * CH;
            const int rho = row0 + rr;
            const int ea = rho >= HL ? 1 : 0;
            const int slot = rr * RS + e * HR + 2 * c;
            const long long g = (2 * ea + e) * QUARTER + (long long)(rho - ea * HL) * HR + 2 * c;
            const float4 w = *reinterpret_cast<const float4*>(tile + slot);
            const float4 q = *reinterpret_cast<const float4*>(ptile + slot);
            float4 v;
            v.x = sc * fmaf(-al, q.x, w.x);
            v.y = sc * fmaf(-al, q.y, w.y);
            v.z = sc * fmaf(-al, q.z, w.z);
            v.w = sc * fmaf(-al, q.w, w.w);
            *reinterpret_cast<float4*>(tile + slot) = v;
            *reinterpret_cast<float4*>(vj + g) = v;
          }
          // every consumer warp's share is combined before any warp reads the rows
          __syncwarp();
          if (lane == 0) mbar_arrive(&comb_bar[s]);
          ok = mbar_wait(&comb_bar[s], comb_use[s] & 1u, p.status);
          ++comb_use[s];
        }
        if (ok)
          r_tile_math<float2, N1R, NHR>(tab, orec, tile, ptile, rows, row0, HL, QUARTER, yb, 1.0f, bprev, prev, warp,
                                        CW);
      } else {
        const float2* pair = reinterpret_cast<const float2*>(reinterpret_cast<const char*>(orec) + OREC_L - 128);
        double dot = 0.0, nw = 0.0, nv = 0.0;
        float2* pbuf = tile + PS::L_TILE_BYTES / 8 + warp * (PS::PBUF_BYTES / 8);
        l_tile_math<float2, N1L, NHL>(tab, orec, tile, pair, HR, m.tile * 8, QUARTER, yb, vj + p.ld, 1.0f,
                                      m.j < p.m - 1, warp, CW, dot, nw, nv, pbuf);
        dot = warp_sum_d(dot);
        nw = warp_sum_d(nw);
        nv = warp_sum_d(nv);
        if (lane == 0) {
          red[q][warp][0] = dot;
          red[q][warp][1] = nw;
          red[q][warp][2] = nv;
        }
      }
    }
    if (!ok) break;
    if (warp == 0 && lane == 0) fmeta[q] = m;
    __syncwarp();
    if (lane == 0) {
      mbar_arrive(&empty_bar[s]);  // this warp no longer reads the stage
      mbar_arrive(&cdone_bar[q]);
    }
  }
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static std::once_flag once;
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  std::call_once(once, [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q{};
    const cudaError_t err = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q);
    if (err == cudaSuccess && q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
    else
      cudaGetLastError();
  });
  if (!fn) fail(RPM_E_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
  return fn;
}

// 5-D map of the basis buffer: (r, eB, l, eA, slot) with strides (element,
// N/4, HR, N/2, ld) elements and a box of 8 r x 2 eB x BL l, so that one box
// lands as [l][eB][8 r] rows of 16 elements.
template <class PS>
CUtensorMap basis_map(const float2* V, long long nslots, long long ld) {
  CUtensorMap map;
  const cuuint64_t q = (cuuint64_t)PS::HL * PS::HR;
  cuuint64_t dims[5] = {(cuuint64_t)PS::HR, 2, (cuuint64_t)PS::HL, 2, (cuuint64_t)nslots};
  cuuint64_t strides[4] = {q * 8, (cuuint64_t)PS::HR * 8, 2 * q * 8, (cuuint64_t)ld * 8};
  cuuint32_t box[5] = {8, 2, (cuuint32_t)PS::BL, 1, 1};
  cuuint32_t estr[5] = {1, 1, 1, 1, 1};
  if (nslots < 1 || nslots > 0x7fffffffLL) fail(RPM_E_UNSUPPORTED, "basis too large for the tensor map");
  const CUresult r = encode_fn()(&map, CU_TENSOR_MAP_DATA_TYPE_UINT64, 5, const_cast<float2*>(V), dims, strides, box,
                                 estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                                 CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS)
    fail(RPM_E_CUDA, "cuTensorMapEncodeTiled failed for the basis map (" + std::to_string((int)r) + ")");
  return map;
}

template <int N1L, int NHL, int N1R, int NHR, int CW>
void launch_instance(const PersistentLanczos& p, const float2* V_base, long long nslots, cudaStream_t st) {
  using PS = PShape<N1L, NHL, N1R, NHR>;
  static_assert(PS::SMEM <= 227 * 1024, "persistent Lanczos stages exceed shared memory");
  constexpr int kThreads = CW * 32 + 64;
  auto kern = k_lanczos_persistent<N1L, NHL, N1R, NHR, CW>;
  {
    static std::mutex mu;
    static std::vector<int> done;  // devices with the attribute set
    int dev = 0;
    check_cuda(cudaGetDevice(&dev), "cudaGetDevice");
    std::lock_guard<std::mutex> lock(mu);
    bool have = false;
    for (int d : done) have = have || d == dev;
    if (!have) {
      check_cuda(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, PS::SMEM),
                 "persistent Lanczos smem attr");
      int per_sm = 0;
      check_cuda(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kThreads, PS::SMEM), "occupancy");
      if (per_sm < 1) fail(RPM_E_UNSUPPORTED, "persistent Lanczos kernel does not fit on an SM");
      done.push_back(dev);
    }
  }
  const CUtensorMap map = basis_map<PS>(V_base, nslots, p.ld);
  const int ctas = p.ctas > 0 ? std::min(p.ctas, sm_count()) : sm_count();
  kern<<<ctas, kThreads, PS::SMEM, st>>>(map, p);
  check_launch("k_lanczos_persistent");
}

using Launcher = void (*)(const PersistentLanczos&, const float2*, long long, cudaStream_t);

// Consumer warps per CTA (8, 9 or 10; set by rpm_set_persistent_warps): with
// the producer and finisher warps all keep 168 registers per thread; 8 splits
// the full system's 24 pass-R warp tasks evenly (the combine barrier waits
// for the slowest warp), 9 its 36 pass-L tasks, 10 hides more latency.
std::atomic<int> g_consumer_warps{8};

template <int N1L, int NHL, int N1R, int NHR>
Launcher by_warps(int warps) {
  switch (warps) {
    case 9: return launch_instance<N1L, NHL, N1R, NHR, 9>;
    case 10: return launch_instance<N1L, NHL, N1R, NHR, 10>;
    default: return launch_instance<N1L, NHL, N1R, NHR, 8>;
  }
}

Launcher pick(const CubePlan& plan, int* ltiles) {
  if (!plan.fast) return nullptr;
  const int l1 = plan.fl_n1, lh = plan.fl_nh, r1 = plan.fr_n1, rh = plan.fr_nh;
  const int warps = g_consumer_warps.load(std::memory_order_relaxed);
  if (l1 == 2 && lh == 5 && r1 == 1 && rh == 6) {
    if (ltiles) *ltiles = PShape<2, 5, 1, 6>::LT;
    return by_warps<2, 5, 1, 6>(warps);
  }
  if (l1 == 2 && lh == 3 && r1 == 1 && rh == 4) {
    if (ltiles) *ltiles = PShape<2, 3, 1, 4>::LT;
    return by_warps<2, 3, 1, 4>(warps);
  }
  return nullptr;
}

}  // namespace

// 2-D map of a basis buffer [nslots][ld] complex64 (elements as 8-byte words)
// with a box of box_rows consecutive elements of box_slots consecutive slots;
// one tensor copy lands as [slot][box_rows].
CUtensorMap basis_rows_map(const float2* V, long long nslots, long long ld, int box_rows, int box_slots) {
  CUtensorMap map;
  if (nslots < 1 || nslots > 0x7fffffffLL || box_rows < 1 || box_rows > 256 || box_slots < 1 || box_slots > 256 ||
      (box_rows * 8) % 16 != 0 || (ld * 8) % 16 != 0 || (reinterpret_cast<uintptr_t>(V) & 15u))
    fail(RPM_E_UNSUPPORTED, "basis rows map: unsupported sizes or alignment");
  cuuint64_t dims[2] = {(cuuint64_t)ld, (cuuint64_t)nslots};
  cuuint64_t strides[1] = {(cuuint64_t)ld * 8};
  cuuint32_t box[2] = {(cuuint32_t)box_rows, (cuuint32_t)box_slots};
  cuuint32_t estr[2] = {1, 1};
  const CUresult r = encode_fn()(&map, CU_TENSOR_MAP_DATA_TYPE_UINT64, 2, const_cast<float2*>(V), dims, strides, box,
                                 estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                                 CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS)
    fail(RPM_E_CUDA, "cuTensorMapEncodeTiled failed for the basis rows map (" + std::to_string((int)r) + ")");
  return map;
}

int persistent_l_tiles(const CubePlan& plan) {
  int lt = 0;
  return pick(plan, &lt) ? lt : 0;
}

bool launch_lanczos_persistent(const PersistentLanczos& p, const CubePlan& plan, const float2* V_base, long long nslots,
                               cudaStream_t stream) {
  const Launcher fn = pick(plan, nullptr);
  if (!fn) return false;
  if (p.nb < 1 || p.m < 1 || p.gv < 1 || p.j0 < 0 || p.j1 <= p.j0 || p.j1 > p.m)
    fail(RPM_E_INVALID, "persistent Lanczos: empty launch or bad iteration range");
  if (p.part_stride < 3 * persistent_l_tiles(plan)) fail(RPM_E_INVALID, "persistent Lanczos: partial-sum stride");
  auto aligned = [](const void* ptr) { return (reinterpret_cast<uintptr_t>(ptr) & 15u) == 0; };
  if (!aligned(p.V) || !aligned(p.ya) || !aligned(V_base) || (p.ld & 1) || (p.vstride & 1))
    fail(RPM_E_INVALID, "persistent Lanczos: basis and partials need 16-byte alignment");
  fn(p, V_base, nslots, stream);
  return true;
}

}  // namespace rpm

extern "C" int rpm_set_persistent_warps(int consumer_warps) {
  return rpm::guarded([&] {
    if (consumer_warps < 8 || consumer_warps > 10) rpm::fail(RPM_E_INVALID, "consumer warps must be 8, 9 or 10");
    rpm::g_consumer_warps.store(consumer_warps, std::memory_order_relaxed);
  });
}
