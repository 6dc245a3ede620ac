// Shape-specialised H psi passes (complex64 and complex128) for the standard
// radical layout.
//
// Scope: radical-split systems whose tensor axes are ordered
// (electron A, electron B, left nuclei..., right nuclei...) -- the order of
// the reference's production system (rpm_statevector_engine.py:367-469,
// poster_reproduction/core.py:172-229) -- so that the state is the C-order
// array psi[eA][eB][l][r] with l over the left nuclei (HL values) and r over
// the right nuclei (HR values), and whose radicals each list their spin-1
// nuclei before their spin-1/2 nuclei.  The nuclear digit pattern of both
// radicals is a template parameter, so every digit stride, table offset and
// loop bound below is a compile-time constant.
//
// The action is the one of the cube form in hpsi.cu (same tables, same
// merged diagonal / electron-flip coefficients, same pair operator), with
// the two passes in the opposite order:
//   pass R: yb = sf (1 (x) R) psi            pass L: out = sf (L (x) 1 + P) psi + yb
// but the thread mapping is chosen so that every coefficient a warp needs at
// a time is the same for all 32 lanes:
//   * pass R: a CTA stages 16 rows (eA, l) x all (eB, r) of one vector; lane
//     bits 0-3 = row, bit 4 = one of the two outer indices of a warp task.
//     R's coefficients depend on (eB, r) only, which is uniform in a warp
//     task, so they are shared-memory broadcasts.  Each thread holds a
//     register cube (eB x the two fastest spin-1/2 digits) of its row.
//   * pass L: a CTA stages every l of 16 columns (eB x 8 consecutive r);
//     lane = column (+ one spin-1/2 digit of l as lane bit 4).  L's
//     coefficients depend on l only; the lane-bit digit and eB (for the pair
//     operator) are fixed per lane for the whole kernel.
// Partners along register digits come from registers, all others from the
// staged tile (conflict-free: padded rows in pass R, 128-byte rows in pass L).
// Pass R stores its partial row-wise (each lane 32 contiguous bytes); pass L
// reads it column-coalesced, prefetched at the start of each task, and fuses
// <psi, H psi>.  In the fused Lanczos iteration pass R also subtracts
// beta_{j-1} v_{j-1} (staged there for the combine) from the partial, so
// pass L never reads v_{j-1}.  Pass L walks the batch in reverse order so
// that the partials and inputs written or read last are still in L2 when it
// starts.  complex128 runs the same passes with one element per 16-byte copy,
// an odd row stride in 16-byte units, no fused recurrence and one CTA per SM.
#include <mutex>
#include <utility>
#include <vector>

#include "common.cuh"
#include "hpsi.cuh"
#include "hpsi_fast.cuh"

namespace rpm {
namespace {

using namespace fastpass;

// Fused <in_scaled, H in_scaled>: per-block partial; the last block of
// vector b sums the partials in block order (deterministic).
template <class T>
__device__ void finish_dot_fast(const HpsiArgs<T>& a, int b, double mine) {
  __shared__ double red[32];
  __shared__ bool last;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) mine += __shfl_xor_sync(0xffffffffu, mine, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = mine;
  __syncthreads();
  if (threadIdx.x == 0) {
    double tot = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) tot += red[w];
    a.dot_part[(long long)b * gridDim.x + blockIdx.x] = tot;
    __threadfence();
    last = atomicAdd(a.dot_count + b, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (last && threadIdx.x == 0) {
    __threadfence();
    double s = 0.0;
    for (int k = 0; k < (int)gridDim.x; ++k) s += __ldcg(a.dot_part + (long long)b * gridDim.x + k);
    a.dot_out[(long long)b * a.dot_stride] = s;
    a.dot_count[b] = 0;
  }
}

// Fused Lanczos reductions (s0 = <v_j, w'>, s1 = |w'|^2, s2 = |v_j|^2): per
// block partials, then the last block of vector b sums them in block order
// and sets alpha_j, beta_j, the scale and the breakdown flags (LanczosFuse).
__device__ void finish_lanczos(const HpsiArgs<float2>& a, int b, double s0, double s1, double s2) {
  __shared__ double red[3][32];
  __shared__ bool last;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    s0 += __shfl_xor_sync(0xffffffffu, s0, o);
    s1 += __shfl_xor_sync(0xffffffffu, s1, o);
    s2 += __shfl_xor_sync(0xffffffffu, s2, o);
  }
  if ((threadIdx.x & 31) == 0) {
    red[0][threadIdx.x >> 5] = s0;
    red[1][threadIdx.x >> 5] = s1;
    red[2][threadIdx.x >> 5] = s2;
  }
  __syncthreads();
  double* part = a.dot_part + (long long)b * gridDim.x * 3;
  if (threadIdx.x == 0) {
    double t0 = 0.0, t1 = 0.0, t2 = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
      t0 += red[0][w];
      t1 += red[1][w];
      t2 += red[2][w];
    }
    part[blockIdx.x * 3 + 0] = t0;
    part[blockIdx.x * 3 + 1] = t1;
    part[blockIdx.x * 3 + 2] = t2;
    __threadfence();
    last = atomicAdd(a.dot_count + b, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (last && threadIdx.x == 0) {
    __threadfence();
    double t0 = 0.0, t1 = 0.0, t2 = 0.0;
    for (int k = 0; k < (int)gridDim.x; ++k) {
      t0 += __ldcg(part + 3 * k);
      t1 += __ldcg(part + 3 * k + 1);
      t2 += __ldcg(part + 3 * k + 2);
    }
    const LanczosFuse& z = a.lz;
    const double alpha = t2 > 0.0 ? t0 / t2 : 0.0;
    z.alpha_out[(long long)b * z.dstride] = alpha;
    if (!z.last) {
      const double beta = sqrt(fmax(t1 - t0 * alpha, 0.0));  // |w' - alpha v_j|
      z.beta_out[(long long)b * z.dstride] = beta;
      z.scale_out[(long long)b * z.dstride] = beta > 0.0 ? 1.0 / beta : 0.0;
      const double ref = fabs(alpha) + (z.first ? 0.0 : z.beta_prev[(long long)b * z.dstride]);
      const int cap = z.mcap ? z.mcap[(long long)b * z.istride] : 0x7fffffff;
      if (z.j + 1 >= cap) {  // this vector's Krylov cap: its basis ends here
        z.skip[(long long)b * z.istride] = 1;
        z.msize[(long long)b * z.istride] = cap;
      } else if (!(beta > z.breakdown_rel * ref)) {
        z.stop[(long long)b * z.istride] = 1;
        z.skip[(long long)b * z.istride] = 1;
        z.msize[(long long)b * z.istride] = z.j + 1;
      }
    }
    a.dot_count[b] = 0;
  }
}

// ---------------------------------------------------------------------------
// Pass R: stage 16 rows by cp.async (and the fused recurrence's combine),
// then r_tile_math.
// ---------------------------------------------------------------------------
template <class T, int N1, int NH>
__global__ void __launch_bounds__(PassR<T, N1, NH>::WARPS * 32, FastT<T>::MINB)
    fast_pass_r(HpsiArgs<T> a, T* __restrict__ yb) {
  using P = PassR<T, N1, NH>;
  using S = typename P::S;
  using R = typename FastT<T>::R;
  constexpr int K = S::K;
  constexpr int TR = P::TR, HR = P::HR, NO = P::NO, RS = P::RS, EPU = P::EPU;
  constexpr int NT = P::WARPS * 32;
  const int b = blockIdx.y;
  if (skip_vec(a, b)) return;
  const CubeView<T>* view = a.views + (a.sys_of ? a.sys_of[b] : 0);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* tab = reinterpret_cast<T*>(smem_raw);
  ORec<T>* orec = reinterpret_cast<ORec<T>*>(smem_raw + P::TAB_BYTES);
  T* tile = reinterpret_cast<T*>(smem_raw + P::TAB_BYTES + P::OREC_BYTES);
  T* ptile = tile + TR * RS;  // complex64 only
  const int half_l = view->half_l;
  const int row0 = blockIdx.x * TR;
  const int rows = min(TR, 2 * half_l - row0);
  const long long quarter = (long long)half_l * HR;
  const T* x_in = a.in + (long long)b * a.ld;
  constexpr int CH = HR / EPU;  // 16-byte chunks per half row
  const int units = rows * 2 * CH;
  auto unit_at = [&](int idx, int& slot, long long& g) {
    const int rr = idx / (2 * CH), rem = idx - rr * (2 * CH);
    const int e = rem / CH, c = rem - e * CH;
    const int rho = row0 + rr;
    const int ea = rho >= half_l ? 1 : 0;
    const int llo = rho - ea * half_l;
    slot = rr * RS + e * HR + EPU * c;
    g = (2 * ea + e) * quarter + (long long)llo * HR + EPU * c;
  };
  // fused Lanczos (j > 0): the tile receives w'_j and ptile v_{j-1}; below,
  // v_j = (w'_j - alpha_{j-1} v_{j-1}) * scale replaces w'_j in the tile and in `in`
  const bool combine = EPU == 2 && a.lz.on && !a.lz.first;
  const bool with_prev = combine && a.lz.on == 1;  // Arnoldi (on == 2) only rescales
  const T* pv = nullptr;
  if constexpr (EPU == 2) pv = with_prev ? a.lz.prev + (long long)b * a.ld : nullptr;
  for (int idx = threadIdx.x; idx < units; idx += NT) {
    int slot;
    long long g;
    unit_at(idx, slot, g);
    copy16(tile + slot, x_in + g);
    if (with_prev) copy16(ptile + slot, pv + g);
  }
  for (int k = threadIdx.x; k < S::NTAB; k += NT) tab[k] = view->tabR[k];
  __syncthreads();
  build_orec<T, S, K - 2, 4>(tab, orec, NO, threadIdx.x, NT);
  copy_wait_all();
  if constexpr (EPU == 2) if (combine) {
    // each thread combines the units it copied (visible to it after its own wait)
    const float al = with_prev ? (float)a.lz.alpha_prev[(long long)b * a.lz.dstride] : 0.0f;
    const float sc = (float)in_scale(a, b);
    T* xo = const_cast<T*>(x_in);
    for (int idx = threadIdx.x; idx < units; idx += NT) {
      int slot;
      long long g;
      unit_at(idx, slot, g);
      const float4 w = *reinterpret_cast<const float4*>(tile + slot);
      const float4 q = with_prev ? *reinterpret_cast<const float4*>(ptile + slot) : make_float4(0.f, 0.f, 0.f, 0.f);
      float4 v;
      v.x = sc * fmaf(-al, q.x, w.x);
      v.y = sc * fmaf(-al, q.y, w.y);
      v.z = sc * fmaf(-al, q.z, w.z);
      v.w = sc * fmaf(-al, q.w, w.w);
      *reinterpret_cast<float4*>(tile + slot) = v;
      *reinterpret_cast<float4*>(xo + g) = v;
    }
  }
  __syncthreads();
  const R sf = a.lz.on ? R(1) : (R)in_scale(a, b);  // fused: the staged v_j is already scaled
  // Paige's -beta_{j-1} v_{j-1} joins the partial here, where v_{j-1} is staged
  const R bprev = with_prev ? (R)a.lz.beta_prev[(long long)b * a.lz.dstride] : R(0);
  r_tile_math<T, N1, NH>(tab, orec, tile, ptile, rows, row0, half_l, quarter,
                         yb + (long long)b * (a.ya_ld ? a.ya_ld : a.ld), sf, bprev, with_prev, threadIdx.x >> 5,
                         P::WARPS);
}

// ---------------------------------------------------------------------------
// Pass L: stage every l x 16 columns by cp.async, then l_tile_math.
// ---------------------------------------------------------------------------
template <class T, int N1, int NH>
__global__ void __launch_bounds__(PassL<T, N1, NH>::WARPS * 32, FastT<T>::MINB)
    fast_pass_l(HpsiArgs<T> a, const T* __restrict__ yb) {
  using P = PassL<T, N1, NH>;
  using S = typename P::S;
  using R = typename FastT<T>::R;
  constexpr int K = S::K;
  constexpr int HL = P::HL, NO = P::NO, NL = P::NL, EPU = P::EPU;
  constexpr int NT = P::WARPS * 32;
  constexpr int UH = 8 / EPU;  // 16-byte units per (l, electron B) row of 8 columns
  const int b = gridDim.y - 1 - blockIdx.y;
  if (skip_vec(a, b)) return;
  const CubeView<T>* view = a.views + (a.sys_of ? a.sys_of[b] : 0);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* tab = reinterpret_cast<T*>(smem_raw);
  ORec<T>* orec = reinterpret_cast<ORec<T>*>(smem_raw + P::TAB_BYTES);
  T* tile = reinterpret_cast<T*>(smem_raw + P::TAB_BYTES + P::OREC_BYTES);
  const int HR = view->half_r;
  const long long quarter = (long long)HL * HR;
  const int c0 = blockIdx.x * 8;
  const T* x_in = a.in + (long long)b * a.ld;
  for (int idx = threadIdx.x; idx < NL * 2 * UH; idx += NT) {
    const int l = idx / (2 * UH), h = (idx / UH) & 1, q = idx % UH;
    const int ea = l >= HL ? 1 : 0;
    const int llo = l - ea * HL;
    copy16(tile + l * 16 + h * 8 + EPU * q, x_in + (2 * ea + h) * quarter + (long long)llo * HR + c0 + EPU * q);
  }
  for (int k = threadIdx.x; k < S::NTAB; k += NT) tab[k] = view->tabL[k];
  __syncthreads();
  build_orec<T, S, K - 3, 8>(tab, orec, NO, threadIdx.x, NT);
  copy_wait_all();
  __syncthreads();
  const bool fused = EPU == 2 && a.lz.on == 1;
  const bool store = !fused || !a.lz.last;
  const R sf = a.lz.on ? R(1) : (R)in_scale(a, b);  // fused / Arnoldi: pass R wrote the scaled v_j
  double dot = 0.0, nw = 0.0, nv = 0.0;
  l_tile_math<T, N1, NH>(tab, orec, tile, view->pair, HR, c0, quarter, yb + (long long)b * (a.ya_ld ? a.ya_ld : a.ld),
                         a.out + (long long)b * a.ld, sf, store, threadIdx.x >> 5, P::WARPS, dot, nw, nv);
  if constexpr (EPU == 2) {
    if (fused) finish_lanczos(a, b, dot, nw, nv);
    else if (a.dot_part && !a.lz.on) finish_dot_fast(a, b, dot);
  } else {
    if (a.dot_part) finish_dot_fast(a, b, dot);
  }
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
// Raise the dynamic shared-memory limit once per kernel and device, so that
// launches recorded into a CUDA graph issue no attribute calls.
template <class K>
void set_smem(K kern, int bytes) {
  static std::mutex m;
  static std::vector<std::pair<const void*, int>> done;  // (kernel, device)
  int dev = 0;
  check_cuda(cudaGetDevice(&dev), "cudaGetDevice");
  const void* key = reinterpret_cast<const void*>(kern);
  std::lock_guard<std::mutex> lock(m);
  for (const auto& d : done)
    if (d.first == key && d.second == dev) return;
  check_cuda(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes), "fast H psi smem attr");
  done.emplace_back(key, dev);
}

template <class T, int N1, int NH>
void launch_l(const HpsiArgs<T>& a, const T* yb, int half_r, int batch, cudaStream_t st) {
  using P = PassL<T, N1, NH>;
  auto kern = fast_pass_l<T, N1, NH>;
  set_smem(kern, P::SMEM);
  kern<<<dim3(half_r / 8, batch), P::WARPS * 32, P::SMEM, st>>>(a, yb);
  check_launch("fast_pass_l");
}

template <class T, int N1, int NH>
void launch_r(const HpsiArgs<T>& a, T* yb, int half_l, int batch, cudaStream_t st) {
  using P = PassR<T, N1, NH>;
  auto kern = fast_pass_r<T, N1, NH>;
  set_smem(kern, P::SMEM);
  kern<<<dim3((2 * half_l + P::TR - 1) / P::TR, batch), P::WARPS * 32, P::SMEM, st>>>(a, yb);
  check_launch("fast_pass_r");
}

template <class T>
using LaunchL = void (*)(const HpsiArgs<T>&, const T*, int, int, cudaStream_t);
template <class T>
using LaunchR = void (*)(const HpsiArgs<T>&, T*, int, int, cudaStream_t);

// Shared memory a CTA may use (the complex128 tiles are twice as large: a
// pattern whose pass does not fit has no complex128 variant).
constexpr int kFastMaxSmem = 227 * 1024;

template <class T, int N1, int NH>
LaunchL<T> fit_l() {
  return PassL<T, N1, NH>::SMEM <= kFastMaxSmem ? launch_l<T, N1, NH> : nullptr;
}
template <class T, int N1, int NH>
LaunchR<T> fit_r() {
  return PassR<T, N1, NH>::SMEM <= kFastMaxSmem ? launch_r<T, N1, NH> : nullptr;
}

// Instantiated digit patterns (spin-1 count, spin-1/2 count) per radical.
template <class T>
LaunchL<T> pick_l(int n1, int nh) {
  if (n1 == 2 && nh == 5) return fit_l<T, 2, 5>();
  if (n1 == 2 && nh == 3) return fit_l<T, 2, 3>();
  if (n1 == 2 && nh == 4) return fit_l<T, 2, 4>();
  if (n1 == 2 && nh == 6) return fit_l<T, 2, 6>();
  if (n1 == 1 && nh == 5) return fit_l<T, 1, 5>();
  if (n1 == 1 && nh == 6) return fit_l<T, 1, 6>();
  if (n1 == 0 && nh == 6) return fit_l<T, 0, 6>();
  if (n1 == 1 && nh == 3) return fit_l<T, 1, 3>();
  return nullptr;
}
template <class T>
LaunchR<T> pick_r(int n1, int nh) {
  if (n1 == 1 && nh == 6) return fit_r<T, 1, 6>();
  if (n1 == 1 && nh == 4) return fit_r<T, 1, 4>();
  if (n1 == 1 && nh == 5) return fit_r<T, 1, 5>();
  if (n1 == 1 && nh == 3) return fit_r<T, 1, 3>();
  if (n1 == 1 && nh == 2) return fit_r<T, 1, 2>();
  if (n1 == 2 && nh == 5) return fit_r<T, 2, 5>();
  if (n1 == 0 && nh == 6) return fit_r<T, 0, 6>();
  if (n1 == 0 && nh == 3) return fit_r<T, 0, 3>();
  return nullptr;
}

// (spin-1 count, spin-1/2 count) of a cube side when its digits are all
// spin-1 first, then all spin-1/2; {-1, -1} otherwise.
void side_pattern(const CubeSide& s, int& n1, int& nh) {
  n1 = nh = 0;
  int k = 0;
  while (k < s.K && s.dim[k] == 3) ++k, ++n1;
  while (k < s.K && s.dim[k] == 2) ++k, ++nh;
  if (k != s.K) n1 = nh = -1;
}

}  // namespace

// Fills the fast-path fields of `p` for one system (first == true) or checks
// that another system of the same launch has the same shape.
void fast_plan_add(CubePlan& p, const rpm_system* s, bool first) {
  int n1l, nhl, n1r, nhr;
  side_pattern(s->cube_l, n1l, nhl);
  side_pattern(s->cube_r, n1r, nhr);
  bool ok = s->cube && n1l >= 0 && n1r >= 0 && pick_l<float2>(n1l, nhl) && pick_r<float2>(n1r, nhr) &&
            s->half_r % 8 == 0;
  if (ok) {
    // standard layout: offl[l] = eA * N/2 + l_lo * HR, offr[r] = eB * N/4 + r_lo
    const long long n = s->n, hl = s->half_l, hr = s->half_r;
    for (long long l = 0; ok && l < (long long)s->offl.size(); ++l)
      ok = s->offl[l] == (l / hl) * (n / 2) + (l % hl) * hr;
    for (long long r = 0; ok && r < (long long)s->offr.size(); ++r) ok = s->offr[r] == (r / hr) * (n / 4) + (r % hr);
  }
  if (first) {
    p.fast = ok ? 1 : 0;
    p.fl_n1 = n1l;
    p.fl_nh = nhl;
    p.fr_n1 = n1r;
    p.fr_nh = nhr;
    p.f_half_l = s->half_l;
    p.f_half_r = s->half_r;
  } else if (!ok || n1l != p.fl_n1 || nhl != p.fl_nh || n1r != p.fr_n1 || nhr != p.fr_nh || s->half_l != p.f_half_l ||
             s->half_r != p.f_half_r) {
    p.fast = 0;
  }
}

template <class T>
bool cube_fast_usable(const HpsiArgs<T>& a, const CubePlan& p, const T* ya) {
  if (!p.fast) return false;
  const long long yld = a.ya_ld ? a.ya_ld : a.ld;
  auto aligned = [](const void* ptr) { return (reinterpret_cast<uintptr_t>(ptr) & 15u) == 0; };
  if (!aligned(a.in) || !aligned(a.out) || !aligned(ya)) return false;
  if constexpr (FastT<T>::EPU == 2) {
    if ((a.ld & 1) || (yld & 1)) return false;
    if (a.lz.on == 1 && !a.lz.first && !aligned(a.lz.prev)) return false;
  } else {
    if (a.lz.on) return false;  // the fused recurrence is complex64 only
  }
  return pick_l<T>(p.fl_n1, p.fl_nh) && pick_r<T>(p.fr_n1, p.fr_nh);
}

template <class T>
bool launch_cube_fast(const HpsiArgs<T>& a, const CubePlan& p, T* ya, int batch, cudaStream_t st) {
  if (!cube_fast_usable<T>(a, p, ya)) return false;
  const LaunchL<T> fl = pick_l<T>(p.fl_n1, p.fl_nh);
  const LaunchR<T> fr = pick_r<T>(p.fr_n1, p.fr_nh);
  HpsiArgs<T> ar = a;
  ar.dot_part = nullptr;
  fr(ar, ya, p.f_half_l, batch, st);
  fl(a, ya, p.f_half_r, batch, st);
  return true;
}

template bool cube_fast_usable<float2>(const HpsiArgs<float2>&, const CubePlan&, const float2*);
template bool cube_fast_usable<double2>(const HpsiArgs<double2>&, const CubePlan&, const double2*);
template bool launch_cube_fast<float2>(const HpsiArgs<float2>&, const CubePlan&, float2*, int, cudaStream_t);
template bool launch_cube_fast<double2>(const HpsiArgs<double2>&, const CubePlan&, double2*, int, cudaStream_t);

}  // namespace rpm

extern "C" int rpm_system_fast_hpsi(const rpm_system* sys, int* usable) {
  return rpm::guarded([&] {
    if (!sys || !usable) rpm::fail(RPM_E_INVALID, "NULL argument");
    rpm::CubePlan p{};
    if (sys->split && sys->cube) rpm::fast_plan_add(p, sys, true);
    *usable = p.fast;
  });
}
