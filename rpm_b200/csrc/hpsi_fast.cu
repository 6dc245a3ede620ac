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

namespace rpm {
namespace {

constexpr int ipow3(int n) { return n == 0 ? 1 : 3 * ipow3(n - 1); }

// Digit k of a radical's nuclei (k = 0 slowest): spin-1 for k < N1, spin-1/2
// after.  Table offsets follow build_cube_side: [Zd0, Zd1, Zf0, Zf1], then per
// nucleus D (2d), F (2d), X ((2d)^2).
template <int N1, int NH>
struct Shape {
  static constexpr int K = N1 + NH;
  static constexpr int HALF = ipow3(N1) << NH;
  static constexpr int dim(int k) { return k < N1 ? 3 : 2; }
  static constexpr int gs(int k) {
    int s = 1;
    for (int q = K - 1; q > k; --q) s *= dim(q);
    return s;
  }
  static constexpr int offD(int k) {
    int o = 4;
    for (int q = 0; q < k; ++q) o += 4 * dim(q) + 4 * dim(q) * dim(q);
    return o;
  }
  static constexpr int offF(int k) { return offD(k) + 2 * dim(k); }
  static constexpr int offX(int k) { return offD(k) + 4 * dim(k); }
  static constexpr int NTAB = offD(K);
};

// Element type: complex64 stages two elements per 16-byte copy and carries
// the fused Lanczos recurrence; complex128 stages one and runs plain H psi
// (and holds twice the registers per element, so one CTA per SM is assumed).
template <class T> struct FastT;
template <> struct FastT<float2> {
  using R = float;
  static constexpr int EPU = 2;
  static constexpr int MINB = 2;
};
template <> struct FastT<double2> {
  using R = double;
  static constexpr int EPU = 1;
  static constexpr int MINB = 1;
};

// Per outer index: diagonal and electron-flip coefficients merged over the
// electron-only term and every outer digit.
template <class T>
struct ORec {
  typename FastT<T>::R d[2];
  T f[2];
};

constexpr int align16c(int bytes) { return (bytes + 15) & ~15; }

__device__ __forceinline__ void copy16(void* smem_dst, const void* gmem_src) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem_dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void copy_wait_all() { asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory"); }

template <class T>
__device__ __forceinline__ T rmac(typename FastT<T>::R d, T x, T acc) {
  acc.x = fma(d, x.x, acc.x);
  acc.y = fma(d, x.y, acc.y);
  return acc;
}

template <class T>
__device__ __forceinline__ bool skip_vec(const HpsiArgs<T>& a, int b) {
  return a.skip && a.skip[(long long)b * a.skip_stride] != 0;
}
template <class T>
__device__ __forceinline__ double in_scale(const HpsiArgs<T>& a, int b) {
  return a.in_scale ? a.in_scale[(long long)b * a.scale_stride] : 1.0;
}

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
      if (!(beta > z.breakdown_rel * ref)) {
        z.stop[(long long)b * z.istride] = 1;
        z.skip[(long long)b * z.istride] = 1;
        z.msize[(long long)b * z.istride] = z.j + 1;
      }
    }
    a.dot_count[b] = 0;
  }
}

// Merged diagonal / flip coefficients of the two register-cube digits
// (digits K-2 -> bit 1 of i, K-1 -> bit 0 of i).
template <class S, class T>
__device__ __forceinline__ void cube_consts(const T* tab, typename FastT<T>::R (&din)[2][4], T (&fin)[2][4]) {
  constexpr int K = S::K;
#pragma unroll
  for (int e = 0; e < 2; ++e)
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      din[e][i] = tab[S::offD(K - 2) + e * 2 + (i >> 1)].x + tab[S::offD(K - 1) + e * 2 + (i & 1)].x;
      fin[e][i] = cadd(tab[S::offF(K - 2) + e * 2 + (i >> 1)], tab[S::offF(K - 1) + e * 2 + (i & 1)]);
    }
}

// Register-cube transitions of the two cube digits.
template <class S, class T>
__device__ __forceinline__ void cube_inner(const T* tab, const T (&x)[2][4], T (&acc)[2][4]) {
  constexpr int K = S::K;
#pragma unroll
  for (int q = 0; q < 2; ++q) {
    const T* X = tab + S::offX(K - 2 + q);
    const int sh = 1 - q;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int bit = (i >> sh) & 1;
      const int ip = i ^ (1 << sh);
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        acc[e][i] = cfma(X[(e * 2 + bit) * 4 + (1 - bit)], x[0][ip], acc[e][i]);
        acc[e][i] = cfma(X[(e * 2 + bit) * 4 + 2 + (1 - bit)], x[1][ip], acc[e][i]);
      }
    }
  }
}

// acc[e][i] += c[e][ep] * y[ep][i]
template <class T>
__device__ __forceinline__ void partner_mac(const T (&c)[2][2], const T (&y)[2][4], T (&acc)[2][4]) {
#pragma unroll
  for (int ep = 0; ep < 2; ++ep)
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      acc[0][i] = cfma(c[0][ep], y[ep][i], acc[0][i]);
      acc[1][i] = cfma(c[1][ep], y[ep][i], acc[1][i]);
    }
}

// Coefficients of one partner along outer digit k (value m -> mp) for every
// (output electron e, input electron ep).
template <class S, class T>
__device__ __forceinline__ void outer_coefs(const T* tab, int k, int m, int mp, T (&c)[2][2]) {
  const T* X = tab + S::offX(k);
  const int d = S::dim(k);
#pragma unroll
  for (int e = 0; e < 2; ++e)
#pragma unroll
    for (int ep = 0; ep < 2; ++ep) c[e][ep] = X[(e * d + m) * 2 * d + ep * d + mp];
}

// ---------------------------------------------------------------------------
// Pass R: 16 rows (eA, l) x all (eB, r) per CTA; lane bits 0-3 = row, lane
// bit 4 selects one of two outer indices of the warp's task.
// ---------------------------------------------------------------------------
template <class T, int N1, int NH>
struct PassR {
  using S = Shape<N1, NH>;
  static constexpr int EPU = FastT<T>::EPU;
  static constexpr int TR = 16;          // rows per CTA
  static constexpr int HR = S::HALF;
  static constexpr int NO = HR / 4;      // outer indices per row
  static constexpr int NTASK = (NO + 1) / 2;  // warp tasks: two outer indices each
  // padded row stride (elements): an odd number of 16-byte units
  static constexpr int RS = EPU == 2 ? 2 * HR + 2 : 2 * HR + 1;
  static constexpr int TAB_BYTES = align16c(S::NTAB * (int)sizeof(T));
  static constexpr int OREC_BYTES = align16c(NO * (int)sizeof(ORec<T>));
  // tables, records, the tile and (complex64, fused Lanczos) the tile of v_{j-1}
  static constexpr int SMEM = TAB_BYTES + OREC_BYTES + (EPU == 2 ? 2 : 1) * TR * RS * (int)sizeof(T);
  // 8 warps: measured faster than 12 or 16, which force register spills
  static constexpr int WARPS =
      NTASK % 8 == 0 ? 8 : NTASK % 6 == 0 ? 6 : NTASK % 4 == 0 ? 4 : NTASK % 3 == 0 ? 3 : NTASK < 8 ? NTASK : 8;
  static_assert(NH >= 2, "pass R needs two trailing spin-1/2 digits");
};

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
  for (int o = threadIdx.x; o < NO; o += NT) {
    ORec<T> r;
    r.d[0] = tab[0].x;
    r.d[1] = tab[1].x;
    r.f[0] = tab[2];
    r.f[1] = tab[3];
#pragma unroll
    for (int k = 0; k < K - 2; ++k) {
      const int m = (o / (S::gs(k) / 4)) % S::dim(k);
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        r.d[e] += tab[S::offD(k) + e * S::dim(k) + m].x;
        r.f[e] = cadd(r.f[e], tab[S::offF(k) + e * S::dim(k) + m]);
      }
    }
    orec[o] = r;
  }
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

  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int row = lane & 15, hsel = lane >> 4;
  const R sf = a.lz.on ? R(1) : (R)in_scale(a, b);  // fused: the staged v_j is already scaled
  // Paige's -beta_{j-1} v_{j-1} joins the partial here, where v_{j-1} is staged
  const R bprev = with_prev ? (R)a.lz.beta_prev[(long long)b * a.lz.dstride] : R(0);
  const T* rowp = tile + row * RS;
  const T* prowp = ptile + row * RS;
  R din[2][4];
  T fin[2][4];
  cube_consts<S>(tab, din, fin);
  const int rho = row0 + row;
  const int ea = rho >= half_l ? 1 : 0;
  const long long gbase = 2 * ea * quarter + (long long)(rho - ea * half_l) * HR;
  T* y_b = yb + (long long)b * (a.ya_ld ? a.ya_ld : a.ld) + gbase;
  for (int t = warp; t < P::NTASK; t += P::WARPS) {
    const int o = min(2 * t + hsel, NO - 1);  // (odd NO: the spare half repeats the last index, no store)
    const bool active = 2 * t + hsel < NO && row < rows;
    const ORec<T> rec = orec[o];
    auto load = [&](int delta, T (&y)[2][4]) {
#pragma unroll
      for (int ep = 0; ep < 2; ++ep) {
        if constexpr (EPU == 2) {
          const float4 u = *reinterpret_cast<const float4*>(rowp + ep * HR + 4 * o + delta);
          const float4 v = *reinterpret_cast<const float4*>(rowp + ep * HR + 4 * o + delta + 2);
          y[ep][0] = make_float2(u.x, u.y);
          y[ep][1] = make_float2(u.z, u.w);
          y[ep][2] = make_float2(v.x, v.y);
          y[ep][3] = make_float2(v.z, v.w);
        } else {
#pragma unroll
          for (int i = 0; i < 4; ++i) y[ep][i] = rowp[ep * HR + 4 * o + delta + i];
        }
      }
    };
    T x[2][4], acc[2][4];
    load(0, x);
#pragma unroll
    for (int e = 0; e < 2; ++e)
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        acc[e][i] = rmac<T>(rec.d[e] + din[e][i], x[e][i], czero<T>());
        acc[e][i] = cfma(cadd(rec.f[e], fin[e][i]), x[1 - e][i], acc[e][i]);
      }
    cube_inner<S>(tab, x, acc);
#pragma unroll
    for (int k = 0; k < K - 2; ++k) {
      const int m = (o / (S::gs(k) / 4)) % S::dim(k);
#pragma unroll
      for (int tt = 1; tt < S::dim(k); ++tt) {
        const int mp = m + tt >= S::dim(k) ? m + tt - S::dim(k) : m + tt;
        T c[2][2], y[2][4];
        outer_coefs<S>(tab, k, m, mp, c);
        load((mp - m) * S::gs(k), y);
        partner_mac(c, y, acc);
      }
    }
    if (active && EPU == 1) {
#pragma unroll
      for (int e = 0; e < 2; ++e)
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          T v = acc[e][i];
          v.x *= sf;
          v.y *= sf;
          y_b[e * quarter + 4 * o + i] = v;
        }
    }
    if constexpr (EPU == 2) if (active) {
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const long long at = e * quarter + 4 * o;
        float4 w0, w1;
        w0.x = sf * acc[e][0].x;
        w0.y = sf * acc[e][0].y;
        w0.z = sf * acc[e][1].x;
        w0.w = sf * acc[e][1].y;
        w1.x = sf * acc[e][2].x;
        w1.y = sf * acc[e][2].y;
        w1.z = sf * acc[e][3].x;
        w1.w = sf * acc[e][3].y;
        if (with_prev) {
          const float4 q0 = *reinterpret_cast<const float4*>(prowp + e * HR + 4 * o);
          const float4 q1 = *reinterpret_cast<const float4*>(prowp + e * HR + 4 * o + 2);
          w0.x = fmaf(-bprev, q0.x, w0.x);
          w0.y = fmaf(-bprev, q0.y, w0.y);
          w0.z = fmaf(-bprev, q0.z, w0.z);
          w0.w = fmaf(-bprev, q0.w, w0.w);
          w1.x = fmaf(-bprev, q1.x, w1.x);
          w1.y = fmaf(-bprev, q1.y, w1.y);
          w1.z = fmaf(-bprev, q1.z, w1.z);
          w1.w = fmaf(-bprev, q1.w, w1.w);
        }
        *reinterpret_cast<float4*>(y_b + at) = w0;
        *reinterpret_cast<float4*>(y_b + at + 2) = w1;
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Pass L: every l x 16 columns (eB x 8 consecutive r) per CTA; lane bits 0-2
// = r, bit 3 = eB, bit 4 = digit K-3 of l.  Cube = eA x digits K-2, K-1.
// ---------------------------------------------------------------------------
template <class T, int N1, int NH>
struct PassL {
  using S = Shape<N1, NH>;
  static constexpr int EPU = FastT<T>::EPU;
  static constexpr int HL = S::HALF;
  static constexpr int NO = HL / 8;  // outer indices
  static constexpr int NL = 2 * HL;
  static constexpr int TAB_BYTES = align16c(S::NTAB * (int)sizeof(T));
  static constexpr int OREC_BYTES = align16c(NO * (int)sizeof(ORec<T>));
  static constexpr int SMEM = TAB_BYTES + OREC_BYTES + NL * 16 * (int)sizeof(T);
  static constexpr int WARPS =
      NO % 8 == 0 ? 8 : NO % 6 == 0 ? 6 : NO % 9 == 0 ? 9 : NO % 4 == 0 ? 4 : NO % 3 == 0 ? 3 : NO < 8 ? NO : 8;
  static_assert(NH >= 3, "pass L needs three trailing spin-1/2 digits");
};

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
  for (int o = threadIdx.x; o < NO; o += NT) {
    ORec<T> r;
    r.d[0] = tab[0].x;
    r.d[1] = tab[1].x;
    r.f[0] = tab[2];
    r.f[1] = tab[3];
#pragma unroll
    for (int k = 0; k < K - 3; ++k) {
      const int m = (o / (S::gs(k) / 8)) % S::dim(k);
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        r.d[e] += tab[S::offD(k) + e * S::dim(k) + m].x;
        r.f[e] = cadd(r.f[e], tab[S::offF(k) + e * S::dim(k) + m]);
      }
    }
    orec[o] = r;
  }
  copy_wait_all();
  __syncthreads();

  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int j = lane & 7, h = (lane >> 3) & 1, lg = lane >> 4, c = lane & 15;
  const bool fused = EPU == 2 && a.lz.on == 1;
  const bool store = !fused || !a.lz.last;
  const R sf = a.lz.on ? R(1) : (R)in_scale(a, b);  // fused / Arnoldi: pass R wrote the scaled v_j
  // electron-pair operator rows of (e, h): eB-diagonal part merged, eB flip via the partner column
  R dp[2];
  T fp[2], pp[2][2];
#pragma unroll
  for (int e = 0; e < 2; ++e) {
    dp[e] = view->pair[(e * 2 + h) * 4 + e * 2 + h].x;
    fp[e] = view->pair[(e * 2 + h) * 4 + (1 - e) * 2 + h];
#pragma unroll
    for (int ep = 0; ep < 2; ++ep) pp[e][ep] = view->pair[(e * 2 + h) * 4 + ep * 2 + (1 - h)];
  }
  // lane digit K-3
  R dL[2];
  T fL[2], cL[2][2];
#pragma unroll
  for (int e = 0; e < 2; ++e) {
    dL[e] = tab[S::offD(K - 3) + e * 2 + lg].x + dp[e];
    fL[e] = cadd(tab[S::offF(K - 3) + e * 2 + lg], fp[e]);
#pragma unroll
    for (int ep = 0; ep < 2; ++ep) cL[e][ep] = tab[S::offX(K - 3) + (e * 2 + lg) * 4 + ep * 2 + (1 - lg)];
  }
  R din[2][4];
  T fin[2][4];
  cube_consts<S>(tab, din, fin);
  // imaginary diagonal of the pair operator: nonzero only with unequal
  // recombination rates (the non-Hermitian -(i/2) |kS - kT| Q term)
  const bool cdiag = view->pair[0].y != R(0) || view->pair[5].y != R(0) || view->pair[10].y != R(0) ||
                     view->pair[15].y != R(0);
  R gim[2];
#pragma unroll
  for (int e = 0; e < 2; ++e) gim[e] = view->pair[(e * 2 + h) * 4 + e * 2 + h].y;
  const T* col = tile + c;
  const long long cofs = h * quarter + c0 + j;
  const T* y_b = yb + (long long)b * (a.ya_ld ? a.ya_ld : a.ld) + cofs;
  T* y_out = a.out + (long long)b * a.ld + cofs;
  double dot = 0.0, nw = 0.0, nv = 0.0;
  for (int o = warp; o < NO; o += P::WARPS) {
    const ORec<T> rec = orec[o];
    const int lo = o * 8 + lg * 4;  // l of cube element i = 0
    T pb[2][4];  // pass-R partial of the cube (with -beta_{j-1} v_{j-1} when fused), loaded early
#pragma unroll
    for (int e = 0; e < 2; ++e)
#pragma unroll
      for (int i = 0; i < 4; ++i) pb[e][i] = __ldcg(y_b + 2 * e * quarter + (long long)(lo + i) * HR);
    T x[2][4], acc[2][4];
#pragma unroll
    for (int e = 0; e < 2; ++e)
#pragma unroll
      for (int i = 0; i < 4; ++i) x[e][i] = col[(e * HL + lo + i) * 16];
#pragma unroll
    for (int e = 0; e < 2; ++e)
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        acc[e][i] = rmac<T>(rec.d[e] + dL[e] + din[e][i], x[e][i], czero<T>());
        acc[e][i] = cfma(cadd(cadd(rec.f[e], fL[e]), fin[e][i]), x[1 - e][i], acc[e][i]);
        if (cdiag) acc[e][i] = cfma(cmake(R(0), gim[e]), x[e][i], acc[e][i]);
      }
    cube_inner<S>(tab, x, acc);
    auto partner = [&](int delta, int dcol, const T (&cc)[2][2]) {
      T y[2][4];
#pragma unroll
      for (int ep = 0; ep < 2; ++ep)
#pragma unroll
        for (int i = 0; i < 4; ++i) y[ep][i] = tile[(ep * HL + lo + delta + i) * 16 + dcol];
      partner_mac(cc, y, acc);
    };
    partner((1 - 2 * lg) * 4, c, cL);  // lane digit
    partner(0, c ^ 8, pp);             // electron B flip (pair operator)
#pragma unroll
    for (int k = 0; k < K - 3; ++k) {
      const int m = (o / (S::gs(k) / 8)) % S::dim(k);
#pragma unroll
      for (int t = 1; t < S::dim(k); ++t) {
        const int mp = m + t >= S::dim(k) ? m + t - S::dim(k) : m + t;
        T cc[2][2];
        outer_coefs<S>(tab, k, m, mp, cc);
        partner((mp - m) * S::gs(k), c, cc);
      }
    }
    R part = 0, pw = 0, px = 0;
#pragma unroll
    for (int e = 0; e < 2; ++e)
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        T v;
        v.x = fma(sf, acc[e][i].x, pb[e][i].x);
        v.y = fma(sf, acc[e][i].y, pb[e][i].y);  // fused: w' = H v_j - beta_{j-1} v_{j-1}
        if (store) y_out[2 * e * quarter + (long long)(lo + i) * HR] = v;
        part = fma(x[e][i].x, v.x, fma(x[e][i].y, v.y, part));
        pw = fma(v.x, v.x, fma(v.y, v.y, pw));
        px = fma(x[e][i].x, x[e][i].x, fma(x[e][i].y, x[e][i].y, px));
      }
    dot += (double)part * (double)sf;
    nw += (double)pw;
    nv += (double)px;
  }
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
