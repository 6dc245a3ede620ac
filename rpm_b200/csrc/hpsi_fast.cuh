// Device pieces of the shape-specialised H psi passes, shared by the
// per-iteration kernels (hpsi_fast.cu) and the persistent Lanczos kernel
// (lanczos_persistent.cu).  See hpsi_fast.cu for the thread mappings.
#pragma once

#include "common.cuh"
#include "hpsi.cuh"

namespace rpm {
namespace fastpass {

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
// Pass R: 16 rows (eA, l) x all (eB, r) per tile; lane bits 0-3 = row, lane
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


// ---------------------------------------------------------------------------
// Pass L: every l x 16 columns (eB x 8 consecutive r) per tile; lane bits 0-2
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


// Outer records of one staged table (merged diagonal / electron-flip
// coefficients of every outer index); pass R: digits 0..K-3, pass L: 0..K-4.
template <class T, class S, int NOUT, int DIV>
__device__ __forceinline__ void build_orec(const T* tab, ORec<T>* orec, int no, int tid, int nthreads) {
  for (int o = tid; o < no; o += nthreads) {
    ORec<T> r;
    r.d[0] = tab[0].x;
    r.d[1] = tab[1].x;
    r.f[0] = tab[2];
    r.f[1] = tab[3];
#pragma unroll
    for (int k = 0; k < NOUT; ++k) {
      const int m = (o / (S::gs(k) / DIV)) % S::dim(k);
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        r.d[e] += tab[S::offD(k) + e * S::dim(k) + m].x;
        r.f[e] = cadd(r.f[e], tab[S::offF(k) + e * S::dim(k) + m]);
      }
    }
    orec[o] = r;
  }
}

// Pass-R arithmetic of one staged tile: rows row0 .. row0 + rows - 1 of
// vector b, staged at `tile` (row stride RS) with v_{j-1} at `ptile` when
// with_prev; warp `warp` of `nwarps` takes warp tasks warp, warp + nwarps, ...
// Writes the partial sf (1 (x) R) v - bprev v_{j-1} of its rows to y_vec
// (vector b's partial buffer, same layout as the state).
template <class T, int N1, int NH>
__device__ __forceinline__ void r_tile_math(const T* tab, const ORec<T>* orec, const T* tile, const T* ptile, int rows,
                                            int row0, int half_l, long long quarter, T* y_vec,
                                            typename FastT<T>::R sf, typename FastT<T>::R bprev, bool with_prev,
                                            int warp, int nwarps) {
  using P = PassR<T, N1, NH>;
  using S = typename P::S;
  using R = typename FastT<T>::R;
  constexpr int K = S::K;
  constexpr int HR = P::HR, NO = P::NO, RS = P::RS, EPU = P::EPU;
  const int lane = threadIdx.x & 31;
  const int row = lane & 15, hsel = lane >> 4;
  const T* rowp = tile + row * RS;
  const T* prowp = ptile + row * RS;
  R din[2][4];
  T fin[2][4];
  cube_consts<S>(tab, din, fin);
  const int rho = row0 + row;
  const int ea = rho >= half_l ? 1 : 0;
  const long long gbase = 2 * ea * quarter + (long long)(rho - ea * half_l) * HR;
  T* y_b = y_vec + gbase;
  for (int t = warp; t < P::NTASK; t += nwarps) {
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

// Pass-L arithmetic of one staged tile: columns c0 .. c0 + 7 of both
// electron-B halves of vector b, staged at `tile` (16 elements per l); adds
// the pass-R partial y_vec and writes out_vec (when `store`).  `pair` is the
// 4 x 4 electron-pair operator, HR the right radical's half size.
// Accumulates sf <x, out>, |out|^2 and |x|^2 over its elements (x: the staged
// input).  `pbuf` (complex64 only; nullptr: direct loads): this warp's
// 2 KiB shared-memory buffer, into which each task's pass-R partial is copied
// by 16-byte cp.async (L2 only) when the task starts and read back when it
// ends, so the copy's latency overlaps the task's arithmetic without holding
// registers.  Buffer layout: segment ((e 4 + i) 4 + h 2 + lg) of 8 columns.
template <class T, int N1, int NH>
__device__ __forceinline__ void l_tile_math(const T* tab, const ORec<T>* orec, const T* tile, const T* pair, int HR,
                                            int c0, long long quarter, const T* y_vec, T* out_vec,
                                            typename FastT<T>::R sf, bool store, int warp, int nwarps, double& dot,
                                            double& nw, double& nv, T* pbuf = nullptr) {
  using P = PassL<T, N1, NH>;
  using S = typename P::S;
  using R = typename FastT<T>::R;
  constexpr int K = S::K;
  constexpr int HL = P::HL, NO = P::NO;
  const int lane = threadIdx.x & 31;
  const int j = lane & 7, h = (lane >> 3) & 1, lg = lane >> 4, c = lane & 15;
  // electron-pair operator rows of (e, h): eB-diagonal part merged, eB flip via the partner column
  R dp[2];
  T fp[2], pp[2][2];
#pragma unroll
  for (int e = 0; e < 2; ++e) {
    dp[e] = pair[(e * 2 + h) * 4 + e * 2 + h].x;
    fp[e] = pair[(e * 2 + h) * 4 + (1 - e) * 2 + h];
#pragma unroll
    for (int ep = 0; ep < 2; ++ep) pp[e][ep] = pair[(e * 2 + h) * 4 + ep * 2 + (1 - h)];
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
  const bool cdiag = pair[0].y != R(0) || pair[5].y != R(0) || pair[10].y != R(0) ||
                     pair[15].y != R(0);
  R gim[2];
#pragma unroll
  for (int e = 0; e < 2; ++e) gim[e] = pair[(e * 2 + h) * 4 + e * 2 + h].y;
  const T* col = tile + c;
  const long long cofs = h * quarter + c0 + j;
  const T* y_b = y_vec + cofs;
  T* y_out = out_vec + cofs;
  for (int o = warp; o < NO; o += nwarps) {
    const ORec<T> rec = orec[o];
    const int lo = o * 8 + lg * 4;  // l of cube element i = 0
    T pb[2][4];  // pass-R partial of the cube (with -beta_{j-1} v_{j-1} when fused), loaded early
    bool staged = false;
    if constexpr (P::EPU == 2) {
      if (pbuf) {
        // 32 segments of 8 consecutive columns (64 bytes), four 16-byte copies each
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          const int cidx = lane + 32 * k;
          const int seg = cidx >> 2, piece = cidx & 3;
          const int se = seg >> 4, si = (seg >> 2) & 3, sh = (seg >> 1) & 1, sg = seg & 1;
          copy16(pbuf + seg * 8 + 2 * piece,
                 y_vec + (2 * se + sh) * quarter + (long long)(o * 8 + sg * 4 + si) * HR + c0 + 2 * piece);
        }
        asm volatile("cp.async.commit_group;\n" ::: "memory");
        staged = true;
      }
    }
    if (!staged) {
#pragma unroll
      for (int e = 0; e < 2; ++e)
#pragma unroll
        for (int i = 0; i < 4; ++i) pb[e][i] = __ldcg(y_b + 2 * e * quarter + (long long)(lo + i) * HR);
    }
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
    if (staged) {
      // every lane's copies have landed before any lane reads the buffer, and
      // every lane has read it before the next task's copies overwrite it
      asm volatile("cp.async.wait_group 0;\n" ::: "memory");
      __syncwarp();
#pragma unroll
      for (int e = 0; e < 2; ++e)
#pragma unroll
        for (int i = 0; i < 4; ++i) pb[e][i] = pbuf[((e * 4 + i) * 4 + h * 2 + lg) * 8 + j];
      __syncwarp();
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
}

}  // namespace fastpass
}  // namespace rpm
