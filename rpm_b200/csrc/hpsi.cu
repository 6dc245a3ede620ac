// H psi kernels for sm_100a.
//
// Three exact forms of the reference's matrix-free action
// (rpm_statevector_engine.py:95-108 generic, :221-245 radical split):
//
// * Cube form (default for radical-split systems).  The state is viewed as
//   Psi[l, r], l over (electron A, FAD nuclei), r over (electron B, TrpH
//   nuclei).  Two shared-memory-tiled passes:
//     pass L: a tile of all l x 2*TR columns (both electron-B halves) ->
//             L Psi + electron-pair term, written to `ya`;
//     pass R: a tile of TL rows x all r -> Psi R^T, added to `ya`, with an
//             optional fused <psi, H psi> reduction.
//   Inside a tile every thread owns a "cube": both electron values times all
//   2^NI values of the NI fastest spin-1/2 digits of its group, in registers.
//   Terms on those digits are applied register-to-register with warp-uniform
//   coefficient tables; every other nucleus contributes through "partner"
//   cubes read from shared memory (one per alternative value of its digit).
//   All diagonal and electron-flip parts of every term are merged into two
//   per-element coefficients.  No per-nonzero index or value loads remain.
//
// * CSR form: the same two passes driven by CSR rows (fallback when a group
//   term couples two nuclei).
//
// * Generic per-term mode product for systems without a radical split.
#include <algorithm>
#include <atomic>
#include <mutex>
#include <type_traits>
#include <utility>
#include <vector>

#include "common.cuh"
#include "hpsi.cuh"

namespace rpm {

// ---------------------------------------------------------------------------
// Generic form
// ---------------------------------------------------------------------------
template <class T>
__global__ void __launch_bounds__(256) hpsi_generic_kernel(GenericView<T> g, const T* __restrict__ in,
                                                           T* __restrict__ out, long long ld) {
  extern __shared__ unsigned char smem_raw[];
  TermMeta* terms = reinterpret_cast<TermMeta*>(smem_raw);
  for (int t = threadIdx.x; t < g.nterms; t += blockDim.x) terms[t] = g.terms[t];
  __syncthreads();
  const T* x = in + (long long)blockIdx.y * ld;
  T* y = out + (long long)blockIdx.y * ld;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < g.n; i += gridDim.x * blockDim.x) {
    T acc = czero<T>();
    for (int t = 0; t < g.nterms; ++t) {
      const TermMeta& m = terms[t];
      int row = 0, base = i;
      for (int q = 0; q < m.naxes; ++q) {
        const int digit = (i / m.stride[q]) % m.dim[q];
        row += digit * m.lstride[q];
        base -= digit * m.stride[q];
      }
      const T* op = g.ops + m.op_offset + row * m.d;
      const int* co = g.coloff + m.col_offset;
      for (int c = 0; c < m.d; ++c) acc = cfma(__ldg(op + c), x[base + __ldg(co + c)], acc);
    }
    y[i] = acc;
  }
}

// ---------------------------------------------------------------------------
// Shared helpers of the split kernels
// ---------------------------------------------------------------------------
template <class T>
__device__ __forceinline__ T cscale(T v, double s) {
  v.x = (typename Real<T>::type)(v.x * s);
  v.y = (typename Real<T>::type)(v.y * s);
  return v;
}
template <class T>
__device__ __forceinline__ T rmul(typename Real<T>::type r, T v, T acc) {
  acc.x = fma(r, v.x, acc.x);
  acc.y = fma(r, v.y, acc.y);
  return acc;
}

template <class T>
__device__ __forceinline__ bool skip_vector(const HpsiArgs<T>& a, int b) {
  return a.skip && a.skip[(long long)b * a.skip_stride] != 0;
}
template <class T>
__device__ __forceinline__ double input_scale(const HpsiArgs<T>& a, int b) {
  return a.in_scale ? a.in_scale[(long long)b * a.scale_stride] : 1.0;
}

// Block-wide sum of one double (all threads return the total).
__device__ __forceinline__ double block_total(double v, double* red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  double s = 0.0;
  for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w];
  return s;
}

// Fused <in, H in>: per-block partial, the last block of vector b sums them in order.
template <class T>
__device__ void finish_dot(const HpsiArgs<T>& a, int b, double mine) {
  __shared__ double red[32];
  __shared__ bool last;
  const double tot = block_total(mine, red);
  if (threadIdx.x == 0) a.dot_part[(long long)b * gridDim.x + blockIdx.x] = tot;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(a.dot_count + b, 1u) == gridDim.x - 1;
  __syncthreads();
  if (last && threadIdx.x == 0) {
    __threadfence();
    double s = 0.0;
    for (int k = 0; k < (int)gridDim.x; ++k) s += __ldcg(a.dot_part + (long long)b * gridDim.x + k);
    a.dot_out[(long long)b * a.dot_stride] = s;
    a.dot_count[b] = 0;
  }
}

// ---------------------------------------------------------------------------
// Cube form
// ---------------------------------------------------------------------------
// Complex multiply-accumulate of the cube kernels: four FMAs per complex
// product in the state precision (FP32 for complex64, FP64 for complex128).
template <class T> struct CubeArith;

template <>
struct CubeArith<double2> {
  using Coef = double2;
  using R = double;
  __device__ static double2 prep(double2 x) { return x; }
  __device__ static double2 mac(const double2& c, double2 x, double2, double2 acc) { return cfma(c, x, acc); }
  __device__ static double2 rmac(double d, double2 x, double2 acc) {
    acc.x = fma(d, x.x, acc.x);
    acc.y = fma(d, x.y, acc.y);
    return acc;
  }
  __device__ static double2 add(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
  __device__ static double2 from_complex(double2 v) { return v; }
  __device__ static double re(const double2& c) { return c.x; }
};

template <>
struct CubeArith<float2> {
  using Coef = float2;
  using R = float;
  __device__ static float2 prep(float2 x) { return x; }
  __device__ static float2 mac(const float2& c, float2 x, float2, float2 acc) { return cfma(c, x, acc); }
  __device__ static float2 rmac(float d, float2 x, float2 acc) {
    acc.x = fmaf(d, x.x, acc.x);
    acc.y = fmaf(d, x.y, acc.y);
    return acc;
  }
  __device__ static float2 add(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
  __device__ static float2 from_complex(float2 v) { return v; }
  __device__ static float re(const float2& c) { return c.x; }
};

// Per outer index o (all group digits except the NI inner ones), built once
// per CTA in shared memory: the outer digits packed 4 bits each and the
// diagonal / electron-flip coefficients merged over Z and the outer digits.
// Group index g = e * half + C * o + i  (C = 2^NI, i = inner digits).
template <class T>
struct OuterRec {
  typename CubeArith<T>::Coef f[2];
  typename CubeArith<T>::R d[2];
  unsigned lo, hi;
};

__device__ __forceinline__ int align16(int bytes) { return (bytes + 15) & ~15; }

// Asynchronous global -> shared copy of one complex element (cp.async).
template <class T>
__device__ __forceinline__ void async_copy(T* smem_dst, const T* gmem_src) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem_dst);
  if constexpr (sizeof(T) == 16) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem_src) : "memory");
  } else {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem_src) : "memory");
  }
}
__device__ __forceinline__ void async_wait_all() {
  asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
}

// Copy one group's CubeSide and its coefficient table into shared memory.
template <class Coef>
__device__ __forceinline__ void load_side(const CubeSide& src, const Coef* tab_src, CubeSide& side, Coef* tab) {
  const int* s = reinterpret_cast<const int*>(&src);
  int* d = reinterpret_cast<int*>(&side);
  for (int k = threadIdx.x; k < (int)(sizeof(CubeSide) / sizeof(int)); k += blockDim.x) d[k] = s[k];
  __syncthreads();
  for (int k = threadIdx.x; k < side.ntab; k += blockDim.x) tab[k] = tab_src[k];
}

template <class T, int NI>
__device__ __forceinline__ void build_outer(const CubeSide& side, const typename CubeArith<T>::Coef* tab,
                                            OuterRec<T>* otab, int n_outer) {
  using A = CubeArith<T>;
  const int nout = side.K - NI;
  for (int o = threadIdx.x; o < n_outer; o += blockDim.x) {
    OuterRec<T> rec;
    rec.d[0] = A::re(tab[0]);
    rec.d[1] = A::re(tab[1]);
    rec.f[0] = tab[2];
    rec.f[1] = tab[3];
    int rem = o;
    unsigned lo = 0, hi = 0;
    for (int k = nout - 1; k >= 0; --k) {
      const int d = side.dim[k];
      const int m = rem % d;
      rem /= d;
      if (k < 8) lo |= (unsigned)m << (4 * k);
      else hi |= (unsigned)m << (4 * (k - 8));
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        rec.d[e] += A::re(tab[side.offD[k] + e * d + m]);
        rec.f[e] = A::add(rec.f[e], tab[side.offF[k] + e * d + m]);
      }
    }
    rec.lo = lo;
    rec.hi = hi;
    otab[o] = rec;
  }
}

// Diagonal and electron-flip coefficients contributed by the inner digits:
// the same for every cube of a CTA, so computed once per thread.
template <class T, int NI>
struct InnerConst {
  typename CubeArith<T>::R d[2][1 << NI];
  typename CubeArith<T>::Coef f[2][1 << NI];
  __device__ InnerConst(const CubeSide& side, const typename CubeArith<T>::Coef* tab) {
    using A = CubeArith<T>;
#pragma unroll
    for (int e = 0; e < 2; ++e)
#pragma unroll
      for (int i = 0; i < (1 << NI); ++i) {
        // first inner digit, then the others
        typename A::Coef fl = tab[side.offF[side.K - NI] + e * 2 + ((i >> (NI - 1)) & 1)];
        typename A::R dg = A::re(tab[side.offD[side.K - NI] + e * 2 + ((i >> (NI - 1)) & 1)]);
#pragma unroll
        for (int q = 1; q < NI; ++q) {
          const int k = side.K - NI + q;
          const int bit = (i >> (NI - 1 - q)) & 1;
          dg += A::re(tab[side.offD[k] + e * 2 + bit]);
          fl = A::add(fl, tab[side.offF[k] + e * 2 + bit]);
        }
        d[e][i] = dg;
        f[e][i] = fl;
      }
  }
};

// Register-cube update shared by both passes.  `at(e, i, delta)` returns the
// element (electron e, inner i) of the cube whose outer index is shifted by
// `delta` (delta = 0: the thread's own cube).
template <class T, int NI, class At>
__device__ __forceinline__ void cube_apply(const CubeSide& side, const typename CubeArith<T>::Coef* tab,
                                           const InnerConst<T, NI>& ic, const OuterRec<T>& rec,
                                           const typename CubeArith<T>::R (&dout)[2],
                                           const typename CubeArith<T>::Coef (&fout)[2], const T (&x)[2][1 << NI],
                                           T (&acc)[2][1 << NI], At at) {
  using A = CubeArith<T>;
  constexpr int C = 1 << NI;
  const int K = side.K;
  T xs[2][C];
#pragma unroll
  for (int e = 0; e < 2; ++e)
#pragma unroll
    for (int i = 0; i < C; ++i) xs[e][i] = A::prep(x[e][i]);
#pragma unroll
  for (int e = 0; e < 2; ++e)
#pragma unroll
    for (int i = 0; i < C; ++i) {
      acc[e][i] = A::rmac(dout[e] + ic.d[e][i], x[e][i], acc[e][i]);
      acc[e][i] = A::mac(A::add(fout[e], ic.f[e][i]), x[1 - e][i], xs[1 - e][i], acc[e][i]);
    }
#pragma unroll
  for (int q = 0; q < NI; ++q) {
    const typename A::Coef* X = tab + side.offX[K - NI + q];
#pragma unroll
    for (int i = 0; i < C; ++i) {
      const int bit = (i >> (NI - 1 - q)) & 1;
      const int ip = i ^ (1 << (NI - 1 - q));
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        acc[e][i] = A::mac(X[(e * 2 + bit) * 4 + (1 - bit)], x[0][ip], xs[0][ip], acc[e][i]);
        acc[e][i] = A::mac(X[(e * 2 + bit) * 4 + 2 + (1 - bit)], x[1][ip], xs[1][ip], acc[e][i]);
      }
    }
  }
  const int nout = K - NI;
  for (int k = 0; k < nout; ++k) {
    const int d = side.dim[k];
    const int m = (int)(((k < 8) ? (rec.lo >> (4 * k)) : (rec.hi >> (4 * (k - 8)))) & 15u);
    const int ostride = side.gs[k] >> NI;
    const typename A::Coef* X = tab + side.offX[k] + (size_t)m * 2 * d;
    for (int mp = 0; mp < d; ++mp) {
      if (mp == m) continue;
      const int delta = (mp - m) * ostride;
      T y[2][C];
#pragma unroll
      for (int e = 0; e < 2; ++e)
#pragma unroll
        for (int i = 0; i < C; ++i) y[e][i] = at(e, i, delta);
#pragma unroll
      for (int ep = 0; ep < 2; ++ep) {
        // coefficients of output electron e from input electron ep
        const typename A::Coef c0 = X[(0 * d) * 2 * d + ep * d + mp];
        const typename A::Coef c1 = X[(1 * d) * 2 * d + ep * d + mp];
#pragma unroll
        for (int i = 0; i < C; ++i) {
          const T ys = A::prep(y[ep][i]);
          acc[0][i] = A::mac(c0, y[ep][i], ys, acc[0][i]);
          acc[1][i] = A::mac(c1, y[ep][i], ys, acc[1][i]);
        }
      }
    }
  }
}

// Shared-memory carve-up of a cube pass: [tab][otab][offA][offB][tile...].
template <class T>
struct CubeSmem {
  typename CubeArith<T>::Coef* tab;
  OuterRec<T>* otab;
  int* offA;
  int* offB;
  T* tile;
  __device__ CubeSmem(unsigned char* raw, int tab_cap, int n_outer_cap, int na, int nb) {
    int pos = 0;
    tab = reinterpret_cast<typename CubeArith<T>::Coef*>(raw + pos);
    pos += align16(tab_cap * (int)sizeof(typename CubeArith<T>::Coef));
    otab = reinterpret_cast<OuterRec<T>*>(raw + pos);
    pos += align16(n_outer_cap * (int)sizeof(OuterRec<T>));
    offA = reinterpret_cast<int*>(raw + pos);
    pos += align16(na * 4);
    offB = reinterpret_cast<int*>(raw + pos);
    pos += align16(nb * 4);
    tile = reinterpret_cast<T*>(raw + pos);
  }
};

template <class T>
inline int cube_smem_prefix(int tab_cap, int n_outer_cap, int na, int nb) {
  auto a16 = [](int b) { return (b + 15) & ~15; };
  return a16(tab_cap * (int)sizeof(typename CubeArith<T>::Coef)) + a16(n_outer_cap * (int)sizeof(OuterRec<T>)) +
         a16(na * 4) + a16(nb * 4);
}

// Pass L: tile = all l rows x W = 2*TR columns, stored [e][i][o][c].
template <class T, int NI, int TR>
__global__ void __launch_bounds__(256) cube_pass_l(HpsiArgs<T> a, T* __restrict__ ya, int tab_cap, int n_outer_cap) {
  using A = CubeArith<T>;
  using R = typename A::R;
  using Coef = typename A::Coef;
  constexpr int C = 1 << NI;
  constexpr int W = 2 * TR;
  const int b = blockIdx.y;
  if (skip_vector(a, b)) return;
  const CubeView<T>* view = a.views + (a.sys_of ? a.sys_of[b] : 0);
  __shared__ CubeSide side;
  __shared__ Coef pair[16];
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int nl = view->nl, half_l = view->half_l, half_r = view->half_r;
  const int no = half_l >> NI;  // outer indices of this group
  CubeSmem<T> sm(smem_raw, tab_cap, n_outer_cap, nl, W);
  const int r0 = blockIdx.x * TR;
  if (threadIdx.x < 16) pair[threadIdx.x] = A::from_complex(view->pair[threadIdx.x]);
  for (int l = threadIdx.x; l < nl; l += blockDim.x) sm.offA[l] = __ldg(view->offl + l);
  if (threadIdx.x < W) {
    const int c = threadIdx.x, j = r0 + (c % TR);
    sm.offB[c] = j < half_r ? __ldg(view->offr + (c / TR) * half_r + j) : -1;
  }
  load_side(view->L, view->tabL, side, sm.tab);  // contains a barrier
  __syncthreads();
  const T* x_in = a.in + (long long)b * a.ld;
  for (int idx = threadIdx.x; idx < nl * W; idx += blockDim.x) {
    const int l = idx / W, c = idx % W;
    const int e = l >= half_l ? 1 : 0;
    const int rem = l - e * half_l;
    T* dst = sm.tile + (((e * C + (rem & (C - 1))) * no + (rem >> NI)) * W + c);
    const int col = sm.offB[c];
    if (col >= 0) async_copy(dst, x_in + sm.offA[l] + col);
    else *dst = czero<T>();
  }
  build_outer<T, NI>(side, sm.tab, sm.otab, no);
  async_wait_all();
  __syncthreads();
  const InnerConst<T, NI> ic(side, sm.tab);
  const R sf = (R)input_scale(a, b);
  const int eoff = sm.offA[half_l] - sm.offA[0];
  int ioff[C];
#pragma unroll
  for (int i = 0; i < C; ++i) ioff[i] = sm.offA[i] - sm.offA[0];
  const int plane = no * W;  // elements per (e, i) plane
  T* y_out = ya + (long long)b * (a.ya_ld ? a.ya_ld : a.ld);
  for (int task = threadIdx.x; task < W * no; task += blockDim.x) {
    const int c = task % W, o = task / W;
    const int col = sm.offB[c];
    if (col < 0) continue;
    const int h = c / TR;
    const OuterRec<T> rec = sm.otab[o];
    R dout[2];
    Coef fout[2];
#pragma unroll
    for (int e = 0; e < 2; ++e) {
      dout[e] = rec.d[e] + A::re(pair[(e * 2 + h) * 4 + e * 2 + h]);
      fout[e] = A::add(rec.f[e], pair[(e * 2 + h) * 4 + (1 - e) * 2 + h]);
    }
    const T* cb = sm.tile + task;  // (e, i) at cb[(e * C + i) * plane]; task == o * W + c
    T x[2][C], acc[2][C];
#pragma unroll
    for (int e = 0; e < 2; ++e)
#pragma unroll
      for (int i = 0; i < C; ++i) {
        x[e][i] = cb[(e * C + i) * plane];
        acc[e][i] = czero<T>();
      }
    cube_apply<T, NI>(side, sm.tab, ic, rec, dout, fout, x, acc,
                      [&](int e, int i, int delta) { return cb[(e * C + i) * plane + delta * W]; });
    // imaginary diagonal of the pair operator: nonzero only with unequal
    // recombination rates (the non-Hermitian -(i/2) |kS - kT| Q term)
#pragma unroll
    for (int e = 0; e < 2; ++e) {
      const R g = (R)pair[(e * 2 + h) * 4 + e * 2 + h].y;
      if (g != (R)0) {
#pragma unroll
        for (int i = 0; i < C; ++i) {
          acc[e][i].x -= g * x[e][i].y;
          acc[e][i].y += g * x[e][i].x;
        }
      }
    }
    const T* cp = cb + (h ? -TR : TR);  // partner column: electron B flipped
#pragma unroll
    for (int ep = 0; ep < 2; ++ep) {
      const Coef p0 = pair[(0 * 2 + h) * 4 + ep * 2 + (1 - h)];
      const Coef p1 = pair[(1 * 2 + h) * 4 + ep * 2 + (1 - h)];
#pragma unroll
      for (int i = 0; i < C; ++i) {
        const T z = cp[(ep * C + i) * plane];
        const T zs = A::prep(z);
        acc[0][i] = A::mac(p0, z, zs, acc[0][i]);
        acc[1][i] = A::mac(p1, z, zs, acc[1][i]);
      }
    }
    const int out0 = sm.offA[o << NI] + col;
#pragma unroll
    for (int e = 0; e < 2; ++e)
#pragma unroll
      for (int i = 0; i < C; ++i) {
        T v = acc[e][i];
        v.x *= sf;
        v.y *= sf;
        y_out[out0 + e * eoff + ioff[i]] = v;
      }
  }
}

// Pass R: tile = TL rows x all r, each row stored [e][i][o]; the pass-L
// partial of the same rows is prefetched into a second tile.
template <class T, int NI, int TL>
__global__ void __launch_bounds__(256) cube_pass_r(HpsiArgs<T> a, const T* __restrict__ ya, int tab_cap,
                                                   int n_outer_cap) {
  using A = CubeArith<T>;
  using R = typename A::R;
  constexpr int C = 1 << NI;
  const int b = blockIdx.y;
  if (skip_vector(a, b)) return;
  const CubeView<T>* view = a.views + (a.sys_of ? a.sys_of[b] : 0);
  __shared__ CubeSide side;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int nl = view->nl, nr = view->nr, half_r = view->half_r;
  const int no = half_r >> NI;
  CubeSmem<T> sm(smem_raw, tab_cap, n_outer_cap, TL, nr);
  T* tile2 = sm.tile + TL * nr;
  const int l0 = blockIdx.x * TL;
  const int rows = min(TL, nl - l0);
  if (threadIdx.x < rows) sm.offA[threadIdx.x] = __ldg(view->offl + l0 + threadIdx.x);
  for (int r = threadIdx.x; r < nr; r += blockDim.x) sm.offB[r] = __ldg(view->offr + r);
  load_side(view->R, view->tabR, side, sm.tab);  // contains a barrier
  __syncthreads();
  const T* x_in = a.in + (long long)b * a.ld;
  const T* yA = ya + (long long)b * (a.ya_ld ? a.ya_ld : a.ld);
  for (int lt = 0; lt < rows; ++lt) {
    const int rowoff = sm.offA[lt];
    for (int r = threadIdx.x; r < nr; r += blockDim.x) {
      const int e = r >= half_r ? 1 : 0;
      const int rem = r - e * half_r;
      const int pos = lt * nr + (e * C + (rem & (C - 1))) * no + (rem >> NI);
      const int addr = rowoff + sm.offB[r];
      async_copy(sm.tile + pos, x_in + addr);
      async_copy(tile2 + pos, yA + addr);
    }
  }
  build_outer<T, NI>(side, sm.tab, sm.otab, no);
  async_wait_all();
  __syncthreads();
  const InnerConst<T, NI> ic(side, sm.tab);
  const R sf = (R)input_scale(a, b);
  const int eoff = sm.offB[half_r] - sm.offB[0];
  int ioff[C];
#pragma unroll
  for (int i = 0; i < C; ++i) ioff[i] = sm.offB[i] - sm.offB[0];
  T* y_out = a.out + (long long)b * a.ld;
  double dot = 0.0;
  for (int task = threadIdx.x; task < rows * no; task += blockDim.x) {
    const int o = task % no, lt = task / no;
    const OuterRec<T> rec = sm.otab[o];
    const R dout[2] = {rec.d[0], rec.d[1]};
    const typename A::Coef fout[2] = {rec.f[0], rec.f[1]};
    const T* row = sm.tile + lt * nr + o;  // (e, i) at row[(e * C + i) * no]
    const T* prow = tile2 + lt * nr + o;
    T x[2][C], acc[2][C];
#pragma unroll
    for (int e = 0; e < 2; ++e)
#pragma unroll
      for (int i = 0; i < C; ++i) {
        x[e][i] = row[(e * C + i) * no];
        acc[e][i] = czero<T>();
      }
    cube_apply<T, NI>(side, sm.tab, ic, rec, dout, fout, x, acc,
                      [&](int e, int i, int delta) { return row[(e * C + i) * no + delta]; });
    const int out0 = sm.offA[lt] + sm.offB[o << NI];
    R part = 0;
#pragma unroll
    for (int e = 0; e < 2; ++e)
#pragma unroll
      for (int i = 0; i < C; ++i) {
        const T p = prow[(e * C + i) * no];
        T v;
        v.x = fma(sf, acc[e][i].x, p.x);
        v.y = fma(sf, acc[e][i].y, p.y);
        y_out[out0 + e * eoff + ioff[i]] = v;
        if (a.dot_part) {
          const T xv = row[(e * C + i) * no];
          part = fma(xv.x, v.x, fma(xv.y, v.y, part));
        }
      }
    dot += (double)part * (double)sf;
  }
  if (a.dot_part) finish_dot(a, b, dot);
}

// ---------------------------------------------------------------------------
// CSR form (fallback for group terms that couple two nuclei)
// ---------------------------------------------------------------------------
template <class T, int TR>
__global__ void __launch_bounds__(512) split_pass_a(SplitView<T> s, const T* __restrict__ in,
                                                    T* __restrict__ ya, long long ld) {
  constexpr int W = 2 * TR;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* pair = reinterpret_cast<T*>(smem_raw);
  T* tile = pair + 16;
  const T* x = in + (long long)blockIdx.y * ld;
  T* y = ya + (long long)blockIdx.y * ld;
  const int r0 = blockIdx.x * TR;
  if (threadIdx.x < 16) pair[threadIdx.x] = s.pair[threadIdx.x];
  for (int idx = threadIdx.x; idx < s.nl * W; idx += blockDim.x) {
    const int l = idx / W, cc = idx % W;
    const int j = r0 + (cc % TR);
    T v = czero<T>();
    if (j < s.half_r) v = x[__ldg(s.offl + l) + __ldg(s.offr + (cc / TR) * s.half_r + j)];
    tile[idx] = v;
  }
  __syncthreads();
  const int cc = threadIdx.x % W;
  const int h = cc / TR;
  const int j = r0 + (cc % TR);
  if (j >= s.half_r) return;  // no barrier below
  const int offr_c = __ldg(s.offr + h * s.half_r + j);
  for (int l = threadIdx.x / W; l < s.nl; l += blockDim.x / W) {
    T acc = czero<T>();
    const int k1 = __ldg(s.lptr + l + 1);
    for (int k = __ldg(s.lptr + l); k < k1; ++k) acc = cfma(__ldg(s.lval + k), tile[__ldg(s.lcol + k) * W + cc], acc);
    const int a = l >= s.half_l ? 1 : 0;
    const int lb = l - a * s.half_l;
    const int cb = cc - h * TR;
#pragma unroll
    for (int a2 = 0; a2 < 2; ++a2)
#pragma unroll
      for (int b2 = 0; b2 < 2; ++b2)
        acc = cfma(pair[(a * 2 + h) * 4 + a2 * 2 + b2], tile[(lb + a2 * s.half_l) * W + cb + b2 * TR], acc);
    y[__ldg(s.offl + l) + offr_c] = acc;
  }
}

template <class T, int TL, int MAXACC>
__global__ void __launch_bounds__(512) split_pass_b(SplitView<T> s, const T* __restrict__ in,
                                                    const T* __restrict__ ya, T* __restrict__ out, long long ld) {
  constexpr int CW = 32 / TL;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* tile = reinterpret_cast<T*>(smem_raw);
  const int nrp = s.nr | 1;
  const long long boff = (long long)blockIdx.y * ld;
  const T* x = in + boff;
  const int l0 = blockIdx.x * TL;
  const int rows = min(TL, s.nl - l0);
  for (int idx = threadIdx.x; idx < rows * s.nr; idx += blockDim.x) {
    const int lt = idx / s.nr, r = idx % s.nr;
    tile[lt * nrp + r] = x[__ldg(s.offl + l0 + lt) + __ldg(s.offr + r)];
  }
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  const int lt = lane % TL, cw = lane / TL;
  const int step = nwarps * CW;
  T acc[MAXACC];
#pragma unroll
  for (int q = 0; q < MAXACC; ++q) {
    acc[q] = czero<T>();
    const int r = warp * CW + cw + q * step;
    if (r < s.nr && lt < rows) {
      T v = czero<T>();
      const int k1 = __ldg(s.rptr + r + 1);
      for (int k = __ldg(s.rptr + r); k < k1; ++k) v = cfma(__ldg(s.rval + k), tile[lt * nrp + __ldg(s.rcol + k)], v);
      acc[q] = v;
    }
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < MAXACC; ++q) {
    const int r = warp * CW + cw + q * step;
    if (r < s.nr && lt < rows) tile[lt * nrp + r] = acc[q];
  }
  __syncthreads();
  const T* yA = ya + boff;
  T* o = out + boff;
  for (int idx = threadIdx.x; idx < rows * s.nr; idx += blockDim.x) {
    const int lt2 = idx / s.nr, r = idx % s.nr;
    const int addr = __ldg(s.offl + l0 + lt2) + __ldg(s.offr + r);
    o[addr] = cadd(tile[lt2 * nrp + r], yA[addr]);
  }
}

// ---------------------------------------------------------------------------
// Launch planning
// ---------------------------------------------------------------------------
int sm_count() {
  static std::mutex m;
  static std::vector<std::pair<int, int>> cache;  // (device, SM count)
  int dev = 0;
  check_cuda(cudaGetDevice(&dev), "cudaGetDevice");
  std::lock_guard<std::mutex> lock(m);
  for (const auto& c : cache)
    if (c.first == dev) return c.second;
  int count = 0;
  check_cuda(cudaDeviceGetAttribute(&count, cudaDevAttrMultiProcessorCount, dev), "cudaDeviceGetAttribute");
  cache.emplace_back(dev, count);
  return count;
}

static constexpr size_t kMaxSmem = 200 * 1024;

// Explicit cube-kernel variant (0 = heuristic), set by rpm_set_cube_tuning;
// one atomic word (a byte per field) so that a launch reads a consistent set.
struct CubeTuning {
  int ni_l, ni_r, tr, tl;
};
static std::atomic<unsigned> g_cube_tuning{0u};

static CubeTuning cube_tuning() {
  const unsigned v = g_cube_tuning.load(std::memory_order_relaxed);
  return CubeTuning{(int)(v & 0xffu), (int)((v >> 8) & 0xffu), (int)((v >> 16) & 0xffu), (int)(v >> 24)};
}

// Raise a kernel's dynamic shared-memory limit only when needed, so that
// launches recorded into a CUDA graph issue no attribute calls once warmed up.
// The attribute belongs to the device's context: the cache is per device.
template <class K>
static void ensure_smem(K kern, size_t bytes, const char* what) {
  struct Done {
    const void* kernel;
    int device;
    size_t bytes;
  };
  static std::mutex m;
  static std::vector<Done> done;
  int dev = 0;
  check_cuda(cudaGetDevice(&dev), "cudaGetDevice");
  const void* key = reinterpret_cast<const void*>(kern);
  std::lock_guard<std::mutex> lock(m);
  for (auto& d : done)
    if (d.kernel == key && d.device == dev) {
      if (d.bytes >= bytes) return;
      check_cuda(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes), what);
      d.bytes = bytes;
      return;
    }
  check_cuda(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes), what);
  done.push_back(Done{key, dev, bytes});
}

template <class T, int NI, int TR>
static bool try_cube_l(const HpsiArgs<T>& a, const CubePlan& p, T* ya, int batch, cudaStream_t st) {
  const int n_outer = NI == 1 ? p.n_outer_l1 : p.n_outer_l2;
  const size_t smem = (size_t)cube_smem_prefix<T>(p.tab_cap, n_outer, p.nl, 2 * TR) + (size_t)p.nl * 2 * TR * sizeof(T);
  if (smem > kMaxSmem) return false;
  auto kern = cube_pass_l<T, NI, TR>;
  ensure_smem(kern, smem, "cube L attr");
  dim3 grid((p.half_r + TR - 1) / TR, batch);
  kern<<<grid, 256, smem, st>>>(a, ya, p.tab_cap, n_outer);
  check_launch("cube_pass_l");
  return true;
}

template <class T, int NI, int TL>
static bool try_cube_r(const HpsiArgs<T>& a, const CubePlan& p, const T* ya, int batch, cudaStream_t st) {
  const int n_outer = NI == 1 ? p.n_outer_r1 : p.n_outer_r2;
  const size_t smem = (size_t)cube_smem_prefix<T>(p.tab_cap, n_outer, TL, p.nr) + (size_t)2 * TL * p.nr * sizeof(T);
  if (smem > kMaxSmem) return false;
  auto kern = cube_pass_r<T, NI, TL>;
  ensure_smem(kern, smem, "cube R attr");
  dim3 grid((p.nl + TL - 1) / TL, batch);
  kern<<<grid, 256, smem, st>>>(a, ya, p.tab_cap, n_outer);
  check_launch("cube_pass_r");
  return true;
}

// Column-tile width for pass L: as wide as shared memory allows, but narrow
// enough that small batches still produce about two CTAs per SM.
template <class T, int NI>
static void cube_l_dispatch(const HpsiArgs<T>& a, const CubePlan& p, T* ya, int batch, cudaStream_t st, int tuned_tr) {
  switch (tuned_tr) {  // explicit choice (autotuner); falls back to the heuristic if it cannot run
    case 8: if (try_cube_l<T, NI, 8>(a, p, ya, batch, st)) return; break;
    case 4: if (try_cube_l<T, NI, 4>(a, p, ya, batch, st)) return; break;
    case 2: if (try_cube_l<T, NI, 2>(a, p, ya, batch, st)) return; break;
    case 1: if (try_cube_l<T, NI, 1>(a, p, ya, batch, st)) return; break;
    default: break;
  }
  const int want = 2 * sm_count();
  auto tiles = [&](int tr) { return ((p.half_r + tr - 1) / tr) * batch; };
  if (tiles(8) >= want && try_cube_l<T, NI, 8>(a, p, ya, batch, st)) return;
  if (tiles(4) >= want && try_cube_l<T, NI, 4>(a, p, ya, batch, st)) return;
  if (tiles(2) >= want && try_cube_l<T, NI, 2>(a, p, ya, batch, st)) return;
  if (try_cube_l<T, NI, 1>(a, p, ya, batch, st)) return;
  fail(RPM_E_UNSUPPORTED, "radical group too large for the cube kernel");
}

template <class T, int NI>
static void cube_r_dispatch(const HpsiArgs<T>& a, const CubePlan& p, const T* ya, int batch, cudaStream_t st,
                            int tuned_tl) {
  switch (tuned_tl) {
    case 16: if (try_cube_r<T, NI, 16>(a, p, ya, batch, st)) return; break;
    case 8: if (try_cube_r<T, NI, 8>(a, p, ya, batch, st)) return; break;
    case 4: if (try_cube_r<T, NI, 4>(a, p, ya, batch, st)) return; break;
    case 2: if (try_cube_r<T, NI, 2>(a, p, ya, batch, st)) return; break;
    case 1: if (try_cube_r<T, NI, 1>(a, p, ya, batch, st)) return; break;
    default: break;
  }
  const int want = 2 * sm_count();
  auto ctas = [&](int tl) { return ((p.nl + tl - 1) / tl) * batch; };
  if (ctas(16) >= want && try_cube_r<T, NI, 16>(a, p, ya, batch, st)) return;
  if (ctas(8) >= want && try_cube_r<T, NI, 8>(a, p, ya, batch, st)) return;
  if (ctas(4) >= want && try_cube_r<T, NI, 4>(a, p, ya, batch, st)) return;
  if (try_cube_r<T, NI, 2>(a, p, ya, batch, st)) return;
  if (try_cube_r<T, NI, 1>(a, p, ya, batch, st)) return;
  fail(RPM_E_UNSUPPORTED, "radical group too large for the cube kernel");
}

template <class T>
void launch_cube(const HpsiArgs<T>& a, const CubePlan& p, T* ya, int batch, cudaStream_t st) {
  const CubeTuning tu = cube_tuning();
  const bool tuned = tu.ni_l || tu.ni_r || tu.tr || tu.tl;
  if (!tuned && launch_cube_fast<T>(a, p, ya, batch, st)) return;
  const int ni_l = tu.ni_l > 0 ? std::min(tu.ni_l, p.ni_l) : p.ni_l;
  const int ni_r = tu.ni_r > 0 ? std::min(tu.ni_r, p.ni_r) : p.ni_r;
  if (ni_l >= 2) {
    HpsiArgs<T> al = a;
    al.dot_part = nullptr;
    cube_l_dispatch<T, 2>(al, p, ya, batch, st, tu.tr);
  } else {
    HpsiArgs<T> al = a;
    al.dot_part = nullptr;
    cube_l_dispatch<T, 1>(al, p, ya, batch, st, tu.tr);
  }
  if (ni_r >= 2) {
    cube_r_dispatch<T, 2>(a, p, ya, batch, st, tu.tl);
  } else {
    cube_r_dispatch<T, 1>(a, p, ya, batch, st, tu.tl);
  }
}

template <class T, int TR>
static bool try_pass_a(const SplitView<T>& s, const T* in, T* ya, int batch, long long ld, cudaStream_t stream) {
  const size_t smem = (16 + (size_t)s.nl * 2 * TR) * sizeof(T);
  if (smem > kMaxSmem) return false;
  auto kern = split_pass_a<T, TR>;
  check_cuda(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
             "cudaFuncSetAttribute(pass A)");
  dim3 grid((s.half_r + TR - 1) / TR, batch);
  kern<<<grid, 512, smem, stream>>>(s, in, ya, ld);
  check_launch("split_pass_a");
  return true;
}

template <class T, int TL, int MAXACC>
static bool try_pass_b(const SplitView<T>& s, const T* in, const T* ya, T* out, int batch, long long ld,
                       cudaStream_t stream) {
  constexpr int CW = 32 / TL;
  const int threads = 512;
  if (s.nr > (threads / 32) * CW * MAXACC) return false;
  const size_t smem = (size_t)TL * (s.nr | 1) * sizeof(T);
  if (smem > kMaxSmem) return false;
  auto kern = split_pass_b<T, TL, MAXACC>;
  check_cuda(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
             "cudaFuncSetAttribute(pass B)");
  dim3 grid((s.nl + TL - 1) / TL, batch);
  kern<<<grid, threads, smem, stream>>>(s, in, ya, out, ld);
  check_launch("split_pass_b");
  return true;
}

template <class T>
static void launch_generic(const GenericView<T>& g, const T* in, T* out, int batch, long long ld, cudaStream_t stream) {
  const size_t smem = (size_t)g.nterms * sizeof(TermMeta);
  if (smem > 48 * 1024) fail(RPM_E_UNSUPPORTED, "too many local terms for the generic kernel");
  const int threads = 256;
  int blocks = (int)std::min<long long>((g.n + threads - 1) / threads, 8LL * sm_count());
  blocks = std::max(blocks, 1);
  dim3 grid(blocks, batch);
  hpsi_generic_kernel<T><<<grid, threads, smem, stream>>>(g, in, out, ld);
  check_launch("hpsi_generic_kernel");
}

template <class T> static const SplitView<T>& split_of(rpm_system* sys);
template <> const SplitView<double2>& split_of<double2>(rpm_system* sys) { return sys->split64; }
template <> const SplitView<float2>& split_of<float2>(rpm_system* sys) { return sys->split32; }
template <class T> static const GenericView<T>& generic_of(rpm_system* sys);
template <> const GenericView<double2>& generic_of<double2>(rpm_system* sys) { return sys->gen64; }
template <> const GenericView<float2>& generic_of<float2>(rpm_system* sys) { return sys->gen32; }
template <class T> const CubeView<T>* cube_dev_of(rpm_system* sys);
template <> const CubeView<double2>* cube_dev_of<double2>(rpm_system* sys) { return sys->cube64_dev; }
template <> const CubeView<float2>* cube_dev_of<float2>(rpm_system* sys) { return sys->cube32_dev; }

bool same_cube_shape(const rpm_system* x, const rpm_system* y) {
  if (x == y) return true;
  if (x->n != y->n || x->nl != y->nl || x->nr != y->nr || x->cube_l.K != y->cube_l.K || x->cube_r.K != y->cube_r.K)
    return false;
  for (int k = 0; k < x->cube_l.K; ++k)
    if (x->cube_l.dim[k] != y->cube_l.dim[k]) return false;
  for (int k = 0; k < x->cube_r.K; ++k)
    if (x->cube_r.dim[k] != y->cube_r.dim[k]) return false;
  return x->offl == y->offl && x->offr == y->offr;
}

// One launch plan covers systems of one shape only: every size, table cap
// and inner-digit count of the plan is then exactly each member's own, so no
// per-view quantity of a launch can differ from the plan it was sized by.
// Batches of uneven sizes launch one plan per shape group.
CubePlan cube_plan(rpm_system* const* systems, int nsys) {
  CubePlan p{};
  p.ni_l = p.ni_r = 2;
  for (int k = 0; k < nsys; ++k) {
    const rpm_system* s = systems[k];
    if (!s->cube) fail(RPM_E_UNSUPPORTED, "system has no cube form");
    if (k > 0 && !same_cube_shape(systems[0], s))
      fail(RPM_E_UNSUPPORTED, "a cube launch plan needs systems of one shape (same dimensions, digits and layout)");
    p.nl = std::max(p.nl, s->nl);
    p.nr = std::max(p.nr, s->nr);
    p.half_r = std::max(p.half_r, s->half_r);
    p.tab_cap = std::max(p.tab_cap, std::max(s->cube_l.ntab, s->cube_r.ntab));
    p.ni_l = std::min(p.ni_l, s->cube64.inner_l);
    p.ni_r = std::min(p.ni_r, s->cube64.inner_r);
    auto outer = [](const CubeSide& side, int ni) {
      int n = 1;
      for (int k = 0; k < side.K - ni; ++k) n *= side.dim[k];
      return n;
    };
    p.n_outer_l1 = std::max(p.n_outer_l1, outer(s->cube_l, 1));
    p.n_outer_l2 = std::max(p.n_outer_l2, outer(s->cube_l, 2));
    p.n_outer_r1 = std::max(p.n_outer_r1, outer(s->cube_r, 1));
    p.n_outer_r2 = std::max(p.n_outer_r2, outer(s->cube_r, 2));
    fast_plan_add(p, s, k == 0);
  }
  p.tab_cap = (p.tab_cap + 1) & ~1;
  if (p.ni_l < 1 || p.ni_r < 1) fail(RPM_E_UNSUPPORTED, "cube kernels need a trailing spin-1/2 digit per radical");
  return p;
}

template <class T>
void launch_hpsi(rpm_system* sys, const T* in, T* out, int batch, long long ld, cudaStream_t stream) {
  if (!sys->on_device) fail(RPM_E_INVALID, "system was created host-only");
  if (batch < 1) return;
  if (sys->split) {
    T* ya = static_cast<T*>(system_scratch(sys, SLOT_YA, (size_t)batch * ld * sizeof(T)));
    if (sys->cube && sys->cube64.inner_l >= 1 && sys->cube64.inner_r >= 1) {
      HpsiArgs<T> a{};
      a.in = in;
      a.out = out;
      a.ld = ld;
      a.views = cube_dev_of<T>(sys);
      rpm_system* one[1] = {sys};
      launch_cube<T>(a, cube_plan(one, 1), ya, batch, stream);
      return;
    }
    const SplitView<T>& s = split_of<T>(sys);
    bool a_ok = try_pass_a<T, 4>(s, in, ya, batch, ld, stream) || try_pass_a<T, 2>(s, in, ya, batch, ld, stream);
    if (a_ok) {
      const bool b_ok = try_pass_b<T, 4, 8>(s, in, ya, out, batch, ld, stream) ||
                        try_pass_b<T, 2, 4>(s, in, ya, out, batch, ld, stream);
      if (b_ok) return;
    }
  }
  launch_generic<T>(generic_of<T>(sys), in, out, batch, ld, stream);
}

template <class T>
void launch_hpsi_scaled(rpm_system* sys, const T* in, T* out, int batch, long long ld, const double* scale_dev,
                        cudaStream_t stream) {
  if (!sys->on_device) fail(RPM_E_INVALID, "system was created host-only");
  if (!sys->split || !sys->cube || sys->cube64.inner_l < 1 || sys->cube64.inner_r < 1 || sys->non_hermitian)
    fail(RPM_E_UNSUPPORTED,
         "scaled H psi needs a Hermitian radical-split system with a trailing spin-1/2 digit per radical");
  if (batch < 1) return;
  T* ya = static_cast<T*>(system_scratch(sys, SLOT_YA, (size_t)batch * ld * sizeof(T)));
  HpsiArgs<T> a{};
  a.in = in;
  a.out = out;
  a.ld = ld;
  a.in_scale = scale_dev;
  a.scale_stride = 0;
  a.views = cube_dev_of<T>(sys);
  rpm_system* one[1] = {sys};
  launch_cube<T>(a, cube_plan(one, 1), ya, batch, stream);
}

template void launch_hpsi_scaled<float2>(rpm_system*, const float2*, float2*, int, long long, const double*,
                                         cudaStream_t);
template void launch_hpsi_scaled<double2>(rpm_system*, const double2*, double2*, int, long long, const double*,
                                          cudaStream_t);
template void launch_hpsi<double2>(rpm_system*, const double2*, double2*, int, long long, cudaStream_t);
template void launch_hpsi<float2>(rpm_system*, const float2*, float2*, int, long long, cudaStream_t);
template void launch_cube<double2>(const HpsiArgs<double2>&, const CubePlan&, double2*, int, cudaStream_t);
template void launch_cube<float2>(const HpsiArgs<float2>&, const CubePlan&, float2*, int, cudaStream_t);

}  // namespace rpm

extern "C" int rpm_set_cube_tuning(int ni_l, int ni_r, int tr, int tl) {
  return rpm::guarded([&] {
    auto ok = [](int v, std::initializer_list<int> allowed) {
      for (int a : allowed)
        if (v == a) return true;
      return false;
    };
    if (!ok(ni_l, {0, 1, 2}) || !ok(ni_r, {0, 1, 2}) || !ok(tr, {0, 1, 2, 4, 8}) || !ok(tl, {0, 1, 2, 4, 8, 16}))
      rpm::fail(RPM_E_INVALID, "cube tuning: ni in {0,1,2}, tr in {0,1,2,4,8}, tl in {0,1,2,4,8,16}");
    rpm::g_cube_tuning.store((unsigned)ni_l | ((unsigned)ni_r << 8) | ((unsigned)tr << 16) | ((unsigned)tl << 24));
  });
}

extern "C" int rpm_hpsi(rpm_system* sys, int precision, const void* psi_dev, void* out_dev, int batch, long long ld,
                        void* stream) {
  return rpm::guarded([&] {
    if (!sys) rpm::fail(RPM_E_INVALID, "system is NULL");
    if (!psi_dev || !out_dev) rpm::fail(RPM_E_INVALID, "NULL state pointer");
    if (batch < 0 || (batch > 0 && ld < sys->n)) rpm::fail(RPM_E_INVALID, "invalid batch or leading dimension");
    if (psi_dev == out_dev) rpm::fail(RPM_E_INVALID, "H psi cannot run in place");
    auto st = static_cast<cudaStream_t>(stream);
    if (precision == RPM_PREC_C128) {
      rpm::launch_hpsi<double2>(sys, static_cast<const double2*>(psi_dev), static_cast<double2*>(out_dev), batch, ld, st);
    } else if (precision == RPM_PREC_C64) {
      rpm::launch_hpsi<float2>(sys, static_cast<const float2*>(psi_dev), static_cast<float2*>(out_dev), batch, ld, st);
    } else {
      rpm::fail(RPM_E_INVALID, "precision must be 64 or 128");
    }
  });
}

// ---------------------------------------------------------------------------
// Allocation-free H psi (rpm_hpsi_noalloc)
//
// For callers that must not allocate device memory while they run: host
// frameworks whose run loop forbids cudaMalloc (their memory comes from a
// pool or arena they own, and a cudaMalloc would synchronise the device and
// take memory outside their accounting), and embedded runtimes with a fixed
// memory budget decided at start-up.  rpm_hpsi grows a per-system cudaMalloc'd buffer
// for the only scratch the radical-split action needs, the partial result
// (batch x ld elements).  This variant uses a fixed array compiled into the
// library instead, so every GPU that loads the library holds those bytes
// until the process exits.
// ---------------------------------------------------------------------------
#include <mutex>

namespace rpm {

constexpr size_t kNoAllocScratchBytes = (size_t)4 << 20;  // 4 MiB per GPU
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kNoAllocMaxDevices = 64;
static void* g_noalloc_address[kNoAllocMaxDevices];
static std::mutex g_noalloc_mutex;

// Device address of g_noalloc_scratch on the current device.  In host code
// the array's name is only a host-side stand-in, so the address is looked up
// once per device, with that device current, and cached for the life of the
// device's primary context: after cudaDeviceReset the cached address is
// stale, so a process that resets a device must not call rpm_hpsi_noalloc on
// it again.
static void* noalloc_scratch() {
  int dev = 0;
  check_cuda(cudaGetDevice(&dev), "cudaGetDevice");
  if (dev < 0 || dev >= kNoAllocMaxDevices) fail(RPM_E_UNSUPPORTED, "rpm_hpsi_noalloc supports device ordinals 0..63");
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if (!g_noalloc_address[dev]) {
    void* p = nullptr;
    check_cuda(cudaGetSymbolAddress(&p, g_noalloc_scratch), "cudaGetSymbolAddress(no-alloc scratch)");
    g_noalloc_address[dev] = p;
  }
  return g_noalloc_address[dev];
}

template <class T>
static void launch_hpsi_noalloc(rpm_system* sys, const T* in, T* out, int batch, long long ld, cudaStream_t stream) {
  if (!sys->on_device) fail(RPM_E_INVALID, "system was created host-only");
  if (batch < 1) return;
  if (!sys->split) {  // the per-term kernel needs no scratch
    launch_generic<T>(generic_of<T>(sys), in, out, batch, ld, stream);
    return;
  }
  const size_t need = (size_t)batch * (size_t)ld * sizeof(T);
  if (need > kNoAllocScratchBytes) {
    fail(RPM_E_UNSUPPORTED, "rpm_hpsi_noalloc: batch x ld x element size = " + std::to_string(need) +
                                " bytes exceeds its fixed 4 MiB scratch; use rpm_hpsi or a smaller batch");
  }
  T* ya = static_cast<T*>(noalloc_scratch());
  // the kernel choice of launch_hpsi: cube form, else the CSR passes, else
  // the per-term kernel (which needs no scratch)
  if (sys->cube && sys->cube64.inner_l >= 1 && sys->cube64.inner_r >= 1) {
    HpsiArgs<T> a{};
    a.in = in;
    a.out = out;
    a.ld = ld;
    a.views = cube_dev_of<T>(sys);
    rpm_system* one[1] = {sys};
    launch_cube<T>(a, cube_plan(one, 1), ya, batch, stream);
    return;
  }
  const SplitView<T>& s = split_of<T>(sys);
  const bool a_ok = try_pass_a<T, 4>(s, in, ya, batch, ld, stream) || try_pass_a<T, 2>(s, in, ya, batch, ld, stream);
  if (a_ok && (try_pass_b<T, 4, 8>(s, in, ya, out, batch, ld, stream) ||
               try_pass_b<T, 2, 4>(s, in, ya, out, batch, ld, stream)))
    return;
  launch_generic<T>(generic_of<T>(sys), in, out, batch, ld, stream);
}

}  // namespace rpm

extern "C" int rpm_hpsi_noalloc(rpm_system* sys, int precision, const void* psi_dev, void* out_dev, int batch,
                                long long ld, void* stream) {
  return rpm::guarded([&] {
    if (!sys) rpm::fail(RPM_E_INVALID, "system is NULL");
    if (!psi_dev || !out_dev) rpm::fail(RPM_E_INVALID, "NULL state pointer");
    if (batch < 0 || (batch > 0 && ld < sys->n)) rpm::fail(RPM_E_INVALID, "invalid batch or leading dimension");
    if (psi_dev == out_dev) rpm::fail(RPM_E_INVALID, "H psi cannot run in place");
    auto st = static_cast<cudaStream_t>(stream);
    if (precision == RPM_PREC_C128) {
      rpm::launch_hpsi_noalloc<double2>(sys, static_cast<const double2*>(psi_dev), static_cast<double2*>(out_dev),
                                        batch, ld, st);
    } else if (precision == RPM_PREC_C64) {
      rpm::launch_hpsi_noalloc<float2>(sys, static_cast<const float2*>(psi_dev), static_cast<float2*>(out_dev), batch,
                                       ld, st);
    } else {
      rpm::fail(RPM_E_INVALID, "precision must be 64 or 128");
    }
  });
}
