// Adjoint sweep for gradients of the singlet yield (rpm_adjoint_*).
//
// The yield on an observation grid t_k = t_0 + k dt is
//   Phi = sum_k w_k <psi_k| P_S |psi_k>,   psi_{k+1} = U_k psi_k,
// with U_k = exp(-i H_k dt) and w_k the Simpson weights times the Haberkorn
// factor exp(-t_k / tau) / tau (equal rates: the decay is a scalar).  The
// adjoint state obeys lambda_K = w_K P_S psi_K and
//   lambda_k = U_k^dag lambda_{k+1} + w_k P_S psi_k,
// and for a parameter p with dH_k/dp = D_k
//   dPhi/dp = sum_k 2 Im int_0^dt <lambda(tau)| D_k |psi(tau)> dtau,
//   lambda(tau) = exp(+i H (dt - tau)) lambda_{k+1},
//   psi(tau)    = exp(+i H (dt - tau)) psi_{k+1}.
//
// One backward sweep walks a run of intervals.  Per interval it builds the
// Taylor basis u_j = (dt H)^j x / j! (j <= degree) of the pair
// x = [lambda_{k+1}; psi_{k+1}] (one batched H psi launch of 2B vectors per
// term, the dt / (j + 1) factor folded into the load), then one kernel forms
// lambda and psi at the Gauss-Legendre nodes of the interval and at its
// start, accumulates the electron-pair transition density
//   M_ab += dt w_q sum_i conj(lambda_q[a, i]) psi_q[b, i]   (a, b = 2 eA + eB)
// (contracted with an electron-pair operator it gives a field derivative),
// and writes psi_k and lambda_k = lambda_k^- + w_k P_S psi_k in FP64 plus the
// next interval's u_0.  Four adjacent lanes hold the four electron-pair
// components of one nuclear index and exchange them by warp shuffles (for M
// and for P_S).  A derivative system D (an operator on nuclei, e.g. the
// quadrupoles) is applied to the psi nodes and <lambda_q| D psi_q> is
// accumulated.  Because lambda(tau) and psi(tau) evolve under the same H,
// <lambda(tau)| H |psi(tau)> is constant over an interval; it is accumulated
// once per interval in FP64 (dt <lambda_{k+1}| H psi_{k+1}>) for derivative
// operators that are most of H (the hyperfine scale), whose node sandwich
// would lose its small imaginary part to rounding.
//
// The basis precision is complex64 or complex128 (the state between
// intervals is always FP64).  The gradient's sensitivity to state errors
// grows with ||dH/dp|| times the horizon, so derivatives with respect to the
// hyperfine scale need the complex128 basis (and FP64-accurate checkpoints);
// field derivatives are well conditioned in complex64.
//
// The forward sweep (rpm_adjoint_forward) propagates psi with the same
// Taylor stepping (coefficients (-i)^j) and records P_S at each new grid
// point; with the complex128 basis it gives FP64-accurate checkpoints and
// populations on a fixed schedule (smooth in the parameters).
#include "hpsi.cuh"

#include <algorithm>
#include <cmath>
#include <complex>
#include <vector>

namespace rpm {

constexpr int kAdjMaxDegree = 24;
constexpr int kAdjMaxNodes = 4;
constexpr int kAdjThreads = 256;
constexpr int kAdjBlocksPerVector = 32;
constexpr int kAdjWarps = kAdjThreads / 32;

template <class T>
struct AdjCoef {
  T node[kAdjMaxNodes][kAdjMaxDegree + 1];  // (i (1 - x_q))^j
  T start[kAdjMaxDegree + 1];               // i^j (backwards) or (-i)^j (forwards)
  double weight[kAdjMaxNodes];              // dt * Gauss-Legendre weight
};

template <class T>
__device__ __forceinline__ T cconj_mul(T a, T b) {  // conj(a) * b
  T r;
  r.x = a.x * b.x + a.y * b.y;
  r.y = a.x * b.y - a.y * b.x;
  return r;
}
template <class T>
__device__ __forceinline__ T shfl_c(T v, int src) {
  v.x = __shfl_sync(0xffffffffu, v.x, src);
  v.y = __shfl_sync(0xffffffffu, v.y, src);
  return v;
}
template <class T>
__device__ __forceinline__ double norm2(T v) {
  return (double)v.x * v.x + (double)v.y * v.y;
}

__global__ void k_adj_set_scales(double* scales, double dt, int degree) {
  const int j = threadIdx.x;
  if (j < degree) scales[j] = dt / (double)(j + 1);
}

// dst[b] = (T) x[b] for B vectors (first n elements).
template <class T>
__global__ void k_adj_convert(const double2* __restrict__ x, T* __restrict__ dst, int B, long long n, long long ld) {
  const int b = blockIdx.y;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    dst[(long long)b * ld + i] = from_d2<T>(x[(long long)b * ld + i]);
}

// lambda += w P_S psi; P_S acts on the electron-pair index e = 2 eA + eB of
// the state (leading axes): (P_S psi)[1] = (psi[1] - psi[2]) / 2 = -(P_S psi)[2].
__global__ void k_adj_source(const double2* __restrict__ xp, double2* __restrict__ xl, int B, long long n4,
                             long long ld, double w) {
  const int b = blockIdx.y;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n4; i += (long long)gridDim.x * blockDim.x) {
    const double2* p = xp + (long long)b * ld;
    double2* l = xl + (long long)b * ld;
    const double2 p1 = p[n4 + i], p2 = p[2 * n4 + i];
    const double sx = 0.5 * w * (p1.x - p2.x), sy = 0.5 * w * (p1.y - p2.y);
    double2 l1 = l[n4 + i], l2 = l[2 * n4 + i];
    l1.x += sx;
    l1.y += sy;
    l2.x -= sx;
    l2.y -= sy;
    l[n4 + i] = l1;
    l[2 * n4 + i] = l2;
  }
}

// One backward interval (see the file comment).  U: degree + 1 slots of 2B
// vectors (lambda part first); slot 0 is rewritten with the new [lambda_k; psi_k].
template <class T, int Q>
__global__ void __launch_bounds__(kAdjThreads) k_adj_combine(
    T* U, double2* __restrict__ xl, double2* __restrict__ xp, T* __restrict__ nodes_p, T* __restrict__ nodes_l,
    double* __restrict__ density, int dens_stride, double* __restrict__ tail, const AdjCoef<T> cf, int degree, int B,
    long long ld, long long n4, double src_weight) {
  using R = typename Real<T>::type;
  const int b = blockIdx.y;
  const int lane = threadIdx.x & 31, e = threadIdx.x & 3, base = lane & ~3;
  const long long slot = 2LL * B * ld;
  T* ul0 = U + (long long)b * ld;
  T* up0 = U + (long long)(B + b) * ld;
  double m[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) m[k] = 0.0;
  double tl[2] = {0.0, 0.0};
  const long long per_round = (long long)gridDim.x * blockDim.x / 4;
  const long long first = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 2;
  const long long rounds = (n4 + per_round - 1) / per_round;
  for (long long r = 0; r < rounds; ++r) {
    const long long i = first + r * per_round;
    const bool act = i < n4;
    const long long at = (long long)e * n4 + (act ? i : 0);
    T lq[Q], pq[Q], ls = czero<T>(), ps = czero<T>();
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      lq[q] = czero<T>();
      pq[q] = czero<T>();
    }
    for (int j = 0; j <= degree; ++j) {
      const T a = act ? ul0[(long long)j * slot + at] : czero<T>();
      const T c = act ? up0[(long long)j * slot + at] : czero<T>();
#pragma unroll
      for (int q = 0; q < Q; ++q) {
        lq[q] = cfma(cf.node[q][j], a, lq[q]);
        pq[q] = cfma(cf.node[q][j], c, pq[q]);
      }
      if (j >= 1) {
        ls = cfma(cf.start[j], a, ls);
        ps = cfma(cf.start[j], c, ps);
      }
      if (j == 0) tl[1] += norm2(c);
      if (j == degree) tl[0] += norm2(c);
    }
    // row e of M: conj(lambda_q[e]) psi_q[c] for c = 0..3 (psi_q[c] from lane base + c)
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      T lw = lq[q];
      lw.x = (R)(lw.x * cf.weight[q]);
      lw.y = (R)(lw.y * cf.weight[q]);
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        const T t = cconj_mul(lw, shfl_c(pq[q], base + c));
        m[2 * c] += (double)t.x;
        m[2 * c + 1] += (double)t.y;
      }
    }
    if (nodes_p && act) {
#pragma unroll
      for (int q = 0; q < Q; ++q) {
        nodes_p[((long long)q * B + b) * ld + at] = pq[q];
        nodes_l[((long long)q * B + b) * ld + at] = lq[q];
      }
    }
    double2 p = act ? xp[(long long)b * ld + at] : make_double2(0.0, 0.0);
    double2 l = act ? xl[(long long)b * ld + at] : make_double2(0.0, 0.0);
    p.x += (double)ps.x;
    p.y += (double)ps.y;
    l.x += (double)ls.x;
    l.y += (double)ls.y;
    const double2 p1 = shfl_c(p, base + 1), p2 = shfl_c(p, base + 2);
    const double sx = 0.5 * src_weight * (p1.x - p2.x), sy = 0.5 * src_weight * (p1.y - p2.y);
    if (e == 1) {
      l.x += sx;
      l.y += sy;
    } else if (e == 2) {
      l.x -= sx;
      l.y -= sy;
    }
    if (act) {
      xp[(long long)b * ld + at] = p;
      xl[(long long)b * ld + at] = l;
      ul0[at] = from_d2<T>(l);
      up0[at] = from_d2<T>(p);
    }
  }
  // reduce: M rows over lanes with the same e, the Taylor norms over the warp
#pragma unroll
  for (int k = 0; k < 8; ++k)
    for (int o = 4; o < 32; o <<= 1) m[k] += __shfl_xor_sync(0xffffffffu, m[k], o);
  for (int o = 1; o < 32; o <<= 1) {
    tl[0] += __shfl_xor_sync(0xffffffffu, tl[0], o);
    tl[1] += __shfl_xor_sync(0xffffffffu, tl[1], o);
  }
  __shared__ double part[kAdjWarps][34];
  const int warp = threadIdx.x >> 5;
  if (lane < 4) {
#pragma unroll
    for (int k = 0; k < 8; ++k) part[warp][lane * 8 + k] = m[k];
  }
  if (lane == 0) {
    part[warp][32] = tl[0];
    part[warp][33] = tl[1];
  }
  __syncthreads();
  if (threadIdx.x < 34) {
    double s = 0.0;
    for (int w = 0; w < kAdjWarps; ++w) s += part[w][threadIdx.x];
    if (threadIdx.x < 32) atomicAdd(density + (long long)b * dens_stride + threadIdx.x, s);
    else atomicAdd(tail + 2 * b + (threadIdx.x - 32), s);
  }
}

// One forward interval: psi_{k+1} = psi_k + sum_{j>=1} (-i)^j u_j (FP64),
// u_0 <- (T) psi_{k+1}, P_S(psi_{k+1}) added to pops[b * pop_ld].
template <class T>
__global__ void __launch_bounds__(kAdjThreads) k_adj_forward(T* U, double2* __restrict__ xp, double* __restrict__ pops,
                                                              long long pop_ld, double* __restrict__ tail,
                                                              const AdjCoef<T> cf, int degree, int B, long long ld,
                                                              long long n4) {
  const int b = blockIdx.y;
  const int lane = threadIdx.x & 31, e = threadIdx.x & 3, base = lane & ~3;
  const long long slot = 2LL * B * ld;
  T* up0 = U + (long long)b * ld;
  double pop = 0.0, tl[2] = {0.0, 0.0};
  const long long per_round = (long long)gridDim.x * blockDim.x / 4;
  const long long first = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 2;
  const long long rounds = (n4 + per_round - 1) / per_round;
  for (long long r = 0; r < rounds; ++r) {
    const long long i = first + r * per_round;
    const bool act = i < n4;
    const long long at = (long long)e * n4 + (act ? i : 0);
    T ps = czero<T>();
    for (int j = 0; j <= degree; ++j) {
      const T c = act ? up0[(long long)j * slot + at] : czero<T>();
      if (j >= 1) ps = cfma(cf.start[j], c, ps);
      if (j == 0) tl[1] += norm2(c);
      if (j == degree) tl[0] += norm2(c);
    }
    double2 p = act ? xp[(long long)b * ld + at] : make_double2(0.0, 0.0);
    p.x += (double)ps.x;
    p.y += (double)ps.y;
    const double2 p2 = shfl_c(p, base + 2);
    if (e == 1) pop += 0.5 * ((p.x - p2.x) * (p.x - p2.x) + (p.y - p2.y) * (p.y - p2.y));
    if (act) {
      xp[(long long)b * ld + at] = p;
      up0[at] = from_d2<T>(p);
    }
  }
  for (int o = 1; o < 32; o <<= 1) {
    pop += __shfl_xor_sync(0xffffffffu, pop, o);
    tl[0] += __shfl_xor_sync(0xffffffffu, tl[0], o);
    tl[1] += __shfl_xor_sync(0xffffffffu, tl[1], o);
  }
  __shared__ double part[kAdjWarps][3];
  const int warp = threadIdx.x >> 5;
  if (lane == 0) {
    part[warp][0] = pop;
    part[warp][1] = tl[0];
    part[warp][2] = tl[1];
  }
  __syncthreads();
  if (threadIdx.x < 3) {
    double s = 0.0;
    for (int w = 0; w < kAdjWarps; ++w) s += part[w][threadIdx.x];
    if (threadIdx.x == 0) atomicAdd(pops + (long long)b * pop_ld, s);
    else atomicAdd(tail + 2 * b + (threadIdx.x - 1), s);
  }
}

// S[b] += sum_q w_q <lambda_q[b] | out_q[b]>  (FP64 accumulation)
template <class T>
__global__ void __launch_bounds__(kAdjThreads) k_adj_dots(const T* __restrict__ nodes_l, const T* __restrict__ outs,
                                                           const AdjCoef<T> cf, int Q, int B, long long n, long long ld,
                                                           double* __restrict__ s, int s_stride) {
  const int b = blockIdx.y;
  double re = 0.0, im = 0.0;
  for (int q = 0; q < Q; ++q) {
    const T* l = nodes_l + ((long long)q * B + b) * ld;
    const T* o = outs + ((long long)q * B + b) * ld;
    double qr = 0.0, qi = 0.0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
      const T t = cconj_mul(l[i], o[i]);
      qr += (double)t.x;
      qi += (double)t.y;
    }
    re += cf.weight[q] * qr;
    im += cf.weight[q] * qi;
  }
  for (int o = 16; o > 0; o >>= 1) {
    re += __shfl_xor_sync(0xffffffffu, re, o);
    im += __shfl_xor_sync(0xffffffffu, im, o);
  }
  __shared__ double part[kAdjWarps][2];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) {
    part[warp][0] = re;
    part[warp][1] = im;
  }
  __syncthreads();
  if (threadIdx.x < 2) {
    double t = 0.0;
    for (int w = 0; w < kAdjWarps; ++w) t += part[w][threadIdx.x];
    atomicAdd(s + (long long)b * s_stride + threadIdx.x, t);
  }
}

// E[b] += dt <lambda[b] | (H psi)[b]>  (FP64 states and product)
__global__ void __launch_bounds__(kAdjThreads) k_adj_energy(const double2* __restrict__ xl,
                                                            const double2* __restrict__ hp, int B, long long n,
                                                            long long ld, double dt, double* __restrict__ e,
                                                            int e_stride) {
  const int b = blockIdx.y;
  double re = 0.0, im = 0.0;
  const double2* l = xl + (long long)b * ld;
  const double2* h = hp + (long long)b * ld;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double2 a = l[i], c = h[i];
    re = fma(a.x, c.x, fma(a.y, c.y, re));
    im = fma(a.x, c.y, fma(-a.y, c.x, im));
  }
  for (int o = 16; o > 0; o >>= 1) {
    re += __shfl_xor_sync(0xffffffffu, re, o);
    im += __shfl_xor_sync(0xffffffffu, im, o);
  }
  __shared__ double part[kAdjWarps][2];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) {
    part[warp][0] = re;
    part[warp][1] = im;
  }
  __syncthreads();
  if (threadIdx.x < 2) {
    double s = 0.0;
    for (int w = 0; w < kAdjWarps; ++w) s += part[w][threadIdx.x];
    atomicAdd(e + (long long)b * e_stride + threadIdx.x, dt * s);
  }
}

}  // namespace rpm

using namespace rpm;

struct rpm_adjoint {
  int B = 0;
  long long n = 0, ld = 0;
  int degree = 0, nodes = 0, precision = 0;
  int device = -1;
  size_t elem = 0;             // bytes per basis element
  void* U = nullptr;           // (degree + 1) x 2B x ld basis elements
  void* node_p = nullptr;      // nodes x B x ld
  void* node_l = nullptr;
  void* node_out = nullptr;
  double2* hpsi64 = nullptr;   // B x ld: H psi_{k+1} in FP64
  double* scales = nullptr;    // degree
  double* tail = nullptr;      // tail_cap doubles
  size_t tail_cap = 0;
  std::vector<double> tail_host;
};

namespace {

void gauss_legendre(int q, double* x, double* w) {
  // nodes on [0, 1], weights summing to one
  switch (q) {
    case 1:
      x[0] = 0.5;
      w[0] = 1.0;
      break;
    case 2: {
      const double d = 0.5 / std::sqrt(3.0);
      x[0] = 0.5 - d;
      x[1] = 0.5 + d;
      w[0] = w[1] = 0.5;
      break;
    }
    case 3: {
      const double d = 0.5 * std::sqrt(0.6);
      x[0] = 0.5 - d;
      x[1] = 0.5;
      x[2] = 0.5 + d;
      w[0] = w[2] = 5.0 / 18.0;
      w[1] = 8.0 / 18.0;
      break;
    }
    default: {
      const double a = std::sqrt(3.0 / 7.0 - 2.0 / 7.0 * std::sqrt(1.2));
      const double c = std::sqrt(3.0 / 7.0 + 2.0 / 7.0 * std::sqrt(1.2));
      const double wa = (18.0 + std::sqrt(30.0)) / 36.0, wc = (18.0 - std::sqrt(30.0)) / 36.0;
      x[0] = 0.5 * (1 - c);
      x[1] = 0.5 * (1 - a);
      x[2] = 0.5 * (1 + a);
      x[3] = 0.5 * (1 + c);
      w[0] = w[3] = 0.5 * wc;
      w[1] = w[2] = 0.5 * wa;
      break;
    }
  }
}

template <class T>
T tcomplex(std::complex<double> z) {
  T v;
  v.x = (typename Real<T>::type)z.real();
  v.y = (typename Real<T>::type)z.imag();
  return v;
}

// direction +1: backward (nodes and start coefficients i^j); -1: forward ((-i)^j)
template <class T>
AdjCoef<T> make_coef(int degree, int nodes, double dt, int direction) {
  AdjCoef<T> cf{};
  double x[kAdjMaxNodes], w[kAdjMaxNodes];
  gauss_legendre(nodes, x, w);
  for (int q = 0; q < nodes; ++q) {
    cf.weight[q] = dt * w[q];
    std::complex<double> z(1.0, 0.0), step(0.0, 1.0 - x[q]);
    for (int j = 0; j <= degree; ++j) {
      cf.node[q][j] = tcomplex<T>(z);
      z *= step;
    }
  }
  std::complex<double> z(1.0, 0.0);
  for (int j = 0; j <= degree; ++j) {
    cf.start[j] = tcomplex<T>(z);
    z *= std::complex<double>(0.0, (double)direction);
  }
  return cf;
}

void check_system(const rpm_adjoint* a, const rpm_system* s, const char* what) {
  if (!s) fail(RPM_E_INVALID, std::string(what) + " is NULL");
  if (!s->on_device) fail(RPM_E_INVALID, std::string(what) + " was created host-only");
  if (s->n != a->n) fail(RPM_E_INVALID, std::string(what) + " has another dimension than the adjoint workspace");
  if (s->ndims < 2 || s->dims[0] != 2 || s->dims[1] != 2)
    fail(RPM_E_UNSUPPORTED, std::string(what) + ": the first two axes must be the electron spins");
}

void check_common(rpm_adjoint* a, rpm_system* const* systems, int nseg, const int* seg_of, int nintervals, double dt) {
  if (!a || !systems || nseg < 1 || (nintervals > 0 && !seg_of)) fail(RPM_E_INVALID, "NULL argument");
  if (!(dt > 0.0) || nintervals < 0) fail(RPM_E_INVALID, "dt must be positive and nintervals nonnegative");
  int dev = -1;
  check_cuda(cudaGetDevice(&dev), "cudaGetDevice");
  if (dev != a->device) fail(RPM_E_INVALID, "adjoint workspace belongs to another device");
  for (int s = 0; s < nseg; ++s) check_system(a, systems[s], "segment system");
  for (int j = 0; j < nintervals; ++j)
    if (seg_of[j] < 0 || seg_of[j] >= nseg) fail(RPM_E_INVALID, "segment index out of range");
}

void ensure_tail(rpm_adjoint* a, size_t need, cudaStream_t st) {
  if (need > a->tail_cap) {
    cudaFree(a->tail);
    a->tail = nullptr;
    a->tail_cap = 0;
    if (cudaMalloc((void**)&a->tail, need * sizeof(double)) != cudaSuccess) {
      cudaGetLastError();
      fail(RPM_E_NOMEM, "adjoint workspace: cudaMalloc failed for the Taylor remainders");
    }
    a->tail_cap = need;
  }
  check_cuda(cudaMemsetAsync(a->tail, 0, need * sizeof(double), st), "cudaMemsetAsync");
}

double read_tail(rpm_adjoint* a, size_t need, cudaStream_t st) {
  a->tail_host.resize(need);
  check_cuda(cudaMemcpyAsync(a->tail_host.data(), a->tail, need * sizeof(double), cudaMemcpyDeviceToHost, st),
             "cudaMemcpyAsync");
  check_cuda(cudaStreamSynchronize(st), "cudaStreamSynchronize");
  double worst = 0.0;
  for (size_t k = 0; k + 1 < need; k += 2) {
    const double last = a->tail_host[k], first = a->tail_host[k + 1];
    if (first > 0.0) worst = std::max(worst, std::sqrt(last / first));
  }
  return worst;
}

// Taylor basis u_{t+1} = H (u_t * dt / (t + 1)) of `count` vectors per slot.
template <class T>
void taylor_basis(rpm_adjoint* a, rpm_system* h, int count, cudaStream_t st) {
  T* U = static_cast<T*>(a->U);
  const long long slot = 2LL * a->B * a->ld;
  for (int t = 0; t < a->degree; ++t)
    launch_hpsi_scaled<T>(h, U + t * slot, U + (t + 1) * slot, count, a->ld, a->scales + t, st);
}

template <class T>
void sweep_impl(rpm_adjoint* a, rpm_system* const* systems, int nseg, rpm_system* const* dsys, int nder,
                const int* seg_of, const double* weights, double dt, int nint, double2* xl, double2* xp,
                double* density, double* deriv, double* energy, double* max_tail, cudaStream_t st) {
  const int B = a->B;
  T* U = static_cast<T*>(a->U);
  const size_t tail_need = (size_t)nint * 2 * B;
  ensure_tail(a, tail_need, st);
  k_adj_set_scales<<<1, 32, 0, st>>>(a->scales, dt, a->degree);
  k_adj_convert<T><<<dim3(kAdjBlocksPerVector * 4, B), kAdjThreads, 0, st>>>(xl, U, B, a->n, a->ld);
  k_adj_convert<T><<<dim3(kAdjBlocksPerVector * 4, B), kAdjThreads, 0, st>>>(xp, U + (long long)B * a->ld, B, a->n,
                                                                             a->ld);
  check_launch("adjoint load");
  const AdjCoef<T> cf = make_coef<T>(a->degree, a->nodes, dt, +1);
  bool any_der = false;
  for (int k = 0; k < nseg * nder; ++k) any_der = any_der || dsys[k] != nullptr;
  T* np = any_der ? static_cast<T*>(a->node_p) : nullptr;
  T* nl = any_der ? static_cast<T*>(a->node_l) : nullptr;
  const dim3 grid(kAdjBlocksPerVector, B);
  for (int j = nint - 1; j >= 0; --j) {
    const int s = seg_of[j];
    rpm_system* h = systems[s];
    if (energy) {
      // <lambda(tau)| H |psi(tau)> is constant over the interval: FP64 once
      launch_hpsi<double2>(h, xp, a->hpsi64, B, a->ld, st);
      k_adj_energy<<<dim3(kAdjBlocksPerVector * 4, B), kAdjThreads, 0, st>>>(xl, a->hpsi64, B, a->n, a->ld, dt,
                                                                             energy + 2 * s, 2 * nseg);
      check_launch("adjoint energy");
    }
    taylor_basis<T>(a, h, 2 * B, st);
    double* dens = density + 32 * s;
    double* tail = a->tail + (size_t)j * 2 * B;
    const long long n4 = a->n / 4;
    switch (a->nodes) {
      case 1:
        k_adj_combine<T, 1><<<grid, kAdjThreads, 0, st>>>(U, xl, xp, np, nl, dens, 32 * nseg, tail, cf, a->degree, B,
                                                          a->ld, n4, weights[j]);
        break;
      case 2:
        k_adj_combine<T, 2><<<grid, kAdjThreads, 0, st>>>(U, xl, xp, np, nl, dens, 32 * nseg, tail, cf, a->degree, B,
                                                          a->ld, n4, weights[j]);
        break;
      case 3:
        k_adj_combine<T, 3><<<grid, kAdjThreads, 0, st>>>(U, xl, xp, np, nl, dens, 32 * nseg, tail, cf, a->degree, B,
                                                          a->ld, n4, weights[j]);
        break;
      default:
        k_adj_combine<T, 4><<<grid, kAdjThreads, 0, st>>>(U, xl, xp, np, nl, dens, 32 * nseg, tail, cf, a->degree, B,
                                                          a->ld, n4, weights[j]);
        break;
    }
    check_launch("adjoint combine");
    for (int r = 0; r < nder; ++r) {
      rpm_system* d = dsys[s * nder + r];
      if (!d) continue;
      T* out = static_cast<T*>(a->node_out);
      launch_hpsi<T>(d, np, out, a->nodes * B, a->ld, st);
      k_adj_dots<T><<<dim3(kAdjBlocksPerVector * 4, B), kAdjThreads, 0, st>>>(nl, out, cf, a->nodes, B, a->n, a->ld,
                                                                              deriv + 2 * (s * nder + r),
                                                                              2 * nseg * nder);
      check_launch("adjoint derivative dots");
    }
  }
  if (max_tail) *max_tail = read_tail(a, tail_need, st);
}

template <class T>
void forward_impl(rpm_adjoint* a, rpm_system* const* systems, const int* seg_of, double dt, int nint, double2* xp,
                  double* pops, long long pop_ld, double* max_tail, cudaStream_t st) {
  const int B = a->B;
  T* U = static_cast<T*>(a->U);
  const size_t tail_need = (size_t)nint * 2 * B;
  ensure_tail(a, tail_need, st);
  check_cuda(cudaMemset2DAsync(pops, (size_t)pop_ld * sizeof(double), 0, (size_t)nint * sizeof(double), B, st),
             "cudaMemset2DAsync");
  k_adj_set_scales<<<1, 32, 0, st>>>(a->scales, dt, a->degree);
  k_adj_convert<T><<<dim3(kAdjBlocksPerVector * 4, B), kAdjThreads, 0, st>>>(xp, U, B, a->n, a->ld);
  check_launch("adjoint forward load");
  const AdjCoef<T> cf = make_coef<T>(a->degree, 1, dt, -1);
  for (int j = 0; j < nint; ++j) {
    taylor_basis<T>(a, systems[seg_of[j]], B, st);
    k_adj_forward<T><<<dim3(kAdjBlocksPerVector, B), kAdjThreads, 0, st>>>(
        U, xp, pops + j, pop_ld, a->tail + (size_t)j * 2 * B, cf, a->degree, B, a->ld, a->n / 4);
    check_launch("adjoint forward step");
  }
  if (max_tail) *max_tail = read_tail(a, tail_need, st);
}

}  // namespace

extern "C" int rpm_adjoint_create(int ntraj, long long n, long long ld, int degree, int nodes, int precision,
                                  rpm_adjoint** out) {
  return guarded([&] {
    if (!out) fail(RPM_E_INVALID, "NULL output handle");
    *out = nullptr;
    if (ntraj < 1 || n < 4 || n % 4 != 0 || ld < n || ld % 2 != 0)
      fail(RPM_E_INVALID, "adjoint workspace: ntraj >= 1, n a positive multiple of 4, even ld >= n");
    if (degree < 1 || degree > kAdjMaxDegree) fail(RPM_E_INVALID, "Taylor degree must be in [1, 24]");
    if (nodes < 1 || nodes > kAdjMaxNodes) fail(RPM_E_INVALID, "quadrature nodes must be in [1, 4]");
    if (precision != RPM_PREC_C64 && precision != RPM_PREC_C128) fail(RPM_E_INVALID, "precision must be 64 or 128");
    int device = 0;
    check_cuda(cudaGetDevice(&device), "cudaGetDevice");
    auto* a = new rpm_adjoint();
    a->B = ntraj;
    a->n = n;
    a->ld = ld;
    a->degree = degree;
    a->nodes = nodes;
    a->precision = precision;
    a->elem = precision == RPM_PREC_C64 ? sizeof(float2) : sizeof(double2);
    a->device = device;
    auto alloc = [&](void** p, size_t bytes, const char* what) {
      if (cudaMalloc(p, bytes) != cudaSuccess) {
        cudaGetLastError();
        fail(RPM_E_NOMEM, std::string("adjoint workspace: cudaMalloc failed for ") + what);
      }
      check_cuda(cudaMemset(*p, 0, bytes), "cudaMemset");
    };
    try {
      const size_t vec = (size_t)ld * a->elem;
      alloc(&a->U, (size_t)(degree + 1) * 2 * ntraj * vec, "the Taylor basis");
      alloc(&a->node_p, (size_t)nodes * ntraj * vec, "the psi nodes");
      alloc(&a->node_l, (size_t)nodes * ntraj * vec, "the lambda nodes");
      alloc(&a->node_out, (size_t)nodes * ntraj * vec, "the derivative outputs");
      alloc((void**)&a->hpsi64, (size_t)ntraj * ld * sizeof(double2), "the FP64 H psi");
      alloc((void**)&a->scales, (size_t)kAdjMaxDegree * sizeof(double), "the Taylor scales");
    } catch (...) {
      cudaFree(a->U);
      cudaFree(a->node_p);
      cudaFree(a->node_l);
      cudaFree(a->node_out);
      cudaFree(a->hpsi64);
      cudaFree(a->scales);
      delete a;
      throw;
    }
    *out = a;
  });
}

extern "C" int rpm_adjoint_destroy(rpm_adjoint* a) {
  return guarded([&] {
    if (!a) return;
    cudaDeviceSynchronize();
    cudaFree(a->U);
    cudaFree(a->node_p);
    cudaFree(a->node_l);
    cudaFree(a->node_out);
    cudaFree(a->hpsi64);
    cudaFree(a->scales);
    cudaFree(a->tail);
    delete a;
  });
}

extern "C" int rpm_adjoint_source(rpm_adjoint* a, const void* psi_dev, void* lambda_dev, double weight, void* stream) {
  return guarded([&] {
    if (!a || !psi_dev || !lambda_dev) fail(RPM_E_INVALID, "NULL argument");
    auto st = static_cast<cudaStream_t>(stream);
    k_adj_source<<<dim3(kAdjBlocksPerVector, a->B), kAdjThreads, 0, st>>>(
        static_cast<const double2*>(psi_dev), static_cast<double2*>(lambda_dev), a->B, a->n / 4, a->ld, weight);
    check_launch("adjoint source");
  });
}

extern "C" int rpm_adjoint_sweep(rpm_adjoint* a, rpm_system* const* systems, int nseg,
                                 rpm_system* const* derivative_systems, int nder, const int* segment_of_interval,
                                 const double* source_weights, double dt, int nintervals, void* lambda_dev,
                                 void* psi_dev, double* density_dev, double* derivative_dev, double* energy_dev,
                                 double* max_tail, void* stream) {
  return guarded([&] {
    check_common(a, systems, nseg, segment_of_interval, nintervals, dt);
    if (!lambda_dev || !psi_dev || !density_dev || (nintervals > 0 && !source_weights))
      fail(RPM_E_INVALID, "NULL argument");
    if (nder < 0 || (nder > 0 && (!derivative_systems || !derivative_dev)))
      fail(RPM_E_INVALID, "derivative systems need an output array");
    for (int k = 0; k < nseg * nder; ++k)
      if (derivative_systems[k]) check_system(a, derivative_systems[k], "derivative system");
    if (max_tail) *max_tail = 0.0;
    if (nintervals == 0) return;
    auto st = static_cast<cudaStream_t>(stream);
    auto* xl = static_cast<double2*>(lambda_dev);
    auto* xp = static_cast<double2*>(psi_dev);
    if (a->precision == RPM_PREC_C64)
      sweep_impl<float2>(a, systems, nseg, derivative_systems, nder, segment_of_interval, source_weights, dt,
                         nintervals, xl, xp, density_dev, derivative_dev, energy_dev, max_tail, st);
    else
      sweep_impl<double2>(a, systems, nseg, derivative_systems, nder, segment_of_interval, source_weights, dt,
                          nintervals, xl, xp, density_dev, derivative_dev, energy_dev, max_tail, st);
  });
}

extern "C" int rpm_adjoint_forward(rpm_adjoint* a, rpm_system* const* systems, int nseg,
                                   const int* segment_of_interval, double dt, int nintervals, void* psi_dev,
                                   double* populations_dev, long long pop_ld, double* max_tail, void* stream) {
  return guarded([&] {
    check_common(a, systems, nseg, segment_of_interval, nintervals, dt);
    if (!psi_dev || (nintervals > 0 && !populations_dev) || pop_ld < nintervals)
      fail(RPM_E_INVALID, "bad population output");
    if (max_tail) *max_tail = 0.0;
    if (nintervals == 0) return;
    auto st = static_cast<cudaStream_t>(stream);
    auto* xp = static_cast<double2*>(psi_dev);
    if (a->precision == RPM_PREC_C64)
      forward_impl<float2>(a, systems, segment_of_interval, dt, nintervals, xp, populations_dev, pop_ld, max_tail, st);
    else
      forward_impl<double2>(a, systems, segment_of_interval, dt, nintervals, xp, populations_dev, pop_ld, max_tail,
                            st);
  });
}
