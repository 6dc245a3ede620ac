// FP64 Krylov machinery for the plain (single-vector, complex128) propagator.
//
//   * Hermitian Lanczos with two classical Gram-Schmidt passes
//     (rpm_statevector_engine.py:651-688), as a fixed launch sequence per
//     basis vector with device-side breakdown flag, so no host round trip
//     happens inside a basis build.
//   * Deterministic reductions: every block writes its partial sums, the
//     last block to finish (atomic ticket) adds them in block order.
//   * Symmetric tridiagonal eigen-decomposition by implicit QR with Wilkinson
//     shifts (Golub & Van Loan, Matrix Computations, sec. 8.3): one thread runs
//     the scalar bulge chase and records the Givens rotations; all threads
//     then apply them to their own rows of the eigenvector matrix.
//   * exp(-i T t) e1 coefficients, embedded error norms and projected singlet
//     populations (rpm_statevector_engine.py:569-609, 690-715, 521-538).
//   * Singlet Gram, state recombination, norms and the Simpson yield
//     (rpm_quantum_needle_jd_sweeps.py:418-420).
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <vector>

#include "common.cuh"
#include "krylov.cuh"

namespace rpm {

constexpr int kThreads = 256;
constexpr int kRowsPerThread = 4;
constexpr int kRowsPerBlock = kThreads * kRowsPerThread;

// ---------------------------------------------------------------------------
// Lanczos kernels (single vector, complex128)
// Device scalars (LanczosScalars) live in SLOT_SMALL.
// ---------------------------------------------------------------------------
struct LanczosScalars {
  unsigned counter[8];
  int stop;       // basis size after a breakdown (0 = running)
  int pad;
  double norm;    // ||state||
  double2 h1[RPM_MAX_KRYLOV];
  double2 h2[RPM_MAX_KRYLOV];
};

// v0 = state / ||state|| ; first launch computes ||state||^2 partials.
__global__ void __launch_bounds__(kThreads) k_norm_partial(const double2* __restrict__ x, long long n,
                                                          double2* partials, LanczosScalars* sc, int init) {
  __shared__ double2 scratch[32];
  __shared__ double2 tot[1];
  double2 acc[1] = {make_double2(0.0, 0.0)};
  const long long base = (long long)blockIdx.x * kRowsPerBlock + threadIdx.x;
#pragma unroll
  for (int r = 0; r < kRowsPerThread; ++r) {
    const long long i = base + (long long)r * kThreads;
    if (i < n) {
      const double2 v = x[i];
      acc[0].x = fma(v.x, v.x, fma(v.y, v.y, acc[0].x));
    }
  }
  block_sum2<1>(acc, scratch, tot);
  if (threadIdx.x == 0) partials[blockIdx.x] = tot[0];
  if (last_block(&sc->counter[0])) {
    __shared__ double2 res[1];
    finish_sums(partials, gridDim.x, 1, res);
    __syncthreads();
    if (threadIdx.x == 0) {
      sc->norm = sqrt(res[0].x);
      if (init) sc->stop = 0;
      if (init && !(sc->norm > 0.0)) sc->stop = -1;
      sc->counter[0] = 0;
    }
  }
}

__global__ void __launch_bounds__(kThreads) k_scale_to(const double2* __restrict__ x, double2* __restrict__ y,
                                                      long long n, const LanczosScalars* sc) {
  if (sc->stop != 0) return;
  const double inv = 1.0 / sc->norm;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double2 v = x[i];
    y[i] = make_double2(v.x * inv, v.y * inv);
  }
}

// alpha_j = Re <v_j, w>
__global__ void __launch_bounds__(kThreads) k_alpha(const double2* __restrict__ v, const double2* __restrict__ w,
                                                   long long n, double2* partials, LanczosScalars* sc, double* alpha,
                                                   int j) {
  if (sc->stop != 0) return;
  __shared__ double2 scratch[32];
  __shared__ double2 tot[1];
  double2 acc[1] = {make_double2(0.0, 0.0)};
  const long long base = (long long)blockIdx.x * kRowsPerBlock + threadIdx.x;
#pragma unroll
  for (int r = 0; r < kRowsPerThread; ++r) {
    const long long i = base + (long long)r * kThreads;
    if (i < n) acc[0] = cfma_conj(v[i], w[i], acc[0]);
  }
  block_sum2<1>(acc, scratch, tot);
  if (threadIdx.x == 0) partials[blockIdx.x] = tot[0];
  if (last_block(&sc->counter[1])) {
    __shared__ double2 res[1];
    finish_sums(partials, gridDim.x, 1, res);
    __syncthreads();
    if (threadIdx.x == 0) {
      alpha[j] = res[0].x;
      sc->counter[1] = 0;
    }
  }
}

// Block dot products  h[k] = <V_k, w>  for k < count over this block's rows,
// with w held in registers.  Results into partials[k * nblocks + block].
__device__ void block_dots(const double2* __restrict__ basis, long long n, int count, const double2 (&w)[kRowsPerThread],
                           double2* partials) {
  __shared__ double2 scratch[32 * 8];
  __shared__ double2 tot[8];
  const long long base = (long long)blockIdx.x * kRowsPerBlock + threadIdx.x;
  for (int k0 = 0; k0 < count; k0 += 8) {
    double2 acc[8];
#pragma unroll
    for (int c = 0; c < 8; ++c) acc[c] = make_double2(0.0, 0.0);
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      if (k0 + c < count) {
        const double2* vk = basis + (size_t)(k0 + c) * n;
#pragma unroll
        for (int r = 0; r < kRowsPerThread; ++r) {
          const long long i = base + (long long)r * kThreads;
          if (i < n) acc[c] = cfma_conj(vk[i], w[r], acc[c]);
        }
      }
    }
    block_sum2<8>(acc, scratch, tot);
    if (threadIdx.x < 8 && k0 + threadIdx.x < count) partials[(size_t)(k0 + threadIdx.x) * gridDim.x + blockIdx.x] = tot[threadIdx.x];
  }
}

// w <- w - alpha_j v_j - beta_{j-1} v_{j-1};  h1 = V[:, :j+1]^H w
__global__ void __launch_bounds__(kThreads) k_update_dots(const double2* __restrict__ basis, double2* __restrict__ w,
                                                         long long n, int j, const double* alpha, const double* beta,
                                                         double2* partials, LanczosScalars* sc) {
  if (sc->stop != 0) return;
  const double a = alpha[j];
  const double b = j > 0 ? beta[j - 1] : 0.0;
  const double2* vj = basis + (size_t)j * n;
  const double2* vp = basis + (size_t)(j > 0 ? j - 1 : 0) * n;
  double2 wr[kRowsPerThread];
  const long long base = (long long)blockIdx.x * kRowsPerBlock + threadIdx.x;
#pragma unroll
  for (int r = 0; r < kRowsPerThread; ++r) {
    const long long i = base + (long long)r * kThreads;
    wr[r] = make_double2(0.0, 0.0);
    if (i < n) {
      double2 x = w[i];
      const double2 v = vj[i];
      x.x -= a * v.x;
      x.y -= a * v.y;
      if (j > 0) {
        const double2 u = vp[i];
        x.x -= b * u.x;
        x.y -= b * u.y;
      }
      wr[r] = x;
      w[i] = x;
    }
  }
  block_dots(basis, n, j + 1, wr, partials);
  if (last_block(&sc->counter[2])) {
    finish_sums(partials, gridDim.x, j + 1, sc->h1);
    __syncthreads();
    if (threadIdx.x == 0) sc->counter[2] = 0;
  }
}

// w <- w - V h ; then (second == 1) h2 = V^H w, or (second == 0) ||w||^2 -> beta_j
__global__ void __launch_bounds__(kThreads) k_axpy_then(const double2* __restrict__ basis, double2* __restrict__ w,
                                                       long long n, int j, int second, int last, double tol,
                                                       double* beta, double2* partials, LanczosScalars* sc) {
  if (sc->stop != 0) return;
  __shared__ double2 h[RPM_MAX_KRYLOV];
  const double2* hsrc = second ? sc->h1 : sc->h2;
  for (int k = threadIdx.x; k <= j; k += blockDim.x) h[k] = hsrc[k];
  __syncthreads();
  double2 wr[kRowsPerThread];
  const long long base = (long long)blockIdx.x * kRowsPerBlock + threadIdx.x;
#pragma unroll
  for (int r = 0; r < kRowsPerThread; ++r) {
    const long long i = base + (long long)r * kThreads;
    wr[r] = make_double2(0.0, 0.0);
    if (i < n) {
      // CGS: w - V h accumulated as one product, then subtracted
      double2 vh = make_double2(0.0, 0.0);
      for (int k = 0; k <= j; ++k) vh = cfma(basis[(size_t)k * n + i], h[k], vh);
      double2 x = w[i];
      x.x -= vh.x;
      x.y -= vh.y;
      wr[r] = x;
      w[i] = x;
    }
  }
  if (second) {
    block_dots(basis, n, j + 1, wr, partials);
    if (last_block(&sc->counter[3])) {
      finish_sums(partials, gridDim.x, j + 1, sc->h2);
      __syncthreads();
      if (threadIdx.x == 0) sc->counter[3] = 0;
    }
    return;
  }
  if (last) return;
  __shared__ double2 scratch[32];
  __shared__ double2 tot[1];
  double2 acc[1] = {make_double2(0.0, 0.0)};
#pragma unroll
  for (int r = 0; r < kRowsPerThread; ++r) acc[0].x = fma(wr[r].x, wr[r].x, fma(wr[r].y, wr[r].y, acc[0].x));
  block_sum2<1>(acc, scratch, tot);
  if (threadIdx.x == 0) partials[blockIdx.x] = tot[0];
  if (last_block(&sc->counter[4])) {
    __shared__ double2 res[1];
    finish_sums(partials, gridDim.x, 1, res);
    __syncthreads();
    if (threadIdx.x == 0) {
      const double bj = sqrt(res[0].x);
      beta[j] = bj;
      if (bj <= tol) sc->stop = j + 1;
      sc->counter[4] = 0;
    }
  }
}

// v_{j+1} = w / beta_j
__global__ void __launch_bounds__(kThreads) k_next_vector(const double2* __restrict__ w, double2* __restrict__ next,
                                                         long long n, const double* beta, int j,
                                                         const LanczosScalars* sc) {
  if (sc->stop != 0) return;
  const double inv = 1.0 / beta[j];
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double2 v = w[i];
    next[i] = make_double2(v.x * inv, v.y * inv);
  }
}

// spectra record layout (doubles): [0] size, [1] status, [2 .. 2+MAXK) eigenvalues,
// then MAXK x MAXK eigenvectors (row i = component i).
__global__ void k_tridiag_spectra(const double* __restrict__ alpha, const double* __restrict__ beta, const int* dims,
                                  double* spectra) {
  extern __shared__ double sm[];
  double* z = sm;                                  // m * m
  double* d = z + RPM_MAX_KRYLOV * RPM_MAX_KRYLOV;  // m
  double* e = d + RPM_MAX_KRYLOV;                  // m
  double2* rot = reinterpret_cast<double2*>(e + RPM_MAX_KRYLOV);
  const int m = dims[blockIdx.x];
  double* rec = spectra + (size_t)blockIdx.x * RPM_SPECTRUM_DOUBLES;
  for (int i = threadIdx.x; i < m; i += blockDim.x) {
    d[i] = alpha[i];
    e[i] = (i + 1 < m) ? beta[i] : 0.0;
  }
  __syncthreads();
  const int status = tridiag_qr(m, d, e, z, m, rot);
  for (int i = threadIdx.x; i < m; i += blockDim.x) rec[2 + i] = d[i];
  for (int idx = threadIdx.x; idx < m * m; idx += blockDim.x) {
    const int i = idx / m, k = idx % m;
    rec[2 + RPM_MAX_KRYLOV + i * RPM_MAX_KRYLOV + k] = z[i * m + k];
  }
  if (threadIdx.x == 0) {
    rec[0] = m;
    rec[1] = status;
  }
}

__global__ void k_krylov_eval(const double* __restrict__ spectra, const rpm_krylov_req* reqs, double safety,
                              double state_norm, const double2* __restrict__ gram, int gram_ld, double2* coef,
                              int coef_ld, double* err_out, double* value_out) {
  __shared__ double2 ph[RPM_MAX_KRYLOV], chi[RPM_MAX_KRYLOV], clo[RPM_MAX_KRYLOV];
  __shared__ double red[kThreads / 32];
  const rpm_krylov_req rq = reqs[blockIdx.x];
  const double* rhi = spectra + (size_t)rq.hi * RPM_SPECTRUM_DOUBLES;
  const int mh = (int)rhi[0];
  spectral_coefficients(rhi, rq.time, ph, chi);
  int ml = 0;
  if (rq.lo >= 0) {
    const double* rlo = spectra + (size_t)rq.lo * RPM_SPECTRUM_DOUBLES;
    ml = (int)rlo[0];
    spectral_coefficients(rlo, rq.time, ph, clo);
  }
  for (int i = threadIdx.x; i < mh; i += blockDim.x) coef[(size_t)blockIdx.x * coef_ld + i] = chi[i];
  // ||c_hi - [c_lo; 0]||
  double acc = 0.0;
  if (rq.lo >= 0) {
    for (int i = threadIdx.x; i < mh; i += blockDim.x) {
      double2 dlt = chi[i];
      if (i < ml) {
        dlt.x -= clo[i].x;
        dlt.y -= clo[i].y;
      }
      acc = fma(dlt.x, dlt.x, fma(dlt.y, dlt.y, acc));
    }
  }
  acc = warp_sum(acc);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w];
    err_out[blockIdx.x] = rq.lo >= 0 ? safety * state_norm * sqrt(s) : 0.0;
  }
  __syncthreads();
  if (gram) {
    // c^H G c
    double v = 0.0;
    for (int i = threadIdx.x; i < mh; i += blockDim.x) {
      double2 gc = make_double2(0.0, 0.0);
      for (int k = 0; k < mh; ++k) gc = cfma(gram[(size_t)i * gram_ld + k], chi[k], gc);
      v += chi[i].x * gc.x + chi[i].y * gc.y;
    }
    v = warp_sum(v);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
      double s = 0.0;
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w];
      value_out[blockIdx.x] = state_norm * state_norm * s;
    }
  }
}

// ---------------------------------------------------------------------------
// Singlet Gram  G = A^H A,  A[:, k] = (V_k[M:2M] - V_k[2M:3M]) / sqrt 2
// ---------------------------------------------------------------------------
constexpr int kGramRows = 32;

__global__ void __launch_bounds__(kThreads) k_gram_partial(const double2* __restrict__ basis, long long n, int m,
                                                          double2* partials) {
  extern __shared__ double2 a[];  // kGramRows x m
  const long long quarter = n / 4;
  const double rs2 = 0.70710678118654752440;
  const int pairs = m * m;
  double2 acc[16];
  const int per = (pairs + blockDim.x - 1) / blockDim.x;  // <= 16 for m <= 64
#pragma unroll
  for (int q = 0; q < 16; ++q) acc[q] = make_double2(0.0, 0.0);
  for (long long r0 = (long long)blockIdx.x * kGramRows; r0 < quarter; r0 += (long long)gridDim.x * kGramRows) {
    __syncthreads();
    for (int idx = threadIdx.x; idx < kGramRows * m; idx += blockDim.x) {
      const int rr = idx / m, k = idx % m;
      const long long i = r0 + rr;
      double2 v = make_double2(0.0, 0.0);
      if (i < quarter) {
        const double2 p = basis[(size_t)k * n + quarter + i];
        const double2 q = basis[(size_t)k * n + 2 * quarter + i];
        v = make_double2((p.x - q.x) * rs2, (p.y - q.y) * rs2);
      }
      a[rr * m + k] = v;
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < 16; ++q) {
      const int pr = threadIdx.x + q * blockDim.x;
      if (q < per && pr < pairs) {
        const int k = pr / m, l = pr % m;
        double2 s = acc[q];
        for (int rr = 0; rr < kGramRows; ++rr) s = cfma_conj(a[rr * m + k], a[rr * m + l], s);
        acc[q] = s;
      }
    }
  }
#pragma unroll
  for (int q = 0; q < 16; ++q) {
    const int pr = threadIdx.x + q * blockDim.x;
    if (q < per && pr < pairs) partials[(size_t)pr * gridDim.x + blockIdx.x] = acc[q];
  }
}

__global__ void k_gram_finish(const double2* __restrict__ partials, int nblocks, int m, double2* gram) {
  const int pr = blockIdx.x * blockDim.x + threadIdx.x;
  if (pr >= m * m) return;
  const int k = pr / m, l = pr % m;
  double2 s = make_double2(0.0, 0.0), t = make_double2(0.0, 0.0);
  for (int b = 0; b < nblocks; ++b) {
    s = cadd(s, partials[(size_t)(k * m + l) * nblocks + b]);
    t = cadd(t, partials[(size_t)(l * m + k) * nblocks + b]);
  }
  // Hermitian symmetrisation 0.5 (G + G^H)
  gram[(size_t)k * m + l] = make_double2(0.5 * (s.x + t.x), 0.5 * (s.y - t.y));
}

static void singlet_gram_launch(rpm_system* sys, const double2* basis, int m, double2* gram, cudaStream_t st) {
  const long long quarter = sys->n / 4;
  int blocks = (int)std::min<long long>((quarter + kGramRows - 1) / kGramRows, 2 * 148);
  blocks = std::max(blocks, 1);
  auto* partials = static_cast<double2*>(system_scratch(sys, SLOT_GRAM, (size_t)blocks * m * m * sizeof(double2)));
  const size_t smem = (size_t)kGramRows * m * sizeof(double2);
  k_gram_partial<<<blocks, kThreads, smem, st>>>(basis, sys->n, m, partials);
  k_gram_finish<<<(m * m + 255) / 256, 256, 0, st>>>(partials, blocks, m, gram);
  check_launch("singlet gram");
}

// ---------------------------------------------------------------------------
// out = scale * V c  (+ ||out||^2)
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads) k_combine(const double2* __restrict__ basis, long long n, int m,
                                                     const double2* __restrict__ coef, double scale,
                                                     double2* __restrict__ out, double2* partials, unsigned* counter,
                                                     double* norm_out) {
  __shared__ double2 c[RPM_MAX_KRYLOV];
  __shared__ double2 scratch[32];
  __shared__ double2 tot[1];
  for (int k = threadIdx.x; k < m; k += blockDim.x) c[k] = coef[k];
  __syncthreads();
  double2 acc[1] = {make_double2(0.0, 0.0)};
  const long long base = (long long)blockIdx.x * kRowsPerBlock + threadIdx.x;
#pragma unroll
  for (int r = 0; r < kRowsPerThread; ++r) {
    const long long i = base + (long long)r * kThreads;
    if (i < n) {
      double2 s = make_double2(0.0, 0.0);
      for (int k = 0; k < m; ++k) s = cfma(basis[(size_t)k * n + i], c[k], s);
      s.x *= scale;
      s.y *= scale;
      out[i] = s;
      acc[0].x = fma(s.x, s.x, fma(s.y, s.y, acc[0].x));
    }
  }
  block_sum2<1>(acc, scratch, tot);
  if (threadIdx.x == 0) partials[blockIdx.x] = tot[0];
  if (last_block(counter)) {
    __shared__ double2 res[1];
    finish_sums(partials, gridDim.x, 1, res);
    __syncthreads();
    if (threadIdx.x == 0) {
      *norm_out = sqrt(res[0].x);
      *counter = 0;
    }
  }
}

// Per-vector reductions over a batch: kind 0 = ||x||^2, kind 1 = singlet population.
__global__ void __launch_bounds__(kThreads) k_batch_reduce(const double2* __restrict__ x, long long n, long long ld,
                                                          int kind, double* out) {
  __shared__ double red[kThreads / 32];
  const double2* v = x + (long long)blockIdx.x * ld;
  double acc = 0.0;
  if (kind == 0) {
    for (long long i = threadIdx.x; i < n; i += blockDim.x) acc = fma(v[i].x, v[i].x, fma(v[i].y, v[i].y, acc));
  } else {
    const long long q = n / 4;
    for (long long i = threadIdx.x; i < q; i += blockDim.x) {
      const double2 a = v[q + i], b = v[2 * q + i];
      const double re = a.x - b.x, im = a.y - b.y;
      acc = fma(re, re, fma(im, im, acc));
    }
    acc *= 0.5;
  }
  acc = warp_sum(acc);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w];
    out[blockIdx.x] = s;
  }
}

// ---------------------------------------------------------------------------
// Simpson yield with Neumaier-compensated FP64 sums (one block per row)
// ---------------------------------------------------------------------------
struct Kahan {
  double s, c;
  __device__ void add(double v) {
    const double t = s + v;
    c += (fabs(s) >= fabs(v)) ? ((s - t) + v) : ((v - t) + s);
    s = t;
  }
};

__device__ __forceinline__ double simpson_integrand(const double* t, const double* p, int k, double tau) {
  return exp(-t[k] / tau) * p[k] / tau;
}

__global__ void k_simpson(const double* __restrict__ t, const double* __restrict__ pops, int n, long long ld,
                          double tau, double* out) {
  __shared__ double ss[kThreads], cs[kThreads];
  const double* p = pops + (long long)blockIdx.x * ld;
  Kahan acc{0.0, 0.0};
  // panels over [0, stop]: odd n -> stop = n - 1, even n -> stop = n - 2 (end correction below)
  const int stop = (n % 2 == 1) ? n - 1 : n - 2;
  if (n >= 3) {
    for (int k = 2 * threadIdx.x; k + 2 <= stop; k += 2 * blockDim.x) {
      const double h0 = t[k + 1] - t[k], h1 = t[k + 2] - t[k + 1];
      const double hs = h0 + h1, hp = h0 * h1, r = h0 / h1;
      const double f0 = simpson_integrand(t, p, k, tau), f1 = simpson_integrand(t, p, k + 1, tau),
                   f2 = simpson_integrand(t, p, k + 2, tau);
      acc.add(hs / 6.0 * (f0 * (2.0 - 1.0 / r) + f1 * (hs * hs / hp) + f2 * (2.0 - r)));
    }
  }
  ss[threadIdx.x] = acc.s;
  cs[threadIdx.x] = acc.c;
  __syncthreads();
  if (threadIdx.x == 0) {
    Kahan tot{0.0, 0.0};
    for (int k = 0; k < (int)blockDim.x; ++k) {
      tot.add(ss[k]);
      tot.add(cs[k]);
    }
    if (n == 2) {
      tot.add(0.5 * (t[1] - t[0]) * (simpson_integrand(t, p, 0, tau) + simpson_integrand(t, p, 1, tau)));
    } else if (n % 2 == 0 && n >= 4) {
      const double a = t[n - 2] - t[n - 3], b = t[n - 1] - t[n - 2];
      const double al = (2 * b * b + 3 * a * b) / (6 * (a + b));
      const double be = (b * b + 3 * a * b) / (6 * a);
      const double et = b * b * b / (6 * a * (a + b));
      tot.add(al * simpson_integrand(t, p, n - 1, tau));
      tot.add(be * simpson_integrand(t, p, n - 2, tau));
      tot.add(-et * simpson_integrand(t, p, n - 3, tau));
    }
    out[blockIdx.x] = tot.s + tot.c;
  }
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
static LanczosScalars* scalars(rpm_system* sys) {
  return static_cast<LanczosScalars*>(system_scratch(sys, SLOT_SMALL, sizeof(LanczosScalars)));
}

static double2* reduce_partials(rpm_system* sys, size_t count) {
  return static_cast<double2*>(system_scratch(sys, SLOT_REDUCE, count * sizeof(double2)));
}

static int row_blocks(long long n) { return (int)((n + kRowsPerBlock - 1) / kRowsPerBlock); }

// Launches a basis build; the size and ||state|| land in the system's
// LanczosScalars (stop: 0 full, j + 1 after a breakdown at j, -1 zero vector).
static void lanczos_basis_launch(rpm_system* sys, const double2* state, int max_dim, double tol, double2* basis,
                                 double* alpha, double* beta, cudaStream_t st) {
  const long long n = sys->n;
  const int m = (int)std::min<long long>(max_dim, n);
  if (m < 1 || m > RPM_MAX_KRYLOV) fail(RPM_E_UNSUPPORTED, "Krylov dimension must be in [1, 128]");
  LanczosScalars* sc = scalars(sys);
  const int nb = row_blocks(n);
  double2* partials = reduce_partials(sys, (size_t)nb * (RPM_MAX_KRYLOV + 1));
  double2* w = static_cast<double2*>(system_scratch(sys, SLOT_WORK, (size_t)n * sizeof(double2)));
  const int ew_blocks = (int)std::min<long long>((n + 255) / 256, 4096);

  k_norm_partial<<<nb, kThreads, 0, st>>>(state, n, partials, sc, 1);
  k_scale_to<<<ew_blocks, 256, 0, st>>>(state, basis, n, sc);
  check_launch("lanczos init");
  for (int j = 0; j < m; ++j) {
    double2* vj = basis + (size_t)j * n;
    launch_hpsi<double2>(sys, vj, w, 1, n, st);
    k_alpha<<<nb, kThreads, 0, st>>>(vj, w, n, partials, sc, alpha, j);
    k_update_dots<<<nb, kThreads, 0, st>>>(basis, w, n, j, alpha, beta, partials, sc);
    k_axpy_then<<<nb, kThreads, 0, st>>>(basis, w, n, j, 1, 0, tol, beta, partials, sc);
    k_axpy_then<<<nb, kThreads, 0, st>>>(basis, w, n, j, 0, j == m - 1, tol, beta, partials, sc);
    if (j + 1 < m) k_next_vector<<<ew_blocks, 256, 0, st>>>(w, basis + (size_t)(j + 1) * n, n, beta, j, sc);
    check_launch("lanczos step");
  }
}

void lanczos_basis(rpm_system* sys, const double2* state, int max_dim, double tol, double2* basis, double* alpha,
                   double* beta, int* actual, double* norm, cudaStream_t st) {
  const int m = (int)std::min<long long>(max_dim, sys->n);
  lanczos_basis_launch(sys, state, max_dim, tol, basis, alpha, beta, st);
  LanczosScalars* sc = scalars(sys);
  struct {
    int stop;
    int pad;
    double norm;
  } info;
  check_cuda(cudaMemcpyAsync(&info, &sc->stop, sizeof(info), cudaMemcpyDeviceToHost, st), "copy lanczos info");
  check_cuda(cudaStreamSynchronize(st), "lanczos sync");
  *norm = info.norm;
  if (info.stop < 0) fail(RPM_E_INVALID, "Cannot propagate the zero vector.");
  *actual = info.stop > 0 ? info.stop : m;
}


// ---------------------------------------------------------------------------
// Plain propagation with the step controller on the device
// ---------------------------------------------------------------------------
// One Krylov step of the reference controller (rpm_statevector_engine.py:
// 717-933) is a fixed launch sequence with one host read at its end: the
// basis, the singlet Gram of the basis, k_plain_control (the spectra of every
// dimension the step's candidate list needs, one warp each; the embedded
// error of every candidate at the trial step; the first one within the
// budget; the coefficient row of the new state and the populations and
// error estimates at the step's observation points), and k_plain_combine
// (the new state and its norm).  The host only keeps the step-size logic.
// records for dimensions <= 64: [0] size, [1] status, eigenvalues, eigenvectors by columns
constexpr int kPlainLD = 64;
constexpr int kPlainRec = 2 + kPlainLD + kPlainLD * kPlainLD;  // doubles per spectra record
constexpr int kPlainWarps = 16;
constexpr int kPlainMaxCand = 15;                             // candidate dimensions per step
constexpr int kPlainMaxDims = 2 * kPlainMaxCand + 1;

struct PlainIn {
  int mode;  // 0: the minimum dimension alone; 1: ladder from the minimum; 2: ladder from minimum + increment
  int target, built, min_dim, max_dim, inc, offset;
  int first, npts;  // observation points times[first, first + npts)
  double trial, budget, safety, t_now;
};

struct PlainOut {
  int status;  // 0 accepted, 1 rejected, 2 the maximum basis is needed, 3 eigen-solver failure, 4 zero vector
  int size, selected, lo, exact, pad;
  double err, norm, new_norm;
};

// c_i(t) = sum_k z_ik exp(-i lambda_k t) z_0k for i < m of one record, by one
// warp into warp-private c (the arithmetic of spectral_coefficients).
static __device__ void warp_coefficients(const double* rec, double t, double2* ph, double2* c) {
  const int lane = threadIdx.x & 31;
  const int m = (int)rec[0];
  const double* lam = rec + 2;
  const double* z = rec + 2 + kPlainLD;
  for (int k = lane; k < m; k += 32) {
    double s, co;
    sincos(lam[k] * t, &s, &co);
    const double w = z[k * kPlainLD];  // first component of eigenvector k
    ph[k] = make_double2(co * w, -s * w);
  }
  __syncwarp();
  for (int i = lane; i < m; i += 32) {
    double2 acc = make_double2(0.0, 0.0);
    for (int k = 0; k < m; ++k) {
      const double zz = z[k * kPlainLD + i];
      acc.x = fma(zz, ph[k].x, acc.x);
      acc.y = fma(zz, ph[k].y, acc.y);
    }
    c[i] = acc;
  }
  __syncwarp();
}

// |c_hi - [c_lo; 0]|^2 over the warp.
static __device__ double warp_diff2(const double2* ch, int mh, const double2* cl, int ml) {
  double acc = 0.0;
  for (int i = threadIdx.x & 31; i < mh; i += 32) {
    double2 d = ch[i];
    if (i < ml) {
      d.x -= cl[i].x;
      d.y -= cl[i].y;
    }
    acc = fma(d.x, d.x, fma(d.y, d.y, acc));
  }
  return warp_sum(acc);
}

constexpr size_t kPlainSmem = sizeof(double) * kPlainWarps * 2 * kPlainLD + sizeof(double2) * kPlainWarps * 4 * kPlainLD;

__global__ void __launch_bounds__(kPlainWarps * 32) k_plain_control(const double* __restrict__ alpha,
                                                                   const double* __restrict__ beta,
                                                                   const LanczosScalars* sc, PlainIn in, double* recs,
                                                                   const double2* __restrict__ gram,
                                                                   const double* __restrict__ times, double* values,
                                                                   double* perr, double2* coef, PlainOut* out) {
  extern __shared__ double psm[];
  __shared__ int s_dims[kPlainMaxDims], s_hi[kPlainMaxCand], s_lo[kPlainMaxCand];
  __shared__ int s_ndims, s_ncand, s_status, s_sel, s_size, s_exact, s_bad;
  __shared__ double s_err[kPlainMaxCand], s_norm;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double* dd = psm + warp * 2 * kPlainLD;
  double* ee = dd + kPlainLD;
  double2* wb = reinterpret_cast<double2*>(psm + kPlainWarps * 2 * kPlainLD) + warp * 4 * kPlainLD;
  double2* rot = wb;
  double2* ph = wb + kPlainLD;
  double2* ch = wb + 2 * kPlainLD;
  double2* cl = wb + 3 * kPlainLD;
  if (threadIdx.x == 0) {
    const int stop = sc->stop;
    s_norm = sc->norm;
    s_bad = 0;
    const int size = stop > 0 ? stop : in.built;
    const int exact = size < in.target;
    int nd = 0, nc = 0;
    auto record = [&](int d) {
      for (int i = 0; i < nd; ++i)
        if (s_dims[i] == d) return i;
      s_dims[nd] = d;
      return nd++;
    };
    // (d, d - offset) as the reference's candidate evaluation (ENG:690-715)
    auto add = [&](int d) {
      d = min(d, size);
      const int lo = max(1, d - in.offset);
      s_hi[nc] = record(d);
      s_lo[nc] = lo == d ? -1 : record(lo);
      ++nc;
    };
    if (stop < 0) {
      nc = 0;
    } else if (exact) {
      s_hi[0] = record(size);
      s_lo[0] = -1;
      nc = 1;
    } else if (in.mode == 0) {
      add(in.min_dim);
    } else {
      int last = 0;
      for (int d = in.mode == 1 ? in.min_dim : in.min_dim + in.inc; d <= in.max_dim; d += in.inc) {
        add(d);
        last = d;
      }
      if (last != in.max_dim) add(in.max_dim);
    }
    s_status = stop < 0 ? 4 : 0;
    s_size = stop < 0 ? 0 : size;
    s_exact = exact;
    s_ndims = nd;
    s_ncand = nc;
  }
  __syncthreads();
  if (s_status == 0) {
    for (int r = warp; r < s_ndims; r += kPlainWarps) {
      const int dim = s_dims[r];
      double* rec = recs + (size_t)r * kPlainRec;
      for (int i = lane; i < dim; i += 32) {
        dd[i] = alpha[i];
        ee[i] = (i + 1 < dim) ? beta[i] : 0.0;
      }
      __syncwarp();
      const int bad = tridiag_qr_warp_cols<false>(dim, dd, ee, rec + 2 + kPlainLD, kPlainLD, rot);
      for (int i = lane; i < dim; i += 32) rec[2 + i] = dd[i];
      if (lane == 0) {
        rec[0] = dim;
        rec[1] = bad;
        if (bad) s_bad = 1;
      }
      __syncwarp();
    }
    __syncthreads();
    for (int c = warp; c < s_ncand; c += kPlainWarps) {
      const double* rh = recs + (size_t)s_hi[c] * kPlainRec;
      double e2 = 0.0;
      if (s_lo[c] >= 0) {
        const double* rl = recs + (size_t)s_lo[c] * kPlainRec;
        warp_coefficients(rh, in.trial, ph, ch);
        warp_coefficients(rl, in.trial, ph, cl);
        e2 = warp_diff2(ch, (int)rh[0], cl, (int)rl[0]);
      }
      if (lane == 0) s_err[c] = s_lo[c] >= 0 ? in.safety * s_norm * sqrt(e2) : 0.0;
      __syncwarp();
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      int sel = -1;
      for (int c = 0; c < s_ncand; ++c)
        if (s_err[c] <= in.budget) {
          sel = c;
          break;
        }
      s_sel = sel;
      s_status = s_bad ? 3 : sel >= 0 ? 0 : (in.mode == 0 && in.max_dim > in.min_dim ? 2 : 1);
    }
    __syncthreads();
  }
  const int status = s_status;
  if (status == 0) {
    const int sel = s_sel;
    const double* rh = recs + (size_t)s_hi[sel] * kPlainRec;
    const double* rl = s_lo[sel] >= 0 ? recs + (size_t)s_lo[sel] * kPlainRec : nullptr;
    const int mh = (int)rh[0], ml = rl ? (int)rl[0] : 0;
    if (warp == 0) {
      warp_coefficients(rh, in.trial, ph, ch);
      for (int i = lane; i < mh; i += 32) coef[i] = ch[i];
    }
    const double nn = s_norm * s_norm;
    for (int p = warp; p < in.npts; p += kPlainWarps) {
      const double dt = times[in.first + p] - in.t_now;
      warp_coefficients(rh, dt, ph, ch);
      double e2 = 0.0;
      if (rl) {
        warp_coefficients(rl, dt, ph, cl);
        e2 = warp_diff2(ch, mh, cl, ml);
      }
      // c^H G c with the singlet Gram of the basis (leading dimension: the basis size)
      double v = 0.0;
      for (int i = lane; i < mh; i += 32) {
        double2 gc = make_double2(0.0, 0.0);
        for (int k = 0; k < mh; ++k) gc = cfma(gram[(size_t)i * in.built + k], ch[k], gc);
        v += ch[i].x * gc.x + ch[i].y * gc.y;
      }
      v = warp_sum(v);
      if (lane == 0) {
        values[in.first + p] = nn * v;
        perr[in.first + p] = rl ? in.safety * s_norm * sqrt(e2) : 0.0;
      }
      __syncwarp();
    }
  }
  if (threadIdx.x == 0) {
    PlainOut o{};
    o.status = status;
    o.size = s_size;
    o.exact = s_exact;
    o.norm = s_norm;
    if (status == 0) {
      const int sel = s_sel;
      o.selected = (int)recs[(size_t)s_hi[sel] * kPlainRec];
      o.lo = s_lo[sel] >= 0 ? (int)recs[(size_t)s_lo[sel] * kPlainRec] : 0;
      o.err = s_err[sel];
    }
    *out = o;
  }
}

// state = ||state|| V c for an accepted step (in place: the basis no longer
// needs the old state), and ||state|| of the result into out->new_norm.
__global__ void __launch_bounds__(kThreads) k_plain_combine(const double2* __restrict__ basis, long long n,
                                                           const double2* __restrict__ coef,
                                                           double2* __restrict__ state, double2* partials,
                                                           unsigned* counter, PlainOut* out) {
  if (out->status != 0) return;
  __shared__ double2 c[kPlainLD];
  __shared__ double2 scratch[32];
  __shared__ double2 tot[1];
  const int m = out->selected;
  const double scale = out->norm;
  for (int k = threadIdx.x; k < m; k += blockDim.x) c[k] = coef[k];
  __syncthreads();
  double2 acc[1] = {make_double2(0.0, 0.0)};
  const long long base = (long long)blockIdx.x * kRowsPerBlock + threadIdx.x;
#pragma unroll
  for (int r = 0; r < kRowsPerThread; ++r) {
    const long long i = base + (long long)r * kThreads;
    if (i < n) {
      double2 s = make_double2(0.0, 0.0);
      for (int k = 0; k < m; ++k) s = cfma(basis[(size_t)k * n + i], c[k], s);
      s.x *= scale;
      s.y *= scale;
      state[i] = s;
      acc[0].x = fma(s.x, s.x, fma(s.y, s.y, acc[0].x));
    }
  }
  block_sum2<1>(acc, scratch, tot);
  if (threadIdx.x == 0) partials[blockIdx.x] = tot[0];
  if (last_block(counter)) {
    __shared__ double2 res[1];
    finish_sums(partials, gridDim.x, 1, res);
    __syncthreads();
    if (threadIdx.x == 0) {
      out->new_norm = sqrt(res[0].x);
      *counter = 0;
    }
  }
}

// Device buffers of one plain propagation (stream-ordered allocation).
struct PlainBuffers {
  cudaStream_t st = nullptr;
  void* base = nullptr;
  double2 *basis = nullptr, *gram = nullptr, *coef = nullptr;
  double *alpha = nullptr, *beta = nullptr, *recs = nullptr, *times = nullptr, *values = nullptr, *perr = nullptr;
  PlainOut* out = nullptr;
  ~PlainBuffers() {
    if (base) cudaFreeAsync(base, st);
  }
};

static void plain_propagate(rpm_system* sys, const rpm_plain_knobs& k, double2* state, const double* times, int ntimes,
                            int cursor0, double norm_error0, double* values_host, double* errors_host,
                            rpm_plain_result* res, cudaStream_t st) {
  const long long n = sys->n;
  const int mmax = (int)std::min<long long>(k.maximum_dimension, n);
  PlainBuffers b;
  b.st = st;
  size_t off = 0;
  auto take = [&](size_t bytes) {
    const size_t at = off;
    off += (bytes + 255) & ~(size_t)255;
    return at;
  };
  const size_t o_basis = take(sizeof(double2) * (size_t)mmax * n), o_gram = take(sizeof(double2) * 64 * 64),
               o_coef = take(sizeof(double2) * kPlainLD), o_alpha = take(sizeof(double) * kPlainLD),
               o_beta = take(sizeof(double) * kPlainLD), o_recs = take(sizeof(double) * kPlainMaxDims * kPlainRec),
               o_times = take(sizeof(double) * ntimes), o_values = take(sizeof(double) * ntimes),
               o_perr = take(sizeof(double) * ntimes), o_out = take(sizeof(PlainOut));
  check_cuda(cudaMallocAsync(&b.base, off, st), "cudaMallocAsync(plain propagation)");
  char* base = static_cast<char*>(b.base);
  b.basis = reinterpret_cast<double2*>(base + o_basis);
  b.gram = reinterpret_cast<double2*>(base + o_gram);
  b.coef = reinterpret_cast<double2*>(base + o_coef);
  b.alpha = reinterpret_cast<double*>(base + o_alpha);
  b.beta = reinterpret_cast<double*>(base + o_beta);
  b.recs = reinterpret_cast<double*>(base + o_recs);
  b.times = reinterpret_cast<double*>(base + o_times);
  b.values = reinterpret_cast<double*>(base + o_values);
  b.perr = reinterpret_cast<double*>(base + o_perr);
  b.out = reinterpret_cast<PlainOut*>(base + o_out);
  // basis slots beyond a breakdown stay finite for the Gram
  check_cuda(cudaMemsetAsync(b.base, 0, off, st), "cudaMemsetAsync(plain propagation)");
  check_cuda(cudaMemcpyAsync(b.times, times, sizeof(double) * ntimes, cudaMemcpyHostToDevice, st), "copy times");
  static bool attr = false;
  if (!attr) {
    check_cuda(cudaFuncSetAttribute(k_plain_control, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kPlainSmem),
               "cudaFuncSetAttribute(k_plain_control)");
    attr = true;
  }
  LanczosScalars* sc = scalars(sys);
  const int nb = row_blocks(n);
  double2* partials = reduce_partials(sys, (size_t)nb * (RPM_MAX_KRYLOV + 1));
  PlainOut o{};
  auto run = [&](const PlainIn& in) {
    lanczos_basis_launch(sys, state, in.target, k.breakdown_tolerance, b.basis, b.alpha, b.beta, st);
    if (in.npts > 0) singlet_gram_launch(sys, b.basis, in.built, b.gram, st);
    k_plain_control<<<1, kPlainWarps * 32, kPlainSmem, st>>>(b.alpha, b.beta, sc, in, b.recs, b.gram, b.times,
                                                            b.values, b.perr, b.coef, b.out);
    k_plain_combine<<<nb, kThreads, 0, st>>>(b.basis, n, b.coef, state, partials, &sc->counter[6], b.out);
    check_launch("plain step");
    check_cuda(cudaMemcpyAsync(&o, b.out, sizeof(PlainOut), cudaMemcpyDeviceToHost, st), "copy step record");
    check_cuda(cudaStreamSynchronize(st), "plain step sync");
  };
  const double t_end = times[ntimes - 1];
  double now = 0.0, acc = 0.0, step = t_end > 0.0 ? std::min(k.initial_step_us, t_end) : 0.0;
  double min_used = 0.0, max_used = 0.0, norm_err = norm_error0;
  int accepted = 0, rejected = 0, maxdim = 0, cursor = cursor0;
  long long matvecs = 0;
  bool prefer_max = false;
  struct Seg {
    int first, count;
    double acc;
  };
  std::vector<Seg> segs;
  res->status = 0;
  while (cursor < ntimes) {
    const double trial = std::min(step, t_end - now);
    if (trial < k.minimum_step_us) {
      res->status = 1;
      break;
    }
    int c = cursor;
    while (c < ntimes && times[c] <= now + trial + 1e-13) ++c;
    PlainIn in{};
    in.mode = prefer_max ? 1 : 0;
    in.target = prefer_max ? k.maximum_dimension : k.minimum_dimension;
    in.built = (int)std::min<long long>(in.target, n);
    in.min_dim = k.minimum_dimension;
    in.max_dim = k.maximum_dimension;
    in.inc = k.dimension_increment;
    in.offset = k.embedded_offset;
    in.first = cursor;
    in.npts = c - cursor;
    in.trial = trial;
    in.budget = k.state_error_budget * trial / std::max(t_end, trial);
    in.safety = k.safety_factor;
    in.t_now = now;
    run(in);
    matvecs += o.size;
    if (o.status == 2) {  // the minimum dimension missed the budget: the maximum basis, ladder from min + increment
      prefer_max = true;
      in.mode = 2;
      in.target = k.maximum_dimension;
      in.built = mmax;
      run(in);
      matvecs += o.size;
    }
    if (o.status == 4) fail(RPM_E_INVALID, "Cannot propagate the zero vector.");
    if (o.status == 3) fail(RPM_E_NUMERIC, "tridiagonal eigen-solver did not converge");
    if (o.status == 1) {
      ++rejected;
      step = 0.5 * trial;
      continue;
    }
    maxdim = std::max(maxdim, o.selected);
    if (o.selected > k.minimum_dimension) prefer_max = true;
    if (c > cursor) segs.push_back({cursor, c - cursor, acc});
    cursor = c;
    now = now + trial;
    acc += o.err;
    min_used = accepted ? std::min(min_used, trial) : trial;
    max_used = accepted ? std::max(max_used, trial) : trial;
    ++accepted;
    norm_err = std::max(norm_err, std::fabs(o.new_norm - 1.0));
    step = o.err < 0.1 * in.budget ? std::min(k.maximum_step_us, 1.5 * trial) : trial;
  }
  std::vector<double> perr(ntimes);
  check_cuda(cudaMemcpyAsync(values_host + cursor0, b.values + cursor0, sizeof(double) * (ntimes - cursor0),
                             cudaMemcpyDeviceToHost, st), "copy values");
  check_cuda(cudaMemcpyAsync(perr.data(), b.perr, sizeof(double) * ntimes, cudaMemcpyDeviceToHost, st), "copy errors");
  check_cuda(cudaStreamSynchronize(st), "plain propagation sync");
  for (const Seg& s : segs)
    for (int i = s.first; i < s.first + s.count; ++i) errors_host[i] = s.acc + perr[i];
  res->accepted_steps = accepted;
  res->rejected_steps = rejected;
  res->matvecs = matvecs;
  res->maximum_krylov_dimension = maxdim;
  res->minimum_step_us = min_used;
  res->maximum_step_us = max_used;
  res->accumulated_state_error = acc;
  res->maximum_norm_error = norm_err;
  res->points_done = cursor;
}
}  // namespace rpm

using namespace rpm;

extern "C" {

int rpm_lanczos_basis(rpm_system* sys, const void* state_dev, int max_dim, double breakdown_tol, void* basis_dev,
                      double* alpha_dev, double* beta_dev, int* actual_host, double* norm_host, void* stream) {
  return guarded([&] {
    if (!sys || !state_dev || !basis_dev || !alpha_dev || !beta_dev || !actual_host || !norm_host)
      fail(RPM_E_INVALID, "NULL argument");
    if (!sys->on_device) fail(RPM_E_INVALID, "system was created host-only");
    if (sys->non_hermitian)
      fail(RPM_E_UNSUPPORTED, "Lanczos needs a Hermitian Hamiltonian; unequal recombination rates run on the "
                              "batched propagator (Arnoldi)");
    lanczos_basis(sys, static_cast<const double2*>(state_dev), max_dim, breakdown_tol, static_cast<double2*>(basis_dev),
                  alpha_dev, beta_dev, actual_host, norm_host, static_cast<cudaStream_t>(stream));
  });
}

int rpm_tridiag_spectra(const double* alpha_dev, const double* beta_dev, int ndims, const int* dims_host,
                        double* spectra_dev, void* stream) {
  return guarded([&] {
    if (!alpha_dev || !beta_dev || !dims_host || !spectra_dev || ndims < 1) fail(RPM_E_INVALID, "bad arguments");
    for (int k = 0; k < ndims; ++k)
      if (dims_host[k] < 1 || dims_host[k] > RPM_MAX_KRYLOV) fail(RPM_E_UNSUPPORTED, "Krylov dimension must be in [1, 128]");
    auto st = static_cast<cudaStream_t>(stream);
    int* d_dims = nullptr;
    check_cuda(cudaMallocAsync(&d_dims, sizeof(int) * ndims, st), "cudaMallocAsync(dims)");
    check_cuda(cudaMemcpyAsync(d_dims, dims_host, sizeof(int) * ndims, cudaMemcpyHostToDevice, st), "copy dims");
    const size_t smem = sizeof(double) * (RPM_MAX_KRYLOV * RPM_MAX_KRYLOV + 2 * RPM_MAX_KRYLOV) +
                        sizeof(double2) * RPM_MAX_KRYLOV;
    check_cuda(cudaFuncSetAttribute(k_tridiag_spectra, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
               "cudaFuncSetAttribute(spectra)");
    k_tridiag_spectra<<<ndims, 128, smem, st>>>(alpha_dev, beta_dev, d_dims, spectra_dev);
    check_launch("k_tridiag_spectra");
    check_cuda(cudaFreeAsync(d_dims, st), "cudaFreeAsync(dims)");
  });
}

int rpm_krylov_eval(const double* spectra_dev, int nreq, const rpm_krylov_req* reqs_host, double safety,
                    double state_norm, const void* gram_dev, int gram_ld, void* coef_dev, int coef_ld,
                    double* err_host, double* value_host, void* stream) {
  return guarded([&] {
    if (!spectra_dev || nreq < 1 || !reqs_host || !coef_dev || !err_host) fail(RPM_E_INVALID, "bad arguments");
    if (gram_dev && !value_host) fail(RPM_E_INVALID, "value_host required with a Gram matrix");
    auto st = static_cast<cudaStream_t>(stream);
    const size_t req_bytes = sizeof(rpm_krylov_req) * nreq;
    void* dbuf = nullptr;
    check_cuda(cudaMallocAsync(&dbuf, req_bytes + sizeof(double) * 2 * nreq, st), "cudaMallocAsync(eval)");
    auto* d_req = static_cast<rpm_krylov_req*>(dbuf);
    auto* d_err = reinterpret_cast<double*>(static_cast<char*>(dbuf) + req_bytes);
    double* d_val = d_err + nreq;
    check_cuda(cudaMemcpyAsync(d_req, reqs_host, req_bytes, cudaMemcpyHostToDevice, st), "copy reqs");
    k_krylov_eval<<<nreq, kThreads, 0, st>>>(spectra_dev, d_req, safety, state_norm,
                                              static_cast<const double2*>(gram_dev), gram_ld,
                                              static_cast<double2*>(coef_dev), coef_ld, d_err, d_val);
    check_launch("k_krylov_eval");
    check_cuda(cudaMemcpyAsync(err_host, d_err, sizeof(double) * nreq, cudaMemcpyDeviceToHost, st), "copy err");
    if (gram_dev)
      check_cuda(cudaMemcpyAsync(value_host, d_val, sizeof(double) * nreq, cudaMemcpyDeviceToHost, st), "copy values");
    check_cuda(cudaFreeAsync(dbuf, st), "cudaFreeAsync(eval)");
    check_cuda(cudaStreamSynchronize(st), "eval sync");
  });
}

int rpm_singlet_gram(rpm_system* sys, const void* basis_dev, int m, void* gram_dev, void* stream) {
  return guarded([&] {
    if (!sys || !basis_dev || !gram_dev) fail(RPM_E_INVALID, "NULL argument");
    if (m < 1 || m > 64) fail(RPM_E_UNSUPPORTED, "Gram size must be in [1, 64]");
    if (sys->ndims < 2 || sys->dims[0] != 2 || sys->dims[1] != 2)
      fail(RPM_E_INVALID, "The first two axes must be the two electron spins.");
    singlet_gram_launch(sys, static_cast<const double2*>(basis_dev), m, static_cast<double2*>(gram_dev),
                        static_cast<cudaStream_t>(stream));
  });
}

int rpm_plain_propagate(rpm_system* sys, const rpm_plain_knobs* knobs, void* state_dev, const double* times_host,
                        int ntimes, int cursor0, double norm_error0, double* values_host, double* state_errors_host,
                        rpm_plain_result* result, void* stream) {
  return guarded([&] {
    if (!sys || !knobs || !state_dev || !times_host || !values_host || !state_errors_host || !result)
      fail(RPM_E_INVALID, "NULL argument");
    if (!sys->on_device) fail(RPM_E_INVALID, "system was created host-only");
    if (sys->non_hermitian)
      fail(RPM_E_UNSUPPORTED, "Lanczos needs a Hermitian Hamiltonian; unequal recombination rates run on the "
                              "batched propagator (Arnoldi)");
    if (sys->ndims < 2 || sys->dims[0] != 2 || sys->dims[1] != 2)
      fail(RPM_E_INVALID, "The first two axes must be the two electron spins.");
    const rpm_plain_knobs& k = *knobs;
    if (k.minimum_dimension <= k.embedded_offset || k.embedded_offset < 0)
      fail(RPM_E_INVALID, "minimum_dimension must exceed embedded_offset.");
    if (k.maximum_dimension < k.minimum_dimension)
      fail(RPM_E_INVALID, "maximum_dimension must not be smaller than minimum_dimension.");
    if (k.maximum_dimension > kPlainLD) fail(RPM_E_UNSUPPORTED, "device-driven steps support Krylov dimension <= 64");
    if (k.dimension_increment < 1) fail(RPM_E_INVALID, "dimension_increment must be positive");
    if ((k.maximum_dimension - k.minimum_dimension) / k.dimension_increment + 2 > kPlainMaxCand)
      fail(RPM_E_UNSUPPORTED, "device-driven steps support at most 15 candidate dimensions");
    if (ntimes < 1 || cursor0 < 0 || cursor0 > ntimes) fail(RPM_E_INVALID, "bad observation range");
    for (int i = 0; i < ntimes; ++i)
      if (!(times_host[i] >= 0.0) || (i && !(times_host[i] > times_host[i - 1])))
        fail(RPM_E_INVALID, "Observation times must be nonnegative and strictly increasing.");
    *result = rpm_plain_result{};
    plain_propagate(sys, k, static_cast<double2*>(state_dev), times_host, ntimes, cursor0, norm_error0, values_host,
                    state_errors_host, result, static_cast<cudaStream_t>(stream));
  });
}

int rpm_combine(rpm_system* sys, const void* basis_dev, int m, const void* coef_dev, double scale, void* out_dev,
                double* norm_host, void* stream) {
  return guarded([&] {
    if (!sys || !basis_dev || !coef_dev || !out_dev) fail(RPM_E_INVALID, "NULL argument");
    if (m < 1 || m > RPM_MAX_KRYLOV) fail(RPM_E_UNSUPPORTED, "Krylov dimension must be in [1, 128]");
    auto st = static_cast<cudaStream_t>(stream);
    const int nb = row_blocks(sys->n);
    double2* partials = reduce_partials(sys, (size_t)nb * (RPM_MAX_KRYLOV + 1));
    LanczosScalars* sc = scalars(sys);
    k_combine<<<nb, kThreads, 0, st>>>(static_cast<const double2*>(basis_dev), sys->n, m,
                                       static_cast<const double2*>(coef_dev), scale, static_cast<double2*>(out_dev),
                                       partials, &sc->counter[5], &sc->norm);
    check_launch("k_combine");
    if (norm_host) {
      check_cuda(cudaMemcpyAsync(norm_host, &sc->norm, sizeof(double), cudaMemcpyDeviceToHost, st), "copy norm");
      check_cuda(cudaStreamSynchronize(st), "combine sync");
    }
  });
}

static int batch_reduce(long long n, const void* psi, int batch, long long ld, int kind, double* host,
                        void* stream) {
  return guarded([&] {
    if (!psi || !host || batch < 1 || n < 1 || ld < n) fail(RPM_E_INVALID, "bad arguments");
    if (kind == 1 && n % 4 != 0) fail(RPM_E_INVALID, "The first two axes must be the two electron spins.");
    auto st = static_cast<cudaStream_t>(stream);
    double* d_out = nullptr;
    check_cuda(cudaMallocAsync(&d_out, sizeof(double) * batch, st), "cudaMallocAsync(reduce)");
    k_batch_reduce<<<batch, kThreads, 0, st>>>(static_cast<const double2*>(psi), n, ld, kind, d_out);
    check_launch("k_batch_reduce");
    check_cuda(cudaMemcpyAsync(host, d_out, sizeof(double) * batch, cudaMemcpyDeviceToHost, st), "copy reduce");
    check_cuda(cudaFreeAsync(d_out, st), "cudaFreeAsync(reduce)");
    check_cuda(cudaStreamSynchronize(st), "reduce sync");
  });
}

int rpm_singlet_population(const void* psi_dev, long long n, int batch, long long ld, double* values_host,
                           void* stream) {
  return batch_reduce(n, psi_dev, batch, ld, 1, values_host, stream);
}

int rpm_norm(rpm_system* sys, const void* psi_dev, double* norm_host, void* stream) {
  if (!sys) {
    set_last_error("system is NULL");
    return RPM_E_INVALID;
  }
  const int rc = batch_reduce(sys->n, psi_dev, 1, sys->n, 0, norm_host, stream);
  if (rc == RPM_OK) *norm_host = std::sqrt(*norm_host);
  return rc;
}

int rpm_simpson_yield(const double* times_dev, const double* pops_dev, int n, int batch, long long ld,
                      double lifetime_us, double* yields_dev, void* stream) {
  return guarded([&] {
    if (!times_dev || !pops_dev || !yields_dev || n < 1 || batch < 1 || ld < n || !(lifetime_us > 0.0))
      fail(RPM_E_INVALID, "bad arguments");
    auto st = static_cast<cudaStream_t>(stream);
    k_simpson<<<batch, kThreads, 0, st>>>(times_dev, pops_dev, n, ld, lifetime_us, yields_dev);
    check_launch("k_simpson");
  });
}

}  // extern "C"

namespace rpm {

// out = (1 (x) ... (x) U (x) ... (x) 1) in for a d x d operator U on one axis
// (any operator; used for instantaneous unitaries between propagation segments).
__global__ void __launch_bounds__(256) k_apply_local(const double2* __restrict__ in, double2* __restrict__ out,
                                                    long long n, long long ld, long long stride, int d,
                                                    const double2* __restrict__ op) {
  const double2* u = op;  // d x d, read through the read-only cache
  const double2* x = in + (long long)blockIdx.y * ld;
  double2* y = out + (long long)blockIdx.y * ld;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int digit = (int)((i / stride) % d);
    const long long base = i - (long long)digit * stride;
    double2 acc = make_double2(0.0, 0.0);
    for (int c = 0; c < d; ++c) acc = cfma(__ldg(u + digit * d + c), x[base + (long long)c * stride], acc);
    y[i] = acc;
  }
}

}  // namespace rpm

extern "C" int rpm_apply_local_operator(const int* dims, int ndims, int axis, const double* op_host, const void* in_dev,
                                        void* out_dev, int batch, long long ld, void* stream) {
  return guarded([&] {
    if (!dims || ndims < 1 || ndims > RPM_MAX_AXES || !op_host || !in_dev || !out_dev || batch < 1)
      fail(RPM_E_INVALID, "bad arguments");
    if (axis < 0 || axis >= ndims) fail(RPM_E_INVALID, "axis out of range");
    if (in_dev == out_dev) fail(RPM_E_INVALID, "local operator cannot be applied in place");
    long long n = 1, stride = 1;
    for (int a = 0; a < ndims; ++a) {
      if (dims[a] < 1) fail(RPM_E_INVALID, "Every tensor dimension must be positive.");
      n *= dims[a];
    }
    for (int a = ndims - 1; a > axis; --a) stride *= dims[a];
    if (ld < n) fail(RPM_E_INVALID, "leading dimension smaller than the state");
    const int d = dims[axis];
    if (d > RPM_MAX_LOCAL_DIM) fail(RPM_E_UNSUPPORTED, "axis dimension above 64");
    auto st = static_cast<cudaStream_t>(stream);
    double2* d_op = nullptr;
    check_cuda(cudaMallocAsync(&d_op, sizeof(double2) * d * d, st), "cudaMallocAsync(op)");
    check_cuda(cudaMemcpyAsync(d_op, op_host, sizeof(double2) * d * d, cudaMemcpyHostToDevice, st), "copy op");
    const int blocks = (int)std::min<long long>((n + 255) / 256, 4096);
    k_apply_local<<<dim3(blocks, batch), 256, 0, st>>>(static_cast<const double2*>(in_dev),
                                                       static_cast<double2*>(out_dev), n, ld, stride, d, d_op);
    check_launch("k_apply_local");
    check_cuda(cudaFreeAsync(d_op, st), "cudaFreeAsync(op)");
  });
}
