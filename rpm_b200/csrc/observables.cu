// Stored-state observables: reduced density matrices of a bipartition.
//
// For a pure state psi and a split of its tensor axes into a kept part A
// (index a) and a traced part C (index c), M[a][c] = psi[offa[a] + offc[c]]
// and rho_A = M M^H, i.e. rho_A[a][b] = sum_c psi[a, c] conj(psi[b, c]).
// Its eigenvalues are the squared Schmidt coefficients, which give the
// reference's entanglement observables (poster_reproduction/core.py:311-365):
//   * pure_log_negativity(state, dims, left_axes) = 2 log2(sum sigma / |sigma|)
//     with sigma = sqrt(eig(rho_A)) for A = left_axes (or its complement);
//   * reduced_electron_density(state, dims) = rho of the electron pair
//     (A = axes 0, 1), hermitised.
// Two kernels, FP64 throughout:
//   * small A (da <= 4): one CTA per state, threads stride over c, each
//     holds the da (da + 1) / 2 upper-triangle sums, block reduction in a
//     fixed order (deterministic);
//   * any A: one CTA per (state, 32 x 32 tile of the upper triangle),
//     contraction over c in chunks of 32 staged in shared memory, 2 x 2
//     outputs per thread; the lower triangle is written mirrored.
#include "common.cuh"

namespace rpm {
namespace {

constexpr int kSmallThreads = 256;

__device__ __forceinline__ double2 cmul_conj_b(double2 x, double2 y) {  // x * conj(y)
  return make_double2(x.x * y.x + x.y * y.y, x.y * y.x - x.x * y.y);
}

template <int DA>
__global__ void __launch_bounds__(kSmallThreads) k_rdm_small(const double2* __restrict__ states, long long ld,
                                                             const long long* __restrict__ offa,
                                                             const long long* __restrict__ offc, long long dc,
                                                             double2* __restrict__ rho) {
  constexpr int NP = DA * (DA + 1) / 2;
  __shared__ double2 red[kSmallThreads / 32][NP];
  __shared__ long long oa[DA];
  const double2* psi = states + (long long)blockIdx.x * ld;
  if (threadIdx.x < DA) oa[threadIdx.x] = offa[threadIdx.x];
  __syncthreads();
  double2 acc[NP];
#pragma unroll
  for (int p = 0; p < NP; ++p) acc[p] = make_double2(0.0, 0.0);
  for (long long c = threadIdx.x; c < dc; c += blockDim.x) {
    const long long base = offc[c];
    double2 v[DA];
#pragma unroll
    for (int a = 0; a < DA; ++a) v[a] = psi[oa[a] + base];
    int p = 0;
#pragma unroll
    for (int a = 0; a < DA; ++a)
#pragma unroll
      for (int b = a; b < DA; ++b, ++p) acc[p] = cadd(acc[p], cmul_conj_b(v[a], v[b]));
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int p = 0; p < NP; ++p) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      acc[p].x += __shfl_xor_sync(0xffffffffu, acc[p].x, o);
      acc[p].y += __shfl_xor_sync(0xffffffffu, acc[p].y, o);
    }
    if (lane == 0) red[warp][p] = acc[p];
  }
  __syncthreads();
  if (threadIdx.x < NP) {
    double2 s = make_double2(0.0, 0.0);
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s = cadd(s, red[w][threadIdx.x]);
    int a = 0, rem = threadIdx.x;
    while (rem >= DA - a) {
      rem -= DA - a;
      ++a;
    }
    const int b = a + rem;
    double2* out = rho + (long long)blockIdx.x * DA * DA;
    out[a * DA + b] = s;
    out[b * DA + a] = make_double2(s.x, -s.y);
  }
}

constexpr int kTile = 32;

__global__ void __launch_bounds__(256) k_rdm_tiled(const double2* __restrict__ states, long long ld,
                                                   const long long* __restrict__ offa, int da,
                                                   const long long* __restrict__ offc, long long dc, int ntiles,
                                                   double2* __restrict__ rho) {
  __shared__ double2 ta[kTile][kTile + 1];  // [c][a]
  __shared__ double2 tb[kTile][kTile + 1];  // [c][b]
  // upper-triangle tile (ti <= tj) of this block
  int ti = 0, rem = blockIdx.x;
  while (rem >= ntiles - ti) {
    rem -= ntiles - ti;
    ++ti;
  }
  const int tj = ti + rem;
  const double2* psi = states + (long long)blockIdx.y * ld;
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;  // 16 x 16 threads, 2 x 2 outputs each
  double2 acc[2][2];
#pragma unroll
  for (int p = 0; p < 2; ++p)
#pragma unroll
    for (int q = 0; q < 2; ++q) acc[p][q] = make_double2(0.0, 0.0);
  for (long long c0 = 0; c0 < dc; c0 += kTile) {
    __syncthreads();
    for (int idx = threadIdx.x; idx < kTile * kTile; idx += blockDim.x) {
      const int cc = idx / kTile, aa = idx % kTile;
      const long long c = c0 + cc;
      const int a = ti * kTile + aa, b = tj * kTile + aa;
      double2 va = make_double2(0.0, 0.0), vb = make_double2(0.0, 0.0);
      if (c < dc) {
        const long long oc = offc[c];
        if (a < da) va = psi[offa[a] + oc];
        if (b < da) vb = psi[offa[b] + oc];
      }
      ta[cc][aa] = va;
      tb[cc][aa] = vb;
    }
    __syncthreads();
#pragma unroll 4
    for (int cc = 0; cc < kTile; ++cc) {
      const double2 a0 = ta[cc][ty], a1 = ta[cc][ty + 16];
      const double2 b0 = tb[cc][tx], b1 = tb[cc][tx + 16];
      acc[0][0] = cadd(acc[0][0], cmul_conj_b(a0, b0));
      acc[0][1] = cadd(acc[0][1], cmul_conj_b(a0, b1));
      acc[1][0] = cadd(acc[1][0], cmul_conj_b(a1, b0));
      acc[1][1] = cadd(acc[1][1], cmul_conj_b(a1, b1));
    }
  }
  double2* out = rho + (long long)blockIdx.y * da * da;
#pragma unroll
  for (int p = 0; p < 2; ++p)
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      const int a = ti * kTile + ty + 16 * p, b = tj * kTile + tx + 16 * q;
      if (a < da && b < da && (ti != tj || a <= b)) {
        out[(long long)a * da + b] = acc[p][q];
        if (a != b) out[(long long)b * da + a] = make_double2(acc[p][q].x, -acc[p][q].y);
      }
    }
}

// Schmidt norms from the eigenvectors U of rho_A (per state, da x da,
// column i = eigenvector i): sigma2[i] = sum_c |sum_a conj(U[a][i]) M[a][c]|^2.
// Computing W = U^H M and its row norms keeps small Schmidt values accurate
// to ~eps |M| (the eigenvalues of rho_A themselves only resolve sqrt(eps)).
template <int DA>
__global__ void __launch_bounds__(kSmallThreads) k_schmidt_small(const double2* __restrict__ states, long long ld,
                                                                 const long long* __restrict__ offa,
                                                                 const long long* __restrict__ offc, long long dc,
                                                                 const double2* __restrict__ u,
                                                                 double* __restrict__ sigma2) {
  __shared__ double red[kSmallThreads / 32][DA];
  __shared__ long long oa[DA];
  __shared__ double2 us[DA * DA];
  const double2* psi = states + (long long)blockIdx.x * ld;
  if (threadIdx.x < DA) oa[threadIdx.x] = offa[threadIdx.x];
  if (threadIdx.x < DA * DA) us[threadIdx.x] = u[(long long)blockIdx.x * DA * DA + threadIdx.x];
  __syncthreads();
  double acc[DA];
#pragma unroll
  for (int i = 0; i < DA; ++i) acc[i] = 0.0;
  for (long long c = threadIdx.x; c < dc; c += blockDim.x) {
    const long long base = offc[c];
    double2 v[DA];
#pragma unroll
    for (int a = 0; a < DA; ++a) v[a] = psi[oa[a] + base];
#pragma unroll
    for (int i = 0; i < DA; ++i) {
      double2 w = make_double2(0.0, 0.0);
#pragma unroll
      for (int a = 0; a < DA; ++a) {
        const double2 q = us[a * DA + i];  // conj(q) * v
        w.x = fma(q.x, v[a].x, fma(q.y, v[a].y, w.x));
        w.y = fma(q.x, v[a].y, fma(-q.y, v[a].x, w.y));
      }
      acc[i] = fma(w.x, w.x, fma(w.y, w.y, acc[i]));
    }
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int i = 0; i < DA; ++i) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc[i] += __shfl_xor_sync(0xffffffffu, acc[i], o);
    if (lane == 0) red[warp][i] = acc[i];
  }
  __syncthreads();
  if (threadIdx.x < DA) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w][threadIdx.x];
    sigma2[(long long)blockIdx.x * DA + threadIdx.x] = t;
  }
}

// General da: one CTA per (state, 32-row tile of i); W tile = U^H M tile with
// the contraction over a staged 32 at a time; |W|^2 summed over c per row.
__global__ void __launch_bounds__(256) k_schmidt_tiled(const double2* __restrict__ states, long long ld,
                                                       const long long* __restrict__ offa, int da,
                                                       const long long* __restrict__ offc, long long dc,
                                                       const double2* __restrict__ u, double* __restrict__ sigma2) {
  __shared__ double2 ut[kTile][kTile + 1];  // [a][i]
  __shared__ double2 mt[kTile][kTile + 1];  // [a][c]
  __shared__ double rows[kTile][17];
  const int ti = blockIdx.x;
  const long long s = blockIdx.y;
  const double2* psi = states + s * ld;
  const double2* us = u + s * (long long)da * da;
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;  // ty: i (two rows), tx: c (two columns)
  double norm2[2] = {0.0, 0.0};
  for (long long c0 = 0; c0 < dc; c0 += kTile) {
    double2 w[2][2];
#pragma unroll
    for (int p = 0; p < 2; ++p)
#pragma unroll
      for (int q = 0; q < 2; ++q) w[p][q] = make_double2(0.0, 0.0);
    for (int a0 = 0; a0 < da; a0 += kTile) {
      __syncthreads();
      for (int idx = threadIdx.x; idx < kTile * kTile; idx += blockDim.x) {
        const int r = idx / kTile, k = idx % kTile;
        const int a = a0 + r, i = ti * kTile + k;
        const long long c = c0 + k;
        ut[r][k] = (a < da && i < da) ? us[(long long)a * da + i] : make_double2(0.0, 0.0);
        mt[r][k] = (a < da && c < dc) ? psi[offa[a] + offc[c]] : make_double2(0.0, 0.0);
      }
      __syncthreads();
#pragma unroll 4
      for (int r = 0; r < kTile; ++r) {
#pragma unroll
        for (int p = 0; p < 2; ++p) {
          const double2 q = ut[r][ty + 16 * p];
#pragma unroll
          for (int qq = 0; qq < 2; ++qq) {
            const double2 v = mt[r][tx + 16 * qq];
            w[p][qq].x = fma(q.x, v.x, fma(q.y, v.y, w[p][qq].x));
            w[p][qq].y = fma(q.x, v.y, fma(-q.y, v.x, w[p][qq].y));
          }
        }
      }
    }
#pragma unroll
    for (int p = 0; p < 2; ++p)
#pragma unroll
      for (int qq = 0; qq < 2; ++qq) norm2[p] = fma(w[p][qq].x, w[p][qq].x, fma(w[p][qq].y, w[p][qq].y, norm2[p]));
  }
  // sum the 16 column-threads of each row in a fixed order
  rows[ty][tx] = norm2[0];
  rows[ty + 16][tx] = norm2[1];
  __syncthreads();
  if (threadIdx.x < kTile) {
    const int i = ti * kTile + threadIdx.x;
    double t = 0.0;
    for (int k = 0; k < 16; ++k) t += rows[threadIdx.x][k];
    if (i < da) sigma2[s * da + i] = t;
  }
}

// Transition lines of one radical, deposited with linear interpolation onto a
// centred frequency grid (rpm_quantum_needle_reproduction.py:128-170):
// line (i, j) has frequency lam[i] - lam[j] and weight sp[i][j] sq[j][i] *
// scale; grid bin = frequency / delta + half_width.  FP64 atomics (the order
// of additions is not fixed: results agree to rounding).
__global__ void k_bin_lines(const double* __restrict__ lam, const double2* __restrict__ sp,
                            const double2* __restrict__ sq, int d, double scale, double delta, long long half_width,
                            long long size, double2* __restrict__ grid, int* __restrict__ bad) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)d * d) return;
  const int i = (int)(idx / d), j = (int)(idx - (long long)i * d);
  const double2 a = sp[(long long)i * d + j], b = sq[(long long)j * d + i];
  const double cx = (a.x * b.x - a.y * b.y) * scale, cy = (a.x * b.y + a.y * b.x) * scale;
  const double pos = (lam[i] - lam[j]) / delta + (double)half_width;
  const double fl = floor(pos);
  const long long lower = (long long)fl;
  const double frac = pos - fl;
  if (lower < 0 || lower + 1 >= size) {
    atomicExch(bad, 1);
    return;
  }
  atomicAdd(&grid[lower].x, cx * (1.0 - frac));
  atomicAdd(&grid[lower].y, cy * (1.0 - frac));
  atomicAdd(&grid[lower + 1].x, cx * frac);
  atomicAdd(&grid[lower + 1].y, cy * frac);
}

}  // namespace
}  // namespace rpm

extern "C" int rpm_bin_transition_lines(const double* lam_dev, const void* sp_dev, const void* sq_dev, int d,
                                        double scale, double delta, long long half_width, void* grid_dev,
                                        int* bad_dev, void* stream) {
  return rpm::guarded([&] {
    if (!lam_dev || !sp_dev || !sq_dev || !grid_dev || !bad_dev) rpm::fail(RPM_E_INVALID, "NULL pointer");
    if (d < 1 || !(delta > 0.0) || half_width < 1) rpm::fail(RPM_E_INVALID, "invalid line-binning arguments");
    const long long lines = (long long)d * d;
    const long long blocks = (lines + 255) / 256;
    rpm::k_bin_lines<<<(unsigned)blocks, 256, 0, static_cast<cudaStream_t>(stream)>>>(
        lam_dev, static_cast<const double2*>(sp_dev), static_cast<const double2*>(sq_dev), d, scale, delta,
        half_width, 2 * half_width + 1, static_cast<double2*>(grid_dev), bad_dev);
    rpm::check_launch("k_bin_lines");
  });
}

extern "C" int rpm_schmidt_norms(const void* states_dev, long long nstates, long long ld, const long long* offa_dev,
                                 int da, const long long* offc_dev, long long dc, const void* u_dev, double* sigma2_dev,
                                 void* stream) {
  return rpm::guarded([&] {
    if (!states_dev || !offa_dev || !offc_dev || !u_dev || !sigma2_dev) rpm::fail(RPM_E_INVALID, "NULL pointer");
    if (nstates < 0 || da < 1 || dc < 1 || ld < 1) rpm::fail(RPM_E_INVALID, "invalid sizes");
    if (nstates == 0) return;
    auto st = static_cast<cudaStream_t>(stream);
    const auto* s = static_cast<const double2*>(states_dev);
    const auto* u = static_cast<const double2*>(u_dev);
    if (da <= 4 && nstates <= 2147483647LL) {
      switch (da) {
        case 1: rpm::k_schmidt_small<1><<<(unsigned)nstates, rpm::kSmallThreads, 0, st>>>(s, ld, offa_dev, offc_dev, dc, u, sigma2_dev); break;
        case 2: rpm::k_schmidt_small<2><<<(unsigned)nstates, rpm::kSmallThreads, 0, st>>>(s, ld, offa_dev, offc_dev, dc, u, sigma2_dev); break;
        case 3: rpm::k_schmidt_small<3><<<(unsigned)nstates, rpm::kSmallThreads, 0, st>>>(s, ld, offa_dev, offc_dev, dc, u, sigma2_dev); break;
        default: rpm::k_schmidt_small<4><<<(unsigned)nstates, rpm::kSmallThreads, 0, st>>>(s, ld, offa_dev, offc_dev, dc, u, sigma2_dev); break;
      }
      rpm::check_launch("k_schmidt_small");
      return;
    }
    if (nstates > 65535) rpm::fail(RPM_E_UNSUPPORTED, "at most 65535 states per call for kept dimensions above 4");
    const int nt = (da + rpm::kTile - 1) / rpm::kTile;
    rpm::k_schmidt_tiled<<<dim3(nt, (unsigned)nstates), 256, 0, st>>>(s, ld, offa_dev, da, offc_dev, dc, u, sigma2_dev);
    rpm::check_launch("k_schmidt_tiled");
  });
}

extern "C" int rpm_reduced_density(const void* states_dev, long long nstates, long long ld,
                                   const long long* offa_dev, int da, const long long* offc_dev, long long dc,
                                   void* rho_dev, void* stream) {
  return rpm::guarded([&] {
    if (!states_dev || !offa_dev || !offc_dev || !rho_dev) rpm::fail(RPM_E_INVALID, "NULL pointer");
    if (nstates < 0 || da < 1 || dc < 1 || ld < 1) rpm::fail(RPM_E_INVALID, "invalid sizes");
    if (nstates == 0) return;
    if (nstates > 65535LL * 65535LL) rpm::fail(RPM_E_UNSUPPORTED, "too many states in one call");
    auto st = static_cast<cudaStream_t>(stream);
    const auto* s = static_cast<const double2*>(states_dev);
    auto* r = static_cast<double2*>(rho_dev);
    if (da <= 4 && nstates <= 2147483647LL) {
      switch (da) {
        case 1: rpm::k_rdm_small<1><<<(unsigned)nstates, rpm::kSmallThreads, 0, st>>>(s, ld, offa_dev, offc_dev, dc, r); break;
        case 2: rpm::k_rdm_small<2><<<(unsigned)nstates, rpm::kSmallThreads, 0, st>>>(s, ld, offa_dev, offc_dev, dc, r); break;
        case 3: rpm::k_rdm_small<3><<<(unsigned)nstates, rpm::kSmallThreads, 0, st>>>(s, ld, offa_dev, offc_dev, dc, r); break;
        default: rpm::k_rdm_small<4><<<(unsigned)nstates, rpm::kSmallThreads, 0, st>>>(s, ld, offa_dev, offc_dev, dc, r); break;
      }
      rpm::check_launch("k_rdm_small");
      return;
    }
    if (nstates > 65535) rpm::fail(RPM_E_UNSUPPORTED, "at most 65535 states per call for kept dimensions above 4");
    const int nt = (da + rpm::kTile - 1) / rpm::kTile;
    const int nup = nt * (nt + 1) / 2;
    rpm::k_rdm_tiled<<<dim3(nup, (unsigned)nstates), 256, 0, st>>>(s, ld, offa_dev, da, offc_dev, dc, nt, r);
    rpm::check_launch("k_rdm_tiled");
  });
}
