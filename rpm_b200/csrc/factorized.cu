// Kernels of the factorized exact oracle (rpm_quantum_needle_reproduction.py:
// 93-240): batched Hermitian eigen-decompositions of the radical
// Hamiltonians (FAD 576, TrpH 384 dimensions; one matrix per field
// orientation), eigenbasis spin operators (complex products A^H B) and the
// FFT convolution of the binned transition spectra.  All FP64.
//
// Eigen-decomposition (one CTA per matrix):
//   k_he_tridiag  Householder reduction Q^H A Q = T with a real symmetric
//                 tridiagonal T (the reflectors of LAPACK's zlarfg / zhetd2,
//                 lower form: H = I - tau v v^H, v[0] = 1, H^H [a; x] = [b; 0]
//                 with b real), the full trailing matrix updated by the
//                 Hermitian rank-2 update;
//   k_he_tridiag_eig  implicit symmetric tridiagonal QR with Wilkinson shifts
//                 (krylov.cuh tridiag_qr) with the eigenvectors of T;
//   k_he_back     V = Q Z, the reflectors applied to Z in reverse order, 32
//                 columns per CTA.
// Eigenvalues come out in QR order and are sorted ascending with their
// vectors (k_he_sort), as LAPACK returns them.
#include <algorithm>
#include <cfloat>
#include <vector>

#include "common.cuh"
#include "krylov.cuh"

namespace rpm {
namespace {

constexpr int kHeThreads = 1024;
constexpr int kHeMaxN = 1024;

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }

__device__ __forceinline__ double warp_reduce(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Sum over the block (every thread returns the total).
__device__ double block_reduce_sum(double v, double* red) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  __syncthreads();
  v = warp_reduce(v);
  if (lane == 0) red[warp] = v;
  __syncthreads();
  if (warp == 0) {
    double t = lane < nw ? red[lane] : 0.0;
    t = warp_reduce(t);
    if (lane == 0) red[0] = t;
  }
  __syncthreads();
  return red[0];
}

// Householder reduction of matrix b: a (n x n, row-major, overwritten), d, e
// (n, n - 1 real), house (n x n: row k holds v_k, v_k[j] for j > k, v_k[k+1]
// = 1), tau (n - 1 complex).
__global__ void __launch_bounds__(kHeThreads) k_he_tridiag(double2* a_all, int n, double* d_all, double* e_all,
                                                          double2* house_all, double2* tau_all) {
  __shared__ double2 v[kHeMaxN], w[kHeMaxN];
  __shared__ double red[32];
  __shared__ double2 s_tau;
  __shared__ double s_beta;
  const size_t nn = (size_t)n * n;
  double2* a = a_all + blockIdx.x * nn;
  double* d = d_all + (size_t)blockIdx.x * n;
  double* e = e_all + (size_t)blockIdx.x * n;
  double2* house = house_all + blockIdx.x * nn;
  double2* tau = tau_all + (size_t)blockIdx.x * n;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int k = 0; k + 1 < n; ++k) {
    const int m = n - k - 1;  // trailing size
    // x = A[k+1:, k] = conj(A[k, k+1:]) (A Hermitian, full storage)
    double part = 0.0;
    for (int j = 1 + threadIdx.x; j < m; j += blockDim.x) {
      const double2 x = a[(size_t)k * n + k + 1 + j];
      part += x.x * x.x + x.y * x.y;
    }
    const double xnorm2 = block_reduce_sum(part, red);
    if (threadIdx.x == 0) {
      const double2 alpha = cconj(a[(size_t)k * n + k + 1]);
      if (xnorm2 == 0.0 && alpha.y == 0.0) {
        s_tau = make_double2(0.0, 0.0);
        s_beta = alpha.x;
      } else {
        const double beta = -copysign(sqrt(alpha.x * alpha.x + alpha.y * alpha.y + xnorm2), alpha.x);
        s_tau = make_double2((beta - alpha.x) / beta, -alpha.y / beta);
        s_beta = beta;
        // 1 / (alpha - beta)
        const double2 den = make_double2(alpha.x - beta, alpha.y);
        const double dd = den.x * den.x + den.y * den.y;
        w[0] = make_double2(den.x / dd, -den.y / dd);
      }
    }
    __syncthreads();
    const double2 t = s_tau;
    const bool reflect = t.x != 0.0 || t.y != 0.0;
    const double2 scale = w[0];
    __syncthreads();
    for (int j = threadIdx.x; j < m; j += blockDim.x) {
      double2 vj = make_double2(1.0, 0.0);
      if (j > 0) vj = reflect ? cmul(cconj(a[(size_t)k * n + k + 1 + j]), scale) : make_double2(0.0, 0.0);
      v[j] = vj;
      house[(size_t)k * n + k + 1 + j] = vj;
    }
    if (threadIdx.x == 0) {
      tau[k] = t;
      d[k] = a[(size_t)k * n + k].x;
      e[k] = s_beta;
    }
    __syncthreads();
    if (reflect) {
      // w = tau A22 v, one warp per row (lanes over the row's columns)
      for (int i = warp; i < m; i += nw) {
        const double2* row = a + (size_t)(k + 1 + i) * n + k + 1;
        double sx = 0.0, sy = 0.0;
        for (int j = lane; j < m; j += 32) {
          const double2 p = cmul(row[j], v[j]);
          sx += p.x;
          sy += p.y;
        }
        sx = warp_reduce(sx);
        sy = warp_reduce(sy);
        if (lane == 0) w[i] = cmul(t, make_double2(sx, sy));
      }
      __syncthreads();
      // alpha = -1/2 tau (w^H v); w += alpha v
      double px = 0.0, py = 0.0;
      for (int j = threadIdx.x; j < m; j += blockDim.x) {
        const double2 p = cmul(cconj(w[j]), v[j]);
        px += p.x;
        py += p.y;
      }
      const double wx = block_reduce_sum(px, red);
      const double wy = block_reduce_sum(py, red);
      const double2 al = cmul(make_double2(-0.5 * t.x, -0.5 * t.y), make_double2(wx, wy));
      for (int j = threadIdx.x; j < m; j += blockDim.x) {
        const double2 p = cmul(al, v[j]);
        w[j] = make_double2(w[j].x + p.x, w[j].y + p.y);
      }
      __syncthreads();
      // A22 -= v w^H + w v^H (full storage)
      for (size_t idx = threadIdx.x; idx < (size_t)m * m; idx += blockDim.x) {
        const int i = (int)(idx / m), j = (int)(idx - (size_t)i * m);
        const double2 p = cmul(v[i], cconj(w[j]));
        const double2 q = cmul(w[i], cconj(v[j]));
        double2& x = a[(size_t)(k + 1 + i) * n + k + 1 + j];
        x = make_double2(x.x - p.x - q.x, x.y - p.y - q.y);
      }
      __syncthreads();
    }
  }
  if (threadIdx.x == 0) d[n - 1] = a[(size_t)(n - 1) * n + n - 1].x;
}

// Eigenvalues and eigenvectors of the tridiagonal T of matrix b: z (n x n,
// row i = component i), eigenvalues into d (QR order), status[b] = 0 on
// convergence.
__global__ void __launch_bounds__(256) k_he_tridiag_eig(double* d_all, double* e_all, double* z_all, int n,
                                                       int* status) {
  __shared__ double ds[kHeMaxN], es[kHeMaxN];
  __shared__ double2 rot[kHeMaxN];
  double* d = d_all + (size_t)blockIdx.x * n;
  const double* e = e_all + (size_t)blockIdx.x * n;
  double* z = z_all + (size_t)blockIdx.x * n * n;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    ds[i] = d[i];
    es[i] = i + 1 < n ? e[i] : 0.0;
  }
  __syncthreads();
  const int bad = tridiag_qr(n, ds, es, z, n, rot);
  for (int i = threadIdx.x; i < n; i += blockDim.x) d[i] = ds[i];
  if (threadIdx.x == 0) status[blockIdx.x] = bad;
}

// Ascending order of the eigenvalues: perm[r] = index of the r-th smallest
// (ties by index), sorted values into w.
__global__ void __launch_bounds__(256) k_he_sort(const double* d_all, int n, int* perm_all, double* w_all) {
  const double* d = d_all + (size_t)blockIdx.x * n;
  int* perm = perm_all + (size_t)blockIdx.x * n;
  double* w = w_all + (size_t)blockIdx.x * n;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const double x = d[i];
    int r = 0;
    for (int j = 0; j < n; ++j) {
      const double y = d[j];
      r += (y < x || (y == x && j < i)) ? 1 : 0;
    }
    perm[r] = i;
    w[r] = x;
  }
}

// V = Q Z[:, perm]: 32 output columns per CTA (lanes), 8 row groups (warps);
// the reflectors H_k = I - tau_k v_k v_k^H applied for k = n-2 .. 0.
__global__ void __launch_bounds__(256) k_he_back(const double* z_all, const int* perm_all, const double2* house_all,
                                                const double2* tau_all, int n, double2* v_all) {
  __shared__ double2 part[8][32];
  const size_t nn = (size_t)n * n;
  const int b = blockIdx.y;
  const double* z = z_all + b * nn;
  const int* perm = perm_all + (size_t)b * n;
  const double2* house = house_all + b * nn;
  const double2* tau = tau_all + (size_t)b * n;
  double2* v = v_all + b * nn;
  const int lane = threadIdx.x & 31, g = threadIdx.x >> 5;
  const int c = blockIdx.x * 32 + lane;
  const bool col = c < n;
  const int src = col ? perm[c] : 0;
  for (int i = g; i < n; i += 8)
    if (col) v[(size_t)i * n + c] = make_double2(z[(size_t)i * n + src], 0.0);
  __syncthreads();
  for (int k = n - 2; k >= 0; --k) {
    const double2 t = tau[k];
    if (t.x == 0.0 && t.y == 0.0) continue;  // uniform: H_k = I
    const double2* hv = house + (size_t)k * n;
    double2 s = make_double2(0.0, 0.0);
    if (col)
      for (int i = k + 1 + g; i < n; i += 8) {
        const double2 p = cmul(cconj(hv[i]), v[(size_t)i * n + c]);
        s.x += p.x;
        s.y += p.y;
      }
    part[g][lane] = s;
    __syncthreads();
    double2 tot = make_double2(0.0, 0.0);
#pragma unroll
    for (int q = 0; q < 8; ++q) tot = make_double2(tot.x + part[q][lane].x, tot.y + part[q][lane].y);
    const double2 ts = cmul(t, tot);
    if (col)
      for (int i = k + 1 + g; i < n; i += 8) {
        const double2 p = cmul(hv[i], ts);
        double2& x = v[(size_t)i * n + c];
        x = make_double2(x.x - p.x, x.y - p.y);
      }
    __syncthreads();
  }
}

// C = A^H B for square n x n complex matrices (row-major), 16 x 16 tiles;
// grid (tiles, tiles, batch).
__global__ void __launch_bounds__(256) k_zgemm_hn(const double2* a_all, const double2* b_all, double2* c_all,
                                                 int n) {
  __shared__ double2 at[16][17], bt[16][17];
  const size_t nn = (size_t)n * n;
  const double2* a = a_all + blockIdx.z * nn;
  const double2* b = b_all + blockIdx.z * nn;
  double2* c = c_all + blockIdx.z * nn;
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const int i = blockIdx.y * 16 + ty, j = blockIdx.x * 16 + tx;
  double2 acc = make_double2(0.0, 0.0);
  for (int k0 = 0; k0 < n; k0 += 16) {
    // at[kk][ii] = A[k0 + kk][i0 + ii], bt[kk][jj] = B[k0 + kk][j0 + jj]
    const int kk = ty, ii = tx;
    const int ka = k0 + kk;
    at[kk][ii] = (ka < n && blockIdx.y * 16 + ii < n) ? a[(size_t)ka * n + blockIdx.y * 16 + ii] : make_double2(0.0, 0.0);
    bt[kk][ii] = (ka < n && blockIdx.x * 16 + ii < n) ? b[(size_t)ka * n + blockIdx.x * 16 + ii] : make_double2(0.0, 0.0);
    __syncthreads();
#pragma unroll
    for (int q = 0; q < 16; ++q) {
      const double2 x = cconj(at[q][ty]), y = bt[q][tx];
      acc.x = fma(x.x, y.x, fma(-x.y, y.y, acc.x));
      acc.y = fma(x.x, y.y, fma(x.y, y.x, acc.y));
    }
    __syncthreads();
  }
  if (i < n && j < n) c[(size_t)i * n + j] = acc;
}

// Radix-2 FFT (power-of-two n, batch of rows): bit-reversal permutation, then
// log2 n butterfly passes in place; sign -1 forward, +1 inverse (unscaled).
__global__ void k_fft_bitrev(const double2* in, double2* out, int n, int logn, long long total) {
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    const long long row = t / n;
    const int i = (int)(t - row * n);
    const int r = (int)(__brev((unsigned)i) >> (32 - logn));
    out[row * n + r] = in[t];
  }
}
__global__ void k_fft_pass(double2* x, int n, int half, double sign, long long total_half) {
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total_half;
       t += (long long)gridDim.x * blockDim.x) {
    const long long row = t / (n / 2);
    const int j = (int)(t - row * (n / 2));
    const int pos = j % half, grp = j / half;
    const long long i0 = row * n + (long long)grp * 2 * half + pos, i1 = i0 + half;
    double s, c;
    sincospi(sign * (double)pos / (double)half, &s, &c);
    const double2 u = x[i0], v = x[i1];
    const double2 w = make_double2(c * v.x - s * v.y, c * v.y + s * v.x);
    x[i0] = make_double2(u.x + w.x, u.y + w.y);
    x[i1] = make_double2(u.x - w.x, u.y - w.y);
  }
}
// acc += x * y (element-wise), or x *= scale
__global__ void k_fft_mac(double2* acc, const double2* x, const double2* y, long long total) {
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    const double2 p = cmul(x[t], y[t]);
    acc[t] = make_double2(acc[t].x + p.x, acc[t].y + p.y);
  }
}

int grid_for(long long work) { return (int)std::max(1LL, std::min((work + 255) / 256, 65535LL * 4)); }

}  // namespace
}  // namespace rpm

using namespace rpm;

extern "C" {

int rpm_he_eigh_workspace(int n, int batch, long long* bytes) {
  return guarded([&] {
    if (n < 2 || n > kHeMaxN || batch < 1 || !bytes) fail(RPM_E_INVALID, "eigh: need 2 <= n <= 1024, batch >= 1");
    const long long nn = (long long)n * n;
    // d, e, perm (as double), tau (2 doubles), status; house (complex) and z (real)
    *bytes = (long long)batch * ((3 * n + 2 * n + 1) * 8 + nn * 16 + nn * 8) + 7 * 256;  // + alignment of 7 parts
  });
}

int rpm_he_eigh(int n, int batch, void* a_dev, double* w_dev, void* v_dev, void* work_dev, cudaStream_t stream) {
  return guarded([&] {
    long long need = 0;
    if (rpm_he_eigh_workspace(n, batch, &need) != RPM_OK) fail(RPM_E_INVALID, "eigh: bad sizes");
    if (!a_dev || !w_dev || !v_dev || !work_dev) fail(RPM_E_INVALID, "eigh: null pointer");
    const long long nn = (long long)n * n;
    char* p = static_cast<char*>(work_dev);
    auto take = [&](long long bytes) {
      char* q = p;
      p += (bytes + 255) / 256 * 256;
      return q;
    };
    double* d = reinterpret_cast<double*>(take((long long)batch * n * 8));
    double* e = reinterpret_cast<double*>(take((long long)batch * n * 8));
    int* perm = reinterpret_cast<int*>(take((long long)batch * n * 8));
    double2* tau = reinterpret_cast<double2*>(take((long long)batch * n * 16));
    int* status = reinterpret_cast<int*>(take((long long)batch * 8));
    double2* house = reinterpret_cast<double2*>(take((long long)batch * nn * 16));
    double* z = reinterpret_cast<double*>(take((long long)batch * nn * 8));
    (void)need;
    k_he_tridiag<<<batch, kHeThreads, 0, stream>>>(static_cast<double2*>(a_dev), n, d, e, house, tau);
    k_he_tridiag_eig<<<batch, 256, 0, stream>>>(d, e, z, n, status);
    k_he_sort<<<batch, 256, 0, stream>>>(d, n, perm, w_dev);
    k_he_back<<<dim3((n + 31) / 32, batch), 256, 0, stream>>>(z, perm, house, tau, n, static_cast<double2*>(v_dev));
    check_launch("eigh");
    std::vector<int> st(batch);
    check_cuda(cudaMemcpyAsync(st.data(), status, sizeof(int) * batch, cudaMemcpyDeviceToHost, stream), "eigh status");
    check_cuda(cudaStreamSynchronize(stream), "eigh sync");
    for (int b = 0; b < batch; ++b)
      if (st[b]) fail(RPM_E_NUMERIC, "eigh: the tridiagonal QR did not converge");
  });
}

int rpm_zgemm_hn(int n, int batch, const void* a_dev, const void* b_dev, void* c_dev, cudaStream_t stream) {
  return guarded([&] {
    if (n < 1 || batch < 1 || !a_dev || !b_dev || !c_dev) fail(RPM_E_INVALID, "zgemm_hn: bad arguments");
    const int t = (n + 15) / 16;
    k_zgemm_hn<<<dim3(t, t, batch), 256, 0, stream>>>(static_cast<const double2*>(a_dev),
                                                      static_cast<const double2*>(b_dev), static_cast<double2*>(c_dev),
                                                      n);
    check_launch("zgemm_hn");
  });
}

int rpm_fft_pow2(int n, int batch, void* data_dev, void* scratch_dev, int inverse, cudaStream_t stream) {
  return guarded([&] {
    if (n < 2 || (n & (n - 1)) || batch < 1 || !data_dev || !scratch_dev)
      fail(RPM_E_INVALID, "fft: n must be a power of two >= 2");
    int logn = 0;
    while ((1 << logn) < n) ++logn;
    const long long total = (long long)n * batch;
    double2* x = static_cast<double2*>(data_dev);
    double2* s = static_cast<double2*>(scratch_dev);
    k_fft_bitrev<<<grid_for(total), 256, 0, stream>>>(x, s, n, logn, total);
    for (int half = 1; half < n; half *= 2)
      k_fft_pass<<<grid_for(total / 2), 256, 0, stream>>>(s, n, half, inverse ? 1.0 : -1.0, total / 2);
    check_cuda(cudaMemcpyAsync(x, s, sizeof(double2) * total, cudaMemcpyDeviceToDevice, stream), "fft copy");
    check_launch("fft");
  });
}

int rpm_spectrum_mac(long long count, void* acc_dev, const void* x_dev, const void* y_dev, cudaStream_t stream) {
  return guarded([&] {
    if (count < 1 || !acc_dev || !x_dev || !y_dev) fail(RPM_E_INVALID, "spectrum_mac: bad arguments");
    k_fft_mac<<<grid_for(count), 256, 0, stream>>>(static_cast<double2*>(acc_dev), static_cast<const double2*>(x_dev),
                                                   static_cast<const double2*>(y_dev), count);
    check_launch("spectrum_mac");
  });
}

}  // extern "C"
