// Device helpers shared by the plain and batched Krylov kernels.
#pragma once

#include <cfloat>

#include "common.cuh"

namespace rpm {

// ---------------------------------------------------------------------------
// Block reduction helpers
// ---------------------------------------------------------------------------
static __device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Reduce `count` double2 values held by every thread over the block; thread
// 0..count-1 of warp 0 ends up with the block totals in `out` (shared memory).
template <int COUNT>
static __device__ __forceinline__ void block_sum2(double2 (&v)[COUNT], double2* scratch /*[32][COUNT]*/, double2* out) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int c = 0; c < COUNT; ++c) {
    v[c].x = warp_sum(v[c].x);
    v[c].y = warp_sum(v[c].y);
  }
  if (lane == 0) {
#pragma unroll
    for (int c = 0; c < COUNT; ++c) scratch[warp * COUNT + c] = v[c];
  }
  __syncthreads();
  if (threadIdx.x < COUNT) {
    double2 s = make_double2(0.0, 0.0);
    for (int w = 0; w < nw; ++w) s = cadd(s, scratch[w * COUNT + threadIdx.x]);
    out[threadIdx.x] = s;
  }
  __syncthreads();
}

// Last-block completion.  Returns true in exactly one block (the last to
// arrive); that block sees every other block's partials.
static __device__ __forceinline__ bool last_block(unsigned* counter) {
  __shared__ bool is_last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned ticket = atomicAdd(counter, 1u);
    is_last = (ticket == gridDim.x - 1);
  }
  __syncthreads();
  if (is_last) __threadfence();
  return is_last;
}

// Sum partials[k * nblocks + b] over b in order, for k < count, into out[k].
static __device__ void finish_sums(const double2* partials, int nblocks, int count, double2* out) {
  for (int k = threadIdx.x; k < count; k += blockDim.x) {
    double2 s = make_double2(0.0, 0.0);
    const double2* p = partials + (size_t)k * nblocks;
    for (int b = 0; b < nblocks; ++b) s = cadd(s, __ldcg(p + b));
    out[k] = s;
  }
}

// ---------------------------------------------------------------------------
// Tridiagonal eigen-decomposition (implicit QR, Wilkinson shift)
// ---------------------------------------------------------------------------
// d[0..m), e[0..m-1): diagonal / off-diagonal (overwritten: d -> eigenvalues).
// z: m x m eigenvectors, row-major with leading dimension ldz.
// rot: scratch for m-1 rotations.  Must be called by all threads of a block.
// Returns 0 on convergence, 1 otherwise.
static __device__ int tridiag_qr(int m, double* d, double* e, double* z, int ldz, double2* rot) {
  __shared__ int s_p, s_q, s_state;
  for (int idx = threadIdx.x; idx < m * m; idx += blockDim.x) {
    const int i = idx / m, k = idx % m;
    z[i * ldz + k] = (i == k) ? 1.0 : 0.0;
  }
  if (threadIdx.x == 0) s_state = 0;
  __syncthreads();
  int sweeps = 0;
  while (true) {
    if (threadIdx.x == 0) {
      // deflate negligible couplings
      for (int i = 0; i + 1 < m; ++i) {
        if (fabs(e[i]) <= DBL_EPSILON * (fabs(d[i]) + fabs(d[i + 1])) || fabs(e[i]) < DBL_MIN) e[i] = 0.0;
      }
      int q = m - 1;
      while (q > 0 && e[q - 1] == 0.0) --q;
      if (q == 0) {
        s_state = 1;  // converged
      } else if (++sweeps > 40 * m) {
        s_state = 2;  // no convergence
      } else {
        int p = q - 1;
        while (p > 0 && e[p - 1] != 0.0) --p;
        // Wilkinson shift from the trailing 2x2 block of [p, q]
        const double delta = 0.5 * (d[q - 1] - d[q]);
        const double eq = e[q - 1];
        const double denom = delta + copysign(hypot(delta, eq), delta);
        const double mu = d[q] - eq * eq / denom;
        double x = d[p] - mu, y = e[p];
        for (int k = p; k < q; ++k) {
          double c = 1.0, s = 0.0;
          const double r = hypot(x, y);
          if (r > 0.0) {
            c = x / r;
            s = y / r;
          }
          if (k > p) e[k - 1] = r;
          const double a = d[k], b = e[k], cc = d[k + 1];
          d[k] = c * c * a + 2.0 * c * s * b + s * s * cc;
          d[k + 1] = s * s * a - 2.0 * c * s * b + c * c * cc;
          e[k] = c * s * (cc - a) + (c * c - s * s) * b;
          if (k + 1 < q) {
            x = e[k];
            y = s * e[k + 1];
            e[k + 1] = c * e[k + 1];
          }
          rot[k] = make_double2(c, s);
        }
        s_p = p;
        s_q = q;
      }
    }
    __syncthreads();
    if (s_state != 0) break;
    const int p = s_p, q = s_q;
    for (int i = threadIdx.x; i < m; i += blockDim.x) {
      double* row = z + i * ldz;
      double zk = row[p];
      for (int k = p; k < q; ++k) {
        const double2 cs = rot[k];
        const double zk1 = row[k + 1];
        row[k] = cs.x * zk + cs.y * zk1;
        zk = -cs.y * zk + cs.x * zk1;
      }
      row[q] = zk;
    }
    __syncthreads();
  }
  const int state = s_state;
  __syncthreads();
  return state == 1 ? 0 : 1;
}

// ---------------------------------------------------------------------------
// Tridiagonal eigen-decomposition by one warp
// ---------------------------------------------------------------------------
// Implicit symmetric tridiagonal QR with Wilkinson shifts (Golub & Van Loan,
// section 8.3) run by ONE warp: every lane tests its off-diagonal entries
// for deflation and the active block [p, q] comes from two ballots; lane 0
// computes the shift and chases the bulge; every lane applies the sweep's
// rotations to its rows of the eigenvector matrix.  d, e: diagonal and
// off-diagonal (d -> eigenvalues); m <= 64.  z: m x m eigenvector matrix
// stored by columns, z[k * ldz + i] = component i of eigenvector k, so that
// the lanes' row updates touch consecutive addresses.  FAST = true normalises
// the rotations with rsqrt and carries the entries the next rotation reads in
// registers; FAST = false keeps the block-wide solver's arithmetic exactly
// (hypot and two divisions, operands re-read from memory), so that the plain
// path's decisions stay those matched to the reference.  Returns 0 on
// convergence.
template <bool FAST>
static __device__ int tridiag_qr_warp_cols(int m, double* d, double* e, double* z, int ldz, double2* rot) {
  const int lane = threadIdx.x & 31;
  for (int idx = lane; idx < m * m; idx += 32) {
    const int k = idx / m, i = idx - k * m;
    z[k * ldz + i] = (i == k) ? 1.0 : 0.0;
  }
  __syncwarp();
  int sweeps = 0;
  while (true) {
    // deflation: e[i] negligible against its neighbours on the diagonal
    bool nz[2];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int i = lane + 32 * h;
      nz[h] = false;
      if (i + 1 < m) {
        const double ei = e[i];
        if (fabs(ei) <= DBL_EPSILON * (fabs(d[i]) + fabs(d[i + 1])) || fabs(ei) < DBL_MIN) e[i] = 0.0;
        else nz[h] = true;
      }
    }
    const unsigned long long nzm = (unsigned long long)__ballot_sync(0xffffffffu, nz[0]) |
                                   ((unsigned long long)__ballot_sync(0xffffffffu, nz[1]) << 32);
    __syncwarp();
    // q - 1: the last nonzero off-diagonal; p: the start of its unreduced block
    const int q = nzm ? 64 - __clzll(nzm) : 0;
    if (q == 0) return 0;
    if (++sweeps > 40 * m) return 1;
    const unsigned long long below = q >= 2 ? (~nzm) & ((1ull << (q - 1)) - 1ull) : 0ull;
    const int p = below ? 64 - __clzll(below) : 0;
    if (lane == 0 && !FAST) {
      const double delta = 0.5 * (d[q - 1] - d[q]);
      const double eq = e[q - 1];
      const double denom = delta + copysign(hypot(delta, eq), delta);
      const double mu = d[q] - eq * eq / denom;
      double x = d[p] - mu, y = e[p];
      for (int k = p; k < q; ++k) {
        double c = 1.0, sn = 0.0;
        const double r = hypot(x, y);
        if (r > 0.0) {
          c = x / r;
          sn = y / r;
        }
        if (k > p) e[k - 1] = r;
        const double a = d[k], bb = e[k], cc = d[k + 1];
        d[k] = c * c * a + 2.0 * c * sn * bb + sn * sn * cc;
        d[k + 1] = sn * sn * a - 2.0 * c * sn * bb + c * c * cc;
        e[k] = c * sn * (cc - a) + (c * c - sn * sn) * bb;
        if (k + 1 < q) {
          x = e[k];
          y = sn * e[k + 1];
          e[k + 1] = c * e[k + 1];
        }
        rot[k] = make_double2(c, sn);
      }
    }
    if (lane == 0 && FAST) {
      const double delta = 0.5 * (d[q - 1] - d[q]);
      const double eq = e[q - 1];
      const double denom = delta + copysign(hypot(delta, eq), delta);
      const double mu = d[q] - eq * eq / denom;
      double x = d[p] - mu, y = e[p];
      double a = d[p], bb = e[p];  // d[k] and e[k] as the previous rotation left them
      for (int k = p; k < q; ++k) {
        const double cc = d[k + 1];
        const double en = k + 1 < q ? e[k + 1] : 0.0;
        double c = 1.0, sn = 0.0, r = 0.0;
        const double rr = fma(x, x, y * y);
        if (rr > 0.0) {
          const double inv = rsqrt(rr);
          c = x * inv;
          sn = y * inv;
          r = rr * inv;
        }
        if (k > p) e[k - 1] = r;
        const double dk = c * c * a + 2.0 * c * sn * bb + sn * sn * cc;
        const double dk1 = sn * sn * a - 2.0 * c * sn * bb + c * c * cc;
        const double ek = c * sn * (cc - a) + (c * c - sn * sn) * bb;
        d[k] = dk;
        d[k + 1] = dk1;
        e[k] = ek;
        if (k + 1 < q) {
          x = ek;
          y = sn * en;
          bb = c * en;
          e[k + 1] = bb;
        }
        a = dk1;
        rot[k] = make_double2(c, sn);
      }
    }
    __syncwarp();
    for (int i = lane; i < m; i += 32) {
      double zk = z[p * ldz + i];
      for (int k = p; k < q; ++k) {
        const double2 cs = rot[k];
        const double zk1 = z[(k + 1) * ldz + i];
        z[k * ldz + i] = cs.x * zk + cs.y * zk1;
        zk = -cs.y * zk + cs.x * zk1;
      }
      z[q * ldz + i] = zk;
    }
    __syncwarp();
  }
}

// c = exp(-i T t) e1 from a spectra record, into shared `c` (m entries).
// Record layout with leading dimension LD: [0] size, [1] status, [2, 2+LD)
// eigenvalues, then LD x LD eigenvectors (row i = component i).
template <int LD = RPM_MAX_KRYLOV>
static __device__ void spectral_coefficients(const double* rec, double t, double2* ph, double2* c) {
  const int m = (int)rec[0];
  const double* lam = rec + 2;
  const double* z = rec + 2 + LD;
  for (int k = threadIdx.x; k < m; k += blockDim.x) {
    double s, co;
    sincos(lam[k] * t, &s, &co);
    const double w = z[k];  // first component of eigenvector k
    ph[k] = make_double2(co * w, -s * w);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < m; i += blockDim.x) {
    const double* zi = z + i * LD;
    double2 acc = make_double2(0.0, 0.0);
    for (int k = 0; k < m; ++k) {
      acc.x = fma(zi[k], ph[k].x, acc.x);
      acc.y = fma(zi[k], ph[k].y, acc.y);
    }
    c[i] = acc;
  }
  __syncthreads();
}

}  // namespace rpm
