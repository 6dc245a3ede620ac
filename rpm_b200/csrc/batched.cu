// Batched mixed-precision Krylov propagation (many trajectories per launch).
//
// One "trajectory" is one state vector of one system (field orientation /
// system size) propagated over the observation grid.  Precision follows the
// split the hot path needs:
//   * the Lanczos basis and every H psi are complex64 with FP32 accumulation;
//   * alpha/beta reductions, the state between Krylov steps (complex128),
//     its recombination psi = ||psi|| V c, the tridiagonal eigen-solve,
//     exp(-i T t) e1, the error control and the singlet Gram/populations are
//     FP64.
// Each Krylov step is a fixed kernel sequence over all trajectories:
//   start -> m x [H psi (pass L, pass R + alpha), update + beta]
//         -> control -> rebuild -> gram -> observe
// captured once as a CUDA graph and replayed until every trajectory reached
// the last observation time.  Per-trajectory controller state lives on the
// device; the host only polls a done-counter.
//
// Step control (per trajectory): with the Krylov basis of dimension m fixed,
// the embedded error err(dt) = safety * ||psi|| * ||c_m(dt) - [c_{m-off}(dt); 0]||
// (the reference's estimate, rpm_statevector_engine.py:690-715) is evaluated
// for trial steps, and the largest dt <= min(max_step, T - t) with
// err(dt) <= budget * dt / T is taken.  Because the basis does not depend on
// dt, no step is ever rejected.
#include <algorithm>
#include <atomic>
#include <cfloat>
#include <cmath>
#include <memory>

#include "common.cuh"
#include "hpsi.cuh"
#include "krylov.cuh"

namespace rpm {

constexpr int kBMaxK = 64;    // Krylov dimension cap of the batched path
constexpr int kMaxPts = 256;  // observation points per Krylov step
constexpr int kEwThreads = 256;
constexpr int kEwPer = 8;                         // elements per thread
constexpr int kEwChunk = kEwThreads * kEwPer;     // elements per block
constexpr int kRecDoubles = 2 + kBMaxK + kBMaxK * kBMaxK;  // one spectra record (LD = kBMaxK)
constexpr size_t kArnCtlSmem = sizeof(double2) * 3 * kBMaxK * kBMaxK;  // Arnoldi controller scratch

struct TrajState {
  double t_now, dt, norm, new_norm2, acc_err, step_err, max_norm_err;
  double min_step, max_step, hint, scale;
  double wnorm2;  // Arnoldi: |H v_j|^2 before the Gram-Schmidt projection
  double alpha[kBMaxK];
  double beta[kBMaxK];
  long long n, matvecs;
  int cursor, npts, done, stop, skip, msize, steps, sys;
  int status;
  int cgs_done;  // Arnoldi: the first projection kept the norm (no second pass)
  int mcap;      // this trajectory's Krylov dimension (<= the batch's m)
  int pad_;
};
static_assert(sizeof(TrajState) % 8 == 0, "TrajState must be a whole number of doubles");
static_assert(sizeof(TrajState) % 4 == 0, "TrajState must be a whole number of ints");
constexpr int kStateDoubles = sizeof(TrajState) / 8;
constexpr int kStateInts = sizeof(TrajState) / 4;

struct BatchDev {
  TrajState* st;
  int ntraj, m, offset;
  double safety, budget, max_step, min_step, t_end, breakdown_rel;
  const double* times;
  int ntimes;
  long long ld;
  float2* V;        // [traj][m + 1][ld]
  double2* psi;     // [traj][ld]
  double2* coef;    // [traj][kMaxPts + 1][kBMaxK]; row kMaxPts = endpoint
  double* perr;     // [traj][kMaxPts]
  double* part;     // [traj][nblk][2]
  unsigned* count;  // [traj] completion counters (elementwise reductions)
  double2* gpart;   // [traj][gblk][kBMaxK * kBMaxK]
  double* values;   // [traj][ntimes]
  double* errs;     // [traj][ntimes]
  int nblk, gblk;
  int* active;      // trajectories not yet done
  // persistent Lanczos kernel: per-trajectory progress / tile counters and
  // L-tile partial sums, one dequeue counter per launch, sticky wait status
  int* prog;
  unsigned* pcnt;
  double* ppart;
  int ppart_stride;
  unsigned* work;
  int nwork;
  int* kstatus;
  // Arnoldi (non-Hermitian systems: unequal recombination rates)
  int arnoldi;
  double grid_h;    // uniform observation spacing
  double2* hess;    // [traj][kBMaxK + 1][kBMaxK] Hessenberg matrix H(i, j)
  double2* hcur;    // [traj][kBMaxK] projections of the current Gram-Schmidt pass
  double2* adots;   // [traj][nblk][kBMaxK] block partials of the projections
  double2* expm;    // [traj][2][kBMaxK * kBMaxK] exp(-i H h) of T_M and T_(M-offset)
};

__device__ __forceinline__ bool traj_last_block(unsigned* counter) {
  __shared__ bool is_last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) is_last = atomicAdd(counter, 1u) == gridDim.x - 1;
  __syncthreads();
  if (is_last) __threadfence();
  return is_last;
}

__device__ __forceinline__ double block_sum(double v, double* red) {
  v = warp_sum(v);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  double s = 0.0;
  for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w];
  return s;
}

// Sum two partial slots over the blocks of trajectory b, in block order.
__device__ __forceinline__ double2 sum_parts(const BatchDev& B, int b) {
  double2 s = make_double2(0.0, 0.0);
  const double* p = B.part + (size_t)b * B.nblk * 2;
  for (int k = 0; k < (int)gridDim.x; ++k) {
    s.x += __ldcg(p + 2 * k);
    s.y += __ldcg(p + 2 * k + 1);
  }
  return s;
}

// ---------------------------------------------------------------------------
// Set-up: state fields, ||psi0|| and P_S(psi0)
// ---------------------------------------------------------------------------
__global__ void k_b_setup(BatchDev B, const int* sys_of, const long long* n_of, const int* cap_of,
                          double initial_step) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= B.ntraj) return;
  TrajState& s = B.st[b];
  int* raw = reinterpret_cast<int*>(&s);
  for (int k = 0; k < kStateInts; ++k) raw[k] = 0;
  s.sys = sys_of[b];
  s.n = n_of[b];
  s.hint = initial_step;
  s.min_step = DBL_MAX;
  s.mcap = max(2, min(B.m, cap_of[b] > 0 ? cap_of[b] : B.m));
  s.msize = s.mcap;
  s.scale = 1.0;
  B.count[b] = 0;
}

__global__ void __launch_bounds__(kEwThreads) k_b_init(BatchDev B) {
  __shared__ double red[32];
  const int b = blockIdx.y;
  TrajState& s = B.st[b];
  const long long n = s.n, q = n / 4;
  const double2* x = B.psi + (size_t)b * B.ld;
  double nn = 0.0, ps = 0.0;
  for (long long i = (long long)blockIdx.x * kEwChunk + threadIdx.x; i < n && i < (long long)(blockIdx.x + 1) * kEwChunk;
       i += kEwThreads) {
    const double2 v = x[i];
    nn = fma(v.x, v.x, fma(v.y, v.y, nn));
    if (i >= q && i < 2 * q) {
      const double2 w = x[i + q];
      const double re = v.x - w.x, im = v.y - w.y;
      ps = fma(re, re, fma(im, im, ps));
    }
  }
  nn = block_sum(nn, red);
  ps = block_sum(ps, red);
  if (threadIdx.x == 0) {
    B.part[((size_t)b * B.nblk + blockIdx.x) * 2] = nn;
    B.part[((size_t)b * B.nblk + blockIdx.x) * 2 + 1] = 0.5 * ps;
  }
  if (traj_last_block(B.count + b) && threadIdx.x == 0) {
    const double2 tot = sum_parts(B, b);
    s.norm = sqrt(tot.x);
    s.max_norm_err = fabs(s.norm - 1.0);
    if (B.times[0] == 0.0) {
      B.values[(size_t)b * B.ntimes] = tot.y;
      B.errs[(size_t)b * B.ntimes] = 0.0;
      s.cursor = 1;
    }
    if (!(s.norm > 0.0) || !isfinite(s.norm)) {
      s.status = 1;
      s.done = 1;
    }
    if (s.cursor >= B.ntimes) s.done = 1;
    s.skip = s.done;
    if (s.done) atomicSub(B.active, 1);
    B.count[b] = 0;
  }
}

// ---------------------------------------------------------------------------
// Krylov step kernels
// ---------------------------------------------------------------------------
// v0 = psi / ||psi|| (complex64)
__global__ void __launch_bounds__(kEwThreads) k_b_start(BatchDev B) {
  const int b = blockIdx.y;
  TrajState& s = B.st[b];
  if (blockIdx.x == 0) {  // persistent-kernel counters start from zero every Krylov step
    if (threadIdx.x == 0) {
      B.prog[b] = 0;
      B.pcnt[b] = 0;
    }
    if (b == 0)
      for (int k = threadIdx.x; k < B.nwork; k += blockDim.x) B.work[k] = 0u;
  }
  if (s.done) return;
  const double inv = 1.0 / s.norm;
  const double2* x = B.psi + (size_t)b * B.ld;
  float2* v0 = B.V + (size_t)b * (B.m + 1) * B.ld;
  const long long end = min(s.n, (long long)(blockIdx.x + 1) * kEwChunk);
  for (long long i = (long long)blockIdx.x * kEwChunk + threadIdx.x; i < end; i += kEwThreads) {
    const double2 v = x[i];
    v0[i] = make_float2((float)(v.x * inv), (float)(v.y * inv));
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    s.stop = 0;
    s.skip = 0;
    s.msize = s.mcap;
    s.scale = 1.0;
  }
}

// v_j <- scale * V_j (in place);  w = V_{j+1} - alpha_j v_j - beta_{j-1} v_{j-1};
// beta_j = ||w||, scale = 1 / beta_j; breakdown when beta_j is at round-off level.
__global__ void __launch_bounds__(kEwThreads) k_b_update(BatchDev B, int j, int b0) {
  __shared__ double red[32];
  const int b = blockIdx.y + b0;
  TrajState& s = B.st[b];
  if (s.skip) return;
  const float sc = (float)s.scale;
  const float a = (float)s.alpha[j];
  const float bp = j > 0 ? (float)s.beta[j - 1] : 0.0f;
  float2* base = B.V + (size_t)b * (B.m + 1) * B.ld;
  float2* vj = base + (size_t)j * B.ld;
  float2* wn = base + (size_t)(j + 1) * B.ld;
  const float2* vp = base + (size_t)(j > 0 ? j - 1 : 0) * B.ld;
  const bool last = (j == B.m - 1);
  double nn = 0.0;
  const long long end = min(s.n, (long long)(blockIdx.x + 1) * kEwChunk);
  for (long long i = (long long)blockIdx.x * kEwChunk + threadIdx.x; i < end; i += kEwThreads) {
    float2 v = vj[i];
    v.x *= sc;
    v.y *= sc;
    vj[i] = v;
    if (!last) {
      float2 w = wn[i];
      w.x = fmaf(-a, v.x, w.x);
      w.y = fmaf(-a, v.y, w.y);
      if (j > 0) {
        const float2 u = vp[i];
        w.x = fmaf(-bp, u.x, w.x);
        w.y = fmaf(-bp, u.y, w.y);
      }
      wn[i] = w;
      nn = fma((double)w.x, (double)w.x, fma((double)w.y, (double)w.y, nn));
    }
  }
  if (last) return;
  nn = block_sum(nn, red);
  if (threadIdx.x == 0) B.part[((size_t)b * B.nblk + blockIdx.x) * 2] = nn;
  if (traj_last_block(B.count + b) && threadIdx.x == 0) {
    double tot = 0.0;
    const double* p = B.part + (size_t)b * B.nblk * 2;
    for (int k = 0; k < (int)gridDim.x; ++k) tot += __ldcg(p + 2 * k);
    const double bj = sqrt(tot);
    s.beta[j] = bj;
    s.scale = bj > 0.0 ? 1.0 / bj : 0.0;
    const double ref = fabs(s.alpha[j]) + (j > 0 ? s.beta[j - 1] : 0.0);
    if (j + 1 >= s.mcap) {  // this trajectory's Krylov cap: its basis ends here
      s.skip = 1;
      s.msize = s.mcap;
    } else if (!(bj > B.breakdown_rel * ref)) {
      s.stop = 1;
      s.skip = 1;
      s.msize = j + 1;
    }
    B.count[b] = 0;
  }
}

// ---------------------------------------------------------------------------
// Per-trajectory controller (one CTA of four warps per trajectory)
// ---------------------------------------------------------------------------
// One warp: c = exp(-i T_hi t) e1 (into `c` when non-null) and the embedded
// error safety * norm * |c_hi(t) - [c_lo(t); 0]| (0 when `exact`), the
// reference's estimate (rpm_statevector_engine.py:690-715).  ph: 2 * kBMaxK
// warp-private scratch.  Records: [0] size, [1] status, [2, 2 + kBMaxK)
// eigenvalues, then the eigenvectors by columns (tridiag_qr_warp_cols, ld kBMaxK).
__device__ double warp_step_error(const double* rec_hi, const double* rec_lo, bool exact, double t, double safety,
                                  double norm, double2* ph, double2* c) {
  const int lane = threadIdx.x & 31;
  const int mh = (int)rec_hi[0], ml = exact ? 0 : (int)rec_lo[0];
  const double* lh = rec_hi + 2;
  const double* zh = rec_hi + 2 + kBMaxK;
  const double* ll = rec_lo + 2;
  const double* zl = rec_lo + 2 + kBMaxK;
  for (int k = lane; k < mh + ml; k += 32) {
    const bool hi = k < mh;
    const int kk = hi ? k : k - mh;
    double sv, cv;
    sincos((hi ? lh : ll)[kk] * t, &sv, &cv);
    const double w = (hi ? zh : zl)[kk * kBMaxK];  // first component of eigenvector kk
    ph[k] = make_double2(cv * w, -sv * w);
  }
  __syncwarp();
  double acc = 0.0;
  for (int i = lane; i < mh; i += 32) {
    double2 ch = make_double2(0.0, 0.0), cl = make_double2(0.0, 0.0);
    for (int k = 0; k < mh; ++k) {
      const double zz = zh[k * kBMaxK + i];
      ch.x = fma(zz, ph[k].x, ch.x);
      ch.y = fma(zz, ph[k].y, ch.y);
    }
    if (c) c[i] = ch;
    if (i < ml) {
      for (int k = 0; k < ml; ++k) {
        const double zz = zl[k * kBMaxK + i];
        cl.x = fma(zz, ph[mh + k].x, cl.x);
        cl.y = fma(zz, ph[mh + k].y, cl.y);
      }
    }
    const double dx = ch.x - cl.x, dy = ch.y - cl.y;
    acc = fma(dx, dx, fma(dy, dy, acc));
  }
  acc = warp_sum(acc);
  __syncwarp();
  return exact ? 0.0 : safety * norm * sqrt(acc);
}

// Per trajectory: spectra of T_M and T_{M-offset} (one warp each), the
// largest step dt <= dt_max with err(dt) <= budget * dt / T (bracket, then
// 5-way multisection in log dt with four trial steps per round, one per
// warp, to a relative width of 5e-4), and the coefficient rows of the
// step's observation points (one point per warp at a time).
// Dynamic shared memory: two spectra records (hi, lo) of the krylov.cuh layout.
__global__ void __launch_bounds__(128) k_b_control(BatchDev B) {
  extern __shared__ double sm[];
  __shared__ double2 ph[4][2 * kBMaxK];
  __shared__ double2 rot[2][kBMaxK];
  __shared__ double dd[2][kBMaxK], ee[2][kBMaxK];
  __shared__ double cand[4];
  __shared__ int okf[4];
  __shared__ double s_dt, s_lo, s_hi;
  __shared__ int s_state, s_np;
  const int b = blockIdx.x;
  TrajState& s = B.st[b];
  if (s.done) return;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double* rec_hi = sm;
  double* rec_lo = sm + kRecDoubles;
  const int M = s.msize;
  const bool exact = s.stop != 0;
  const int ML = max(1, M - B.offset);
  if (warp < (exact ? 1 : 2)) {
    const int dim = warp == 0 ? M : ML;
    double* rec = warp == 0 ? rec_hi : rec_lo;
    for (int i = lane; i < dim; i += 32) {
      dd[warp][i] = s.alpha[i];
      ee[warp][i] = (i + 1 < dim) ? s.beta[i] : 0.0;
    }
    __syncwarp();
    const int bad = tridiag_qr_warp_cols<true>(dim, dd[warp], ee[warp], rec + 2 + kBMaxK, kBMaxK, rot[warp]);
    for (int i = lane; i < dim; i += 32) rec[2 + i] = dd[warp][i];
    if (lane == 0) {
      rec[0] = dim;
      rec[1] = bad;
      if (bad) s.status = 2;
    }
  }
  __syncthreads();
  const double t_now = s.t_now;
  const double remaining = B.t_end - t_now;
  double dt_max = fmin(B.max_step, remaining);
  // keep the observation points of one step within the coefficient buffer
  if (s.cursor + kMaxPts - 1 < B.ntimes) dt_max = fmin(dt_max, B.times[s.cursor + kMaxPts - 1] - t_now);
  const double norm = s.norm;
  if (threadIdx.x == 0) {
    const double g = fmin(s.hint, 0.5 * dt_max);
    cand[0] = dt_max;
    cand[1] = g;
    cand[2] = 0.25 * g;
    cand[3] = 0.0625 * g;
    s_state = 0;  // 0: first round, 1: going down, 2: multisection, 3: done, 4: underflow
    s_lo = 0.0;
    s_hi = dt_max;
  }
  __syncthreads();
  for (int round = 0; round < 64; ++round) {
    {
      const double err = warp_step_error(rec_hi, rec_lo, exact, cand[warp], B.safety, norm, ph[warp], nullptr);
      if (lane == 0) okf[warp] = err <= B.budget * cand[warp] / B.t_end;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      int st = s_state;
      if (st == 0 && okf[0]) {
        s_dt = dt_max;
        st = 3;
      } else if (st == 0 || st == 1) {
        int k0 = st == 0 ? 1 : 0, found = -1;
        for (int k = k0; k < 4; ++k)
          if (okf[k]) {
            found = k;
            break;
          }
        if (found >= 0) {
          s_lo = cand[found];
          s_hi = found == k0 ? s_hi : cand[found - 1];
          if (found == k0 && st == 0) s_hi = dt_max;
          st = 2;
        } else {
          s_hi = cand[3];
          const double base = cand[3];
          if (base * 0.25 < B.min_step) {
            st = 4;
          } else {
            for (int k = 0; k < 4; ++k) cand[k] = base * pow(0.25, k + 1);
            st = 1;
          }
        }
      } else if (st == 2) {
        for (int k = 0; k < 4; ++k) {
          if (okf[k]) s_lo = cand[k];
          else {
            s_hi = cand[k];
            break;
          }
        }
      }
      if (st == 2) {
        if (s_lo < B.min_step) {
          st = 4;
        } else if (s_hi <= s_lo * 1.0005) {
          s_dt = s_lo;
          st = 3;
        } else {
          const double l0 = log(s_lo), w = log(s_hi) - l0;
          for (int k = 0; k < 4; ++k) cand[k] = exp(l0 + w * (k + 1) / 5.0);
        }
      }
      s_state = st;
    }
    __syncthreads();
    if (s_state >= 3) break;
  }
  if (s_state != 3) {
    if (threadIdx.x == 0) {
      s.status = 3;  // step underflow (or no bracket within the round limit)
      s.done = 1;
      s.skip = 1;
      atomicSub(B.active, 1);
    }
    return;
  }
  double dt = s_dt;
  if (remaining - dt < 1e-12) dt = remaining;
  double2* rows = B.coef + (size_t)b * (kMaxPts + 1) * kBMaxK;
  // observation points inside (t_now, t_now + dt]
  if (threadIdx.x == 0) {
    int np = 0;
    const double t_end_step = t_now + dt;
    while (s.cursor + np < B.ntimes && np < kMaxPts && B.times[s.cursor + np] <= t_end_step + 1e-13) ++np;
    s_np = np;
  }
  __syncthreads();
  const int np = s_np;
  // point p < np: row p; p == np: the endpoint (row kMaxPts)
  for (int p = warp; p <= np; p += 4) {
    const bool endpoint = p == np;
    const double tau = endpoint ? dt : B.times[s.cursor + p] - t_now;
    double2* row = rows + (size_t)(endpoint ? kMaxPts : p) * kBMaxK;
    const double err = warp_step_error(rec_hi, rec_lo, exact, tau, B.safety, norm, ph[warp], row);
    for (int i = M + lane; i < kBMaxK; i += 32) row[i] = make_double2(0.0, 0.0);
    if (lane == 0) {
      if (endpoint) {
        s.dt = dt;
        s.step_err = err;
        s.npts = np;
      } else {
        B.perr[(size_t)b * kMaxPts + p] = err;
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Arnoldi (non-Hermitian H: unequal recombination rates)
// ---------------------------------------------------------------------------
// Classical Gram-Schmidt of w = V_(j+1) (H v_j from the passes) against
// v_0..v_j: projections in FP64 from FP32 products, accumulated into column j
// of the Hessenberg matrix.  A second pass runs only when the first lost more
// than 1 - 1/sqrt(2) of the norm (the Kahan-Parlett / DGKS criterion, "twice
// is enough"); the last pass's norm gives H(j+1, j) and the next scale.
__global__ void __launch_bounds__(kEwThreads) k_b_arn_dots(BatchDev B, int j, int pass) {
  __shared__ double2 red[kEwThreads / 32][kBMaxK];
  __shared__ double rn[kEwThreads / 32];
  const int b = blockIdx.y;
  TrajState& s = B.st[b];
  if (s.skip || (pass == 2 && s.cgs_done)) return;
  const float2* base = B.V + (size_t)b * (B.m + 1) * B.ld;
  const float2* w = base + (size_t)(j + 1) * B.ld;
  const long long i0 = (long long)blockIdx.x * kEwChunk + threadIdx.x;
  float2 wv[kEwPer];
#pragma unroll
  for (int k = 0; k < kEwPer; ++k) {
    const long long e = i0 + (long long)k * kEwThreads;
    wv[k] = e < s.n ? w[e] : make_float2(0.f, 0.f);
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (pass == 1) {  // |w|^2 before the projection (second-pass criterion)
    double nn = 0.0;
#pragma unroll
    for (int k = 0; k < kEwPer; ++k) nn = fma((double)wv[k].x, (double)wv[k].x, fma((double)wv[k].y, (double)wv[k].y, nn));
    nn = warp_sum(nn);
    if (lane == 0) rn[warp] = nn;
  }
  for (int i = 0; i <= j; ++i) {
    const float2* v = base + (size_t)i * B.ld;
    double2 acc = make_double2(0.0, 0.0);
#pragma unroll
    for (int k = 0; k < kEwPer; ++k) {
      const long long e = i0 + (long long)k * kEwThreads;
      if (e < s.n) {
        const float2 q = v[e];  // conj(q) * w
        acc.x += (double)q.x * wv[k].x + (double)q.y * wv[k].y;
        acc.y += (double)q.x * wv[k].y - (double)q.y * wv[k].x;
      }
    }
    acc.x = warp_sum(acc.x);
    acc.y = warp_sum(acc.y);
    if (lane == 0) red[warp][i] = acc;
  }
  __syncthreads();
  double2* part = B.adots + ((size_t)b * B.nblk + blockIdx.x) * kBMaxK;
  for (int i = threadIdx.x; i <= j; i += blockDim.x) {
    double2 t = make_double2(0.0, 0.0);
    for (int w2 = 0; w2 < kEwThreads / 32; ++w2) t = cadd(t, red[w2][i]);
    part[i] = t;
  }
  if (pass == 1 && threadIdx.x == 0) {
    double t = 0.0;
    for (int w2 = 0; w2 < kEwThreads / 32; ++w2) t += rn[w2];
    B.part[((size_t)b * B.nblk + blockIdx.x) * 2 + 1] = t;
  }
  if (traj_last_block(B.count + b)) {
    if (pass == 1 && threadIdx.x == 0) {
      double t = 0.0;
      for (int k = 0; k < (int)gridDim.x; ++k) t += __ldcg(B.part + ((size_t)b * B.nblk + k) * 2 + 1);
      s.wnorm2 = t;
    }
    for (int i = threadIdx.x; i <= j; i += blockDim.x) {
      double2 t = make_double2(0.0, 0.0);
      for (int k = 0; k < (int)gridDim.x; ++k) t = cadd(t, __ldcg(B.adots + ((size_t)b * B.nblk + k) * kBMaxK + i));
      B.hcur[(size_t)b * kBMaxK + i] = t;
      double2& h = B.hess[((size_t)b * (kBMaxK + 1) + i) * kBMaxK + j];
      h = pass == 1 ? t : cadd(h, t);
    }
    if (threadIdx.x == 0) B.count[b] = 0;
  }
}

// v_j <- scale * V_j in place for trajectories b0 + blockIdx.y (Arnoldi on
// the general cube kernels; the shape-specialised passes do this while staging).
__global__ void __launch_bounds__(kEwThreads) k_b_arn_scale(BatchDev B, int j, int b0) {
  const int b = blockIdx.y + b0;
  TrajState& s = B.st[b];
  if (s.skip) return;
  const float sc = (float)s.scale;
  float2* v = B.V + (size_t)b * (B.m + 1) * B.ld + (size_t)j * B.ld;
  const long long end = min(s.n, (long long)(blockIdx.x + 1) * kEwChunk);
  for (long long i = (long long)blockIdx.x * kEwChunk + threadIdx.x; i < end; i += kEwThreads) {
    float2 x = v[i];
    x.x *= sc;
    x.y *= sc;
    v[i] = x;
  }
}

__global__ void __launch_bounds__(kEwThreads) k_b_arn_axpy(BatchDev B, int j, int pass) {
  __shared__ float2 hc[kBMaxK];
  __shared__ double red[32];
  const int b = blockIdx.y;
  TrajState& s = B.st[b];
  if (s.skip || (pass == 2 && s.cgs_done)) return;
  for (int i = threadIdx.x; i <= j; i += blockDim.x) {
    const double2 t = B.hcur[(size_t)b * kBMaxK + i];
    hc[i] = make_float2((float)t.x, (float)t.y);
  }
  __syncthreads();
  float2* base = B.V + (size_t)b * (B.m + 1) * B.ld;
  float2* w = base + (size_t)(j + 1) * B.ld;
  double nn = 0.0;
  const long long end = min(s.n, (long long)(blockIdx.x + 1) * kEwChunk);
  for (long long e = (long long)blockIdx.x * kEwChunk + threadIdx.x; e < end; e += kEwThreads) {
    float2 x = w[e];
    for (int i = 0; i <= j; ++i) x = cfma(make_float2(-hc[i].x, -hc[i].y), base[(size_t)i * B.ld + e], x);
    w[e] = x;
    nn = fma((double)x.x, (double)x.x, fma((double)x.y, (double)x.y, nn));
  }
  nn = block_sum(nn, red);
  if (threadIdx.x == 0) B.part[((size_t)b * B.nblk + blockIdx.x) * 2] = nn;
  if (traj_last_block(B.count + b) && threadIdx.x == 0) {
    double tot = 0.0;
    for (int k = 0; k < (int)gridDim.x; ++k) tot += __ldcg(B.part + ((size_t)b * B.nblk + k) * 2);
    if (pass == 1) {
      // "twice is enough" (Kahan-Parlett / DGKS): a projection that keeps more
      // than 1/sqrt(2) of the norm needs no second Gram-Schmidt pass
      s.cgs_done = tot > 0.5 * s.wnorm2 ? 1 : 0;
      if (!s.cgs_done) {
        B.count[b] = 0;
        return;
      }
    }
    const double beta = sqrt(tot);
    B.hess[((size_t)b * (kBMaxK + 1) + j + 1) * kBMaxK + j] = make_double2(beta, 0.0);
    s.scale = beta > 0.0 ? 1.0 / beta : 0.0;
    if (j + 1 >= s.mcap && j + 1 < B.m) {  // this trajectory's Krylov cap: its basis ends here
      s.skip = 1;
      s.msize = s.mcap;
    } else if (j + 1 < B.m) {
      const double2 hd = B.hess[((size_t)b * (kBMaxK + 1) + j) * kBMaxK + j];
      double ref = hypot(hd.x, hd.y);
      if (j > 0) ref += B.hess[((size_t)b * (kBMaxK + 1) + j) * kBMaxK + j - 1].x;
      if (!(beta > B.breakdown_rel * ref)) {
        s.stop = 1;
        s.skip = 1;
        s.msize = j + 1;
      }
    }
    B.count[b] = 0;
  }
}

// ---------------------------------------------------------------------------
// Periodic reorthogonalisation of the Lanczos recurrence (reorth_policy 1)
// ---------------------------------------------------------------------------
// After iteration j the next vector is r = w'_(j+1) - alpha_j v_j, with w' held
// in V_(j+1).  One classical Gram-Schmidt pass against v_0 .. v_j:
// k_b_reo_dots forms d_i = <v_i, r> (FP64 sums of FP32 products, per-block
// partials summed in block order by the last block), k_b_reo_axpy stores
// w' - sum_i d_i v_i (so that r becomes r - sum_i d_i v_i) and, after the
// second pass, sets beta_j = |r| and the next scale (the reference runs two
// such passes every iteration, rpm_statevector_engine.py:675-676).
__global__ void __launch_bounds__(kEwThreads) k_b_reo_dots(BatchDev B, int j) {
  __shared__ double2 red[kEwThreads / 32][kBMaxK];
  const int b = blockIdx.y;
  TrajState& s = B.st[b];
  if (s.skip) return;
  const float2* base = B.V + (size_t)b * (B.m + 1) * B.ld;
  const float2* w = base + (size_t)(j + 1) * B.ld;
  const float2* vj = base + (size_t)j * B.ld;
  const float al = (float)s.alpha[j];
  const long long i0 = (long long)blockIdx.x * kEwChunk + threadIdx.x;
  float2 rv[kEwPer];
#pragma unroll
  for (int k = 0; k < kEwPer; ++k) {
    const long long e = i0 + (long long)k * kEwThreads;
    rv[k] = make_float2(0.f, 0.f);
    if (e < s.n) {
      const float2 x = w[e], v = vj[e];
      rv[k] = make_float2(fmaf(-al, v.x, x.x), fmaf(-al, v.y, x.y));
    }
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int i = 0; i <= j; ++i) {
    const float2* v = base + (size_t)i * B.ld;
    double2 acc = make_double2(0.0, 0.0);
#pragma unroll
    for (int k = 0; k < kEwPer; ++k) {
      const long long e = i0 + (long long)k * kEwThreads;
      if (e < s.n) {
        const float2 q = v[e];  // conj(q) * r
        acc.x += (double)q.x * rv[k].x + (double)q.y * rv[k].y;
        acc.y += (double)q.x * rv[k].y - (double)q.y * rv[k].x;
      }
    }
    acc.x = warp_sum(acc.x);
    acc.y = warp_sum(acc.y);
    if (lane == 0) red[warp][i] = acc;
  }
  __syncthreads();
  double2* part = B.adots + ((size_t)b * B.nblk + blockIdx.x) * kBMaxK;
  for (int i = threadIdx.x; i <= j; i += blockDim.x) {
    double2 t = make_double2(0.0, 0.0);
    for (int w2 = 0; w2 < kEwThreads / 32; ++w2) t = cadd(t, red[w2][i]);
    part[i] = t;
  }
  if (traj_last_block(B.count + b)) {
    for (int i = threadIdx.x; i <= j; i += blockDim.x) {
      double2 t = make_double2(0.0, 0.0);
      for (int k = 0; k < (int)gridDim.x; ++k) t = cadd(t, __ldcg(B.adots + ((size_t)b * B.nblk + k) * kBMaxK + i));
      B.hcur[(size_t)b * kBMaxK + i] = t;
    }
    if (threadIdx.x == 0) B.count[b] = 0;
  }
}

__global__ void __launch_bounds__(kEwThreads) k_b_reo_axpy(BatchDev B, int j, int last_pass) {
  __shared__ float2 hc[kBMaxK];
  __shared__ double red[32];
  const int b = blockIdx.y;
  TrajState& s = B.st[b];
  if (s.skip) return;
  for (int i = threadIdx.x; i <= j; i += blockDim.x) {
    const double2 t = B.hcur[(size_t)b * kBMaxK + i];
    hc[i] = make_float2((float)t.x, (float)t.y);
  }
  __syncthreads();
  float2* base = B.V + (size_t)b * (B.m + 1) * B.ld;
  float2* w = base + (size_t)(j + 1) * B.ld;
  const float2* vj = base + (size_t)j * B.ld;
  const float al = (float)s.alpha[j];
  double nn = 0.0;
  const long long end = min(s.n, (long long)(blockIdx.x + 1) * kEwChunk);
  for (long long e = (long long)blockIdx.x * kEwChunk + threadIdx.x; e < end; e += kEwThreads) {
    float2 x = w[e];
    for (int i = 0; i <= j; ++i) x = cfma(make_float2(-hc[i].x, -hc[i].y), base[(size_t)i * B.ld + e], x);
    w[e] = x;
    const float2 v = vj[e];
    const float rx = fmaf(-al, v.x, x.x), ry = fmaf(-al, v.y, x.y);
    nn = fma((double)rx, (double)rx, fma((double)ry, (double)ry, nn));
  }
  if (!last_pass) return;
  nn = block_sum(nn, red);
  if (threadIdx.x == 0) B.part[((size_t)b * B.nblk + blockIdx.x) * 2] = nn;
  if (traj_last_block(B.count + b) && threadIdx.x == 0) {
    double tot = 0.0;
    for (int k = 0; k < (int)gridDim.x; ++k) tot += __ldcg(B.part + ((size_t)b * B.nblk + k) * 2);
    const double beta = sqrt(tot);
    s.beta[j] = beta;
    s.scale = beta > 0.0 ? 1.0 / beta : 0.0;
    const double ref = fabs(s.alpha[j]) + (j > 0 ? s.beta[j - 1] : 0.0);
    if (j + 1 >= s.mcap) {  // this trajectory's Krylov cap: its basis ends here
      s.skip = 1;
      s.msize = s.mcap;
    } else if (!(beta > B.breakdown_rel * ref)) {
      s.stop = 1;
      s.skip = 1;
      s.msize = j + 1;
    }
    B.count[b] = 0;
  }
}

// Matrix product C = A X for n x n complex matrices in shared memory (row-major).
__device__ void cmatmul(int n, const double2* A, const double2* X, double2* C) {
  for (int idx = threadIdx.x; idx < n * n; idx += blockDim.x) {
    const int r = idx / n, c = idx - r * n;
    double2 acc = make_double2(0.0, 0.0);
    for (int k = 0; k < n; ++k) acc = cfma(A[r * n + k], X[k * n + c], acc);
    C[idx] = acc;
  }
  __syncthreads();
}

// E = exp(-i H h) for the leading n x n block of the Hessenberg matrix:
// scaling and squaring with an 18-term Taylor polynomial (norm of the scaled
// matrix at most 1/2: truncation below 1e-22).  P, Q, R: n x n scratch.
__device__ void hessenberg_expm(const double2* hess, int n, double h, double2* P, double2* Q, double2* R,
                                double2* out) {
  __shared__ double s_norm;
  for (int idx = threadIdx.x; idx < n * n; idx += blockDim.x) {
    const int r = idx / n, c = idx - r * n;
    const double2 v = hess[(size_t)r * kBMaxK + c];
    P[idx] = make_double2(v.y * h, -v.x * h);  // -i h H
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double best = 0.0;
    for (int c = 0; c < n; ++c) {
      double col = 0.0;
      for (int r = 0; r < n; ++r) col += hypot(P[r * n + c].x, P[r * n + c].y);
      best = fmax(best, col);
    }
    s_norm = best;
  }
  __syncthreads();
  int sq = 0;
  double scale = 1.0;
  while (s_norm * scale > 0.5 && sq < 60) {
    scale *= 0.5;
    ++sq;
  }
  for (int idx = threadIdx.x; idx < n * n; idx += blockDim.x) {
    P[idx].x *= scale;
    P[idx].y *= scale;
    Q[idx] = make_double2((idx / n == idx % n) ? 1.0 : 0.0, 0.0);
  }
  __syncthreads();
  // Horner: Q = I + P/1 (I + P/2 (I + ... (I + P/18)))
  for (int k = 18; k >= 1; --k) {
    cmatmul(n, P, Q, R);
    const double inv = 1.0 / k;
    for (int idx = threadIdx.x; idx < n * n; idx += blockDim.x) {
      const bool diag = idx / n == idx % n;
      Q[idx] = make_double2(R[idx].x * inv + (diag ? 1.0 : 0.0), R[idx].y * inv);
    }
    __syncthreads();
  }
  for (int t = 0; t < sq; ++t) {
    cmatmul(n, Q, Q, R);
    for (int idx = threadIdx.x; idx < n * n; idx += blockDim.x) Q[idx] = R[idx];
    __syncthreads();
  }
  for (int idx = threadIdx.x; idx < n * n; idx += blockDim.x) out[idx] = Q[idx];
  __syncthreads();
}

// Arnoldi controller (one CTA per trajectory): exponentials of T_M and
// T_(M-offset) over one observation spacing h, then marching c(k h) =
// E^k e1 over the uniform observation grid; the step is the largest k h
// whose embedded error (the reference's estimate, rpm_statevector_engine.py:
// 690-715) meets budget * k h / T.  Every grid point of the step is an
// observation point.  Dynamic shared memory: three kBMaxK^2 complex buffers.
__global__ void __launch_bounds__(128) k_b_control_arn(BatchDev B) {
  extern __shared__ double2 scratch[];
  __shared__ double2 chi[kBMaxK], clo[kBMaxK], nhi[kBMaxK], nlo[kBMaxK];
  __shared__ double red[32];
  __shared__ int s_k;
  const int b = blockIdx.x;
  TrajState& s = B.st[b];
  if (s.done) return;
  const int M = s.msize;
  const bool exact = s.stop != 0;
  const int ML = max(1, M - B.offset);
  double2* P = scratch;
  double2* Q = P + kBMaxK * kBMaxK;
  double2* R = Q + kBMaxK * kBMaxK;
  double2* Ehi = B.expm + (size_t)b * 2 * kBMaxK * kBMaxK;
  double2* Elo = Ehi + kBMaxK * kBMaxK;
  const double* hess_d = reinterpret_cast<const double*>(B.hess + (size_t)b * (kBMaxK + 1) * kBMaxK);
  hessenberg_expm(reinterpret_cast<const double2*>(hess_d), M, B.grid_h, P, Q, R, Ehi);
  if (!exact) hessenberg_expm(reinterpret_cast<const double2*>(hess_d), ML, B.grid_h, P, Q, R, Elo);
  const double t_now = s.t_now;
  const double remaining = B.t_end - t_now;
  const double dt_max = fmin(B.max_step, remaining);
  int kmax = (int)floor(dt_max / B.grid_h + 1e-9);
  kmax = min(kmax, kMaxPts);
  kmax = min(kmax, B.ntimes - s.cursor);
  for (int i = threadIdx.x; i < kBMaxK; i += blockDim.x) {
    chi[i] = make_double2(i == 0 ? 1.0 : 0.0, 0.0);
    clo[i] = chi[i];
  }
  if (threadIdx.x == 0) s_k = 0;
  __syncthreads();
  double2* rows = B.coef + (size_t)b * (kMaxPts + 1) * kBMaxK;
  const double norm = s.norm;
  for (int k = 1; k <= kmax; ++k) {
    // threads 0-63: hi system, 64-127: lo system
    const int t = threadIdx.x;
    if (t < M) {
      double2 acc = make_double2(0.0, 0.0);
      for (int c = 0; c < M; ++c) acc = cfma(Ehi[t * M + c], chi[c], acc);
      nhi[t] = acc;
    } else if (t >= 64 && t - 64 < ML && !exact) {
      const int r = t - 64;
      double2 acc = make_double2(0.0, 0.0);
      for (int c = 0; c < ML; ++c) acc = cfma(Elo[r * ML + c], clo[c], acc);
      nlo[r] = acc;
    }
    __syncthreads();
    double acc = 0.0;
    for (int i = threadIdx.x; i < M; i += blockDim.x) {
      chi[i] = nhi[i];
      if (!exact) {
        if (i < ML) clo[i] = nlo[i];
        const double2 lo = i < ML ? nlo[i] : make_double2(0.0, 0.0);
        const double dx = nhi[i].x - lo.x, dy = nhi[i].y - lo.y;
        acc = fma(dx, dx, fma(dy, dy, acc));
      }
    }
    acc = block_sum(acc, red);
    const double err = exact ? 0.0 : B.safety * norm * sqrt(acc);
    const double tk = k * B.grid_h;
    if (!(err <= B.budget * tk / B.t_end)) break;  // uniform: every thread sees the same sum
    for (int i = threadIdx.x; i < kBMaxK; i += blockDim.x) rows[(size_t)(k - 1) * kBMaxK + i] = i < M ? chi[i] : make_double2(0.0, 0.0);
    if (threadIdx.x == 0) {
      B.perr[(size_t)b * kMaxPts + k - 1] = err;
      s_k = k;
      s.step_err = err;
    }
    __syncthreads();
  }
  __syncthreads();
  const int kk = s_k;
  if (kk == 0) {
    if (threadIdx.x == 0) {
      s.status = 3;  // the first observation spacing already exceeds the error budget
      s.done = 1;
      s.skip = 1;
      atomicSub(B.active, 1);
    }
    return;
  }
  for (int i = threadIdx.x; i < kBMaxK; i += blockDim.x)
    rows[(size_t)kMaxPts * kBMaxK + i] = rows[(size_t)(kk - 1) * kBMaxK + i];
  if (threadIdx.x == 0) {
    double dt = kk * B.grid_h;
    if (remaining - dt < 1e-12) dt = remaining;
    s.dt = dt;
    s.npts = kk;
  }
}

// psi = ||psi|| V c_end (FP64 accumulation); ||psi||^2 into new_norm2.
__global__ void __launch_bounds__(kEwThreads) k_b_rebuild(BatchDev B) {
  __shared__ double2 cc[kBMaxK];
  __shared__ double red[32];
  const int b = blockIdx.y;
  TrajState& s = B.st[b];
  if (s.done) return;
  const int M = s.msize;
  const double2* row = B.coef + ((size_t)b * (kMaxPts + 1) + kMaxPts) * kBMaxK;
  for (int k = threadIdx.x; k < M; k += blockDim.x) cc[k] = make_double2(row[k].x * s.norm, row[k].y * s.norm);
  __syncthreads();
  const float2* V = B.V + (size_t)b * (B.m + 1) * B.ld;
  double2* x = B.psi + (size_t)b * B.ld;
  double nn = 0.0;
  // the thread's kEwPer elements are summed side by side (independent loads
  // and accumulation chains per basis vector); each element's sum runs over
  // k in ascending order
  const long long i0 = (long long)blockIdx.x * kEwChunk + threadIdx.x;
  const long long end = min(s.n, (long long)(blockIdx.x + 1) * kEwChunk);
  double2 acc[kEwPer];
#pragma unroll
  for (int e = 0; e < kEwPer; ++e) acc[e] = make_double2(0.0, 0.0);
  for (int k = 0; k < M; ++k) {
    const float2* vk = V + (size_t)k * B.ld;
    const double2 ck = cc[k];
    float2 v[kEwPer];
#pragma unroll
    for (int e = 0; e < kEwPer; ++e) {
      const long long i = i0 + (long long)e * kEwThreads;
      v[e] = i < end ? vk[i] : make_float2(0.f, 0.f);
    }
#pragma unroll
    for (int e = 0; e < kEwPer; ++e) acc[e] = cfma(ck, make_double2(v[e].x, v[e].y), acc[e]);
  }
#pragma unroll
  for (int e = 0; e < kEwPer; ++e) {
    const long long i = i0 + (long long)e * kEwThreads;
    if (i < end) {
      x[i] = acc[e];
      nn = fma(acc[e].x, acc[e].x, fma(acc[e].y, acc[e].y, nn));
    }
  }
  nn = block_sum(nn, red);
  if (threadIdx.x == 0) B.part[((size_t)b * B.nblk + blockIdx.x) * 2] = nn;
  if (traj_last_block(B.count + b) && threadIdx.x == 0) {
    double tot = 0.0;
    const double* p = B.part + (size_t)b * B.nblk * 2;
    for (int k = 0; k < (int)gridDim.x; ++k) tot += __ldcg(p + 2 * k);
    s.new_norm2 = tot;
    B.count[b] = 0;
  }
}

// Singlet Gram partials  G_kl = sum_q conj(a_k(q)) a_l(q),
// a_k(q) = (V_k[n/4 + q] - V_k[n/2 + q]) / sqrt 2, over this block's rows.
// Register-tiled: thread (u, g) owns the 4x4 tile u of the upper triangle
// (tile row <= tile column; the Hermitian lower half is written mirrored)
// for the rows g, g + NG, ... of each staged chunk.  Products and sums are
// FP32 within one chunk and FP64 across chunks and row groups.
constexpr int kGramChunk = 64;   // rows per staged chunk
constexpr int kGramGroups = 8;   // at most this many row groups per block
__global__ void __launch_bounds__(256) k_b_gram(BatchDev B) {
  // staged chunk; reused for the row-group sum (needed only when NG > 1,
  // i.e. at most 128 tiles: 16 x 128 double2 = 32 KiB <= the chunk's bytes)
  __shared__ __align__(16) float2 a[kGramChunk][kBMaxK + 2];
  double2(*red)[128] = reinterpret_cast<double2(*)[128]>(&a[0][0]);
  static_assert(sizeof(a) >= 16 * 128 * sizeof(double2), "row-group buffer does not fit");
  const int b = blockIdx.y;
  TrajState& s = B.st[b];
  if (s.done) return;
  const int M = s.msize;
  const int T = (M + 3) / 4;             // tiles per side
  const int NU = T * (T + 1) / 2;        // upper-triangle tiles
  const int NG = min(kGramGroups, max(1, (int)blockDim.x / NU));
  const int u = threadIdx.x % NU, g = threadIdx.x / NU;
  const bool worker = g < NG;
  int ti = 0, rem = u;
  while (rem >= T - ti) {
    rem -= T - ti;
    ++ti;
  }
  const int tj = ti + rem;
  const long long q4 = s.n / 4;
  const float2* V = B.V + (size_t)b * (B.m + 1) * B.ld;
  const float rs2 = 0.70710678118654752440f;
  double2 acc[4][4];
#pragma unroll
  for (int p = 0; p < 4; ++p)
#pragma unroll
    for (int q = 0; q < 4; ++q) acc[p][q] = make_double2(0.0, 0.0);
  const int KP = 4 * T;  // staged columns (zero beyond M)
  for (long long r0 = (long long)blockIdx.x * kGramChunk; r0 < q4; r0 += (long long)gridDim.x * kGramChunk) {
    __syncthreads();
    for (int idx = threadIdx.x; idx < kGramChunk * KP; idx += blockDim.x) {
      const int k = idx / kGramChunk, rr = idx % kGramChunk;
      const long long qq = r0 + rr;
      float2 v = make_float2(0.f, 0.f);
      if (qq < q4 && k < M) {
        const float2 p1 = V[(size_t)k * B.ld + q4 + qq];
        const float2 p2 = V[(size_t)k * B.ld + 2 * q4 + qq];
        v = make_float2((p1.x - p2.x) * rs2, (p1.y - p2.y) * rs2);
      }
      a[rr][k] = v;
    }
    __syncthreads();
    if (worker) {
      float2 cs[4][4];
#pragma unroll
      for (int p = 0; p < 4; ++p)
#pragma unroll
        for (int q = 0; q < 4; ++q) cs[p][q] = make_float2(0.f, 0.f);
      for (int rr = g; rr < kGramChunk; rr += NG) {
        const float4 u01 = *reinterpret_cast<const float4*>(&a[rr][4 * ti]);
        const float4 u23 = *reinterpret_cast<const float4*>(&a[rr][4 * ti + 2]);
        const float4 v01 = *reinterpret_cast<const float4*>(&a[rr][4 * tj]);
        const float4 v23 = *reinterpret_cast<const float4*>(&a[rr][4 * tj + 2]);
        const float2 uu[4] = {make_float2(u01.x, u01.y), make_float2(u01.z, u01.w), make_float2(u23.x, u23.y),
                              make_float2(u23.z, u23.w)};
        const float2 vv[4] = {make_float2(v01.x, v01.y), make_float2(v01.z, v01.w), make_float2(v23.x, v23.y),
                              make_float2(v23.z, v23.w)};
#pragma unroll
        for (int p = 0; p < 4; ++p)
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            cs[p][q].x = fmaf(uu[p].x, vv[q].x, fmaf(uu[p].y, vv[q].y, cs[p][q].x));
            cs[p][q].y = fmaf(uu[p].x, vv[q].y, fmaf(-uu[p].y, vv[q].x, cs[p][q].y));
          }
      }
#pragma unroll
      for (int p = 0; p < 4; ++p)
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          acc[p][q].x += cs[p][q].x;
          acc[p][q].y += cs[p][q].y;
        }
    }
  }
  // sum the row groups in FP64, one group at a time (NG > 1 implies NU <= 128)
  if (NG > 1) {
    __syncthreads();  // the chunk buffer is reused
    for (int gg = 0; gg < NG; ++gg) {
      if (worker && g == gg) {
#pragma unroll
        for (int p = 0; p < 4; ++p)
#pragma unroll
          for (int q = 0; q < 4; ++q) red[p * 4 + q][u] = gg ? cadd(red[p * 4 + q][u], acc[p][q]) : acc[p][q];
      }
      __syncthreads();
    }
  }
  double2* out = B.gpart + ((size_t)b * B.gblk + blockIdx.x) * kBMaxK * kBMaxK;  // compact M x M
  if (worker && g == 0) {
#pragma unroll
    for (int p = 0; p < 4; ++p)
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int k = 4 * ti + p, l = 4 * tj + q;
        if (k < M && l < M) {
          const double2 v = NG > 1 ? red[p * 4 + q][u] : acc[p][q];
          out[k * M + l] = v;
          if (ti != tj) out[l * M + k] = make_double2(v.x, -v.y);
        }
      }
  }
}

// Populations at the step's observation points and the controller update.
__global__ void __launch_bounds__(256) k_b_observe(BatchDev B) {
  extern __shared__ double2 G[];  // M x M
  const int b = blockIdx.x;
  TrajState& s = B.st[b];
  if (s.done) return;
  const int M = s.msize;
  const int pairs = M * M;
  for (int pr = threadIdx.x; pr < pairs; pr += blockDim.x) {
    double2 t = make_double2(0.0, 0.0);
    const double2* p = B.gpart + (size_t)b * B.gblk * kBMaxK * kBMaxK + pr;
    for (int k = 0; k < B.gblk; ++k) t = cadd(t, p[(size_t)k * kBMaxK * kBMaxK]);
    G[pr] = t;
  }
  __syncthreads();
  const double n2 = s.norm * s.norm;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const double2* rows = B.coef + (size_t)b * (kMaxPts + 1) * kBMaxK;
  for (int p = warp; p < s.npts; p += nw) {
    const double2* cv = rows + (size_t)p * kBMaxK;
    double v = 0.0;
    for (int i = lane; i < M; i += 32) {
      // (G c)_i with G Hermitian-symmetrised on the fly
      double2 gc = make_double2(0.0, 0.0);
      for (int k = 0; k < M; ++k) {
        const double2 g1 = G[i * M + k], g2 = G[k * M + i];
        const double2 g = make_double2(0.5 * (g1.x + g2.x), 0.5 * (g1.y - g2.y));
        gc = cfma(g, cv[k], gc);
      }
      v += cv[i].x * gc.x + cv[i].y * gc.y;
    }
    v = warp_sum(v);
    if (lane == 0) {
      const int at = s.cursor + p;
      B.values[(size_t)b * B.ntimes + at] = n2 * v;
      B.errs[(size_t)b * B.ntimes + at] = s.acc_err + B.perr[(size_t)b * kMaxPts + p];
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    s.t_now += s.dt;
    s.cursor += s.npts;
    s.acc_err += s.step_err;
    s.steps += 1;
    s.matvecs += s.msize;
    s.min_step = fmin(s.min_step, s.dt);
    s.max_step = fmax(s.max_step, s.dt);
    s.hint = s.dt;
    s.norm = sqrt(s.new_norm2);
    s.max_norm_err = fmax(s.max_norm_err, fabs(s.norm - 1.0));
    if (!isfinite(s.norm)) s.status = 4;
    if (s.cursor >= B.ntimes || s.status != 0) {
      s.done = 1;
      s.skip = 1;
      atomicSub(B.active, 1);
    }
  }
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
}  // namespace rpm

#include "gram_tc.cuh"

struct rpm_batch {
  std::vector<rpm_system*> systems;
  rpm_batch_config cfg{};
  // maxima over all systems of the batch, for buffer sizing only (launches
  // use the plan of their shape group)
  int max_nl = 0, max_half_r = 0;
  rpm::CubeView<float2>* views_dev = nullptr;
  long long ld = 0;
  // buffers (grown on demand)
  int cap_traj = 0, cap_times = 0;
  void* buf = nullptr;
  size_t buf_bytes = 0;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int graph_traj = -1, graph_times = -1;
  // Work is issued on a private non-blocking stream (graph capture is not
  // allowed on the legacy default stream), ordered after the caller's stream
  // on entry and before it on exit through events.
  cudaStream_t work = nullptr;
  cudaEvent_t ev_in = nullptr, ev_out = nullptr;
  // The singlet Gram depends only on the basis: it runs on `side`, forked
  // from and joined back into `work`, concurrently with the controller.
  cudaStream_t side = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  // Measurement: a timed event pair around the H psi of Lanczos iteration 1 of
  // every Krylov step (recorded inside the graph), sampled at each poll while
  // every trajectory is still running; and the number of kernels launched.
  cudaEvent_t probe0 = nullptr, probe1 = nullptr;
  double probe_ms_sum = 0.0;
  long long probe_samples = 0;
  long long kernel_launches = 0, replays = 0;
  int launches_per_step = 0;
  int probe_iters = 1;      // Lanczos iterations between the probe events
  bool fused = false;       // every group runs the fused passes
  bool persistent = false;  // every group runs the persistent Lanczos kernel
  bool gram_tc = false;     // the singlet Gram runs on the tensor cores (k_b_gram_tc)
  // Consecutive trajectories whose systems share one shape (digit pattern and
  // layout) form a group; each group's H psi is one launch pair with its own
  // plan, on the shape-specialised passes when the shape allows.
  struct ShapeGroup {
    int b0, nb;
    rpm::CubePlan plan;
    bool records;  // every member carries the outer-index records of the persistent kernel
  };
  std::vector<ShapeGroup> groups;
  int dot_stride = 1;  // partial-sum slots per trajectory
  std::vector<int> caps;  // Krylov cap per system (0: the batch's dimension)
};

namespace rpm {

// Which kernel forms the singlet Gram (rpm_set_gram_kernel): 0 the CUDA-core
// k_b_gram, 1 the tensor-core k_b_gram_tc where the batch allows it.
static std::atomic<int> g_gram_kernel{1};

// The singlet Gram of the step's basis, on the side stream (it overlaps the
// controller and the rebuild).
static void launch_gram(const rpm_batch* Bh, const BatchDev& B) {
  if (Bh->gram_tc) {
    const CUtensorMap map = basis_rows_map(B.V, (long long)B.ntraj * (B.m + 1), B.ld, gramtc::kGC, B.m + 1);
    gramtc::k_b_gram_tc<<<dim3(B.gblk, B.ntraj), gramtc::kThreads, gramtc::kSmemBytes, Bh->side>>>(map, B);
  }
  else
    k_b_gram<<<dim3(B.gblk, B.ntraj), 256, 0, Bh->side>>>(B);
}

static void free_graph(rpm_batch* B) {
  if (B->exec) cudaGraphExecDestroy(B->exec);
  if (B->graph) cudaGraphDestroy(B->graph);
  B->exec = nullptr;
  B->graph = nullptr;
  B->graph_traj = B->graph_times = -1;
}

struct Layout {
  size_t st, V, coef, perr, part, count, gpart, ya, dotpart, dotcount, times, sysof, nof, active, hess, hcur, adots,
      expm, prog, pcnt, ppart, work, kstatus, capof, total;
};

static Layout layout(const rpm_batch* B, int ntraj, int ntimes, int nblk, int gblk, int dot_blocks, int ppart_stride,
                     int nwork) {
  Layout L{};
  size_t pos = 0;
  auto take = [&](size_t bytes) {
    const size_t at = pos;
    pos += (bytes + 255) & ~(size_t)255;
    return at;
  };
  const int m = B->cfg.krylov_dim;
  L.st = take(sizeof(TrajState) * ntraj);
  L.V = take(sizeof(float2) * (size_t)ntraj * (m + 1) * B->ld);
  L.coef = take(sizeof(double2) * (size_t)ntraj * (kMaxPts + 1) * kBMaxK);
  L.perr = take(sizeof(double) * (size_t)ntraj * kMaxPts);
  L.part = take(sizeof(double) * (size_t)ntraj * nblk * 2);
  L.count = take(sizeof(unsigned) * ntraj);
  L.gpart = take(sizeof(double2) * (size_t)ntraj * gblk * kBMaxK * kBMaxK);
  L.ya = take(sizeof(float2) * (size_t)ntraj * B->ld);
  L.dotpart = take(sizeof(double) * (size_t)ntraj * dot_blocks);
  L.dotcount = take(sizeof(unsigned) * ntraj);
  L.times = take(sizeof(double) * ntimes);
  L.sysof = take(sizeof(int) * ntraj);
  L.nof = take(sizeof(long long) * ntraj);
  L.active = take(sizeof(int));
  L.hess = take(sizeof(double2) * (size_t)ntraj * (kBMaxK + 1) * kBMaxK);
  L.hcur = take(sizeof(double2) * (size_t)ntraj * kBMaxK);
  L.adots = take(sizeof(double2) * (size_t)ntraj * nblk * kBMaxK);
  L.expm = take(sizeof(double2) * (size_t)ntraj * 2 * kBMaxK * kBMaxK);
  L.prog = take(sizeof(int) * ntraj);
  L.pcnt = take(sizeof(unsigned) * ntraj);
  L.ppart = take(sizeof(double) * (size_t)ntraj * ppart_stride);
  L.work = take(sizeof(unsigned) * (size_t)nwork);
  L.kstatus = take(sizeof(int));
  L.capof = take(sizeof(int) * ntraj);
  L.total = pos;
  return L;
}

// Launch arguments of trajectories b0, b0 + 1, ... (every per-trajectory
// pointer advanced by b0); `dstride` partial-sum slots per trajectory.
static HpsiArgs<float2> group_args(const HpsiArgs<float2>& a, int b0, int dstride) {
  HpsiArgs<float2> c = a;
  const long long s = b0;
  c.in += s * a.ld;
  c.out += s * a.ld;
  if (c.in_scale) c.in_scale += s * a.scale_stride;
  if (c.skip) c.skip += s * a.skip_stride;
  if (c.sys_of) c.sys_of += s;
  if (c.dot_out) c.dot_out += s * a.dot_stride;
  if (c.dot_part) c.dot_part += s * dstride;
  if (c.dot_count) c.dot_count += s;
  LanczosFuse& z = c.lz;
  if (z.prev) z.prev += s * a.ld;
  if (z.alpha_prev) z.alpha_prev += s * z.dstride;
  if (z.beta_prev) z.beta_prev += s * z.dstride;
  if (z.alpha_out) z.alpha_out += s * z.dstride;
  if (z.beta_out) z.beta_out += s * z.dstride;
  if (z.scale_out) z.scale_out += s * z.dstride;
  if (z.stop) z.stop += s * z.istride;
  if (z.skip) z.skip += s * z.istride;
  if (z.msize) z.msize += s * z.istride;
  if (z.mcap) z.mcap += s * z.istride;
  return c;
}

static void record_step(rpm_batch* Bh, const BatchDev& B, const Layout& L, cudaStream_t st) {
  char* base = static_cast<char*>(Bh->buf);
  const int m = B.m;
  dim3 ew(B.nblk, B.ntraj);
  k_b_start<<<ew, kEwThreads, 0, st>>>(B);
  HpsiArgs<float2> a{};
  a.ld = (long long)(m + 1) * B.ld;
  a.ya_ld = B.ld;
  a.in_scale = &B.st[0].scale;
  a.scale_stride = kStateDoubles;
  a.skip = &B.st[0].skip;
  a.skip_stride = kStateInts;
  a.views = Bh->views_dev;
  a.sys_of = reinterpret_cast<const int*>(base + L.sysof);
  a.dot_stride = kStateDoubles;
  a.dot_part = reinterpret_cast<double*>(base + L.dotpart);
  a.dot_count = reinterpret_cast<unsigned*>(base + L.dotcount);
  float2* ya = reinterpret_cast<float2*>(base + L.ya);
  const int probe_j = m > 1 ? 1 : 0;
  cudaStreamCaptureStatus capturing = cudaStreamCaptureStatusNone;
  check_cuda(cudaStreamIsCapturing(st, &capturing), "capture status");
  const unsigned probe_flags = capturing == cudaStreamCaptureStatusActive ? cudaEventRecordExternal : 0u;
  const int D = Bh->dot_stride;
  // Per shape group: the shape-specialised passes carry the Lanczos
  // recurrence themselves (LanczosFuse: no update kernel); otherwise H psi on
  // the general cube kernels + k_b_update.  Non-Hermitian systems (unequal
  // recombination rates) run Arnoldi instead.
  a.in = B.V;
  a.out = B.V + B.ld;
  std::vector<char> gfused(Bh->groups.size());
  bool all_fused = true;
  for (size_t g = 0; g < Bh->groups.size(); ++g) {
    const auto& G = Bh->groups[g];
    gfused[g] = cube_fast_usable(group_args(a, G.b0, D), G.plan, ya + (size_t)G.b0 * B.ld) ? 1 : 0;
    all_fused = all_fused && gfused[g];
  }
  int per_iter = 0;
  for (size_t g = 0; g < Bh->groups.size(); ++g) per_iter += gfused[g] ? 2 : 3;
  if (B.arnoldi) {
    for (int j = 0; j < m; ++j) {
      a.in = B.V + (size_t)j * B.ld;
      a.out = B.V + (size_t)(j + 1) * B.ld;
      LanczosFuse& z = a.lz;
      z = LanczosFuse{};
      z.first = j == 0;
      z.last = j == m - 1;
      z.j = j;
      a.dot_out = nullptr;
      a.dot_part = nullptr;
      if (j == probe_j) check_cuda(cudaEventRecordWithFlags(Bh->probe0, st, probe_flags), "probe record");
      for (size_t g = 0; g < Bh->groups.size(); ++g) {
        const auto& G = Bh->groups[g];
        HpsiArgs<float2> ak = group_args(a, G.b0, D);
        float2* yk = ya + (size_t)G.b0 * B.ld;
        if (gfused[g]) {
          ak.lz.on = 2;  // pass R scales v_j (written back) while staging
          if (!launch_cube_fast(ak, G.plan, yk, G.nb, st)) fail(RPM_E_INVALID, "H psi passes unavailable");
        } else {
          // one shape per launch: H (scale V_j), then V_j *= scale
          launch_cube<float2>(ak, G.plan, yk, G.nb, st);
          k_b_arn_scale<<<dim3(B.nblk, G.nb), kEwThreads, 0, st>>>(B, j, G.b0);
        }
      }
      if (j == probe_j) check_cuda(cudaEventRecordWithFlags(Bh->probe1, st, probe_flags), "probe record");
      for (int pass = 1; pass <= 2; ++pass) {
        k_b_arn_dots<<<ew, kEwThreads, 0, st>>>(B, j, pass);
        k_b_arn_axpy<<<ew, kEwThreads, 0, st>>>(B, j, pass);
      }
    }
    Bh->fused = false;
    Bh->persistent = false;
    Bh->probe_iters = 1;
    Bh->launches_per_step = 1 + (per_iter + 4) * m + 4;
    check_cuda(cudaEventRecord(Bh->ev_fork, st), "fork record");
    check_cuda(cudaStreamWaitEvent(Bh->side, Bh->ev_fork, 0), "fork wait");
    launch_gram(Bh, B);
    check_cuda(cudaEventRecord(Bh->ev_join, Bh->side), "join record");
    k_b_control_arn<<<B.ntraj, 128, kArnCtlSmem, st>>>(B);
    k_b_rebuild<<<ew, kEwThreads, 0, st>>>(B);
    check_cuda(cudaStreamWaitEvent(st, Bh->ev_join, 0), "join wait");
    k_b_observe<<<B.ntraj, 256, sizeof(double2) * kBMaxK * kBMaxK, st>>>(B);
    check_launch("batched Arnoldi step");
    return;
  }
  // Shape groups with a persistent Lanczos kernel run every iteration of the
  // step in one launch; the others launch their passes per iteration.
  // Periodic reorthogonalisation after iterations P-1, 2P-1, ... (< m-1)
  // covers every trajectory at once: with it, either every group runs the
  // persistent kernel (in segments between the reorthogonalisations) or none.
  const int reo = Bh->cfg.reorth_policy == RPM_REORTH_PERIODIC && Bh->cfg.reorth_period > 0 ? Bh->cfg.reorth_period : 0;
  std::vector<char> gpers(Bh->groups.size());
  int npers = 0;
  for (size_t g = 0; g < Bh->groups.size(); ++g) {
    gpers[g] = Bh->cfg.lanczos_kernel == RPM_LANCZOS_PERSISTENT && gfused[g] && Bh->groups[g].records &&
               persistent_l_tiles(Bh->groups[g].plan) > 0;
    npers += gpers[g];
  }
  if (reo > 0 && npers != (int)Bh->groups.size()) {
    std::fill(gpers.begin(), gpers.end(), 0);
    npers = 0;
  }
  const bool all_pers = npers == (int)Bh->groups.size();
  auto reorth_after = [&](int j) { return reo > 0 && (j + 1) % reo == 0 && j + 1 < m; };
  auto reorthogonalise = [&](int j) {
    for (int pass = 1; pass <= 2; ++pass) {
      k_b_reo_dots<<<ew, kEwThreads, 0, st>>>(B, j);
      k_b_reo_axpy<<<ew, kEwThreads, 0, st>>>(B, j, pass == 2 ? 1 : 0);
    }
    check_launch("batched reorthogonalisation");
  };
  const int nseg = reo > 0 ? (m + reo - 1) / reo : 1;  // segments of the persistent launches
  if (all_pers) check_cuda(cudaEventRecordWithFlags(Bh->probe0, st, probe_flags), "probe record");
  for (int seg = 0; seg < nseg && npers > 0; ++seg) {
    const int j0 = reo > 0 ? seg * reo : 0;
    const int j1 = reo > 0 ? std::min(m, (seg + 1) * reo) : m;
    for (size_t g = 0; g < Bh->groups.size(); ++g) {
      if (!gpers[g]) continue;
      const auto& G = Bh->groups[g];
      PersistentLanczos P{};
      P.V = B.V + (size_t)G.b0 * (m + 1) * B.ld;
      P.ld = B.ld;
      P.vstride = (long long)(m + 1) * B.ld;
      P.slot0 = (long long)G.b0 * (m + 1);
      P.m = m;
      P.nb = G.nb;
      // wavefront groups: the requested size, or equal groups of at most 16
      // vectors (48 vectors: three of 16, 0.1675 ms per iteration against
      // 0.1755 ms for four of 12; a partial last group costs more)
      if (Bh->cfg.wavefront > 0) {
        P.gv = Bh->cfg.wavefront;
      } else {
        const int ngroups = (G.nb + 15) / 16;
        P.gv = (G.nb + ngroups - 1) / ngroups;
      }
      P.j0 = j0;
      P.j1 = j1;
      P.views = Bh->views_dev;
      P.sys_of = reinterpret_cast<const int*>(base + L.sysof) + G.b0;
      P.alpha = &B.st[G.b0].alpha[0];
      P.beta = &B.st[G.b0].beta[0];
      P.scale = &B.st[G.b0].scale;
      P.dstride = kStateDoubles;
      P.stop = &B.st[G.b0].stop;
      P.skip = &B.st[G.b0].skip;
      P.msize = &B.st[G.b0].msize;
      P.mcap = &B.st[G.b0].mcap;
      P.istride = kStateInts;
      P.breakdown_rel = B.breakdown_rel;
      P.ya = ya + (size_t)G.b0 * B.ld;
      P.prog = B.prog + G.b0;
      P.cnt = B.pcnt + G.b0;
      P.part = B.ppart + (size_t)G.b0 * B.ppart_stride;
      P.part_stride = B.ppart_stride;
      P.work = B.work + g * nseg + seg;
      P.status = B.kstatus;
      P.ctas = Bh->cfg.persistent_ctas;
      if (!launch_lanczos_persistent(P, G.plan, B.V, (long long)B.ntraj * (m + 1), st))
        fail(RPM_E_INVALID, "persistent Lanczos kernel unavailable");
    }
    if (all_pers && reorth_after(j1 - 1)) reorthogonalise(j1 - 1);
  }
  if (all_pers) {
    check_cuda(cudaEventRecordWithFlags(Bh->probe1, st, probe_flags), "probe record");
    Bh->probe_iters = m;
  } else {
    Bh->probe_iters = 1;
  }
  for (int j = 0; j < m && !all_pers; ++j) {
    a.in = B.V + (size_t)j * B.ld;
    a.out = B.V + (size_t)(j + 1) * B.ld;
    // While capturing, external records become event-record nodes of the graph.
    if (j == probe_j) check_cuda(cudaEventRecordWithFlags(Bh->probe0, st, probe_flags), "probe record");
    LanczosFuse& z = a.lz;
    z = LanczosFuse{};
    z.on = 1;
    z.first = j == 0;
    z.last = j == m - 1;
    z.j = j;
    z.prev = j > 0 ? B.V + (size_t)(j - 1) * B.ld : nullptr;
    z.alpha_prev = j > 0 ? &B.st[0].alpha[j - 1] : nullptr;
    z.beta_prev = j > 0 ? &B.st[0].beta[j - 1] : nullptr;
    z.alpha_out = &B.st[0].alpha[j];
    z.beta_out = &B.st[0].beta[j];
    z.scale_out = &B.st[0].scale;
    z.stop = &B.st[0].stop;
    z.skip = &B.st[0].skip;
    z.msize = &B.st[0].msize;
    z.mcap = &B.st[0].mcap;
    z.dstride = kStateDoubles;
    z.istride = kStateInts;
    z.breakdown_rel = B.breakdown_rel;
    for (size_t g = 0; g < Bh->groups.size(); ++g) {
      if (gpers[g]) continue;
      const auto& G = Bh->groups[g];
      HpsiArgs<float2> ak = group_args(a, G.b0, D);
      float2* yk = ya + (size_t)G.b0 * B.ld;
      if (gfused[g]) {
        ak.dot_out = nullptr;
        if (!launch_cube_fast(ak, G.plan, yk, G.nb, st)) fail(RPM_E_INVALID, "fused Lanczos passes unavailable");
      } else {
        ak.lz = LanczosFuse{};
        ak.dot_out = &B.st[G.b0].alpha[j];
        launch_cube<float2>(ak, G.plan, yk, G.nb, st);
        k_b_update<<<dim3(B.nblk, G.nb), kEwThreads, 0, st>>>(B, j, G.b0);
      }
    }
    if (reorth_after(j)) reorthogonalise(j);
    if (j == probe_j) check_cuda(cudaEventRecordWithFlags(Bh->probe1, st, probe_flags), "probe record");
  }
  const bool fused = all_fused;
  Bh->fused = fused;
  Bh->persistent = all_pers;
  int per_iter_rest = 0;
  for (size_t g = 0; g < Bh->groups.size(); ++g)
    if (!gpers[g]) per_iter_rest += gfused[g] ? 2 : 3;
  const int nreo = reo > 0 ? (m - 1) / reo : 0;  // iterations j = P-1, 2P-1, ... <= m-2
  Bh->launches_per_step = 1 + npers * nseg + per_iter_rest * m + 4 * nreo + 4;
  const size_t ctl_smem = sizeof(double) * 2 * kRecDoubles;
  check_cuda(cudaEventRecord(Bh->ev_fork, st), "fork record");
  check_cuda(cudaStreamWaitEvent(Bh->side, Bh->ev_fork, 0), "fork wait");
  launch_gram(Bh, B);
  check_cuda(cudaEventRecord(Bh->ev_join, Bh->side), "join record");
  k_b_control<<<B.ntraj, 128, ctl_smem, st>>>(B);
  k_b_rebuild<<<ew, kEwThreads, 0, st>>>(B);
  check_cuda(cudaStreamWaitEvent(st, Bh->ev_join, 0), "join wait");
  k_b_observe<<<B.ntraj, 256, sizeof(double2) * kBMaxK * kBMaxK, st>>>(B);
  check_launch("batched step");
}

static void run_batch(rpm_batch* Bh, int ntraj, const int* sys_of, void* psi, const double* times_host, int ntimes,
                      double* values, double* errs, rpm_batch_stats* stats, cudaStream_t caller) {
  const rpm_batch_config& cfg = Bh->cfg;
  cudaStream_t st = Bh->work;
  check_cuda(cudaEventRecord(Bh->ev_in, caller), "record entry event");
  check_cuda(cudaStreamWaitEvent(st, Bh->ev_in, 0), "wait entry event");
  if (ntraj < 1 || ntimes < 1) fail(RPM_E_INVALID, "At least one trajectory and one observation time are required.");
  for (int k = 0; k < ntimes; ++k) {
    if (!(times_host[k] >= 0.0) || (k && !(times_host[k] > times_host[k - 1])))
      fail(RPM_E_INVALID, "Observation times must be nonnegative and strictly increasing.");
  }
  std::vector<long long> n_of(ntraj);
  std::vector<int> cap_of(ntraj, 0);
  for (int b = 0; b < ntraj; ++b) {
    if (sys_of[b] < 0 || sys_of[b] >= (int)Bh->systems.size()) fail(RPM_E_INVALID, "system index out of range");
    n_of[b] = Bh->systems[sys_of[b]]->n;
    if (!Bh->caps.empty()) cap_of[b] = Bh->caps[sys_of[b]];
  }
  const int nblk = (int)((Bh->ld + kEwChunk - 1) / kEwChunk);
  const int gblk = std::max(1, std::min(32, (int)((Bh->ld / 4 + kGramChunk - 1) / kGramChunk)));
  // tensor-core Gram: 16-byte aligned bulk copies need n / 4 even, and the
  // basis (m + 1 vectors) fits the 64 rows per real part of its operand
  Bh->gram_tc = g_gram_kernel.load(std::memory_order_relaxed) == 1 && cfg.krylov_dim + 1 <= gramtc::kMaxBasis;
  for (int b = 0; b < ntraj && Bh->gram_tc; ++b) Bh->gram_tc = n_of[b] % 8 == 0;
  // shape groups: runs of consecutive trajectories whose systems share a shape
  Bh->groups.clear();
  for (int b = 0; b < ntraj;) {
    int e = b + 1;
    while (e < ntraj && same_cube_shape(Bh->systems[sys_of[e]], Bh->systems[sys_of[b]])) ++e;
    std::vector<rpm_system*> members;
    for (int k = b; k < e; ++k) {
      rpm_system* sk = Bh->systems[sys_of[k]];
      if (std::find(members.begin(), members.end(), sk) == members.end()) members.push_back(sk);
    }
    bool records = true;
    for (const rpm_system* sk : members) records = records && sk->cube32.orecR && sk->cube32.orecL;
    Bh->groups.push_back({b, e - b, cube_plan(members.data(), (int)members.size()), records});
    b = e;
  }
  // partial-sum slots per trajectory: general pass R (grid.x <= nl) or fused pass L (3 per block)
  const int dot_blocks = std::max({Bh->max_nl, 3 * (Bh->max_half_r / 8), 1});
  Bh->dot_stride = dot_blocks;
  int lt_max = 1;
  for (const auto& G : Bh->groups) lt_max = std::max(lt_max, persistent_l_tiles(G.plan));
  const int ppart_stride = 3 * lt_max;
  const int reo_period = cfg.reorth_policy == RPM_REORTH_PERIODIC && cfg.reorth_period > 0 ? cfg.reorth_period : 0;
  const int nseg_max = reo_period > 0 ? (cfg.krylov_dim + reo_period - 1) / reo_period : 1;
  const int nwork = (int)Bh->groups.size() * std::max(1, nseg_max);
  const Layout L = layout(Bh, ntraj, ntimes, nblk, gblk, dot_blocks, ppart_stride, nwork);
  if (L.total > Bh->buf_bytes) {
    free_graph(Bh);
    if (Bh->buf) check_cuda(cudaFree(Bh->buf), "cudaFree(batch)");
    Bh->buf = nullptr;
    check_cuda(cudaMalloc(&Bh->buf, L.total), "cudaMalloc(batch)");
    Bh->buf_bytes = L.total;
  }
  char* base = static_cast<char*>(Bh->buf);
  check_cuda(cudaMemsetAsync(base + L.count, 0, sizeof(unsigned) * ntraj, st), "memset counters");
  check_cuda(cudaMemsetAsync(base + L.dotcount, 0, sizeof(unsigned) * ntraj, st), "memset counters");
  check_cuda(cudaMemsetAsync(base + L.kstatus, 0, sizeof(int), st), "memset status");
  check_cuda(cudaMemcpyAsync(base + L.times, times_host, sizeof(double) * ntimes, cudaMemcpyHostToDevice, st), "times");
  check_cuda(cudaMemcpyAsync(base + L.sysof, sys_of, sizeof(int) * ntraj, cudaMemcpyHostToDevice, st), "sys_of");
  check_cuda(cudaMemcpyAsync(base + L.nof, n_of.data(), sizeof(long long) * ntraj, cudaMemcpyHostToDevice, st), "n_of");
  check_cuda(cudaMemcpyAsync(base + L.capof, cap_of.data(), sizeof(int) * ntraj, cudaMemcpyHostToDevice, st),
             "cap_of");
  check_cuda(cudaMemcpyAsync(base + L.active, &ntraj, sizeof(int), cudaMemcpyHostToDevice, st), "active");

  BatchDev B{};
  B.st = reinterpret_cast<TrajState*>(base + L.st);
  B.ntraj = ntraj;
  B.m = cfg.krylov_dim;
  B.offset = cfg.embedded_offset;
  B.safety = cfg.safety_factor;
  B.budget = cfg.state_error_budget;
  B.max_step = cfg.maximum_step_us;
  B.min_step = cfg.minimum_step_us;
  B.t_end = times_host[ntimes - 1];
  B.breakdown_rel = cfg.breakdown_relative;
  B.times = reinterpret_cast<const double*>(base + L.times);
  B.ntimes = ntimes;
  B.ld = Bh->ld;
  B.V = reinterpret_cast<float2*>(base + L.V);
  B.psi = static_cast<double2*>(psi);
  B.coef = reinterpret_cast<double2*>(base + L.coef);
  B.perr = reinterpret_cast<double*>(base + L.perr);
  B.part = reinterpret_cast<double*>(base + L.part);
  B.count = reinterpret_cast<unsigned*>(base + L.count);
  B.gpart = reinterpret_cast<double2*>(base + L.gpart);
  B.values = values;
  B.errs = errs;
  B.nblk = nblk;
  B.gblk = gblk;
  B.active = reinterpret_cast<int*>(base + L.active);
  B.hess = reinterpret_cast<double2*>(base + L.hess);
  B.hcur = reinterpret_cast<double2*>(base + L.hcur);
  B.adots = reinterpret_cast<double2*>(base + L.adots);
  B.expm = reinterpret_cast<double2*>(base + L.expm);
  B.prog = reinterpret_cast<int*>(base + L.prog);
  B.pcnt = reinterpret_cast<unsigned*>(base + L.pcnt);
  B.ppart = reinterpret_cast<double*>(base + L.ppart);
  B.ppart_stride = ppart_stride;
  B.work = reinterpret_cast<unsigned*>(base + L.work);
  B.nwork = nwork;
  B.kstatus = reinterpret_cast<int*>(base + L.kstatus);
  B.arnoldi = 0;
  for (rpm_system* sy : Bh->systems) B.arnoldi |= sy->non_hermitian ? 1 : 0;
  B.grid_h = 0.0;
  if (B.arnoldi) {
    // the Arnoldi controller marches over a uniform observation grid that
    // starts at 0 or one spacing
    if (ntimes < 2) fail(RPM_E_INVALID, "unequal recombination rates need at least two observation times");
    const double h = times_host[1] - times_host[0];
    const double k0 = times_host[0] / h;
    if (!(h > 0.0) || !(std::fabs(k0) < 1e-9 || std::fabs(k0 - 1.0) < 1e-9))
      fail(RPM_E_INVALID, "unequal recombination rates need observation times k h starting at 0 or h");
    for (int k = 0; k < ntimes; ++k)
      if (std::fabs(times_host[k] - (k + k0) * h) > 1e-9 * h * (k + 1))
        fail(RPM_E_INVALID, "unequal recombination rates need uniformly spaced observation times");
    B.grid_h = h;
    check_cuda(cudaMemsetAsync(B.hess, 0, sizeof(double2) * (size_t)ntraj * (kBMaxK + 1) * kBMaxK, st), "memset hess");
    check_cuda(cudaFuncSetAttribute(k_b_control_arn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kArnCtlSmem),
               "Arnoldi control attr");
  }

  k_b_setup<<<(ntraj + 127) / 128, 128, 0, st>>>(B, reinterpret_cast<const int*>(base + L.sysof),
                                                 reinterpret_cast<const long long*>(base + L.nof),
                                                 reinterpret_cast<const int*>(base + L.capof), cfg.initial_step_us);
  k_b_init<<<dim3(nblk, ntraj), kEwThreads, 0, st>>>(B);
  check_launch("batched init");
  const size_t ctl_smem = sizeof(double) * 2 * kRecDoubles;
  check_cuda(cudaFuncSetAttribute(k_b_control, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ctl_smem),
             "control attr");
  if (Bh->gram_tc)
    check_cuda(cudaFuncSetAttribute(gramtc::k_b_gram_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    gramtc::kSmemBytes),
               "tensor-core Gram attr");
  check_cuda(cudaFuncSetAttribute(k_b_observe, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)(sizeof(double2) * kBMaxK * kBMaxK)),
             "observe attr");

  const bool use_graph = cfg.use_graph != 0;
  if (use_graph) {
    // one eager step sets every kernel attribute before capture
    record_step(Bh, B, L, st);
    free_graph(Bh);
    check_cuda(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal), "begin capture");
    record_step(Bh, B, L, st);
    check_cuda(cudaStreamEndCapture(st, &Bh->graph), "end capture");
    check_cuda(cudaGraphInstantiate(&Bh->exec, Bh->graph, 0), "graph instantiate");
  }
  int active = ntraj;
  long long replays = use_graph ? 1 : 0;  // the eager warm-up step above
  Bh->kernel_launches += 2 + (use_graph ? Bh->launches_per_step : 0);
  const long long max_replays = cfg.max_steps > 0 ? cfg.max_steps : 10000000LL;
  while (active > 0) {
    for (int r = 0; r < 4; ++r) {
      if (use_graph) check_cuda(cudaGraphLaunch(Bh->exec, st), "graph launch");
      else record_step(Bh, B, L, st);
      ++replays;
      Bh->kernel_launches += Bh->launches_per_step;
    }
    int kstatus = 0;
    check_cuda(cudaMemcpyAsync(&active, base + L.active, sizeof(int), cudaMemcpyDeviceToHost, st), "poll");
    check_cuda(cudaMemcpyAsync(&kstatus, base + L.kstatus, sizeof(int), cudaMemcpyDeviceToHost, st), "poll");
    check_cuda(cudaStreamSynchronize(st), "poll sync");
    if (kstatus) fail(RPM_E_TIMEOUT, "persistent Lanczos or tensor-core Gram kernel: a device wait gave up (time limit)");
    if (active == ntraj) {
      float ms = 0.f;
      if (cudaEventElapsedTime(&ms, Bh->probe0, Bh->probe1) == cudaSuccess) {
        Bh->probe_ms_sum += ms;
        ++Bh->probe_samples;
      } else {
        cudaGetLastError();
      }
    }
    if (replays > max_replays) fail(RPM_E_NUMERIC, "batched propagation exceeded the step limit");
  }
  Bh->replays += replays;
  std::vector<TrajState> host(ntraj);
  check_cuda(cudaMemcpyAsync(host.data(), B.st, sizeof(TrajState) * ntraj, cudaMemcpyDeviceToHost, st), "stats");
  check_cuda(cudaStreamSynchronize(st), "stats sync");
  check_cuda(cudaEventRecord(Bh->ev_out, st), "record exit event");
  check_cuda(cudaStreamWaitEvent(caller, Bh->ev_out, 0), "wait exit event");
  for (int b = 0; b < ntraj; ++b) {
    rpm_batch_stats& o = stats[b];
    o.accepted_steps = host[b].steps;
    o.rejected_steps = 0;
    o.matvecs = host[b].matvecs;
    o.maximum_krylov_dimension = host[b].mcap;
    o.minimum_step_us = host[b].steps ? host[b].min_step : 0.0;
    o.maximum_step_us = host[b].max_step;
    o.accumulated_state_error = host[b].acc_err;
    o.maximum_norm_error = host[b].max_norm_err;
    o.status = host[b].status;
  }
}

// Frees everything a batch owns (also a partly created one) and the batch.
static void release_batch(rpm_batch* batch) {
  free_graph(batch);
  if (batch->work) cudaStreamSynchronize(batch->work);
  if (batch->side) cudaStreamSynchronize(batch->side);
  if (batch->buf) cudaFree(batch->buf);
  if (batch->views_dev) cudaFree(batch->views_dev);
  if (batch->ev_fork) cudaEventDestroy(batch->ev_fork);
  if (batch->ev_join) cudaEventDestroy(batch->ev_join);
  if (batch->side) cudaStreamDestroy(batch->side);
  if (batch->ev_in) cudaEventDestroy(batch->ev_in);
  if (batch->ev_out) cudaEventDestroy(batch->ev_out);
  if (batch->probe0) cudaEventDestroy(batch->probe0);
  if (batch->probe1) cudaEventDestroy(batch->probe1);
  if (batch->work) cudaStreamDestroy(batch->work);
  delete batch;
}

}  // namespace rpm

using namespace rpm;

extern "C" {

int rpm_set_gram_kernel(int kernel) {
  return rpm::guarded([&] {
    if (kernel != 0 && kernel != 1) rpm::fail(RPM_E_INVALID, "Gram kernel must be 0 (CUDA cores) or 1 (tensor cores)");
    rpm::g_gram_kernel.store(kernel, std::memory_order_relaxed);
  });
}

int rpm_batch_create(rpm_system* const* systems, int nsys, const rpm_batch_config* cfg, rpm_batch** out) {
  return guarded([&] {
    if (!out || !systems || nsys < 1 || !cfg) fail(RPM_E_INVALID, "bad arguments");
    *out = nullptr;
    if (cfg->krylov_dim < 2 || cfg->krylov_dim > kBMaxK) fail(RPM_E_UNSUPPORTED, "batched Krylov dimension must be in [2, 64]");
    if (cfg->embedded_offset < 1 || cfg->embedded_offset >= cfg->krylov_dim)
      fail(RPM_E_INVALID, "embedded offset must be in [1, krylov_dim)");
    if (!(cfg->state_error_budget > 0.0) || !(cfg->maximum_step_us > 0.0)) fail(RPM_E_INVALID, "bad step controls");
    std::unique_ptr<rpm_batch, void (*)(rpm_batch*)> B(new rpm_batch(), release_batch);
    B->cfg = *cfg;
    std::vector<CubeView<float2>> views;
    for (int k = 0; k < nsys; ++k) {
      rpm_system* s = systems[k];
      if (!s || !s->on_device) fail(RPM_E_INVALID, "every system must be on the device");
      if (!s->cube) fail(RPM_E_UNSUPPORTED, "the batched path needs the radical-split cube form");
      if (s->ndims < 2 || s->dims[0] != 2 || s->dims[1] != 2)
        fail(RPM_E_INVALID, "The first two axes must be the two electron spins.");
      if (s->cube64.inner_l < 1 || s->cube64.inner_r < 1)
        fail(RPM_E_UNSUPPORTED, "cube kernels need a trailing spin-1/2 digit per radical");
      B->systems.push_back(s);
      views.push_back(s->cube32);
      B->ld = std::max(B->ld, s->n);
      B->max_nl = std::max(B->max_nl, s->nl);
      B->max_half_r = std::max(B->max_half_r, s->half_r);
    }
    B->ld = (B->ld + 63) & ~63LL;
    check_cuda(cudaStreamCreateWithFlags(&B->work, cudaStreamNonBlocking), "create batch stream");
    check_cuda(cudaEventCreateWithFlags(&B->ev_in, cudaEventDisableTiming), "create event");
    check_cuda(cudaEventCreateWithFlags(&B->ev_out, cudaEventDisableTiming), "create event");
    check_cuda(cudaStreamCreateWithFlags(&B->side, cudaStreamNonBlocking), "create batch stream");
    check_cuda(cudaEventCreateWithFlags(&B->ev_fork, cudaEventDisableTiming), "create event");
    check_cuda(cudaEventCreateWithFlags(&B->ev_join, cudaEventDisableTiming), "create event");
    check_cuda(cudaEventCreate(&B->probe0), "create probe event");
    check_cuda(cudaEventCreate(&B->probe1), "create probe event");
    check_cuda(cudaMalloc(&B->views_dev, sizeof(CubeView<float2>) * nsys), "cudaMalloc(views)");
    check_cuda(cudaMemcpy(B->views_dev, views.data(), sizeof(CubeView<float2>) * nsys, cudaMemcpyHostToDevice),
               "copy views");
    *out = B.release();
  });
}

int rpm_batch_leading_dimension(const rpm_batch* batch, long long* ld) {
  return guarded([&] {
    if (!batch || !ld) fail(RPM_E_INVALID, "bad arguments");
    *ld = batch->ld;
  });
}

int rpm_batch_propagate(rpm_batch* batch, int ntraj, const int* sys_of_host, void* psi_dev, const double* times_host,
                        int ntimes, double* values_dev, double* state_errors_dev, rpm_batch_stats* stats_host,
                        void* stream) {
  return guarded([&] {
    if (!batch || !sys_of_host || !psi_dev || !times_host || !values_dev || !state_errors_dev || !stats_host)
      fail(RPM_E_INVALID, "NULL argument");
    run_batch(batch, ntraj, sys_of_host, psi_dev, times_host, ntimes, values_dev, state_errors_dev, stats_host,
              static_cast<cudaStream_t>(stream));
  });
}

int rpm_batch_counters(rpm_batch* batch, int reset, long long* kernel_launches, long long* step_replays,
                       double* hpsi_ms_mean, long long* hpsi_samples) {
  return guarded([&] {
    if (!batch) fail(RPM_E_INVALID, "batch is NULL");
    if (kernel_launches) *kernel_launches = batch->kernel_launches;
    if (step_replays) *step_replays = batch->replays;
    if (hpsi_ms_mean)
      *hpsi_ms_mean = batch->probe_samples ? batch->probe_ms_sum / batch->probe_samples / batch->probe_iters : 0.0;
    if (hpsi_samples) *hpsi_samples = batch->probe_samples;
    if (reset) {
      batch->kernel_launches = batch->replays = batch->probe_samples = 0;
      batch->probe_ms_sum = 0.0;
    }
  });
}

int rpm_batch_lanczos_kind(const rpm_batch* batch, int* kind) {
  return guarded([&] {
    if (!batch || !kind) fail(RPM_E_INVALID, "bad arguments");
    *kind = batch->persistent ? 0 : batch->fused ? 1 : 2;
  });
}

int rpm_batch_set_krylov_caps(rpm_batch* batch, const int* caps, int nsys) {
  return guarded([&] {
    if (!batch) fail(RPM_E_INVALID, "batch is NULL");
    if (nsys == 0 || !caps) {
      batch->caps.clear();
      return;
    }
    if (nsys != (int)batch->systems.size()) fail(RPM_E_INVALID, "one Krylov cap per system of the batch is required");
    for (int k = 0; k < nsys; ++k)
      if (caps[k] != 0 && (caps[k] < 2 || caps[k] > batch->cfg.krylov_dim))
        fail(RPM_E_INVALID, "Krylov caps must be 0 or in [2, krylov_dim]");
    batch->caps.assign(caps, caps + nsys);
  });
}

int rpm_batch_set_budget(rpm_batch* batch, double state_error_budget) {
  return guarded([&] {
    if (!batch) fail(RPM_E_INVALID, "batch is NULL");
    if (!(state_error_budget > 0.0)) fail(RPM_E_INVALID, "the state-error budget must be positive");
    batch->cfg.state_error_budget = state_error_budget;
  });
}

int rpm_batch_destroy(rpm_batch* batch) {
  return guarded([&] {
    if (!batch) return;
    release_batch(batch);
  });
}

}  // extern "C"
