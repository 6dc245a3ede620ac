// Shared definitions for the librpm_b200 CUDA sources (sm_100a).
#pragma once

#include <cuda_runtime.h>

#include <complex>
#include <cstdint>
#include <cstdio>
#include <new>
#include <string>
#include <vector>

#include "../../include/rpm_b200.h"

namespace rpm {

using cd = std::complex<double>;

// ---------------------------------------------------------------------------
// Error reporting: a thread-local message plus the int status returned by the
// C ABI.  Internal code throws rpm::Error; every extern "C" function catches.
// ---------------------------------------------------------------------------
struct Error {
  int code;
  std::string message;
};

void set_last_error(const std::string& message);
[[noreturn]] void fail(int code, const std::string& message);
void check_cuda(cudaError_t status, const char* what);
void check_launch(const char* what);

// Run `body`, translating rpm::Error / allocation failures into a status code.
template <class F>
int guarded(F&& body) {
  try {
    body();
    return RPM_OK;
  } catch (const Error& e) {
    set_last_error(e.message);
    return e.code;
  } catch (const std::bad_alloc&) {
    set_last_error("host allocation failed");
    return RPM_E_NOMEM;
  } catch (...) {
    set_last_error("unexpected internal error");
    return RPM_E_INVALID;
  }
}

// ---------------------------------------------------------------------------
// Complex helpers (interleaved float2 / double2)
// ---------------------------------------------------------------------------
template <class T> struct Real;
template <> struct Real<float2> { using type = float; };
template <> struct Real<double2> { using type = double; };

__host__ __device__ __forceinline__ float2 cmake(float re, float im) { return make_float2(re, im); }
__host__ __device__ __forceinline__ double2 cmake(double re, double im) { return make_double2(re, im); }

template <class T>
__host__ __device__ __forceinline__ T czero() {
  T z;
  z.x = 0;
  z.y = 0;
  return z;
}

// acc + a * b
__device__ __forceinline__ float2 cfma(float2 a, float2 b, float2 acc) {
  acc.x = fmaf(a.x, b.x, acc.x);
  acc.x = fmaf(-a.y, b.y, acc.x);
  acc.y = fmaf(a.x, b.y, acc.y);
  acc.y = fmaf(a.y, b.x, acc.y);
  return acc;
}
__device__ __forceinline__ double2 cfma(double2 a, double2 b, double2 acc) {
  acc.x = fma(a.x, b.x, acc.x);
  acc.x = fma(-a.y, b.y, acc.x);
  acc.y = fma(a.x, b.y, acc.y);
  acc.y = fma(a.y, b.x, acc.y);
  return acc;
}
// acc + conj(a) * b
__device__ __forceinline__ double2 cfma_conj(double2 a, double2 b, double2 acc) {
  acc.x = fma(a.x, b.x, acc.x);
  acc.x = fma(a.y, b.y, acc.x);
  acc.y = fma(a.x, b.y, acc.y);
  acc.y = fma(-a.y, b.x, acc.y);
  return acc;
}
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 to_d2(float2 a) { return make_double2(a.x, a.y); }
__device__ __forceinline__ double2 to_d2(double2 a) { return a; }
template <class T> __device__ __forceinline__ T from_d2(double2 a);
template <> __device__ __forceinline__ double2 from_d2<double2>(double2 a) { return a; }
template <> __device__ __forceinline__ float2 from_d2<float2>(double2 a) {
  return make_float2((float)a.x, (float)a.y);
}

// ---------------------------------------------------------------------------
// Device view of a radical-split Hamiltonian (see system.cu).
//   state index  i = offl[l] + offr[r]
//   l = a * half_l + (left nuclei),  r = b * half_r + (right nuclei)
//   (H psi)[l, r] = sum_l' L[l, l'] psi[l', r] + sum_r' R[r, r'] psi[l, r']
//                 + sum_{a'b'} P[(a b),(a' b')] psi[l + (a'-a) half_l, r + (b'-b) half_r]
// ---------------------------------------------------------------------------
template <class T>
struct SplitView {
  int nl, nr, half_l, half_r;
  const int* offl;  // nl
  const int* offr;  // nr
  const int* lptr;  // nl + 1
  const int* lcol;
  const T* lval;
  const int* rptr;  // nr + 1
  const int* rcol;
  const T* rval;
  T pair[16];  // row-major over (a b) x (a' b')
};

// Device view of the generic per-term form (used when no split is given).
struct TermMeta {
  int naxes;
  int d;             // local dimension
  int op_offset;     // into the op arrays (complex elements)
  int col_offset;    // into the column-offset table (d entries)
  int stride[RPM_MAX_TERM_AXES];  // tensor stride of each active axis
  int dim[RPM_MAX_TERM_AXES];     // its dimension
  int lstride[RPM_MAX_TERM_AXES]; // stride inside the local index
};

template <class T>
struct GenericView {
  int nterms;
  int n;
  const TermMeta* terms;
  const T* ops;
  const int* coloff;  // for each term: memory offset of local column c relative to the row-zero base
};

// ---------------------------------------------------------------------------
// "Cube" form of one radical group (see hpsi.cu).  The group index is
//   g = e * half + sum_k n_k * gs[k]      (e: electron digit, n_k: nuclei)
// and every group term acts on {e}, {n_k} or {e, n_k}.  Per nucleus k the
// combined 2d x 2d block O_k on (e, n_k) is split into
//   D_k[e][m]            = Re O_k[(e,m),(e,m)]          (merged diagonal)
//   F_k[e][m]            = O_k[(e,m),(1-e,m)]           (merged electron flip)
//   X_k[(e,m),(e',m')]   = O_k[(e,m),(e',m')], m' != m  (nuclear transitions)
// The electron-only operator Z adds Zd[e] = Re Z[e][e] and Zf[e] = Z[e][1-e].
// Table layout (complex entries): [Zd0, Zd1, Zf0, Zf1], then per nucleus
// D (2d), F (2d), X ((2d)^2) at offD/offF/offX.
// ---------------------------------------------------------------------------
constexpr int kCubeMaxDigits = 16;
constexpr int kCubeMaxTable = 2048;

struct CubeSide {
  int K;        // nuclear digits in the group
  int half;     // group size / 2 (electron stride)
  int n_outer;  // product of the dims of the outer digits (all but the last NI)
  int ntab;     // table length in complex entries
  int dim[kCubeMaxDigits];
  int gs[kCubeMaxDigits];
  int offD[kCubeMaxDigits], offF[kCubeMaxDigits], offX[kCubeMaxDigits];
};

// Coefficient storage of the cube tables (same precision as the state).
template <class T> struct CubeCoef { using type = T; };

template <class T>
struct CubeView {
  CubeSide L, R;
  const typename CubeCoef<T>::type* tabL;
  const typename CubeCoef<T>::type* tabR;
  T pair[16];  // (a b) x (a' b') electron-pair operator
  const int* offl;
  const int* offr;
  int nl, nr, half_l, half_r;
  int inner_l, inner_r;  // usable trailing spin-1/2 digits per side
  // complex64 views of shapes with shape-specialised passes: per outer index
  // the merged diagonal / electron-flip records of pass R (outer digits
  // 0..K-3 of the right radical) and pass L (0..K-4 of the left), laid out as
  // {float d[2]; float2 f[2]} (24 bytes) and padded to 16 bytes, the pass-L
  // records followed by the 16 float2 of the pair operator; else null
  const void* orecR;
  const void* orecL;
  int orec_bytes_r, orec_bytes_l;
};

}  // namespace rpm

// The opaque system object of the C ABI.
struct rpm_system {
  int ndims = 0;
  int dims[RPM_MAX_AXES] = {};
  long long n = 0;
  bool split = false;
  bool on_device = false;
  int device = -1;

  // host tables -------------------------------------------------------------
  int nl = 0, nr = 0, half_l = 0, half_r = 0;
  std::vector<long long> offl, offr;
  std::vector<int> lptr, lcol, rptr, rcol;
  std::vector<rpm::cd> lval, rval;
  rpm::cd pair[16];
  // Haberkorn recombination with unequal rates (rpm_system_set_recombination):
  // pair = pair_base - (i/2) |kS - kT| Q, Q = P_S (kS > kT) or P_T (kT > kS);
  // the common decay exp(-min(kS, kT) t / 2) of the state is factored out.
  rpm::cd pair_base[16];
  bool recombination = false;
  bool non_hermitian = false;
  double rate_singlet = 0.0, rate_triplet = 0.0;
  std::vector<rpm::TermMeta> terms;
  std::vector<rpm::cd> ops;
  std::vector<int> coloff;

  // device copies -----------------------------------------------------------
  rpm::SplitView<double2> split64{};
  rpm::SplitView<float2> split32{};
  rpm::GenericView<double2> gen64{};
  rpm::GenericView<float2> gen32{};
  // cube form (valid when `cube` is true)
  bool cube = false;
  rpm::CubeSide cube_l{}, cube_r{};
  std::vector<rpm::cd> cube_tab_l, cube_tab_r;
  rpm::CubeView<double2> cube64{};
  rpm::CubeView<float2> cube32{};
  rpm::CubeView<double2>* cube64_dev = nullptr;  // device copy of cube64
  rpm::CubeView<float2>* cube32_dev = nullptr;
  std::vector<void*> allocations;

  // scratch buffers, one per slot, grown on demand (cudaMalloc'd) ---------
  void* scratch[8] = {};
  size_t scratch_bytes[8] = {};
};

namespace rpm {
// Scratch slots of a system.  Each slot is a grow-only device buffer, zeroed
// when (re)allocated and freed by rpm_system_destroy.
enum Slot : int {
  SLOT_YA = 0,        // pass-A partial of the radical-split H psi
  SLOT_REDUCE = 1,    // block partials + completion counters of reductions
  SLOT_WORK = 2,      // Lanczos work vector
  SLOT_SMALL = 3,     // small device scalars (alpha, beta, h coefficients, flags)
  SLOT_GRAM = 4,      // Gram partials
};
void* system_scratch(rpm_system* sys, int slot, size_t bytes);
// H psi launchers (hpsi.cu).  `scale_dev`, when non-null, multiplies the input
// by 1/scale_dev[0] on load (used to fold normalisation into H psi).
template <class T>
void launch_hpsi(rpm_system* sys, const T* in, T* out, int batch, long long ld, cudaStream_t stream);
}  // namespace rpm
