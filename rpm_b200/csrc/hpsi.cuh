// Launch interface of the H psi kernels (hpsi.cu), shared with batched.cu.
#pragma once

#include "common.cuh"

namespace rpm {

// Fused Lanczos recurrence of the shape-specialised complex64 passes (off
// when `on` is 0).  Iteration j of vector b, in Paige's ordering:
//   pass R stages v_j = (w'_j - alpha_{j-1} v_{j-1}) * in_scale (j > 0) from
//          `in` (holding w'_j) and `prev`, and writes v_j back into `in`;
//   pass R also subtracts beta_{j-1} v_{j-1} from its partial;
//   pass L writes w'_{j+1} = H v_j - beta_{j-1} v_{j-1} into `out` (not for
//          the last iteration) and reduces <v_j, w'>, |w'|^2 and |v_j|^2;
//          its last block sets alpha_j = <v_j, w'> / |v_j|^2 and
//          beta_j = |w' - alpha_j v_j|, scale = 1 / beta_j, and flags a
//          breakdown (beta_j <= breakdown_rel (|alpha_j| + beta_{j-1})).
// Per-vector scalars of vector b live at ptr + b * dstride (doubles) or
// ptr + b * istride (ints).
// on == 2 (Arnoldi): pass R only scales (v_j = in * in_scale, written back,
// no v_{j-1} term) and pass L stores H v_j unchanged, without reductions.
struct LanczosFuse {
  int on, first, last, j;
  const float2* prev;  // v_{j-1} of vector b at prev + b * ld (unused when first)
  const double* alpha_prev;
  const double* beta_prev;
  double* alpha_out;
  double* beta_out;
  double* scale_out;
  int* stop;
  int* skip;
  int* msize;
  int dstride, istride;
  double breakdown_rel;
};

// Arguments of one batched H psi launch.  Vector b of the batch is read from
// in + b*ld and written to out + b*ld; everything else is optional.
template <class T>
struct HpsiArgs {
  const T* in;
  T* out;
  long long ld;
  long long ya_ld;  // stride of the pass-L scratch per vector (0: same as ld)
  const double* in_scale;  // input multiplier of vector b at in_scale[b*scale_stride]
  int scale_stride;
  const int* skip;         // vector b untouched when skip[b*skip_stride] != 0
  int skip_stride;
  const CubeView<T>* views;  // device array of system views
  const int* sys_of;         // view index of vector b (NULL: view 0)
  // fused <in_scaled, H in_scaled> of vector b into dot_out[b*dot_stride]
  double* dot_out;
  int dot_stride;
  double* dot_part;     // gridDim.x partials per vector (three per block with `lz`)
  unsigned* dot_count;  // one completion counter per vector (zero on entry)
  LanczosFuse lz;       // complex64 shape-specialised passes only
};

// Shape limits of one launch over one or more systems.
struct CubePlan {
  int nl, nr, half_r, tab_cap;
  int ni_l, ni_r;  // inner digits used per side
  int n_outer_l1, n_outer_l2, n_outer_r1, n_outer_r2;  // outer-index counts for NI = 1, 2
  // shape-specialised complex64 passes (hpsi_fast.cu): usable when every
  // system of the launch has the standard axis order and the same digit
  // pattern (spin-1 count, spin-1/2 count) per radical
  int fast;
  int fl_n1, fl_nh, fr_n1, fr_nh, f_half_l, f_half_r;
};

int sm_count();
// Same dimensions, digit pattern and layout (offset tables) of the two radicals.
bool same_cube_shape(const rpm_system* x, const rpm_system* y);
// Launch plan over systems of ONE shape (fails with RPM_E_UNSUPPORTED otherwise).
CubePlan cube_plan(rpm_system* const* systems, int nsys);
void fast_plan_add(CubePlan& p, const rpm_system* s, bool first);
// Launches the specialised passes; false (nothing launched) when the plan or
// the pointers/strides (16-byte alignment) do not allow them.
template <class T>
bool launch_cube_fast(const HpsiArgs<T>& a, const CubePlan& p, T* ya, int batch, cudaStream_t stream);
template <class T>
bool cube_fast_usable(const HpsiArgs<T>& a, const CubePlan& p, const T* ya);
// Two passes: pass L into `ya` (batch x ld scratch), pass R into a.out.
template <class T>
void launch_cube(const HpsiArgs<T>& a, const CubePlan& p, T* ya, int batch, cudaStream_t stream);
// out = H (in * scale_dev[0]) for `batch` vectors of one Hermitian cube-form
// system (every vector uses the same device scale).
template <class T>
void launch_hpsi_scaled(rpm_system* sys, const T* in, T* out, int batch, long long ld, const double* scale_dev,
                        cudaStream_t stream);

}  // namespace rpm
