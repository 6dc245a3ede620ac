// Launch interface of the H psi kernels (hpsi.cu), shared with batched.cu.
#pragma once

#include <cuda.h>

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
  const int* mcap;  // Krylov cap of vector b (null: the batch's); the
                    // iteration j = cap - 1 ends the vector's basis
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

// One persistent launch runs the Lanczos iterations j0 <= j < j1 of a Krylov
// step for the trajectories of one shape group on the shape-specialised
// complex64 passes (lanczos_persistent.cu).  Vector b (0-based in the group)
// keeps its basis at V + b * vstride + j * ld, its pass-R partial at
// ya + b * ld and its scalars in the batch's per-trajectory records
// (ptr + b * dstride [+ j] for doubles, ptr + b * istride for ints).
// prog/cnt/part/work/status are device scratch: prog, cnt and *work start at
// zero for every Krylov step (k_b_start), *status at zero for every
// propagation (nonzero: a wait gave up).
struct PersistentLanczos {
  float2* V;
  long long ld, vstride;
  long long slot0;  // tensor-map slot of (vector 0, j = 0): vector b, slot j is slot0 + b (m + 1) + j
  int m, nb, gv;    // Krylov dimension, vectors, vectors per wavefront group
  int j0, j1;       // iterations j0 <= j < j1 of this launch (a segment of 0 .. m-1)
  const CubeView<float2>* views;
  const int* sys_of;
  double* alpha;  // alpha_j of vector b at alpha[b * dstride + j]
  double* beta;
  double* scale;  // 1 / beta_{j-1} of vector b at scale[b * dstride]
  int dstride;
  int* stop;
  int* skip;
  int* msize;
  const int* mcap;  // Krylov cap of vector b at mcap[b * istride]
  int istride;
  double breakdown_rel;
  float2* ya;
  int* prog;       // per vector: phases completed (R of iteration j -> 2j + 1, L -> 2j + 2)
  unsigned* cnt;   // per vector: tiles completed in the current phase
  double* part;    // per vector: [L tile][3] partial sums at part + b * part_stride
  int part_stride;
  unsigned* work;  // dequeue counter of this launch
  int* status;     // sticky wait-timeout flag
  int ctas;        // CTAs of the launch (<= 0: one per SM)
};

// Launches the persistent Lanczos kernel for the plan's shape; false (nothing
// launched) when no persistent instance exists for it.  `V_base` and
// `nslots` describe the whole basis buffer ([nslots][ld] complex64) that the
// tensor map covers.
bool launch_lanczos_persistent(const PersistentLanczos& p, const CubePlan& plan, const float2* V_base,
                               long long nslots, cudaStream_t stream);
// L tiles per vector and iteration of the persistent kernel for a shape (8
// columns per electron-B half each), 0 when the shape has no instance.
int persistent_l_tiles(const CubePlan& plan);
// 2-D tensor map of a basis buffer [nslots][ld] complex64: a box of box_rows
// consecutive elements of box_slots consecutive slots lands as [slot][box_rows].
CUtensorMap basis_rows_map(const float2* V, long long nslots, long long ld, int box_rows, int box_slots);

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
