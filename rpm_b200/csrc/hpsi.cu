// H psi kernels for sm_100a.
//
// Two forms, both exact re-designs of the reference's matrix-free action:
//
// * Generic per-term mode product (rpm_statevector_engine.py:95-108): every
//   thread owns output elements and applies each local term as a strided
//   gather of its d neighbours along the term's axes.
//
// * Radical split (rpm_statevector_engine.py:221-245): the state is viewed as
//   Psi[l, r] with l over (electron A, FAD nuclei) and r over (electron B,
//   TrpH nuclei).  Two shared-memory-tiled passes:
//     pass A: a tile of all l rows x 2*TR columns (both electron-B halves of
//             TR right indices) -> L Psi + pair-term, written to `ya`;
//     pass B: a tile of TL rows x all r columns -> Psi R^T, added to `ya`.
//   Operator values are read warp-uniformly (one row of L per warp, one row
//   of R per warp step), and pass B pads the shared row stride to an odd
//   number of elements so lanes on different rows hit different banks.
#include <algorithm>

#include "common.cuh"

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
// Radical split, pass A: L Psi + pair term over a tile of all rows.
//   grid: x = column tiles (TR right indices of each electron half),
//         y = vector in batch, z = row slices (each CTA loads the whole tile
//         but computes rows [z*nl/Z, (z+1)*nl/Z)).
// ---------------------------------------------------------------------------
template <class T, int TR>
__global__ void __launch_bounds__(512) split_pass_a(SplitView<T> s, const T* __restrict__ in,
                                                    T* __restrict__ ya, long long ld) {
  constexpr int W = 2 * TR;
  extern __shared__ unsigned char smem_raw[];
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
  const int rows_per = (s.nl + gridDim.z - 1) / gridDim.z;
  const int l_begin = blockIdx.z * rows_per;
  const int l_end = min(s.nl, l_begin + rows_per);
  const int cc = threadIdx.x % W;
  const int h = cc / TR;
  const int j = r0 + (cc % TR);
  if (j >= s.half_r) return;  // no barrier below
  const int offr_c = __ldg(s.offr + h * s.half_r + j);
  for (int l = l_begin + threadIdx.x / W; l < l_end; l += blockDim.x / W) {
    T acc = czero<T>();
    const int k1 = __ldg(s.lptr + l + 1);
    for (int k = __ldg(s.lptr + l); k < k1; ++k) acc = cfma(__ldg(s.lval + k), tile[__ldg(s.lcol + k) * W + cc], acc);
    const int a = l >= s.half_l ? 1 : 0;
    const int lb = l - a * s.half_l;
    const int cb = cc - h * TR;
#pragma unroll
    for (int a2 = 0; a2 < 2; ++a2) {
#pragma unroll
      for (int b2 = 0; b2 < 2; ++b2) {
        acc = cfma(pair[(a * 2 + h) * 4 + a2 * 2 + b2], tile[(lb + a2 * s.half_l) * W + cb + b2 * TR], acc);
      }
    }
    y[__ldg(s.offl + l) + offr_c] = acc;
  }
}

// ---------------------------------------------------------------------------
// Radical split, pass B: out = ya + Psi R^T over tiles of TL full rows.
//   Lane layout: TL rows x CW columns per warp step (TL * CW == 32).
//   Accumulators stay in registers until the tile has been consumed, then
//   overwrite it in shared memory for a coalesced write-out.
// ---------------------------------------------------------------------------
template <class T, int TL, int MAXACC>
__global__ void __launch_bounds__(512) split_pass_b(SplitView<T> s, const T* __restrict__ in,
                                                    const T* __restrict__ ya, T* __restrict__ out, long long ld) {
  constexpr int CW = 32 / TL;
  extern __shared__ unsigned char smem_raw[];
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
      T a = czero<T>();
      const int k1 = __ldg(s.rptr + r + 1);
      for (int k = __ldg(s.rptr + r); k < k1; ++k) a = cfma(__ldg(s.rval + k), tile[lt * nrp + __ldg(s.rcol + k)], a);
      acc[q] = a;
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
static int sm_count() {
  static int count = 0;
  if (!count) {
    int dev = 0;
    check_cuda(cudaGetDevice(&dev), "cudaGetDevice");
    check_cuda(cudaDeviceGetAttribute(&count, cudaDevAttrMultiProcessorCount, dev), "cudaDeviceGetAttribute");
  }
  return count;
}

static constexpr size_t kMaxSmem = 220 * 1024;

template <class T, int TR>
static bool try_pass_a(const SplitView<T>& s, const T* in, T* ya, int batch, long long ld, cudaStream_t stream) {
  const size_t smem = (16 + (size_t)s.nl * 2 * TR) * sizeof(T);
  if (smem > kMaxSmem) return false;
  auto kern = split_pass_a<T, TR>;
  check_cuda(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
             "cudaFuncSetAttribute(pass A)");
  const int tiles = (s.half_r + TR - 1) / TR;
  // Slice rows when the batch alone does not fill the GPU.
  int z = 1;
  const int ctas = tiles * batch;
  while (ctas * z < 2 * sm_count() && z < 16 && s.nl / (z * 2) >= 32) z *= 2;
  dim3 grid(tiles, batch, z);
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

template <class SV>
static const SV& split_of(rpm_system* sys);
template <>
const SplitView<double2>& split_of<SplitView<double2>>(rpm_system* sys) { return sys->split64; }
template <>
const SplitView<float2>& split_of<SplitView<float2>>(rpm_system* sys) { return sys->split32; }

template <class T>
static const GenericView<T>& generic_of(rpm_system* sys);
template <>
const GenericView<double2>& generic_of<double2>(rpm_system* sys) { return sys->gen64; }
template <>
const GenericView<float2>& generic_of<float2>(rpm_system* sys) { return sys->gen32; }

template <class T>
void launch_hpsi(rpm_system* sys, const T* in, T* out, int batch, long long ld, cudaStream_t stream) {
  if (!sys->on_device) fail(RPM_E_INVALID, "system was created host-only");
  if (batch < 1) return;
  if (sys->split) {
    const SplitView<T>& s = split_of<SplitView<T>>(sys);
    // pass-A partial result lives in the system scratch (batch x ld elements)
    T* ya = static_cast<T*>(system_scratch(sys, SLOT_YA, (size_t)batch * ld * sizeof(T)));
    bool a_ok;
    if (sizeof(T) == 8) {
      a_ok = try_pass_a<T, 8>(s, in, ya, batch, ld, stream) || try_pass_a<T, 4>(s, in, ya, batch, ld, stream) ||
             try_pass_a<T, 2>(s, in, ya, batch, ld, stream);
    } else {
      a_ok = try_pass_a<T, 4>(s, in, ya, batch, ld, stream) || try_pass_a<T, 2>(s, in, ya, batch, ld, stream);
    }
    if (a_ok) {
      bool b_ok;
      if (batch >= 8) {
        b_ok = (sizeof(T) == 8 ? try_pass_b<T, 32, 32>(s, in, ya, out, batch, ld, stream)
                               : try_pass_b<T, 16, 16>(s, in, ya, out, batch, ld, stream)) ||
               try_pass_b<T, 4, 8>(s, in, ya, out, batch, ld, stream);
      } else {
        b_ok = try_pass_b<T, 4, 8>(s, in, ya, out, batch, ld, stream) ||
               try_pass_b<T, 2, 4>(s, in, ya, out, batch, ld, stream);
      }
      if (b_ok) return;
    }
  }
  launch_generic<T>(generic_of<T>(sys), in, out, batch, ld, stream);
}

template void launch_hpsi<double2>(rpm_system*, const double2*, double2*, int, long long, cudaStream_t);
template void launch_hpsi<float2>(rpm_system*, const float2*, float2*, int, long long, cudaStream_t);

}  // namespace rpm

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
