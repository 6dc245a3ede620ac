// System construction: validation of local terms, the radical-split CSR tables
// and the generic per-term tables, and their upload to the device.
//
// Follows rpm_statevector_engine.py:46-93 (term checks) and :142-219 (radical
// split), re-designed as host-built CSR + offset tables consumed by the
// sm_100a H psi kernels in hpsi.cu.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <numeric>
#include <set>

#include "common.cuh"

namespace rpm {

static thread_local std::string g_last_error;

void set_last_error(const std::string& message) { g_last_error = message; }

void fail(int code, const std::string& message) { throw Error{code, message}; }

void check_cuda(cudaError_t status, const char* what) {
  if (status != cudaSuccess) {
    fail(RPM_E_CUDA, std::string(what) + ": " + cudaGetErrorString(status));
  }
}

void check_launch(const char* what) { check_cuda(cudaGetLastError(), what); }

void* system_scratch(rpm_system* sys, int slot, size_t bytes) {
  if (slot < 0 || slot >= 8) fail(RPM_E_INVALID, "bad scratch slot");
  if (bytes <= sys->scratch_bytes[slot]) return sys->scratch[slot];
  if (sys->scratch[slot]) {
    // cudaFree waits for work in flight that may still use the old buffer
    check_cuda(cudaFree(sys->scratch[slot]), "cudaFree(scratch)");
    sys->scratch[slot] = nullptr;
    sys->scratch_bytes[slot] = 0;
  }
  size_t grown = std::max(bytes, (size_t)1 << 16);
  check_cuda(cudaMalloc(&sys->scratch[slot], grown), "cudaMalloc(scratch)");
  check_cuda(cudaMemset(sys->scratch[slot], 0, grown), "cudaMemset(scratch)");
  sys->scratch_bytes[slot] = grown;
  return sys->scratch[slot];
}

// Row-major tensor strides.
static std::vector<long long> tensor_strides(const int* dims, int ndims) {
  std::vector<long long> s(ndims, 1);
  for (int a = ndims - 2; a >= 0; --a) s[a] = s[a + 1] * dims[a + 1];
  return s;
}

// Sparse accumulation of the operator restricted to one axis group.  `group`
// lists tensor axes in the group's own (row-major) digit order; each term is
// given by its positions inside the group.
struct GroupTerm {
  std::vector<int> pos;  // positions in the group
  const cd* op;
  int d;
};

static void build_group_csr(const std::vector<int>& gdims, const std::vector<GroupTerm>& gterms,
                            std::vector<int>& ptr, std::vector<int>& col, std::vector<cd>& val) {
  const int ng = (int)gdims.size();
  long long size = 1;
  for (int v : gdims) size *= v;
  std::vector<long long> gstride(ng, 1);
  for (int p = ng - 2; p >= 0; --p) gstride[p] = gstride[p + 1] * gdims[p + 1];
  ptr.assign(size + 1, 0);
  col.clear();
  val.clear();
  std::vector<std::pair<int, cd>> row;
  std::vector<int> digit(ng);
  for (long long g = 0; g < size; ++g) {
    row.clear();
    long long rem = g;
    for (int p = 0; p < ng; ++p) {
      digit[p] = (int)(rem / gstride[p]);
      rem %= gstride[p];
    }
    for (const GroupTerm& t : gterms) {
      const int k = (int)t.pos.size();
      // local row index and the base index with the active digits cleared
      int lrow = 0;
      long long base = g;
      for (int q = 0; q < k; ++q) {
        lrow = lrow * gdims[t.pos[q]] + digit[t.pos[q]];
        base -= (long long)digit[t.pos[q]] * gstride[t.pos[q]];
      }
      for (int c = 0; c < t.d; ++c) {
        cd v = t.op[(size_t)lrow * t.d + c];
        if (v == cd(0.0, 0.0)) continue;
        long long target = base;
        int cc = c;
        for (int q = k - 1; q >= 0; --q) {
          const int dq = gdims[t.pos[q]];
          target += (long long)(cc % dq) * gstride[t.pos[q]];
          cc /= dq;
        }
        row.emplace_back((int)target, v);
      }
    }
    std::sort(row.begin(), row.end(), [](const auto& x, const auto& y) { return x.first < y.first; });
    for (size_t i = 0; i < row.size();) {
      size_t j = i;
      cd sum = 0.0;
      while (j < row.size() && row[j].first == row[i].first) sum += row[j++].second;
      if (sum != cd(0.0, 0.0)) {
        col.push_back(row[i].first);
        val.push_back(sum);
      }
      i = j;
    }
    ptr[g + 1] = (int)col.size();
  }
}

// Cube tables of one radical group (see CubeSide in common.cuh).  Returns
// false when a group term acts on anything but {e}, {n_k} or {e, n_k}.
static bool build_cube_side(const std::vector<int>& gdims, const std::vector<GroupTerm>& gterms, CubeSide& side,
                            std::vector<cd>& tab, int& inner) {
  const int K = (int)gdims.size() - 1;
  if (K < 1 || K > kCubeMaxDigits || gdims[0] != 2) return false;
  side = CubeSide{};
  side.K = K;
  long long stride = 1;
  for (int k = K - 1; k >= 0; --k) {
    side.dim[k] = gdims[k + 1];
    side.gs[k] = (int)stride;
    stride *= gdims[k + 1];
  }
  side.half = (int)stride;
  cd Z[2][2] = {};
  std::vector<std::vector<cd>> O(K);
  for (int k = 0; k < K; ++k) O[k].assign((size_t)4 * side.dim[k] * side.dim[k], 0.0);
  for (const GroupTerm& t : gterms) {
    if (t.pos.size() == 1 && t.pos[0] == 0) {
      for (int a = 0; a < 2; ++a)
        for (int b = 0; b < 2; ++b) Z[a][b] += t.op[a * 2 + b];
    } else if (t.pos.size() == 1) {
      const int k = t.pos[0] - 1, d = side.dim[k];
      for (int e = 0; e < 2; ++e)
        for (int m = 0; m < d; ++m)
          for (int mp = 0; mp < d; ++mp) O[k][(size_t)(e * d + m) * 2 * d + e * d + mp] += t.op[m * d + mp];
    } else if (t.pos.size() == 2 && (t.pos[0] == 0 || t.pos[1] == 0)) {
      const bool e_first = t.pos[0] == 0;
      const int k = (e_first ? t.pos[1] : t.pos[0]) - 1, d = side.dim[k];
      for (int e = 0; e < 2; ++e)
        for (int m = 0; m < d; ++m)
          for (int ep = 0; ep < 2; ++ep)
            for (int mp = 0; mp < d; ++mp) {
              const int row = e_first ? e * d + m : m * 2 + e;
              const int col = e_first ? ep * d + mp : mp * 2 + ep;
              O[k][(size_t)(e * d + m) * 2 * d + ep * d + mp] += t.op[(size_t)row * 2 * d + col];
            }
    } else {
      return false;
    }
  }
  tab.assign(4, 0.0);
  tab[0] = Z[0][0].real();
  tab[1] = Z[1][1].real();
  tab[2] = Z[0][1];
  tab[3] = Z[1][0];
  for (int k = 0; k < K; ++k) {
    const int d = side.dim[k];
    side.offD[k] = (int)tab.size();
    for (int e = 0; e < 2; ++e)
      for (int m = 0; m < d; ++m) tab.push_back(O[k][(size_t)(e * d + m) * 2 * d + e * d + m].real());
    side.offF[k] = (int)tab.size();
    for (int e = 0; e < 2; ++e)
      for (int m = 0; m < d; ++m) tab.push_back(O[k][(size_t)(e * d + m) * 2 * d + (1 - e) * d + m]);
    side.offX[k] = (int)tab.size();
    tab.insert(tab.end(), O[k].begin(), O[k].end());
  }
  side.ntab = (int)tab.size();
  if (side.ntab > kCubeMaxTable) return false;
  inner = 0;
  while (inner < K && side.dim[K - 1 - inner] == 2) ++inner;
  return true;
}

template <class T>
static T* upload(rpm_system* sys, const void* src, size_t bytes) {
  void* p = nullptr;
  if (bytes == 0) bytes = 16;
  check_cuda(cudaMalloc(&p, bytes), "cudaMalloc(system table)");
  sys->allocations.push_back(p);
  if (src) check_cuda(cudaMemcpy(p, src, bytes, cudaMemcpyHostToDevice), "cudaMemcpy(system table)");
  return static_cast<T*>(p);
}

// Outer-index records of the shape-specialised passes (see CubeView): for
// outer index o the electron-only diagonal / flip entries plus those of the
// outer digits k < nout, digit value (o / (gs[k] / div)) % dim[k], summed in
// FP32 in digit order (the order the passes' own record builder uses).
static std::vector<float> outer_records(const CubeSide& side, const std::vector<float2>& tab, int nout, int div) {
  const int no = side.half / div;
  std::vector<float> out((size_t)no * 6 + 2, 0.0f);  // + padding to 16 bytes when no is odd
  for (int o = 0; o < no; ++o) {
    float d[2] = {tab[0].x, tab[1].x};
    float2 f[2] = {tab[2], tab[3]};
    for (int k = 0; k < nout; ++k) {
      const int m = (o / (side.gs[k] / div)) % side.dim[k];
      for (int e = 0; e < 2; ++e) {
        d[e] += tab[side.offD[k] + e * side.dim[k] + m].x;
        const float2 g = tab[side.offF[k] + e * side.dim[k] + m];
        f[e].x += g.x;
        f[e].y += g.y;
      }
    }
    float* r = out.data() + (size_t)o * 6;
    r[0] = d[0];
    r[1] = d[1];
    r[2] = f[0].x;
    r[3] = f[0].y;
    r[4] = f[1].x;
    r[5] = f[1].y;
  }
  out.resize(((size_t)no * 24 + 15) / 16 * 4);
  return out;
}

static std::vector<double2> to_d2(const std::vector<cd>& v) {
  std::vector<double2> out(v.size());
  for (size_t i = 0; i < v.size(); ++i) out[i] = make_double2(v[i].real(), v[i].imag());
  return out;
}
static std::vector<float2> to_f2(const std::vector<cd>& v) {
  std::vector<float2> out(v.size());
  for (size_t i = 0; i < v.size(); ++i) out[i] = make_float2((float)v[i].real(), (float)v[i].imag());
  return out;
}

static void upload_system(rpm_system* sys) {
  check_cuda(cudaGetDevice(&sys->device), "cudaGetDevice");
  // generic per-term tables (always present)
  {
    auto* terms = upload<TermMeta>(sys, sys->terms.data(), sys->terms.size() * sizeof(TermMeta));
    auto ops64 = to_d2(sys->ops);
    auto ops32 = to_f2(sys->ops);
    auto* o64 = upload<double2>(sys, ops64.data(), ops64.size() * sizeof(double2));
    auto* o32 = upload<float2>(sys, ops32.data(), ops32.size() * sizeof(float2));
    auto* coff = upload<int>(sys, sys->coloff.data(), sys->coloff.size() * sizeof(int));
    sys->gen64 = GenericView<double2>{(int)sys->terms.size(), (int)sys->n, terms, o64, coff};
    sys->gen32 = GenericView<float2>{(int)sys->terms.size(), (int)sys->n, terms, o32, coff};
  }
  if (sys->split) {
    std::vector<int> offl(sys->offl.begin(), sys->offl.end()), offr(sys->offr.begin(), sys->offr.end());
    const int* d_offl = upload<int>(sys, offl.data(), offl.size() * sizeof(int));
    const int* d_offr = upload<int>(sys, offr.data(), offr.size() * sizeof(int));
    const int* d_lptr = upload<int>(sys, sys->lptr.data(), sys->lptr.size() * sizeof(int));
    const int* d_lcol = upload<int>(sys, sys->lcol.data(), sys->lcol.size() * sizeof(int));
    const int* d_rptr = upload<int>(sys, sys->rptr.data(), sys->rptr.size() * sizeof(int));
    const int* d_rcol = upload<int>(sys, sys->rcol.data(), sys->rcol.size() * sizeof(int));
    auto l64 = to_d2(sys->lval), r64 = to_d2(sys->rval);
    auto l32 = to_f2(sys->lval), r32 = to_f2(sys->rval);
    SplitView<double2> s64{};
    SplitView<float2> s32{};
    s64.nl = s32.nl = sys->nl;
    s64.nr = s32.nr = sys->nr;
    s64.half_l = s32.half_l = sys->half_l;
    s64.half_r = s32.half_r = sys->half_r;
    s64.offl = s32.offl = d_offl;
    s64.offr = s32.offr = d_offr;
    s64.lptr = s32.lptr = d_lptr;
    s64.lcol = s32.lcol = d_lcol;
    s64.rptr = s32.rptr = d_rptr;
    s64.rcol = s32.rcol = d_rcol;
    s64.lval = upload<double2>(sys, l64.data(), l64.size() * sizeof(double2));
    s64.rval = upload<double2>(sys, r64.data(), r64.size() * sizeof(double2));
    s32.lval = upload<float2>(sys, l32.data(), l32.size() * sizeof(float2));
    s32.rval = upload<float2>(sys, r32.data(), r32.size() * sizeof(float2));
    for (int k = 0; k < 16; ++k) {
      s64.pair[k] = make_double2(sys->pair[k].real(), sys->pair[k].imag());
      s32.pair[k] = make_float2((float)sys->pair[k].real(), (float)sys->pair[k].imag());
    }
    sys->split64 = s64;
    sys->split32 = s32;
    if (sys->cube) {
      auto tl64 = to_d2(sys->cube_tab_l), tr64 = to_d2(sys->cube_tab_r);
      auto tl32 = to_f2(sys->cube_tab_l), tr32 = to_f2(sys->cube_tab_r);
      CubeView<double2>& c64 = sys->cube64;
      CubeView<float2>& c32 = sys->cube32;
      c64.L = c32.L = sys->cube_l;
      c64.R = c32.R = sys->cube_r;
      c64.tabL = upload<double2>(sys, tl64.data(), tl64.size() * sizeof(double2));
      c64.tabR = upload<double2>(sys, tr64.data(), tr64.size() * sizeof(double2));
      c32.tabL = upload<float2>(sys, tl32.data(), tl32.size() * sizeof(float2));
      c32.tabR = upload<float2>(sys, tr32.data(), tr32.size() * sizeof(float2));
      for (int k = 0; k < 16; ++k) {
        c64.pair[k] = s64.pair[k];
        c32.pair[k] = s32.pair[k];
      }
      c64.offl = c32.offl = d_offl;
      c64.offr = c32.offr = d_offr;
      c64.nl = c32.nl = sys->nl;
      c64.nr = c32.nr = sys->nr;
      c64.half_l = c32.half_l = sys->half_l;
      c64.half_r = c32.half_r = sys->half_r;
      c64.orecR = c64.orecL = c32.orecR = c32.orecL = nullptr;
      c64.orec_bytes_r = c64.orec_bytes_l = c32.orec_bytes_r = c32.orec_bytes_l = 0;
      const CubeSide& cl = sys->cube_l;
      const CubeSide& cr = sys->cube_r;
      if (c32.inner_r >= 2 && c32.inner_l >= 3 && cr.half % 4 == 0 && cl.half % 8 == 0) {
        const std::vector<float> rr = outer_records(cr, tr32, cr.K - 2, 4);
        std::vector<float> rl = outer_records(cl, tl32, cl.K - 3, 8);
        // the electron-pair operator follows the pass-L records (staged together)
        for (int k = 0; k < 16; ++k) {
          rl.push_back(c32.pair[k].x);
          rl.push_back(c32.pair[k].y);
        }
        c32.orecR = upload<float>(sys, rr.data(), rr.size() * sizeof(float));
        c32.orecL = upload<float>(sys, rl.data(), rl.size() * sizeof(float));
        c32.orec_bytes_r = (int)(rr.size() * sizeof(float));
        c32.orec_bytes_l = (int)(rl.size() * sizeof(float));  // records (padded to 16 bytes) + 128 pair bytes
      }
      sys->cube64_dev = upload<CubeView<double2>>(sys, &c64, sizeof(c64));
      sys->cube32_dev = upload<CubeView<float2>>(sys, &c32, sizeof(c32));
    }
  }
  sys->on_device = true;
}

static void free_system(rpm_system* sys) {
  for (void* p : sys->allocations) cudaFree(p);
  sys->allocations.clear();
  for (int k = 0; k < 8; ++k) {
    if (sys->scratch[k]) cudaFree(sys->scratch[k]);
    sys->scratch[k] = nullptr;
    sys->scratch_bytes[k] = 0;
  }
}

static rpm_system* create_system(const int* dims, int ndims, const rpm_term* terms, int nterms, const int* left,
                                 int nleft, const int* right, int nright, double tol, int host_only) {
  if (!dims || ndims < 1 || ndims > RPM_MAX_AXES) fail(RPM_E_INVALID, "Every tensor dimension must be positive.");
  long long n = 1;
  for (int a = 0; a < ndims; ++a) {
    if (dims[a] < 1) fail(RPM_E_INVALID, "Every tensor dimension must be positive.");
    n *= dims[a];
    if (n > (1LL << 30)) fail(RPM_E_UNSUPPORTED, "state dimension exceeds 2^30");
  }
  if (nterms < 0 || (nterms > 0 && !terms)) fail(RPM_E_INVALID, "invalid term list");
  auto sys = std::make_unique<rpm_system>();
  sys->ndims = ndims;
  std::copy(dims, dims + ndims, sys->dims);
  sys->n = n;
  const auto strides = tensor_strides(dims, ndims);

  // --- term validation and generic tables (ENG:67-93) ----------------------
  for (int t = 0; t < nterms; ++t) {
    const rpm_term& term = terms[t];
    if (term.naxes < 1 || term.naxes > RPM_MAX_TERM_AXES) {
      fail(term.naxes < 1 ? RPM_E_INVALID : RPM_E_UNSUPPORTED, "Local term must have 1 to 4 unique active axes.");
    }
    std::set<int> seen;
    int d = 1;
    for (int q = 0; q < term.naxes; ++q) {
      const int a = term.axes[q];
      if (a < 0 || a >= ndims) fail(RPM_E_INVALID, "Local term contains an out-of-range axis.");
      if (!seen.insert(a).second) fail(RPM_E_INVALID, "Local term must have unique active axes.");
      d *= dims[a];
    }
    if (d > RPM_MAX_LOCAL_DIM) fail(RPM_E_UNSUPPORTED, "local operator side exceeds 64");
    if (!term.op) fail(RPM_E_INVALID, "local term operator is NULL");
    const cd* op = reinterpret_cast<const cd*>(term.op);
    double norm2 = 0.0, anti2 = 0.0;
    for (int r = 0; r < d; ++r) {
      for (int c = 0; c < d; ++c) {
        const cd v = op[(size_t)r * d + c];
        if (!std::isfinite(v.real()) || !std::isfinite(v.imag())) fail(RPM_E_INVALID, "Local term has non-finite entries.");
        norm2 += std::norm(v);
        anti2 += std::norm(v - std::conj(op[(size_t)c * d + r]));
      }
    }
    if (std::sqrt(anti2) > tol * std::max(1.0, std::sqrt(norm2))) fail(RPM_E_NOT_HERMITIAN, "Local term is not Hermitian.");

    TermMeta meta{};
    meta.naxes = term.naxes;
    meta.d = d;
    meta.op_offset = (int)sys->ops.size();
    meta.col_offset = (int)sys->coloff.size();
    int ls = 1;
    for (int q = term.naxes - 1; q >= 0; --q) {
      meta.stride[q] = (int)strides[term.axes[q]];
      meta.dim[q] = dims[term.axes[q]];
      meta.lstride[q] = ls;
      ls *= dims[term.axes[q]];
    }
    for (int c = 0; c < d; ++c) {
      long long off = 0;
      for (int q = 0; q < term.naxes; ++q) off += (long long)((c / meta.lstride[q]) % meta.dim[q]) * meta.stride[q];
      sys->coloff.push_back((int)off);
    }
    sys->ops.insert(sys->ops.end(), op, op + (size_t)d * d);
    sys->terms.push_back(meta);
  }

  // --- radical split (ENG:159-219) -----------------------------------------
  if (nleft > 0 || nright > 0) {
    if (nleft < 1 || nright < 1 || !left || !right) fail(RPM_E_INVALID, "Full-pair axis groups must be nonempty and disjoint.");
    std::vector<int> lg(left, left + nleft), rg(right, right + nright);
    std::set<int> ls(lg.begin(), lg.end()), rs(rg.begin(), rg.end());
    if ((int)ls.size() != nleft || (int)rs.size() != nright) fail(RPM_E_INVALID, "Full-pair axis groups must be nonempty and disjoint.");
    for (int a : lg)
      if (rs.count(a)) fail(RPM_E_INVALID, "Full-pair axis groups must be nonempty and disjoint.");
    std::set<int> all(ls);
    all.insert(rs.begin(), rs.end());
    if ((int)all.size() != ndims || *all.begin() != 0 || *all.rbegin() != ndims - 1)
      fail(RPM_E_INVALID, "Full-pair axis groups must partition every tensor axis.");
    if (dims[lg[0]] != 2 || dims[rg[0]] != 2) fail(RPM_E_INVALID, "The electron-pair axes must both have dimension two.");
    std::map<int, int> lpos, rpos;
    for (int p = 0; p < nleft; ++p) lpos[lg[p]] = p;
    for (int p = 0; p < nright; ++p) rpos[rg[p]] = p;
    std::vector<GroupTerm> lterms, rterms;
    for (int k = 0; k < 16; ++k) sys->pair[k] = 0.0;
    for (int t = 0; t < nterms; ++t) {
      const rpm_term& term = terms[t];
      const cd* op = reinterpret_cast<const cd*>(term.op);
      bool in_l = true, in_r = true;
      for (int q = 0; q < term.naxes; ++q) {
        in_l = in_l && lpos.count(term.axes[q]);
        in_r = in_r && rpos.count(term.axes[q]);
      }
      GroupTerm gt{{}, op, sys->terms[t].d};
      if (in_l) {
        for (int q = 0; q < term.naxes; ++q) gt.pos.push_back(lpos[term.axes[q]]);
        lterms.push_back(gt);
      } else if (in_r) {
        for (int q = 0; q < term.naxes; ++q) gt.pos.push_back(rpos[term.axes[q]]);
        rterms.push_back(gt);
      } else if (term.naxes == 2 && term.axes[0] == lg[0] && term.axes[1] == rg[0]) {
        for (int k = 0; k < 16; ++k) sys->pair[k] += op[k];
      } else {
        fail(RPM_E_INVALID, "Cross-radical terms must act on the configured electron pair.");
      }
    }
    std::vector<int> ldims, rdims;
    for (int a : lg) ldims.push_back(dims[a]);
    for (int a : rg) rdims.push_back(dims[a]);
    build_group_csr(ldims, lterms, sys->lptr, sys->lcol, sys->lval);
    build_group_csr(rdims, rterms, sys->rptr, sys->rcol, sys->rval);
    int inner_l = 0, inner_r = 0;
    sys->cube = build_cube_side(ldims, lterms, sys->cube_l, sys->cube_tab_l, inner_l) &&
                build_cube_side(rdims, rterms, sys->cube_r, sys->cube_tab_r, inner_r);
    sys->cube64.inner_l = sys->cube32.inner_l = inner_l;
    sys->cube64.inner_r = sys->cube32.inner_r = inner_r;
    auto offsets = [&](const std::vector<int>& g, const std::vector<int>& gd) {
      long long size = 1;
      for (int v : gd) size *= v;
      std::vector<long long> off(size, 0);
      for (long long idx = 0; idx < size; ++idx) {
        long long rem = idx, o = 0;
        for (int p = (int)g.size() - 1; p >= 0; --p) {
          o += (rem % gd[p]) * strides[g[p]];
          rem /= gd[p];
        }
        off[idx] = o;
      }
      return off;
    };
    sys->offl = offsets(lg, ldims);
    sys->offr = offsets(rg, rdims);
    sys->nl = (int)sys->offl.size();
    sys->nr = (int)sys->offr.size();
    sys->half_l = sys->nl / 2;
    sys->half_r = sys->nr / 2;
    sys->split = true;
  }
  if (!host_only) upload_system(sys.get());
  return sys.release();
}

}  // namespace rpm

using rpm::guarded;

extern "C" {

const char* rpm_last_error(void) { return rpm::g_last_error.c_str(); }

int rpm_version(void) { return 1; }

int rpm_device_count(int* count) {
  return guarded([&] {
    if (!count) rpm::fail(RPM_E_INVALID, "count is NULL");
    int c = 0;
    if (cudaGetDeviceCount(&c) != cudaSuccess) {
      cudaGetLastError();
      c = 0;
    }
    *count = c;
  });
}

int rpm_system_create(const int* dims, int ndims, const rpm_term* terms, int nterms, const int* left_axes, int nleft,
                      const int* right_axes, int nright, double hermitian_tolerance, int host_only, rpm_system** out) {
  return guarded([&] {
    if (!out) rpm::fail(RPM_E_INVALID, "out is NULL");
    *out = nullptr;
    *out = rpm::create_system(dims, ndims, terms, nterms, left_axes, nleft, right_axes, nright, hermitian_tolerance,
                              host_only);
  });
}

int rpm_system_destroy(rpm_system* sys) {
  return guarded([&] {
    if (!sys) return;
    rpm::free_system(sys);
    delete sys;
  });
}

int rpm_system_info(const rpm_system* sys, long long* dimension, int* split, int* nl, int* nr, int* nnz_left,
                    int* nnz_right) {
  return guarded([&] {
    if (!sys) rpm::fail(RPM_E_INVALID, "system is NULL");
    if (dimension) *dimension = sys->n;
    if (split) *split = sys->split ? 1 : 0;
    if (nl) *nl = sys->nl;
    if (nr) *nr = sys->nr;
    if (nnz_left) *nnz_left = (int)sys->lcol.size();
    if (nnz_right) *nnz_right = (int)sys->rcol.size();
  });
}

int rpm_system_set_recombination(rpm_system* sys, double singlet_rate, double triplet_rate) {
  return guarded([&] {
    if (!sys) rpm::fail(RPM_E_INVALID, "system is NULL");
    if (!sys->split) rpm::fail(RPM_E_UNSUPPORTED, "recombination needs a radical-split system");
    if (!(singlet_rate >= 0.0) || !(triplet_rate >= 0.0) || !std::isfinite(singlet_rate) ||
        !std::isfinite(triplet_rate))
      rpm::fail(RPM_E_INVALID, "Recombination rates must be finite and nonnegative.");
    if (!sys->recombination)
      for (int k = 0; k < 16; ++k) sys->pair_base[k] = sys->pair[k];
    // P_S on (eA, eB) in the order (uu, ud, du, dd): |S> = (|ud> - |du>) / sqrt 2
    double ps[16] = {};
    ps[1 * 4 + 1] = ps[2 * 4 + 2] = 0.5;
    ps[1 * 4 + 2] = ps[2 * 4 + 1] = -0.5;
    const bool singlet_faster = singlet_rate >= triplet_rate;
    const double delta = std::fabs(singlet_rate - triplet_rate);
    for (int k = 0; k < 16; ++k) {
      const double q = singlet_faster ? ps[k] : ((k % 5 == 0) ? 1.0 : 0.0) - ps[k];  // P_T = 1 - P_S
      sys->pair[k] = sys->pair_base[k] - rpm::cd(0.0, 0.5 * delta * q);
    }
    sys->recombination = true;
    sys->non_hermitian = delta > 0.0;
    sys->rate_singlet = singlet_rate;
    sys->rate_triplet = triplet_rate;
    if (sys->on_device) {
      for (int k = 0; k < 16; ++k) {
        const double2 v = make_double2(sys->pair[k].real(), sys->pair[k].imag());
        sys->split64.pair[k] = v;
        sys->split32.pair[k] = make_float2((float)v.x, (float)v.y);
        sys->cube64.pair[k] = v;
        sys->cube32.pair[k] = make_float2((float)v.x, (float)v.y);
      }
      if (sys->cube && sys->cube32.orecL) {
        // the copy of the pair operator that follows the pass-L outer records
        float2 pair32[16];
        for (int k = 0; k < 16; ++k) pair32[k] = sys->cube32.pair[k];
        char* dst = static_cast<char*>(const_cast<void*>(sys->cube32.orecL)) + sys->cube32.orec_bytes_l - sizeof(pair32);
        rpm::check_cuda(cudaMemcpy(dst, pair32, sizeof(pair32), cudaMemcpyHostToDevice), "update pair operator");
      }
      if (sys->cube) {
        rpm::check_cuda(cudaMemcpy(sys->cube64_dev, &sys->cube64, sizeof(sys->cube64), cudaMemcpyHostToDevice),
                   "update cube view");
        rpm::check_cuda(cudaMemcpy(sys->cube32_dev, &sys->cube32, sizeof(sys->cube32), cudaMemcpyHostToDevice),
                   "update cube view");
      }
    }
  });
}

int rpm_system_recombination(const rpm_system* sys, double* singlet_rate, double* triplet_rate, int* non_hermitian) {
  return guarded([&] {
    if (!sys) rpm::fail(RPM_E_INVALID, "system is NULL");
    if (singlet_rate) *singlet_rate = sys->rate_singlet;
    if (triplet_rate) *triplet_rate = sys->rate_triplet;
    if (non_hermitian) *non_hermitian = sys->non_hermitian ? 1 : 0;
  });
}

int rpm_system_split_tables(const rpm_system* sys, int* lptr, int* lcol, double* lval, int* rptr, int* rcol,
                            double* rval, long long* offl, long long* offr, double* pair) {
  return guarded([&] {
    if (!sys) rpm::fail(RPM_E_INVALID, "system is NULL");
    if (!sys->split) rpm::fail(RPM_E_INVALID, "system has no radical split");
    auto cp = [](auto* dst, const auto& src) {
      if (dst) std::memcpy(dst, src.data(), src.size() * sizeof(src[0]));
    };
    cp(lptr, sys->lptr);
    cp(lcol, sys->lcol);
    cp(rptr, sys->rptr);
    cp(rcol, sys->rcol);
    cp(offl, sys->offl);
    cp(offr, sys->offr);
    if (lval) std::memcpy(lval, sys->lval.data(), sys->lval.size() * sizeof(rpm::cd));
    if (rval) std::memcpy(rval, sys->rval.data(), sys->rval.size() * sizeof(rpm::cd));
    if (pair) std::memcpy(pair, sys->pair, sizeof(sys->pair));
  });
}

}  // extern "C"
