// Host side of the B200 lifting DWT: catalogue, step-program resolution,
// argument checks, axis planning, host-pointer staging and the C ABI of
// include/lifted_capi.h.
#include <cuda_runtime.h>

#include "lw_pdl.hpp"

#include <algorithm>
#include <atomic>
#include <cfloat>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/lifted_capi.h"
#include "lw_host.hpp"
#include "lw_cache.cuh"
#include "lw_launch.hpp"
#include "lw_reg.hpp"

static_assert(LDBL_MANT_DIG == 64,
              "the coefficient casts reproduce x86-64 80-bit long double "
              "arithmetic (1.0L / c in src/lifted-common.hpp:951-963)");

namespace lw {

// ---------------------------------------------------------------------------
// Catalogue (generated from the reference's src/lifted-wavelets.hpp).
#define LW_K_GEN K_GEN
#define LW_K_UNIT K_UNIT
#define LW_K_REPEAT K_REPEAT
#define LW_K_SCALE K_SCALE
#define LW_EVENS 0
#define LW_ODDS 1
#define LW_PM_ADD 0
#define LW_PM_SUB 1
#include "wavelet_catalogue.inc"

namespace {

const StepRow kCatSteps[] = {
#define LW_CATALOGUE_STEPS
#include "wavelet_catalogue.inc"
#undef LW_CATALOGUE_STEPS
};

struct CatWavelet {
  const char* name;
  uint32_t value, width, first, count;
};

const CatWavelet kCatWavelets[] = {
#define LW_CATALOGUE_WAVELETS
#include "wavelet_catalogue.inc"
#undef LW_CATALOGUE_WAVELETS
};

constexpr size_t kNumWavelets = sizeof(kCatWavelets) / sizeof(kCatWavelets[0]);

const CatWavelet* find_wavelet(uint32_t value) {
  for (const auto& w : kCatWavelets)
    if (w.value == value) return &w;
  return nullptr;
}

thread_local std::string g_last_error;
std::atomic<uint64_t> g_launches{0};
std::atomic<uint64_t> g_family[KF_COUNT] = {};
const char* const kFamilyNames[KF_COUNT] = {"line", "reg", "wrow", "wrow2", "wtile",
                                            "col", "batch", "copy", "blur"};
std::atomic<int64_t> g_opt_force_global{0};
std::atomic<int64_t> g_opt_max_global_ctas{296};
std::atomic<int64_t> g_opt_fast_path{1};
std::atomic<int64_t> g_opt_tma_strided{1};
std::atomic<int64_t> g_opt_tma_packed{1};
std::atomic<int64_t> g_opt_tma_stacked{1};
std::atomic<int64_t> g_opt_long_batched{1};
std::atomic<int64_t> g_opt_wrow_split{1};
std::atomic<int64_t> g_opt_overlap{1};
std::atomic<int64_t> g_opt_row_windows{1};
std::atomic<int64_t> g_opt_generic{1};
std::atomic<int64_t> g_opt_l2_hints{0};
std::atomic<int64_t> g_opt_col_row_order{1};
std::atomic<int64_t> g_opt_batch_nd_mode{0};
std::atomic<int64_t> g_opt_edge_always{0};
std::atomic<int64_t> g_opt_overlap_graphs{0};
std::atomic<int64_t> g_opt_zero_steps{1};

}  // namespace

int set_error(int status, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return status;
}

void clear_error() { g_last_error.clear(); }
void count_launches(uint64_t n) { g_launches += n; }
void count_family(int fam, uint64_t n) {
  if (fam >= 0 && fam < KF_COUNT) g_family[fam] += n;
}
uint64_t family_count(int fam) {
  return fam >= 0 && fam < KF_COUNT ? g_family[fam].load() : 0;
}
int family_index(const char* name) {
  for (int i = 0; name && i < KF_COUNT; ++i)
    if (!std::strcmp(name, kFamilyNames[i])) return i;
  return -1;
}

int catalogue_program(uint32_t wavelet, Program* prog) {
  const CatWavelet* w = find_wavelet(wavelet);
  if (!w) return set_error(LIFTED_EINVAL, "unknown wavelet value %u", wavelet);
  prog->rows.assign(kCatSteps + w->first, kCatSteps + w->first + w->count);
  prog->width = w->width;
  prog->cat_index = (int)(w - kCatWavelets);
  return LIFTED_OK;
}

int user_program(const lifted_step_t* steps, size_t nsteps, size_t width,
                 Program* prog) {
  if (nsteps > (size_t)MAX_STEPS)
    return set_error(LIFTED_EINVAL, "step program longer than %d steps",
                     MAX_STEPS);
  if (nsteps && !steps) return set_error(LIFTED_EINVAL, "null step program");
  prog->rows.clear();
  for (size_t k = 0; k < nsteps; ++k) {
    const lifted_step_t& u = steps[k];
    StepRow r{};
    if (u.kind > 3 || u.target > 1)
      return set_error(LIFTED_EINVAL, "step %zu: bad kind/target", k);
    if (u.kind == K_SCALE && (u.ntaps < 1 || u.ntaps > 2))
      return set_error(LIFTED_EINVAL, "step %zu: scale takes 1 or 2 factors", k);
    if ((u.kind == K_GEN || u.kind == K_REPEAT) &&
        (u.ntaps < 1 || u.ntaps > (uint32_t)MAX_TAPS))
      return set_error(LIFTED_EINVAL, "step %zu: 1..%d taps", k, MAX_TAPS);
    if (u.offset < -(1 << 20) || u.offset > (1 << 20))
      return set_error(LIFTED_EINVAL, "step %zu: offset out of range", k);
    r.kind = (int)u.kind;
    r.target = (int)u.target;
    r.offset = u.offset;
    r.ntaps = u.kind == K_UNIT ? 1 : (int)u.ntaps;
    r.pm = u.unit_sub ? 1 : 0;
    for (int t = 0; t < MAX_TAPS; ++t) r.c[t] = (long double)u.coef[t];
    prog->rows.push_back(r);
  }
  prog->width = width;
  return LIFTED_OK;
}

// Resolves a step program for element type T and transform op, in execution
// order (src/lifted-common.hpp:798-964 for the per-step data,
// src/lifted-drivers-inl.hpp:51-63 for the order).
template <typename T>
void resolve_program(const Program& prog, int op, int across,
                     DevProgram<T>* out) {
  std::memset(out, 0, sizeof(*out));
  const bool normal = (op == TF_F || op == TF_I);
  const bool fwd_tf = (op == TF_F || op == TF_FA);
  const bool fwd_loop = (op == TF_F || op == TF_IA);
  const int ns = (int)prog.rows.size();
  out->nsteps = ns;
  out->normal = normal ? 1 : 0;
  out->fwd_driver = fwd_loop ? 1 : 0;
  out->across = across ? 1 : 0;
  for (int k = 0; k < ns; ++k) {
    const StepRow& r = prog.rows[fwd_loop ? k : ns - 1 - k];
    DevStep<T>& d = out->st[k];
    d.kind = r.kind;
    d.ntaps = r.ntaps;
    if (r.kind == K_SCALE) {
      const long double a = r.c[0];
      const long double b = r.ntaps == 2 ? r.c[1] : r.c[0];
      const T s_mul = (T)a, s_div = (T)(1.0L / a);
      const T d_div = (T)b, d_mul = (T)(1.0L / b);
      d.sm = fwd_tf ? s_mul : s_div;
      d.dm = fwd_tf ? d_mul : d_div;
      continue;
    }
    const int N = r.ntaps;
    const int offset = r.offset;
    const int maxo = N - 1 + offset;
    const int n_front = offset < 0 ? -offset : 0;
    const int n_back = maxo < 0 ? 0 : maxo;
    const int offset_r = -maxo;
    const int maxo_r = N - 1 + offset_r;
    const int n_front_r = offset_r < 0 ? -offset_r : 0;
    const int n_back_r = maxo_r < 0 ? 0 : maxo_r;
    const int target = normal ? 1 /*odds*/ : 0 /*evens*/;
    d.y_is_d = (r.target == target) ? 1 : 0;
    d.off = normal ? offset : offset_r;
    d.fold_off = offset;
    d.nf = normal ? n_front : n_front_r;
    d.nb = normal ? n_back : n_back_r;
    if (r.kind == K_UNIT) {
      // unit_op_from_tf_t (src/lifted-steps-inl.hpp:623-626)
      d.sub = fwd_tf ? r.pm : !r.pm;
    } else {
      d.sub = fwd_tf ? 0 : 1;  // op_from_tf (src/lifted-steps-inl.hpp:75-77)
    }
    if (r.kind == K_GEN) {
      for (int t = 0; t < N; ++t) {
        const T v = (T)r.c[normal ? t : N - 1 - t];
        d.c[t] = v;
      }
    } else if (r.kind == K_REPEAT) {
      d.c[0] = (T)r.c[0];
    }
  }
}

template void resolve_program<float>(const Program&, int, int,
                                     DevProgram<float>*);
template void resolve_program<double>(const Program&, int, int,
                                      DevProgram<double>*);

// max_level (src/lifted-common.hpp:1099-1108); (size_t)-1 for width 1.
size_t max_level(size_t width, size_t n) {
  if (width == 0) return 0;
  if (width == 1) return (size_t)-1;
  if (n < width - 1) return 0;
  size_t lvl = 0;
  while (n >= 2 * (width - 1)) {
    lvl += 1;
    n = (n + 1) / 2;
  }
  return lvl;
}

namespace {

// True when the reference's index map would not return, divide by zero, or
// hand back an index outside the band for this call.
bool bad_index_call(int bc, int64_t i, int64_t n) {
  if (bc == BC_PERIODIC || bc == BC_SYMMETRIC) return n == 0;
  if (bc == BC_REFLECT) return n == 0 || (n == 1 && (i < 0 || i >= 1));
  return false;
}


// Replays the index computations of one level of one step program (the loop
// bounds of src/lifted-steps-inl.hpp:500-615, 754-885, 1011-1126) without
// data, and reports whether any of them is one on which the reference hangs,
// divides by zero or indexes out of bounds.
bool level_degenerate(const Program& prog, int op, int bc, int64_t m) {
  const int64_t nd = m / 2, ns = m - nd;
  const bool normal = (op == TF_F || op == TF_I);
  for (const StepRow& r : prog.rows) {
    if (r.kind == K_SCALE) continue;
    const int64_t N = r.ntaps, offset = r.offset;
    const int64_t maxo = N - 1 + offset;
    const int64_t n_front = offset < 0 ? -offset : 0;
    const int64_t n_back = maxo < 0 ? 0 : maxo;
    const int64_t offset_r = -maxo;
    const int64_t maxo_r = N - 1 + offset_r;
    const int64_t n_front_r = offset_r < 0 ? -offset_r : 0;
    const int64_t n_back_r = maxo_r < 0 ? 0 : maxo_r;
    const int target = normal ? 1 : 0;
    const bool same = r.target == target;
    const int64_t nx = same ? ns : nd, ny = same ? nd : ns;
    const int64_t nf = normal ? n_front : n_front_r;
    const int64_t nb = normal ? n_back : n_back_r;
    const int64_t off = normal ? offset : offset_r;
    const int64_t n1 = std::min(nf, ny);
    const int64_t n2 = nd > nb ? nd - nb : 0;
    const int64_t ntap = r.kind == K_UNIT ? 1 : N;
    if (normal) {
      // The boundary-mapped loops [0,n1) and [n2,ny) evaluate i+off+k.
      for (int64_t i = 0; i < n1; ++i)
        for (int64_t k = 0; k < ntap; ++k)
          if (bad_index_call(bc, i + off + k, nx)) return true;
      for (int64_t i = n2; i < ny; ++i)
        for (int64_t k = 0; k < ntap; ++k)
          if (bad_index_call(bc, i + off + k, nx)) return true;
    } else {
      // Front fold i in [offset, 0): index_of(i, ny).
      for (int64_t i = offset, j = 0; i < 0; ++i, ++j) {
        if (r.kind == K_UNIT && j >= nx) break;
        if (bad_index_call(bc, i, ny)) return true;
      }
      // Back fold i in [nd, nx - off): index_of(i, ny); Constant with an
      // empty band yields size_t(-1) and the reference writes y[-1]; a unit
      // step reads x[j] without a bounds check.
      for (int64_t i = nd, j = nd + off; i < nx - off; ++i, ++j) {
        if (bad_index_call(bc, i, ny)) return true;
        if (bc == BC_CONSTANT && ny == 0) return true;
        if (r.kind == K_UNIT) {
          const int64_t io = host_bc_index(bc, i, ny);
          if (io != ny && io != i && (j < 0 || j >= nx)) return true;
        }
      }
    }
  }
  return false;
}

}  // namespace

bool line_degenerate(const Program& prog, int op, int bc, int64_t n,
                     size_t levels) {
  int64_t m = n;
  for (size_t l = 0; l < levels; ++l) {
    if (level_degenerate(prog, op, bc, m)) return true;
    m = m - m / 2;
  }
  return false;
}

// ---------------------------------------------------------------------------
// Pointer classification and staging.
namespace {

bool is_device_pointer(const void* p) {
  if (!p) return false;
  cudaPointerAttributes a;
  cudaError_t e = cudaPointerGetAttributes(&a, p);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

// Element span [lo, hi] covered by a strided array.
void span_of(size_t ndim, const size_t* shape, const ptrdiff_t* stride,
             int64_t* lo, int64_t* hi) {
  int64_t a = 0, b = 0;
  for (size_t d = 0; d < ndim; ++d) {
    int64_t ext = (int64_t)(shape[d] - 1) * (int64_t)stride[d];
    if (ext < 0) a += ext;
    else b += ext;
  }
  *lo = a;
  *hi = b;
}

bool dense(size_t ndim, const size_t* shape, const ptrdiff_t* stride) {
  int64_t lo, hi, numel = 1;
  for (size_t d = 0; d < ndim; ++d) numel *= (int64_t)shape[d];
  span_of(ndim, shape, stride, &lo, &hi);
  return hi - lo + 1 == numel;
}

}  // namespace

bool device_pointer(const void* p) { return is_device_pointer(p); }

// The reference's index maps on inputs that pass bad_index_call (so the
// loops terminate); returns n for "skip".
int64_t host_bc_index(int bc, int64_t i, int64_t n) {
  switch (bc) {
    case BC_ZERO: return (i < 0 || i >= n) ? n : i;
    case BC_CONSTANT: return i < 0 ? 0 : (i >= n ? n - 1 : i);
    case BC_PERIODIC: return (int64_t)((uint64_t)i % (uint64_t)n);
    case BC_SYMMETRIC:
      while (i >= n || i < 0) i = i < 0 ? -(i + 1) : 2 * (n - 1) - (i - 1);
      return i;
    default:
      while (i >= n || i < 0) i = i < 0 ? -i : 2 * (n - 1) - i;
      return i;
  }
}

// ---------------------------------------------------------------------------
// Axis passes.
namespace {

template <typename T>
int run_axis_pass(const Program& prog, int op, int bc, int across,
                  size_t ndim, const int64_t* shape, const int64_t* sin,
                  const int64_t* sout, size_t ax, size_t levels, const T* in,
                  T* out, cudaStream_t stream, const PassOptions& opt) {
  if (levels == 0) return LIFTED_OK;  // the reference returns at once
  LineParams<T> p;
  std::memset(&p, 0, sizeof(p));
  p.in = in;
  p.out = out;
  LineGeom& g = p.g;
  g.n = shape[ax];
  g.sin = sin[ax];
  g.sout = sout[ax];
  // other dims, fastest (smallest |stride_out|) first
  std::vector<size_t> dims;
  for (size_t d = 0; d < ndim; ++d)
    if (d != ax) dims.push_back(d);
  std::stable_sort(dims.begin(), dims.end(), [&](size_t a, size_t b) {
    return std::llabs(sout[a]) < std::llabs(sout[b]);
  });
  g.nlines = 1;
  g.nother = 0;
  for (size_t d : dims) {
    if (shape[d] == 1) continue;
    g.oshape[g.nother] = shape[d];
    g.oin[g.nother] = sin[d];
    g.oout[g.nother] = sout[d];
    g.nother++;
    g.nlines *= shape[d];
  }
  p.levels = (int32_t)levels;
  p.bc = bc;
  resolve_program<T>(prog, op, across, &p.prog);
  p.zfast = zero_fast_ok(p.prog, bc, g.n, (int)levels) ? 1 : 0;

  if (opt.fast_path && !opt.force_global && !opt.no_alloc) {
    // Overlap of source and destination spans (in place, or aliasing).
    int64_t ilo = 0, ihi = 0, olo = 0, ohi = 0;
    for (size_t d = 0; d < ndim; ++d) {
      const int64_t ei = (shape[d] - 1) * sin[d], eo = (shape[d] - 1) * sout[d];
      (ei < 0 ? ilo : ihi) += ei;
      (eo < 0 ? olo : ohi) += eo;
    }
    const char* ib = (const char*)(in + ilo);
    const char* ie = (const char*)(in + ihi + 1);
    const char* ob = (const char*)(out + olo);
    const char* oe = (const char*)(out + ohi + 1);
    const bool overlap = ib < oe && ob < ie;
    RegPassArgs<T> ra;
    ra.prog = &p.prog;
    ra.wi = prog.cat_index;
    ra.op = op;
    ra.bc = bc;
    ra.levels = (int)levels;
    ra.g = g;
    ra.in = in;
    ra.out = out;
    ra.in_place = overlap;
    RegStats st;
    const int rc = plan_reg_pass<T>(ra, stream, &st);
    count_launches((uint64_t)st.launches);
    if (rc == 1) return LIFTED_OK;
    if (rc < 0)
      return set_error(LIFTED_ECUDA, "register-path launch failed (%d): %s", rc,
                       rc <= -1000 ? cudaGetErrorString((cudaError_t)(-rc - 1000))
                                   : "planning error");
  }

  const int64_t n = g.n;
  const int64_t pitch = n;
  const int64_t pitch_b = n - n / 2;
  const size_t line_bytes = (size_t)(pitch + pitch_b) * sizeof(T);
  // Lines too long for one CTA's shared memory: many CTAs per line through
  // the batch engine (level-group tiles), when the lines are contiguous and
  // source and destination do not overlap.
  if (line_bytes > kMaxDynSmem && prog.cat_index >= 0 && bc == BC_ZERO && !opt.force_global &&
      !opt.no_alloc && opt.fast_path && g_opt_long_batched.load()) {
    int64_t ilo = 0, ihi = 0, olo = 0, ohi = 0;
    for (size_t d = 0; d < ndim; ++d) {
      const int64_t ei = (shape[d] - 1) * sin[d], eo = (shape[d] - 1) * sout[d];
      (ei < 0 ? ilo : ihi) += ei;
      (eo < 0 ? olo : ohi) += eo;
    }
    const bool overlap = (const char*)(in + ilo) < (const char*)(out + ohi + 1) &&
                         (const char*)(out + olo) < (const char*)(in + ihi + 1);
    if (!overlap) {
      const int rc = run_lines_batched<T>(wavelet_value((size_t)prog.cat_index), op, bc, g,
                                          (int)levels, in, out, stream);
      if (rc == 1) return LIFTED_OK;
      if (rc < 0) return LIFTED_ECUDA;
    }
  }
  const bool contiguous_axis = (std::llabs(g.sin) == 1);
  int block = 256;
  int W = 1;
  size_t smem = 0;
  int grid = 1;
  T* scratch = nullptr;
  if (line_bytes <= kMaxDynSmem && !opt.force_global) {
    p.use_smem = 1;
    // Batch short lines; batch strided lines across for coalescing.
    const size_t budget = contiguous_axis ? 48 * 1024 : 96 * 1024;
    int64_t w_fit = (int64_t)std::max<size_t>(1, budget / line_bytes);
    int64_t w_want = contiguous_axis ? std::max<int64_t>(1, 4096 / n) : 32;
    W = (int)std::min<int64_t>({w_fit, w_want, 64, g.nlines});
    if ((size_t)W * line_bytes > kMaxDynSmem) W = 1;
    smem = (size_t)W * line_bytes;
    const int64_t work = (int64_t)W * n;
    block = work >= 4096 ? 512 : (work >= 1024 ? 256 : 128);
    int64_t groups = (g.nlines + W - 1) / W;
    grid = (int)std::min<int64_t>(groups, 148 * 32);
  } else {
    p.use_smem = 0;
    W = 1;
    block = 512;
    int64_t groups = g.nlines;
    grid = (int)std::min<int64_t>(groups, opt.max_global_ctas);
    const size_t bytes = (size_t)grid * line_bytes;
    if (opt.scratch) {
      // Caller-provided scratch of fixed size: as many CTAs as lines fit.
      const size_t fit = opt.scratch_bytes / line_bytes;
      if (fit < 1)
        return set_error(LIFTED_ETOOLARGE,
                         "a line of %lld elements needs %zu bytes of scratch; "
                         "only %zu are available",
                         (long long)n, line_bytes, opt.scratch_bytes);
      if ((size_t)grid > fit) grid = (int)fit;
      scratch = (T*)opt.scratch;
    } else {
      cudaError_t e = scratch_alloc((void**)&scratch, bytes, stream);
      if (e != cudaSuccess)
        return set_error(LIFTED_ENOMEM, "cudaMallocAsync(%zu): %s", bytes,
                         cudaGetErrorString(e));
    }
  }
  p.W = W;
  p.pitch = pitch;
  p.pitch_b = pitch_b;
  p.scratch = scratch;
  p.nlines_per_cta_stride = (int64_t)grid * W;
  cudaError_t e = launch_line(p, grid, block, smem, stream);
  count_launches(1);
  count_family(KF_LINE, 1);
  if (scratch && !opt.scratch) scratch_free(scratch, stream);
  if (e != cudaSuccess)
    return set_error(LIFTED_ECUDA, "line kernel launch: %s",
                     cudaGetErrorString(e));
  return LIFTED_OK;
}

template <typename T>
int copy_strided(size_t ndim, const int64_t* shape, const int64_t* sin,
                 const int64_t* sout, const T* in, T* out,
                 cudaStream_t stream) {
  CopyParams<T> p;
  std::memset(&p, 0, sizeof(p));
  p.in = in;
  p.out = out;
  p.total = 1;
  // fastest-varying (last) dim first
  for (size_t k = 0; k < ndim; ++k) {
    size_t d = ndim - 1 - k;
    p.shape[k] = shape[d];
    p.sin[k] = sin[d];
    p.sout[k] = sout[d];
    p.total *= shape[d];
  }
  p.ndim = (int32_t)ndim;
  cudaError_t e = launch_copy(p, stream);
  count_launches(1);
  count_family(KF_COPY, 1);
  if (e != cudaSuccess)
    return set_error(LIFTED_ECUDA, "copy kernel launch: %s",
                     cudaGetErrorString(e));
  return LIFTED_OK;
}

}  // namespace

template <typename T>
bool zero_fast_ok(const DevProgram<T>& prog, int bc, int64_t n, int levels) {
  if (bc != BC_ZERO || !g_opt_zero_steps.load()) return false;
  int64_t m = n;
  for (int l = 0; l < levels; ++l) {
    const int64_t nd = m / 2, ns = m - nd;
    for (int k = 0; k < prog.nsteps; ++k) {
      const DevStep<T>& st = prog.st[k];
      if (st.kind == K_SCALE) continue;
      const int64_t ny = st.y_is_d ? nd : ns;
      const int64_t n1 = std::min<int64_t>(st.nf, ny);
      const int64_t n2 = nd > st.nb ? nd - st.nb : 0;
      if (n1 > n2) return false;
    }
    m = ns;
  }
  return true;
}
template bool zero_fast_ok<float>(const DevProgram<float>&, int, int64_t, int);
template bool zero_fast_ok<double>(const DevProgram<double>&, int, int64_t, int);

// Validation shared by both drivers.
int check_common(uint32_t op, uint32_t bc, size_t ndim, const size_t* shape,
                 const ptrdiff_t* sin, const ptrdiff_t* sout, size_t naxes,
                 const size_t* axes) {
  if (op > 3) return set_error(LIFTED_EINVAL, "unknown transform %u", op);
  if (bc > 4) return set_error(LIFTED_EINVAL, "unknown boundary condition %u", bc);
  if (ndim == 0 || ndim > (size_t)MAX_NDIM)
    return set_error(LIFTED_EINVAL, "ndim %zu outside 1..%d", ndim, MAX_NDIM);
  if (!shape || !sin || !sout)
    return set_error(LIFTED_EINVAL, "null shape/stride");
  if (naxes && !axes) return set_error(LIFTED_EINVAL, "null axes");
  for (size_t i = 0; i < naxes; ++i)
    if (axes[i] >= ndim)
      return set_error(LIFTED_EINVAL, "axis %zu is beyond the array's %zu dims",
                       axes[i], ndim);
  for (size_t d = 0; d < ndim; ++d)
    if (shape[d] > ((size_t)1 << 40))
      return set_error(LIFTED_EINVAL, "dimension %zu too large", d);
  return LIFTED_OK;
}

// Resolves and checks the per-axis levels of the separable driver
// (level 0 = max_level, src/lifted-drivers-inl.hpp:459-463).
int resolve_sep_levels(const Program& prog, uint32_t op, uint32_t bc,
                       const size_t* shape, size_t naxes, const size_t* axes,
                       const size_t* levels, std::vector<size_t>* lv) {
  lv->assign(naxes, 0);
  for (size_t i = 0; i < naxes; ++i) {
    size_t l = levels[i];
    const size_t len = shape[axes[i]];
    if (l == 0) {
      if (prog.width == 1)
        return set_error(LIFTED_EDEGENERATE,
                         "level 0 with a width-1 wavelet: the reference's "
                         "max_level never returns");
      l = max_level(prog.width, len);
    }
    if (l > (size_t)MAX_LEVELS)
      return set_error(LIFTED_EINVAL, "%zu levels exceeds %d", l, MAX_LEVELS);
    if (line_degenerate(prog, (int)op, (int)bc, (int64_t)len, l))
      return set_error(LIFTED_EDEGENERATE,
                       "axis %zu (length %zu, %zu levels): the reference hangs "
                       "or indexes out of bounds on a band this short",
                       axes[i], len, l);
    (*lv)[i] = l;
  }
  return LIFTED_OK;
}

// Separable driver (general_nd, src/lifted-drivers-inl.hpp:417-486).
template <typename T>
int sep_device(const Program& prog, uint32_t op, uint32_t bc, size_t ndim,
               const size_t* shape, const ptrdiff_t* sin,
               const ptrdiff_t* sout, size_t naxes, const size_t* axes,
               const std::vector<size_t>& lv, const T* in, T* out,
               cudaStream_t stream, const PassOptions& opt) {
  int64_t sh[MAX_NDIM], si[MAX_NDIM], so[MAX_NDIM];
  for (size_t d = 0; d < ndim; ++d) {
    sh[d] = (int64_t)shape[d];
    si[d] = sin[d];
    so[d] = sout[d];
  }
  for (size_t i = 0; i < naxes; ++i) {
    const T* src = i == 0 ? in : out;
    const int64_t* ss = i == 0 ? si : so;
    int rc = run_axis_pass<T>(prog, (int)op, (int)bc, /*across=*/1, ndim, sh,
                              ss, so, axes[i], lv[i], src, out, stream, opt);
    if (rc) return rc;
  }
  return LIFTED_OK;
}

// Level shapes of the non-separable driver
// (src/lifted-drivers-inl.hpp:529-540), checked.
int resolve_nonsep_levels(const Program& prog, uint32_t op, uint32_t bc,
                          size_t ndim, const size_t* shape, size_t naxes,
                          const size_t* axes, size_t level,
                          std::vector<std::vector<int64_t>>* shp) {
  if (naxes == 0) return set_error(LIFTED_EINVAL, "no axes");
  size_t lvl = level;
  if (lvl == 0) {
    if (prog.width == 1)
      return set_error(LIFTED_EDEGENERATE,
                       "level 0 with a width-1 wavelet: the reference's "
                       "max_level never returns");
    size_t min_n = shape[axes[0]];
    for (size_t i = 1; i < naxes; ++i) min_n = std::min(min_n, shape[axes[i]]);
    lvl = max_level(prog.width, min_n);
    if (lvl == 0)
      return set_error(LIFTED_EDEGENERATE,
                       "max_level resolves to 0: the reference indexes an "
                       "empty level list");
  }
  if (lvl > (size_t)MAX_LEVELS)
    return set_error(LIFTED_EINVAL, "%zu levels exceeds %d", lvl, MAX_LEVELS);
  shp->assign(lvl, std::vector<int64_t>(ndim));
  for (size_t d = 0; d < ndim; ++d) (*shp)[0][d] = (int64_t)shape[d];
  for (size_t l = 1; l < lvl; ++l) {
    (*shp)[l] = (*shp)[l - 1];
    for (size_t i = 0; i < naxes; ++i) {
      size_t a = axes[i];
      (*shp)[l][a] = (*shp)[l - 1][a] - (*shp)[l - 1][a] / 2;
    }
  }
  for (size_t l = 0; l < lvl; ++l)
    for (size_t i = 0; i < naxes; ++i)
      if (line_degenerate(prog, (int)op, (int)bc, (*shp)[l][axes[i]], 1))
        return set_error(LIFTED_EDEGENERATE,
                         "level %zu axis %zu: the reference hangs or indexes "
                         "out of bounds on a band this short",
                         l, axes[i]);
  return LIFTED_OK;
}

// Non-separable driver (general_nd, src/lifted-drivers-inl.hpp:488-610).
template <typename T>
int nonsep_device(const Program& prog, uint32_t op, uint32_t bc, size_t ndim,
                  const ptrdiff_t* sin, const ptrdiff_t* sout, size_t naxes,
                  const size_t* axes,
                  const std::vector<std::vector<int64_t>>& shp, const T* in,
                  T* out, cudaStream_t stream, const PassOptions& opt) {
  int64_t si[MAX_NDIM], so[MAX_NDIM];
  for (size_t d = 0; d < ndim; ++d) {
    si[d] = sin[d];
    so[d] = sout[d];
  }
  const size_t lvl = shp.size();
  const bool fwd_loop = (op == TF_F || op == TF_IA);
  const T* src = in;
  const int64_t* ssrc = si;
  if (!fwd_loop && (const void*)in != (const void*)out) {
    int rc = copy_strided<T>(ndim, shp[0].data(), si, so, in, out, stream);
    if (rc) return rc;
    src = out;
    ssrc = so;
  }
  for (size_t l = 0; l < lvl; ++l) {
    const std::vector<int64_t>& sh = fwd_loop ? shp[l] : shp[lvl - 1 - l];
    for (size_t i = 0; i < naxes; ++i) {
      const size_t ax = axes[i];
      // Lines along a unit-stride output axis take the reference's Along
      // form, whose adjoint back region runs the direct loop first
      // (src/lifted-drivers-inl.hpp:580,595-602).
      const int across = (so[ax] == 1) ? 0 : 1;
      const T* tsrc = i == 0 ? src : out;
      const int64_t* ts = i == 0 ? ssrc : so;
      int rc = run_axis_pass<T>(prog, (int)op, (int)bc, across, ndim,
                                sh.data(), ts, so, ax, 1, tsrc, out, stream,
                                opt);
      if (rc) return rc;
    }
    src = out;
    ssrc = so;
  }
  return LIFTED_OK;
}

// Entry shared by every C ABI function: validation, empty arrays, host
// staging, then the device driver.
template <typename T>
int lwt_entry(const Program& prog, bool separable, uint32_t op, uint32_t bc,
              size_t ndim, const size_t* shape, const ptrdiff_t* sin,
              const ptrdiff_t* sout, size_t naxes, const size_t* axes,
              const size_t* levels, size_t level, const T* in, T* out,
              void* stream_v, const PassOptions& opt) {
  clear_error();
  int rc = check_common(op, bc, ndim, shape, sin, sout, naxes, axes);
  if (rc) return rc;
  if (separable && naxes && !levels)
    return set_error(LIFTED_EINVAL, "null levels");
  size_t numel = 1;
  for (size_t d = 0; d < ndim; ++d) numel *= shape[d];
  if (numel == 0) return LIFTED_OK;  // empty arrays: nothing to transform
  if (!in || !out) return set_error(LIFTED_EINVAL, "null data pointer");
  // Every check that needs no GPU runs before the first CUDA call.
  std::vector<size_t> lv;
  std::vector<std::vector<int64_t>> shp;
  rc = separable ? resolve_sep_levels(prog, op, bc, shape, naxes, axes, levels, &lv)
                 : resolve_nonsep_levels(prog, op, bc, ndim, shape, naxes, axes,
                                         level, &shp);
  if (rc) return rc;
  cudaStream_t stream = (cudaStream_t)stream_v;

  const bool dev_in = is_device_pointer(in);
  const bool dev_out = is_device_pointer(out);
  auto run = [&](const T* din, T* dout) {
    return separable
               ? sep_device<T>(prog, op, bc, ndim, shape, sin, sout, naxes,
                               axes, lv, din, dout, stream, opt)
               : nonsep_device<T>(prog, op, bc, ndim, sin, sout, naxes, axes,
                                  shp, din, dout, stream, opt);
  };
  if (dev_in && dev_out) return run(in, out);
  if (opt.no_alloc)
    return set_error(LIFTED_EINVAL,
                     "host pointers need staging buffers; this entry point "
                     "allocates nothing");

  // Host (or mixed) pointers: stage through device memory.
  int64_t ilo, ihi, olo, ohi;
  span_of(ndim, shape, sin, &ilo, &ihi);
  span_of(ndim, shape, sout, &olo, &ohi);
  const bool same = (const void*)in == (const void*)out;
  const size_t ibytes = (size_t)(ihi - ilo + 1) * sizeof(T);
  const size_t obytes = (size_t)(ohi - olo + 1) * sizeof(T);
  T* dbuf_in = nullptr;
  T* dbuf_out = nullptr;
  cudaError_t e;
  auto fail = [&](const char* what, cudaError_t err) {
    if (dbuf_in && !dev_in) scratch_free(dbuf_in, stream);
    if (dbuf_out && !dev_out && dbuf_out != dbuf_in) scratch_free(dbuf_out, stream);
    cudaStreamSynchronize(stream);
    return set_error(err == cudaErrorMemoryAllocation ? LIFTED_ENOMEM
                                                      : LIFTED_ECUDA,
                     "%s: %s", what, cudaGetErrorString(err));
  };
  const T* din = in;
  T* dout = out;
  if (!dev_in) {
    e = scratch_alloc((void**)&dbuf_in, ibytes, stream);
    if (e != cudaSuccess) return fail("cudaMallocAsync(in)", e);
    e = cudaMemcpyAsync(dbuf_in, in + ilo, ibytes, cudaMemcpyHostToDevice,
                        stream);
    if (e != cudaSuccess) return fail("cudaMemcpyAsync(H2D in)", e);
    din = dbuf_in - ilo;
  }
  if (!dev_out) {
    if (same && !dev_in) {
      dbuf_out = dbuf_in;
    } else {
      e = scratch_alloc((void**)&dbuf_out, obytes, stream);
      if (e != cudaSuccess) return fail("cudaMallocAsync(out)", e);
      // Prefill when the transform may leave elements of the span untouched:
      // gaps between strided elements, or a first axis with 0 levels (the
      // reference then leaves `out` as it was and later axes read it).
      bool prefill = !dense(ndim, shape, sout) || naxes == 0;
      if (separable && naxes > 0 && lv[0] == 0) prefill = true;
      if (prefill) {
        e = cudaMemcpyAsync(dbuf_out, out + olo, obytes,
                            cudaMemcpyHostToDevice, stream);
        if (e != cudaSuccess) return fail("cudaMemcpyAsync(H2D out)", e);
      }
    }
    dout = dbuf_out - olo;
  }
  rc = run(din, dout);
  if (rc == LIFTED_OK && !dev_out) {
    e = cudaMemcpyAsync(out + olo, dbuf_out, obytes, cudaMemcpyDeviceToHost,
                        stream);
    if (e != cudaSuccess) return fail("cudaMemcpyAsync(D2H out)", e);
  }
  if (dbuf_in) scratch_free(dbuf_in, stream);
  if (dbuf_out && dbuf_out != dbuf_in) scratch_free(dbuf_out, stream);
  e = cudaStreamSynchronize(stream);
  if (rc == LIFTED_OK && e != cudaSuccess)
    return set_error(LIFTED_ECUDA, "cudaStreamSynchronize: %s",
                     cudaGetErrorString(e));
  return rc;
}

template int lwt_entry<float>(const Program&, bool, uint32_t, uint32_t,
                              size_t, const size_t*, const ptrdiff_t*,
                              const ptrdiff_t*, size_t, const size_t*,
                              const size_t*, size_t, const float*, float*,
                              void*, const PassOptions&);
template int lwt_entry<double>(const Program&, bool, uint32_t, uint32_t,
                               size_t, const size_t*, const ptrdiff_t*,
                               const ptrdiff_t*, size_t, const size_t*,
                               const size_t*, size_t, const double*, double*,
                               void*, const PassOptions&);

size_t wavelet_count() { return kNumWavelets; }
uint32_t wavelet_value(size_t i) {
  return i < kNumWavelets ? kCatWavelets[i].value : 0xffffffffu;
}
size_t wavelet_width(uint32_t w) {
  const CatWavelet* c = find_wavelet(w);
  return c ? c->width : 0;
}
const char* last_error() { return g_last_error.c_str(); }

PassOptions default_options() {
  PassOptions o;
  o.force_global = g_opt_force_global.load() != 0;
  o.max_global_ctas = (int)g_opt_max_global_ctas.load();
  o.fast_path = g_opt_fast_path.load() != 0;
  return o;
}

int set_option(const char* name, int64_t value) {
  if (!name) return set_error(LIFTED_EINVAL, "null option name");
  if (!std::strcmp(name, "force_global_scratch")) {
    g_opt_force_global = value ? 1 : 0;
  } else if (!std::strcmp(name, "fast_path")) {
    g_opt_fast_path = value ? 1 : 0;
  } else if (!std::strcmp(name, "tma_strided")) {
    g_opt_tma_strided = value ? 1 : 0;
  } else if (!std::strcmp(name, "tma_packed")) {
    g_opt_tma_packed = value ? 1 : 0;
  } else if (!std::strcmp(name, "tma_stacked")) {
    g_opt_tma_stacked = value ? 1 : 0;
  } else if (!std::strcmp(name, "long_lines_batched")) {
    g_opt_long_batched = value ? 1 : 0;
  } else if (!std::strcmp(name, "wrow_split")) {
    g_opt_wrow_split = value ? 1 : 0;
  } else if (!std::strcmp(name, "overlap_launches")) {
    g_opt_overlap = value ? 1 : 0;
  } else if (!std::strcmp(name, "row_windows")) {
    g_opt_row_windows = value ? 1 : 0;
  } else if (!std::strcmp(name, "generic_kernels")) {
    g_opt_generic = value ? 1 : 0;
  } else if (!std::strcmp(name, "l2_hints")) {
    g_opt_l2_hints = value ? 1 : 0;
  } else if (!std::strcmp(name, "col_row_order")) {
    g_opt_col_row_order = value ? 1 : 0;
  } else if (!std::strcmp(name, "overlap_in_graphs")) {
    if (value < 0 || value > 2) return set_error(LIFTED_EINVAL, "overlap_in_graphs outside 0..2");
    g_opt_overlap_graphs = value;
  } else if (!std::strcmp(name, "zero_step_code")) {
    g_opt_zero_steps = value ? 1 : 0;
  } else if (!std::strcmp(name, "edge_kernels_always")) {
    g_opt_edge_always = value ? 1 : 0;
  } else if (!std::strcmp(name, "batch_nd_mode")) {
    if (value < 0 || value > 2) return set_error(LIFTED_EINVAL, "batch_nd_mode outside 0..2");
    g_opt_batch_nd_mode = value;
  } else if (!std::strcmp(name, "max_global_ctas")) {
    if (value < 1 || value > 65535)
      return set_error(LIFTED_EINVAL, "max_global_ctas outside 1..65535");
    g_opt_max_global_ctas = value;
  } else {
    return set_error(LIFTED_EINVAL, "unknown option '%s'", name);
  }
  return LIFTED_OK;
}
uint64_t launch_count() { return g_launches.load(); }
bool col_enabled() { return g_opt_tma_strided.load() != 0; }
bool col_packed() { return g_opt_tma_packed.load() != 0; }
bool col_stacked() { return g_opt_tma_stacked.load() != 0; }
bool col_row_order() { return g_opt_col_row_order.load() != 0; }
int batch_nd_mode() { return (int)g_opt_batch_nd_mode.load(); }
bool edge_kernels_always() { return g_opt_edge_always.load() != 0; }
bool wrow2_enabled() { return g_opt_wrow_split.load() != 0; }
bool pdl_enabled() { return g_opt_overlap.load() != 0; }
bool pdl_in_graphs(int kind) {
  const int64_t v = g_opt_overlap_graphs.load();
  return v == 1 || (v == 2 && kind == 1);
}
bool wtile_enabled() { return g_opt_row_windows.load() != 0; }
bool generic_enabled() { return g_opt_generic.load() != 0; }
int l2_hint_code() {
  return g_opt_l2_hints.load() ? l2_code(L2_FIRST, L2_LAST) : l2_code(L2_NORMAL, L2_NORMAL);
}

}  // namespace lw

// ---------------------------------------------------------------------------
// C ABI.
extern "C" {

#define LW_SEP(T, SUF)                                                        \
  LIFTED_CAPI int lifted_lwt_sep_##SUF(                                       \
      uint32_t wavelet, uint32_t op, uint32_t bc, size_t ndim,               \
      const size_t* shape, const ptrdiff_t* stride_in,                        \
      const ptrdiff_t* stride_out, size_t naxes, const size_t* axes,          \
      const size_t* levels, const T* in, T* out, void* stream) {              \
    lw::clear_error();                                                        \
    lw::Program prog;                                                         \
    int rc = lw::catalogue_program(wavelet, &prog);                           \
    if (rc) return rc;                                                        \
    return lw::lwt_entry<T>(prog, true, op, bc, ndim, shape, stride_in,       \
                            stride_out, naxes, axes, levels, 0, in, out,      \
                            stream, lw::default_options());                       \
  }
LW_SEP(float, f32)
LW_SEP(double, f64)
#undef LW_SEP

#define LW_NONSEP(T, SUF)                                                     \
  LIFTED_CAPI int lifted_lwt_##SUF(                                           \
      uint32_t wavelet, uint32_t op, uint32_t bc, size_t ndim,               \
      const size_t* shape, const ptrdiff_t* stride_in,                        \
      const ptrdiff_t* stride_out, size_t naxes, const size_t* axes,          \
      size_t level, const T* in, T* out, void* stream) {                      \
    lw::clear_error();                                                        \
    lw::Program prog;                                                         \
    int rc = lw::catalogue_program(wavelet, &prog);                           \
    if (rc) return rc;                                                        \
    return lw::lwt_entry<T>(prog, false, op, bc, ndim, shape, stride_in,      \
                            stride_out, naxes, axes, nullptr, level, in, out, \
                            stream, lw::default_options());                       \
  }
LW_NONSEP(float, f32)
LW_NONSEP(double, f64)
#undef LW_NONSEP

#define LW_PROG(T, SUF)                                                       \
  LIFTED_CAPI int lifted_lwt_sep_program_##SUF(                               \
      const lifted_step_t* steps, size_t nsteps, size_t width, uint32_t op,   \
      uint32_t bc, size_t ndim, const size_t* shape,                          \
      const ptrdiff_t* stride_in, const ptrdiff_t* stride_out, size_t naxes,  \
      const size_t* axes, const size_t* levels, const T* in, T* out,          \
      void* stream) {                                                         \
    lw::clear_error();                                                        \
    lw::Program prog;                                                         \
    int rc = lw::user_program(steps, nsteps, width, &prog);                   \
    if (rc) return rc;                                                        \
    return lw::lwt_entry<T>(prog, true, op, bc, ndim, shape, stride_in,       \
                            stride_out, naxes, axes, levels, 0, in, out,      \
                            stream, lw::default_options());                       \
  }
LW_PROG(float, f32)
LW_PROG(double, f64)
#undef LW_PROG

LIFTED_CAPI size_t lifted_max_level(size_t width, size_t n) {
  return lw::max_level(width, n);
}
LIFTED_CAPI size_t lifted_wavelet_width(uint32_t wavelet) {
  return lw::wavelet_width(wavelet);
}
LIFTED_CAPI size_t lifted_wavelet_count(void) { return lw::wavelet_count(); }
LIFTED_CAPI uint32_t lifted_wavelet_value(size_t index) {
  return lw::wavelet_value(index);
}
LIFTED_CAPI const char* lifted_status_string(int status) {
  switch (status) {
    case LIFTED_OK: return "ok";
    case LIFTED_EINVAL: return "invalid argument";
    case LIFTED_EDEGENERATE:
      return "input on which the reference hangs or indexes out of bounds";
    case LIFTED_ENOTIMPL: return "not implemented";
    case LIFTED_ECUDA: return "CUDA runtime error";
    case LIFTED_ENOMEM: return "out of device memory";
    case LIFTED_ETIMEOUT: return "device-side wait timed out";
    case LIFTED_ETOOLARGE: return "request exceeds a fixed limit";
    default: return "unknown status";
  }
}
LIFTED_CAPI const char* lifted_last_error(void) { return lw::last_error(); }
LIFTED_CAPI uint64_t lifted_launch_count(void) { return lw::launch_count(); }
LIFTED_CAPI uint64_t lifted_kernel_launch_count(const char* family) {
  return lw::family_count(lw::family_index(family));
}
LIFTED_CAPI int lifted_device_check(void* stream) {
  lw::clear_error();
  const int v = lw::check_col_errors((cudaStream_t)stream);
  if (v < 0) return lw::set_error(LIFTED_ECUDA, "device status check failed");
  if (v > 0)
    return lw::set_error(LIFTED_ETIMEOUT,
                         "a strided-pass kernel gave up waiting for a staging copy");
  return LIFTED_OK;
}
LIFTED_CAPI int lifted_set_option(const char* name, int64_t value) {
  lw::clear_error();
  return lw::set_option(name, value);
}

}  // extern "C"
