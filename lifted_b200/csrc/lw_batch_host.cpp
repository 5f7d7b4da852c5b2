// Host side of the batched uneven-length transform: the planner that cuts
// every signal into work items (lw_batch.hpp), the plan object, its launch
// (plain or replayed from a captured CUDA graph), the autotuner of tile
// width and levels per tile group, and the C ABI of include/lifted_capi.h.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/lifted_capi.h"
#include "lw_batch.hpp"
#include "lw_host.hpp"
#include "lw_launch.hpp"

struct lifted_batch_plan {
  int dtype = 4;  // element bytes
  int op = 0, bc = 0;
  int device = -1;             // bound on first run
  std::vector<char> progs_host;  // resolved programs, uploaded on first run
  size_t progs_bytes = 0;
  std::vector<lw::BatchItem> items;
  std::vector<int32_t> item_phase;
  void* d_items = nullptr;
  void* d_progs = nullptr;
  int32_t* d_sync = nullptr;  // [head, error, counters...]
  void* d_scratch = nullptr;
  int64_t ncounters = 0;
  size_t scratch_bytes = 0;
  int64_t buf_elems = 0;
  size_t smem = 0;
  int block = 256, grid = 1;
  int32_t spin_limit = 4000000;
  int64_t ntile = 0, nwhole = 0, nwhole_global = 0, nsignals = 0;
  int64_t max_in = 0, max_out = 0;  // highest element index + 1 touched
  // completion of the last run, so that a run on another stream starts after it
  cudaEvent_t last = nullptr;
  // device buffers from the stream-ordered pool (plans the library caches
  // for long lines), freed stream-ordered after the last run
  bool pooled = false;
  // batches of nD images (line items): axis pass geometries, and the
  // per-CTA global slots of lines longer than shared memory holds
  bool nd = false;
  bool nd_inplace_ok = false;  // the table may run with in == out
  std::vector<lw::BatchAxisGeom> geos;
  void* d_geos = nullptr;
  int64_t slot_elems = 0;
  int64_t slot_off = 0;
  // captured graph of one run and the pointers it was captured with
  cudaGraphExec_t gexec = nullptr;
  const void* g_in = nullptr;
  void* g_out = nullptr;
};

namespace lw {

namespace {

struct TuneKey {
  uint32_t wavelet;
  int dtype, op, log2len;
  int64_t stride;
  bool operator<(const TuneKey& o) const {
    if (wavelet != o.wavelet) return wavelet < o.wavelet;
    if (dtype != o.dtype) return dtype < o.dtype;
    if (op != o.op) return op < o.op;
    if (log2len != o.log2len) return log2len < o.log2len;
    return stride < o.stride;
  }
};
struct TuneVal {
  int tile, levels;
  double us;
};

std::mutex g_tune_mu;
std::map<TuneKey, TuneVal> g_tune;

int ilog2(uint64_t n) {
  int l = 0;
  while (n > 1) {
    n >>= 1;
    ++l;
  }
  return l;
}

// Per-level reach (pairs, per side) of a resolved program: the sum over its
// lifting steps of how far a step's taps reach to the left and right.
template <typename T>
int program_reach(const DevProgram<T>& p) {
  int l = 0, r = 0;
  for (int k = 0; k < p.nsteps; ++k) {
    const DevStep<T>& s = p.st[k];
    if (s.kind == K_SCALE) continue;
    const int nt = s.kind == K_UNIT ? 1 : s.ntaps;
    l += s.off < 0 ? -s.off : 0;
    r += (s.off + nt - 1) > 0 ? (s.off + nt - 1) : 0;
  }
  return l > r ? l : r;
}

// Halo (level-0 samples of the group's band, per side) that K levels with
// this reach need: reach pairs at level l are reach * 2^l samples; plus one
// 2^K margin, rounded up to a multiple of 2^K.
int64_t group_halo(int reach, int K) {
  int64_t h = 0;
  for (int l = 1; l <= K; ++l) h += (int64_t)reach << l;
  const int64_t a = (int64_t)1 << K;
  h += a;
  return (h + a - 1) / a * a;
}

// The uniform Zero-boundary form holds on a band of length m when the front
// and back loops of every step do not overlap (src/lifted-steps-inl.hpp:
// 409-410; n1 <= n2).
template <typename T>
bool band_uniform(const DevProgram<T>& p, int64_t m) {
  const int64_t nd = m / 2, ns = m - nd;
  for (int k = 0; k < p.nsteps; ++k) {
    const DevStep<T>& s = p.st[k];
    if (s.kind == K_SCALE) continue;
    const int64_t ny = s.y_is_d ? nd : ns;
    const int64_t n1 = std::min<int64_t>(s.nf, ny);
    const int64_t n2 = nd > s.nb ? nd - s.nb : 0;
    if (n2 < n1 + 2) return false;
  }
  return true;
}

constexpr int64_t kBandAlign = 32;  // elements (128 bytes of float32)

struct Defaults {
  int64_t whole_max, tile;
  int block;
};
// Measured on B200 over 10,000 uneven float32 signals (all catalogue
// wavelets, lengths 2^8..2^20): 4096-sample tiles and whole items with
// 128-thread CTAs (seven per SM) beat larger tiles and CTAs; float64 keeps
// the same bytes per tile.
template <typename T>
Defaults defaults() {
  if (sizeof(T) == 4) return {4096, 4096, 128};
  return {2048, 2048, 128};
}

// Levels per tile group for a wavelet: the tuned value for the nearest
// tuned length of the same (wavelet, dtype, op), else the largest K <= 6
// whose halo costs at most 1/8 of the tile.
template <typename T>
void pick_group(uint32_t wavelet, int op, int64_t len, int reach,
                const lifted_batch_tuning_t* tu, int64_t* tile, int* K) {
  const Defaults df = defaults<T>();
  int64_t t = (tu && tu->tile) ? (int64_t)tu->tile : 0;
  int k = (tu && tu->tile_levels) ? (int)tu->tile_levels : 0;
  if (!t || !k) {
    std::lock_guard<std::mutex> g(g_tune_mu);
    const int lg = ilog2((uint64_t)len);
    int best_d = 1 << 30;
    for (const auto& kv : g_tune) {
      if (kv.first.wavelet != wavelet || kv.first.dtype != (int)sizeof(T) ||
          kv.first.op != op || kv.first.stride != 1)
        continue;
      const int d = std::abs(kv.first.log2len - lg);
      if (d < best_d) {
        best_d = d;
        if (!t) t = kv.second.tile;
        if (!k) k = kv.second.levels;
      }
    }
  }
  if (!t) t = df.tile;
  if (!k) {
    k = 1;
    for (int kk = 6; kk >= 1; --kk)
      if (2 * group_halo(reach, kk) * 8 <= t) {
        k = kk;
        break;
      }
  }
  const int64_t a = (int64_t)1 << k;
  t = std::max<int64_t>(a, t / a * a);
  *tile = t;
  *K = k;
}

template <typename T>
int plan_create(uint32_t op, uint32_t bc, size_t nsig,
                const lifted_signal_t* sigs, const lifted_batch_tuning_t* tu,
                lifted_batch_plan** out) {
  if (!out) return set_error(LIFTED_EINVAL, "null plan pointer");
  *out = nullptr;
  if (op > 3) return set_error(LIFTED_EINVAL, "unknown transform %u", op);
  if (bc > 4) return set_error(LIFTED_EINVAL, "unknown boundary condition %u", bc);
  if (nsig && !sigs) return set_error(LIFTED_EINVAL, "null signal table");
  const Defaults df = defaults<T>();
  const int64_t whole_max =
      (tu && tu->whole_max) ? (int64_t)tu->whole_max : df.whole_max;
  const int block = (tu && tu->block) ? (int)tu->block : df.block;
  if (block < 64 || block > 512 || block % 32)
    return set_error(LIFTED_EINVAL, "block size %d not in 64..512 (multiple of 32)", block);
  if (whole_max < 64 || whole_max > (int64_t)1 << 24)
    return set_error(LIFTED_EINVAL, "whole_max %lld out of range", (long long)whole_max);

  auto plan = std::make_unique<lifted_batch_plan>();
  plan->dtype = (int)sizeof(T);
  plan->op = (int)op;
  plan->bc = (int)bc;
  plan->nsignals = (int64_t)nsig;

  std::map<uint32_t, int> pidx;
  std::vector<Program> hprogs;
  std::vector<DevProgram<T>> dprogs;
  std::vector<int> reach;
  const bool fwd = (op == TF_F || op == TF_IA);
  const bool zero = (bc == BC_ZERO);
  std::vector<BatchItem>& items = plan->items;
  std::vector<int32_t>& phase = plan->item_phase;
  std::vector<int64_t> work;
  int64_t scratch = 0;  // elements
  int64_t buf = 0;      // shared band capacity needed (elements)
  int32_t nctr = 0;

  auto add = [&](const BatchItem& it, int32_t ph, int64_t w) {
    items.push_back(it);
    phase.push_back(ph);
    work.push_back(w);
  };

  for (size_t si = 0; si < nsig; ++si) {
    const lifted_signal_t& s = sigs[si];
    auto f = pidx.find(s.wavelet);
    int pi;
    if (f == pidx.end()) {
      Program pr;
      int rc = catalogue_program(s.wavelet, &pr);
      if (rc) return set_error(rc, "signal %zu: unknown wavelet value %u", si, s.wavelet);
      DevProgram<T> dp;
      resolve_program<T>(pr, (int)op, /*across=*/1, &dp);
      pi = (int)dprogs.size();
      pidx[s.wavelet] = pi;
      hprogs.push_back(pr);
      dprogs.push_back(dp);
      reach.push_back(program_reach(dp));
    } else {
      pi = f->second;
    }
    const int64_t n = (int64_t)s.length;
    if (n == 0) continue;
    size_t L = s.levels;
    if (L == 0) {
      if (hprogs[pi].width == 1)
        return set_error(LIFTED_EDEGENERATE,
                         "signal %zu: level 0 with a width-1 wavelet (the "
                         "reference's max_level never returns)", si);
      L = max_level(hprogs[pi].width, (size_t)n);
      if (L == 0) continue;  // the reference returns at once
    }
    if (L > (size_t)MAX_LEVELS)
      return set_error(LIFTED_EINVAL, "signal %zu: %zu levels exceeds %d", si, L, MAX_LEVELS);
    if (line_degenerate(hprogs[pi], (int)op, (int)bc, n, L))
      return set_error(LIFTED_EDEGENERATE,
                       "signal %zu (length %lld, %zu levels): the reference "
                       "hangs or indexes out of bounds on a band this short",
                       si, (long long)n, L);
    plan->max_in = std::max<int64_t>(plan->max_in, (int64_t)s.in_offset + n);
    plan->max_out = std::max<int64_t>(plan->max_out, (int64_t)s.out_offset + n);
    std::vector<int64_t> m(L + 1);
    m[0] = n;
    for (size_t l = 0; l < L; ++l) m[l + 1] = m[l] - m[l] / 2;

    BatchItem base;
    std::memset(&base, 0, sizeof(base));
    base.prog = pi;
    base.sig = (int32_t)si;
    base.n0 = n;
    base.in_off = (int64_t)s.in_offset;
    base.out_off = (int64_t)s.out_offset;
    base.wait_ctr = -1;
    base.done_ctr = -1;
    base.gbuf = -1;

    // first level whose band a whole item holds
    size_t lw = 0;
    while (lw < L && m[lw] > whole_max) ++lw;

    if (lw == 0 || !zero) {
      BatchItem it = base;
      it.kind = fwd ? BI_WHOLE_FWD : BI_WHOLE_REV;
      it.lev0 = 0;
      it.nlev = (int32_t)L;
      it.zfast = zero_fast_ok(dprogs[pi], (int)bc, m[0], (int)L) ? 1 : 0;
      it.src_sel = BS_IN;
      it.src_off = base.in_off;
      it.dst_sel = BS_OUT;
      it.dst_off = base.out_off;
      const int64_t need = m[0] + (m[0] - m[0] / 2);
      if (m[0] > whole_max) {
        it.gbuf = scratch;
        scratch += need;
        plan->nwhole_global++;
      } else {
        buf = std::max(buf, need);
      }
      add(it, 1, n);
      plan->nwhole++;
      continue;
    }

    // tile groups over levels [0, lw), then a whole item for [lw, L)
    struct Group {
      int a, K;
      int64_t tile, halo;
    };
    std::vector<Group> groups;
    for (int a = 0; a < (int)lw;) {
      int64_t tile;
      int K;
      pick_group<T>(sigs[si].wavelet, (int)op, m[a], reach[pi], tu, &tile, &K);
      K = std::min<int>(K, (int)lw - a);
      const int64_t al = (int64_t)1 << K;
      tile = std::max<int64_t>(al, tile / al * al);
      const int64_t halo = group_halo(reach[pi], K);
      for (int l = a; l < a + K; ++l)
        if (!band_uniform(dprogs[pi], m[l]))
          return set_error(LIFTED_EINVAL, "signal %zu: band of %lld too short for tiles",
                           si, (long long)m[l]);
      groups.push_back({a, K, tile, halo});
      buf = std::max<int64_t>(buf, 3 * ((tile + 2 * halo + 1) / 2 + 1));
      a += K;
    }
    // scratch bands at the group boundaries inside [1, L)
    std::map<int, int64_t> band_off;
    for (const Group& g : groups) {
      const int b = g.a + g.K;
      if (b < (int)L && !band_off.count(b)) {
        // 128-byte aligned: no cache line holds parts of two bands
        scratch = (scratch + kBandAlign - 1) / kBandAlign * kBandAlign;
        band_off[b] = scratch;
        scratch += m[b];
      }
    }
    if (lw < L) buf = std::max<int64_t>(buf, m[lw] + (m[lw] - m[lw] / 2));

    const int G = (int)groups.size();
    if (fwd) {
      int32_t prev = -1, prev_n = 0;
      for (int gi = 0; gi < G; ++gi) {
        const Group& g = groups[gi];
        const int64_t mb = m[g.a];
        const int64_t nt = (mb + g.tile - 1) / g.tile;
        const int32_t ctr = nctr++;
        for (int64_t t = 0; t < nt; ++t) {
          BatchItem it = base;
          it.kind = BI_TILE_FWD;
          it.lev0 = g.a;
          it.nlev = g.K;
          it.src_sel = g.a == 0 ? BS_IN : BS_SCRATCH;
          it.src_off = g.a == 0 ? base.in_off : band_off[g.a];
          const int b = g.a + g.K;
          it.dst_sel = b == (int)L ? BS_OUT : BS_SCRATCH;
          it.dst_off = b == (int)L ? base.out_off : band_off[b];
          it.wait_ctr = prev;
          it.wait_target = prev_n;
          it.done_ctr = ctr;
          it.t0 = t * g.tile;
          it.t1 = std::min(mb, (t + 1) * g.tile);
          it.halo = g.halo;
          add(it, 2 * gi, it.t1 - it.t0 + 2 * g.halo);
          plan->ntile++;
        }
        prev = ctr;
        prev_n = (int32_t)nt;
      }
      if (lw < L) {
        BatchItem it = base;
        it.kind = BI_WHOLE_FWD;
        it.lev0 = (int32_t)lw;
        it.nlev = (int32_t)(L - lw);
        it.zfast = zero_fast_ok(dprogs[pi], (int)bc, m[lw], (int)(L - lw)) ? 1 : 0;
        it.src_sel = BS_SCRATCH;
        it.src_off = band_off[(int)lw];
        it.dst_sel = BS_OUT;
        it.dst_off = base.out_off;
        it.wait_ctr = prev;
        it.wait_target = prev_n;
        add(it, 2 * G, m[lw]);
        plan->nwhole++;
      }
    } else {
      int32_t prev = -1, prev_n = 0;
      if (lw < L) {
        BatchItem it = base;
        it.kind = BI_WHOLE_REV;
        it.lev0 = (int32_t)lw;
        it.nlev = (int32_t)(L - lw);
        it.zfast = zero_fast_ok(dprogs[pi], (int)bc, m[lw], (int)(L - lw)) ? 1 : 0;
        it.src_sel = BS_IN;
        it.src_off = base.in_off;
        it.dst_sel = BS_SCRATCH;
        it.dst_off = band_off[(int)lw];
        it.done_ctr = nctr++;
        prev = it.done_ctr;
        prev_n = 1;
        add(it, 0, m[lw]);
        plan->nwhole++;
      }
      for (int h = 0; h < G; ++h) {
        const Group& g = groups[G - 1 - h];
        const int64_t mb = m[g.a];
        const int64_t nt = (mb + g.tile - 1) / g.tile;
        const int32_t ctr = nctr++;
        const int b = g.a + g.K;
        for (int64_t t = 0; t < nt; ++t) {
          BatchItem it = base;
          it.kind = BI_TILE_REV;
          it.lev0 = g.a;
          it.nlev = g.K;
          it.src_sel = b == (int)L ? BS_IN : BS_SCRATCH;
          it.src_off = b == (int)L ? base.in_off : band_off[b];
          it.dst_sel = g.a == 0 ? BS_OUT : BS_SCRATCH;
          it.dst_off = g.a == 0 ? base.out_off : band_off[g.a];
          it.wait_ctr = prev;
          it.wait_target = prev_n;
          it.done_ctr = ctr;
          it.t0 = t * g.tile;
          it.t1 = std::min(mb, (t + 1) * g.tile);
          it.halo = g.halo;
          add(it, 2 + 2 * h, it.t1 - it.t0 + 2 * g.halo);
          plan->ntile++;
        }
        prev = ctr;
        prev_n = (int32_t)nt;
      }
    }
  }

  // Queue order: by phase (every producer group before its consumers), then
  // largest work first within a phase.
  std::vector<size_t> ord(items.size());
  for (size_t i = 0; i < ord.size(); ++i) ord[i] = i;
  std::stable_sort(ord.begin(), ord.end(), [&](size_t a, size_t b) {
    if (phase[a] != phase[b]) return phase[a] < phase[b];
    return work[a] > work[b];
  });
  {
    std::vector<BatchItem> it2(items.size());
    std::vector<int32_t> ph2(items.size());
    for (size_t i = 0; i < ord.size(); ++i) {
      it2[i] = items[ord[i]];
      ph2[i] = phase[ord[i]];
    }
    items.swap(it2);
    phase.swap(ph2);
  }

  plan->ncounters = nctr;
  plan->buf_elems = std::max<int64_t>(buf, 3 * 64);
  plan->buf_elems = (plan->buf_elems + 3) / 3 * 3;
  plan->smem = batch_smem_bytes<T>(plan->buf_elems);
  if (plan->smem > kMaxDynSmem)
    return set_error(LIFTED_EINVAL,
                     "batch tiles need %zu bytes of shared memory (limit %zu): "
                     "lower the tile width or whole_max", plan->smem, kMaxDynSmem);
  plan->block = block;
  if (tu && tu->spin_limit) plan->spin_limit = tu->spin_limit > 0 ? tu->spin_limit : 0;
  plan->scratch_bytes = (size_t)scratch * sizeof(T);

  plan->progs_bytes = dprogs.size() * sizeof(DevProgram<T>);
  plan->progs_host.assign((const char*)dprogs.data(), (const char*)dprogs.data() + plan->progs_bytes);
  *out = plan.release();
  return LIFTED_OK;
}

// Binds the plan to the current device on its first run: launch shape from
// the kernel's occupancy, device copies of the queue and programs, scratch.
template <typename T>
int ensure_device(lifted_batch_plan* p, cudaStream_t stream = nullptr) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return set_error(LIFTED_ECUDA, "no CUDA device");
  }
  if (p->device >= 0) {
    if (dev != p->device)
      return set_error(LIFTED_EINVAL, "plan bound to device %d, current device is %d",
                       p->device, dev);
    return LIFTED_OK;
  }
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int occ = batch_occupancy((int)sizeof(T), p->block, p->smem);
  if (occ < 1)
    return set_error(LIFTED_ECUDA, "batch kernel cannot run with %d threads and "
                     "%zu bytes of shared memory", p->block, p->smem);
  p->grid = (int)std::min<int64_t>((int64_t)sms * occ, (int64_t)p->items.size());
  cudaError_t e;
  auto alloc = [&](void** ptr, size_t bytes) {
    return p->pooled ? scratch_alloc(ptr, bytes, stream) : cudaMalloc(ptr, bytes);
  };
  auto upload = [&](void* dst, const void* src, size_t bytes) {
    // pageable source: the call returns once the data is staged
    return p->pooled ? cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, stream)
                     : cudaMemcpy(dst, src, bytes, cudaMemcpyHostToDevice);
  };
  auto release = [&](void* ptr) {
    if (!ptr) return;
    if (p->pooled) scratch_free(ptr, stream);
    else cudaFree(ptr);
  };
  if (p->slot_elems > 0) {
    // one global slot per resident CTA for line items too long for shared
    // memory, after the plan's own scratch bands
    p->slot_off = ((int64_t)(p->scratch_bytes / sizeof(T)) + kBandAlign - 1) / kBandAlign *
                  kBandAlign;
    p->slot_elems = (p->slot_elems + kBandAlign - 1) / kBandAlign * kBandAlign;
    p->scratch_bytes = (size_t)(p->slot_off + (int64_t)p->grid * p->slot_elems) * sizeof(T);
  }
  e = alloc(&p->d_items, p->items.size() * sizeof(BatchItem));
  if (e == cudaSuccess && !p->geos.empty())
    e = alloc(&p->d_geos, p->geos.size() * sizeof(BatchAxisGeom));
  if (e == cudaSuccess && !p->geos.empty())
    e = upload(p->d_geos, p->geos.data(), p->geos.size() * sizeof(BatchAxisGeom));
  if (e == cudaSuccess) e = alloc(&p->d_progs, p->progs_bytes);
  if (e == cudaSuccess) e = alloc((void**)&p->d_sync, (size_t)(2 + p->ncounters) * sizeof(int32_t));
  if (e == cudaSuccess && p->scratch_bytes) e = alloc(&p->d_scratch, p->scratch_bytes);
  if (e == cudaSuccess) e = upload(p->d_items, p->items.data(), p->items.size() * sizeof(BatchItem));
  if (e == cudaSuccess) e = upload(p->d_progs, p->progs_host.data(), p->progs_bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    release(p->d_items);
    release(p->d_progs);
    release(p->d_sync);
    release(p->d_scratch);
    release(p->d_geos);
    p->d_items = p->d_progs = p->d_scratch = p->d_geos = nullptr;
    p->d_sync = nullptr;
    return set_error(e == cudaErrorMemoryAllocation ? LIFTED_ENOMEM : LIFTED_ECUDA,
                     "batch plan buffers: %s", cudaGetErrorString(e));
  }
  if (cudaEventCreateWithFlags(&p->last, cudaEventDisableTiming) != cudaSuccess) {
    cudaGetLastError();
    p->last = nullptr;
  }
  p->device = dev;
  return LIFTED_OK;
}

template <typename T>
int plan_run(lifted_batch_plan* p, const T* in, T* out, cudaStream_t stream,
             bool count = true, bool spans_checked = false) {
  if (p->items.empty()) return LIFTED_OK;
  if (!device_pointer(in) || !device_pointer(out))
    return set_error(LIFTED_EINVAL, "batch transforms take device (or managed) pointers");
  // in and out must not overlap: tiles read input other tiles' outputs would
  // clobber; a batch of nD images may also run with in == out when every
  // image is transformed in place
  const char* ib = (const char*)in;
  const char* ie = (const char*)(in + p->max_in);
  const char* ob = (const char*)out;
  const char* oe = (const char*)(out + p->max_out);
  const bool inplace = p->nd && (const void*)in == (const void*)out && p->nd_inplace_ok;
  if (!spans_checked && !inplace && ib < oe && ob < ie)
    return set_error(LIFTED_EINVAL, "batch input and output overlap");
  int rc = ensure_device<T>(p, stream);
  if (rc) return rc;
  // runs of one plan share its queue and counters: order them on the GPU
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(stream, &cap) != cudaSuccess) cudaGetLastError();
  const bool capturing = cap != cudaStreamCaptureStatusNone;
  if (p->last && !capturing) cudaStreamWaitEvent(stream, p->last, 0);
  cudaError_t e = cudaMemsetAsync(p->d_sync, 0, (size_t)(2 + p->ncounters) * sizeof(int32_t), stream);
  if (e != cudaSuccess) return set_error(LIFTED_ECUDA, "batch reset: %s", cudaGetErrorString(e));
  BatchParams<T> bp;
  std::memset(&bp, 0, sizeof(bp));
  bp.in = in;
  bp.out = out;
  bp.scratch = (T*)p->d_scratch;
  bp.items = (const BatchItem*)p->d_items;
  bp.progs = (const DevProgram<T>*)p->d_progs;
  bp.head = p->d_sync;
  bp.error = p->d_sync + 1;
  bp.counters = p->d_sync + 2;
  bp.nitems = (int32_t)p->items.size();
  bp.bc = p->bc;
  bp.buf_elems = p->buf_elems;
  bp.spin_limit = p->spin_limit;
  bp.geos = (const BatchAxisGeom*)p->d_geos;
  bp.slot_off = p->slot_off;
  bp.slot_elems = p->slot_elems;
  e = launch_batch(bp, p->grid, p->block, p->smem, stream);
  if (count) {
    count_launches(1);
    count_family(KF_BATCH, 1);
  }
  if (e != cudaSuccess) return set_error(LIFTED_ECUDA, "batch kernel launch: %s", cudaGetErrorString(e));
  if (p->last && !capturing) cudaEventRecord(p->last, stream);
  return LIFTED_OK;
}

int plan_run_any(lifted_batch_plan* p, const void* in, void* out, cudaStream_t s,
                 bool count = true) {
  if (p->dtype == 4) return plan_run<float>(p, (const float*)in, (float*)out, s, count);
  return plan_run<double>(p, (const double*)in, (double*)out, s, count);
}

int plan_graph(lifted_batch_plan* p, const void* in, void* out, cudaStream_t stream) {
  if (p->items.empty()) return LIFTED_OK;
  if (!p->gexec || p->g_in != in || p->g_out != out) {
    // device buffers exist before capture (no allocation or copy inside it)
    const int rc0 = p->dtype == 4 ? ensure_device<float>(p) : ensure_device<double>(p);
    if (rc0) return rc0;
    if (p->gexec) {
      cudaGraphExecDestroy(p->gexec);
      p->gexec = nullptr;
    }
    cudaStream_t cs;
    cudaError_t e = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking);
    if (e != cudaSuccess) return set_error(LIFTED_ECUDA, "capture stream: %s", cudaGetErrorString(e));
    e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) {
      cudaStreamDestroy(cs);
      return set_error(LIFTED_ECUDA, "begin capture: %s", cudaGetErrorString(e));
    }
    // the captured launch is counted when the graph is replayed
    int rc = plan_run_any(p, in, out, cs, /*count=*/false);
    cudaGraph_t g = nullptr;
    e = cudaStreamEndCapture(cs, &g);
    cudaStreamDestroy(cs);
    if (rc) {
      if (g) cudaGraphDestroy(g);
      return rc;
    }
    if (e != cudaSuccess) return set_error(LIFTED_ECUDA, "end capture: %s", cudaGetErrorString(e));
    e = cudaGraphInstantiate(&p->gexec, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
      p->gexec = nullptr;
      return set_error(LIFTED_ECUDA, "graph instantiate: %s", cudaGetErrorString(e));
    }
    p->g_in = in;
    p->g_out = out;
  }
  cudaError_t e = cudaGraphLaunch(p->gexec, stream);
  count_launches(1);
  count_family(KF_BATCH, 1);
  if (e != cudaSuccess) return set_error(LIFTED_ECUDA, "graph launch: %s", cudaGetErrorString(e));
  return LIFTED_OK;
}

// ---------------------------------------------------------------------------
// Long contiguous lines of an axis pass as a batch (each line one signal).

struct LinesKey {
  std::string k;
  bool operator<(const LinesKey& o) const { return k < o.k; }
};
std::mutex g_lines_mu;
std::map<LinesKey, lifted_batch_plan*> g_lines_plans;
std::vector<LinesKey> g_lines_order;  // insertion order, oldest first
constexpr size_t kLinesPlans = 16;

}  // namespace

template <typename T>
int run_lines_batched(uint32_t wavelet, int op, int bc, const LineGeom& g, int levels,
                      const T* in, T* out, cudaStream_t stream) {
  if (g.sin != 1 || g.sout != 1 || levels < 1 || g.nlines < 1) return 0;
  for (int d = 0; d < g.nother; ++d)
    if (g.oin[d] < 0 || g.oout[d] < 0) return 0;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  char buf[96];
  std::string key;
  std::snprintf(buf, sizeof(buf), "%d|%d|%u|%d|%d|%d|%lld|%lld|", dev, (int)sizeof(T), wavelet,
                op, bc, levels, (long long)g.n, (long long)g.nlines);
  key = buf;
  for (int d = 0; d < g.nother; ++d) {
    std::snprintf(buf, sizeof(buf), "%lld,%lld,%lld;", (long long)g.oshape[d],
                  (long long)g.oin[d], (long long)g.oout[d]);
    key += buf;
  }
  std::lock_guard<std::mutex> lk(g_lines_mu);
  lifted_batch_plan* plan = nullptr;
  auto it = g_lines_plans.find({key});
  if (it != g_lines_plans.end()) {
    plan = it->second;
  } else {
    std::vector<lifted_signal_t> sig((size_t)g.nlines);
    for (int64_t L = 0; L < g.nlines; ++L) {
      int64_t r = L, bi = 0, bo = 0;
      for (int d = 0; d < g.nother; ++d) {
        const int64_t q = r / g.oshape[d];
        const int64_t idx = r - q * g.oshape[d];
        r = q;
        bi += idx * g.oin[d];
        bo += idx * g.oout[d];
      }
      sig[L].wavelet = wavelet;
      sig[L].levels = (uint32_t)levels;
      sig[L].length = (uint64_t)g.n;
      sig[L].in_offset = (uint64_t)bi;
      sig[L].out_offset = (uint64_t)bo;
    }
    // a new plan allocates: not inside a stream capture
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(stream, &cap) != cudaSuccess) cudaGetLastError();
    if (cap != cudaStreamCaptureStatusNone) return 0;
    const int rc = plan_create<T>((uint32_t)op, (uint32_t)bc, sig.size(), sig.data(), nullptr, &plan);
    if (rc) {
      clear_error();
      return 0;  // not eligible: the general path handles it
    }
    plan->pooled = true;
    if (g_lines_plans.size() >= kLinesPlans) {
      const LinesKey old = g_lines_order.front();
      g_lines_order.erase(g_lines_order.begin());
      lifted_batch_plan* victim = g_lines_plans[old];
      g_lines_plans.erase(old);
      lifted_batch_plan_destroy(victim);  // stream-ordered after its last run
    }
    g_lines_plans[{key}] = plan;
    g_lines_order.push_back({key});
  }
  const int rc = plan_run<T>(plan, in, out, stream);
  if (rc) return -1;
  return 1;
}

template int run_lines_batched<float>(uint32_t, int, int, const LineGeom&, int, const float*,
                                      float*, cudaStream_t);
template int run_lines_batched<double>(uint32_t, int, int, const LineGeom&, int,
                                       const double*, double*, cudaStream_t);

// ---------------------------------------------------------------------------
// Batches of nD images (lifted_lwt_batch_nd_*) as one persistent launch.
//
// Every image is a dense C-order array transformed separably over all of its
// axes in order (src/lifted-drivers-inl.hpp:417-486: the first axis reads
// `in`, later axes work in place on `out`).  Its pass along an axis is cut
// into line items of W whole lines each; the items of the image's next axis
// wait (bounded) on a completion counter that the items of this axis
// increment, and the queue holds every image's first-axis items before any
// second-axis item, and so on, so every wait ends.  Images of any shape,
// wavelet and level counts share the launch.

namespace {

template <typename T>
int plan_create_nd(uint32_t op, uint32_t bc, size_t nimg, const lifted_image_t* ims,
                   const lifted_batch_tuning_t* tu, lifted_batch_plan** out) {
  *out = nullptr;
  if (op > 3) return set_error(LIFTED_EINVAL, "unknown transform %u", op);
  if (bc > 4) return set_error(LIFTED_EINVAL, "unknown boundary condition %u", bc);
  // shared-memory budget per CTA (elements) and CTA size: lines of an axis
  // pass are grouped up to this budget (a line needs 1.5 of its length)
  const int64_t budget = (tu && tu->whole_max) ? (int64_t)tu->whole_max * 3 / 2
                                              : (int64_t)(48 * 1024) / (int64_t)sizeof(T);
  const int block = (tu && tu->block) ? (int)tu->block : 256;
  if (block < 64 || block > 512 || block % 32)
    return set_error(LIFTED_EINVAL, "block size %d not in 64..512 (multiple of 32)", block);
  if (nimg && !ims) return set_error(LIFTED_EINVAL, "null image table");
  // shapes; outputs pairwise disjoint; whether the table runs in place
  // (in == out): every image's input span equals its output span or misses
  // it, and meets no other image's output span
  struct Span {
    uint64_t lo, hi;
    size_t img;
  };
  std::vector<Span> outs, ins;
  for (size_t i = 0; i < nimg; ++i) {
    const lifted_image_t& im = ims[i];
    if (im.ndim < 1 || im.ndim > 4)
      return set_error(LIFTED_EINVAL, "image %zu: ndim %u outside 1..4", i, im.ndim);
    uint64_t n = 1;
    for (uint32_t d = 0; d < im.ndim; ++d) {
      if (im.shape[d] == 0) return set_error(LIFTED_EINVAL, "image %zu: empty axis %u", i, d);
      if (n > (UINT64_MAX >> 2) / im.shape[d])
        return set_error(LIFTED_EINVAL, "image %zu: size overflow", i);
      n *= im.shape[d];
    }
    outs.push_back({im.out_offset, im.out_offset + n, i});
    ins.push_back({im.in_offset, im.in_offset + n, i});
  }
  std::sort(outs.begin(), outs.end(), [](const Span& a, const Span& b) { return a.lo < b.lo; });
  for (size_t k = 1; k < outs.size(); ++k)
    if (outs[k].lo < outs[k - 1].hi)
      return set_error(LIFTED_EINVAL, "images %zu and %zu have overlapping outputs",
                       outs[k - 1].img, outs[k].img);
  bool inplace_ok = true;
  for (const Span& a : ins) {
    auto it = std::upper_bound(outs.begin(), outs.end(), a.lo,
                               [](uint64_t v, const Span& o) { return v < o.hi; });
    for (; it != outs.end() && it->lo < a.hi && inplace_ok; ++it)
      if (it->img != a.img || it->lo != a.lo) inplace_ok = false;
  }
  auto plan = std::make_unique<lifted_batch_plan>();
  plan->dtype = (int)sizeof(T);
  plan->op = (int)op;
  plan->bc = (int)bc;
  plan->nd = true;
  plan->nd_inplace_ok = inplace_ok;
  plan->nsignals = (int64_t)nimg;
  std::map<uint32_t, int> pidx;
  std::vector<DevProgram<T>> dprogs;
  std::vector<BatchItem>& items = plan->items;
  std::vector<int32_t>& phase = plan->item_phase;
  std::vector<int64_t> work;
  int64_t buf = 0;
  int32_t nctr = 0;
  const bool fwd = (op == TF_F || op == TF_IA);
  for (size_t ii = 0; ii < nimg; ++ii) {
    const lifted_image_t& im = ims[ii];
    Program pr;
    int rc = catalogue_program(im.wavelet, &pr);
    if (rc) return set_error(rc, "image %zu: unknown wavelet value %u", ii, im.wavelet);
    int pi;
    auto f = pidx.find(im.wavelet);
    if (f == pidx.end()) {
      DevProgram<T> dp;
      resolve_program<T>(pr, (int)op, /*across=*/1, &dp);
      pi = (int)dprogs.size();
      pidx[im.wavelet] = pi;
      dprogs.push_back(dp);
    } else {
      pi = f->second;
    }
    const size_t nd = im.ndim;
    size_t shape[4], axes[4], lv_in[4];
    int64_t stride[4];
    int64_t numel = 1;
    for (size_t d = 0; d < nd; ++d) {
      shape[d] = (size_t)im.shape[d];
      axes[d] = d;
      lv_in[d] = im.levels[d];
      numel *= (int64_t)im.shape[d];
    }
    int64_t st = 1;
    for (size_t d = nd; d-- > 0;) {
      stride[d] = st;
      st *= (int64_t)shape[d];
    }
    std::vector<size_t> lv;
    rc = resolve_sep_levels(pr, op, bc, shape, nd, axes, lv_in, &lv);
    if (rc) return set_error(rc, "image %zu: %s", ii, last_error());
    plan->max_in = std::max<int64_t>(plan->max_in, (int64_t)im.in_offset + numel);
    plan->max_out = std::max<int64_t>(plan->max_out, (int64_t)im.out_offset + numel);
    // axes that run (levels > 0), in order
    std::vector<size_t> run;
    for (size_t a = 0; a < nd; ++a)
      if (lv[a] > 0) run.push_back(a);
    int32_t prev = -1, prev_n = 0;
    for (size_t k = 0; k < run.size(); ++k) {
      const size_t a = run[k];
      const int64_t n = (int64_t)shape[a];
      BatchAxisGeom g;
      std::memset(&g, 0, sizeof(g));
      g.n = n;
      g.sa = stride[a];
      int no = 0;
      for (size_t d = nd; d-- > 0;) {
        if (d == a) continue;
        g.oshape[no] = (int64_t)shape[d];
        g.ostride[no] = stride[d];
        ++no;
      }
      for (; no < 3; ++no) {
        g.oshape[no] = 1;
        g.ostride[no] = 0;
      }
      const int32_t gi = (int32_t)plan->geos.size();
      plan->geos.push_back(g);
      const int64_t nlines = numel / n;
      const int64_t need = n + (n - n / 2);
      const bool strided = g.sa != 1;
      int64_t W;
      int64_t gbuf = -1;
      if (need > budget) {
        W = 1;
        gbuf = -2;
        plan->slot_elems = std::max(plan->slot_elems, need);
        plan->nwhole_global++;
      } else {
        // at most 64 lines (the kernel's per-item line table)
        const int64_t want = strided ? 32 : std::min<int64_t>(64, std::max<int64_t>(1, 4096 / n));
        W = std::min<int64_t>({want, budget / need, nlines});
        W = std::max<int64_t>(W, 1);
        buf = std::max(buf, W * need);
      }
      const int64_t nit = (nlines + W - 1) / W;
      if (nit > (int64_t)INT32_MAX / 2 || (int64_t)items.size() + nit > (int64_t)INT32_MAX / 2)
        return set_error(LIFTED_EINVAL, "image %zu: too many line items", ii);
      const int32_t ctr = k + 1 < run.size() ? nctr++ : -1;
      const int32_t zf = zero_fast_ok(dprogs[pi], (int)bc, n, (int)lv[a]) ? 1 : 0;
      for (int64_t t = 0; t < nit; ++t) {
        BatchItem it;
        std::memset(&it, 0, sizeof(it));
        it.kind = fwd ? BI_LINES_FWD : BI_LINES_REV;
        it.prog = pi;
        it.sig = (int32_t)ii;
        it.lev0 = 0;
        it.nlev = (int32_t)lv[a];
        it.src_sel = a == 0 ? BS_IN : BS_OUT;
        it.dst_sel = BS_OUT;
        it.wait_ctr = prev;
        it.wait_target = prev_n;
        it.done_ctr = ctr;
        it.geo = gi;
        it.zfast = zf;
        it.n0 = n;
        it.in_off = (int64_t)im.in_offset;
        it.out_off = (int64_t)im.out_offset;
        it.src_off = it.src_sel == BS_IN ? it.in_off : it.out_off;
        it.dst_off = it.out_off;
        it.t0 = t * W;
        it.t1 = std::min(nlines, (t + 1) * W);
        it.gbuf = gbuf;
        items.push_back(it);
        phase.push_back((int32_t)k);
        work.push_back((it.t1 - it.t0) * n);
        plan->nwhole++;
      }
      prev = ctr;
      prev_n = (int32_t)nit;
    }
  }
  // queue order: by axis position (every producer before its consumers),
  // then largest work first
  std::vector<size_t> ord(items.size());
  for (size_t i = 0; i < ord.size(); ++i) ord[i] = i;
  std::stable_sort(ord.begin(), ord.end(), [&](size_t a, size_t b) {
    if (phase[a] != phase[b]) return phase[a] < phase[b];
    return work[a] > work[b];
  });
  {
    std::vector<BatchItem> it2(items.size());
    std::vector<int32_t> ph2(items.size());
    for (size_t i = 0; i < ord.size(); ++i) {
      it2[i] = items[ord[i]];
      ph2[i] = phase[ord[i]];
    }
    items.swap(it2);
    phase.swap(ph2);
  }
  plan->ncounters = nctr;
  plan->buf_elems = std::max<int64_t>(buf, 3 * 64);
  plan->buf_elems = (plan->buf_elems + 3) / 3 * 3;
  plan->smem = batch_smem_bytes<T>(plan->buf_elems);
  if (plan->smem > kMaxDynSmem)
    return set_error(LIFTED_EINVAL, "line items need %zu bytes of shared memory (limit %zu)",
                     plan->smem, kMaxDynSmem);
  plan->block = block;
  if (tu && tu->spin_limit) plan->spin_limit = tu->spin_limit > 0 ? tu->spin_limit : 0;
  plan->scratch_bytes = 0;
  plan->progs_bytes = dprogs.size() * sizeof(DevProgram<T>);
  plan->progs_host.assign((const char*)dprogs.data(),
                          (const char*)dprogs.data() + plan->progs_bytes);
  *out = plan.release();
  return LIFTED_OK;
}

std::mutex g_nd_mu;
std::map<std::string, lifted_batch_plan*> g_nd_plans;
std::vector<std::string> g_nd_order;  // insertion order, oldest first
constexpr size_t kNdPlans = 8;

}  // namespace

template <typename T>
int run_batch_nd(uint32_t op, uint32_t bc, size_t nimg, const lifted_image_t* ims, const T* in,
                 T* out, cudaStream_t stream, bool* ran) {
  *ran = false;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return set_error(LIFTED_ECUDA, "no CUDA device");
  }
  std::string key;
  key.reserve(64 + nimg * sizeof(lifted_image_t));
  char hdr[64];
  std::snprintf(hdr, sizeof(hdr), "%d|%d|%u|%u|", dev, (int)sizeof(T), op, bc);
  key = hdr;
  key.append((const char*)ims, nimg * sizeof(lifted_image_t));
  std::lock_guard<std::mutex> lk(g_nd_mu);
  lifted_batch_plan* plan = nullptr;
  auto it = g_nd_plans.find(key);
  if (it != g_nd_plans.end()) {
    plan = it->second;
  } else {
    // a new plan allocates: not inside a stream capture
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(stream, &cap) != cudaSuccess) cudaGetLastError();
    if (cap != cudaStreamCaptureStatusNone) return LIFTED_OK;
    const int rc = plan_create_nd<T>(op, bc, nimg, ims, nullptr, &plan);
    if (rc) return rc;
    plan->pooled = true;
    if (g_nd_plans.size() >= kNdPlans) {
      const std::string old = g_nd_order.front();
      g_nd_order.erase(g_nd_order.begin());
      lifted_batch_plan* victim = g_nd_plans[old];
      g_nd_plans.erase(old);
      lifted_batch_plan_destroy(victim);  // stream-ordered after its last run
    }
    g_nd_plans[key] = plan;
    g_nd_order.push_back(key);
  }
  *ran = true;
  // the caller checked every image's input against the other images' outputs
  return plan_run<T>(plan, in, out, stream, /*count=*/true, /*spans_checked=*/true);
}

template int run_batch_nd<float>(uint32_t, uint32_t, size_t, const lifted_image_t*,
                                 const float*, float*, cudaStream_t, bool*);
template int run_batch_nd<double>(uint32_t, uint32_t, size_t, const lifted_image_t*,
                                  const double*, double*, cudaStream_t, bool*);

namespace {

// ---------------------------------------------------------------------------
// Autotuner.

template <typename T>
int autotune(uint32_t op, uint32_t bc, size_t nw, const uint32_t* wavelets,
             size_t length, size_t total, cudaStream_t stream) {
  if (!nw || !wavelets || length < 2)
    return set_error(LIFTED_EINVAL, "autotune needs wavelets and a length >= 2");
  const size_t nsig = std::max<size_t>(1, total / length);
  const size_t numel = nsig * length;
  T* din = nullptr;
  T* dout = nullptr;
  cudaError_t e = cudaMalloc(&din, numel * sizeof(T));
  if (e == cudaSuccess) e = cudaMalloc(&dout, numel * sizeof(T));
  if (e == cudaSuccess) e = cudaMemsetAsync(din, 0, numel * sizeof(T), stream);
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (e == cudaSuccess) e = cudaEventCreate(&e0);
  if (e == cudaSuccess) e = cudaEventCreate(&e1);
  int rc = LIFTED_OK;
  if (e != cudaSuccess) rc = set_error(LIFTED_ENOMEM, "autotune buffers: %s", cudaGetErrorString(e));
  const int64_t tiles[] = {2048, 4096, 8192, 16384};
  for (size_t wi = 0; wi < nw && rc == LIFTED_OK; ++wi) {
    std::vector<lifted_signal_t> sig(nsig);
    for (size_t i = 0; i < nsig; ++i) {
      sig[i].wavelet = wavelets[wi];
      sig[i].levels = 0;
      sig[i].length = length;
      sig[i].in_offset = i * length;
      sig[i].out_offset = i * length;
    }
    double best = 1e30;
    TuneVal bv{0, 0, 0};
    bool whole_only = false;
    for (int64_t t : tiles) {
      if (whole_only) break;
      for (int K = 1; K <= 6; ++K) {
        lifted_batch_tuning_t tu{};
        tu.tile = (uint32_t)t;
        tu.tile_levels = (uint32_t)K;
        lifted_batch_plan* p = nullptr;
        if (plan_create<T>(op, bc, nsig, sig.data(), &tu, &p) != LIFTED_OK) {
          clear_error();
          continue;
        }
        if (p->ntile == 0) {  // nothing tiled: the length fits a whole item
          lifted_batch_plan_destroy(p);
          whole_only = true;
          break;
        }
        float ms = 1e30f;
        int r = LIFTED_OK;
        for (int rep = 0; rep < 5 && r == LIFTED_OK; ++rep) {
          cudaEventRecord(e0, stream);
          r = plan_run<T>(p, din, dout, stream);
          cudaEventRecord(e1, stream);
          cudaEventSynchronize(e1);
          float x = 0;
          cudaEventElapsedTime(&x, e0, e1);
          if (rep >= 2) ms = std::min(ms, x);
        }
        lifted_batch_plan_destroy(p);
        if (r != LIFTED_OK) {
          rc = r;
          break;
        }
        if (ms < best) {
          best = ms;
          bv = {(int)t, K, ms * 1e3};
        }
      }
    }
    if (rc == LIFTED_OK && bv.tile) {
      TuneKey k{wavelets[wi], (int)sizeof(T), (int)op, ilog2(length), 1};
      std::lock_guard<std::mutex> g(g_tune_mu);
      g_tune[k] = bv;
    }
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (din) cudaFree(din);
  if (dout) cudaFree(dout);
  return rc;
}

}  // namespace

}  // namespace lw

// ---------------------------------------------------------------------------
// C ABI.
using lw::set_error;

extern "C" {

LIFTED_CAPI int lifted_batch_plan_create_f32(uint32_t op, uint32_t bc, size_t nsignals,
                                             const lifted_signal_t* signals,
                                             const lifted_batch_tuning_t* tuning,
                                             lifted_batch_plan_t** plan) {
  lw::clear_error();
  return lw::plan_create<float>(op, bc, nsignals, signals, tuning, plan);
}
LIFTED_CAPI int lifted_batch_plan_create_f64(uint32_t op, uint32_t bc, size_t nsignals,
                                             const lifted_signal_t* signals,
                                             const lifted_batch_tuning_t* tuning,
                                             lifted_batch_plan_t** plan) {
  lw::clear_error();
  return lw::plan_create<double>(op, bc, nsignals, signals, tuning, plan);
}

LIFTED_CAPI int lifted_batch_plan_create_nd_f32(uint32_t op, uint32_t bc, size_t nimages,
                                                const lifted_image_t* images,
                                                const lifted_batch_tuning_t* tuning,
                                                lifted_batch_plan_t** plan) {
  lw::clear_error();
  if (!plan) return lw::set_error(LIFTED_EINVAL, "null plan pointer");
  return lw::plan_create_nd<float>(op, bc, nimages, images, tuning, plan);
}
LIFTED_CAPI int lifted_batch_plan_create_nd_f64(uint32_t op, uint32_t bc, size_t nimages,
                                                const lifted_image_t* images,
                                                const lifted_batch_tuning_t* tuning,
                                                lifted_batch_plan_t** plan) {
  lw::clear_error();
  if (!plan) return lw::set_error(LIFTED_EINVAL, "null plan pointer");
  return lw::plan_create_nd<double>(op, bc, nimages, images, tuning, plan);
}

LIFTED_CAPI int lifted_batch_run(lifted_batch_plan_t* plan, const void* in, void* out,
                                 void* stream) {
  lw::clear_error();
  if (!plan) return set_error(LIFTED_EINVAL, "null plan");
  return lw::plan_run_any(plan, in, out, (cudaStream_t)stream);
}

LIFTED_CAPI int lifted_batch_run_graph(lifted_batch_plan_t* plan, const void* in, void* out,
                                       void* stream) {
  lw::clear_error();
  if (!plan) return set_error(LIFTED_EINVAL, "null plan");
  return lw::plan_graph(plan, in, out, (cudaStream_t)stream);
}

LIFTED_CAPI int lifted_batch_check(lifted_batch_plan_t* plan, void* stream) {
  lw::clear_error();
  if (!plan) return set_error(LIFTED_EINVAL, "null plan");
  if (plan->items.empty()) return LIFTED_OK;
  cudaError_t e = cudaStreamSynchronize((cudaStream_t)stream);
  int32_t err = 0;
  if (e == cudaSuccess)
    e = cudaMemcpy(&err, plan->d_sync + 1, sizeof(err), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return set_error(LIFTED_ECUDA, "batch check: %s", cudaGetErrorString(e));
  if (err)
    return set_error(LIFTED_ETIMEOUT,
                     "batch item %d gave up waiting for its input band", err - 1);
  return LIFTED_OK;
}

LIFTED_CAPI int lifted_batch_plan_info(const lifted_batch_plan_t* plan,
                                       lifted_batch_info_t* info) {
  if (!plan || !info) return set_error(LIFTED_EINVAL, "null argument");
  info->nsignals = (uint64_t)plan->nsignals;
  info->nitems = (uint64_t)plan->items.size();
  info->ntiles = (uint64_t)plan->ntile;
  info->nwhole = (uint64_t)plan->nwhole;
  info->nwhole_global = (uint64_t)plan->nwhole_global;
  info->ncounters = (uint64_t)plan->ncounters;
  info->scratch_bytes = (uint64_t)plan->scratch_bytes;
  info->shared_bytes = (uint64_t)plan->smem;
  info->grid = (uint32_t)plan->grid;
  info->block = (uint32_t)plan->block;
  return LIFTED_OK;
}

LIFTED_CAPI int lifted_batch_plan_item(const lifted_batch_plan_t* plan, size_t index,
                                       int64_t* fields, size_t nfields) {
  if (!plan || !fields) return set_error(LIFTED_EINVAL, "null argument");
  if (index >= plan->items.size()) return set_error(LIFTED_EINVAL, "item index out of range");
  const lw::BatchItem& it = plan->items[index];
  const int64_t v[] = {it.kind, it.prog, it.sig, it.lev0, it.nlev, it.src_sel,
                       it.dst_sel, it.wait_ctr, it.wait_target, it.done_ctr,
                       it.n0, it.in_off, it.out_off, it.src_off, it.dst_off,
                       it.t0, it.t1, it.halo, it.gbuf, plan->item_phase[index], it.geo};
  const size_t n = sizeof(v) / sizeof(v[0]);
  for (size_t i = 0; i < nfields && i < n; ++i) fields[i] = v[i];
  return LIFTED_OK;
}

LIFTED_CAPI int lifted_batch_plan_geo(const lifted_batch_plan_t* plan, size_t index,
                                      int64_t* fields, size_t nfields) {
  if (!plan || !fields) return set_error(LIFTED_EINVAL, "null argument");
  if (index >= plan->geos.size()) return set_error(LIFTED_EINVAL, "geometry index out of range");
  const lw::BatchAxisGeom& g = plan->geos[index];
  const int64_t v[] = {g.n, g.sa, g.oshape[0], g.oshape[1], g.oshape[2],
                       g.ostride[0], g.ostride[1], g.ostride[2]};
  const size_t n = sizeof(v) / sizeof(v[0]);
  for (size_t i = 0; i < nfields && i < n; ++i) fields[i] = v[i];
  return LIFTED_OK;
}

LIFTED_CAPI void lifted_batch_plan_destroy(lifted_batch_plan_t* plan) {
  if (!plan) return;
  if (plan->gexec) cudaGraphExecDestroy(plan->gexec);
  void* bufs[5] = {plan->d_items, plan->d_progs, plan->d_sync, plan->d_scratch, plan->d_geos};
  if (plan->pooled) {
    // free on the legacy stream after the plan's last run
    if (plan->last) cudaStreamWaitEvent(nullptr, plan->last, 0);
    for (void* b : bufs)
      if (b) cudaFreeAsync(b, nullptr);
  } else {
    for (void* b : bufs)
      if (b) cudaFree(b);
  }
  if (plan->last) cudaEventDestroy(plan->last);
  cudaGetLastError();
  delete plan;
}

#define LW_BATCH_ONESHOT(T, SUF)                                                    \
  LIFTED_CAPI int lifted_lwt_batch_##SUF(uint32_t op, uint32_t bc, size_t nsignals,  \
                                         const lifted_signal_t* signals,            \
                                         const T* in, T* out, void* stream) {        \
    lifted_batch_plan_t* p = nullptr;                                               \
    int rc = lifted_batch_plan_create_##SUF(op, bc, nsignals, signals, nullptr, &p);\
    if (rc) return rc;                                                              \
    rc = lifted_batch_run(p, in, out, stream);                                      \
    if (!rc) rc = lifted_batch_check(p, stream);                                    \
    std::string keep = lw::last_error();                                            \
    lifted_batch_plan_destroy(p);                                                   \
    if (rc) set_error(rc, "%s", keep.c_str());                                      \
    return rc;                                                                      \
  }
LW_BATCH_ONESHOT(float, f32)
LW_BATCH_ONESHOT(double, f64)

LIFTED_CAPI int lifted_batch_autotune(uint32_t dtype_bytes, uint32_t op, uint32_t bc,
                                      size_t nwavelets, const uint32_t* wavelets,
                                      size_t length, size_t total, void* stream) {
  lw::clear_error();
  if (dtype_bytes == 4)
    return lw::autotune<float>(op, bc, nwavelets, wavelets, length, total, (cudaStream_t)stream);
  if (dtype_bytes == 8)
    return lw::autotune<double>(op, bc, nwavelets, wavelets, length, total, (cudaStream_t)stream);
  return set_error(LIFTED_EINVAL, "dtype_bytes must be 4 or 8");
}

LIFTED_CAPI int lifted_batch_tune_save(const char* path) {
  if (!path) return set_error(LIFTED_EINVAL, "null path");
  FILE* f = std::fopen(path, "w");
  if (!f) return set_error(LIFTED_EINVAL, "cannot write %s", path);
  std::lock_guard<std::mutex> g(lw::g_tune_mu);
  std::fprintf(f, "[\n");
  size_t i = 0;
  for (const auto& kv : lw::g_tune) {
    std::fprintf(f,
                 "  {\"wavelet\": %u, \"dtype_bytes\": %d, \"op\": %d, \"log2_length\": %d, "
                 "\"stride\": %lld, \"tile\": %d, \"tile_levels\": %d, \"us\": %.3f}%s\n",
                 kv.first.wavelet, kv.first.dtype, kv.first.op, kv.first.log2len,
                 (long long)kv.first.stride, kv.second.tile, kv.second.levels, kv.second.us,
                 ++i < lw::g_tune.size() ? "," : "");
  }
  std::fprintf(f, "]\n");
  std::fclose(f);
  return LIFTED_OK;
}

LIFTED_CAPI int lifted_batch_tune_load(const char* path, size_t* loaded) {
  if (!path) return set_error(LIFTED_EINVAL, "null path");
  if (loaded) *loaded = 0;
  FILE* f = std::fopen(path, "r");
  if (!f) return set_error(LIFTED_EINVAL, "cannot read %s", path);
  char line[512];
  int n = 0;
  std::lock_guard<std::mutex> g(lw::g_tune_mu);
  while (std::fgets(line, sizeof(line), f)) {
    unsigned w;
    int dt, op, lg, tile, lv;
    long long st;
    double us;
    if (std::sscanf(line,
                    " {\"wavelet\": %u, \"dtype_bytes\": %d, \"op\": %d, \"log2_length\": %d, "
                    "\"stride\": %lld, \"tile\": %d, \"tile_levels\": %d, \"us\": %lf",
                    &w, &dt, &op, &lg, &st, &tile, &lv, &us) == 8) {
      if (tile < 2 || lv < 1 || lv > lw::MAX_LEVELS) continue;
      lw::g_tune[{w, dt, op, lg, (int64_t)st}] = {tile, lv, us};
      ++n;
    }
  }
  std::fclose(f);
  if (loaded) *loaded = (size_t)n;
  return LIFTED_OK;
}

LIFTED_CAPI void lifted_batch_tune_clear(void) {
  std::lock_guard<std::mutex> g(lw::g_tune_mu);
  lw::g_tune.clear();
}

}  // extern "C"
