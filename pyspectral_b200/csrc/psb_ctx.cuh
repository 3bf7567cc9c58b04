// Host-side context shared by the translation units of libpyspectral_b200:
// grid constants, FFT plans and twiddle pools, wavenumber/mask tables on the
// device, the scratch arena and launch helpers.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <type_traits>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/pyspectral_b200.h"
#include "psb_physics.cuh"

// Launch shape of one pass picked by the autotuner: tile (columns per CTA, or
// pencils per CTA for the z pass), its transform's radix order, and whether
// that order needs the wide (radix 6/12/16) kernels.
struct psb_pass_shape {
  int tile = 0;
  psb::FFTPlan plan{};
  bool wide = false;
};
// Shapes of the five passes (x-inverse, y-inverse, z, y-forward, x-forward) of
// a 3/2-padded closure's RHS.
struct psb_tuned {
  psb_pass_shape pass[5];
};

struct psb_ctx {
  int N1 = 0, N2 = 0, N3 = 0, N3h = 0;
  int prec = 64;
  int dev = 0;
  cudaStream_t stream = nullptr;
  double L1 = 0, L2 = 0, L3 = 0, dx = 0, dy = 0, dz = 0, Delta = 0;
  int kc = 0;
  // device tables (double): N grid, 2x grid, MHD dealias masks, Gf masks
  double *kx = nullptr, *ky = nullptr, *kz = nullptr;
  double *kxf = nullptr, *kyf = nullptr, *kzf = nullptr;
  double *mx = nullptr, *my = nullptr, *mz = nullptr;
  double *gx = nullptr, *gy = nullptr, *gz = nullptr;
  int kz_mhd = 0;  // retained k3 count of the 2/3 rule
  int dtau_kf = -1;  // test-filter wavenumber of the cached dynamic-tau masks
  int dsmag_kl = -1;  // test-filter cutoff of the cached dynamic-Smagorinsky masks
  void* tw_d = nullptr;  // Cx<double> pool
  void* tw_f = nullptr;  // Cx<float> pool
  std::map<int, psb::FFTPlan> plans;
  struct Buf {
    void* p = nullptr;
    size_t bytes = 0;
  };
  std::map<std::string, Buf> scratch;
  std::map<int, psb_tuned> tuned;  // autotuned launch shapes by closure (psb_autotune)
  double* red_dev = nullptr;   // reduction partials
  double* red_host = nullptr;  // pinned
  size_t red_cap = 0;
  std::string err;
  std::vector<void*> owned;  // table allocations
  // launch accounting: every kernel launch counts; with timing on, each
  // launch is bracketed by CUDA events on the context stream and tagged
  // with its compulsory HBM bytes (inputs read once + outputs written once)
  unsigned long long launches = 0;
  int timing = 0;
  int use_tma = 1;          // stage eligible pass inputs with bulk tensor copies
  int use_zrr = 1;          // register-direct z-pass for two-pass (R1, 16) schedules
  int* dstatus = nullptr;   // device status word (a bounded wait gave up), owned
  struct Rec {
    std::string name;
    double bytes;
    cudaEvent_t a, b;
  };
  std::vector<Rec> recs;
  std::vector<cudaEvent_t> ev_free;
};

namespace psbh {

using psb::Cx;
using psb::FFTPlan;

inline int fail(psb_ctx* c, int code, const std::string& msg) {
  c->err = msg;
  return code;
}

inline int cuda_ok(psb_ctx* c, cudaError_t e, const char* what) {
  if (e == cudaSuccess) return PSB_OK;
  return fail(c, PSB_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

inline int launch_ok(psb_ctx* c, const char* what) { return cuda_ok(c, cudaGetLastError(), what); }

#define PSB_TRY(expr)              \
  do {                             \
    int _s = (expr);               \
    if (_s != PSB_OK) return _s;   \
  } while (0)

inline const FFTPlan* plan_for(psb_ctx* c, int L) {
  auto it = c->plans.find(L);
  return it == c->plans.end() ? nullptr : &it->second;
}

template <typename T>
inline const Cx<T>* twiddles(psb_ctx* c) {
  return reinterpret_cast<const Cx<T>*>(sizeof(T) == 8 ? c->tw_d : c->tw_f);
}

// Named scratch buffer of at least `n` complex elements (grows; contents undefined).
template <typename T>
inline Cx<T>* scratch(psb_ctx* c, const char* name, size_t n, int* status) {
  const size_t bytes = n * sizeof(Cx<T>);
  auto& b = c->scratch[name];
  if (b.bytes < bytes) {
    if (b.p) cudaFree(b.p);
    b.p = nullptr;
    b.bytes = 0;
    cudaError_t e = cudaMalloc(&b.p, bytes);
    if (e != cudaSuccess) {
      *status = fail(c, PSB_ERR_CUDA, std::string("scratch ") + name + ": " + cudaGetErrorString(e));
      return nullptr;
    }
    b.bytes = bytes;
  }
  return reinterpret_cast<Cx<T>*>(b.p);
}

inline cudaEvent_t take_event(psb_ctx* c) {
  if (!c->ev_free.empty()) {
    cudaEvent_t e = c->ev_free.back();
    c->ev_free.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}

// Bracket one kernel launch: count it and, when timing is on, record events.
struct LaunchScope {
  psb_ctx* c;
  psb_ctx::Rec rec;
  bool on;
  LaunchScope(psb_ctx* ctx, const char* name, double bytes) : c(ctx), on(ctx->timing != 0) {
    ++c->launches;
    if (on) {
      rec.name = name;
      rec.bytes = bytes;
      rec.a = take_event(c);
      rec.b = take_event(c);
      cudaEventRecord(rec.a, c->stream);
    }
  }
  ~LaunchScope() {
    if (on) {
      cudaEventRecord(rec.b, c->stream);
      c->recs.push_back(rec);
    }
  }
};

// Boxes of rows of a TMA-staged pass: the fewest that divide L with at most 256 rows each.
inline int tma_boxes(int L) {
  for (int nb = 1; nb <= 8; ++nb)
    if (L % nb == 0 && L / nb <= 256) return nb;
  return 0;
}

inline int count_mapped(const psb::RowMap& m, int rows) {
  int n = 0;
  for (int i = 0; i < rows; ++i) n += m.lo > i ? 1 : (i >= m.hi ? 1 : 0);
  return n;
}

constexpr size_t kSmemBudget = 100 * 1024;

// Raise a kernel's dynamic shared-memory limit once per (kernel, device); a
// fixed table, so that launching never allocates host memory either.  The
// table is process-wide and shared by every context, so it is guarded by a
// mutex: host threads that launch on different contexts may meet here.
struct SmemCache {
  const void* fn[512];
  int dev[512];
  size_t bytes[512];
  int n = 0;
  std::mutex mu;
};
inline SmemCache& smem_cache() {
  static SmemCache c;
  return c;
}
template <typename K>
inline void set_smem(K kernel, size_t smem) {
  if (smem <= 48 * 1024) return;
  int dev = 0;
  cudaGetDevice(&dev);
  SmemCache& c = smem_cache();
  const void* f = reinterpret_cast<const void*>(kernel);
  std::lock_guard<std::mutex> lk(c.mu);
  for (int i = 0; i < c.n; ++i)
    if (c.fn[i] == f && c.dev[i] == dev) {
      if (c.bytes[i] >= smem) return;
      cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      c.bytes[i] = smem;
      return;
    }
  cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (c.n < 512) {
    c.fn[c.n] = f;
    c.dev[c.n] = dev;
    c.bytes[c.n] = smem;
    ++c.n;
  }
}

// Launch of a pipeline kernel (axis, z and x-forward passes) with
// programmatic stream serialisation: it may start while the previous kernel
// in the stream drains; the kernels wait for their predecessor (pdl_wait)
// before touching pipeline data.
template <typename... KArgs, typename... Args>
inline cudaError_t launch_pdl(void (*kernel)(KArgs...), dim3 grid, int block, size_t smem, cudaStream_t stream,
                              Args... args) {
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = grid;
  cfg.blockDim = dim3((unsigned)block);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, args...);
}

// Grid of a persistent kernel: at most (resident CTAs per SM) x SMs of the
// current device, and no more CTAs than there are tiles.  The kernel asks for
// the largest shared-memory carveout first: under 48 KB per CTA the default
// carveout would otherwise leave room for fewer CTAs than the registers and
// shared memory allow (one per SM was seen).  Results are cached per
// (kernel, device, shared memory) in a fixed table.
struct OccCache {
  const void* fn[256];
  int dev[256];
  size_t smem[256];
  int per[256], nsm[256];
  int n = 0;
};
inline OccCache& occ_cache() {
  static OccCache c;
  return c;
}
template <typename K>
inline long long persistent_grid(K kernel, size_t smem, long long ntiles) {
  int dev = 0;
  cudaGetDevice(&dev);
  OccCache& oc = occ_cache();
  const void* f = reinterpret_cast<const void*>(kernel);
  for (int i = 0; i < oc.n; ++i)
    if (oc.fn[i] == f && oc.dev[i] == dev && oc.smem[i] == smem)
      return std::min<long long>(ntiles, (long long)oc.per[i] * oc.nsm[i]);
  int nsm = 0, per = 0;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout, (int)cudaSharedmemCarveoutMaxShared);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, 256, smem) != cudaSuccess || per < 1 || nsm < 1) {
    (void)cudaGetLastError();
    return ntiles;
  }
  if (oc.n < 256) {
    oc.fn[oc.n] = f;
    oc.dev[oc.n] = dev;
    oc.smem[oc.n] = smem;
    oc.per[oc.n] = per;
    oc.nsm[oc.n] = nsm;
    ++oc.n;
  }
  return std::min<long long>(ntiles, (long long)per * nsm);
}

inline int pow2_floor(int x) {
  int p = 1;
  while (p * 2 <= x) p *= 2;
  return p;
}

// columns per CTA for strided passes
// nouter > 0: also shrink the tile until the grid has ~2 CTAs per SM (148 SMs)
inline int pick_ct(int ncols, int F, int L, size_t esz, int nouter = 0) {
  int ct = 32;
  int cap = pow2_floor(ncols < 1 ? 1 : ncols);
  if (ncols > cap) cap *= 2;
  if (ct > cap) ct = cap;
  while (ct > 1 && (size_t)(L + 2 * L * F * ct) * esz > kSmemBudget) ct /= 2;
  if (nouter > 0)
    while (ct > 4 && (long long)((ncols + ct - 1) / ct) * nouter < 2 * 148) ct /= 2;
  return ct;
}

// radix 6/12/16 passes need the wide kernel instantiations
inline bool plan_is_wide_h(const psb::FFTPlan& p) {
  for (int s = 0; s < p.npass; ++s)
    if (p.radix[s] > 8 || p.radix[s] == 6) return true;
  return false;
}

// sh: an autotuned shape (TUNABLE launch sites only) or null for the default
template <typename T, bool INV, class Pre, bool TUNABLE = false>
int launch_axis(psb_ctx* c, psb::AxisArgs<T> a, Pre pre, const char* what, const psb_pass_shape* sh = nullptr) {
  const size_t esz = sizeof(Cx<T>);
  const int L = a.plan.L;
  a.col_tile = pick_ct(a.ncols, Pre::F_DST, L, esz, a.nouter);
  if (sh && sh->tile) {
    a.col_tile = sh->tile;
    a.plan = sh->plan;
  }
  const size_t smem = (size_t)(L + 2 * L * Pre::F_DST * a.col_tile) * esz;
  dim3 grid((a.ncols + a.col_tile - 1) / a.col_tile, a.nouter);
  const double bytes = (double)esz * a.nouter * a.ncols *
                       ((double)Pre::F_SRC * count_mapped(a.in_map, a.in_rows) + (double)Pre::F_DST * a.out_rows);
  auto go = [&](auto k) {
    set_smem(k, smem);
    LaunchScope scope(c, what, bytes);
    launch_pdl(k, grid, 256, smem, c->stream, a, pre);
    return launch_ok(c, what);
  };
  // A compiled two-pass schedule on a tunable pass whose Pre forms each field
  // on load: registers straight from and to global memory around a single
  // shared-memory exchange (psb::axis_rr_body).
  if constexpr (TUNABLE && psb::pre_fieldwise<Pre>::value) {
    const size_t rsmem = (size_t)(L + (size_t)L * Pre::F_DST * a.col_tile) * esz;
    auto gor = [&](auto k) {
      set_smem(k, rsmem);
      LaunchScope scope(c, what, bytes);
      launch_pdl(k, grid, 256, rsmem, c->stream, a, pre);
      return launch_ok(c, what);
    };
    switch (psb::fixed_plan_id(a.plan)) {
#define PSB_FIXED_CASE(ID, ...)                                                                       \
  case ID:                                                                                            \
    if constexpr (psb::fixed_plan_compiled<T, ID>::value && psb::FixedPlan<ID>::Radices::NP == 2) \
      return gor(psb::axis_pass_rr_kernel<T, INV, Pre, ID>);                                          \
    break;
      PSB_FIXED_PLANS(PSB_FIXED_CASE)
#undef PSB_FIXED_CASE
      default:
        break;
    }
  }
  // Rows read unchanged (a plain copy, every row at its own position): the
  // tile is staged by bulk tensor copies when the view meets TMA's rules.
  if constexpr (std::is_same<Pre, psb::PreCopy<T>>::value) {
    const int nbox = tma_boxes(L);
    CUtensorMap map;
    const bool plain_rows = a.in_rows == L && a.in_map.lo >= L;
    // every box lands on a 128-byte boundary: the buffer's start, and box b at b*(L/nbox) rows
    const bool boxes_aligned = nbox == 1 || ((size_t)(L / nbox) * a.col_tile * esz) % 128 == 0;
    if (c->use_tma && plain_rows && nbox > 0 && boxes_aligned && (a.col_tile * esz) % 16 == 0 &&
        !(sh && sh->wide)) {
      const long long dims[4] = {a.ncols, 1, a.in_rows, a.nouter};
      const long long strides[3] = {a.in_rstride, a.in_rstride, a.in_ostride};
      const int box[4] = {a.col_tile, 1, L / nbox, 1};
      if (tma::encode4d(&map, a.in, (int)esz, dims, strides, box)) {
        const size_t tsmem = psb::tma_buf_offset<T>(L) + (size_t)2 * L * a.col_tile * esz;
        auto got = [&](auto k) {
          set_smem(k, tsmem);
          LaunchScope scope(c, what, bytes);
          launch_pdl(k, grid, 256, tsmem, c->stream, a, map, nbox, c->dstatus);
          return launch_ok(c, what);
        };
        switch (psb::fixed_plan_id(a.plan)) {
#define PSB_FIXED_CASE(ID, ...) \
  case ID:                      \
    if constexpr (psb::fixed_plan_compiled<T, ID>::value) return got(psb::axis_pass_tma_kernel<T, INV, ID>); \
    break;
          PSB_FIXED_PLANS(PSB_FIXED_CASE)
#undef PSB_FIXED_CASE
          default:
            break;
        }
        if (!plan_is_wide_h(a.plan)) return got(psb::axis_pass_tma_kernel<T, INV, 0>);
      }
    }
  }
  if constexpr (TUNABLE) {
    switch (psb::fixed_plan_id(a.plan)) {
#define PSB_FIXED_CASE(ID, ...) \
  case ID:                      \
    if constexpr (psb::fixed_plan_compiled<T, ID>::value) return go(psb::axis_pass_kernel<T, INV, Pre, false, ID>); \
    break;
      PSB_FIXED_PLANS(PSB_FIXED_CASE)
#undef PSB_FIXED_CASE
      default:
        break;
    }
    if (sh && sh->wide) return go(psb::axis_pass_kernel<T, INV, Pre, true>);
  }
  return go(psb::axis_pass_kernel<T, INV, Pre>);
}

template <typename T, class Phys, bool TUNABLE = false>
int launch_z(psb_ctx* c, psb::ZArgs<T> z, Phys phys, const char* what, double extra_bytes = 0.0,
             const psb_pass_shape* sh = nullptr) {
  const size_t esz = sizeof(Cx<T>);
  const int M = z.plan.L;
  constexpr int FMAX = Phys::F_IN > Phys::F_OUT ? Phys::F_IN : Phys::F_OUT;
  constexpr size_t extra = (size_t)psb::phys_is_block<Phys>::extra;
  (void)esz;
  auto smem_for = [&](int P) { return psb::zpass_smem_bytes<T>(FMAX, P, M, extra); };
  int P = psb::phys_default_ppc<Phys>::value;
  while (P > 1 && smem_for(P) > kSmemBudget) P /= 2;
  while (P > 1 && (z.npencils + P - 1) / P < 2 * 148) P /= 2;
  if (sh && sh->tile) {
    P = sh->tile;
    z.plan = sh->plan;
  } else if constexpr (psb::phys_fixed_fft<Phys>::value && sizeof(T) == 4) {
    // default shape: the register-direct z pass where its schedule exists
    if ((P & 1) == 0 && c->use_zrr) psb::zrr_default_plan(z.plan);
  }
  z.ppc = P;
  const size_t smem = smem_for(P);
  const long long grid = (z.npencils + P - 1) / P;
  double bytes = extra_bytes + (double)esz * z.npencils * Phys::F_OUT * z.out_kz;
  // a field formed as d/dz of another input re-reads that input's line: no new bytes
  for (int f = 0; f < Phys::F_IN; ++f)
    if (!z.dz[f]) bytes += (double)esz * z.npencils * z.in_kz[f];
  auto go = [&](auto k) {
    set_smem(k, smem);
    const long long g = persistent_grid(k, smem, grid);
    LaunchScope scope(c, what, bytes);
    launch_pdl(k, dim3((unsigned)g), 256, smem, c->stream, z, phys);
    return launch_ok(c, what);
  };
  // A compiled two-pass schedule (R1, 16) with pencils paired per packed line
  // (P even): the register-direct z-pass, whose transforms read the packed
  // spectra from and write them to global memory (psb::zpass_rr_tile).
  if constexpr (psb::phys_fixed_fft<Phys>::value && sizeof(T) == 4) {
    if ((P & 1) == 0 && c->use_zrr) {
      switch (psb::fixed_plan_id(z.plan)) {
#define PSB_FIXED_CASE(ID, ...)                                                                   \
  case ID:                                                                                        \
    if constexpr (psb::zrr_plan<ID>::value && psb::zrr_plan<ID>::R2 == 16)                      \
      return go(psb::zpass_rr_kernel<T, Phys, ID>);                                               \
    break;
        PSB_FIXED_PLANS(PSB_FIXED_CASE)
#undef PSB_FIXED_CASE
        default:
          break;
      }
    }
  }
  if constexpr (psb::phys_fixed_fft<Phys>::value) {
    switch (psb::fixed_plan_id(z.plan)) {
#define PSB_FIXED_CASE(ID, ...) \
  case ID:                      \
    if constexpr (psb::fixed_plan_compiled<T, ID>::value) return go(psb::zpass_kernel<T, Phys, false, ID>); \
    break;
      PSB_FIXED_PLANS(PSB_FIXED_CASE)
#undef PSB_FIXED_CASE
      default:
        break;
    }
  }
  if constexpr (TUNABLE) {
    if (sh && sh->wide) return go(psb::zpass_kernel<T, Phys, true>);
  }
  return go(psb::zpass_kernel<T, Phys>);
}

// bytes: the transform input plus the epilogue's own state traffic (epi.io_bytes)
template <typename T, class Epi, bool TUNABLE = false>
int launch_epi(psb_ctx* c, psb::XEpiArgs<T> e, Epi epi, const char* what, const psb_pass_shape* sh = nullptr) {
  const size_t esz = sizeof(Cx<T>);
  const int L = e.plan.L;
  e.col_tile = pick_ct(e.kz, Epi::F_IN, L, esz, e.n2);
  if (sh && sh->tile) {
    e.col_tile = sh->tile;
    e.plan = sh->plan;
  }
  const int ntile = (e.kz + e.col_tile - 1) / e.col_tile;
  e.main_blocks = ntile * e.n2;
  int extra = 0;
  if (e.n3h > e.kz) {
    const long long pts = (long long)e.n1 * e.n2 * (e.n3h - e.kz);
    extra = (int)std::min<long long>((pts + 255) / 256, 1024);
  }
  const size_t smem = (size_t)(L + 2 * L * Epi::F_IN * e.col_tile) * esz;
  const double bytes = epi.io_bytes((long long)e.n1 * e.n2 * e.n3h) + (double)esz * Epi::F_IN * L * e.n2 * e.kz;
  auto go = [&](auto k) {
    set_smem(k, smem);
    LaunchScope scope(c, what, bytes);
    launch_pdl(k, dim3((unsigned)(e.main_blocks + extra)), 256, smem, c->stream, e, epi);
    return launch_ok(c, what);
  };
  // a compiled two-pass schedule: the first pass loads straight from global memory
  if constexpr (TUNABLE) {
    switch (psb::fixed_plan_id(e.plan)) {
#define PSB_FIXED_CASE(ID, ...)                                                                       \
  case ID:                                                                                            \
    if constexpr (psb::fixed_plan_compiled<T, ID>::value && psb::FixedPlan<ID>::Radices::NP == 2) \
      return go(psb::xfwd_epi_rr_kernel<T, Epi, ID>);                                                 \
    break;
      PSB_FIXED_PLANS(PSB_FIXED_CASE)
#undef PSB_FIXED_CASE
      default:
        break;
    }
  }
  // the input tile (ct columns x F fields x L rows) staged by bulk tensor copies
  {
    const int nbox = tma_boxes(L);
    CUtensorMap map;
    const bool boxes_aligned = nbox == 1 || ((size_t)(L / nbox) * Epi::F_IN * e.col_tile * esz) % 128 == 0;
    if (c->use_tma && nbox > 0 && boxes_aligned && (e.col_tile * esz) % 16 == 0 && !(sh && sh->wide)) {
      const long long dims[4] = {e.kz, Epi::F_IN, L, e.n2};
      const long long strides[3] = {e.in_fstride, e.in_rstride, e.in_ostride};
      const int box[4] = {e.col_tile, Epi::F_IN, L / nbox, 1};
      if (tma::encode4d(&map, e.in, (int)esz, dims, strides, box)) {
        const size_t tsmem = psb::tma_buf_offset<T>(L) + (size_t)2 * L * Epi::F_IN * e.col_tile * esz;
        auto got = [&](auto k) {
          set_smem(k, tsmem);
          LaunchScope scope(c, what, bytes);
          launch_pdl(k, dim3((unsigned)(e.main_blocks + extra)), 256, tsmem, c->stream, e, epi, map, nbox,
                     c->dstatus);
          return launch_ok(c, what);
        };
        switch (psb::fixed_plan_id(e.plan)) {
#define PSB_FIXED_CASE(ID, ...) \
  case ID:                      \
    if constexpr (psb::fixed_plan_compiled<T, ID>::value) return got(psb::xfwd_epi_tma_kernel<T, Epi, ID>); \
    break;
          PSB_FIXED_PLANS(PSB_FIXED_CASE)
#undef PSB_FIXED_CASE
          default:
            break;
        }
        if (!plan_is_wide_h(e.plan)) return got(psb::xfwd_epi_tma_kernel<T, Epi, 0>);
      }
    }
  }
  if constexpr (TUNABLE) {
    switch (psb::fixed_plan_id(e.plan)) {
#define PSB_FIXED_CASE(ID, ...) \
  case ID:                      \
    if constexpr (psb::fixed_plan_compiled<T, ID>::value) return go(psb::xfwd_epi_kernel<T, Epi, false, ID>); \
    break;
      PSB_FIXED_PLANS(PSB_FIXED_CASE)
#undef PSB_FIXED_CASE
      default:
        break;
    }
    if (sh && sh->wide) return go(psb::xfwd_epi_kernel<T, Epi, true>);
  }
  return go(psb::xfwd_epi_kernel<T, Epi>);
}

// The fewest-pass schedule of n over radices {16, 12, 8, 6, 4, 3, 2}.
inline std::vector<int> fewest_passes(int n) {
  if (n == 1) return {};
  std::vector<int> best;
  bool found = false;
  for (int r : {16, 12, 8, 6, 4, 3, 2}) {
    if (n % r) continue;
    std::vector<int> rest = fewest_passes(n / r);
    if (n / r != 1 && rest.empty()) continue;
    rest.insert(rest.begin(), r);
    if (!found || rest.size() < best.size()) {
      best = rest;
      found = true;
    }
  }
  return best;
}

// Candidate schedules of a length: every order of the default schedule's
// radices and of the fewest-pass schedule's (distinct permutations).
inline std::vector<FFTPlan> radix_orders(const FFTPlan& p) {
  std::vector<FFTPlan> out;
  auto add_perms = [&](std::vector<int> r) {
    std::sort(r.begin(), r.end());
    int n = 0;
    do {
      FFTPlan q = p;
      q.npass = (int)r.size();
      for (int s = 0; s < q.npass; ++s) q.radix[s] = r[s];
      bool dup = false;
      for (const FFTPlan& o : out)
        if (o.npass == q.npass && std::equal(o.radix, o.radix + o.npass, q.radix)) dup = true;
      if (!dup) out.push_back(q);
    } while (std::next_permutation(r.begin(), r.end()) && ++n < 24);
  };
  add_perms(std::vector<int>(p.radix, p.radix + p.npass));
  add_perms(fewest_passes(p.L));
  // every other two-pass schedule with radices 6..16 (e.g. 12 x 8 beside 16 x 6)
  for (int r : {16, 12, 8, 6})
    if (p.L % r == 0 && p.L / r != r) {
      const int q = p.L / r;
      if (q == 16 || q == 12 || q == 8 || q == 6) add_perms({r, q});
    }
  return out;
}

// z-pass inputs of a 3/2-padded pipeline: NIN fields from the y-pass output B
// (field stride fsP, Kz stored k3 per pencil), with the z derivatives a Pre
// leaves to the z-pass (pre_z_derived) formed from their stored field.
template <typename T, class Pre, int NIN>
void set_z_inputs(psb::ZArgs<T>& z, const Cx<T>* B, long long fsP, int Kz, const double* k3) {
  static_assert(NIN == psb::pre_b_fields<Pre>::value + psb::pre_z_derived<Pre>::value, "z-pass inputs mismatch");
  for (int f = 0; f < NIN; ++f) {
    int src = f;
    bool der = false;
    if constexpr (psb::pre_z_derived<Pre>::value > 0) Pre::zsrc(f, src, der);
    z.in[f] = B + src * fsP;
    z.in_pstride[f] = Kz;
    z.in_kz[f] = Kz;
    z.dz[f] = der ? 1 : 0;
  }
  z.k3 = k3;
}

inline psb::RowMap map_id(int L) { return psb::RowMap{L, L, 0}; }
// pad/unpad (3/2): drops index N/2 (PySpectral/src/padding.py:2-25)
inline psb::RowMap map_pad32(int N) { return psb::RowMap{N / 2, N / 2 + 1, 3 * N / 2 - N}; }
// pad_2x/unpad_2x: keeps N/2 as the -N/2 mode (PySpectral/src/padding.py:28-49)
inline psb::RowMap map_pad2x(int N) { return psb::RowMap{N / 2, N / 2, N}; }
// unpad(pad()) followed by pad_2x: Nyquist dropped, upper half shifted by N
inline psb::RowMap map_pad2x_nyq0(int N) { return psb::RowMap{N / 2, N / 2 + 1, N}; }

}  // namespace psbh
