// Batched ensembles: many independent runs of one grid size, precision and
// closure advanced together, every pass of the RK4 step one launch over all
// runs (the run index is a grid dimension; each run reads its own argument
// block from device memory).  No counterpart in the reference, which advances
// one run per process (PySpectral/src/PySpec_3d.py:96-144).
//
// Launch shapes are chosen by an autotuner: for every pass it times the
// candidate column tiles (x/y passes), pencils per CTA (z-pass) and radix
// orders of the transform length on the batch's own data, and keeps the
// fastest.  Timing reads the runs' states and writes only scratch (the last
// pass runs a middle-stage update on scratch copies), so tuning leaves the
// runs' states untouched.
#include <algorithm>
#include <array>
#include <type_traits>
#include <cstring>

#include "psb_ctx.cuh"
#include "psb_grid.cuh"

using namespace psb;
using namespace psbh;

struct psb_batch {
  psb_ctx* c = nullptr;
  int closure = 0;
  int nruns = 0;
  std::vector<void*> state, comp;
  std::vector<psb_params> params;
  void* arena = nullptr;  // per-run scratch: A, B, C, D, Q0, RHS (tuning)
  size_t arena_bytes = 0;
  void* dargs = nullptr;  // device argument blocks
  size_t dargs_bytes = 0;
  bool dirty = true;
  // launch shape per pass: 0 x-inverse, 1 y-inverse, 2 z, 3 y-forward, 4 x-forward
  std::array<int, 5> tile{{0, 0, 0, 0, 0}};
  std::array<FFTPlan, 5> plan{};
  bool tuned = false;
  std::vector<char> host;  // staging of the argument blocks
};

namespace {

template <typename T>
KTabs<T> ktab(const double* a, const double* b, const double* c) {
  KTabs<T> k;
  k.k1 = a;
  k.k2 = b;
  k.k3 = c;
  return k;
}

// Sizes of one run's buffers (complex elements).
struct Dims {
  int N1, N2, N3, N3h, M1, M2, M3, Kz;
  long long nA, nB, nC, nD, nQ;
};
// Fi / Fb: fields after the x / y pass, Fo: z-pass outputs
Dims dims(const psb_ctx* c, int Fi, int Fb, int Fo) {
  Dims d;
  d.N1 = c->N1;
  d.N2 = c->N2;
  d.N3 = c->N3;
  d.N3h = c->N3h;
  d.M1 = 3 * d.N1 / 2;
  d.M2 = 3 * d.N2 / 2;
  d.M3 = 3 * d.N3 / 2;
  d.Kz = d.N3 / 2;
  d.nA = (long long)Fi * d.M1 * d.N2 * d.Kz;
  d.nB = (long long)Fb * d.M1 * d.M2 * d.Kz;
  d.nC = (long long)Fo * d.M1 * d.M2 * d.Kz;
  d.nD = (long long)Fo * d.M1 * d.N2 * d.Kz;
  d.nQ = 3LL * d.N1 * d.N2 * d.N3h;
  return d;
}
long long al(long long n) { return (n + 63) / 64 * 64; }

template <typename T, class Pre, class Phys, class Epi>
struct Batch {
  static constexpr int Fi = Pre::F_DST, Fb = pre_b_fields<Pre>::value, Fo = Phys::F_OUT;
  using YP = pre_ypass<T, Pre>;
  using YPre = typename YP::type;
  psb_batch* b;
  psb_ctx* c;
  Dims d;
  int R;
  // device views
  AxisArgs<T>*ax, *ay, *ayf;
  ZArgs<T>* az;
  XEpiArgs<T>* ae;
  Pre* pre;
  YPre* ypre;  // y-inverse pass
  PreCopy<T>* cpy;
  Phys* phys;
  Epi* epi;  // [5][R]: stages 0..3, then a middle stage on scratch copies (tuning)

  static size_t arg_bytes(int R) {
    return al(sizeof(AxisArgs<T>) * R) * 3 + al(sizeof(ZArgs<T>) * R) + al(sizeof(XEpiArgs<T>) * R) +
           al(sizeof(Pre) * R) + al(sizeof(YPre) * R) + al(sizeof(PreCopy<T>) * R) + al(sizeof(Phys) * R) +
           al(sizeof(Epi) * R * 5);
  }
  static size_t run_bytes(const Dims& d) { return sizeof(Cx<T>) * (al(d.nA) + al(d.nB) + al(d.nC) + al(d.nD) + 2 * al(d.nQ)); }

  Cx<T>* run_buf(int r, int which) const {
    Cx<T>* base = reinterpret_cast<Cx<T>*>(reinterpret_cast<char*>(b->arena) + (size_t)r * run_bytes(d));
    const long long off[6] = {0, al(d.nA), al(d.nA) + al(d.nB), al(d.nA) + al(d.nB) + al(d.nC),
                              al(d.nA) + al(d.nB) + al(d.nC) + al(d.nD),
                              al(d.nA) + al(d.nB) + al(d.nC) + al(d.nD) + al(d.nQ)};
    return base + off[which];
  }

  void views(char* base) {
    char* p = base;
    auto take = [&](size_t n) {
      char* q = p;
      p += al(n);
      return q;
    };
    ax = reinterpret_cast<AxisArgs<T>*>(take(sizeof(AxisArgs<T>) * R));
    ay = reinterpret_cast<AxisArgs<T>*>(take(sizeof(AxisArgs<T>) * R));
    ayf = reinterpret_cast<AxisArgs<T>*>(take(sizeof(AxisArgs<T>) * R));
    az = reinterpret_cast<ZArgs<T>*>(take(sizeof(ZArgs<T>) * R));
    ae = reinterpret_cast<XEpiArgs<T>*>(take(sizeof(XEpiArgs<T>) * R));
    pre = reinterpret_cast<Pre*>(take(sizeof(Pre) * R));
    ypre = reinterpret_cast<YPre*>(take(sizeof(YPre) * R));
    cpy = reinterpret_cast<PreCopy<T>*>(take(sizeof(PreCopy<T>) * R));
    phys = reinterpret_cast<Phys*>(take(sizeof(Phys) * R));
    epi = reinterpret_cast<Epi*>(take(sizeof(Epi) * R * 5));
  }

  // Argument blocks of every run (host copy, then one upload).
  int build(const Pre& pre0, Phys (*mkphys)(psb_ctx*, const psb_params&),
            Epi (*mkepi)(psb_ctx*, StepIO<T>, const psb_params&)) {
    const size_t ab = arg_bytes(R);
    b->host.assign(ab, 0);
    views(b->host.data());
    const long long fsN = (long long)d.N1 * d.N2 * d.N3h;
    const double s32 = std::sqrt(std::pow(1.5, 3) * std::sqrt((double)d.N1 * d.N2 * d.N3));
    const double rk[4] = {1. / 4, 1. / 3, 1. / 2, 1.};
    for (int r = 0; r < R; ++r) {
      const Cx<T>* Q = reinterpret_cast<const Cx<T>*>(b->state[r]);
      Cx<T>*A = run_buf(r, 0), *B = run_buf(r, 1), *C = run_buf(r, 2), *D = run_buf(r, 3);
      AxisArgs<T> a{};
      a.plan = b->plan[0];
      a.tw = twiddles<T>(c);
      a.scale = (T)1;
      a.in = Q;
      a.out = A;
      a.in_fstride = fsN;
      a.in_ostride = d.N3h;
      a.in_rstride = (long long)d.N2 * d.N3h;
      a.out_fstride = (long long)d.M1 * d.N2 * d.Kz;
      a.out_ostride = d.Kz;
      a.out_rstride = (long long)d.N2 * d.Kz;
      a.nouter = d.N2;
      a.ncols = d.Kz;
      a.col_tile = b->tile[0];
      a.in_rows = d.N1;
      a.out_rows = d.M1;
      a.in_map = map_pad32(d.N1);
      a.out_map = map_id(d.M1);
      a.k_row = c->kx;
      a.k_outer = c->ky;
      a.k_col = c->kz;
      ax[r] = a;
      AxisArgs<T> y{};
      y.plan = b->plan[1];
      y.tw = twiddles<T>(c);
      y.scale = (T)1;
      y.in = A;
      y.out = B;
      y.in_ostride = (long long)d.N2 * d.Kz;
      y.in_rstride = d.Kz;
      y.out_ostride = (long long)d.M2 * d.Kz;
      y.out_rstride = d.Kz;
      y.nouter = YP::groups * d.M1;
      y.in_fstride = (long long)YP::in_fields * d.M1 * d.N2 * d.Kz;
      y.out_fstride = (long long)YP::out_fields * d.M1 * d.M2 * d.Kz;
      y.k_row = c->ky;
      y.ncols = d.Kz;
      y.col_tile = b->tile[1];
      y.in_rows = d.N2;
      y.out_rows = d.M2;
      y.in_map = map_pad32(d.N2);
      y.out_map = map_id(d.M2);
      ay[r] = y;
      ZArgs<T> z{};
      const long long fsP = (long long)d.M1 * d.M2 * d.Kz;
      set_z_inputs<T, Pre, Phys::F_IN>(z, B, fsP, d.Kz, c->kz);
      for (int g = 0; g < Fo; ++g) {
        z.out[g] = C + g * fsP;
        z.out_pstride[g] = d.Kz;
      }
      z.out_kz = d.Kz;
      z.npencils = (long long)d.M1 * d.M2;
      z.ppc = b->tile[2];
      z.fac = (T)(s32 / ((double)d.M1 * d.M2 * d.M3));
      z.plan = b->plan[2];
      z.tw = twiddles<T>(c);
      az[r] = z;
      AxisArgs<T> yf{};
      yf.plan = b->plan[3];
      yf.tw = twiddles<T>(c);
      yf.scale = (T)1;
      yf.in = C;
      yf.out = D;
      yf.in_ostride = (long long)d.M2 * d.Kz;
      yf.in_rstride = d.Kz;
      yf.out_ostride = (long long)d.N2 * d.Kz;
      yf.out_rstride = d.Kz;
      yf.nouter = Fo * d.M1;
      yf.ncols = d.Kz;
      yf.col_tile = b->tile[3];
      yf.in_rows = d.M2;
      yf.out_rows = d.N2;
      yf.in_map = map_id(d.M2);
      yf.out_map = map_pad32(d.N2);
      ayf[r] = yf;
      XEpiArgs<T> e{};
      e.in = D;
      e.in_fstride = (long long)d.M1 * d.N2 * d.Kz;
      e.in_rstride = (long long)d.N2 * d.Kz;
      e.in_ostride = d.Kz;
      e.n1 = d.N1;
      e.n2 = d.N2;
      e.n3h = d.N3h;
      e.kz = d.Kz;
      e.col_tile = b->tile[4];
      e.out_map = map_pad32(d.N1);
      e.main_blocks = ((d.Kz + e.col_tile - 1) / e.col_tile) * d.N2;
      e.plan = b->plan[4];
      e.tw = twiddles<T>(c);
      ae[r] = e;
      pre[r] = pre0;
      ypre[r] = YPre{};
      cpy[r] = PreCopy<T>{};
      phys[r] = mkphys(c, b->params[r]);
      for (int i = 0; i < 5; ++i) {
        StepIO<T> io{};
        io.Q = reinterpret_cast<Cx<T>*>(b->state[r]);
        io.Q0 = run_buf(r, 4);
        io.comp = reinterpret_cast<Cx<T>*>(b->comp[r]);
        io.fstride = fsN;
        io.n2 = d.N2;
        io.n3h = d.N3h;
        if (i < 4) {
          io.mode = i == 0 ? kStage1 : (i == 3 ? kStageLast : kStageMid);
          io.dtc = (T)(b->params[r].dt * rk[i]);
        } else {
          // tuning: the traffic of a middle RK stage (state, Q0 and the
          // compensation read, state written) on scratch copies only
          io.mode = kStageMid;
          io.dtc = (T)(b->params[r].dt * rk[1]);
          io.Q = run_buf(r, 5);
          io.Q0 = run_buf(r, 4);
          io.comp = b->comp[r] ? run_buf(r, 5) : nullptr;
        }
        epi[i * R + r] = mkepi(c, io, b->params[r]);
      }
    }
    // The argument blocks are read by every kernel of the previous steps that
    // may still be queued on the context stream (a non-blocking stream, not
    // ordered with the legacy default stream): drain it before rewriting
    // them, then upload on that stream so the next launches follow the copy.
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    PSB_TRY(cuda_ok(c, cudaStreamIsCapturing(c->stream, &cap), "batch arguments: capture status"));
    if (cap != cudaStreamCaptureStatusNone)
      return fail(c, PSB_ERR_ARG, "psb_batch: runs changed while the stream is being captured; set them first");
    PSB_TRY(cuda_ok(c, cudaStreamSynchronize(c->stream), "batch arguments: drain the stream"));
    if (b->dargs_bytes < ab) {
      if (b->dargs) cudaFree(b->dargs);
      b->dargs = nullptr;
      b->dargs_bytes = 0;
      PSB_TRY(cuda_ok(c, cudaMalloc(&b->dargs, ab), "batch arguments"));
      b->dargs_bytes = ab;
    }
    PSB_TRY(cuda_ok(c, cudaMemcpyAsync(b->dargs, b->host.data(), ab, cudaMemcpyHostToDevice, c->stream),
                    "batch arguments upload"));
    views(reinterpret_cast<char*>(b->dargs));
    return PSB_OK;
  }

  // ---- launches -----------------------------------------------------------
  size_t smem_axis(int L, int F, int ct) const { return (size_t)(L + 2 * L * F * ct) * sizeof(Cx<T>); }
  size_t smem_z(int P) const {
    constexpr int FMAX = Phys::F_IN > Phys::F_OUT ? Phys::F_IN : Phys::F_OUT;
    return zpass_smem_bytes<T>(FMAX, P, d.M3, (size_t)phys_is_block<Phys>::extra);
  }
  // radix 6/12/16 passes need the wide kernel instantiations
  bool wide(int pass) const {
    const FFTPlan& p = b->plan[pass];
    for (int s = 0; s < p.npass; ++s)
      if (p.radix[s] > 8 || p.radix[s] == 6) return true;
    return false;
  }
  // fix(integral_constant<int, ID>) when the pass's plan is a compiled-in
  // schedule ID (for this precision), else def().
  template <class Fix, class Def>
  int by_plan(int pass, Fix fix, Def def) {
    switch (fixed_plan_id(b->plan[pass])) {
#define PSB_FIXED_CASE(ID, ...)                                                             \
  case ID:                                                                                  \
    if constexpr (fixed_plan_compiled<T, ID>::value) return fix(std::integral_constant<int, ID>{}); \
    break;
      PSB_FIXED_PLANS(PSB_FIXED_CASE)
#undef PSB_FIXED_CASE
      default:
        break;
    }
    return def();
  }
  template <bool W>
  int launch_w(int pass, int stage) {
    const size_t esz = sizeof(Cx<T>);
    switch (pass) {
      case 0: {
        const int ct = b->tile[0];
        dim3 g((d.Kz + ct - 1) / ct, d.N2, R);
        const size_t sm = smem_axis(d.M1, Fi, ct);
        auto go = [&](auto k) {
          set_smem(k, sm);
          LaunchScope s(c, "batch x-inverse", (double)R * esz * d.N2 * d.Kz * (3.0 * d.N1 + (double)Fi * d.M1));
          launch_pdl(k, g, 256, sm, c->stream, (const AxisArgs<T>*)ax, (const Pre*)pre);
          return launch_ok(c, "batch x-inverse");
        };
        return by_plan(
            0, [&](auto id) { return go(axis_pass_batch<T, true, Pre, false, decltype(id)::value>); },
            [&] { return go(axis_pass_batch<T, true, Pre, W>); });
      }
      case 1:
      case 3: {
        const bool inv = pass == 1;
        const int ct = b->tile[pass];
        // y-inverse: YP::groups outer groups of YPre::F_DST lines per column
        const int G = inv ? YP::groups : Fo, F = inv ? Fb : Fo;
        dim3 g((d.Kz + ct - 1) / ct, G * d.M1, R);
        const size_t sm = smem_axis(d.M2, inv ? YPre::F_DST : 1, ct);
        const double by = (double)R * esz * F * d.M1 * d.Kz * (double)(d.N2 + d.M2);
        if (inv) {
          auto go = [&](auto k) {
            set_smem(k, sm);
            LaunchScope s(c, "batch y-inverse", by);
            launch_pdl(k, g, 256, sm, c->stream, (const AxisArgs<T>*)ay, (const YPre*)ypre);
            return launch_ok(c, "batch y-inverse");
          };
          return by_plan(
              1, [&](auto id) { return go(axis_pass_batch<T, true, YPre, false, decltype(id)::value>); },
              [&] { return go(axis_pass_batch<T, true, YPre, W>); });
        }
        auto go = [&](auto k) {
          set_smem(k, sm);
          LaunchScope s(c, "batch y-forward", by);
          launch_pdl(k, g, 256, sm, c->stream, (const AxisArgs<T>*)ayf, (const PreCopy<T>*)cpy);
          return launch_ok(c, "batch y-forward");
        };
        return by_plan(
            3, [&](auto id) { return go(axis_pass_batch<T, false, PreCopy<T>, false, decltype(id)::value>); },
            [&] { return go(axis_pass_batch<T, false, PreCopy<T>, W>); });
      }
      case 2: {
        const int P = b->tile[2];
        const long long np = (long long)d.M1 * d.M2;
        const long long items = (np + P - 1) / P * R;
        const size_t sm = smem_z(P);
        // persistent over (run, tile): at most the resident CTAs of the device
        auto go = [&](auto k) {
          set_smem(k, sm);
          const long long g = persistent_grid(k, sm, items);
          LaunchScope s(c, "batch z-fused", (double)R * esz * np * d.Kz * (Fb + Fo));
          launch_pdl(k, dim3((unsigned)g), 256, sm, c->stream, (const ZArgs<T>*)az, (const Phys*)phys, R);
          return launch_ok(c, "batch z-fused");
        };
        // a compiled two-pass (R1, 16) schedule with pencils paired: register-direct
        if constexpr (phys_fixed_fft<Phys>::value && sizeof(T) == 4) {
          if ((P & 1) == 0 && c->use_zrr) {
            switch (fixed_plan_id(b->plan[2])) {
#define PSB_FIXED_CASE(ID, ...)                                                   \
  case ID:                                                                        \
    if constexpr (zrr_plan<ID>::value && zrr_plan<ID>::R2 == 16) return go(zpass_rr_batch<T, Phys, ID>); \
    break;
              PSB_FIXED_PLANS(PSB_FIXED_CASE)
#undef PSB_FIXED_CASE
              default:
                break;
            }
          }
        }
        if constexpr (phys_fixed_fft<Phys>::value)
          return by_plan(
              2, [&](auto id) { return go(zpass_batch<T, Phys, false, decltype(id)::value>); },
              [&] { return go(zpass_batch<T, Phys, W>); });
        return go(zpass_batch<T, Phys, W>);
      }
      default: {
        const int ct = b->tile[4];
        const int ntile = (d.Kz + ct - 1) / ct;
        const int mainb = ntile * d.N2;
        const long long pts = (long long)d.N1 * d.N2 * (d.N3h - d.Kz);
        const int extra = (int)std::min<long long>((pts + 255) / 256, 1024);
        dim3 g(mainb + extra, R);
        const size_t sm = smem_axis(d.M1, Fo, ct);
        const double by = (double)R * (esz * Fo * d.M1 * d.N2 * d.Kz + esz * 3.0 * d.N1 * d.N2 * d.N3h *
                                                                           3.0);
        auto go = [&](auto k) {
          set_smem(k, sm);
          LaunchScope s(c, "batch x-forward+epilogue", by);
          launch_pdl(k, g, 256, sm, c->stream, (const XEpiArgs<T>*)ae, (const Epi*)(epi + (size_t)stage * R));
          return launch_ok(c, "batch x-forward+epilogue");
        };
        return by_plan(
            4, [&](auto id) { return go(xfwd_epi_batch<T, Epi, false, decltype(id)::value>); },
            [&] { return go(xfwd_epi_batch<T, Epi, W>); });
      }
    }
  }

  int launch(int pass, int stage) { return wide(pass) ? launch_w<true>(pass, stage) : launch_w<false>(pass, stage); }

  int step(int nsteps) {
    for (int s = 0; s < nsteps; ++s)
      for (int i = 0; i < 4; ++i)
        for (int pass = 0; pass < 5; ++pass) PSB_TRY(launch(pass, i));
    return PSB_OK;
  }

  // ---- autotuning -----------------------------------------------------------
  // Mean time of `reps` launches of one pass (RHS-mode epilogue), ms.
  int time_pass(int pass, int reps, float* ms) {
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    int st = launch(pass, 4);  // warm-up (and shape check)
    if (st == PSB_OK) {
      cudaEventRecord(e0, c->stream);
      for (int k = 0; k < reps && st == PSB_OK; ++k) st = launch(pass, 4);
      cudaEventRecord(e1, c->stream);
      cudaEventSynchronize(e1);
      cudaEventElapsedTime(ms, e0, e1);
      *ms /= reps;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return st;
  }

  int autotune(const Pre& pre0, Phys (*mkphys)(psb_ctx*, const psb_params&),
               Epi (*mkepi)(psb_ctx*, StepIO<T>, const psb_params&)) {
    const size_t esz = sizeof(Cx<T>);
    const int Ls[5] = {d.M1, d.M2, d.M3, d.M2, d.M1};
    const int Fs[5] = {Fi, YPre::F_DST, 0, 1, Fo};
    // RHS-mode passes read the runs' states and write only scratch; run one
    // full RHS first so that every intermediate buffer holds real data.
    for (int pass = 0; pass < 5; ++pass) PSB_TRY(launch(pass, 4));
    for (int pass = 0; pass < 5; ++pass) {
      std::vector<int> tiles;
      if (pass == 2) {
        for (int P : {1, 2, 4, 8})
          if (P <= phys_max_ppc<Phys>::value && smem_z(P) <= kSmemBudget) tiles.push_back(P);
      } else {
        for (int ct : {2, 4, 8, 16, 32})
          if (ct <= std::max(2, 2 * d.Kz) && smem_axis(Ls[pass], Fs[pass], ct) <= kSmemBudget) tiles.push_back(ct);
      }
      const std::vector<FFTPlan> orders = radix_orders(*plan_for(c, Ls[pass]));
      // the default shape is the incumbent; a candidate must beat it by 3%,
      // and the winner is re-timed against it before it is kept
      const int t0 = b->tile[pass];
      const FFTPlan p0 = b->plan[pass];
      float base = 0;
      PSB_TRY(time_pass(pass, 8, &base));
      float best = 0.97f * base;
      int bt = t0;
      FFTPlan bp = p0;
      for (int t : tiles)
        for (const FFTPlan& q : orders) {
          b->tile[pass] = t;
          b->plan[pass] = q;
          PSB_TRY(build(pre0, mkphys, mkepi));
          float ms = 0;
          PSB_TRY(time_pass(pass, 6, &ms));
          if (ms < best) {
            best = ms;
            bt = t;
            bp = q;
          }
        }
      b->tile[pass] = bt;
      b->plan[pass] = bp;
      PSB_TRY(build(pre0, mkphys, mkepi));
      if (bt != t0 || bp.npass != p0.npass || !std::equal(bp.radix, bp.radix + bp.npass, p0.radix)) {
        float again = 0, def = 0;
        PSB_TRY(time_pass(pass, 10, &again));
        b->tile[pass] = t0;
        b->plan[pass] = p0;
        PSB_TRY(build(pre0, mkphys, mkepi));
        PSB_TRY(time_pass(pass, 10, &def));
        if (again < 0.98f * def) {
          b->tile[pass] = bt;
          b->plan[pass] = bp;
          PSB_TRY(build(pre0, mkphys, mkepi));
        }
      }
    }
    (void)esz;
    b->tuned = true;
    return PSB_OK;
  }
};

// per-closure functor makers
template <typename T>
PhysProducts<T> mk_products(psb_ctx*, const psb_params&) {
  return PhysProducts<T>{};
}
template <typename T>
PhysSmag<T> mk_smag(psb_ctx* c, const psb_params&) {
  return PhysSmag<T>{(T)(0.16 * c->Delta * 0.16 * c->Delta)};
}
template <typename T, int ACT, int H>
PhysLearned<T, ACT, H> mk_learned(psb_ctx* c, const psb_params& p) {
  const double s32 = std::sqrt(std::pow(1.5, 3) * std::sqrt((double)c->N1 * c->N2 * c->N3));
  return PhysLearned<T, ACT, H>{reinterpret_cast<const float*>(p.mlp_params),
                                reinterpret_cast<const float*>(p.mlp_norm), (T)s32,
                                (float)(p.les_delta > 0 ? p.les_delta : c->Delta)};
}
template <typename T, bool SMAG>
EpiNS<T, SMAG> mk_epi(psb_ctx* c, StepIO<T> io, const psb_params& p) {
  return EpiNS<T, SMAG>{io, ktab<T>(c->kx, c->ky, c->kz), (T)p.nu, p.rotate, (T)p.Om1, (T)p.Om2, (T)p.Om3,
                        SMAG ? 0 : 1, c->N1 / 2, c->N2 / 2, c->N3 / 2};
}

// Default launch shapes: the single-run rules of the library.
// Fz: z-pass inputs (with the fields it derives itself); Fy / Gy: lines per
// column and outer groups of the y-inverse pass
void default_shapes(psb_batch* b, int Fi, int Fb, int Fz, int Fo, int Fy, int Gy, size_t esz, int ppc,
                    size_t zextra) {
  psb_ctx* c = b->c;
  const Dims d = dims(c, Fi, Fb, Fo);
  b->tile[0] = pick_ct(d.Kz, Fi, d.M1, esz, d.N2);
  b->tile[1] = pick_ct(d.Kz, Fy, d.M2, esz, Gy * d.M1);
  b->tile[3] = pick_ct(d.Kz, 1, d.M2, esz, Fo * d.M1);
  b->tile[4] = pick_ct(d.Kz, Fo, d.M1, esz, d.N2);
  const int FMAX = std::max(Fz, Fo);
  int P = ppc;
  auto sm = [&](int P) { return (size_t)(d.M3 + 2 * (size_t)((FMAX * P + 1) / 2) * d.M3) * esz + zextra; };
  while (P > 1 && sm(P) > kSmemBudget) P /= 2;
  // at least ~2 CTAs per SM over the whole batch (the single-run rule at nruns = 1)
  const long long np = (long long)d.M1 * d.M2;
  while (P > 1 && (np + P - 1) / P * b->nruns < 2 * 148) P /= 2;
  b->tile[2] = P;
  b->plan[0] = *plan_for(c, d.M1);
  b->plan[1] = *plan_for(c, d.M2);
  b->plan[2] = *plan_for(c, d.M3);
  b->plan[3] = *plan_for(c, d.M2);
  b->plan[4] = *plan_for(c, d.M1);
}

template <typename T, class Pre, class Phys, class Epi>
int run_batch(psb_batch* b, int nsteps, bool tune, Pre pre0, Phys (*mkphys)(psb_ctx*, const psb_params&),
              Epi (*mkepi)(psb_ctx*, StepIO<T>, const psb_params&)) {
  psb_ctx* c = b->c;
  using BT = Batch<T, Pre, Phys, Epi>;
  BT x;
  x.b = b;
  x.c = c;
  x.d = dims(c, BT::Fi, BT::Fb, BT::Fo);
  x.R = b->nruns;
  const size_t need = BT::run_bytes(x.d) * (size_t)b->nruns;
  if (b->arena_bytes < need) {
    if (b->arena) cudaFree(b->arena);
    b->arena = nullptr;
    b->arena_bytes = 0;
    PSB_TRY(cuda_ok(c, cudaMalloc(&b->arena, need), "batch scratch"));
    b->arena_bytes = need;
  }
  if (b->plan[0].L == 0) {
    default_shapes(b, BT::Fi, BT::Fb, Phys::F_IN, BT::Fo, BT::YPre::F_DST, BT::YP::groups, sizeof(Cx<T>),
                   phys_default_ppc<Phys>::value, (size_t)phys_is_block<Phys>::extra);
    // the register-direct z pass's schedule where it exists (as for single runs)
    if constexpr (phys_fixed_fft<Phys>::value && sizeof(T) == 4)
      if ((b->tile[2] & 1) == 0 && c->use_zrr) zrr_default_plan(b->plan[2]);
  }
  if (b->dirty) {
    PSB_TRY(x.build(pre0, mkphys, mkepi));
    b->dirty = false;
  } else {
    x.views(reinterpret_cast<char*>(b->dargs));
  }
  if (tune) return x.autotune(pre0, mkphys, mkepi);
  return x.step(nsteps);
}

template <typename T>
int dispatch(psb_batch* b, int nsteps, bool tune) {
  switch (b->closure) {
    case PSB_DNS:
      return run_batch<T>(b, nsteps, tune, PreCopyN<T, 3>{}, &mk_products<T>, &mk_epi<T, false>);
    case PSB_SMAG:
      return run_batch<T>(b, nsteps, tune, PreStrain<T>{}, &mk_smag<T>, &mk_epi<T, true>);
    case PSB_LEARNED:
      // every run of a learned batch has the activation and width of run 0 (psb_batch_set_run)
      if (b->params[0].mlp_act == PSB_ACT_GELU)
        return run_batch<T>(b, nsteps, tune, PreGradXY<T>{}, &mk_learned<T, kActGelu, 64>, &mk_epi<T, false>);
      if (b->params[0].mlp_hidden == 32)
        return run_batch<T>(b, nsteps, tune, PreGradXY<T>{}, &mk_learned<T, kActRelu, 32>, &mk_epi<T, false>);
      return run_batch<T>(b, nsteps, tune, PreGradXY<T>{}, &mk_learned<T, kActRelu, 64>, &mk_epi<T, false>);
    default:
      return fail(b->c, PSB_ERR_UNSUPPORTED, "psb_batch: closure not batched (DNS, SMAG, LEARNED are)");
  }
}

// ---------------------------------------------------------------------------
// Persistent ensemble: every batch of an ensemble (grid sizes and closures may
// differ) advanced by ONE cooperative launch per call.  The kernel walks the
// RK4 stages and the five passes of each; a pass's work items -- the CTA tiles
// of that pass over every run of every batch -- are spread over the CTAs, and
// a bounded grid barrier separates consecutive passes (a pass reads what the
// previous one wrote).  Each item runs the same tile body as the batched
// launches (runtime transform schedules, every radix), with the batch's own
// argument blocks, so the results equal the batched step's up to the
// schedule's rounding.
// ---------------------------------------------------------------------------
constexpr int kEnsMaxGroups = 4;
enum EnsKind : int { kEnsDns = 0, kEnsSmag = 1, kEnsLearnedR32 = 2 };

struct EnsGroup {
  int kind;
  int R;
  int nx[5], ny[5];  // tiles of a pass per run: nx x ny (pass 4: nx = main + extra blocks)
  long long items[5];
  const void *ax, *ay, *ayf, *az, *ae, *pre, *ypre, *cpy, *phys, *epi;
};
struct EnsDesc {
  int ngroups;
  EnsGroup g[kEnsMaxGroups];
};

// staged: the z items' (group, run) whose twiddles and Phys extra the CTA's
// shared memory holds (-1: none); a z item stages only when it changes.
template <typename T, class Pre, class Phys, class Epi>
__device__ __forceinline__ void ens_item(const EnsGroup& g, int q, int pass, int stage, long long i, int& staged) {
  using YP = pre_ypass<T, Pre>;
  using YPre = typename YP::type;
  const long long per = (long long)g.nx[pass] * g.ny[pass];
  const int r = (int)(i / per);
  const int rem = (int)(i - (long long)r * per);
  const int by = rem / g.nx[pass], bx = rem - by * g.nx[pass];
  switch (pass) {
    case 0:
      axis_pass_body<T, true, Pre, true>(static_cast<const AxisArgs<T>*>(g.ax)[r], static_cast<const Pre*>(g.pre)[r],
                                         bx, by);
      break;
    case 1:
      axis_pass_body<T, true, YPre, true>(static_cast<const AxisArgs<T>*>(g.ay)[r],
                                          static_cast<const YPre*>(g.ypre)[r], bx, by);
      break;
    case 2: {
      const ZArgs<T>& a = static_cast<const ZArgs<T>*>(g.az)[r];
      const Phys& ph = static_cast<const Phys*>(g.phys)[r];
      const int key = q * 65536 + r;
      if (key != staged) {
        zpass_setup<T, Phys>(a, ph);
        staged = key;
      }
      zpass_tile<T, Phys, true>(a, ph, bx);
      break;
    }
    case 3:
      axis_pass_body<T, false, PreCopy<T>, true>(static_cast<const AxisArgs<T>*>(g.ayf)[r],
                                                 static_cast<const PreCopy<T>*>(g.cpy)[r], bx, by);
      break;
    default:
      xfwd_epi_body<T, Epi, true>(static_cast<const XEpiArgs<T>*>(g.ae)[r],
                                  static_cast<const Epi*>(g.epi)[(size_t)stage * g.R + r], bx, g.nx[4]);
      break;
  }
}

template <typename T>
__global__ void __launch_bounds__(256, 2) ens_persistent_kernel(const EnsDesc* __restrict__ D, GridBar* gb,
                                                                int* status, int nsteps, unsigned limit) {
  const int ng = D->ngroups;
  for (int step = 0; step < nsteps; ++step)
    for (int stage = 0; stage < 4; ++stage)
      for (int pass = 0; pass < 5; ++pass) {
        long long total = 0;
        for (int q = 0; q < ng; ++q) total += D->g[q].items[pass];
        int staged = -1;  // the previous pass's items reused the shared memory
        for (long long it = blockIdx.x; it < total; it += gridDim.x) {
          long long i = it;
          int q = 0;
          while (q < ng - 1 && i >= D->g[q].items[pass]) i -= D->g[q++].items[pass];
          const EnsGroup& g = D->g[q];
          switch (g.kind) {
            case kEnsDns:
              ens_item<T, PreCopyN<T, 3>, PhysProducts<T>, EpiNS<T, false>>(g, q, pass, stage, i, staged);
              break;
            case kEnsSmag:
              ens_item<T, PreStrain<T>, PhysSmag<T>, EpiNS<T, true>>(g, q, pass, stage, i, staged);
              break;
            default:
              ens_item<T, PreGradXY<T>, PhysLearned<T, kActRelu, 32>, EpiNS<T, false>>(g, q, pass, stage, i, staged);
              break;
          }
          __syncthreads();  // the next item reuses the shared memory
        }
        if (!grid_barrier(gb, gridDim.x, limit, status)) return;
      }
}

// Host view of one batch for the ensemble: its device argument blocks, items and shared memory.
template <typename T, class Pre, class Phys, class Epi>
size_t ens_group(psb_batch* b, int kind, EnsGroup& g) {
  using BT = Batch<T, Pre, Phys, Epi>;
  BT x;
  x.b = b;
  x.c = b->c;
  x.d = dims(b->c, BT::Fi, BT::Fb, BT::Fo);
  x.R = b->nruns;
  x.views(reinterpret_cast<char*>(b->dargs));
  const Dims& d = x.d;
  g.kind = kind;
  g.R = b->nruns;
  g.ax = x.ax;
  g.ay = x.ay;
  g.ayf = x.ayf;
  g.az = x.az;
  g.ae = x.ae;
  g.pre = x.pre;
  g.ypre = x.ypre;
  g.cpy = x.cpy;
  g.phys = x.phys;
  g.epi = x.epi;
  const int* t = b->tile.data();
  g.nx[0] = (d.Kz + t[0] - 1) / t[0];
  g.ny[0] = d.N2;
  g.nx[1] = (d.Kz + t[1] - 1) / t[1];
  g.ny[1] = BT::YP::groups * d.M1;
  g.nx[2] = (int)(((long long)d.M1 * d.M2 + t[2] - 1) / t[2]);
  g.ny[2] = 1;
  g.nx[3] = (d.Kz + t[3] - 1) / t[3];
  g.ny[3] = BT::Fo * d.M1;
  const int mainb = ((d.Kz + t[4] - 1) / t[4]) * d.N2;
  const long long pts = (long long)d.N1 * d.N2 * (d.N3h - d.Kz);
  g.nx[4] = mainb + (int)std::min<long long>((pts + 255) / 256, 1024);
  g.ny[4] = 1;
  for (int k = 0; k < 5; ++k) g.items[k] = (long long)g.nx[k] * g.ny[k] * g.R;
  size_t sm = 0;
  sm = std::max(sm, x.smem_axis(d.M1, BT::Fi, t[0]));
  sm = std::max(sm, x.smem_axis(d.M2, BT::YPre::F_DST, t[1]));
  sm = std::max(sm, x.smem_z(t[2]));
  sm = std::max(sm, x.smem_axis(d.M2, 1, t[3]));
  sm = std::max(sm, x.smem_axis(d.M1, BT::Fo, t[4]));
  return sm;
}

}  // namespace

extern "C" {

int psb_batch_create(psb_ctx* c, int closure, int nruns, psb_batch** out) {
  if (!c || !out) return PSB_ERR_ARG;
  *out = nullptr;
  if (nruns <= 0 || nruns > 65535) return fail(c, PSB_ERR_ARG, "psb_batch_create: nruns must be in 1..65535");
  if (closure != PSB_DNS && closure != PSB_SMAG && closure != PSB_LEARNED)
    return fail(c, PSB_ERR_UNSUPPORTED, "psb_batch_create: closure not batched (DNS, SMAG, LEARNED are)");
  psb_batch* b = new psb_batch();
  b->c = c;
  b->closure = closure;
  b->nruns = nruns;
  b->state.assign(nruns, nullptr);
  b->comp.assign(nruns, nullptr);
  b->params.assign(nruns, psb_params{});
  *out = b;
  return PSB_OK;
}

int psb_batch_set_run(psb_batch* b, int r, void* state, void* comp, const psb_params* p) {
  if (!b) return PSB_ERR_ARG;
  if (r < 0 || r >= b->nruns || !state || !p) return fail(b->c, PSB_ERR_ARG, "psb_batch_set_run: bad argument");
  if (b->closure == PSB_LEARNED && (!p->mlp_params || !p->mlp_norm))
    return fail(b->c, PSB_ERR_ARG, "psb_batch_set_run: PSB_LEARNED needs mlp_params and mlp_norm");
  if (b->closure == PSB_LEARNED && p->mlp_act != PSB_ACT_GELU && p->mlp_act != PSB_ACT_RELU)
    return fail(b->c, PSB_ERR_ARG, "psb_batch_set_run: mlp_act must be PSB_ACT_GELU or PSB_ACT_RELU");
  if (b->closure == PSB_LEARNED &&
      !(p->mlp_hidden == 0 || p->mlp_hidden == 64 || (p->mlp_hidden == 32 && p->mlp_act == PSB_ACT_RELU)))
    return fail(b->c, PSB_ERR_ARG, "psb_batch_set_run: mlp_hidden must be 64 (0), or 32 with PSB_ACT_RELU");
  if (b->closure == PSB_LEARNED)
    for (int q = 0; q < b->nruns; ++q)
      if (q != r && b->state[q] &&
          (b->params[q].mlp_act != p->mlp_act || (b->params[q].mlp_hidden == 32) != (p->mlp_hidden == 32)))
        return fail(b->c, PSB_ERR_ARG,
                    "psb_batch_set_run: every run of a learned batch needs the same mlp_act and mlp_hidden");
  b->state[r] = state;
  b->comp[r] = comp;
  b->params[r] = *p;
  b->dirty = true;
  return PSB_OK;
}

int psb_batch_autotune(psb_batch* b) {
  if (!b) return PSB_ERR_ARG;
  for (int r = 0; r < b->nruns; ++r)
    if (!b->state[r]) return fail(b->c, PSB_ERR_ARG, "psb_batch_autotune: run without state");
  PSB_TRY(cuda_ok(b->c, cudaSetDevice(b->c->dev), "cudaSetDevice"));
  return b->c->prec == 64 ? dispatch<double>(b, 0, true) : dispatch<float>(b, 0, true);
}

int psb_batch_step_rk4(psb_batch* b, int nsteps) {
  if (!b) return PSB_ERR_ARG;
  if (nsteps < 0) return fail(b->c, PSB_ERR_ARG, "psb_batch_step_rk4: nsteps < 0");
  for (int r = 0; r < b->nruns; ++r)
    if (!b->state[r]) return fail(b->c, PSB_ERR_ARG, "psb_batch_step_rk4: run without state");
  PSB_TRY(cuda_ok(b->c, cudaSetDevice(b->c->dev), "cudaSetDevice"));
  return b->c->prec == 64 ? dispatch<double>(b, nsteps, false) : dispatch<float>(b, nsteps, false);
}

int psb_batch_shape(const psb_batch* b, int pass, int* tile, int* radices, int maxr) {
  if (!b || pass < 0 || pass > 4 || !tile) return PSB_ERR_ARG;
  *tile = b->tile[pass];
  const FFTPlan& p = b->plan[pass];
  for (int s = 0; s < maxr; ++s) radices[s] = s < p.npass ? p.radix[s] : 0;
  return PSB_OK;
}

int psb_tuned_shape(const psb_ctx* c, int closure, int pass, int* tile, int* radices, int maxr) {
  if (!c || pass < 0 || pass > 4 || !tile) return PSB_ERR_ARG;
  const auto it = c->tuned.find(closure);
  if (it == c->tuned.end()) {
    *tile = 0;
    for (int s = 0; s < maxr; ++s) radices[s] = 0;
    return PSB_OK;
  }
  const psb_pass_shape& sh = it->second.pass[pass];
  *tile = sh.tile;
  for (int s = 0; s < maxr; ++s) radices[s] = s < sh.plan.npass ? sh.plan.radix[s] : 0;
  return PSB_OK;
}

int psb_autotune_clear(psb_ctx* c, int closure) {
  if (!c) return PSB_ERR_ARG;
  c->tuned.erase(closure);
  return PSB_OK;
}

struct psb_ensemble {
  psb_ctx* c = nullptr;  // the first batch's context: stream and device
  std::vector<psb_batch*> batches;
  void* dev = nullptr;  // EnsDesc, then GridBar, then the status word
  int prec = 64;
  EnsDesc uploaded{};   // the descriptor on the device (uploads happen only when it changes)
  bool have = false;
};

int psb_ensemble_create(psb_batch* const* batches, int nbatch, psb_ensemble** out) {
  if (!batches || !out || nbatch < 1) return PSB_ERR_ARG;
  *out = nullptr;
  psb_ctx* c = batches[0] ? batches[0]->c : nullptr;
  if (!c) return PSB_ERR_ARG;
  if (nbatch > kEnsMaxGroups) return fail(c, PSB_ERR_ARG, "psb_ensemble_create: at most 4 batches");
  for (int i = 0; i < nbatch; ++i) {
    const psb_batch* b = batches[i];
    if (!b || b->c->dev != c->dev || b->c->prec != c->prec)
      return fail(c, PSB_ERR_ARG, "psb_ensemble_create: every batch on one device and precision");
    const bool learned_ok = b->closure == PSB_LEARNED && b->params[0].mlp_act == PSB_ACT_RELU &&
                            b->params[0].mlp_hidden == 32;
    if (b->closure != PSB_DNS && b->closure != PSB_SMAG && !learned_ok)
      return fail(c, PSB_ERR_UNSUPPORTED,
                  "psb_ensemble_create: batches of PSB_DNS, PSB_SMAG or PSB_LEARNED (ReLU, width 32)");
  }
  PSB_TRY(cuda_ok(c, cudaSetDevice(c->dev), "cudaSetDevice"));
  psb_ensemble* e = new psb_ensemble();
  e->c = c;
  e->prec = c->prec;
  e->batches.assign(batches, batches + nbatch);
  cudaError_t err = cudaMalloc(&e->dev, sizeof(EnsDesc) + sizeof(GridBar) + 16);
  if (err == cudaSuccess) err = cudaMemset(e->dev, 0, sizeof(EnsDesc) + sizeof(GridBar) + 16);  // status 0
  if (err != cudaSuccess) {
    delete e;
    return fail(c, PSB_ERR_CUDA, std::string("psb_ensemble_create: ") + cudaGetErrorString(err));
  }
  *out = e;
  return PSB_OK;
}

}  // extern "C"

template <typename T>
static int ens_step(psb_ensemble* e, int nsteps, unsigned limit) {
  psb_ctx* c = e->c;
  EnsDesc h{};
  h.ngroups = (int)e->batches.size();
  size_t smem = 0;
  for (int i = 0; i < h.ngroups; ++i) {
    psb_batch* b = e->batches[i];
    PSB_TRY(psb_batch_step_rk4(b, 0));  // (re)build the argument blocks of a changed batch
    if (b->closure == PSB_DNS)
      smem = std::max(smem, ens_group<T, PreCopyN<T, 3>, PhysProducts<T>, EpiNS<T, false>>(b, kEnsDns, h.g[i]));
    else if (b->closure == PSB_SMAG)
      smem = std::max(smem, ens_group<T, PreStrain<T>, PhysSmag<T>, EpiNS<T, true>>(b, kEnsSmag, h.g[i]));
    else
      smem = std::max(smem, ens_group<T, PreGradXY<T>, PhysLearned<T, kActRelu, 32>, EpiNS<T, false>>(
                                b, kEnsLearnedR32, h.g[i]));
  }
  auto k = ens_persistent_kernel<T>;
  if (smem > 48 * 1024)
    PSB_TRY(cuda_ok(c, cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                    "ensemble shared memory"));
  int per = 0, nsm = 0;
  PSB_TRY(cuda_ok(c, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k, 256, smem), "ensemble occupancy"));
  PSB_TRY(cuda_ok(c, cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, c->dev), "SM count"));
  if (per < 1) return fail(c, PSB_ERR_SHAPE, "psb_ensemble_step_rk4: the tiles' shared memory leaves no CTA per SM");
  unsigned grid = (unsigned)(per * nsm);
  char* dv = static_cast<char*>(e->dev);
  EnsDesc* dd = reinterpret_cast<EnsDesc*>(dv);
  GridBar* gb = reinterpret_cast<GridBar*>(dv + sizeof(EnsDesc));
  int* status = reinterpret_cast<int*>(dv + sizeof(EnsDesc) + sizeof(GridBar));
  // the descriptor changes only when a batch's runs or shapes do: upload it
  // then (not while the stream is captured), after the stream drains
  if (!e->have || std::memcmp(&h, &e->uploaded, sizeof(EnsDesc)) != 0) {
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    PSB_TRY(cuda_ok(c, cudaStreamIsCapturing(c->stream, &cap), "capture status"));
    if (cap != cudaStreamCaptureStatusNone)
      return fail(c, PSB_ERR_ARG, "psb_ensemble_step_rk4: step once outside a stream capture first");
    PSB_TRY(cuda_ok(c, cudaStreamSynchronize(c->stream), "ensemble: drain the stream"));
    PSB_TRY(cuda_ok(c, cudaMemcpy(dd, &h, sizeof(EnsDesc), cudaMemcpyHostToDevice), "ensemble descriptor"));
    e->uploaded = h;
    e->have = true;
  }
  PSB_TRY(cuda_ok(c, cudaMemsetAsync(gb, 0, sizeof(GridBar), c->stream), "grid barrier reset"));
  if (nsteps == 0) return PSB_OK;
  void* args[] = {&dd, &gb, &status, &nsteps, &limit};
  {
    LaunchScope ls(c, "ensemble persistent", 0.0);
    PSB_TRY(cuda_ok(c, cudaLaunchCooperativeKernel((const void*)k, dim3(grid), dim3(256), args, smem, c->stream),
                    "ensemble persistent launch"));
  }
  return PSB_OK;
}

extern "C" {

int psb_ensemble_step_rk4(psb_ensemble* e, int nsteps, unsigned poll_limit) {
  if (!e) return PSB_ERR_ARG;
  if (nsteps < 0) return fail(e->c, PSB_ERR_ARG, "psb_ensemble_step_rk4: nsteps < 0");
  PSB_TRY(cuda_ok(e->c, cudaSetDevice(e->c->dev), "cudaSetDevice"));
  const unsigned limit = poll_limit ? poll_limit : (1u << 26);
  return e->prec == 64 ? ens_step<double>(e, nsteps, limit) : ens_step<float>(e, nsteps, limit);
}

int psb_ensemble_status(psb_ensemble* e, int* status) {
  if (!e || !status) return PSB_ERR_ARG;
  psb_ctx* c = e->c;
  PSB_TRY(cuda_ok(c, cudaSetDevice(c->dev), "cudaSetDevice"));
  int* st = reinterpret_cast<int*>(static_cast<char*>(e->dev) + sizeof(EnsDesc) + sizeof(GridBar));
  int h = 0;
  PSB_TRY(cuda_ok(c, cudaMemcpyAsync(&h, st, sizeof(int), cudaMemcpyDeviceToHost, c->stream), "status read"));
  PSB_TRY(cuda_ok(c, cudaMemsetAsync(st, 0, sizeof(int), c->stream), "status clear"));
  PSB_TRY(cuda_ok(c, cudaStreamSynchronize(c->stream), "status sync"));
  *status = h;
  return PSB_OK;
}

int psb_ensemble_destroy(psb_ensemble* e) {
  if (!e) return PSB_ERR_ARG;
  cudaSetDevice(e->c->dev);
  if (e->dev) cudaFree(e->dev);
  delete e;
  return PSB_OK;
}

int psb_batch_destroy(psb_batch* b) {
  if (!b) return PSB_ERR_ARG;
  cudaSetDevice(b->c->dev);
  if (b->arena) cudaFree(b->arena);
  if (b->dargs) cudaFree(b->dargs);
  delete b;
  return PSB_OK;
}

}  // extern "C"
