// DNS right-hand side without any device allocation.
//
// Who needs this: callers that must not allocate device memory at the time
// they evaluate the RHS.  Examples are host applications whose own pool
// allocator has reserved the device memory up front, so that a cudaMalloc
// from a library fails with out-of-memory, and time-critical loops that
// cannot afford the implicit device synchronisation of cudaMalloc/cudaFree.
// psb_rhs allocates its scratch on first use; psb_rhs_dns_noalloc instead
// works in a fixed scratch array that is part of the library image.
//
// The scratch is a file-scope __device__ array of kNoAllocBytes.  Every GPU
// that loads this part of the library holds it until the process exits.  Host
// code cannot use the array's name as a device address, so the first call on
// each device (with that device current) looks the address up with
// cudaGetSymbolAddress and caches it; make that first call before any stream
// capture.  All calls share the one array: calls that overlap on the GPU (two
// streams, two host threads) race on it and must be serialised by the caller.
// Every scratch element the pipeline reads is written earlier in the same
// call, so nothing needs clearing between calls.  The caller's current device
// is restored before the call returns.  Launches are counted and, with
// psb_timing_enable on, timed like those of psb_rhs (same pass names).
#include <mutex>

#include "psb_ctx.cuh"

using namespace psb;
using namespace psbh;

namespace {

// DNS scratch of a 32^3 FP64 grid: (3+3+6+6) pencil buffers of 48 x {32|48} x 16 complex.
constexpr size_t kNoAllocBytes = 8847360;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
void* g_noalloc_ptr[kMaxDevices] = {};

size_t align256(size_t b) { return (b + 255) / 256 * 256; }

template <typename T>
size_t noalloc_bytes(const psb_ctx* c) {
  const size_t M1 = 3 * c->N1 / 2, M2 = 3 * c->N2 / 2, Kz = c->N3 / 2, N2 = c->N2;
  const size_t e = sizeof(Cx<T>);
  return align256(3 * M1 * N2 * Kz * e) + align256(3 * M1 * M2 * Kz * e) + align256(6 * M1 * M2 * Kz * e) +
         align256(6 * M1 * N2 * Kz * e);
}

template <typename T, bool INV, class Pre>
int axis(psb_ctx* c, AxisArgs<T> a, Pre pre, const char* what) {
  const size_t esz = sizeof(Cx<T>);
  const int L = a.plan.L;
  a.col_tile = pick_ct(a.ncols, Pre::F_DST, L, esz);
  const size_t smem = (size_t)(L + 2 * L * Pre::F_DST * a.col_tile) * esz;
  dim3 grid((a.ncols + a.col_tile - 1) / a.col_tile, a.nouter);
  const double bytes = (double)esz * a.nouter * a.ncols *
                       ((double)Pre::F_SRC * count_mapped(a.in_map, a.in_rows) + (double)Pre::F_DST * a.out_rows);
  auto k = axis_pass_kernel<T, INV, Pre>;
  set_smem(k, smem);
  LaunchScope scope(c, what, bytes);
  k<<<grid, 256, smem, c->stream>>>(a, pre);
  return launch_ok(c, what);
}

// Restores the caller's current device when the entry point returns.
struct DeviceGuard {
  int prev = -1;
  DeviceGuard() {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
  }
  ~DeviceGuard() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

template <typename T>
int dns_noalloc(psb_ctx* c, const Cx<T>* Q, Cx<T>* rhs, const psb_params* p, unsigned char* base) {
  const int N1 = c->N1, N2 = c->N2, N3 = c->N3, N3h = c->N3h;
  const int M1 = 3 * N1 / 2, M2 = 3 * N2 / 2, M3 = 3 * N3 / 2, Kz = N3 / 2;
  const size_t e = sizeof(Cx<T>);
  Cx<T>* A = reinterpret_cast<Cx<T>*>(base);
  Cx<T>* B = reinterpret_cast<Cx<T>*>(base + align256((size_t)3 * M1 * N2 * Kz * e));
  Cx<T>* C = reinterpret_cast<Cx<T>*>(reinterpret_cast<unsigned char*>(B) + align256((size_t)3 * M1 * M2 * Kz * e));
  Cx<T>* D = reinterpret_cast<Cx<T>*>(reinterpret_cast<unsigned char*>(C) + align256((size_t)6 * M1 * M2 * Kz * e));
  const Cx<T>* tw = twiddles<T>(c);
  AxisArgs<T> a{};
  a.plan = *plan_for(c, M1);
  a.tw = tw;
  a.scale = (T)1;
  a.in = Q;
  a.out = A;
  a.in_fstride = (long long)N1 * N2 * N3h;
  a.in_ostride = N3h;
  a.in_rstride = (long long)N2 * N3h;
  a.out_fstride = (long long)M1 * N2 * Kz;
  a.out_ostride = Kz;
  a.out_rstride = (long long)N2 * Kz;
  a.nouter = N2;
  a.ncols = Kz;
  a.in_rows = N1;
  a.out_rows = M1;
  a.in_map = map_pad32(N1);
  a.out_map = map_id(M1);
  PSB_TRY((axis<T, true>(c, a, PreCopyN<T, 3>{}, "x-inverse")));
  AxisArgs<T> b{};
  b.plan = *plan_for(c, M2);
  b.tw = tw;
  b.scale = (T)1;
  b.in = A;
  b.out = B;
  b.in_ostride = (long long)N2 * Kz;
  b.in_rstride = Kz;
  b.out_ostride = (long long)M2 * Kz;
  b.out_rstride = Kz;
  b.nouter = 3 * M1;
  b.ncols = Kz;
  b.in_rows = N2;
  b.out_rows = M2;
  b.in_map = map_pad32(N2);
  b.out_map = map_id(M2);
  PSB_TRY((axis<T, true>(c, b, PreCopy<T>{}, "y-inverse")));
  ZArgs<T> z{};
  const long long fsP = (long long)M1 * M2 * Kz;
  for (int f = 0; f < 3; ++f) {
    z.in[f] = B + f * fsP;
    z.in_pstride[f] = Kz;
    z.in_kz[f] = Kz;
  }
  for (int g = 0; g < 6; ++g) {
    z.out[g] = C + g * fsP;
    z.out_pstride[g] = Kz;
  }
  z.out_kz = Kz;
  z.npencils = (long long)M1 * M2;
  const double s32 = std::sqrt(std::pow(1.5, 3) * std::sqrt((double)N1 * N2 * N3));
  z.fac = (T)(s32 / ((double)M1 * M2 * M3));
  z.plan = *plan_for(c, M3);
  z.tw = tw;
  {
    auto smem_for = [&](int P) { return zpass_smem_bytes<T>(6, P, M3, 0); };
    int P = 8;
    while (P > 1 && smem_for(P) > kSmemBudget) P /= 2;
    while (P > 1 && (z.npencils + P - 1) / P < 2 * 148) P /= 2;
    z.ppc = P;
    auto k = zpass_kernel<T, PhysProducts<T>>;
    set_smem(k, smem_for(P));
    const double zbytes = (double)e * z.npencils * Kz * (3.0 + 6.0);
    LaunchScope scope(c, "z-fused", zbytes);
    k<<<(unsigned)((z.npencils + P - 1) / P), 256, smem_for(P), c->stream>>>(z, PhysProducts<T>{});
    PSB_TRY(launch_ok(c, "z-fused"));
  }
  AxisArgs<T> d{};
  d.plan = *plan_for(c, M2);
  d.tw = tw;
  d.scale = (T)1;
  d.in = C;
  d.out = D;
  d.in_ostride = (long long)M2 * Kz;
  d.in_rstride = Kz;
  d.out_ostride = (long long)N2 * Kz;
  d.out_rstride = Kz;
  d.nouter = 6 * M1;
  d.ncols = Kz;
  d.in_rows = M2;
  d.out_rows = N2;
  d.in_map = map_id(M2);
  d.out_map = map_pad32(N2);
  PSB_TRY((axis<T, false>(c, d, PreCopy<T>{}, "y-forward")));
  StepIO<T> io{};
  io.Q = const_cast<Cx<T>*>(Q);
  io.rhs_out = rhs;
  io.fstride = (long long)N1 * N2 * N3h;
  io.n2 = N2;
  io.n3h = N3h;
  io.mode = kRHS;
  KTabs<T> kt;
  kt.k1 = c->kx;
  kt.k2 = c->ky;
  kt.k3 = c->kz;
  EpiNS<T, false> epi{io, kt, (T)p->nu, p->rotate, (T)p->Om1, (T)p->Om2, (T)p->Om3, 1, N1 / 2, N2 / 2, N3 / 2};
  XEpiArgs<T> ea{};
  ea.in = D;
  ea.in_fstride = (long long)M1 * N2 * Kz;
  ea.in_rstride = (long long)N2 * Kz;
  ea.in_ostride = Kz;
  ea.n1 = N1;
  ea.n2 = N2;
  ea.n3h = N3h;
  ea.kz = Kz;
  ea.out_map = map_pad32(N1);
  ea.plan = *plan_for(c, M1);
  ea.tw = tw;
  ea.col_tile = pick_ct(Kz, 6, M1, e);
  const int ntile = (Kz + ea.col_tile - 1) / ea.col_tile;
  ea.main_blocks = ntile * N2;
  const long long pts = (long long)N1 * N2 * (N3h - Kz);
  const int extra = (int)std::min<long long>((pts + 255) / 256, 1024);
  const size_t smem = (size_t)(M1 + 2 * M1 * 6 * ea.col_tile) * e;
  auto k = xfwd_epi_kernel<T, EpiNS<T, false>>;
  set_smem(k, smem);
  const double ebytes = epi.io_bytes((long long)N1 * N2 * N3h) + (double)e * 6 * M1 * N2 * Kz;
  LaunchScope scope(c, "x-forward+epilogue", ebytes);
  k<<<ea.main_blocks + extra, 256, smem, c->stream>>>(ea, epi);
  return launch_ok(c, "x-forward+epilogue");
}

}  // namespace

extern "C" int psb_rhs_dns_noalloc(psb_ctx* c, const void* state, void* rhs, const psb_params* p) {
  if (!c) return PSB_ERR_ARG;
  if (!state || !rhs || !p) return fail(c, PSB_ERR_ARG, "psb_rhs_dns_noalloc: null argument");
  const size_t need = c->prec == 64 ? noalloc_bytes<double>(c) : noalloc_bytes<float>(c);
  if (need > kNoAllocBytes)
    return fail(c, PSB_ERR_SHAPE,
                "psb_rhs_dns_noalloc: grid needs " + std::to_string(need) + " scratch bytes, the fixed array holds " +
                    std::to_string(kNoAllocBytes) + " (N1*N2*N3 up to 32^3 in FP64, 2*32^3 in FP32); use psb_rhs");
  if (c->dev < 0 || c->dev >= kMaxDevices) return fail(c, PSB_ERR_ARG, "psb_rhs_dns_noalloc: device index too large");
  DeviceGuard restore;
  PSB_TRY(cuda_ok(c, cudaSetDevice(c->dev), "cudaSetDevice"));
  void* base = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_ptr[c->dev]) {
      void* ptr = nullptr;
      PSB_TRY(cuda_ok(c, cudaGetSymbolAddress(&ptr, g_noalloc_scratch), "cudaGetSymbolAddress(noalloc scratch)"));
      g_noalloc_ptr[c->dev] = ptr;
    }
    base = g_noalloc_ptr[c->dev];
  }
  if (c->prec == 64)
    return dns_noalloc<double>(c, reinterpret_cast<const Cx<double>*>(state), reinterpret_cast<Cx<double>*>(rhs), p,
                               static_cast<unsigned char*>(base));
  return dns_noalloc<float>(c, reinterpret_cast<const Cx<float>*>(state), reinterpret_cast<Cx<float>*>(rhs), p,
                            static_cast<unsigned char*>(base));
}
