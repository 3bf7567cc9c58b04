// C ABI of libpyspectral_b200: context lifetime, the RHS / RK4 entry points,
// FP64 diagnostics and plain transforms.  See include/pyspectral_b200.h.
#include <cstring>
#include <mutex>

#include "psb_ctx.cuh"

using namespace psb;
using namespace psbh;

namespace psbh {
template <typename T>
int rhs_dispatch(psb_ctx* c, int closure, StepIO<T> io, const psb_params* p, double* tau_out);
template <typename T>
StepIO<T> make_io(psb_ctx* c, void* Q, void* Q0, void* comp, void* rhs, void* read_out, void* w0, int mode,
                  double dtc);
template <typename T>
int sgs_dns_run(psb_ctx* c, const void* fields, void* w0, void* tau6);
template <typename T>
int products_run(psb_ctx* c, const void* fields, void* out6);
template <typename T>
int products_filtered_run(psb_ctx* c, const void* fields, void* out6);
int si_step(psb_ctx* c, void* Q, void* H, void* read_out, const psb_params* p);
}  // namespace psbh

namespace {

std::mutex g_create_mu;
std::string g_create_err;

bool smooth23(int L) {
  if (L < 2) return false;
  while (L % 2 == 0) L /= 2;
  while (L % 3 == 0) L /= 3;
  return L == 1;
}

// Default radix schedule: radix 8 first, then 4, 2, 3 (the fastest default
// measured on B200 at these lengths: larger radices raise register pressure
// more than they save passes).  The batch autotuner also tries the
// fewest-pass schedules over {16, 12, 8, 6, 4, 3, 2} and every radix order.
FFTPlan make_plan(int L) {
  FFTPlan p{};
  p.L = L;
  int n = L;
  while (n % 8 == 0) {
    p.radix[p.npass++] = 8;
    n /= 8;
  }
  while (n % 4 == 0) {
    p.radix[p.npass++] = 4;
    n /= 4;
  }
  while (n % 2 == 0) {
    p.radix[p.npass++] = 2;
    n /= 2;
  }
  while (n % 3 == 0) {
    p.radix[p.npass++] = 3;
    n /= 3;
  }
  return p;
}

// W_L^k = exp(-2 pi i k/L) in extended precision; exact at multiples of pi/2
void twiddle_table(int L, std::vector<long double>& re, std::vector<long double>& im) {
  re.resize(L);
  im.resize(L);
  const long double pi = 3.141592653589793238462643383279502884L;
  for (int k = 0; k < L; ++k) {
    long double c, s;
    if ((4LL * k) % L == 0) {
      const int q = (int)((4LL * k) / L) & 3;
      const long double cs[4] = {1, 0, -1, 0}, sn[4] = {0, 1, 0, -1};
      c = cs[q];
      s = sn[q];
    } else {
      const long double ang = 2.0L * pi * (long double)k / (long double)L;
      c = cosl(ang);
      s = sinl(ang);
    }
    re[k] = c;
    im[k] = -s;
  }
}

template <typename T>
__global__ void finite_count_kernel(const T* __restrict__ d, long long n, unsigned long long* cnt) {
  unsigned long long local = 0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    if (!isfinite(d[i])) ++local;
  if (local) atomicAdd(cnt, local);
}

// ---- reductions -------------------------------------------------------------
enum RedKind { kEnergy = 0, kEnstrophy = 1, kCross = 2 };

template <typename T>
__global__ void __launch_bounds__(256) reduce_kernel(const Cx<T>* __restrict__ a, const Cx<T>* __restrict__ b,
                                                     int kind, int filt, const double* __restrict__ k1,
                                                     const double* __restrict__ k2, const double* __restrict__ k3,
                                                     const double* __restrict__ g1, const double* __restrict__ g2,
                                                     const double* __restrict__ g3, int N1, int N2, int N3,
                                                     double* __restrict__ partial) {
  const int n3h = N3 / 2 + 1;
  const long long npts = (long long)N1 * N2 * n3h, fs = npts;
  double acc = 0.0;
  for (long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x; s < npts;
       s += (long long)gridDim.x * blockDim.x) {
    const int i3 = (int)(s % n3h);
    if (i3 >= N3 / 2 && i3 != 0) continue;  // k3 = N3/2 excluded (PySpectral/src/Classes.py:653-658)
    const long long t = s / n3h;
    const int i2 = (int)(t % N2), i1 = (int)(t / N2);
    const double w = i3 == 0 ? 1.0 : 2.0;
    const double g = filt ? g1[i1] * g2[i2] * g3[i3] : 1.0;
    double v = 0.0;
    if (kind == kEnergy) {
      for (int f = 0; f < 3; ++f) {
        const Cx<T> u = a[f * fs + s];
        v += (double)u.x * u.x + (double)u.y * u.y;
      }
      v *= g * g;
    } else if (kind == kCross) {
      for (int f = 0; f < 3; ++f) {
        const Cx<T> u = a[f * fs + s], B = b[f * fs + s];
        v += (double)u.x * B.x + (double)u.y * B.y;
      }
      v *= g * g;
    } else {
      const double kk1 = k1[i1], kk2 = k2[i2], kk3 = k3[i3];
      const Cx<T> u = a[s], vv = a[fs + s], ww = a[2 * fs + s];
      // omega = i k x u (PySpectral/src/Classes.py:734-736)
      const double o1x = -(kk2 * ww.y - kk3 * vv.y), o1y = kk2 * ww.x - kk3 * vv.x;
      const double o2x = -(kk3 * u.y - kk1 * ww.y), o2y = kk3 * u.x - kk1 * ww.x;
      const double o3x = -(kk1 * vv.y - kk2 * u.y), o3y = kk1 * vv.x - kk2 * u.x;
      v = (o1x * o1x + o1y * o1y + o2x * o2x + o2y * o2y + o3x * o3x + o3y * o3y) * g * g;
    }
    acc += w * v;
  }
  __shared__ double red[256];
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int h = blockDim.x / 2; h > 0; h >>= 1) {
    if ((int)threadIdx.x < h) red[threadIdx.x] += red[threadIdx.x + h];
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[blockIdx.x] = red[0];
}

// serial spectrum: int8 shell index with wrap, k3=N/2 excluded (PySpectral/src/Classes.py:762-797)
template <typename T>
__global__ void __launch_bounds__(256) spectrum_kernel(const Cx<T>* __restrict__ a, int filt,
                                                       const double* __restrict__ g1, const double* __restrict__ g2,
                                                       const double* __restrict__ g3, int N1, int N2, int N3,
                                                       int nbins, double* __restrict__ spec) {
  const int n3h = N3 / 2 + 1;
  const long long npts = (long long)N1 * N2 * n3h, fs = npts;
  for (long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x; s < npts;
       s += (long long)gridDim.x * blockDim.x) {
    const int i3 = (int)(s % n3h);
    if (i3 >= N3 / 2 && i3 != 0) continue;
    const long long t = s / n3h;
    const int i2 = (int)(t % N2), i1 = (int)(t / N2);
    const long long n1 = i1 < N1 / 2 ? i1 : i1 - N1, n2 = i2 < N2 / 2 ? i2 : i2 - N2, n3 = i3;
    const double km = rint(sqrt((double)(n1 * n1 + n2 * n2 + n3 * n3)));
    int bin = (int)(signed char)(long long)km;
    if (bin < 0) bin += nbins;
    if (bin < 0 || bin >= nbins) continue;
    const double w = i3 == 0 ? 1.0 : 2.0;
    const double g = filt ? g1[i1] * g2[i2] * g3[i3] : 1.0;
    for (int f = 0; f < 3; ++f) {
      const Cx<T> u = a[f * fs + s];
      atomicAdd(&spec[bin * 3 + f], w * g * g * ((double)u.x * u.x + (double)u.y * u.y));
    }
  }
}

// energy transfer spectra (PySpectral/src/Classes.py:988-1239), binned like
// spectrum_kernel, Nyquist modes of the state zeroed (they contribute
// nothing); spec[2 bin] += Re, spec[2 bin + 1] += Im.
//  mode 0 (computeTransfer): sum_i conj(u_i) (-i k_j P_ij - i k_i p), P the
//    3/2-dealiased products, p = ksqr_i (-k_i k_j P_ij);
//  mode 1 (computeTransfer_resolved): the same with u -> Gf u (P of Gf u);
//  mode 2 (computeTransfer_SGS): Re sum_i conj(Gf u_i) W_i (W = w0).
//  two_d (the *_2D variants, src/Classes.py:1043-1092,1152-1205,1241-1270):
//  the k3 = 0 plane only, bins rint(sqrt(k1^2 + k2^2)), components u and v,
//  weight 1.
template <typename T>
__global__ void __launch_bounds__(256) transfer_kernel(const Cx<T>* __restrict__ a, const Cx<T>* __restrict__ P,
                                                       int mode, int two_d, const double* __restrict__ gx,
                                                       const double* __restrict__ gy, const double* __restrict__ gz,
                                                       const double* __restrict__ kx, const double* __restrict__ ky,
                                                       const double* __restrict__ kz, int N1, int N2, int N3,
                                                       int nbins, double* __restrict__ spec) {
  const int n3h = N3 / 2 + 1;
  const long long npts = (long long)N1 * N2 * n3h, fs = npts;
  for (long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x; s < npts;
       s += (long long)gridDim.x * blockDim.x) {
    const int i3 = (int)(s % n3h);
    if (i3 >= N3 / 2 && i3 != 0) continue;
    if (two_d && i3 != 0) continue;
    const long long t = s / n3h;
    const int i2 = (int)(t % N2), i1 = (int)(t / N2);
    if (i1 == N1 / 2 || i2 == N2 / 2) continue;
    const long long n1 = i1 < N1 / 2 ? i1 : i1 - N1, n2 = i2 < N2 / 2 ? i2 : i2 - N2, n3 = i3;
    const double kh = two_d ? sqrt(kx[i1] * kx[i1] + ky[i2] * ky[i2]) : sqrt((double)(n1 * n1 + n2 * n2 + n3 * n3));
    int bin = (int)(signed char)(long long)rint(kh);
    if (bin < 0) bin += nbins;
    if (bin < 0 || bin >= nbins) continue;
    const double gf = mode ? gx[i1] * gy[i2] * gz[i3] : 1.0;
    const int ncomp = two_d ? 2 : 3;
    const double wgt = i3 == 0 ? 1.0 : 2.0;
    if (mode == 2) {
      double re = 0.0;
      for (int i = 0; i < ncomp; ++i) {
        const Cx<T> u = a[i * fs + s], q = P[i * fs + s];
        re += gf * ((double)u.x * q.x + (double)u.y * q.y);
      }
      atomicAdd(&spec[2 * bin], wgt * re);
      continue;
    }
    const double k[3] = {kx[i1], ky[i2], kz[i3]};
    double pr[6][2];
#pragma unroll
    for (int m = 0; m < 6; ++m) {
      const Cx<T> v = P[m * fs + s];
      pr[m][0] = v.x;
      pr[m][1] = v.y;
    }
    // P order 11, 22, 33, 12, 13, 23
    const int idx[3][3] = {{0, 3, 4}, {3, 1, 5}, {4, 5, 2}};
    const double ksi = 1.0 / (k[0] * k[0] + k[1] * k[1] + k[2] * k[2] + 1.0e-50);
    double ph[2];
#pragma unroll
    for (int c = 0; c < 2; ++c)
      ph[c] = ksi * (-k[0] * k[0] * pr[0][c] - k[1] * k[1] * pr[1][c] - k[2] * k[2] * pr[2][c] -
                     2.0 * k[0] * k[1] * pr[3][c] - 2.0 * k[0] * k[2] * pr[4][c] - 2.0 * k[1] * k[2] * pr[5][c]);
    double re = 0.0, im = 0.0;
    for (int i = 0; i < ncomp; ++i) {
      // z = k_j P_ij + k_i p; the advection term is -i z = (z.y, -z.x)
      double zx = k[i] * ph[0], zy = k[i] * ph[1];
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        zx += k[j] * pr[idx[i][j]][0];
        zy += k[j] * pr[idx[i][j]][1];
      }
      const Cx<T> u = a[i * fs + s];
      const double ux = gf * u.x, uy = gf * u.y;
      const double ax = zy, ay = -zx;
      re += ux * ax + uy * ay;  // conj(u) * (-i z)
      im += ux * ay - uy * ax;
    }
    atomicAdd(&spec[2 * bin], wgt * re);
    atomicAdd(&spec[2 * bin + 1], wgt * im);
  }
}

// MPI spectrum: int16 shells, all k3 (PySpectral/src_MPI/Classes.py:370-408)
template <typename T>
__global__ void __launch_bounds__(256) spectrum_mpi_kernel(const Cx<T>* __restrict__ a, int N1, int N2, int N3,
                                                           int nbins, double* __restrict__ spec) {
  const int n3h = N3 / 2 + 1;
  const long long npts = (long long)N1 * N2 * n3h, fs = npts;
  for (long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x; s < npts;
       s += (long long)gridDim.x * blockDim.x) {
    const int i3 = (int)(s % n3h);
    const long long t = s / n3h;
    const int i2 = (int)(t % N2), i1 = (int)(t / N2);
    const long long n1 = i1 < N1 / 2 ? i1 : i1 - N1, n2 = i2 < N2 / 2 ? i2 : i2 - N2, n3 = i3;
    int bin = (int)(short)(long long)rint(sqrt((double)(n1 * n1 + n2 * n2 + n3 * n3)));
    if (bin < 0 || bin >= nbins) continue;
    const double w = i3 == 0 ? 1.0 : 2.0;
    double e = 0.0;
    for (int f = 0; f < 3; ++f) {
      const Cx<T> u = a[f * fs + s];
      e += (double)u.x * u.x + (double)u.y * u.y;
    }
    atomicAdd(&spec[bin], w * e);
  }
}

// physical-space max for compute_dt (PySpectral/src/Classes.py:689-692)
template <typename T>
struct PhysCFL {
  static constexpr int F_IN = 3, F_OUT = 0;
  double idx, idy, idz;
  unsigned long long* out;
  __device__ __forceinline__ void operator()(long long, int, const T* in, T*) const {
    const double v = fabs((double)in[0]) * idx + fabs((double)in[1]) * idy + fabs((double)in[2]) * idz;
    atomicMax(out, __double_as_longlong(v));
  }
};

template <typename T>
struct PhysStoreReal {
  static constexpr int F_IN = 1, F_OUT = 0;
  T* phys;
  int n3;
  __device__ __forceinline__ void operator()(long long pen, int z, const T* in, T*) const { phys[pen * n3 + z] = in[0]; }
};

template <typename T>
struct PhysLoadReal {
  static constexpr int F_IN = 0, F_OUT = 1;
  const T* phys;
  int n3;
  __device__ __forceinline__ void operator()(long long pen, int z, const T*, T* out) const {
    out[0] = phys[pen * n3 + z];
  }
};

template <typename T>
int inverse_xy(psb_ctx* c, const Cx<T>* spec, int nf, int kz, Cx<T>** Bout) {
  const int N1 = c->N1, N2 = c->N2, N3h = c->N3h;
  int st = PSB_OK;
  Cx<T>* A = scratch<T>(c, "tr.A", (size_t)nf * N1 * N2 * kz, &st);
  Cx<T>* B = scratch<T>(c, "tr.B", (size_t)nf * N1 * N2 * kz, &st);
  if (st != PSB_OK) return st;
  AxisArgs<T> a{};
  a.plan = *plan_for(c, N1);
  a.tw = twiddles<T>(c);
  a.scale = (T)1;
  a.in = spec;
  a.out = A;
  a.in_fstride = (long long)N1 * N2 * N3h;
  a.in_ostride = N3h;
  a.in_rstride = (long long)N2 * N3h;
  a.out_fstride = (long long)N1 * N2 * kz;
  a.out_ostride = kz;
  a.out_rstride = (long long)N2 * kz;
  a.nouter = N2;
  a.ncols = kz;
  a.in_rows = N1;
  a.out_rows = N1;
  a.in_map = map_id(N1);
  a.out_map = map_id(N1);
  if (nf == 3) {
    PSB_TRY((launch_axis<T, true>(c, a, PreCopyN<T, 3>{}, "c2r x")));
  } else {
    PSB_TRY((launch_axis<T, true>(c, a, PreCopy<T>{}, "c2r x")));
  }
  AxisArgs<T> b{};
  b.plan = *plan_for(c, N2);
  b.tw = twiddles<T>(c);
  b.scale = (T)1;
  b.in = A;
  b.out = B;
  b.in_ostride = (long long)N2 * kz;
  b.in_rstride = kz;
  b.out_ostride = (long long)N2 * kz;
  b.out_rstride = kz;
  b.nouter = nf * N1;
  b.ncols = kz;
  b.in_rows = N2;
  b.out_rows = N2;
  b.in_map = map_id(N2);
  b.out_map = map_id(N2);
  PSB_TRY((launch_axis<T, true>(c, b, PreCopy<T>{}, "c2r y")));
  *Bout = B;
  return PSB_OK;
}

template <typename T>
int c2r_impl(psb_ctx* c, const void* spec, void* phys, int nfields) {
  const int N1 = c->N1, N2 = c->N2, N3 = c->N3, N3h = c->N3h;
  for (int f = 0; f < nfields; ++f) {
    const Cx<T>* s = reinterpret_cast<const Cx<T>*>(spec) + (size_t)f * N1 * N2 * N3h;
    T* ph = reinterpret_cast<T*>(phys) + (size_t)f * N1 * N2 * N3;
    Cx<T>* B = nullptr;
    PSB_TRY(inverse_xy<T>(c, s, 1, N3h, &B));
    ZArgs<T> z{};
    z.in[0] = B;
    z.in_pstride[0] = N3h;
    z.in_kz[0] = N3h;
    z.out_kz = 0;
    z.npencils = (long long)N1 * N2;
    z.fac = (T)(1.0 / ((double)N1 * N2 * N3));
    z.plan = *plan_for(c, N3);
    z.tw = twiddles<T>(c);
    PSB_TRY(launch_z<T>(c, z, PhysStoreReal<T>{ph, N3}, "c2r z"));
  }
  return PSB_OK;
}

template <typename T>
int r2c_impl(psb_ctx* c, const void* phys, void* spec, int nfields) {
  const int N1 = c->N1, N2 = c->N2, N3 = c->N3, N3h = c->N3h;
  int st = PSB_OK;
  Cx<T>* A = scratch<T>(c, "tr.A", (size_t)N1 * N2 * N3h, &st);
  Cx<T>* B = scratch<T>(c, "tr.B", (size_t)N1 * N2 * N3h, &st);
  if (st != PSB_OK) return st;
  for (int f = 0; f < nfields; ++f) {
    const T* ph = reinterpret_cast<const T*>(phys) + (size_t)f * N1 * N2 * N3;
    Cx<T>* out = reinterpret_cast<Cx<T>*>(spec) + (size_t)f * N1 * N2 * N3h;
    ZArgs<T> z{};
    z.out[0] = A;
    z.out_pstride[0] = N3h;
    z.out_kz = N3h;
    z.npencils = (long long)N1 * N2;
    z.fac = (T)1;
    z.plan = *plan_for(c, N3);
    z.tw = twiddles<T>(c);
    PSB_TRY(launch_z<T>(c, z, PhysLoadReal<T>{ph, N3}, "r2c z"));
    AxisArgs<T> b{};
    b.plan = *plan_for(c, N2);
    b.tw = twiddles<T>(c);
    b.scale = (T)1;
    b.in = A;
    b.out = B;
    b.in_ostride = (long long)N2 * N3h;
    b.in_rstride = N3h;
    b.out_ostride = (long long)N2 * N3h;
    b.out_rstride = N3h;
    b.nouter = N1;
    b.ncols = N3h;
    b.in_rows = N2;
    b.out_rows = N2;
    b.in_map = map_id(N2);
    b.out_map = map_id(N2);
    PSB_TRY((launch_axis<T, false>(c, b, PreCopy<T>{}, "r2c y")));
    AxisArgs<T> a{};
    a.plan = *plan_for(c, N1);
    a.tw = twiddles<T>(c);
    a.scale = (T)1;
    a.in = B;
    a.out = out;
    a.in_ostride = N3h;
    a.in_rstride = (long long)N2 * N3h;
    a.out_ostride = N3h;
    a.out_rstride = (long long)N2 * N3h;
    a.nouter = N2;
    a.ncols = N3h;
    a.in_rows = N1;
    a.out_rows = N1;
    a.in_map = map_id(N1);
    a.out_map = map_id(N1);
    PSB_TRY((launch_axis<T, false>(c, a, PreCopy<T>{}, "r2c x")));
  }
  return PSB_OK;
}

// ---- slab-decomposed transforms of the MPI solver -------------------------
// One rank of P holds the spectra of an x slab, (Npx, N2, N3/2+1), and the
// physical field of a y slab, (N1, Npy, N3): FFTclass.myifft3D / myfft3D,
// PySpectral/src_MPI/Classes.py:244-258.  Between the halves the caller runs
// an all-to-all of equal blocks (block p of the send buffer to rank p).
// Inverse: the DFT along y of the x slab is written in the blocked layout
// (P, Npx, Npy, Kz) -- block p holds the rows of rank p's y slab -- so that
// every block is contiguous; the block received from rank p holds p's x slab,
// so the received buffer is (N1, Npy, Kz) in order, transformed along x and
// (c2r) along z.  Forward: r2c along z and the DFT along x of the y slab give
// (N1, Npy, Kz) = (P, Npx, Npy, Kz) in order; after the exchange block p holds
// rank p's y rows, which the y pass reads blocked.
template <typename T>
struct SlabY {
  const Cx<T>* in;
  Cx<T>* out;
  int N2, Npx, Npy, Kz, ct;
  int blocked_out;  // 1: natural in, blocked out (inverse); 0: blocked in, natural out
  FFTPlan plan;
  const Cx<T>* tw;
};

// element (x, y, k3) of a slab: natural (Npx, N2, Kz) or blocked (P, Npx, Npy, Kz)
template <typename T>
__device__ __forceinline__ long long slab_off(const SlabY<T>& a, bool blocked, int x, int y, int k) {
  if (!blocked) return ((long long)x * a.N2 + y) * a.Kz + k;
  const int p = y / a.Npy, yy = y - p * a.Npy;
  return (((long long)p * a.Npx + x) * a.Npy + yy) * a.Kz + k;
}

// grid (ceil(Kz/ct), Npx); a CTA transforms ct consecutive k3 columns of one
// x along y (ct a power of two dividing the CTA); smem = (N2 + 2 N2 ct) complex
template <typename T, bool INV>
__global__ void __launch_bounds__(256) slab_y_kernel(SlabY<T> a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Cx<T>* tw = reinterpret_cast<Cx<T>*>(smem_raw);
  const int L = a.N2, ct = a.ct;
  Cx<T>* bufA = tw + L;
  Cx<T>* bufB = bufA + (size_t)L * ct;
  const int x = blockIdx.y;
  stage_twiddles(tw, a.tw, a.plan);
  const int c = threadIdx.x % ct, r0 = threadIdx.x / ct, dr = blockDim.x / ct;
  const int k = blockIdx.x * ct + c;
  const bool ok = k < a.Kz;
  const bool bin = a.blocked_out == 0;
  for (int y = r0; y < L; y += dr) bufA[(size_t)y * ct + c] = ok ? a.in[slab_off(a, bin, x, y, k)] : mk<T>(0, 0);
  __syncthreads();
  const Cx<T>* res = block_fft<T, INV, false>(bufA, bufB, a.plan, tw, ct, 1, ct, true);
  if (!ok) return;
  for (int y = r0; y < L; y += dr) a.out[slab_off(a, !bin, x, y, k)] = res[(size_t)y * ct + c];
}

int slab_check(psb_ctx* c, int P, const char* what) {
  if (P < 1 || c->N1 % P != 0 || c->N2 % P != 0)
    return fail(c, PSB_ERR_SHAPE, std::string(what) + ": N1 and N2 must be multiples of nprocs");
  return PSB_OK;
}

template <typename T>
int slab_y_impl(psb_ctx* c, int P, const void* in, void* out, bool inverse) {
  const size_t esz = sizeof(Cx<T>);
  SlabY<T> a{};
  a.in = reinterpret_cast<const Cx<T>*>(in);
  a.out = reinterpret_cast<Cx<T>*>(out);
  a.N2 = c->N2;
  a.Npx = c->N1 / P;
  a.Npy = c->N2 / P;
  a.Kz = c->N3h;
  a.blocked_out = inverse ? 1 : 0;
  a.plan = *plan_for(c, c->N2);
  a.tw = twiddles<T>(c);
  a.ct = pick_ct(a.Kz, 1, a.N2, esz, a.Npx);
  const size_t smem = (size_t)(a.N2 + 2 * (size_t)a.N2 * a.ct) * esz;
  const dim3 grid((unsigned)((a.Kz + a.ct - 1) / a.ct), (unsigned)a.Npx);
  const char* what = inverse ? "slab y-inverse" : "slab y-forward";
  auto k = inverse ? slab_y_kernel<T, true> : slab_y_kernel<T, false>;
  set_smem(k, smem);
  LaunchScope scope(c, what, 2.0 * esz * a.Npx * a.N2 * a.Kz);
  k<<<grid, 256, smem, c->stream>>>(a);
  return launch_ok(c, what);
}

// x pass of a y slab (N1 rows x Npy outer x Kz columns, natural order)
template <typename T>
AxisArgs<T> slab_x_args(psb_ctx* c, int P, const Cx<T>* in, Cx<T>* out) {
  const int N1 = c->N1, Npy = c->N2 / P, Kz = c->N3h;
  AxisArgs<T> a{};
  a.plan = *plan_for(c, N1);
  a.tw = twiddles<T>(c);
  a.scale = (T)1;
  a.in = in;
  a.out = out;
  a.in_ostride = Kz;
  a.in_rstride = (long long)Npy * Kz;
  a.out_ostride = Kz;
  a.out_rstride = (long long)Npy * Kz;
  a.nouter = Npy;
  a.ncols = Kz;
  a.in_rows = N1;
  a.out_rows = N1;
  a.in_map = map_id(N1);
  a.out_map = map_id(N1);
  return a;
}

// received blocks (N1, Npy, Kz) -> physical y slab (N1, Npy, N3): inverse DFT
// along x, c2r along z, the whole 1/(N1 N2 N3) of the reference's ifft/irfft2
template <typename T>
int slab_xz_inverse(psb_ctx* c, int P, const void* recv, void* phys) {
  const int N1 = c->N1, Npy = c->N2 / P, N3 = c->N3, Kz = c->N3h;
  int st = PSB_OK;
  Cx<T>* A = scratch<T>(c, "slab.A", (size_t)N1 * Npy * Kz, &st);
  if (st != PSB_OK) return st;
  PSB_TRY((launch_axis<T, true>(c, slab_x_args<T>(c, P, reinterpret_cast<const Cx<T>*>(recv), A), PreCopy<T>{},
                                "slab x-inverse")));
  ZArgs<T> z{};
  z.in[0] = A;
  z.in_pstride[0] = Kz;
  z.in_kz[0] = Kz;
  z.out_kz = 0;
  z.npencils = (long long)N1 * Npy;
  z.fac = (T)(1.0 / ((double)N1 * c->N2 * N3));
  z.plan = *plan_for(c, N3);
  z.tw = twiddles<T>(c);
  return launch_z<T>(c, z, PhysStoreReal<T>{reinterpret_cast<T*>(phys), N3}, "slab z c2r");
}

// physical y slab (N1, Npy, N3) -> send (N1, Npy, Kz): r2c along z, DFT along x
template <typename T>
int slab_xz_forward(psb_ctx* c, int P, const void* phys, void* send) {
  const int N1 = c->N1, Npy = c->N2 / P, N3 = c->N3, Kz = c->N3h;
  int st = PSB_OK;
  Cx<T>* A = scratch<T>(c, "slab.A", (size_t)N1 * Npy * Kz, &st);
  if (st != PSB_OK) return st;
  ZArgs<T> z{};
  z.out[0] = A;
  z.out_pstride[0] = Kz;
  z.out_kz = Kz;
  z.npencils = (long long)N1 * Npy;
  z.fac = (T)1;
  z.plan = *plan_for(c, N3);
  z.tw = twiddles<T>(c);
  PSB_TRY(launch_z<T>(c, z, PhysLoadReal<T>{reinterpret_cast<const T*>(phys), N3}, "slab z r2c"));
  return launch_axis<T, false>(c, slab_x_args<T>(c, P, A, reinterpret_cast<Cx<T>*>(send)), PreCopy<T>{},
                               "slab x-forward");
}

template <typename T, int F>
struct PhysStoreN {
  static constexpr int F_IN = F, F_OUT = 0;
  T* phys;
  long long fs;
  int n3;
  __device__ __forceinline__ void operator()(long long pen, int z, const T* in, T*) const {
#pragma unroll
    for (int f = 0; f < F; ++f) phys[f * fs + pen * n3 + z] = in[f];
  }
};

// physical u (and its gradients) on the N grid, irfftn(uhat)*sqrt(N1 N2 N3)
template <typename T, class Pre>
int physical_impl(psb_ctx* c, const void* fields, void* out, Pre pre) {
  constexpr int F = Pre::F_DST;
  const int N1 = c->N1, N2 = c->N2, N3 = c->N3, N3h = c->N3h;
  int st = PSB_OK;
  Cx<T>* A = scratch<T>(c, "phys.A", (size_t)F * N1 * N2 * N3h, &st);
  Cx<T>* B = scratch<T>(c, "phys.B", (size_t)F * N1 * N2 * N3h, &st);
  if (st != PSB_OK) return st;
  AxisArgs<T> a{};
  a.plan = *plan_for(c, N1);
  a.tw = twiddles<T>(c);
  a.scale = (T)1;
  a.in = reinterpret_cast<const Cx<T>*>(fields);
  a.out = A;
  a.in_fstride = (long long)N1 * N2 * N3h;
  a.in_ostride = N3h;
  a.in_rstride = (long long)N2 * N3h;
  a.out_fstride = (long long)N1 * N2 * N3h;
  a.out_ostride = N3h;
  a.out_rstride = (long long)N2 * N3h;
  a.nouter = N2;
  a.ncols = N3h;
  a.in_rows = N1;
  a.out_rows = N1;
  a.in_map = map_id(N1);
  a.out_map = map_id(N1);
  a.k_row = c->kx;
  a.k_outer = c->ky;
  a.k_col = c->kz;
  PSB_TRY((launch_axis<T, true>(c, a, pre, "physical x")));
  AxisArgs<T> b{};
  b.plan = *plan_for(c, N2);
  b.tw = twiddles<T>(c);
  b.scale = (T)1;
  b.in = A;
  b.out = B;
  b.in_ostride = (long long)N2 * N3h;
  b.in_rstride = N3h;
  b.out_ostride = (long long)N2 * N3h;
  b.out_rstride = N3h;
  b.nouter = F * N1;
  b.ncols = N3h;
  b.in_rows = N2;
  b.out_rows = N2;
  b.in_map = map_id(N2);
  b.out_map = map_id(N2);
  PSB_TRY((launch_axis<T, true>(c, b, PreCopy<T>{}, "physical y")));
  ZArgs<T> z{};
  const long long fs = (long long)N1 * N2 * N3h;
  for (int f = 0; f < F; ++f) {
    z.in[f] = B + f * fs;
    z.in_pstride[f] = N3h;
    z.in_kz[f] = N3h;
  }
  z.npencils = (long long)N1 * N2;
  z.fac = (T)(std::sqrt((double)N1 * N2 * N3) / ((double)N1 * N2 * N3));
  z.plan = *plan_for(c, N3);
  z.tw = twiddles<T>(c);
  PhysStoreN<T, F> ph{reinterpret_cast<T*>(out), (long long)N1 * N2 * N3, N3};
  return launch_z<T>(c, z, ph, "physical z", (double)sizeof(T) * F * N1 * N2 * N3);
}

template <typename T>
__global__ void resample_kernel(const Cx<T>* __restrict__ src, int N1, int N2, int N3, Cx<T>* __restrict__ dst,
                                int n1, int n2, int n3, int nf, int kc, T scale) {
  const int h3 = n3 / 2 + 1, H3 = N3 / 2 + 1;
  const long long npts = (long long)n1 * n2 * h3;
  for (long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x; s < npts * nf;
       s += (long long)gridDim.x * blockDim.x) {
    const int f = (int)(s / npts);
    const long long q = s - f * npts;
    const int i3 = (int)(q % h3);
    const long long t = q / h3;
    const int i2 = (int)(t % n2), i1 = (int)(t / n2);
    const int k1 = i1 < n1 / 2 ? i1 : i1 - n1, k2 = i2 < n2 / 2 ? i2 : i2 - n2, k3 = i3;
    Cx<T> v = mk<T>(0, 0);
    const bool keep = abs(k1) < kc && abs(k2) < kc && k3 < kc && abs(k1) < N1 / 2 && abs(k2) < N2 / 2 &&
                      k3 < N3 / 2 && !(i1 == n1 / 2) && !(i2 == n2 / 2);
    if (keep) {
      const int j1 = k1 >= 0 ? k1 : k1 + N1, j2 = k2 >= 0 ? k2 : k2 + N2;
      v = scale * src[(long long)f * N1 * N2 * H3 + ((long long)j1 * N2 + j2) * H3 + k3];
    }
    dst[s] = v;
  }
}

template <typename T>
int cfl_impl(psb_ctx* c, const void* fields, double* vmax) {
  const int N1 = c->N1, N2 = c->N2, N3 = c->N3, N3h = c->N3h;
  Cx<T>* B = nullptr;
  PSB_TRY(inverse_xy<T>(c, reinterpret_cast<const Cx<T>*>(fields), 3, N3h, &B));
  int st = PSB_OK;
  unsigned long long* dmax =
      reinterpret_cast<unsigned long long*>(scratch<double>(c, "cfl.max", 1, &st));
  if (st != PSB_OK) return st;
  PSB_TRY(cuda_ok(c, cudaMemsetAsync(dmax, 0, sizeof(unsigned long long), c->stream), "memset"));
  ZArgs<T> z{};
  const long long fs = (long long)N1 * N2 * N3h;
  for (int f = 0; f < 3; ++f) {
    z.in[f] = B + f * fs;
    z.in_pstride[f] = N3h;
    z.in_kz[f] = N3h;
  }
  z.npencils = (long long)N1 * N2;
  // irfftn(uhat)*sqrt(N1 N2 N3) (PySpectral/src/Classes.py:689-691)
  z.fac = (T)(std::sqrt((double)N1 * N2 * N3) / ((double)N1 * N2 * N3));
  z.plan = *plan_for(c, N3);
  z.tw = twiddles<T>(c);
  PSB_TRY(launch_z<T>(c, z, PhysCFL<T>{1.0 / c->dx, 1.0 / c->dy, 1.0 / c->dz, dmax}, "cfl z"));
  unsigned long long h = 0;
  PSB_TRY(cuda_ok(c, cudaMemcpyAsync(&h, dmax, sizeof(h), cudaMemcpyDeviceToHost, c->stream), "cfl copy"));
  PSB_TRY(cuda_ok(c, cudaStreamSynchronize(c->stream), "cfl sync"));
  std::memcpy(vmax, &h, sizeof(double));
  return PSB_OK;
}

constexpr int kRedBlocks = 296;

int ensure_red(psb_ctx* c, size_t n) {
  if (c->red_cap >= n) return PSB_OK;
  if (c->red_dev) cudaFree(c->red_dev);
  if (c->red_host) cudaFreeHost(c->red_host);
  c->red_dev = nullptr;
  c->red_host = nullptr;
  c->red_cap = 0;
  PSB_TRY(cuda_ok(c, cudaMalloc(&c->red_dev, n * sizeof(double)), "reduction buffer"));
  PSB_TRY(cuda_ok(c, cudaMallocHost(&c->red_host, n * sizeof(double)), "reduction host buffer"));
  c->red_cap = n;
  return PSB_OK;
}

template <typename T>
int reduce_impl(psb_ctx* c, const void* a, const void* b, int kind, int filt, double* sum) {
  PSB_TRY(ensure_red(c, kRedBlocks));
  reduce_kernel<T><<<kRedBlocks, 256, 0, c->stream>>>(reinterpret_cast<const Cx<T>*>(a),
                                                       reinterpret_cast<const Cx<T>*>(b), kind, filt, c->kx, c->ky,
                                                       c->kz, c->gx, c->gy, c->gz, c->N1, c->N2, c->N3, c->red_dev);
  PSB_TRY(launch_ok(c, "reduce"));
  PSB_TRY(cuda_ok(c, cudaMemcpyAsync(c->red_host, c->red_dev, kRedBlocks * sizeof(double), cudaMemcpyDeviceToHost,
                                     c->stream),
                  "reduce copy"));
  PSB_TRY(cuda_ok(c, cudaStreamSynchronize(c->stream), "reduce sync"));
  double s = 0.0;
  for (int i = 0; i < kRedBlocks; ++i) s += c->red_host[i];
  *sum = s;
  return PSB_OK;
}

int check_ctx(psb_ctx* c) { return c ? PSB_OK : PSB_ERR_ARG; }

int set_device(psb_ctx* c) { return cuda_ok(c, cudaSetDevice(c->dev), "cudaSetDevice"); }

}  // namespace

// ===========================================================================
extern "C" {

const char* psb_create_error(void) {
  std::lock_guard<std::mutex> g(g_create_mu);
  return g_create_err.c_str();
}

int psb_ctx_create(const psb_grid* g, int precision, int device, psb_ctx** out) {
  auto cfail = [](const std::string& m, int code) {
    std::lock_guard<std::mutex> lk(g_create_mu);
    g_create_err = m;
    return code;
  };
  if (!g || !out) return cfail("null argument", PSB_ERR_ARG);
  *out = nullptr;
  if (precision != 32 && precision != 64) return cfail("precision must be 32 or 64", PSB_ERR_ARG);
  const int Ns[3] = {g->N1, g->N2, g->N3};
  for (int n : Ns) {
    if (n < 8 || n % 4 != 0) return cfail("grid sizes must be multiples of 4 and >= 8", PSB_ERR_SHAPE);
    if (!smooth23(n) || !smooth23(3 * n / 2) || !smooth23(2 * n))
      return cfail("grid size " + std::to_string(n) + ": N, 3N/2 and 2N must factor as 2^a 3^b", PSB_ERR_SHAPE);
    if (2 * n > 1024 || 3 * n / 2 > 1024) return cfail("grid size too large (max 512)", PSB_ERR_SHAPE);
  }
  if (!(g->L1 > 0 && g->L2 > 0 && g->L3 > 0)) return cfail("L1, L2, L3 must be positive", PSB_ERR_ARG);
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev)
    return cfail("no such CUDA device", PSB_ERR_CUDA);
  if (cudaSetDevice(device) != cudaSuccess) return cfail("cudaSetDevice failed", PSB_ERR_CUDA);
  psb_ctx* c = new psb_ctx();
  c->N1 = g->N1;
  c->N2 = g->N2;
  c->N3 = g->N3;
  c->N3h = g->N3 / 2 + 1;
  c->prec = precision;
  c->dev = device;
  c->L1 = g->L1;
  c->L2 = g->L2;
  c->L3 = g->L3;
  c->dx = g->dx;
  c->dy = g->dy;
  c->dz = g->dz;
  c->kc = g->kc;
  c->Delta = std::pow(g->dx * g->dy * g->dz, 1.0 / 3.0);
  // plans + twiddles for N, 3N/2, 2N and 3N of each axis (3N: the second-order
  // finite memory model's products on the 3/2-padded 2x grid)
  std::vector<int> Ls;
  for (int n : Ns)
    for (int L : {n, 3 * n / 2, 2 * n, 3 * n})
      if (std::find(Ls.begin(), Ls.end(), L) == Ls.end()) Ls.push_back(L);
  std::vector<Cx<double>> twd;
  std::vector<Cx<float>> twf;
  for (int L : Ls) {
    FFTPlan p = make_plan(L);
    p.tw_off = (int)twd.size();
    std::vector<long double> re, im;
    twiddle_table(L, re, im);
    for (int k = 0; k < L; ++k) {
      twd.push_back(mk<double>((double)re[k], (double)im[k]));
      twf.push_back(mk<float>((float)re[k], (float)im[k]));
    }
    c->plans[L] = p;
  }
  auto upload = [&](const void* h, size_t bytes, void** d) -> bool {
    if (cudaMalloc(d, bytes) != cudaSuccess) return false;
    c->owned.push_back(*d);
    return cudaMemcpy(*d, h, bytes, cudaMemcpyHostToDevice) == cudaSuccess;
  };
  bool ok = upload(twd.data(), twd.size() * sizeof(Cx<double>), &c->tw_d) &&
            upload(twf.data(), twf.size() * sizeof(Cx<float>), &c->tw_f);
  // wavenumbers with the reference's float operations:
  // fftshift(linspace(-N/2,N/2-1,N)) * 2. * pi / L  (PySpectral/src/Classes.py:565-570)
  const double PI = 3.141592653589793;
  auto kvec = [&](int n, double L, bool half, bool twice) {
    std::vector<double> k;
    if (half) {
      const int m = twice ? n + 1 : n / 2 + 1;
      for (int i = 0; i < m; ++i) k.push_back((double)i * 2. * PI / L);
    } else {
      const int m = twice ? 2 * n : n;
      for (int i = 0; i < m; ++i) {
        const int idx = i < m / 2 ? i : i - m;
        k.push_back((double)idx * 2. * PI / L);
      }
    }
    return k;
  };
  std::vector<double> k1 = kvec(c->N1, c->L1, false, false), k2 = kvec(c->N2, c->L2, false, false),
                      k3 = kvec(c->N3, c->L3, true, false);
  std::vector<double> k1f = kvec(c->N1, c->L1, false, true), k2f = kvec(c->N2, c->L2, false, true),
                      k3f = kvec(c->N3, c->L3, true, true);
  ok = ok && upload(k1.data(), k1.size() * 8, (void**)&c->kx) && upload(k2.data(), k2.size() * 8, (void**)&c->ky) &&
       upload(k3.data(), k3.size() * 8, (void**)&c->kz) && upload(k1f.data(), k1f.size() * 8, (void**)&c->kxf) &&
       upload(k2f.data(), k2f.size() * 8, (void**)&c->kyf) && upload(k3f.data(), k3f.size() * 8, (void**)&c->kzf);
  // 2/3-rule masks (PySpectral/src_MPI/Classes.py:206-218)
  std::vector<double> mx(c->N1, 1.0), my(c->N2, 1.0), mz(c->N3h, 1.0);
  for (int i = 0; i < c->N1; ++i)
    if (std::fabs(k1[i]) >= (c->N1 / 2) * 2. / 3. * 2. * PI / c->L1) mx[i] = 0.0;
  for (int i = 0; i < c->N2; ++i)
    if (std::fabs(k2[i]) >= (c->N2 / 2) * 2. / 3. * 2. * PI / c->L2) my[i] = 0.0;
  c->kz_mhd = c->N3h;
  if (c->N3 != 2) {
    c->kz_mhd = (int)((c->N3 / 2) * 2. / 3.);
    for (int i = c->kz_mhd; i < c->N3h; ++i) mz[i] = 0.0;
  }
  // sharp cutoff Gf per axis (PySpectral/src/Classes.py:584-588)
  std::vector<double> gx(c->N1, 0.0), gy(c->N2, 0.0), gz(c->N3h, 0.0);
  const int kc = c->kc;
  for (int i = 0; i < c->N1; ++i) gx[i] = (i < kc || i >= c->N1 - kc + 1) ? 1.0 : 0.0;
  for (int i = 0; i < c->N2; ++i) gy[i] = (i < kc || i >= c->N2 - kc + 1) ? 1.0 : 0.0;
  for (int i = 0; i < c->N3h; ++i) gz[i] = i < kc ? 1.0 : 0.0;
  ok = ok && upload(mx.data(), mx.size() * 8, (void**)&c->mx) && upload(my.data(), my.size() * 8, (void**)&c->my) &&
       upload(mz.data(), mz.size() * 8, (void**)&c->mz) && upload(gx.data(), gx.size() * 8, (void**)&c->gx) &&
       upload(gy.data(), gy.size() * 8, (void**)&c->gy) && upload(gz.data(), gz.size() * 8, (void**)&c->gz);
  // device status word: raised by a kernel whose bounded wait gave up
  const int zero_status = 0;
  ok = ok && upload(&zero_status, sizeof(int), (void**)&c->dstatus);
  if (!ok) {
    std::string m = std::string("table upload failed: ") + cudaGetErrorString(cudaGetLastError());
    psb_ctx_destroy(c);
    return cfail(m, PSB_ERR_CUDA);
  }
  *out = c;
  return PSB_OK;
}

int psb_ctx_destroy(psb_ctx* c) {
  if (!c) return PSB_ERR_ARG;
  cudaSetDevice(c->dev);
  for (auto& kv : c->scratch)
    if (kv.second.p) cudaFree(kv.second.p);
  for (void* p : c->owned) cudaFree(p);
  if (c->red_dev) cudaFree(c->red_dev);
  if (c->red_host) cudaFreeHost(c->red_host);
  delete c;
  return PSB_OK;
}

int psb_ctx_set_tma(psb_ctx* c, int enable) {
  PSB_TRY(check_ctx(c));
  c->use_tma = enable ? 1 : 0;
  return PSB_OK;
}

int psb_ctx_set_zrr(psb_ctx* c, int enable) {
  PSB_TRY(check_ctx(c));
  c->use_zrr = enable ? 1 : 0;
  return PSB_OK;
}

int psb_device_status(psb_ctx* c, int* status) {
  PSB_TRY(check_ctx(c));
  if (!status) return fail(c, PSB_ERR_ARG, "psb_device_status: null argument");
  PSB_TRY(set_device(c));
  int h = 0;
  PSB_TRY(cuda_ok(c, cudaMemcpyAsync(&h, c->dstatus, sizeof(int), cudaMemcpyDeviceToHost, c->stream), "status read"));
  PSB_TRY(cuda_ok(c, cudaMemsetAsync(c->dstatus, 0, sizeof(int), c->stream), "status clear"));
  PSB_TRY(cuda_ok(c, cudaStreamSynchronize(c->stream), "status sync"));
  *status = h;
  return PSB_OK;
}

int psb_ctx_set_stream(psb_ctx* c, void* stream) {
  PSB_TRY(check_ctx(c));
  c->stream = reinterpret_cast<cudaStream_t>(stream);
  return PSB_OK;
}

const char* psb_last_error(const psb_ctx* c) { return c ? c->err.c_str() : "null context"; }

static int closure_fields(int closure, const psb_params* p) {
  if (closure == PSB_FM1) return 3 + 3 * (p && p->fm_nsub > 0 ? p->fm_nsub : 1);
  if (closure == PSB_FM2) return 3 + 6 * (p && p->fm_nsub > 0 ? p->fm_nsub : 1);
  return closure == PSB_MHD || closure == PSB_MHD_TMODEL || closure == PSB_CM1 ? 6 : 3;
}

int psb_rhs(psb_ctx* c, int closure, const void* state, void* rhs, void* w0, void* read_out, const psb_params* p,
            double* tau_out) {
  PSB_TRY(check_ctx(c));
  if (!state || !rhs || !p) return fail(c, PSB_ERR_ARG, "psb_rhs: null argument");
  PSB_TRY(set_device(c));
  if (c->prec == 64) {
    StepIO<double> io = make_io<double>(c, const_cast<void*>(state), nullptr, nullptr, rhs, read_out, w0, kRHS, 0.0);
    return rhs_dispatch<double>(c, closure, io, p, tau_out);
  }
  StepIO<float> io = make_io<float>(c, const_cast<void*>(state), nullptr, nullptr, rhs, read_out, w0, kRHS, 0.0);
  return rhs_dispatch<float>(c, closure, io, p, tau_out);
}

int psb_prepare(psb_ctx* c, int closure) {
  PSB_TRY(check_ctx(c));
  psb_params p{};
  p.nu = 0;
  p.eta = -1;
  PSB_TRY(set_device(c));
  const size_t n = (size_t)closure_fields(closure, &p) * c->N1 * c->N2 * c->N3h;
  int st = PSB_OK;
  if (c->prec == 64) {
    scratch<double>(c, "rk.Q0", n, &st);
    if (st != PSB_OK) return st;
    StepIO<double> io{};
    return rhs_dispatch<double>(c, closure, io, &p, nullptr);
  }
  scratch<float>(c, "rk.Q0", n, &st);
  if (st != PSB_OK) return st;
  StepIO<float> io{};
  return rhs_dispatch<float>(c, closure, io, &p, nullptr);
}

int psb_step_si(psb_ctx* c, void* state, void* H, void* read_out, const psb_params* p, int nsteps) {
  PSB_TRY(check_ctx(c));
  if (!state || !H || !p || nsteps < 0) return fail(c, PSB_ERR_ARG, "psb_step_si: bad argument");
  PSB_TRY(set_device(c));
  for (int s = 0; s < nsteps; ++s) PSB_TRY(si_step(c, state, H, s == nsteps - 1 ? read_out : nullptr, p));
  return PSB_OK;
}

int psb_step_rk4(psb_ctx* c, int closure, void* state, void* comp, void* read_out, const psb_params* p, int nsteps) {
  PSB_TRY(check_ctx(c));
  if (!state || !p || nsteps < 0) return fail(c, PSB_ERR_ARG, "psb_step_rk4: bad argument");
  PSB_TRY(set_device(c));
  const double rk[4] = {1. / 4, 1. / 3, 1. / 2, 1.};
  const size_t n = (size_t)closure_fields(closure, p) * c->N1 * c->N2 * c->N3h;
  int st = PSB_OK;
  for (int s = 0; s < nsteps; ++s) {
    for (int i = 0; i < 4; ++i) {
      const int mode = i == 0 ? kStage1 : (i == 3 ? kStageLast : kStageMid);
      void* rd = (i == 3 && s == nsteps - 1) ? read_out : nullptr;
      const double dtc = p->dt * rk[i];
      if (c->prec == 64) {
        Cx<double>* Q0 = scratch<double>(c, "rk.Q0", n, &st);
        if (st != PSB_OK) return st;
        StepIO<double> io = make_io<double>(c, state, Q0, comp, nullptr, rd, nullptr, mode, dtc);
        PSB_TRY(rhs_dispatch<double>(c, closure, io, p, nullptr));
      } else {
        Cx<float>* Q0 = scratch<float>(c, "rk.Q0", n, &st);
        if (st != PSB_OK) return st;
        StepIO<float> io = make_io<float>(c, state, Q0, comp, nullptr, rd, nullptr, mode, dtc);
        PSB_TRY(rhs_dispatch<float>(c, closure, io, p, nullptr));
      }
    }
  }
  return PSB_OK;
}

int psb_energy(psb_ctx* c, const void* f, int flags, double* out) {
  PSB_TRY(check_ctx(c));
  if (!f || !out) return fail(c, PSB_ERR_ARG, "psb_energy: null argument");
  PSB_TRY(set_device(c));
  double s = 0;
  const int filt = (flags & PSB_FILTER_GF) ? 1 : 0;
  PSB_TRY(c->prec == 64 ? reduce_impl<double>(c, f, nullptr, kEnergy, filt, &s)
                        : reduce_impl<float>(c, f, nullptr, kEnergy, filt, &s));
  const double nnn = (double)c->N1 * c->N2 * c->N3;
  *out = (flags & PSB_NORM_MPI) ? 0.5 * s / (nnn * nnn) : 0.5 * s / nnn;
  return PSB_OK;
}

int psb_enstrophy(psb_ctx* c, const void* f, int flags, double* out) {
  PSB_TRY(check_ctx(c));
  if (!f || !out) return fail(c, PSB_ERR_ARG, "psb_enstrophy: null argument");
  PSB_TRY(set_device(c));
  double s = 0;
  const int filt = (flags & PSB_FILTER_GF) ? 1 : 0;
  PSB_TRY(c->prec == 64 ? reduce_impl<double>(c, f, nullptr, kEnstrophy, filt, &s)
                        : reduce_impl<float>(c, f, nullptr, kEnstrophy, filt, &s));
  const double nnn = (double)c->N1 * c->N2 * c->N3;
  *out = (flags & PSB_NORM_MPI) ? 0.5 * s / (nnn * nnn) : 0.5 * s / nnn;
  return PSB_OK;
}

int psb_cross_helicity(psb_ctx* c, const void* u, const void* b, int flags, double* out) {
  PSB_TRY(check_ctx(c));
  if (!u || !b || !out) return fail(c, PSB_ERR_ARG, "psb_cross_helicity: null argument");
  PSB_TRY(set_device(c));
  double s = 0;
  const int filt = (flags & PSB_FILTER_GF) ? 1 : 0;
  PSB_TRY(c->prec == 64 ? reduce_impl<double>(c, u, b, kCross, filt, &s)
                        : reduce_impl<float>(c, u, b, kCross, filt, &s));
  const double nnn = (double)c->N1 * c->N2 * c->N3;
  *out = (flags & PSB_NORM_MPI) ? s / (nnn * nnn) : s / nnn;
  return PSB_OK;
}

int psb_spectrum_nbins(const psb_ctx* c, int flags, int* nbins) {
  if (!c || !nbins) return PSB_ERR_ARG;
  if (flags & PSB_TRANSFER_2D) {
    // kmax = round(max rint(sqrt(k1^2 + k2^2))) over the k3 = 0 plane (src/Classes.py:1080-1082)
    const double k1 = ((double)(c->N1 / 2) * 2.0) * M_PI / c->L1, k2 = ((double)(c->N2 / 2) * 2.0) * M_PI / c->L2;
    *nbins = (int)std::rint(std::sqrt(k1 * k1 + k2 * k2)) + 1;
    return PSB_OK;
  }
  // kmax = round(max over k3 in [1, N3/2) of rint(|k|)) (PySpectral/src/Classes.py:764-768)
  const double n1 = c->N1 / 2, n2 = c->N2 / 2, n3 = c->N3 / 2 - 1;
  *nbins = (int)std::rint(std::sqrt(n1 * n1 + n2 * n2 + n3 * n3)) + 1;
  return PSB_OK;
}

int psb_spectrum(psb_ctx* c, const void* f, int flags, double* out, int nbins) {
  PSB_TRY(check_ctx(c));
  if (!f || !out || nbins <= 0) return fail(c, PSB_ERR_ARG, "psb_spectrum: bad argument");
  PSB_TRY(set_device(c));
  PSB_TRY(ensure_red(c, (size_t)3 * nbins));
  PSB_TRY(cuda_ok(c, cudaMemsetAsync(c->red_dev, 0, sizeof(double) * 3 * nbins, c->stream), "memset"));
  const int filt = (flags & PSB_FILTER_GF) ? 1 : 0;
  if (c->prec == 64)
    spectrum_kernel<double><<<kRedBlocks, 256, 0, c->stream>>>(reinterpret_cast<const Cx<double>*>(f), filt, c->gx,
                                                                 c->gy, c->gz, c->N1, c->N2, c->N3, nbins,
                                                                 c->red_dev);
  else
    spectrum_kernel<float><<<kRedBlocks, 256, 0, c->stream>>>(reinterpret_cast<const Cx<float>*>(f), filt, c->gx,
                                                                c->gy, c->gz, c->N1, c->N2, c->N3, nbins, c->red_dev);
  PSB_TRY(launch_ok(c, "spectrum"));
  PSB_TRY(cuda_ok(c, cudaMemcpyAsync(c->red_host, c->red_dev, sizeof(double) * 3 * nbins, cudaMemcpyDeviceToHost,
                                     c->stream),
                  "spectrum copy"));
  PSB_TRY(cuda_ok(c, cudaStreamSynchronize(c->stream), "spectrum sync"));
  const double nnn = (double)c->N1 * c->N2 * c->N3;
  for (int i = 0; i < 3 * nbins; ++i) out[i] = c->red_host[i] / nnn;
  return PSB_OK;
}

int psb_transfer(psb_ctx* c, const void* f, const void* w0, int flags, double* out, int nbins) {
  PSB_TRY(check_ctx(c));
  if (!f || !out || nbins <= 0) return fail(c, PSB_ERR_ARG, "psb_transfer: bad argument");
  PSB_TRY(set_device(c));
  const int mode = w0 ? 2 : ((flags & PSB_FILTER_GF) ? 1 : 0);
  const void* Pp = w0;
  if (mode < 2) {
    const size_t esz = c->prec == 64 ? 16 : 8;
    const size_t nP = (size_t)6 * c->N1 * c->N2 * c->N3h;
    auto& buf = c->scratch["transfer.P"];
    if (buf.bytes < nP * esz) {
      if (buf.p) cudaFree(buf.p);
      buf.p = nullptr;
      buf.bytes = 0;
      PSB_TRY(cuda_ok(c, cudaMalloc(&buf.p, nP * esz), "transfer scratch"));
      buf.bytes = nP * esz;
    }
    if (mode == 0)
      PSB_TRY(c->prec == 64 ? products_run<double>(c, f, buf.p) : products_run<float>(c, f, buf.p));
    else
      PSB_TRY(c->prec == 64 ? products_filtered_run<double>(c, f, buf.p)
                            : products_filtered_run<float>(c, f, buf.p));
    Pp = buf.p;
  }
  PSB_TRY(ensure_red(c, (size_t)2 * nbins));
  PSB_TRY(cuda_ok(c, cudaMemsetAsync(c->red_dev, 0, sizeof(double) * 2 * nbins, c->stream), "memset"));
  ++c->launches;
  if (c->prec == 64)
    transfer_kernel<double><<<kRedBlocks, 256, 0, c->stream>>>(
        reinterpret_cast<const Cx<double>*>(f), reinterpret_cast<const Cx<double>*>(Pp), mode,
        (flags & PSB_TRANSFER_2D) ? 1 : 0, c->gx, c->gy, c->gz,
        c->kx, c->ky, c->kz, c->N1, c->N2, c->N3, nbins, c->red_dev);
  else
    transfer_kernel<float><<<kRedBlocks, 256, 0, c->stream>>>(
        reinterpret_cast<const Cx<float>*>(f), reinterpret_cast<const Cx<float>*>(Pp), mode,
        (flags & PSB_TRANSFER_2D) ? 1 : 0, c->gx, c->gy, c->gz,
        c->kx, c->ky, c->kz, c->N1, c->N2, c->N3, nbins, c->red_dev);
  PSB_TRY(launch_ok(c, "transfer"));
  PSB_TRY(cuda_ok(c, cudaMemcpyAsync(c->red_host, c->red_dev, sizeof(double) * 2 * nbins, cudaMemcpyDeviceToHost,
                                     c->stream),
                  "transfer copy"));
  PSB_TRY(cuda_ok(c, cudaStreamSynchronize(c->stream), "transfer sync"));
  const double nnn = (double)c->N1 * c->N2 * c->N3;
  for (int i = 0; i < 2 * nbins; ++i) out[i] = c->red_host[i] / nnn;
  return PSB_OK;
}

int psb_spectrum_mpi(psb_ctx* c, const void* f, double* out, int nbins) {
  PSB_TRY(check_ctx(c));
  if (!f || !out || nbins <= 0) return fail(c, PSB_ERR_ARG, "psb_spectrum_mpi: bad argument");
  PSB_TRY(set_device(c));
  PSB_TRY(ensure_red(c, (size_t)nbins));
  PSB_TRY(cuda_ok(c, cudaMemsetAsync(c->red_dev, 0, sizeof(double) * nbins, c->stream), "memset"));
  if (c->prec == 64)
    spectrum_mpi_kernel<double><<<kRedBlocks, 256, 0, c->stream>>>(reinterpret_cast<const Cx<double>*>(f), c->N1,
                                                                     c->N2, c->N3, nbins, c->red_dev);
  else
    spectrum_mpi_kernel<float><<<kRedBlocks, 256, 0, c->stream>>>(reinterpret_cast<const Cx<float>*>(f), c->N1,
                                                                    c->N2, c->N3, nbins, c->red_dev);
  PSB_TRY(launch_ok(c, "spectrum_mpi"));
  PSB_TRY(cuda_ok(c, cudaMemcpyAsync(c->red_host, c->red_dev, sizeof(double) * nbins, cudaMemcpyDeviceToHost,
                                     c->stream),
                  "spectrum copy"));
  PSB_TRY(cuda_ok(c, cudaStreamSynchronize(c->stream), "spectrum sync"));
  const double nnn = (double)c->N1 * c->N2 * c->N3;
  for (int i = 0; i < nbins; ++i) out[i] = c->red_host[i] / (nnn * nnn);
  return PSB_OK;
}

int psb_cfl_dt(psb_ctx* c, const void* f, double cfl, double nu, double* dt_out) {
  PSB_TRY(check_ctx(c));
  if (!dt_out) return fail(c, PSB_ERR_ARG, "psb_cfl_dt: null argument");
  if (!(cfl > 0)) {
    *dt_out = -cfl;
    return PSB_OK;
  }
  if (!f) return fail(c, PSB_ERR_ARG, "psb_cfl_dt: null field");
  PSB_TRY(set_device(c));
  double vmax = 0;
  PSB_TRY(c->prec == 64 ? cfl_impl<double>(c, f, &vmax) : cfl_impl<float>(c, f, &vmax));
  double dt = cfl / (vmax + 1e-10);
  if (nu > 0) {
    const double cap = 0.634 / (1. / (c->dx * c->dx) + 1. / (c->dy * c->dy) + 1. / (c->dz * c->dz)) / nu * cfl / 1.35;
    dt = std::min(dt, cap);
  }
  *dt_out = dt;
  return PSB_OK;
}

int psb_sgs_dns(psb_ctx* c, const void* f, void* w0, void* tau6) {
  PSB_TRY(check_ctx(c));
  if (!f || !w0) return fail(c, PSB_ERR_ARG, "psb_sgs_dns: null argument");
  PSB_TRY(set_device(c));
  return c->prec == 64 ? sgs_dns_run<double>(c, f, w0, tau6) : sgs_dns_run<float>(c, f, w0, tau6);
}

int psb_fft_r2c(psb_ctx* c, const void* phys, void* spec, int nfields) {
  PSB_TRY(check_ctx(c));
  if (!phys || !spec || nfields <= 0) return fail(c, PSB_ERR_ARG, "psb_fft_r2c: bad argument");
  PSB_TRY(set_device(c));
  return c->prec == 64 ? r2c_impl<double>(c, phys, spec, nfields) : r2c_impl<float>(c, phys, spec, nfields);
}

int psb_fft_c2r(psb_ctx* c, const void* spec, void* phys, int nfields) {
  PSB_TRY(check_ctx(c));
  if (!phys || !spec || nfields <= 0) return fail(c, PSB_ERR_ARG, "psb_fft_c2r: bad argument");
  PSB_TRY(set_device(c));
  return c->prec == 64 ? c2r_impl<double>(c, spec, phys, nfields) : c2r_impl<float>(c, spec, phys, nfields);
}

int psb_slab_ifft_y(psb_ctx* c, int nprocs, const void* uhat, void* send) {
  PSB_TRY(check_ctx(c));
  if (!uhat || !send) return fail(c, PSB_ERR_ARG, "psb_slab_ifft_y: null argument");
  PSB_TRY(slab_check(c, nprocs, "psb_slab_ifft_y"));
  PSB_TRY(set_device(c));
  return c->prec == 64 ? slab_y_impl<double>(c, nprocs, uhat, send, true)
                        : slab_y_impl<float>(c, nprocs, uhat, send, true);
}

int psb_slab_ifft_xz(psb_ctx* c, int nprocs, const void* recv, void* u) {
  PSB_TRY(check_ctx(c));
  if (!recv || !u) return fail(c, PSB_ERR_ARG, "psb_slab_ifft_xz: null argument");
  PSB_TRY(slab_check(c, nprocs, "psb_slab_ifft_xz"));
  PSB_TRY(set_device(c));
  return c->prec == 64 ? slab_xz_inverse<double>(c, nprocs, recv, u) : slab_xz_inverse<float>(c, nprocs, recv, u);
}

int psb_slab_fft_xz(psb_ctx* c, int nprocs, const void* u, void* send) {
  PSB_TRY(check_ctx(c));
  if (!u || !send) return fail(c, PSB_ERR_ARG, "psb_slab_fft_xz: null argument");
  PSB_TRY(slab_check(c, nprocs, "psb_slab_fft_xz"));
  PSB_TRY(set_device(c));
  return c->prec == 64 ? slab_xz_forward<double>(c, nprocs, u, send) : slab_xz_forward<float>(c, nprocs, u, send);
}

int psb_slab_fft_y(psb_ctx* c, int nprocs, const void* recv, void* uhat) {
  PSB_TRY(check_ctx(c));
  if (!recv || !uhat) return fail(c, PSB_ERR_ARG, "psb_slab_fft_y: null argument");
  PSB_TRY(slab_check(c, nprocs, "psb_slab_fft_y"));
  PSB_TRY(set_device(c));
  return c->prec == 64 ? slab_y_impl<double>(c, nprocs, recv, uhat, false)
                        : slab_y_impl<float>(c, nprocs, recv, uhat, false);
}

int psb_check_finite(psb_ctx* c, const void* data, long long n, long long* count) {
  PSB_TRY(check_ctx(c));
  if (!data || !count || n < 0) return fail(c, PSB_ERR_ARG, "psb_check_finite: bad argument");
  PSB_TRY(set_device(c));
  int st = PSB_OK;
  unsigned long long* d = reinterpret_cast<unsigned long long*>(scratch<double>(c, "finite.cnt", 1, &st));
  if (st != PSB_OK) return st;
  PSB_TRY(cuda_ok(c, cudaMemsetAsync(d, 0, sizeof(unsigned long long), c->stream), "memset"));
  if (c->prec == 64)
    finite_count_kernel<double><<<kRedBlocks, 256, 0, c->stream>>>(reinterpret_cast<const double*>(data), 2 * n, d);
  else
    finite_count_kernel<float><<<kRedBlocks, 256, 0, c->stream>>>(reinterpret_cast<const float*>(data), 2 * n, d);
  PSB_TRY(launch_ok(c, "finite"));
  unsigned long long h = 0;
  PSB_TRY(cuda_ok(c, cudaMemcpyAsync(&h, d, sizeof(h), cudaMemcpyDeviceToHost, c->stream), "finite copy"));
  PSB_TRY(cuda_ok(c, cudaStreamSynchronize(c->stream), "finite sync"));
  *count = (long long)h;
  return h ? fail(c, PSB_ERR_NONFINITE, "non-finite values found") : PSB_OK;
}

int psb_physical_fields(psb_ctx* c, const void* f, int what, void* out) {
  PSB_TRY(check_ctx(c));
  if (!f || !out || (what != 0 && what != 1)) return fail(c, PSB_ERR_ARG, "psb_physical_fields: bad argument");
  PSB_TRY(set_device(c));
  if (c->prec == 64)
    return what ? physical_impl<double>(c, f, out, PreGrad<double>{})
                : physical_impl<double>(c, f, out, PreCopyN<double, 3>{});
  return what ? physical_impl<float>(c, f, out, PreGrad<float>{}) : physical_impl<float>(c, f, out, PreCopyN<float, 3>{});
}

int psb_products(psb_ctx* c, const void* f, void* out6) {
  PSB_TRY(check_ctx(c));
  if (!f || !out6) return fail(c, PSB_ERR_ARG, "psb_products: null argument");
  PSB_TRY(set_device(c));
  return c->prec == 64 ? products_run<double>(c, f, out6) : products_run<float>(c, f, out6);
}

int psb_spectral_resample(const void* src, int N1, int N2, int N3, void* dst, int n1, int n2, int n3, int nfields,
                          int kc, double scale, int precision, void* stream) {
  if (!src || !dst || nfields <= 0 || N1 < 2 || N2 < 2 || N3 < 2 || n1 < 2 || n2 < 2 || n3 < 2 || kc < 1)
    return PSB_ERR_ARG;
  if (precision != 32 && precision != 64) return PSB_ERR_ARG;
  const long long n = (long long)n1 * n2 * (n3 / 2 + 1) * nfields;
  const int blocks = (int)std::min<long long>((n + 255) / 256, 4096);
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (precision == 64)
    resample_kernel<double><<<blocks, 256, 0, s>>>(reinterpret_cast<const Cx<double>*>(src), N1, N2, N3,
                                                   reinterpret_cast<Cx<double>*>(dst), n1, n2, n3, nfields, kc, scale);
  else
    resample_kernel<float><<<blocks, 256, 0, s>>>(reinterpret_cast<const Cx<float>*>(src), N1, N2, N3,
                                                  reinterpret_cast<Cx<float>*>(dst), n1, n2, n3, nfields, kc,
                                                  (float)scale);
  return cudaGetLastError() == cudaSuccess ? PSB_OK : PSB_ERR_CUDA;
}

int psb_launch_count(const psb_ctx* c, unsigned long long* n) {
  if (!c || !n) return PSB_ERR_ARG;
  *n = c->launches;
  return PSB_OK;
}

int psb_timing_enable(psb_ctx* c, int on) {
  PSB_TRY(check_ctx(c));
  for (auto& r : c->recs) {
    c->ev_free.push_back(r.a);
    c->ev_free.push_back(r.b);
  }
  c->recs.clear();
  c->timing = on ? 1 : 0;
  return PSB_OK;
}

int psb_timing_count(psb_ctx* c, int* n) {
  PSB_TRY(check_ctx(c));
  if (!n) return fail(c, PSB_ERR_ARG, "psb_timing_count: null argument");
  PSB_TRY(set_device(c));
  PSB_TRY(cuda_ok(c, cudaStreamSynchronize(c->stream), "timing sync"));
  *n = (int)c->recs.size();
  return PSB_OK;
}

int psb_timing_get(psb_ctx* c, int i, char* name, int name_len, double* ms, double* bytes) {
  PSB_TRY(check_ctx(c));
  if (i < 0 || i >= (int)c->recs.size() || !ms || !bytes) return fail(c, PSB_ERR_ARG, "psb_timing_get: bad index");
  const auto& r = c->recs[i];
  float t = 0.f;
  PSB_TRY(cuda_ok(c, cudaEventElapsedTime(&t, r.a, r.b), "event elapsed"));
  *ms = t;
  *bytes = r.bytes;
  if (name && name_len > 0) {
    std::strncpy(name, r.name.c_str(), name_len - 1);
    name[name_len - 1] = 0;
  }
  return PSB_OK;
}

}  // extern "C"
