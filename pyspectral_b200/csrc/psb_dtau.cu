// Dynamic tau-model (PySpectral/src/RHSfunctions.py:592-878).
//
// Runs the PL / PLQL pipelines twice -- on u and on the test-filtered u --
// keeps the Leonard pieces on the compact test-filter box, reduces the three
// complex energy balances LE, PLQLE_filt, filt_PLQLE in FP64 on the device,
// forms tau = |LE| / (|PLQLE_filt| - |filt_PLQLE| + 1e-5) on the device and
// finishes RHS = unpad_2x(PL) + max(0,tau) PLQL (+ Coriolis) with the RK stage
// update.  No host round trip inside the RHS.
#include "psb_ctx.cuh"

using namespace psb;
using namespace psbh;

namespace psbh {
template <typename T>
int mem_stage_pl(psb_ctx* c, const Cx<T>* Qin, const psb_params* p, const char* tag, const double* filt, int kfp,
                 Cx<T>* PLp, Cx<T>* Lbox, int kfb, Cx<T>** B2, Cx<T>** E);
template <typename T>
int mem_stage_plql(psb_ctx* c, Cx<T>* B2, Cx<T>* E, EpiPLQL<T> epi);
}  // namespace psbh

namespace {

__device__ __forceinline__ int box_to_idx(int b, int kf, int M) { return b < kf ? b : M - (2 * kf - 1) + b; }

// sums[0..5] = (LE, PLQLE_filt, filt_PLQLE) as (re, im) pairs, then tau[0]=raw, tau[1]=clamped
template <typename T>
__global__ void __launch_bounds__(256) dtau_sums_kernel(const Cx<T>* __restrict__ Q, const Cx<T>* __restrict__ Lu,
                                                        const Cx<T>* __restrict__ Lf,
                                                        const Cx<T>* __restrict__ PLQL,
                                                        const Cx<T>* __restrict__ PLQLf, int N1, int N2, int N3,
                                                        int n3h, int kf, double* __restrict__ out) {
  const int nb = 2 * kf - 1;
  const long long npts = (long long)nb * nb * kf;
  const long long fsN = (long long)N1 * N2 * n3h;
  const long long fsB = npts;
  double acc[6] = {0, 0, 0, 0, 0, 0};
  for (long long idx = threadIdx.x; idx < npts; idx += blockDim.x) {
    const int i3 = (int)(idx % kf);
    const long long t = idx / kf;
    const int b2 = (int)(t % nb), b1 = (int)(t / nb);
    const int n1 = box_to_idx(b1, kf, N1), n2 = box_to_idx(b2, kf, N2);
    const double w = i3 == 0 ? 1.0 : (i3 < N3 / 2 ? 2.0 : 0.0);
    const long long s = ((long long)n1 * N2 + n2) * n3h + i3;
#pragma unroll
    for (int f = 0; f < 3; ++f) {
      const Cx<T> u = Q[f * fsN + s];
      const Cx<T> L = Lu[f * fsB + idx] - Lf[f * fsB + idx];
      const Cx<T> a = PLQLf[f * fsN + s];
      const Cx<T> b = PLQL[f * fsN + s];
      // x * conj(u)
      acc[0] += w * ((double)L.x * u.x + (double)L.y * u.y);
      acc[1] += w * ((double)L.y * u.x - (double)L.x * u.y);
      acc[2] += w * ((double)a.x * u.x + (double)a.y * u.y);
      acc[3] += w * ((double)a.y * u.x - (double)a.x * u.y);
      acc[4] += w * ((double)b.x * u.x + (double)b.y * u.y);
      acc[5] += w * ((double)b.y * u.x - (double)b.x * u.y);
    }
  }
  __shared__ double red[6][256];
#pragma unroll
  for (int m = 0; m < 6; ++m) red[m][threadIdx.x] = acc[m];
  __syncthreads();
  for (int h = blockDim.x / 2; h > 0; h >>= 1) {
    if ((int)threadIdx.x < h)
#pragma unroll
      for (int m = 0; m < 6; ++m) red[m][threadIdx.x] += red[m][threadIdx.x + h];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const double nnn = (double)N1 * N2 * N3;
    double s[6];
    for (int m = 0; m < 6; ++m) {
      s[m] = red[m][0] / nnn;
      out[m] = s[m];
    }
    const double le = hypot(s[0], s[1]), pf = hypot(s[2], s[3]), fp = hypot(s[4], s[5]);
    const double tau = le / (pf - fp + 1.0e-5);
    out[6] = tau;
    out[7] = tau > 0.0 ? tau : 0.0;
  }
}

template <typename T>
__global__ void __launch_bounds__(256) dtau_combine_kernel(StepIO<T> io, const Cx<T>* __restrict__ PLp,
                                                           const Cx<T>* __restrict__ PLQL,
                                                           const double* __restrict__ taus, int N1, int N2,
                                                           int N3, int rotate, T Om1, T Om2, T Om3) {
  const long long npts = (long long)N1 * N2 * io.n3h;
  const T tc = (T)taus[7];
  for (long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x; s < npts;
       s += (long long)gridDim.x * blockDim.x) {
    const int i3 = (int)(s % io.n3h);
    const long long t = s / io.n3h;
    const int i2 = (int)(t % N2), i1 = (int)(t / N2);
    Cx<T> u = io.Q[s], v = io.Q[io.fstride + s], w = io.Q[2 * io.fstride + s];
    if (i1 == N1 / 2 || i2 == N2 / 2 || i3 == N3 / 2) u = v = w = mk<T>(0, 0);
    const Cx<T> w0u = tc * PLQL[s], w0v = tc * PLQL[io.fstride + s], w0w = tc * PLQL[2 * io.fstride + s];
    Cx<T> ru = PLp[s] + w0u, rv = PLp[io.fstride + s] + w0v, rw = PLp[2 * io.fstride + s] + w0w;
    if (rotate) {
      ru = ru + (T)2 * (Om3 * v - Om2 * w);
      rv = rv + (T)2 * (Om1 * w - Om3 * u);
      rw = rw + (T)2 * (Om2 * u - Om1 * v);
    }
    if (io.w0_out) {
      io.w0_out[s] = w0u;
      io.w0_out[io.fstride + s] = w0v;
      io.w0_out[2 * io.fstride + s] = w0w;
    }
    if (io.read_out) {
      io.read_out[s] = u;
      io.read_out[io.fstride + s] = v;
      io.read_out[2 * io.fstride + s] = w;
    }
    io.finish(s, 0, ru);
    io.finish(s, 1, rv);
    io.finish(s, 2, rw);
  }
}

template <typename T>
int dtau_rhs(psb_ctx* c, StepIO<T> io, const psb_params* p, double* tau_out) {
  const int N1 = c->N1, N2 = c->N2, N3 = c->N3, N3h = c->N3h;
  const int kf = p->kf > 0 ? p->kf : (int)(c->kc * 2.0 / 3.0);
  const double two_pi = 2.0 * M_PI;
  if (c->L1 != two_pi || c->L2 != two_pi || c->L3 != two_pi)
    return fail(c, PSB_ERR_UNSUPPORTED, "dynamic tau-model requires L1=L2=L3=2*pi");
  if (kf < 2 || 2 * kf > N1 || 2 * kf > N2 || 2 * kf > N3)
    return fail(c, PSB_ERR_ARG, "dynamic tau-model: test filter kf out of range");
  int st = PSB_OK;
  const size_t nN = (size_t)3 * N1 * N2 * N3h;
  const size_t nb = (size_t)(2 * kf - 1) * (2 * kf - 1) * kf;
  Cx<T>* PLp = scratch<T>(c, "mem.PLp", nN, &st);
  Cx<T>* PLQL = scratch<T>(c, "dtau.PLQL", nN, &st);
  Cx<T>* PLQLf = scratch<T>(c, "dtau.PLQLf", nN, &st);
  Cx<T>* Lu = scratch<T>(c, "dtau.Lu", 3 * nb, &st);
  Cx<T>* Lf = scratch<T>(c, "dtau.Lf", 3 * nb, &st);
  // test filter masks (N grid): |k| < kf per axis (PySpectral/src/Classes.py:131-146)
  double* filt = reinterpret_cast<double*>(scratch<double>(c, "dtau.filt", (size_t)(N1 + N2 + N3h), &st));
  double* sums = reinterpret_cast<double*>(scratch<double>(c, "dtau.sums", 4, &st));
  if (st != PSB_OK) return st;
  if (c->dtau_kf != kf) {
    std::vector<double> h(N1 + N2 + N3h);
    std::vector<double> k1(N1), k2(N2), k3(N3h);
    cudaMemcpy(k1.data(), c->kx, N1 * sizeof(double), cudaMemcpyDeviceToHost);
    cudaMemcpy(k2.data(), c->ky, N2 * sizeof(double), cudaMemcpyDeviceToHost);
    cudaMemcpy(k3.data(), c->kz, N3h * sizeof(double), cudaMemcpyDeviceToHost);
    for (int i = 0; i < N1; ++i) h[i] = std::fabs(k1[i]) >= kf ? 0.0 : 1.0;
    for (int i = 0; i < N2; ++i) h[N1 + i] = std::fabs(k2[i]) >= kf ? 0.0 : 1.0;
    for (int i = 0; i < N3h; ++i) h[N1 + N2 + i] = std::fabs(k3[i]) >= kf ? 0.0 : 1.0;
    PSB_TRY(cuda_ok(c, cudaMemcpy(filt, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice), "filter upload"));
    c->dtau_kf = kf;
  }
  Cx<T>*B2u = nullptr, *Eu = nullptr, *B2f = nullptr, *Ef = nullptr;
  const Cx<T>* Qin = io.Q;
  if (!Qin) {  // allocation only
    PSB_TRY(mem_stage_pl<T>(c, nullptr, p, "memu", nullptr, 0, PLp, Lu, kf, &B2u, &Eu));
    PSB_TRY(mem_stage_pl<T>(c, nullptr, p, "memf", filt, kf, nullptr, Lf, kf, &B2f, &Ef));
    EpiPLQL<T> e{};
    return mem_stage_plql<T>(c, nullptr, nullptr, e);
  }
  PSB_TRY(cuda_ok(c, cudaMemsetAsync(PLp, 0, nN * sizeof(Cx<T>), c->stream), "memset"));
  PSB_TRY(mem_stage_pl<T>(c, Qin, p, "memu", nullptr, 0, PLp, Lu, kf, &B2u, &Eu));
  EpiPLQL<T> e{};
  e.io = io;
  e.k.k1 = c->kx;
  e.k.k2 = c->ky;
  e.k.k3 = c->kz;
  e.PLp = PLp;
  e.coef = (T)0;
  e.ny1 = N1 / 2;
  e.ny2 = N2 / 2;
  e.ny3 = N3 / 2;
  e.plql_out = PLQL;
  PSB_TRY(mem_stage_plql<T>(c, B2u, Eu, e));
  PSB_TRY(mem_stage_pl<T>(c, Qin, p, "memf", filt, kf, nullptr, Lf, kf, &B2f, &Ef));
  e.plql_out = PLQLf;
  PSB_TRY(mem_stage_plql<T>(c, B2f, Ef, e));
  dtau_sums_kernel<T><<<1, 256, 0, c->stream>>>(Qin, Lu, Lf, PLQL, PLQLf, N1, N2, N3, N3h, kf, sums);
  PSB_TRY(launch_ok(c, "dtau sums"));
  const long long npts = (long long)N1 * N2 * N3h;
  const int blocks = (int)std::min<long long>((npts + 255) / 256, 4096);
  dtau_combine_kernel<T><<<blocks, 256, 0, c->stream>>>(io, PLp, PLQL, sums, N1, N2, N3, p->rotate, (T)p->Om1,
                                                         (T)p->Om2, (T)p->Om3);
  PSB_TRY(launch_ok(c, "dtau combine"));
  if (tau_out) {
    double h[8];
    PSB_TRY(cuda_ok(c, cudaMemcpyAsync(h, sums, sizeof(h), cudaMemcpyDeviceToHost, c->stream), "tau copy"));
    PSB_TRY(cuda_ok(c, cudaStreamSynchronize(c->stream), "tau sync"));
    *tau_out = h[6];
  }
  return PSB_OK;
}

}  // namespace

namespace psbh {
int dtau_rhs_d(psb_ctx* c, StepIO<double> io, const psb_params* p, double* tau_out) {
  return dtau_rhs<double>(c, io, p, tau_out);
}
int dtau_rhs_f(psb_ctx* c, StepIO<float> io, const psb_params* p, double* tau_out) {
  return dtau_rhs<float>(c, io, p, tau_out);
}
}  // namespace psbh
