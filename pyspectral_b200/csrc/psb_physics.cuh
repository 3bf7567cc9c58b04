// Pointwise physics of the right-hand sides: spectral expanders run on load by
// the x-inverse pass, physical-space products run inside the z-pass, spectral
// epilogues (projection, viscosity, closure, Coriolis, RK stage) run after the
// last forward pass.  Every formula cites the reference line it restates.
#pragma once
#include "psb_passes.cuh"

namespace psb {

// ---- precision helpers ---------------------------------------------------
// FP64 keeps the reference's ksqr = k.k + 1e-50 and ksqr_i = 1/ksqr
// (PySpectral/src/Classes.py:576-577).  In FP32 1e-50 flushes to zero, so the
// k=0 mode uses ksqr_i = 0; every term it multiplies vanishes there anyway.
template <typename T>
__device__ __forceinline__ void ksq_pair(T k1, T k2, T k3, T& ksq, T& ksqi) {
  if constexpr (sizeof(T) == 8) {
    ksq = k1 * k1 + k2 * k2 + k3 * k3 + 1.0e-50;
    ksqi = 1.0 / ksq;
  } else {
    ksq = k1 * k1 + k2 * k2 + k3 * k3;
    ksqi = ksq > (T)0 ? (T)1 / ksq : (T)0;
  }
}

// -i*k*X and i*k*X
template <typename T>
__device__ __forceinline__ Cx<T> mik(T k, Cx<T> X) { return mk<T>(k * X.y, -k * X.x); }
template <typename T>
__device__ __forceinline__ Cx<T> pik(T k, Cx<T> X) { return mk<T>(-k * X.y, k * X.x); }

// ---- RK stage bookkeeping --------------------------------------------------
enum StageMode : int { kRHS = 0, kStage1 = 1, kStageMid = 2, kStageLast = 3 };

template <typename T>
struct StepIO {
  Cx<T>* Q;         // state (read; updated in RK modes)
  Cx<T>* Q0;        // step start state (written in stage 1)
  Cx<T>* comp;      // Kahan compensation (FP32 runs) or null
  Cx<T>* rhs_out;   // RHS output (kRHS) or null
  Cx<T>* read_out;  // state as read by this RHS (the reference's main.uhat) or null
  Cx<T>* w0_out;    // closure force (main.w0_*) or null
  long long fstride;
  int n2, n3h;
  int mode;
  T dtc;  // dt * rk4const[i]
  __device__ __forceinline__ long long sidx(int i1, int i2, int i3) const {
    return ((long long)i1 * n2 + i2) * n3h + i3;
  }
  // compulsory state traffic over npts points and nf fields
  __host__ double bytes(long long npts, int nf) const {
    double n = 1.0;  // read Q
    if (mode == kRHS) n += 1.0;
    else n += 2.0 + (comp ? (mode == kStageLast ? 2.0 : 1.0) : 0.0);
    if (read_out) n += 1.0;
    double b = n * (double)sizeof(Cx<T>) * npts * nf;
    if (w0_out) b += (double)sizeof(Cx<T>) * npts * 3;
    return b;
  }
  // Q = Q0 + dt*c*RHS  (PySpectral/src/PySpec_3d.py:104), Kahan-compensated when comp != null.
  __device__ __forceinline__ void finish(long long s, int f, Cx<T> R) const {
    const long long e = f * fstride + s;
    if (mode == kRHS) {
      rhs_out[e] = R;
      return;
    }
    Cx<T> base;
    if (mode == kStage1) {
      base = Q[e];
      Q0[e] = base;
    } else {
      base = Q0[e];
    }
    const Cx<T> inc = dtc * R;
    if (comp == nullptr) {
      Q[e] = base + inc;
    } else {
      const Cx<T> c = comp[e];
      const Cx<T> y = inc - c;
      const Cx<T> t = base + y;
      if (mode == kStageLast) comp[e] = (t - base) - y;
      Q[e] = t;
    }
  }
};

// ---- 3/2-padded Navier-Stokes: DNS and Smagorinsky --------------------------
template <typename T, int F>
struct PreCopyN {
  static constexpr int F_SRC = F, F_DST = F;
  static constexpr bool FIELDWISE = true;
  __device__ void operator()(int, int, int, const AxisArgs<T>&, const Cx<T>* s, Cx<T>* d) const {
#pragma unroll
    for (int f = 0; f < F; ++f) d[f] = s[f];
  }
  // field g of row i, column col, read from the row's inputs (in: the outer index's base)
  __device__ __forceinline__ Cx<T> field(int g, int i, int, int col, const AxisArgs<T>& a, const Cx<T>* in) const {
    return in[g * a.in_fstride + i * a.in_rstride + col];
  }
};

// (u,v,w) -> (u,v,w,S11,S22,S33,S12,S13,S23), S_ij = (i/2)(k_j u_i + k_i u_j)
// (PySpectral/src/RHSfunctions.py:174-179)
template <typename T>
struct PreStrain {
  static constexpr int F_SRC = 3, F_DST = 9;
  static constexpr bool FIELDWISE = true;
  __device__ __forceinline__ Cx<T> field(int g, int i, int o, int col, const AxisArgs<T>& a, const Cx<T>* in) const {
    auto src = [&](int f) { return in[f * a.in_fstride + i * a.in_rstride + col]; };
    const T k[3] = {(T)a.k_row[i], (T)a.k_outer[o], (T)a.k_col[col]};
    if (g < 3) return src(g);
    if (g < 6) return pik(k[g - 3], src(g - 3));
    const int p = g == 6 ? 0 : (g == 7 ? 0 : 1), q = g == 6 ? 1 : 2;  // S_pq
    return (T)0.5 * (pik(k[q], src(p)) + pik(k[p], src(q)));
  }
  __device__ void operator()(int i, int o, int c, const AxisArgs<T>& a, const Cx<T>* s, Cx<T>* d) const {
    const T k1 = (T)a.k_row[i], k2 = (T)a.k_outer[o], k3 = (T)a.k_col[c];
    d[0] = s[0];
    d[1] = s[1];
    d[2] = s[2];
    d[3] = pik(k1, s[0]);
    d[4] = pik(k2, s[1]);
    d[5] = pik(k3, s[2]);
    d[6] = (T)0.5 * (pik(k2, s[0]) + pik(k1, s[1]));
    d[7] = (T)0.5 * (pik(k3, s[0]) + pik(k1, s[2]));
    d[8] = (T)0.5 * (pik(k3, s[1]) + pik(k2, s[2]));
  }
};

// u_i u_j in physical space (PySpectral/src/RHSfunctions.py:18-23)
template <typename T>
struct PhysProducts {
  static constexpr int F_IN = 3, F_OUT = 6;
  __device__ __forceinline__ void operator()(long long, int, const T* in, T* out) const {
    const T u = in[0], v = in[1], w = in[2];
    out[0] = u * u;
    out[1] = v * v;
    out[2] = w * w;
    out[3] = u * v;
    out[4] = u * w;
    out[5] = v * w;
  }
};

// Products plus the Smagorinsky stress tau_ij = -2 (Cs Delta)^2 |S| S_ij
// (PySpectral/src/RHSfunctions.py:195-212, Cs = 0.16 at :197).
template <typename T>
struct PhysSmag {
  static constexpr int F_IN = 9, F_OUT = 12;
  T csd2;  // 0.16*Delta*0.16*Delta
  __device__ __forceinline__ void operator()(long long, int, const T* in, T* out) const {
    const T u = in[0], v = in[1], w = in[2];
    out[0] = u * u;
    out[1] = v * v;
    out[2] = w * w;
    out[3] = u * v;
    out[4] = u * w;
    out[5] = v * w;
    const T S11 = in[3], S22 = in[4], S33 = in[5], S12 = in[6], S13 = in[7], S23 = in[8];
    const T sm = sqrt((T)2 * (S11 * S11 + S22 * S22 + S33 * S33 + (T)2 * S12 * S12 + (T)2 * S13 * S13 +
                              (T)2 * S23 * S23));
    const T m2nut = (T)-2 * (csd2 * fabs(sm));
    out[6] = m2nut * S11;
    out[7] = m2nut * S22;
    out[8] = m2nut * S33;
    out[9] = m2nut * S12;
    out[10] = m2nut * S13;
    out[11] = m2nut * S23;
  }
};

template <typename T>
struct KTabs {
  const double *k1, *k2, *k3;
};

// DNS / Smagorinsky epilogue (PySpectral/src/RHSfunctions.py:29-50, :164-232)
template <typename T, bool SMAG>
struct EpiNS {
  static constexpr int F_IN = SMAG ? 12 : 6;
  __host__ double io_bytes(long long npts) const { return io.bytes(npts, 3); }
  StepIO<T> io;
  KTabs<T> k;
  T nu;
  int rotate;
  T Om1, Om2, Om3;
  int zero_nyq;  // unpad(pad(uhat)) on read (:10-12); absent in SMAG
  int ny1, ny2, ny3;
  __device__ void operator()(int i1, int i2, int i3, const Cx<T>* P) const {
    const long long s = io.sidx(i1, i2, i3);
    Cx<T> u = io.Q[s], v = io.Q[io.fstride + s], w = io.Q[2 * io.fstride + s];
    if (zero_nyq && (i1 == ny1 || i2 == ny2 || i3 == ny3)) u = v = w = mk<T>(0, 0);
    const T k1 = (T)k.k1[i1], k2 = (T)k.k2[i2], k3 = (T)k.k3[i3];
    T ksq, ksqi;
    ksq_pair(k1, k2, k3, ksq, ksqi);
    const Cx<T> uu = P[0], vv = P[1], ww = P[2], uv = P[3], uw = P[4], vw = P[5];
    Cx<T> ph = ksqi * ((-k1 * k1) * uu - (k2 * k2) * vv - (k3 * k3) * ww - ((T)2 * k1 * k2) * uv -
                       ((T)2 * k1 * k3) * uw - ((T)2 * k2 * k3) * vw);
    Cx<T> cu = mk<T>(0, 0), cv = cu, cw = cu;
    if (rotate) {
      cu = Om3 * v - Om2 * w;
      cv = Om1 * w - Om3 * u;
      cw = Om2 * u - Om1 * v;
      // phat -= 2 ksqr_i 1j (k . (u x Om)) (:33-36)
      const Cx<T> kd = k1 * cu + k2 * cv + k3 * cw;
      ph = ph - ((T)2 * ksqi) * mul_i(kd);
    }
    Cx<T> ru = mik(k1, uu) + mik(k2, uv) + mik(k3, uw) + mik(k1, ph) - (nu * ksq) * u;
    Cx<T> rv = mik(k1, uv) + mik(k2, vv) + mik(k3, vw) + mik(k2, ph) - (nu * ksq) * v;
    Cx<T> rw = mik(k1, uw) + mik(k2, vw) + mik(k3, ww) + mik(k3, ph) - (nu * ksq) * w;
    if constexpr (SMAG) {
      // projected SGS divergence (:215-222); note 1j*k_i*(1j*ksqr_i*(kk:tau))
      const Cx<T> t11 = P[6], t22 = P[7], t33 = P[8], t12 = P[9], t13 = P[10], t23 = P[11];
      const Cx<T> kk = (k1 * k1) * t11 + (k2 * k2) * t22 + (k3 * k3) * t33 + ((T)2 * k1 * k2) * t12 +
                       ((T)2 * k1 * k3) * t13 + ((T)2 * k2 * k3) * t23;
      const Cx<T> proj = mul_i(ksqi * kk);
      const Cx<T> w0u = mik(k1, t11) + mik(k2, t12) + mik(k3, t13) + pik(k1, proj);
      const Cx<T> w0v = mik(k1, t12) + mik(k2, t22) + mik(k3, t23) + pik(k2, proj);
      const Cx<T> w0w = mik(k1, t13) + mik(k2, t23) + mik(k3, t33) + pik(k3, proj);
      ru = ru + w0u;
      rv = rv + w0v;
      rw = rw + w0w;
      if (io.w0_out) {
        io.w0_out[s] = w0u;
        io.w0_out[io.fstride + s] = w0v;
        io.w0_out[2 * io.fstride + s] = w0w;
      }
    }
    if (rotate) {  // + 2 u x Om (:47-50)
      ru = ru + (T)2 * cu;
      rv = rv + (T)2 * cv;
      rw = rw + (T)2 * cw;
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
};

// ---- MHD (2/3 rule, unpadded), PySpectral/src_MPI/RHSfunctions.py:95-175 ------
template <typename T>
struct PreMask6 {
  static constexpr int F_SRC = 6, F_DST = 6;
  const double *m1, *m2, *m3;
  __device__ void operator()(int i, int o, int c, const AxisArgs<T>&, const Cx<T>* s, Cx<T>* d) const {
    const T m = (T)(m1[i] * m2[o] * m3[c]);
#pragma unroll
    for (int f = 0; f < 6; ++f) d[f] = m * s[f];
  }
};

// (u_i u_j - B_i B_j) and u x B (:117-134; the momentum and pressure terms are
// linear in NL - MHDNL, so the difference is transformed once).
template <typename T>
struct PhysMHD {
  static constexpr int F_IN = 6, F_OUT = 9;
  __device__ __forceinline__ void operator()(long long, int, const T* in, T* out) const {
    const T u = in[0], v = in[1], w = in[2], b1 = in[3], b2 = in[4], b3 = in[5];
    out[0] = u * u - b1 * b1;
    out[1] = v * v - b2 * b2;
    out[2] = w * w - b3 * b3;
    out[3] = u * v - b1 * b2;
    out[4] = u * w - b1 * b3;
    out[5] = v * w - b2 * b3;
    out[6] = v * b3 - w * b2;
    out[7] = w * b1 - u * b3;
    out[8] = u * b2 - v * b1;
  }
};

template <typename T>
struct EpiMHD {
  static constexpr int F_IN = 9;
  __host__ double io_bytes(long long npts) const {
    return io.bytes(npts, 6) + (force ? (double)sizeof(Cx<T>) * npts * 3 : 0.0);
  }
  StepIO<T> io;
  KTabs<T> k;
  const double *m1, *m2, *m3;
  const Cx<T>* force;  // 3 fields or null
  T nu, eta;
  __device__ void operator()(int i1, int i2, int i3, const Cx<T>* P) const {
    const long long s = io.sidx(i1, i2, i3);
    const T D = (T)(m1[i1] * m2[i2] * m3[i3]);
    Cx<T> st[6];
#pragma unroll
    for (int f = 0; f < 6; ++f) st[f] = D * io.Q[f * io.fstride + s];
    const T k1 = (T)k.k1[i1], k2 = (T)k.k2[i2], k3 = (T)k.k3[i3];
    T ksq, ksqi;
    ksq_pair(k1, k2, k3, ksq, ksqi);
    const Cx<T> n0 = P[0], n1 = P[1], n2 = P[2], n3 = P[3], n4 = P[4], n5 = P[5];
    const Cx<T> x0 = P[6], x1 = P[7], x2 = P[8];
    const Cx<T> ph = ksqi * ((-k1 * k1) * n0 - (k2 * k2) * n1 - (k3 * k3) * n2 - ((T)2 * k1 * k2) * n3 -
                             ((T)2 * k1 * k3) * n4 - ((T)2 * k2 * k3) * n5);
    Cx<T> f0 = mk<T>(0, 0), f1 = f0, f2 = f0;
    if (force) {
      f0 = force[s];
      f1 = force[io.fstride + s];
      f2 = force[2 * io.fstride + s];
    }
    Cx<T> r[6];
    r[0] = D * (mik(k1, n0) + mik(k2, n3) + mik(k3, n4) + mik(k1, ph) - (nu * ksq) * st[0] + f0);
    r[1] = D * (mik(k1, n3) + mik(k2, n1) + mik(k3, n5) + mik(k2, ph) - (nu * ksq) * st[1] + f1);
    r[2] = D * (mik(k1, n4) + mik(k2, n5) + mik(k3, n2) + mik(k3, ph) - (nu * ksq) * st[2] + f2);
    r[3] = D * ((pik(k2, x2) - pik(k3, x1)) - (eta * ksq) * st[3]);
    r[4] = D * ((pik(k3, x0) - pik(k1, x2)) - (eta * ksq) * st[4]);
    r[5] = D * ((pik(k1, x1) - pik(k2, x0)) - (eta * ksq) * st[5]);
    if (io.read_out) {
#pragma unroll
      for (int f = 0; f < 6; ++f) io.read_out[f * io.fstride + s] = st[f];
    }
#pragma unroll
    for (int f = 0; f < 6; ++f) io.finish(s, f, r[f]);
  }
};

// ---- 2x-padded memory closures: t-model, static/dynamic tau-model -----------
// (PySpectral/src/RHSfunctions.py:240-363, :366-497, :592-878)

// 2x-grid index -> N-grid index under unpad_2x (PySpectral/src/padding.py:28-38)
__device__ __forceinline__ int unpad2x_idx(int i, int N) {
  return i < N / 2 ? i : (i >= 2 * N - N / 2 ? i - N : -1);
}
// membership of the resolved set p of seperateModes (PySpectral/src/padding.py:67-79)
__device__ __forceinline__ bool in_p_axis(int i, int N) { return i < N / 2 || i > 2 * N - N / 2; }

// PL on the full 2x grid, split into the q part (inverse-transformed next) and
// unpad_2x(PL) (the resolved RHS).  Optional: the test-filtered Leonard term of
// the dynamic model is stored on the compact G2 box.
template <typename T>
struct EpiPL {
  static constexpr int F_IN = 6;
  // npts = 2x-grid points: q part written everywhere, resolved state read / PL_p written on the N grid
  __host__ double io_bytes(long long npts) const {
    const double e = (double)sizeof(Cx<T>);
    return e * 3 * npts * (PLfull ? 2.0 : 1.0) + e * 3 * fstride_n * (PLp ? 2.0 : 1.0);
  }
  const Cx<T>* Q;  // N-grid state (3 fields)
  long long fstride_n;
  int N1, N2, N3, n3h;
  int nf2, nf3h;  // 2x-grid sizes: rows_y = 2*N2, k3 count N3+1
  long long fstride_2x;
  KTabs<T> kf;  // 2x-grid wavenumbers
  T nu;
  int rotate;
  T Om1, Om2, Om3;
  const double* filt;  // N-grid test filter per axis (nullptr = no filter): [N1 | N2 | n3h]
  int kfp;             // test-filter split size for the q part (0 = seperateModes)
  Cx<T>* PLq;          // (3, 2N1, 2N2, N3+1)
  Cx<T>* PLp;          // (3, N1, N2, n3h) unpad_2x(PL), may be null
  Cx<T>* Lbox;         // (3, 2kfb-1, 2kfb-1, kfb) Leonard pieces, or null
  int kfb;             // box half-size (test-filter kf)
  Cx<T>* PLfull;       // (3, 2N1, 2N2, N3+1) PL on the whole 2x grid, or null
  __device__ void operator()(int i1, int i2, int i3, const Cx<T>* P) const {
    const int n1 = unpad2x_idx(i1, N1), n2 = unpad2x_idx(i2, N2);
    const int n3 = i3 < N3 / 2 ? i3 : -1;
    Cx<T> u = mk<T>(0, 0), v = u, w = u;
    // pad_2x(unpad(pad(uhat))) [optionally test-filtered first]
    if (n1 >= 0 && n2 >= 0 && n3 >= 0 && n1 != N1 / 2 && n2 != N2 / 2) {
      const long long s = ((long long)n1 * N2 + n2) * n3h + n3;
      T g = (T)1;
      if (filt) g = (T)(filt[n1] * filt[N1 + n2] * filt[N1 + N2 + n3]);
      u = g * Q[s];
      v = g * Q[fstride_n + s];
      w = g * Q[2 * fstride_n + s];
    }
    const T k1 = (T)kf.k1[i1], k2 = (T)kf.k2[i2], k3 = (T)kf.k3[i3];
    T ksq, ksqi;
    ksq_pair(k1, k2, k3, ksq, ksqi);
    const Cx<T> uu = P[0], vv = P[1], ww = P[2], uv = P[3], uw = P[4], vw = P[5];
    Cx<T> ph = ksqi * ((-k1 * k1) * uu - (k2 * k2) * vv - (k3 * k3) * ww - ((T)2 * k1 * k2) * uv -
                       ((T)2 * k1 * k3) * uw - ((T)2 * k2 * k3) * vw);
    if (rotate) {
      const Cx<T> cu = Om3 * v - Om2 * w, cv = Om1 * w - Om3 * u, cw = Om2 * u - Om1 * v;
      ph = ph - ((T)2 * ksqi) * mul_i(k1 * cu + k2 * cv + k3 * cw);
    }
    const Cx<T> au = mik(k1, uu) + mik(k2, uv) + mik(k3, uw);
    const Cx<T> av = mik(k1, uv) + mik(k2, vv) + mik(k3, vw);
    const Cx<T> aw = mik(k1, uw) + mik(k2, vw) + mik(k3, ww);
    const Cx<T> pu = au + mik(k1, ph) - (nu * ksq) * u;
    const Cx<T> pv = av + mik(k2, ph) - (nu * ksq) * v;
    const Cx<T> pw = aw + mik(k3, ph) - (nu * ksq) * w;
    bool inp;
    if (kfp > 0) {  // seperateModes_testFilter (PySpectral/src/padding.py:52-64)
      const int M1 = 2 * N1, M2 = 2 * N2;
      inp = (i1 < kfp || i1 >= M1 - kfp + 1) && (i2 < kfp || i2 >= M2 - kfp + 1) && i3 < kfp;
    } else {
      inp = in_p_axis(i1, N1) && in_p_axis(i2, N2) && i3 < N3 / 2;
    }
    const long long s2 = ((long long)i1 * nf2 + i2) * nf3h + i3;
    const Cx<T> z = mk<T>(0, 0);
    PLq[s2] = inp ? z : pu;
    PLq[fstride_2x + s2] = inp ? z : pv;
    PLq[2 * fstride_2x + s2] = inp ? z : pw;
    if (PLfull) {
      PLfull[s2] = pu;
      PLfull[fstride_2x + s2] = pv;
      PLfull[2 * fstride_2x + s2] = pw;
    }
    if (PLp && n1 >= 0 && n2 >= 0 && n3 >= 0) {
      const long long s = ((long long)n1 * N2 + n2) * n3h + n3;
      PLp[s] = pu;
      PLp[fstride_n + s] = pv;
      PLp[2 * fstride_n + s] = pw;
    }
    if (Lbox) {
      // test_filter_2x(-1j k_j (u_i u_j)^ + 1j k_i phat) (PySpectral/src/RHSfunctions.py:813-819)
      const int M1 = 2 * N1, M2 = 2 * N2;
      const int b1 = i1 < kfb ? i1 : (i1 > M1 - kfb ? i1 - M1 + 2 * kfb - 1 : -1);
      const int b2 = i2 < kfb ? i2 : (i2 > M2 - kfb ? i2 - M2 + 2 * kfb - 1 : -1);
      if (b1 >= 0 && b2 >= 0 && i3 < kfb) {
        const int nb = 2 * kfb - 1;
        const long long sb = ((long long)b1 * nb + b2) * kfb + i3;
        const long long fb = (long long)nb * nb * kfb;
        Lbox[sb] = au + pik(k1, ph);
        Lbox[fb + sb] = av + pik(k2, ph);
        Lbox[2 * fb + sb] = aw + pik(k3, ph);
      }
    }
  }
};

// u_j * (PL_q)_i, nine products (PySpectral/src/RHSfunctions.py:325-335)
template <typename T>
struct PhysPLQL {
  static constexpr int F_IN = 6, F_OUT = 9;
  __device__ __forceinline__ void operator()(long long, int, const T* in, T* out) const {
#pragma unroll
    for (int j = 0; j < 3; ++j)
#pragma unroll
      for (int i = 0; i < 3; ++i) out[3 * j + i] = in[j] * in[3 + i];
  }
};

// PLQL on the N grid and the memory-closure RHS = unpad_2x(PL) + coef*PLQL
// (PySpectral/src/RHSfunctions.py:338-358).  With coef_ptr set the PLQL field
// is stored and the RHS is formed later (dynamic tau-model).
template <typename T>
struct EpiPLQL {
  static constexpr int F_IN = 9;
  __host__ double io_bytes(long long npts) const {
    if (plql_out) return (double)sizeof(Cx<T>) * npts * 3;
    return io.bytes(npts, 3) + (double)sizeof(Cx<T>) * npts * 3;  // + PL_p read
  }
  StepIO<T> io;
  KTabs<T> k;
  const Cx<T>* PLp;
  T coef;
  int rotate;
  T Om1, Om2, Om3;
  int ny1, ny2, ny3;
  Cx<T>* plql_out;  // if non-null: store PLQL and stop
  __device__ void operator()(int i1, int i2, int i3, const Cx<T>* P) const {
    const long long s = io.sidx(i1, i2, i3);
    const T k1 = (T)k.k1[i1], k2 = (T)k.k2[i2], k3 = (T)k.k3[i3];
    T ksq, ksqi;
    ksq_pair(k1, k2, k3, ksq, ksqi);
    const Cx<T> upu = P[0], upv = P[1], upw = P[2], vpu = P[3], vpv = P[4], vpw = P[5], wpu = P[6],
                wpv = P[7], wpw = P[8];
    const Cx<T> pt = ((T)2 * ksqi) * ((k1 * k1) * upu + (k2 * k2) * vpv + (k3 * k3) * wpw +
                                      (k1 * k2) * (upv + vpu) + (k1 * k3) * (upw + wpu) + (k2 * k3) * (vpw + wpv));
    const Cx<T> Lu = mik(k1, upu) + mik(k2, vpu) + mik(k3, wpu) + mik(k1, upu) + mik(k2, upv) + mik(k3, upw) +
                     pik(k1, pt);
    const Cx<T> Lv = mik(k1, upv) + mik(k2, vpv) + mik(k3, wpv) + mik(k1, vpu) + mik(k2, vpv) + mik(k3, vpw) +
                     pik(k2, pt);
    const Cx<T> Lw = mik(k1, upw) + mik(k2, vpw) + mik(k3, wpw) + mik(k1, wpu) + mik(k2, wpv) + mik(k3, wpw) +
                     pik(k3, pt);
    if (plql_out) {
      plql_out[s] = Lu;
      plql_out[io.fstride + s] = Lv;
      plql_out[2 * io.fstride + s] = Lw;
      return;
    }
    Cx<T> u = io.Q[s], v = io.Q[io.fstride + s], w = io.Q[2 * io.fstride + s];
    if (i1 == ny1 || i2 == ny2 || i3 == ny3) u = v = w = mk<T>(0, 0);
    const Cx<T> w0u = coef * Lu, w0v = coef * Lv, w0w = coef * Lw;
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
};

// PLQL on the whole 2x grid (the second-order finite memory model needs its
// q part there): the formula of EpiPLQL with the 2x-grid wavenumbers
// (PySpectral/src/RHSfunctions.py:1131-1147), then
//   PLQLq  = seperateModes(PLQL)[1] on the 2x grid (inverse-transformed next),
//   PLQLn  = unpad_2x(PLQL) and PLQLqn = unpad_2x(PLQLq) on the N grid
// (the k3 = N3/2 plane of the N-grid outputs is not written: unpad_2x leaves it zero).
template <typename T>
struct EpiPLQLFull {
  static constexpr int F_IN = 9;
  __host__ double io_bytes(long long npts) const {
    return (double)sizeof(Cx<T>) * (3.0 * npts + 6.0 * fstride_n);
  }
  KTabs<T> kf;  // 2x-grid wavenumbers
  int N1, N2, N3, n3h;
  int nf2, nf3h;
  long long fstride_2x, fstride_n;
  Cx<T>* PLQLq;
  Cx<T>* PLQLn;
  Cx<T>* PLQLqn;
  __device__ void operator()(int i1, int i2, int i3, const Cx<T>* P) const {
    const T k1 = (T)kf.k1[i1], k2 = (T)kf.k2[i2], k3 = (T)kf.k3[i3];
    T ksq, ksqi;
    ksq_pair(k1, k2, k3, ksq, ksqi);
    const Cx<T> upu = P[0], upv = P[1], upw = P[2], vpu = P[3], vpv = P[4], vpw = P[5], wpu = P[6],
                wpv = P[7], wpw = P[8];
    const Cx<T> pt = ((T)2 * ksqi) * ((k1 * k1) * upu + (k2 * k2) * vpv + (k3 * k3) * wpw +
                                      (k1 * k2) * (upv + vpu) + (k1 * k3) * (upw + wpu) + (k2 * k3) * (vpw + wpv));
    const Cx<T> L[3] = {
        mik(k1, upu) + mik(k2, vpu) + mik(k3, wpu) + mik(k1, upu) + mik(k2, upv) + mik(k3, upw) + pik(k1, pt),
        mik(k1, upv) + mik(k2, vpv) + mik(k3, wpv) + mik(k1, vpu) + mik(k2, vpv) + mik(k3, vpw) + pik(k2, pt),
        mik(k1, upw) + mik(k2, vpw) + mik(k3, wpw) + mik(k1, wpu) + mik(k2, wpv) + mik(k3, wpw) + pik(k3, pt)};
    const bool inp = in_p_axis(i1, N1) && in_p_axis(i2, N2) && i3 < N3 / 2;
    const long long s2 = ((long long)i1 * nf2 + i2) * nf3h + i3;
    const Cx<T> z = mk<T>(0, 0);
#pragma unroll
    for (int c = 0; c < 3; ++c) PLQLq[c * fstride_2x + s2] = inp ? z : L[c];
    const int n1 = unpad2x_idx(i1, N1), n2 = unpad2x_idx(i2, N2);
    if (n1 >= 0 && n2 >= 0 && i3 < N3 / 2) {
      const long long s = ((long long)n1 * N2 + n2) * n3h + i3;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        PLQLn[c * fstride_n + s] = L[c];
        PLQLqn[c * fstride_n + s] = inp ? z : L[c];
      }
    }
  }
};

// ---- MHD t-model (no reference counterpart) ----------------------------------
// The t-model construction of PySpectral/src/RHSfunctions.py:240-363 applied to
// the MHD operator of PySpectral/src_MPI/RHSfunctions.py:95-175: resolved set
// p = the 2/3-rule set, L evaluated without aliasing on the 2x grid, QL its q
// part, PLQL the linearisation of L about (u, B) in the direction QL.

// Nonlinear MHD operator from the nine product spectra (u_iu_j - B_iB_j for
// 11,22,33,12,13,23, then u x B): momentum with the pressure projection and the
// induction curl, as in EpiMHD without dissipation, forcing and mask.
template <typename T>
__device__ __forceinline__ void mhd_nonlinear(T k1, T k2, T k3, T ksqi, const Cx<T>* P, Cx<T>* r) {
  const Cx<T> ph = ksqi * ((-k1 * k1) * P[0] - (k2 * k2) * P[1] - (k3 * k3) * P[2] - ((T)2 * k1 * k2) * P[3] -
                           ((T)2 * k1 * k3) * P[4] - ((T)2 * k2 * k3) * P[5]);
  r[0] = mik(k1, P[0]) + mik(k2, P[3]) + mik(k3, P[4]) + mik(k1, ph);
  r[1] = mik(k1, P[3]) + mik(k2, P[1]) + mik(k3, P[5]) + mik(k2, ph);
  r[2] = mik(k1, P[4]) + mik(k2, P[5]) + mik(k3, P[2]) + mik(k3, ph);
  r[3] = pik(k2, P[8]) - pik(k3, P[7]);
  r[4] = pik(k3, P[6]) - pik(k1, P[8]);
  r[5] = pik(k1, P[7]) - pik(k2, P[6]);
}

// 2x-grid epilogue: QL = L(u, B) on the modes outside the 2/3-rule set.
template <typename T>
struct EpiMHDQ {
  static constexpr int F_IN = 9;
  __host__ double io_bytes(long long npts) const { return (double)sizeof(Cx<T>) * 6 * npts; }
  KTabs<T> kf;                 // 2x-grid wavenumbers
  const double *m1, *m2, *m3;  // N-grid 2/3-rule masks
  int N1, N2, n3h;             // N-grid sizes (k3 count N3/2+1)
  int nf2, nf3h;               // 2x-grid rows along y, k3 count
  long long fstride_2x;
  T scale;  // 2x-grid transform sums -> N-grid convention (1/8)
  Cx<T>* QL;  // (6, 2N1, 2N2, N3+1)
  __device__ void operator()(int i1, int i2, int i3, const Cx<T>* P) const {
    const int n1 = unpad2x_idx(i1, N1), n2 = unpad2x_idx(i2, N2);
    const bool resolved = n1 >= 0 && n2 >= 0 && i3 < n3h && m1[n1] * m2[n2] * m3[i3] != 0.0;
    const long long s = ((long long)i1 * nf2 + i2) * nf3h + i3;
    Cx<T> r[6];
    if (resolved) {
#pragma unroll
      for (int f = 0; f < 6; ++f) r[f] = mk<T>(0, 0);
    } else {
      Cx<T> Ps[9];
#pragma unroll
      for (int m = 0; m < 9; ++m) Ps[m] = scale * P[m];
      const T k1 = (T)kf.k1[i1], k2 = (T)kf.k2[i2], k3 = (T)kf.k3[i3];
      T ksq, ksqi;
      ksq_pair(k1, k2, k3, ksq, ksqi);
      mhd_nonlinear(k1, k2, k3, ksqi, Ps, r);
    }
#pragma unroll
    for (int f = 0; f < 6; ++f) QL[f * fstride_2x + s] = r[f];
  }
};

// Linearised MHD products about (u, B) in the direction (q, r) = QL:
// u_i q_j + q_i u_j - B_i r_j - r_i B_j and q x B + u x r.
template <typename T>
struct PhysMHDLin {
  static constexpr int F_IN = 12, F_OUT = 9;
  __device__ __forceinline__ void operator()(long long, int, const T* in, T* out) const {
    const T u = in[0], v = in[1], w = in[2], b1 = in[3], b2 = in[4], b3 = in[5];
    const T q1 = in[6], q2 = in[7], q3 = in[8], r1 = in[9], r2 = in[10], r3 = in[11];
    out[0] = (T)2 * (u * q1 - b1 * r1);
    out[1] = (T)2 * (v * q2 - b2 * r2);
    out[2] = (T)2 * (w * q3 - b3 * r3);
    out[3] = u * q2 + q1 * v - b1 * r2 - r1 * b2;
    out[4] = u * q3 + q1 * w - b1 * r3 - r1 * b3;
    out[5] = v * q3 + q2 * w - b2 * r3 - r2 * b3;
    out[6] = (q2 * b3 - q3 * b2) + (v * r3 - w * r2);
    out[7] = (q3 * b1 - q1 * b3) + (w * r1 - u * r3);
    out[8] = (q1 * b2 - q2 * b1) + (u * r2 - v * r1);
  }
};

// N-grid epilogue: RHS = (plain MHD RHS, precomputed) + Ct t D PLQL, then the
// RK stage update.
template <typename T>
struct EpiMHDT {
  static constexpr int F_IN = 9;
  __host__ double io_bytes(long long npts) const {
    return io.bytes(npts, 6) + (double)sizeof(Cx<T>) * 6 * npts + (w0_out ? (double)sizeof(Cx<T>) * 6 * npts : 0.0);
  }
  StepIO<T> io;
  KTabs<T> k;
  const double *m1, *m2, *m3;
  const Cx<T>* rhs6;  // plain MHD RHS (6 fields)
  T coef;             // Ct t / 8 (2x-grid sums -> N-grid convention)
  Cx<T>* w0_out;      // memory term (6 fields) or null
  __device__ void operator()(int i1, int i2, int i3, const Cx<T>* P) const {
    const long long s = io.sidx(i1, i2, i3);
    const T D = (T)(m1[i1] * m2[i2] * m3[i3]);
    const T k1 = (T)k.k1[i1], k2 = (T)k.k2[i2], k3 = (T)k.k3[i3];
    T ksq, ksqi;
    ksq_pair(k1, k2, k3, ksq, ksqi);
    Cx<T> r[6];
    mhd_nonlinear(k1, k2, k3, ksqi, P, r);
#pragma unroll
    for (int f = 0; f < 6; ++f) {
      const Cx<T> w0 = (coef * D) * r[f];
      if (w0_out) w0_out[f * io.fstride + s] = w0;
      io.finish(s, f, rhs6[f * io.fstride + s] + w0);
    }
  }
};

}  // namespace psb

// ---- learned subgrid closure (no counterpart in the reference) -------------
#include "psb_mlp.cuh"

namespace psb {

// (u,v,w) -> (u,v,w, du_i/dx_j = i k_j u_i for i,j = 1..3), gradient order
// g[3*i + j]; the spectral expander of the learned closure's x-inverse pass.
template <typename T>
struct PreGrad {
  static constexpr int F_SRC = 3, F_DST = 12;
  __device__ void operator()(int i, int o, int c, const AxisArgs<T>& a, const Cx<T>* s, Cx<T>* d) const {
    const T k[3] = {(T)a.k_row[i], (T)a.k_outer[o], (T)a.k_col[c]};
#pragma unroll
    for (int f = 0; f < 3; ++f) d[f] = s[f];
#pragma unroll
    for (int f = 0; f < 3; ++f)
#pragma unroll
      for (int j = 0; j < 3; ++j) d[3 + 3 * f + j] = pik(k[j], s[f]);
  }
};

// y-inverse pass of the velocity-gradient pipeline: the CTA of component q
// (outer index q*M1 + x) reads u_q and its x derivative (fields q and 3+q of
// the x pass) and writes u_q, du_q/dx and du_q/dy = i k_y u_q (fields q, 3+q
// and 6+q): the y derivative is formed on load (derivatives commute with the
// x transform, so the x pass need not carry it) and every source field is
// read once.  GROUPS outer groups; input and output field strides of 3 fields.
template <typename T>
struct PreYGrad {
  static constexpr int F_SRC = 2, F_DST = 3, GROUPS = 3, IN_FIELDS = 3, OUT_FIELDS = 3;
  static constexpr bool FIELDWISE = true;
  __device__ __forceinline__ Cx<T> field(int g, int i, int, int col, const AxisArgs<T>& a, const Cx<T>* in) const {
    const Cx<T> v = in[(g == 1 ? a.in_fstride : 0) + i * a.in_rstride + col];
    return g == 2 ? pik((T)a.k_row[i], v) : v;
  }
  __device__ void operator()(int i, int, int, const AxisArgs<T>& a, const Cx<T>* s, Cx<T>* d) const {
    d[0] = s[0];
    d[1] = s[1];
    d[2] = pik((T)a.k_row[i], s[0]);
  }
};

// (u,v,w) -> (u,v,w, du_i/dx) on the x-inverse pass; the y-inverse pass
// (PreYGrad) adds du_i/dy and the z-pass forms du_i/dz = i k3 u_i itself, so
// the x pass carries 6 fields and the y pass 9 instead of 12.  z-pass input
// order is PreGrad's: u,v,w then g[3*i + j]; after the y pass the stored
// fields are (u, v, w, ux, vx, wx, uy, vy, wy).
template <typename T>
struct PreGradXY {
  static constexpr int F_SRC = 3, F_DST = 6, F_B = 9, Z_DERIVED = 3;
  static constexpr bool FIELDWISE = true;
  __device__ __forceinline__ Cx<T> field(int g, int i, int, int col, const AxisArgs<T>& a, const Cx<T>* in) const {
    const Cx<T> v = in[(g < 3 ? g : g - 3) * a.in_fstride + i * a.in_rstride + col];
    return g < 3 ? v : pik((T)a.k_row[i], v);
  }
  using YPass = PreYGrad<T>;
  __device__ void operator()(int i, int, int, const AxisArgs<T>& a, const Cx<T>* s, Cx<T>* d) const {
    const T k1 = (T)a.k_row[i];
#pragma unroll
    for (int f = 0; f < 3; ++f) {
      d[f] = s[f];
      d[3 + f] = pik(k1, s[f]);
    }
  }
  // z-pass input f (0..11) -> stored field and whether it is differentiated along z
  __host__ static void zsrc(int f, int& src, bool& der) {
    if (f < 3) {
      src = f;
      der = false;
      return;
    }
    const int i = (f - 3) / 3, j = (f - 3) % 3;
    der = j == 2;
    src = der ? i : 3 + 3 * j + i;
  }
};

// Products u_i u_j plus the MLP subgrid stress, summed so that one forward
// transform per component carries both: out_ij = u_i u_j + tau_ij / s^2 in the
// reference's real-space scaling (real-space arrays equal physical / s).
// The MLP runs warp-cooperatively on tensor cores over all points of the CTA.
// ACT: the network's hidden activation (kActRelu or kActGelu); a separate
// kernel per activation keeps the ReLU kernel free of the GELU's registers.
// H: the network's hidden width (32 or 64).
template <typename T, int ACT = kActRelu, int H = 64>
struct PhysLearned {
  static constexpr int F_IN = 12, F_OUT = 6;
  static constexpr bool BLOCK = true;
  static constexpr int EXTRA_SMEM = (int)((sizeof(MlpFwdSmem<H>) + 15) / 16 * 16);
  // 4 pencils per CTA by default (3 CTAs per SM at 3N/2 = 96, FP32); the
  // autotuner also tries 8 (fuller transform passes, 2 CTAs per SM)
  static constexpr int DEFAULT_PPC = 4, MAX_PPC = 8;
  const float* params;
  const float* norm;
  T sphys;      // s: physical = real-space * s
  float delta;  // filter width fed to the MLP
  __device__ void setup(unsigned char* extra) const {
    mlp_stage_fwd<H>(*reinterpret_cast<MlpFwdSmem<H>*>(extra), params, norm);
  }
  __device__ void block(const Cx<T>* R, Cx<T>* W, int P, int M, int LS, T fac, long long, long long,
                        unsigned char* extra) const {
    block_act(R, W, P, M, LS, fac, extra);
  }
  // Each warp takes tiles of 16 consecutive points (pencil-major); a lane
  // holds rows g and g+8 of a tile and locates them once per tile.
  __device__ __forceinline__ void block_act(const Cx<T>* R, Cx<T>* W, int P, int M, int LS, T fac,
                                            unsigned char* extra) const {
    const MlpFwdSmem<H>& s = *reinterpret_cast<const MlpFwdSmem<H>*>(extra);
    if ((M & 7) == 0 && (P & 1) == 0) {
      block_tiles(reinterpret_cast<const T*>(R), reinterpret_cast<T*>(W), P, M, LS, fac, s);
      return;
    }
    const int npts = P * M;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    const int nw = blockDim.x >> 5;
    const T is2 = (T)1 / (sphys * sphys);
    const T fs = fac * sphys;
    for (int pt0 = warp * 16; pt0 < npts; pt0 += nw * 16) {
      // rows g and g+8 of the tile: pencil p, position z
      int rp[2], rz[2];
      bool ok[2];
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int pt = pt0 + g + 8 * h;
        ok[h] = pt < npts;
        rp[h] = ok[h] ? pt / M : 0;
        rz[h] = ok[h] ? pt - rp[h] * M : 0;
      }
      auto val = [&](int f, int h) -> T {
        const int r = f * P + rp[h];
        const Cx<T> v = R[(size_t)(r >> 1) * LS + rz[h]];
        return (r & 1) ? v.y : v.x;
      };
      uint32_t xa[4];
      mlp_xfrag(s, xa, [&](int r, int f) -> float {
        const int h = r >= 8 ? 1 : 0;
        if (!ok[h]) return s.xmean[f];
        return f < 9 ? (float)(val(3 + f, h) * fs) : delta;
      });
      float y[4];
      mlp_forward_fast<ACT, H>(s, xa, y);
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int c = 2 * t + (e & 1);
        const int h = e < 2 ? 0 : 1;
        if (c >= kMlpOut || !ok[h]) continue;
        const int ii = c < 3 ? c : (c == 5 ? 1 : 0);
        const int jj = c < 3 ? c : (c == 3 ? 1 : 2);
        const T tau = (T)(y[e] * s.ystd[c] + s.ymean[c]);
        const T o = (fac * val(ii, h)) * (fac * val(jj, h)) + tau * is2;
        const int r = c * P + rp[h];
        reinterpret_cast<T*>(W + (size_t)(r >> 1) * LS + rz[h])[r & 1] = o;
      }
    }
  }
  // The same computation when packed lines pair pencils of one field (P even)
  // and M % 8 == 0: real line (f, p) is half p&1 of packed line f*P/2 + p/2
  // (lines LS apart), so field f of pencil p at z is T element
  // f*P*LS + 2((p/2) LS + z) + (p&1).  A tile is 16 consecutive T elements of
  // a packed line -- 8 consecutive z of a pencil pair, both halves -- so the
  // 8 rows a lane group reads are consecutive words and, with the field
  // stride P*LS = 28 (mod 32) words at P = 4 (LS = 7 mod 16), the 32 lanes of a
  // feature gather (8 rows x 4 features) hit 32 different banks.  Each lane keeps the
  // offsets, normalisation and output coefficients of its fragment slots in
  // registers; per tile it computes one base index per row.
  __device__ __forceinline__ void block_tiles(const T* __restrict__ R, T* __restrict__ W, int P, int M, int LS,
                                              T fac, const MlpFwdSmem<H>& s) const {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    const int nw = blockDim.x >> 5;
    const int fst = P * LS;
    const T is2 = (T)1 / (sphys * sphys);
    const T fs = fac * sphys;
    // feature slot q = 2 hk + e holds feature f = 2t + 8hk + e: a gradient
    // (f < 9, physical field 3 + f), the filter width (f = 9) or padding
    int foff[4];
    float fm[4], fi[4], fc[4];
    bool fg[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int f = 2 * t + 8 * (q >> 1) + (q & 1);
      fg[q] = f < 9;
      foff[q] = fg[q] ? (3 + f) * fst : 0;
      fm[q] = f < kMlpIn ? s.xmean[f] : 0.f;
      fi[q] = f < kMlpIn ? s.xistd[f] : 0.f;
      fc[q] = f == 9 ? (delta - s.xmean[f]) * s.xistd[f] : 0.f;
    }
    // output slot e2 = e & 1: column c = 2t + e2 (valid for c < 6) = u_ii u_jj + tau_c / s^2
    int ooff[2], ioff[2], joff[2];
    float ys[2], ym[2];
#pragma unroll
    for (int e2 = 0; e2 < 2; ++e2) {
      const int c = 2 * t + e2;
      const int ii = c < 3 ? c : (c == 5 ? 1 : 0);
      const int jj = c < 3 ? c : (c == 3 ? 1 : 2);
      ooff[e2] = c * fst;
      ioff[e2] = ii * fst;
      joff[e2] = jj * fst;
      ys[e2] = c < kMlpOut ? s.ystd[c] : 0.f;
      ym[e2] = c < kMlpOut ? s.ymean[c] : 0.f;
    }
    const bool out_ok = t < 3;
    const int tpp = M >> 3, ntile = (P >> 1) * tpp;
    for (int tile = warp; tile < ntile; tile += nw) {
      const int pp = tile / tpp;  // pencil pair
      const int z0 = (tile - pp * tpp) << 3;
      const int b0 = 2 * (pp * LS + z0) + g;  // row g; row g + 8 is b0 + 8
      float v[8];
#pragma unroll
      for (int hr = 0; hr < 2; ++hr)
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const float x = (float)(R[b0 + 8 * hr + foff[q]] * fs);
          v[hr * 4 + q] = fg[q] ? (x - fm[q]) * fi[q] : fc[q];
        }
      uint32_t xa[4];
      xa[0] = pack_bf16(v[0], v[1]);  // row g,   k 2t..2t+1
      xa[1] = pack_bf16(v[4], v[5]);  // row g+8, k 2t..2t+1
      xa[2] = pack_bf16(v[2], v[3]);  // row g,   k 2t+8..
      xa[3] = pack_bf16(v[6], v[7]);  // row g+8, k 2t+8..
      float y[4];
      mlp_forward_fast<ACT, H>(s, xa, y);
      if (out_ok) {
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const int e2 = e & 1;
          const int b = b0 + 8 * (e >> 1);
          const T tau = (T)(y[e] * ys[e2] + ym[e2]);
          W[b + ooff[e2]] = (fac * R[b + ioff[e2]]) * (fac * R[b + joff[e2]]) + tau * is2;
        }
      }
    }
  }
};

template <typename T>
struct phys_fixed_fft<PhysProducts<T>> {
  static constexpr bool value = true;
};
template <typename T>
struct phys_fixed_fft<PhysSmag<T>> {
  static constexpr bool value = true;
};
// (the GELU network keeps the runtime schedules: it is not the shipped model)
template <typename T, int H>
struct phys_fixed_fft<PhysLearned<T, kActRelu, H>> {
  static constexpr bool value = true;
};

}  // namespace psb
