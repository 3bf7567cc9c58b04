// Block-cooperative mixed-radix FFT in shared memory (sm_100a).
//
// A CTA transforms `nlines` independent lines of length L (L = 2^a 3^b) held in
// shared memory.  The algorithm is the Stockham auto-sort formulation: pass s
// combines R = radix[s] sub-transforms of length Ns into length Ns*R, reading
// element j + r*L/R and writing (j/Ns)*Ns*R + j%Ns + r*Ns, so the result comes
// out in natural order with one ping-pong buffer and one __syncthreads per
// pass.  Twiddles come from a table W_L^k = exp(-2 pi i k / L) computed on the
// host in extended precision and staged into shared memory by the caller.
//
// Used by every transform of the pseudo-spectral right-hand side: the 3/2- and
// 2x-padded real-to-complex transforms that replace pyFFTW's plans of
// PySpectral/src/Classes.py:590-625, and the unpadded transforms of the MHD
// solver (PySpectral/src_MPI/Classes.py:246-258).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace psb {

template <typename T>
struct alignas(2 * sizeof(T)) Cx {
  T x, y;
};

template <typename T>
__host__ __device__ __forceinline__ Cx<T> mk(T a, T b) {
  Cx<T> r;
  r.x = a;
  r.y = b;
  return r;
}
template <typename T>
__device__ __forceinline__ Cx<T> operator+(Cx<T> a, Cx<T> b) { return mk<T>(a.x + b.x, a.y + b.y); }
template <typename T>
__device__ __forceinline__ Cx<T> operator-(Cx<T> a, Cx<T> b) { return mk<T>(a.x - b.x, a.y - b.y); }
template <typename T>
__device__ __forceinline__ Cx<T> operator*(T s, Cx<T> a) { return mk<T>(s * a.x, s * a.y); }
template <typename T>
__device__ __forceinline__ Cx<T> cmul(Cx<T> a, Cx<T> b) {
  return mk<T>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <typename T>
__device__ __forceinline__ Cx<T> conjg(Cx<T> a) { return mk<T>(a.x, -a.y); }
// i*a and -i*a
template <typename T>
__device__ __forceinline__ Cx<T> mul_i(Cx<T> a) { return mk<T>(-a.y, a.x); }
template <typename T>
__device__ __forceinline__ Cx<T> mul_mi(Cx<T> a) { return mk<T>(a.y, -a.x); }

constexpr int kMaxPasses = 12;

// Radix schedule of one transform length (host-built).
struct FFTPlan {
  int L;
  int npass;
  int radix[kMaxPasses];
  int tw_off;  // offset of this length's twiddle table in the pool
};

// ---- small DFTs ----------------------------------------------------------
// Forward uses exp(-2 pi i m r / R); INV uses the conjugate.
template <typename T, bool INV>
__device__ __forceinline__ Cx<T> rot_mi(Cx<T> a) {  // multiply by -i (fwd) / +i (inv)
  return INV ? mul_i(a) : mul_mi(a);
}

template <typename T, bool INV>
__device__ __forceinline__ void dft2(Cx<T>& a, Cx<T>& b) {
  Cx<T> t = a - b;
  a = a + b;
  b = t;
}

template <typename T, bool INV>
__device__ __forceinline__ void dft4(Cx<T>& v0, Cx<T>& v1, Cx<T>& v2, Cx<T>& v3) {
  Cx<T> t0 = v0 + v2, t1 = v0 - v2, t2 = v1 + v3, t3 = rot_mi<T, INV>(v1 - v3);
  v0 = t0 + t2;
  v2 = t0 - t2;
  v1 = t1 + t3;
  v3 = t1 - t3;
}

template <typename T, bool INV>
__device__ __forceinline__ void dft3(Cx<T>& v0, Cx<T>& v1, Cx<T>& v2) {
  // sin(2 pi / 3) = sqrt(3)/2
  const T s3 = (T)0.86602540378443864676372317075294;
  Cx<T> s = v1 + v2, d = v1 - v2;
  Cx<T> m = v0 - (T)0.5 * s;
  Cx<T> r = rot_mi<T, INV>(s3 * d);
  v0 = v0 + s;
  v1 = m + r;
  v2 = m - r;
}

template <typename T, bool INV>
__device__ __forceinline__ void dft8(Cx<T>* v) {
  const T h = (T)0.70710678118654752440084436210485;  // sqrt(2)/2
  Cx<T> a[4], b[4];
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    a[r] = v[r] + v[r + 4];
    b[r] = v[r] - v[r + 4];
  }
  // b[r] *= W8^r
  b[1] = INV ? mk<T>(h * (b[1].x - b[1].y), h * (b[1].x + b[1].y))
             : mk<T>(h * (b[1].x + b[1].y), h * (b[1].y - b[1].x));
  b[2] = rot_mi<T, INV>(b[2]);
  b[3] = INV ? mk<T>(-h * (b[3].x + b[3].y), h * (b[3].x - b[3].y))
             : mk<T>(h * (b[3].y - b[3].x), -h * (b[3].x + b[3].y));
  dft4<T, INV>(a[0], a[1], a[2], a[3]);
  dft4<T, INV>(b[0], b[1], b[2], b[3]);
#pragma unroll
  for (int m = 0; m < 4; ++m) {
    v[2 * m] = a[m];
    v[2 * m + 1] = b[m];
  }
}

// cos and sin of 2 pi q / 48 from a quarter-wave table (steps of 7.5 degrees)
struct Trig48 {
  static constexpr double c[13] = {1.0,
                                   0.99144486137381041114455,
                                   0.96592582628906828674974,
                                   0.92387953251128675612818,
                                   0.86602540378443864676372,
                                   0.79335334029123516457751,
                                   0.70710678118654752440084,
                                   0.60876142900872063941609,
                                   0.5,
                                   0.38268343236508977172846,
                                   0.25881904510252076234890,
                                   0.13052619222005159154840,
                                   0.0};
  static constexpr double cosq(int q) {
    q = ((q % 48) + 48) % 48;
    return q <= 12 ? c[q] : (q <= 24 ? -c[24 - q] : (q <= 36 ? -c[q - 24] : c[48 - q]));
  }
  static constexpr double sinq(int q) { return cosq(12 - q); }
};

// x * W_R^M, W_R = exp(-2 pi i / R) (conjugate for INV); 48 % R == 0
template <typename T, bool INV, int M, int R>
__device__ __forceinline__ Cx<T> twc(Cx<T> x) {
  constexpr int q = (M * (48 / R)) % 48;
  if constexpr (q == 0) {
    return x;
  } else {
    constexpr T c = (T)Trig48::cosq(q), s = (T)Trig48::sinq(q);
    return INV ? mk<T>(c * x.x - s * x.y, c * x.y + s * x.x) : mk<T>(c * x.x + s * x.y, c * x.y - s * x.x);
  }
}

template <typename T, int R, bool INV>
__device__ __forceinline__ void small_dft(Cx<T>* v);

// R1 x R2 Cooley-Tukey in registers: X[k1 + R1 k2] =
// sum_n2 W_R2^{n2 k2} W_R^{n2 k1} sum_n1 x[R2 n1 + n2] W_R1^{n1 k1}
template <typename T, int R1, int R2, bool INV>
struct DftCT {
  static constexpr int R = R1 * R2;
  template <int N2>
  __device__ __forceinline__ static void col(const Cx<T>* v, Cx<T>* a) {
    if constexpr (N2 < R2) {
      Cx<T> u[R1];
#pragma unroll
      for (int n1 = 0; n1 < R1; ++n1) u[n1] = v[R2 * n1 + N2];
      small_dft<T, R1, INV>(u);
      tw<N2, 0>(u, a);
      col<N2 + 1>(v, a);
    }
  }
  template <int N2, int K1>
  __device__ __forceinline__ static void tw(const Cx<T>* u, Cx<T>* a) {
    if constexpr (K1 < R1) {
      a[N2 * R1 + K1] = twc<T, INV, N2 * K1, R>(u[K1]);
      tw<N2, K1 + 1>(u, a);
    }
  }
  __device__ __forceinline__ static void run(Cx<T>* v) {
    Cx<T> a[R];
    col<0>(v, a);
#pragma unroll
    for (int k1 = 0; k1 < R1; ++k1) {
      Cx<T> w[R2];
#pragma unroll
      for (int n2 = 0; n2 < R2; ++n2) w[n2] = a[n2 * R1 + k1];
      small_dft<T, R2, INV>(w);
#pragma unroll
      for (int k2 = 0; k2 < R2; ++k2) v[k1 + R1 * k2] = w[k2];
    }
  }
};

template <typename T, int R, bool INV>
__device__ __forceinline__ void small_dft(Cx<T>* v) {
  if constexpr (R == 2) {
    dft2<T, INV>(v[0], v[1]);
  } else if constexpr (R == 3) {
    dft3<T, INV>(v[0], v[1], v[2]);
  } else if constexpr (R == 4) {
    dft4<T, INV>(v[0], v[1], v[2], v[3]);
  } else if constexpr (R == 8) {
    dft8<T, INV>(v);
  } else if constexpr (R == 6) {
    DftCT<T, 2, 3, INV>::run(v);
  } else if constexpr (R == 12) {
    DftCT<T, 4, 3, INV>::run(v);
  } else {
    static_assert(R == 16, "radix 2, 3, 4, 6, 8, 12 or 16");
    DftCT<T, 4, 4, INV>::run(v);
  }
}

// One Stockham pass of radix R over `nlines` lines held at buf[line*ls + j*es]
// (j < L).  Work item (line, j < L/R) reads element j + r*L/R of its line,
// applies the twiddles W_{Ns R}^{r k} (k = j mod Ns), runs the R-point DFT and
// writes element (j - k) R + k + r Ns.  Items are walked as a (fast, slow)
// counter pair advanced by blockDim.x items per iteration without a division
// (fast = line when lines_fast, else j); k follows j modulo Ns the same way
// (Ns divides L/R, so a wrap of j leaves k's step unchanged).
template <typename T, int R, bool INV>
__device__ __forceinline__ void stockham_pass(const Cx<T>* __restrict__ a, Cx<T>* __restrict__ b,
                                              const Cx<T>* __restrict__ tw, int L, int Ns, int nlines, int ls,
                                              int es, bool lines_fast) {
  const int nb = L / R;
  const int tstride = L / (Ns * R);
  const int mf = lines_fast ? nlines : nb;
  const int ms = lines_fast ? nb : nlines;
  const int nt = blockDim.x;
  int f = threadIdx.x % mf, sl = threadIdx.x / mf;
  const int df = nt % mf, ds = nt / mf;
  int j = lines_fast ? sl : f;
  int k = j % Ns;
  const int dk = lines_fast ? ds % Ns : df % Ns;
  const size_t rs = (size_t)nb * es, ws = (size_t)Ns * es;
  while (sl < ms) {
    const int line = lines_fast ? f : sl;
    const Cx<T>* src = a + (size_t)line * ls + (size_t)j * es;
    Cx<T> v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = src[r * rs];
    if (k) {
      const int tstep = k * tstride;
#pragma unroll
      for (int r = 1; r < R; ++r) {
        Cx<T> w = tw[r * tstep];
        if (INV) w.y = -w.y;
        v[r] = cmul(v[r], w);
      }
    }
    small_dft<T, R, INV>(v);
    Cx<T>* dst = b + (size_t)line * ls + (size_t)((j - k) * R + k) * es;
#pragma unroll
    for (int r = 0; r < R; ++r) dst[r * ws] = v[r];
    f += df;
    sl += ds;
    const int carry = f >= mf ? 1 : 0;
    f -= carry * mf;
    sl += carry;
    if (lines_fast) {
      j = sl;
      k += dk + carry;
    } else {
      j = f;
      k += dk;
    }
    if (k >= Ns) k -= Ns;
  }
}

// Transform `nlines` lines held at buf[line*ls + j*es] (j < L).  `a` holds the
// input; `b` is scratch of the same footprint.  Returns the buffer holding the
// result.  lines_fast selects the thread->work mapping: true when consecutive
// lines are adjacent in memory (es > 1, ls == 1), false for contiguous lines.
// Must be called by all threads of the CTA; ends with __syncthreads.
// WIDE compiles the radix 6/12/16 passes in as well (plans that use them must
// run a WIDE instantiation); without it only 2/3/4/8 exist, which keeps the
// register budget of every kernel at what radix 8 needs.
template <typename T, bool INV, bool WIDE = false>
__device__ Cx<T>* block_fft(Cx<T>* a, Cx<T>* b, const FFTPlan& p, const Cx<T>* __restrict__ tw,
                            int nlines, int ls, int es, bool lines_fast) {
  const int L = p.L;
  int Ns = 1;
  for (int s = 0; s < p.npass; ++s) {
    const int R = p.radix[s];
    if constexpr (WIDE) {
      switch (R) {
        case 16: stockham_pass<T, 16, INV>(a, b, tw, L, Ns, nlines, ls, es, lines_fast); break;
        case 12: stockham_pass<T, 12, INV>(a, b, tw, L, Ns, nlines, ls, es, lines_fast); break;
        case 8: stockham_pass<T, 8, INV>(a, b, tw, L, Ns, nlines, ls, es, lines_fast); break;
        case 6: stockham_pass<T, 6, INV>(a, b, tw, L, Ns, nlines, ls, es, lines_fast); break;
        case 4: stockham_pass<T, 4, INV>(a, b, tw, L, Ns, nlines, ls, es, lines_fast); break;
        case 3: stockham_pass<T, 3, INV>(a, b, tw, L, Ns, nlines, ls, es, lines_fast); break;
        default: stockham_pass<T, 2, INV>(a, b, tw, L, Ns, nlines, ls, es, lines_fast); break;
      }
    } else {
      switch (R) {
        case 8: stockham_pass<T, 8, INV>(a, b, tw, L, Ns, nlines, ls, es, lines_fast); break;
        case 4: stockham_pass<T, 4, INV>(a, b, tw, L, Ns, nlines, ls, es, lines_fast); break;
        case 3: stockham_pass<T, 3, INV>(a, b, tw, L, Ns, nlines, ls, es, lines_fast); break;
        default: stockham_pass<T, 2, INV>(a, b, tw, L, Ns, nlines, ls, es, lines_fast); break;
      }
    }
    __syncthreads();
    Cx<T>* t = a;
    a = b;
    b = t;
    Ns *= R;
  }
  return a;
}


// ---- transforms with a compile-time length and schedule --------------------
// The Stockham passes with L, the radix and the sub-transform length Ns known
// to the compiler, over `nlines` lines of length L held at buf[line*ls + j]
// (the z-pass layout: each line contiguous, consecutive lines `ls` elements
// apart; the z pass pads ls to an odd stride, 7 modulo 16, so that the same
// position of consecutive lines falls in different shared-memory banks).
//
// LINES_FAST (used when nlines >= 8): consecutive threads take consecutive
// lines at the same j.  A warp's loads j + r*L/R, its stores (j-k)R + k + r*Ns
// and its twiddle reads (one k per j: a broadcast) then spread over the banks
// by the odd line stride, where in the j-fast order the stores of one line
// land R elements apart and hit one bank up to 16 times per half-warp.
// Otherwise consecutive threads take consecutive j of a line.  Items are
// walked as a (fast, slow) counter pair, without a division.
template <typename T, int R, bool INV, int L, int NS, bool LINES_FAST>
__device__ __forceinline__ void stockham_pass_c(const Cx<T>* __restrict__ a, Cx<T>* __restrict__ b,
                                                const Cx<T>* __restrict__ tw, int nlines, int ls) {
  constexpr int NB = L / R;
  constexpr int TS = L / (NS * R);
  const int mf = LINES_FAST ? nlines : NB;
  const int ms = LINES_FAST ? NB : nlines;
  const int nt = blockDim.x;
  int f = threadIdx.x % mf, sl = threadIdx.x / mf;
  const int df = nt % mf, ds = nt / mf;
  while (sl < ms) {
    const int line = LINES_FAST ? f : sl;
    const int j = LINES_FAST ? sl : f;
    const int k = j % NS;
    const Cx<T>* src = a + line * ls + j;
    Cx<T> v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = src[r * NB];
    if constexpr (NS > 1) {
#pragma unroll
      for (int r = 1; r < R; ++r) {
        Cx<T> w = tw[r * k * TS];
        if (INV) w.y = -w.y;
        v[r] = cmul(v[r], w);
      }
    }
    small_dft<T, R, INV>(v);
    Cx<T>* dst = b + line * ls + (j - k) * R + k;
#pragma unroll
    for (int r = 0; r < R; ++r) dst[r * NS] = v[r];
    f += df;
    sl += ds;
    if (f >= mf) {
      f -= mf;
      ++sl;
    }
  }
}
// Passes R, Rest... starting at sub-transform length NS; returns the buffer
// holding the result.  Ends with __syncthreads.
template <typename T, bool INV, int L, int NS, bool LF, int R, int... Rest>
__device__ __forceinline__ Cx<T>* fft_c(Cx<T>* a, Cx<T>* b, const Cx<T>* __restrict__ tw, int nlines, int ls) {
  stockham_pass_c<T, R, INV, L, NS, LF>(a, b, tw, nlines, ls);
  __syncthreads();
  if constexpr (sizeof...(Rest) == 0)
    return b;
  else
    return fft_c<T, INV, L, NS * R, LF, Rest...>(b, a, tw, nlines, ls);
}

// The same for lines adjacent in memory (element j of line f at f + j*es, the
// axis-pass layout): items walk (line fast, j slow) as a counter pair.
template <typename T, int R, bool INV, int L, int NS>
__device__ __forceinline__ void stockham_pass_cs(const Cx<T>* __restrict__ a, Cx<T>* __restrict__ b,
                                                 const Cx<T>* __restrict__ tw, int nlines, int es) {
  constexpr int NB = L / R;
  constexpr int TS = L / (NS * R);
  const int nt = blockDim.x;
  int f = threadIdx.x % nlines, j = threadIdx.x / nlines;
  const int df = nt % nlines, dj = nt / nlines;
  const int rs = NB * es, ws = NS * es;
  while (j < NB) {
    const int k = j % NS;
    const Cx<T>* src = a + f + j * es;
    Cx<T> v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = src[r * rs];
    if constexpr (NS > 1) {
#pragma unroll
      for (int r = 1; r < R; ++r) {
        Cx<T> w = tw[r * k * TS];
        if (INV) w.y = -w.y;
        v[r] = cmul(v[r], w);
      }
    }
    small_dft<T, R, INV>(v);
    Cx<T>* dst = b + f + ((j - k) * R + k) * es;
#pragma unroll
    for (int r = 0; r < R; ++r) dst[r * ws] = v[r];
    f += df;
    j += dj;
    if (f >= nlines) {
      f -= nlines;
      ++j;
    }
  }
}
template <typename T, bool INV, int L, int NS, int R, int... Rest>
__device__ __forceinline__ Cx<T>* fft_cs(Cx<T>* a, Cx<T>* b, const Cx<T>* __restrict__ tw, int nlines) {
  stockham_pass_cs<T, R, INV, L, NS>(a, b, tw, nlines, nlines);
  __syncthreads();
  if constexpr (sizeof...(Rest) == 0)
    return b;
  else
    return fft_cs<T, INV, L, NS * R, Rest...>(b, a, tw, nlines);
}

// Schedules compiled in with their length (id, L, radices): the default
// schedule of each common 3/2-padded length (48, 72, 96, 192: grids of 32,
// 48, 64 and 128 points) and two-pass orders of it.
#define PSB_FIXED_PLANS(X) \
  X(1, 96, 8, 4, 3)        \
  X(2, 96, 16, 6)          \
  X(3, 96, 6, 16)          \
  X(4, 48, 8, 2, 3)        \
  X(5, 48, 16, 3)          \
  X(6, 48, 3, 16)          \
  X(7, 192, 8, 8, 3)       \
  X(8, 192, 16, 12)        \
  X(9, 192, 12, 16)        \
  X(10, 96, 12, 8)         \
  X(11, 96, 8, 12)         \
  X(12, 48, 8, 6)          \
  X(13, 48, 6, 8)          \
  X(14, 72, 8, 3, 3)       \
  X(15, 72, 6, 12)         \
  X(16, 72, 12, 6)
constexpr int kFixedPlans = 16;

template <int ID>
struct FixedPlan;
template <int R1, int R2 = 0, int R3 = 0>
struct RadixList {
  static constexpr int NP = R3 ? 3 : (R2 ? 2 : 1), A = R1, B = R2;
};
#define PSB_FIXED_PLAN_DEF(ID, LEN, ...)                                                       \
  template <>                                                                                   \
  struct FixedPlan<ID> {                                                                        \
    static constexpr int L = LEN;                                                               \
    using Radices = RadixList<__VA_ARGS__>; /* NP passes; A, B the first two radices */         \
    template <typename T, bool INV>                                                             \
    static __device__ __forceinline__ Cx<T>* run(Cx<T>* a, Cx<T>* b, const Cx<T>* tw, int n,    \
                                                 int ls) {                                      \
      if (n >= 8) return fft_c<T, INV, LEN, 1, true, __VA_ARGS__>(a, b, tw, n, ls);             \
      return fft_c<T, INV, LEN, 1, false, __VA_ARGS__>(a, b, tw, n, ls);                        \
    }                                                                                           \
    template <typename T, bool INV>                                                             \
    static __device__ __forceinline__ Cx<T>* run_adjacent(Cx<T>* a, Cx<T>* b, const Cx<T>* tw, \
                                                          int n) {                              \
      return fft_cs<T, INV, LEN, 1, __VA_ARGS__>(a, b, tw, n);                                  \
    }                                                                                           \
  };
PSB_FIXED_PLANS(PSB_FIXED_PLAN_DEF)
#undef PSB_FIXED_PLAN_DEF

template <int... R>
constexpr int count_radices() {
  return (int)sizeof...(R);
}
// The compiled-in schedules as a compile-time table, and the id of the
// two-pass schedule that runs the radices of `id` in the opposite order (0 if
// `id` is not a two-pass schedule or its reverse is not compiled in).
struct FixedDesc {
  int id, L, n, r[3];
};
#define PSB_FIXED_PLAN_CDESC(ID, LEN, ...) FixedDesc{ID, LEN, count_radices<__VA_ARGS__>(), {__VA_ARGS__}},
constexpr FixedDesc kFixedDescs[] = {PSB_FIXED_PLANS(PSB_FIXED_PLAN_CDESC)};
#undef PSB_FIXED_PLAN_CDESC
constexpr int fixed_plan_reversed(int id) {
  for (const FixedDesc& d : kFixedDescs) {
    if (d.id != id) continue;
    if (d.n != 2) return 0;
    for (const FixedDesc& e : kFixedDescs)
      if (e.L == d.L && e.n == 2 && e.r[0] == d.r[1] && e.r[1] == d.r[0]) return e.id;
  }
  return 0;
}

// Id of the compiled-in schedule equal to p (0 if none).
__host__ inline int fixed_plan_id(const FFTPlan& p) {
  struct D {
    int id, L, n, r[4];
  };
#define PSB_FIXED_PLAN_DESC(ID, LEN, ...) D{ID, LEN, count_radices<__VA_ARGS__>(), {__VA_ARGS__}},
  static const D table[] = {PSB_FIXED_PLANS(PSB_FIXED_PLAN_DESC)};
#undef PSB_FIXED_PLAN_DESC
  for (const D& d : table) {
    if (d.L != p.L || d.n != p.npass) continue;
    bool same = true;
    for (int s = 0; s < d.n; ++s) same = same && d.r[s] == p.radix[s];
    if (same) return d.id;
  }
  return 0;
}

// Stage a length-L twiddle table into shared memory.
template <typename T>
__device__ __forceinline__ void stage_twiddles(Cx<T>* tw_s, const Cx<T>* __restrict__ pool, const FFTPlan& p) {
  for (int k = threadIdx.x; k < p.L; k += blockDim.x) tw_s[k] = pool[p.tw_off + k];
}

}  // namespace psb
