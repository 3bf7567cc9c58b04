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

template <typename T, int R, bool INV>
__device__ __forceinline__ void small_dft(Cx<T>* v) {
  if constexpr (R == 2) {
    dft2<T, INV>(v[0], v[1]);
  } else if constexpr (R == 3) {
    dft3<T, INV>(v[0], v[1], v[2]);
  } else if constexpr (R == 4) {
    dft4<T, INV>(v[0], v[1], v[2], v[3]);
  } else {
    dft8<T, INV>(v);
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
template <typename T, bool INV>
__device__ Cx<T>* block_fft(Cx<T>* a, Cx<T>* b, const FFTPlan& p, const Cx<T>* __restrict__ tw,
                            int nlines, int ls, int es, bool lines_fast) {
  const int L = p.L;
  int Ns = 1;
  for (int s = 0; s < p.npass; ++s) {
    const int R = p.radix[s];
    switch (R) {
      case 8: stockham_pass<T, 8, INV>(a, b, tw, L, Ns, nlines, ls, es, lines_fast); break;
      case 4: stockham_pass<T, 4, INV>(a, b, tw, L, Ns, nlines, ls, es, lines_fast); break;
      case 3: stockham_pass<T, 3, INV>(a, b, tw, L, Ns, nlines, ls, es, lines_fast); break;
      default: stockham_pass<T, 2, INV>(a, b, tw, L, Ns, nlines, ls, es, lines_fast); break;
    }
    __syncthreads();
    Cx<T>* t = a;
    a = b;
    b = t;
    Ns *= R;
  }
  return a;
}

// Stage a length-L twiddle table into shared memory.
template <typename T>
__device__ __forceinline__ void stage_twiddles(Cx<T>* tw_s, const Cx<T>* __restrict__ pool, const FFTPlan& p) {
  for (int k = threadIdx.x; k < p.L; k += blockDim.x) tw_s[k] = pool[p.tw_off + k];
}

}  // namespace psb
