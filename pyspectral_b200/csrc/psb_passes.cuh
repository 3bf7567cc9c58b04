// Pencil passes of the padded 3-D real FFTs, each fused with the pointwise
// work that sits next to it in the reference's dataflow.
//
// Spectral layout  : field-major (F, N1, N2, N3/2+1), k3 contiguous.
// Intermediates    : (F, rows_x, rows_y, Kz) with Kz the retained k3 count, so
//                    every pass reads and writes rows of Kz contiguous complex
//                    values (coalesced, no transposes).
//
//  axis_pass_kernel   one strided axis (x or y): gathers the retained rows
//                     into their padded FFT positions (or the reverse on the
//                     forward side), runs the transform along that axis for a
//                     tile of contiguous columns, scatters the result.  A
//                     `Pre` functor can expand the source fields on load
//                     (e.g. u -> u, S_ij = (i/2)(k_j u_i + k_i u_j)).
//  zpass_kernel       the contiguous axis: c2r of F_IN spectral pencils
//                     (two real lines packed per complex transform), the
//                     physical-space products of a `Phys` functor, r2c of the
//                     F_OUT results truncated to the retained k3 -- physical
//                     space never touches HBM.
//  xfwd_epi_kernel    the last forward pass (x) fused with the spectral
//                     epilogue (`Epi`): pressure projection, viscous term,
//                     closure divergence, Coriolis, RK stage update.
//
// The padding maps reproduce PySpectral/src/padding.py:2-49 (pad/unpad drop
// index N/2 of x and y and the k3=N/2 plane; pad_2x/unpad_2x keep the -N/2
// mode).
#pragma once
#include "psb_fft.cuh"
#include "psb_tma.cuh"

namespace psb {

// Programmatic dependent launch (sm_90+): the pipeline's kernels are launched
// so that the next one may start while this one drains.  Each kernel lets its
// successor launch as soon as all of its own CTAs are running (pdl_trigger:
// by then none of them waits for a free SM, so the successor's waiting CTAs
// cannot starve them), stages what does not depend on its predecessor
// (twiddles, network weights, shared-memory zero fill), and waits for the
// predecessor grid to complete and flush its memory (pdl_wait) before the
// first global read or write of pipeline data.  Both are no-ops in a launch
// without the attribute.
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// Spectral row index i -> FFT position j (or -1 when the row is not carried).
struct RowMap {
  int lo, hi, shift;
  __device__ __forceinline__ int operator()(int i) const { return i < lo ? i : (i >= hi ? i + shift : -1); }
};

constexpr int kMaxZFields = 16;

// Walks the work items (fast, slow) = (id % mf, id / mf) of id = threadIdx.x +
// n * blockDim.x without a division per item.
struct Walk2 {
  int f, s, df, ds, mf;
  __device__ __forceinline__ explicit Walk2(int m) : mf(m) {
    f = threadIdx.x % m;
    s = threadIdx.x / m;
    df = blockDim.x % m;
    ds = blockDim.x / m;
  }
  __device__ __forceinline__ void next() {
    f += df;
    s += ds;
    if (f >= mf) {
      f -= mf;
      ++s;
    }
  }
};

// (field, pencil) of packed real line r = f*P + p; P is a power of two in
// every launch (lp = log2 P), otherwise divide
__device__ __forceinline__ void split_line(int r, int P, int lp, int& f, int& p) {
  if ((P & (P - 1)) == 0) {
    f = r >> lp;
    p = r & (P - 1);
  } else {
    f = r / P;
    p = r - f * P;
  }
}

// Phys functors with `static constexpr bool BLOCK = true` provide
// setup(extra_smem) and block(R, W, P, M, LS, fac, p0, npencils, extra_smem)
// and ask for EXTRA_SMEM bytes behind the z-pass buffers.  R and W hold packed
// real line r (field f, pencil p: r = f*P + p) at component r&1 of complex
// line r>>1, position z at buf[(r>>1)*LS + z] (LS = zline(M)).
template <class P, class = void>
struct phys_is_block {
  static constexpr bool value = false;
  static constexpr int extra = 0;
};
template <class P>
struct phys_is_block<P, decltype((void)P::BLOCK, void())> {
  static constexpr bool value = P::BLOCK;
  static constexpr int extra = P::EXTRA_SMEM;
};

// Upper bound on the pencils per z-pass CTA (Phys::MAX_PPC, default 8).
template <class P, class = void>
struct phys_max_ppc {
  static constexpr int value = 8;
};
template <class P>
struct phys_max_ppc<P, decltype((void)P::MAX_PPC, void())> {
  static constexpr int value = P::MAX_PPC;
};
// Pencils per CTA of the untuned launch shape (Phys::DEFAULT_PPC, else the bound).
template <class P, class = void>
struct phys_default_ppc {
  static constexpr int value = phys_max_ppc<P>::value;
};
template <class P>
struct phys_default_ppc<P, decltype((void)P::DEFAULT_PPC, void())> {
  static constexpr int value = P::DEFAULT_PPC;
};

template <typename T>
struct AxisArgs {
  const Cx<T>* in;
  Cx<T>* out;
  long long in_fstride, in_ostride, in_rstride;
  long long out_fstride, out_ostride, out_rstride;
  int nouter;    // outer (batch) indices
  int ncols;     // contiguous columns per outer index
  int col_tile;  // columns per CTA
  int in_rows, out_rows;
  RowMap in_map, out_map;
  T scale;  // applied on store
  FFTPlan plan;
  const Cx<T>* tw;
  const double* k_row;  // wavenumbers of the input rows (for Pre)
  const double* k_outer;
  const double* k_col;
};

template <typename T>
struct PreCopy {
  static constexpr int F_SRC = 1, F_DST = 1;
  static constexpr bool FIELDWISE = true;
  __device__ void operator()(int, int, int, const AxisArgs<T>&, const Cx<T>* s, Cx<T>* d) const { d[0] = s[0]; }
  __device__ __forceinline__ Cx<T> field(int, int i, int, int col, const AxisArgs<T>& a, const Cx<T>* in) const {
    return in[i * a.in_rstride + col];
  }
};

// Pre functors that can form any one destination field at a row straight
// from the inputs (`field(g, i, o, col, a, in)`), so a pass can load its
// first transform pass's elements from global memory into registers.
template <class P, class = void>
struct pre_fieldwise {
  static constexpr bool value = false;
};
template <class P>
struct pre_fieldwise<P, decltype((void)P::FIELDWISE, void())> {
  static constexpr bool value = P::FIELDWISE;
};

// Row of a row map's position p (the inverse of RowMap), or -1.
__device__ __forceinline__ int row_of(const RowMap& m, int p, int rows) {
  const int i = p < m.lo ? p : (p >= m.hi + m.shift ? p - m.shift : -1);
  return i < rows ? i : -1;
}

// One CTA of an axis pass: column tile bx, outer index by.
// smem = tw[L] + 2 * L*lines
// Transform of `lines` adjacent lines (axis-pass layout): the plan's schedule
// (FP = 0) or the compiled-in schedule FP (which must equal the plan's).
template <typename T, bool INV, bool WIDE, int FP>
__device__ __forceinline__ Cx<T>* axfft(Cx<T>* a, Cx<T>* b, const FFTPlan& p, const Cx<T>* tw, int lines) {
  if constexpr (FP == 0)
    return block_fft<T, INV, WIDE>(a, b, p, tw, lines, 1, lines, true);
  else
    return FixedPlan<FP>::template run_adjacent<T, INV>(a, b, tw, lines);
}

// Transform of a staged tile (F fields x ct columns, position-major in bufA)
// and the store of its output rows.  Must be called by all threads.
template <typename T, bool INV, int F, bool WIDE, int FP>
__device__ __forceinline__ void axis_transform_store(const AxisArgs<T>& a, Cx<T>* bufA, Cx<T>* bufB,
                                                     const Cx<T>* tw, int o, int c0) {
  const int ct = a.col_tile;
  const int lines = F * ct;
  const Cx<T> zero = mk<T>(0, 0);
  const int nt = blockDim.x;
  const int c = threadIdx.x % ct, r0 = threadIdx.x / ct, dr = nt / ct;
  const int col = c0 + c;
  const bool colok = col < a.ncols;
  Cx<T>* res = axfft<T, INV, WIDE, FP>(bufA, bufB, a.plan, tw, lines);
  Cx<T>* outb = a.out + (long long)o * a.out_ostride;
  if (!colok || threadIdx.x >= dr * ct) return;
  const int nrow = a.out_rows * F;
  for (int t = r0; t < nrow; t += dr) {
    const int i = t / F, g = t - i * F;
    const int j = a.out_map(i);
    outb[g * a.out_fstride + i * a.out_rstride + col] = j >= 0 ? a.scale * res[(size_t)j * lines + g * ct + c] : zero;
  }
}

template <typename T>
__device__ __forceinline__ T nan_of() {
  return sizeof(T) == 8 ? (T)__longlong_as_double(0x7ff8000000000000ll) : (T)__int_as_float(0x7fc00000);
}

// Shared memory of a TMA-staged pass ahead of its two transform buffers: the
// twiddles and up to 127 bytes that bring the first buffer to a 128-byte
// boundary of the shared window (bulk tensor copies land on such boundaries;
// the dynamic region starts behind the kernel's static shared variables).
template <typename T>
__host__ __device__ inline size_t tma_buf_offset(int L) {
  return (size_t)L * sizeof(Cx<T>) + 128;
}
// The transform buffer: the first 128-byte boundary of the shared window at
// or after the twiddles' end.
template <typename T>
__device__ __forceinline__ Cx<T>* tma_buf(unsigned char* smem, int L) {
  const uint32_t a = tma::smem_u32(smem) + (uint32_t)(L * sizeof(Cx<T>));
  const uint32_t pad = (128u - (a & 127u)) & 127u;
  return reinterpret_cast<Cx<T>*>(smem + L * sizeof(Cx<T>) + pad);
}
// Issue the copies of a tile of nbox boxes of `rows` rows each (box b: rows
// b*rows.., landing `box_elems` elements after box b-1; x the first column in
// 32-bit words, outer the outer index) unless a destination or the tensor map
// breaks the copy's alignment rules; returns false (nothing issued) then.
template <typename T>
__device__ __forceinline__ bool tma_issue(const CUtensorMap* map, Cx<T>* dst, size_t box_elems, int nbox, int rows,
                                          int x, int outer, uint32_t mb, uint32_t bytes) {
  if ((reinterpret_cast<uintptr_t>(map) & 63) != 0) return false;
  for (int b = 0; b < nbox; ++b)
    if ((tma::smem_u32(dst + (size_t)b * box_elems) & 127u) != 0) return false;
  tma::mbar_arrive_expect(mb, bytes);
  for (int b = 0; b < nbox; ++b)
    tma::load4d(tma::smem_u32(dst + (size_t)b * box_elems), map, x, 0, b * rows, outer, mb);
  return true;
}

template <typename T, bool INV, class Pre, bool WIDE = false, int FP = 0>
__device__ __forceinline__ void axis_pass_body(const AxisArgs<T>& a, const Pre& pre, int bx, int by) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Cx<T>* tw = reinterpret_cast<Cx<T>*>(smem_raw);
  const int L = a.plan.L;
  const int ct = a.col_tile;
  const int lines = Pre::F_DST * ct;
  Cx<T>* bufA = tw + L;
  Cx<T>* bufB = bufA + (size_t)L * lines;
  const int o = by;
  const int c0 = bx * ct;
  pdl_trigger();
  stage_twiddles(tw, a.tw, a.plan);
  const Cx<T> zero = mk<T>(0, 0);
  // A thread keeps one column c of the tile and walks rows with stride nt/ct
  // (launches use power-of-two tiles, which divide the CTA size).
  const int nt = blockDim.x;
  const int c = threadIdx.x % ct, r0 = threadIdx.x / ct, dr = nt / ct;
  const int col = c0 + c;
  const bool colok = col < a.ncols;
  // zero the FFT positions that no input row fills: [lo, hi+shift) and
  // [in_rows+shift, L) of the row map (every map used has in_rows >= hi)
  {
    const RowMap m = a.in_map;
    const int g0 = m.lo < L ? m.lo : L, g1 = min(m.hi + m.shift, L);
    const int t0 = min(a.in_rows + m.shift, L);
    for (int j = g0; j < g1; ++j)
      for (int l = threadIdx.x; l < lines; l += nt) bufA[(size_t)j * lines + l] = zero;
    for (int j = t0; j < L; ++j)
      for (int l = threadIdx.x; l < lines; l += nt) bufA[(size_t)j * lines + l] = zero;
  }
  pdl_wait();
  const Cx<T>* inb = a.in + (long long)o * a.in_ostride;
  // U rows per round: every load of a round is issued before the first store
  constexpr int U = Pre::F_SRC >= 3 ? 2 : (Pre::F_SRC == 2 ? 4 : 8);
  for (int i0 = r0; i0 < a.in_rows; i0 += U * dr) {
    Cx<T> s[U][Pre::F_SRC];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int i = i0 + u * dr;
#pragma unroll
      for (int f = 0; f < Pre::F_SRC; ++f)
        s[u][f] = (colok && i < a.in_rows) ? inb[f * a.in_fstride + i * a.in_rstride + col] : zero;
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int i = i0 + u * dr;
      if (i >= a.in_rows) break;
      const int j = a.in_map(i);
      if (j < 0) continue;
      Cx<T> d[Pre::F_DST];
      if (colok) {
        pre(i, o, col, a, s[u], d);
      } else {
#pragma unroll
        for (int g = 0; g < Pre::F_DST; ++g) d[g] = zero;
      }
#pragma unroll
      for (int g = 0; g < Pre::F_DST; ++g) bufA[(size_t)j * lines + g * ct + c] = d[g];
    }
  }
  __syncthreads();
  axis_transform_store<T, INV, Pre::F_DST, WIDE, FP>(a, bufA, bufB, tw, o, c0);
}

// TMA-staged axis pass for passes that read their rows unchanged (PreCopy,
// identity row map, in_rows = L): one bulk tensor copy per box of rows lands
// the tile [row][col] directly in the transform buffer.  map: a 4-D view
// (columns, 1, rows, outer index) of a.in; nbox boxes of L/nbox rows.
// A copy that does not complete within the poll limit raises *status and the
// CTA writes NaN in place of its tile (after waiting again, bounded, for the
// copy to land).
template <typename T, bool INV, int FP = 0>
__global__ void __launch_bounds__(256) axis_pass_tma_kernel(AxisArgs<T> a, const __grid_constant__ CUtensorMap map,
                                                            int nbox, int* status) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ __align__(8) uint64_t mbar;
  __shared__ int timed_out;
  Cx<T>* tw = reinterpret_cast<Cx<T>*>(smem_raw);
  const int L = a.plan.L;
  const int ct = a.col_tile;
  Cx<T>* bufA = tma_buf<T>(smem_raw, L);
  Cx<T>* bufB = bufA + (size_t)L * ct;
  const int o = blockIdx.y;
  const int c0 = blockIdx.x * ct;
  const uint32_t mb = tma::smem_u32(&mbar);
  pdl_trigger();
  if (threadIdx.x == 0) {
    tma::mbar_init(mb, 1);
    timed_out = 0;
  }
  stage_twiddles(tw, a.tw, a.plan);
  __syncthreads();
  pdl_wait();
  const int rows = L / nbox;
  if (threadIdx.x == 0 &&
      !tma_issue<T>(&map, bufA, (size_t)rows * ct, nbox, rows, c0 * (int)(sizeof(Cx<T>) / 4), o, mb,
                    (uint32_t)((size_t)L * ct * sizeof(Cx<T>))))
    timed_out = 2;  // nothing issued: the barrier's phase will not complete
  __syncthreads();
  if (timed_out == 0 && !tma::mbar_wait(mb, 0, tma::kWaitPolls)) timed_out = 1;
  __syncthreads();
  if (timed_out) {
    if (threadIdx.x == 0) {
      atomicExch(status, timed_out);
      if (timed_out == 1) tma::mbar_wait(mb, 0, tma::kWaitPolls);
    }
    __syncthreads();
    for (int l = threadIdx.x; l < L * ct; l += blockDim.x) bufA[l] = mk<T>(nan_of<T>(), nan_of<T>());
    __syncthreads();
  }
  axis_transform_store<T, INV, 1, false, FP>(a, bufA, bufB, tw, o, c0);
}

// ---------------------------------------------------------------------------
// Two-pass axis transform with global memory on both sides.  For a compiled
// schedule of exactly two radices (L = R1 R2) the first Stockham pass loads
// its R1 elements of a line straight from the input rows (the Pre functor
// forms the line's field on load: `field`), and the second stores its R2
// results straight to the output rows; the only shared-memory traffic is the
// exchange between the passes (one store and one load per element instead of
// the staged tile's six) and the only barrier is the one between them.
// Items walk the lines fast (line = field * ct + column), so consecutive
// threads touch consecutive columns in global memory and consecutive lines
// in the exchange buffer.  smem = L twiddles + L * F * ct elements.
template <typename T, bool INV, class Pre, int FP>
__device__ __forceinline__ void axis_rr_body(const AxisArgs<T>& a, const Pre& pre, int bx, int by) {
  using FPl = FixedPlan<FP>;
  constexpr int L = FPl::L, R1 = FPl::Radices::A, R2 = FPl::Radices::B;
  static_assert(FPl::Radices::NP == 2 && R1 * R2 == L, "two-pass schedules only");
  constexpr int F = Pre::F_DST, NB1 = L / R1, NB2 = L / R2;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Cx<T>* tw = reinterpret_cast<Cx<T>*>(smem_raw);
  const int ct = a.col_tile, lines = F * ct;
  Cx<T>* X = tw + L;
  const int o = by, c0 = bx * ct;
  const Cx<T> zero = mk<T>(0, 0);
  pdl_trigger();
  stage_twiddles(tw, a.tw, a.plan);
  pdl_wait();
  const Cx<T>* inb = a.in + (long long)o * a.in_ostride;
  for (Walk2 w(lines); w.s < NB1; w.next()) {
    const int line = w.f, j1 = w.s;
    const int g = line / ct, col = c0 + (line - g * ct);
    Cx<T> v[R1];
#pragma unroll
    for (int r = 0; r < R1; ++r) {
      const int i = row_of(a.in_map, j1 + r * NB1, a.in_rows);
      v[r] = (i >= 0 && col < a.ncols) ? pre.field(g, i, o, col, a, inb) : zero;
    }
    small_dft<T, R1, INV>(v);
#pragma unroll
    for (int r = 0; r < R1; ++r) X[(size_t)(j1 * R1 + r) * lines + line] = v[r];
  }
  __syncthreads();
  Cx<T>* outb = a.out + (long long)o * a.out_ostride;
  for (Walk2 w(lines); w.s < NB2; w.next()) {
    const int line = w.f, j2 = w.s;
    const int g = line / ct, col = c0 + (line - g * ct);
    const int k = j2 % R1;
    Cx<T> v[R2];
#pragma unroll
    for (int r = 0; r < R2; ++r) v[r] = X[(size_t)(j2 + r * NB2) * lines + line];
    // twiddles W_L^{r k} (sub-transform length R1: the table's stride L / (R1 R2) is 1)
#pragma unroll
    for (int r = 1; r < R2; ++r) {
      Cx<T> t = tw[r * k];
      if (INV) t.y = -t.y;
      v[r] = cmul(v[r], t);
    }
    small_dft<T, R2, INV>(v);
    if (col < a.ncols) {
#pragma unroll
      for (int r = 0; r < R2; ++r) {
        const int i = row_of(a.out_map, (j2 - k) * R2 + k + r * R1, a.out_rows);
        if (i >= 0) outb[g * a.out_fstride + i * a.out_rstride + col] = a.scale * v[r];
      }
    }
  }
  // output rows the map leaves without a position are zero
  const int zlo = a.out_map.lo, zhi = min(a.out_map.hi, a.out_rows);
  for (int t = threadIdx.x; zlo < zhi && t < (zhi - zlo) * lines; t += blockDim.x) {
    const int line = t % lines, i = zlo + t / lines;
    const int g = line / ct, col = c0 + (line - g * ct);
    if (col < a.ncols) outb[g * a.out_fstride + i * a.out_rstride + col] = zero;
  }
}

template <typename T, bool INV, class Pre, int FP>
__global__ void __launch_bounds__(256) axis_pass_rr_kernel(AxisArgs<T> a, Pre pre) {
  axis_rr_body<T, INV, Pre, FP>(a, pre, blockIdx.x, blockIdx.y);
}

// grid = (ceil(ncols/col_tile), nouter)
template <typename T, bool INV, class Pre, bool WIDE = false, int FP = 0>
__global__ void __launch_bounds__(256) axis_pass_kernel(AxisArgs<T> a, Pre pre) {
  axis_pass_body<T, INV, Pre, WIDE, FP>(a, pre, blockIdx.x, blockIdx.y);
}

// Batched: grid = (ceil(ncols/col_tile), nouter, runs); run blockIdx.z takes
// its arguments from A[z] and pre[z] (same tile shape for every run).
template <typename T, bool INV, class Pre, bool WIDE, int FP = 0>
__global__ void __launch_bounds__(256) axis_pass_batch(const AxisArgs<T>* __restrict__ A, const Pre* __restrict__ pre) {
  axis_pass_body<T, INV, Pre, WIDE, FP>(A[blockIdx.z], pre[blockIdx.z], blockIdx.x, blockIdx.y);
}

// ---------------------------------------------------------------------------
template <typename T>
struct ZArgs {
  const Cx<T>* in[kMaxZFields];  // per input field: pencil p at in[f] + p*in_pstride[f]
  long long in_pstride[kMaxZFields];
  int in_kz[kMaxZFields];  // stored k3 entries (0..kz-1); higher k3 are zero
  Cx<T>* out[kMaxZFields];
  long long out_pstride[kMaxZFields];
  int out_kz;  // retained k3 entries on output
  long long npencils;
  int ppc;  // pencils per CTA
  T fac;    // physical normalisation after the inverse transform
  FFTPlan plan;
  const Cx<T>* tw;
  unsigned char dz[kMaxZFields];  // 1: input field f enters as i*k3 times the stored spectrum (a d/dz)
  const double* k3;               // k3 wavenumbers of the stored entries (for dz)
};

// Pre functors may leave derivatives along z to the z-pass: Pre::Z_DERIVED
// extra z-pass inputs, Pre::zsrc(f, src, der) maps z-pass input f to the
// stored field src, differentiated along z when der.
template <class P, class = void>
struct pre_z_derived {
  static constexpr int value = 0;
};
template <class P>
struct pre_z_derived<P, decltype((void)P::Z_DERIVED, void())> {
  static constexpr int value = P::Z_DERIVED;
};
// Fields after the y-inverse pass (Pre::F_B; default: the x pass's F_DST) and
// the y-inverse pass's own Pre (Pre::YPass; default: a copy).
template <class P, class = void>
struct pre_b_fields {
  static constexpr int value = P::F_DST;
};
template <class P>
struct pre_b_fields<P, decltype((void)P::F_B, void())> {
  static constexpr int value = P::F_B;
};
// groups: outer groups of the y pass (x rows each); in_fields / out_fields:
// the pass's field strides in fields (0: one field per CTA, folded into the
// outer index)
template <typename T, class P, class = void>
struct pre_ypass {
  using type = PreCopy<T>;
  static constexpr int groups = pre_b_fields<P>::value, in_fields = 0, out_fields = 0;
};
template <typename T, class P>
struct pre_ypass<T, P, decltype((void)sizeof(typename P::YPass), void())> {
  using type = typename P::YPass;
  static constexpr int groups = type::GROUPS, in_fields = type::IN_FIELDS, out_fields = type::OUT_FIELDS;
};

// Line stride of the z-pass buffers: the (even) transform length padded to
// 7 modulo 16 elements.  The transforms walk the lines fast (psb_fft.cuh), so
// a half-warp touches one position of 16 consecutive lines -- distinct banks
// for any odd stride -- or, with 24 or 12 lines, the tail lines at j and the
// first lines at j + 1: with a stride of 7 (mod 16) those two sets share at
// most one or two banks (a stride of 1 would share seven).  At P = 4 the
// field stride P*LS = 28 (mod 32) words also keeps the MLP's feature gathers
// (8 rows x 4 features per warp instruction) on 32 distinct banks.
__host__ __device__ constexpr int zline(int M) { return M + (((7 - M) % 16) + 16) % 16; }

// Shared memory of one z-pass CTA: twiddles, two buffers of
// nl = ceil(fmax*P/2) packed lines of length M at stride zline(M), and the
// Phys extra (16-byte aligned: M is even).
template <typename T>
__host__ inline size_t zpass_smem_bytes(int fmax, int P, int M, size_t extra) {
  return (size_t)(M + 2 * (size_t)((fmax * P + 1) / 2) * zline(M)) * sizeof(Cx<T>) + extra;
}

// Transform of the z-pass's contiguous lines: the plan's schedule (FP = 0) or
// the compiled-in schedule FP (which must equal the plan's).
template <typename T, bool INV, bool WIDE, int FP>
__device__ __forceinline__ Cx<T>* zfft(Cx<T>* a, Cx<T>* b, const FFTPlan& p, const Cx<T>* tw, int nlines) {
  if constexpr (FP == 0)
    return block_fft<T, INV, WIDE>(a, b, p, tw, nlines, zline(p.L), 1, nlines >= 8);
  else
    return FixedPlan<FP>::template run<T, INV>(a, b, tw, nlines, zline(p.L));
}

// Per-CTA staging of the z-pass: the twiddle table and the Phys extra (the
// MLP's fragment-ordered weights).  Done once per CTA, before its first tile.
template <typename T, class Phys>
__device__ __forceinline__ void zpass_setup(const ZArgs<T>& a, const Phys& phys) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Cx<T>* tw = reinterpret_cast<Cx<T>*>(smem_raw);
  stage_twiddles(tw, a.tw, a.plan);
  if constexpr (phys_is_block<Phys>::value) {
    constexpr int FMAX = Phys::F_IN > Phys::F_OUT ? Phys::F_IN : Phys::F_OUT;
    const int nl = (FMAX * a.ppc + 1) / 2;
    phys.setup(reinterpret_cast<unsigned char*>(tw + a.plan.L + (size_t)2 * nl * zline(a.plan.L)));
  }
}

// The physics of a z-pass tile: physical fields R (F_IN real lines of P
// pencils, packed two per complex line at stride LS) -> the F_OUT results W in
// the same packing.  Block physics (the tensor-core MLP) runs over the CTA's
// points; pointwise physics calls Phys per point.  The last CTA may hold
// fewer than P pencils: its missing pencils produce zeros.
template <typename T, class Phys>
__device__ __forceinline__ void zpass_physics(const ZArgs<T>& a, const Phys& phys, const Cx<T>* R, Cx<T>* W, int P,
                                              int M, int LS, long long p0, unsigned char* extra) {
  constexpr int FI = Phys::F_IN, FO = Phys::F_OUT;
  const int nout = (FO * P + 1) / 2;
  if constexpr (phys_is_block<Phys>::value) {
    // block-cooperative physics (a tensor-core MLP over the CTA's points)
    phys.block(R, W, P, M, LS, a.fac, p0, a.npencils, extra);
    if ((FO * P) & 1) {
      for (int z = threadIdx.x; z < M; z += blockDim.x) reinterpret_cast<T*>(W + (size_t)(nout - 1) * LS + z)[1] = (T)0;
    }
  } else {
    // pointwise physics; the last CTA may hold fewer than P pencils
    for (Walk2 w(M); w.s < P; w.next()) {
      const int z = w.f, p = w.s;
      T vin[FI > 0 ? FI : 1], vout[FO > 0 ? FO : 1];
#pragma unroll
      for (int f = 0; f < FI; ++f) {
        const int r = f * P + p;
        const Cx<T> v = R[(size_t)(r >> 1) * LS + z];
        vin[f] = a.fac * ((r & 1) ? v.y : v.x);
      }
      if (p0 + p < a.npencils) {
        phys(p0 + p, z, vin, vout);
      } else {
#pragma unroll
        for (int g = 0; g < FO; ++g) vout[g] = (T)0;
      }
#pragma unroll
      for (int g = 0; g < FO; ++g) {
        const int r = g * P + p;
        T* w = reinterpret_cast<T*>(W + (size_t)(r >> 1) * LS + z);
        w[r & 1] = vout[g];
      }
      if ((FO * P) & 1) {  // odd count: the last packed line has no partner
        if (p == P - 1) reinterpret_cast<T*>(W + (size_t)(nout - 1) * LS + z)[1] = (T)0;
      }
    }
  }
}

// One tile of the z-pass: pencils bx*ppc ..; smem = zpass_smem_bytes, staged
// by zpass_setup.  Ends with the results stored; the caller synchronises
// before the CTA's next tile reuses the buffers.
template <typename T, class Phys, bool WIDE = false, int FP = 0>
__device__ __forceinline__ void zpass_tile(const ZArgs<T>& a, const Phys& phys, int bx) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Cx<T>* tw = reinterpret_cast<Cx<T>*>(smem_raw);
  constexpr int FI = Phys::F_IN, FO = Phys::F_OUT;
  const int M = a.plan.L;
  const int P = a.ppc;
  constexpr int FMAX = FI > FO ? FI : FO;
  const int nl = (FMAX * P + 1) / 2;
  const int LS = zline(M);
  Cx<T>* X = tw + M;
  Cx<T>* Y = X + (size_t)nl * LS;
  unsigned char* extra = reinterpret_cast<unsigned char*>(Y + (size_t)nl * LS);
  const long long p0 = (long long)bx * P;
  const int lp = __ffs(P) - 1;
  const Cx<T> zero = mk<T>(0, 0);
  const int half = M / 2;
  Cx<T>* R = X;
  if constexpr (FI > 0) {
    const int nin = (FI * P + 1) / 2;
    // pack pairs of Hermitian half-spectra: Z = A + iB, Z[M-k] = conj(A_k) + i conj(B_k);
    // the k=0 and k=M/2 terms keep their real parts only (c2r convention).  The
    // items k = 0..M/2 of every packed line write all M positions of the line
    // (zero where k is beyond the stored k3 range), so nothing needs clearing.
    if ((P & 1) == 0) {
      // P even: packed line c holds pencils p, p+1 (p = 2 (c mod P/2)) of
      // field f = c / (P/2); one warp per line, lanes along k; a warp loads
      // U of its lines before storing any, so their reads overlap
      constexpr int U = 4;
      const int hp = P >> 1, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
      for (int cb = threadIdx.x >> 5; cb < nin; cb += U * nw) {
        const Cx<T>* src[U];
        long long ps[U];
        int kz[U];
        bool oka[U], okb[U], dz[U];
        int kzmax = 0;
        bool anydz = false;
#pragma unroll
        for (int u = 0; u < U; ++u) {
          const int c = cb + u * nw;
          const int f = c < nin ? c / hp : 0, p = 2 * (c - f * hp);
          const long long pa = p0 + p;
          kz[u] = c < nin ? min(a.in_kz[f], half + 1) : 0;
          oka[u] = pa < a.npencils;
          okb[u] = pa + 1 < a.npencils;
          ps[u] = a.in_pstride[f];
          src[u] = a.in[f] + (oka[u] ? pa * ps[u] : 0);
          dz[u] = c < nin && a.dz[f] != 0;
          anydz |= dz[u];
          kzmax = max(kzmax, kz[u]);
        }
        for (int kb = 0; kb < kzmax; kb += 32) {
          const int k = kb + lane;
          Cx<T> A[U], B[U];
#pragma unroll
          for (int u = 0; u < U; ++u) {
            A[u] = (k < kz[u] && oka[u]) ? src[u][k] : zero;
            B[u] = (k < kz[u] && okb[u]) ? src[u][ps[u] + k] : zero;
          }
          // k3 (a table of every stored k3) exists whenever a line is a z derivative
          const T kk = (anydz && k < kzmax) ? (T)a.k3[k] : (T)0;
#pragma unroll
          for (int u = 0; u < U; ++u) {
            if (k >= kz[u]) continue;
            Cx<T> va = A[u], vb = B[u];
            if (dz[u]) {
              va = mk<T>(-kk * va.y, kk * va.x);
              vb = mk<T>(-kk * vb.y, kk * vb.x);
            }
            Cx<T>* Z = X + (size_t)(cb + u * nw) * LS;
            if (k == 0 || k == half) {
              Z[k] = mk<T>(va.x, vb.x);
            } else {
              Z[k] = mk<T>(va.x - vb.y, va.y + vb.x);
              Z[M - k] = mk<T>(va.x + vb.y, vb.x - va.y);
            }
          }
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
          const int c = cb + u * nw;
          if (c >= nin) continue;
          Cx<T>* Z = X + (size_t)c * LS;
          for (int k = kz[u] + lane; k <= M - kz[u]; k += 32) Z[k] = zero;
        }
      }
    } else
    for (Walk2 w(half + 1); w.s < nin; w.next()) {
      const int k = w.f, c = w.s;
      Cx<T> A = zero, B = zero;
#pragma unroll 1
      for (int part = 0; part < 2; ++part) {
        const int r = 2 * c + part;
        if (r >= FI * P) break;
        int f, p;
        split_line(r, P, lp, f, p);
        const long long pen = p0 + p;
        if (pen >= a.npencils || k >= a.in_kz[f]) continue;
        Cx<T> v = a.in[f][pen * a.in_pstride[f] + k];
        if (a.dz[f]) {
          const T kk = (T)a.k3[k];
          v = mk<T>(-kk * v.y, kk * v.x);
        }
        if (part == 0) A = v; else B = v;
      }
      Cx<T>* Z = X + (size_t)c * LS;
      if (k == 0 || k == half) {
        Z[k] = mk<T>(A.x, B.x);
      } else {
        Z[k] = mk<T>(A.x - B.y, A.y + B.x);
        Z[M - k] = mk<T>(A.x + B.y, B.x - A.y);
      }
    }
    __syncthreads();
    R = zfft<T, true, WIDE, FP>(X, Y, a.plan, tw, nin);
  }
  Cx<T>* W = (R == X) ? Y : X;
  const int nout = (FO * P + 1) / 2;
  zpass_physics<T, Phys>(a, phys, R, W, P, M, LS, p0, extra);
  if constexpr (FO > 0) {
    __syncthreads();
    Cx<T>* R2 = zfft<T, false, WIDE, FP>(W, R, a.plan, tw, nout);
    // unpack: A_k = (Z_k + conj(Z_{M-k}))/2, B_k = (Z_k - conj(Z_{M-k}))/(2i)
    const int kzo = a.out_kz;
    if ((P & 1) == 0) {
      // P even: one warp per packed line (field g, pencils p and p+1), lanes along k
      const int hp = P >> 1, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
      for (int c = threadIdx.x >> 5; c < nout; c += nw) {
        const int g = c / hp, p = 2 * (c - g * hp);
        const long long pa = p0 + p;
        const bool oka = pa < a.npencils, okb = pa + 1 < a.npencils;
        const Cx<T>* Z = R2 + (size_t)c * LS;
        Cx<T>* dst = a.out[g] + pa * a.out_pstride[g];
        const long long ps = a.out_pstride[g];
        for (int k = lane; k < kzo; k += 32) {
          const Cx<T> zk = Z[k], zm = Z[k == 0 ? 0 : M - k];
          if (oka) dst[k] = mk<T>((T)0.5 * (zk.x + zm.x), (T)0.5 * (zk.y - zm.y));
          if (okb) dst[ps + k] = mk<T>((T)0.5 * (zk.y + zm.y), (T)0.5 * (zm.x - zk.x));
        }
      }
    } else
    for (Walk2 w(kzo); w.s < nout; w.next()) {
      const int k = w.f, c = w.s;
      const Cx<T>* Z = R2 + (size_t)c * LS;
      const Cx<T> zk = Z[k], zm = Z[k == 0 ? 0 : M - k];
#pragma unroll
      for (int part = 0; part < 2; ++part) {
        const int r = 2 * c + part;
        if (r >= FO * P) break;
        int g, p;
        split_line(r, P, lp, g, p);
        const long long pen = p0 + p;
        if (pen >= a.npencils) continue;
        const Cx<T> v = part == 0 ? mk<T>((T)0.5 * (zk.x + zm.x), (T)0.5 * (zk.y - zm.y))
                                  : mk<T>((T)0.5 * (zk.y + zm.y), (T)0.5 * (zm.x - zk.x));
        a.out[g][pen * a.out_pstride[g] + k] = v;
      }
    }
  }
}

// One CTA, one tile (the batched kernel's unit).
template <typename T, class Phys, bool WIDE = false, int FP = 0>
__device__ __forceinline__ void zpass_body(const ZArgs<T>& a, const Phys& phys, int bx) {
  pdl_trigger();
  zpass_setup<T, Phys>(a, phys);
  pdl_wait();
  zpass_tile<T, Phys, WIDE, FP>(a, phys, bx);
}

// Tiles bx = blockIdx.x, + gridDim.x, ... < ceil(npencils/ppc): any grid
// size covers every tile; a grid of (resident CTAs per SM) x SMs stages the
// twiddles and the Phys extra once per CTA instead of once per tile.
// FP: compiled-in transform schedule (FixedPlan id) equal to a.plan, or 0.
template <typename T, class Phys, bool WIDE = false, int FP = 0>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 3 : 1) zpass_kernel(ZArgs<T> a, Phys phys) {
  pdl_trigger();
  zpass_setup<T, Phys>(a, phys);
  pdl_wait();
  const long long ntiles = (a.npencils + a.ppc - 1) / a.ppc;
  for (long long bx = blockIdx.x; bx < ntiles; bx += gridDim.x) {
    zpass_tile<T, Phys, WIDE, FP>(a, phys, (int)bx);
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// z-pass with global memory on both sides of its transforms.  For a compiled
// two-pass schedule (R1, R2) with R2 = 16 or 8 the inverse runs (R1, R2) and
// the forward (R2, R1), so that both transforms' global-facing passes have R2
// items per packed line, one per lane of an aligned R2-lane group:
//  * inverse pass 1 loads its R1 elements of a packed line, positions
//    j + R2 r, straight from the two pencils' stored spectra (Hermitian
//    packing Z = A + iB, z derivatives i k3 u formed on load): the lanes of a
//    group read R2 consecutive k3 of each pencil;
//  * forward pass 2 hands its R1 results, positions j + R2 r, straight to the
//    unpack A_q = (Z_q + conj Z_{M-q})/2, B_q = (Z_q - conj Z_{M-q})/(2i).
//    For q = j + R2 r (j > 0), M - q = (R2 - j) + R2 (R1 - 1 - r): register
//    R1 - 1 - r of lane R2 - j of the same group, fetched with a warp shuffle
//    (lane 0 pairs with itself: M - R2 r is its register (R1 - r) mod R1).
// A packed line's shared-memory traffic is the exchange inside each transform
// and the physics' reads and writes; the packed spectra never pass through
// shared memory.  P must be even (packed lines pair pencils p, p+1 of one
// field).  smem and staging as zpass_kernel (zpass_smem_bytes, zpass_setup).
template <int FP>
struct zrr_plan {
  using Pl = FixedPlan<FP>;
  static constexpr int R1 = Pl::Radices::A, R2 = Pl::Radices::B, REV = fixed_plan_reversed(FP);
  static constexpr bool value = Pl::Radices::NP == 2 && REV != 0 && (R2 == 16 || R2 == 8);
};

// The default schedule of a register-direct z pass of length p.L: the
// compiled two-pass order (p.L / 16, 16) when there is one (48, 96, 192).
__host__ inline bool zrr_default_plan(FFTPlan& p) {
  for (const FixedDesc& d : kFixedDescs)
    if (d.L == p.L && d.n == 2 && d.r[1] == 16 && fixed_plan_reversed(d.id) != 0) {
      p.npass = 2;
      p.radix[0] = d.r[0];
      p.radix[1] = d.r[1];
      for (int s = 2; s < kMaxPasses; ++s) p.radix[s] = 0;
      return true;
    }
  return false;
}

template <typename T, class Phys, int FP>
__device__ __forceinline__ void zpass_rr_tile(const ZArgs<T>& a, const Phys& phys, int bx) {
  static_assert(zrr_plan<FP>::value, "two-pass schedule (R1, 16 or 8) with its reverse compiled in");
  constexpr int M = FixedPlan<FP>::L, R1 = zrr_plan<FP>::R1, R2 = zrr_plan<FP>::R2;
  constexpr int FI = Phys::F_IN, FO = Phys::F_OUT;
  static_assert(FI > 0 && FO > 0, "a z-pass with inputs and outputs");
  constexpr int FMAX = FI > FO ? FI : FO;
  constexpr int half = M / 2, LS = zline(M);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Cx<T>* tw = reinterpret_cast<Cx<T>*>(smem_raw);
  const int P = a.ppc, hp = P >> 1;
  const int nl = FMAX * hp;
  Cx<T>* X = tw + M;
  Cx<T>* Y = X + (size_t)nl * LS;
  unsigned char* extra = reinterpret_cast<unsigned char*>(Y + (size_t)nl * LS);
  const long long p0 = (long long)bx * P;
  const Cx<T> zero = mk<T>(0, 0);
  const int nin = FI * hp, nout = FO * hp;
  const int gpc = blockDim.x / R2;  // line groups per CTA
  const int j = threadIdx.x % R2, grp = threadIdx.x / R2;
  // ---- inverse pass 1: packed spectra -> registers -> radix R1 -> X
  for (int c = grp; c < nin; c += gpc) {
    const int f = c / hp, p = 2 * (c - f * hp);
    const long long pa = p0 + p;
    const bool oka = pa < a.npencils, okb = pa + 1 < a.npencils;
    const long long ps = a.in_pstride[f];
    const Cx<T>* src = a.in[f] + (oka ? pa * ps : 0);
    const int kz = min(a.in_kz[f], half + 1);
    Cx<T> va[R1], vb[R1];
#pragma unroll
    for (int r = 0; r < R1; ++r) {
      const int n = j + R2 * r;
      const int m = n <= half ? n : M - n;
      va[r] = (m < kz && oka) ? src[m] : zero;
      vb[r] = (m < kz && okb) ? src[ps + m] : zero;
    }
    const bool dz = a.dz[f] != 0;
    Cx<T> v[R1];
#pragma unroll
    for (int r = 0; r < R1; ++r) {
      const int n = j + R2 * r;
      const bool lo = n <= half;
      const int m = lo ? n : M - n;
      Cx<T> A = va[r], B = vb[r];
      if (dz) {
        const T kk = m < kz ? (T)a.k3[m] : (T)0;
        A = mk<T>(-kk * A.y, kk * A.x);
        B = mk<T>(-kk * B.y, kk * B.x);
      }
      if (lo)
        v[r] = (n == 0 || n == half) ? mk<T>(A.x, B.x) : mk<T>(A.x - B.y, A.y + B.x);
      else
        v[r] = mk<T>(A.x + B.y, B.x - A.y);
    }
    small_dft<T, R1, true>(v);
    Cx<T>* Z = X + (size_t)c * LS + j * R1;
#pragma unroll
    for (int r = 0; r < R1; ++r) Z[r] = v[r];
  }
  __syncthreads();
  // ---- inverse pass 2 (X -> Y), the physics (Y -> X), forward pass 1 (X -> Y)
  if (nin >= 8)
    stockham_pass_c<T, R2, true, M, R1, true>(X, Y, tw, nin, LS);
  else
    stockham_pass_c<T, R2, true, M, R1, false>(X, Y, tw, nin, LS);
  __syncthreads();
  zpass_physics<T, Phys>(a, phys, Y, X, P, M, LS, p0, extra);
  __syncthreads();
  if (nout >= 8)
    stockham_pass_c<T, R2, false, M, 1, true>(X, Y, tw, nout, LS);
  else
    stockham_pass_c<T, R2, false, M, 1, false>(X, Y, tw, nout, LS);
  __syncthreads();
  // ---- forward pass 2: Y -> radix R1 (sub-transform length R2) -> unpack -> global.
  // Every lane of a warp runs every round (the shuffles need the whole warp);
  // lanes past the last line compute on zeros and store nothing.
  const int lane = threadIdx.x & 31;
  const int partner = (lane & ~(R2 - 1)) | ((R2 - j) & (R2 - 1));
  const int kzo = a.out_kz;
  for (int cb = 0; cb < nout; cb += gpc) {
    const int c = cb + grp;
    const bool act = c < nout;
    Cx<T> v[R1];
#pragma unroll
    for (int r = 0; r < R1; ++r) v[r] = act ? Y[(size_t)c * LS + j + R2 * r] : zero;
    // twiddles W_M^{r j} (sub-transform length R2: the table's stride is 1)
#pragma unroll
    for (int r = 1; r < R1; ++r) v[r] = cmul(v[r], tw[r * j]);
    small_dft<T, R1, false>(v);
    const int g = act ? c / hp : 0, p = 2 * (c - g * hp);
    const long long pa = p0 + p;
    const bool oka = act && pa < a.npencils, okb = act && pa + 1 < a.npencils;
    const long long ps = a.out_pstride[g];
    Cx<T>* dst = a.out[g] + (oka ? pa * ps : 0);
#pragma unroll
    for (int r = 0; r <= R1 / 2; ++r) {
      if (R2 * r >= kzo) break;  // uniform over the warp
      Cx<T> pv;
      pv.x = __shfl_sync(0xffffffffu, v[R1 - 1 - r].x, partner);
      pv.y = __shfl_sync(0xffffffffu, v[R1 - 1 - r].y, partner);
      const Cx<T> zk = v[r];
      const Cx<T> zm = j == 0 ? v[(R1 - r) % R1] : pv;
      const int q = j + R2 * r;
      if (q < kzo) {
        if (oka) dst[q] = mk<T>((T)0.5 * (zk.x + zm.x), (T)0.5 * (zk.y - zm.y));
        if (okb) dst[ps + q] = mk<T>((T)0.5 * (zk.y + zm.y), (T)0.5 * (zm.x - zk.x));
      }
    }
  }
}

// Persistent register-direct z-pass (tiles as zpass_kernel).
template <typename T, class Phys, int FP>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 3 : 1) zpass_rr_kernel(ZArgs<T> a, Phys phys) {
  pdl_trigger();
  zpass_setup<T, Phys>(a, phys);
  pdl_wait();
  const long long ntiles = (a.npencils + a.ppc - 1) / a.ppc;
  for (long long bx = blockIdx.x; bx < ntiles; bx += gridDim.x) {
    zpass_rr_tile<T, Phys, FP>(a, phys, (int)bx);
    __syncthreads();
  }
}

// Batched z passes, persistent: items (run, tile) = (it / ntiles, it % ntiles)
// for it = blockIdx.x, + gridDim.x, ... < runs * ntiles (run-major, so that a
// CTA's consecutive items share a run); a CTA stages the twiddles and the
// Phys extra (the network's weights) again only when its run changes.  Every
// run of a batch has the same shape (npencils, ppc, plan).
template <typename T, class Phys, bool RR, bool WIDE, int FP>
__device__ __forceinline__ void zpass_batch_body(const ZArgs<T>* __restrict__ A, const Phys* __restrict__ phys,
                                                 int runs) {
  pdl_trigger();
  const long long ntiles = (A[0].npencils + A[0].ppc - 1) / A[0].ppc;
  const long long total = ntiles * runs;
  int staged = -1;
  for (long long it = blockIdx.x; it < total; it += gridDim.x) {
    const int r = (int)(it / ntiles);
    const int bx = (int)(it - (long long)r * ntiles);
    if (r != staged) {
      zpass_setup<T, Phys>(A[r], phys[r]);
      if (staged < 0) pdl_wait();
      staged = r;
    }
    if constexpr (RR)
      zpass_rr_tile<T, Phys, FP>(A[r], phys[r], bx);
    else
      zpass_tile<T, Phys, WIDE, FP>(A[r], phys[r], bx);
    __syncthreads();  // the next item (or the next run's staging) reuses the shared memory
  }
}

template <typename T, class Phys, int FP>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 3 : 1)
    zpass_rr_batch(const ZArgs<T>* __restrict__ A, const Phys* __restrict__ phys, int runs) {
  zpass_batch_body<T, Phys, true, false, FP>(A, phys, runs);
}

template <typename T, class Phys, bool WIDE, int FP = 0>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 3 : 1)
    zpass_batch(const ZArgs<T>* __restrict__ A, const Phys* __restrict__ phys, int runs) {
  zpass_batch_body<T, Phys, false, WIDE, FP>(A, phys, runs);
}

// Closures whose z-pass is compiled with the fixed schedules (the 3/2-padded
// Navier-Stokes closures: DNS products, Smagorinsky, learned); FP64 only with
// the default schedule of each length.
template <class Phys>
struct phys_fixed_fft {
  static constexpr bool value = false;
};
template <typename T, int FP>
struct fixed_plan_compiled {
  static constexpr bool value = sizeof(T) == 4 || FP == 1 || FP == 4 || FP == 7;
};

// ---------------------------------------------------------------------------
template <typename T>
struct XEpiArgs {
  const Cx<T>* in;  // (F, L rows, n2, kz)
  long long in_fstride, in_rstride, in_ostride;
  int n1, n2, n3h;  // spectral output dims (rows, outer, k3 count)
  int kz;           // k3 < kz come from the transform, the rest have zero products
  int col_tile;
  RowMap out_map;  // spectral row -> FFT position
  int main_blocks;
  FFTPlan plan;
  const Cx<T>* tw;
};

// The blocks past main_blocks: columns kz..n3h-1 carry no products.
template <typename T, class Epi>
__device__ __forceinline__ void xfwd_epi_extra(const XEpiArgs<T>& a, const Epi& epi, int bx, int gx) {
  constexpr int F = Epi::F_IN;
  Cx<T> P[F];
  const Cx<T> zero = mk<T>(0, 0);
  const int ncz = a.n3h - a.kz;
  const long long tot = (long long)a.n1 * a.n2 * ncz;
  const int nextra = gx - a.main_blocks;
  for (long long idx = (long long)(bx - a.main_blocks) * blockDim.x + threadIdx.x; idx < tot;
       idx += (long long)nextra * blockDim.x) {
    const int c = (int)(idx % ncz);
    const long long t = idx / ncz;
    const int i2 = (int)(t % a.n2), i1 = (int)(t / a.n2);
#pragma unroll
    for (int f = 0; f < F; ++f) P[f] = zero;
    epi(i1, i2, a.kz + c, P);
  }
}

// Transform of a staged tile and the epilogue on its output rows.  Must be
// called by all threads.
template <typename T, class Epi, bool WIDE, int FP>
__device__ __forceinline__ void xfwd_transform_epi(const XEpiArgs<T>& a, const Epi& epi, Cx<T>* bufA, Cx<T>* bufB,
                                                   const Cx<T>* tw, int o, int c0) {
  constexpr int F = Epi::F_IN;
  Cx<T> P[F];
  const Cx<T> zero = mk<T>(0, 0);
  const int ct = a.col_tile;
  const int lines = F * ct;
  const int nt = blockDim.x;
  const int c = threadIdx.x % ct, r0 = threadIdx.x / ct, dr = nt / ct;
  const int col = c0 + c;
  const bool colok = col < a.kz;
  Cx<T>* res = axfft<T, false, WIDE, FP>(bufA, bufB, a.plan, tw, lines);
  // threads past the last full row of columns would repeat a (row, column)
  // (only when ct does not divide the CTA size): the epilogue is not idempotent
  if (!colok || threadIdx.x >= dr * ct) return;
  for (int i1 = r0; i1 < a.n1; i1 += dr) {
    const int j = a.out_map(i1);
#pragma unroll
    for (int f = 0; f < F; ++f) P[f] = j >= 0 ? res[(size_t)j * lines + f * ct + c] : zero;
    epi(i1, o, col, P);
  }
}

// One CTA of the x-forward epilogue pass: block bx of gx = main_blocks + extra;
// main block b -> (col tile b % ntile, outer b / ntile)
template <typename T, class Epi, bool WIDE = false, int FP = 0>
__device__ __forceinline__ void xfwd_epi_body(const XEpiArgs<T>& a, const Epi& epi, int bx, int gx) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  constexpr int F = Epi::F_IN;
  const Cx<T> zero = mk<T>(0, 0);
  pdl_trigger();
  if (bx >= a.main_blocks) {
    pdl_wait();
    xfwd_epi_extra<T, Epi>(a, epi, bx, gx);
    return;
  }
  Cx<T>* tw = reinterpret_cast<Cx<T>*>(smem_raw);
  const int L = a.plan.L;
  const int ct = a.col_tile;
  const int lines = F * ct;
  Cx<T>* bufA = tw + L;
  Cx<T>* bufB = bufA + (size_t)L * lines;
  const int ntile = (a.kz + ct - 1) / ct;
  const int o = bx / ntile;
  const int c0 = (bx % ntile) * ct;
  stage_twiddles(tw, a.tw, a.plan);
  pdl_wait();
  const Cx<T>* inb = a.in + (long long)o * a.in_ostride;
  // one column c per thread, rows walked with stride nt/ct (as in the axis pass)
  const int nt = blockDim.x;
  const int c = threadIdx.x % ct, r0 = threadIdx.x / ct, dr = nt / ct;
  const int col = c0 + c;
  const bool colok = col < a.kz;
  // 8 loads in flight per thread before their stores
  for (int t0 = r0; t0 < L * F; t0 += 8 * dr) {
    Cx<T> v[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int t = t0 + u * dr;
      const int j = t / F, f = t - j * F;
      v[u] = (colok && t < L * F) ? inb[f * a.in_fstride + j * a.in_rstride + col] : zero;
    }
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int t = t0 + u * dr;
      if (t >= L * F) break;
      const int j = t / F, f = t - j * F;
      bufA[(size_t)j * lines + f * ct + c] = v[u];
    }
  }
  __syncthreads();
  xfwd_transform_epi<T, Epi, WIDE, FP>(a, epi, bufA, bufB, tw, o, c0);
}

// TMA-staged x-forward epilogue pass: the tile (ct columns x F fields x L
// rows of one outer index) arrives by bulk tensor copies of L/nbox rows each
// through map, a 4-D view (columns, fields, rows, outer index) of a.in.  A
// copy that does not complete within the poll limit raises *status and the
// CTA hands NaN to the epilogue in place of its tile.
template <typename T, class Epi, int FP = 0>
__global__ void __launch_bounds__(256) xfwd_epi_tma_kernel(XEpiArgs<T> a, Epi epi,
                                                           const __grid_constant__ CUtensorMap map, int nbox,
                                                           int* status) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ __align__(8) uint64_t mbar;
  __shared__ int timed_out;
  constexpr int F = Epi::F_IN;
  pdl_trigger();
  if ((int)blockIdx.x >= a.main_blocks) {
    pdl_wait();
    xfwd_epi_extra<T, Epi>(a, epi, blockIdx.x, gridDim.x);
    return;
  }
  Cx<T>* tw = reinterpret_cast<Cx<T>*>(smem_raw);
  const int L = a.plan.L;
  const int ct = a.col_tile;
  const int lines = F * ct;
  Cx<T>* bufA = tma_buf<T>(smem_raw, L);
  Cx<T>* bufB = bufA + (size_t)L * lines;
  const int ntile = (a.kz + ct - 1) / ct;
  const int o = blockIdx.x / ntile;
  const int c0 = (blockIdx.x % ntile) * ct;
  const uint32_t mb = tma::smem_u32(&mbar);
  if (threadIdx.x == 0) {
    tma::mbar_init(mb, 1);
    timed_out = 0;
  }
  stage_twiddles(tw, a.tw, a.plan);
  __syncthreads();
  pdl_wait();
  const int rows = L / nbox;
  if (threadIdx.x == 0 &&
      !tma_issue<T>(&map, bufA, (size_t)rows * lines, nbox, rows, c0 * (int)(sizeof(Cx<T>) / 4), o, mb,
                    (uint32_t)((size_t)L * lines * sizeof(Cx<T>))))
    timed_out = 2;  // nothing issued: the barrier's phase will not complete
  __syncthreads();
  if (timed_out == 0 && !tma::mbar_wait(mb, 0, tma::kWaitPolls)) timed_out = 1;
  __syncthreads();
  if (timed_out) {
    if (threadIdx.x == 0) {
      atomicExch(status, timed_out);
      if (timed_out == 1) tma::mbar_wait(mb, 0, tma::kWaitPolls);
    }
    __syncthreads();
    for (int l = threadIdx.x; l < L * lines; l += blockDim.x) bufA[l] = mk<T>(nan_of<T>(), nan_of<T>());
    __syncthreads();
  }
  xfwd_transform_epi<T, Epi, false, FP>(a, epi, bufA, bufB, tw, o, c0);
}

// The x-forward epilogue pass with a two-pass compiled schedule: the first
// pass loads its elements straight from the input rows, the second writes the
// transformed tile to shared memory for the epilogue (which needs every field
// of a point in one thread).  smem = L twiddles + 2 L F ct elements.
template <typename T, class Epi, int FP>
__global__ void __launch_bounds__(256) xfwd_epi_rr_kernel(XEpiArgs<T> a, Epi epi) {
  using FPl = FixedPlan<FP>;
  constexpr int L = FPl::L, R1 = FPl::Radices::A, R2 = FPl::Radices::B;
  static_assert(FPl::Radices::NP == 2 && R1 * R2 == L, "two-pass schedules only");
  constexpr int F = Epi::F_IN, NB1 = L / R1, NB2 = L / R2;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  pdl_trigger();
  if ((int)blockIdx.x >= a.main_blocks) {
    pdl_wait();
    xfwd_epi_extra<T, Epi>(a, epi, blockIdx.x, gridDim.x);
    return;
  }
  Cx<T>* tw = reinterpret_cast<Cx<T>*>(smem_raw);
  const int ct = a.col_tile, lines = F * ct;
  Cx<T>* X = tw + L;
  Cx<T>* Y = X + (size_t)L * lines;
  const int ntile = (a.kz + ct - 1) / ct;
  const int o = blockIdx.x / ntile;
  const int c0 = (blockIdx.x % ntile) * ct;
  const Cx<T> zero = mk<T>(0, 0);
  stage_twiddles(tw, a.tw, a.plan);
  pdl_wait();
  const Cx<T>* inb = a.in + (long long)o * a.in_ostride;
  for (Walk2 w(lines); w.s < NB1; w.next()) {
    const int line = w.f, j1 = w.s;
    const int f = line / ct, col = c0 + (line - f * ct);
    Cx<T> v[R1];
#pragma unroll
    for (int r = 0; r < R1; ++r)
      v[r] = col < a.kz ? inb[f * a.in_fstride + (j1 + r * NB1) * a.in_rstride + col] : zero;
    small_dft<T, R1, false>(v);
#pragma unroll
    for (int r = 0; r < R1; ++r) X[(size_t)(j1 * R1 + r) * lines + line] = v[r];
  }
  __syncthreads();
  for (Walk2 w(lines); w.s < NB2; w.next()) {
    const int line = w.f, j2 = w.s;
    const int k = j2 % R1;
    Cx<T> v[R2];
#pragma unroll
    for (int r = 0; r < R2; ++r) v[r] = X[(size_t)(j2 + r * NB2) * lines + line];
#pragma unroll
    for (int r = 1; r < R2; ++r) v[r] = cmul(v[r], tw[r * k]);
    small_dft<T, R2, false>(v);
#pragma unroll
    for (int r = 0; r < R2; ++r) Y[(size_t)((j2 - k) * R2 + k + r * R1) * lines + line] = v[r];
  }
  __syncthreads();
  const int nt = blockDim.x;
  const int c = threadIdx.x % ct, r0 = threadIdx.x / ct, dr = nt / ct;
  const int col = c0 + c;
  if (col >= a.kz || threadIdx.x >= dr * ct) return;
  Cx<T> P[F];
  for (int i1 = r0; i1 < a.n1; i1 += dr) {
    const int j = a.out_map(i1);
#pragma unroll
    for (int f = 0; f < F; ++f) P[f] = j >= 0 ? Y[(size_t)j * lines + f * ct + c] : zero;
    epi(i1, o, col, P);
  }
}

// grid = main_blocks + extra
template <typename T, class Epi, bool WIDE = false, int FP = 0>
__global__ void __launch_bounds__(256) xfwd_epi_kernel(XEpiArgs<T> a, Epi epi) {
  xfwd_epi_body<T, Epi, WIDE, FP>(a, epi, blockIdx.x, gridDim.x);
}

// Batched: grid = (main_blocks + extra, runs); run blockIdx.y reads A[y], epi[y].
template <typename T, class Epi, bool WIDE, int FP = 0>
__global__ void __launch_bounds__(256) xfwd_epi_batch(const XEpiArgs<T>* __restrict__ A, const Epi* __restrict__ epi) {
  xfwd_epi_body<T, Epi, WIDE, FP>(A[blockIdx.y], epi[blockIdx.y], blockIdx.x, gridDim.x);
}

}  // namespace psb
