// Tensor-memory-accelerator (TMA) staging of pipeline tiles (sm_100a).
//
// A pass that reads its input rows unchanged (the forward y pass, the x pass
// of the spectral epilogue, the plain inverse y pass) loads a CTA's whole
// tile -- ct contiguous columns x F fields x the rows of one outer index --
// with bulk tensor copies straight into the shared-memory transform buffer,
// instead of a load/store per element through registers.  The tensor map
// covers only this GPU's own memory and the copies carry no cluster
// multicast.
//
// Device side: one elected thread arms an mbarrier with the byte count and
// issues the copies; every thread waits on the barrier's phase with a bounded
// number of polls (a wait that gives up raises the launch's error flag and the
// CTA skips its tile instead of hanging).
// Host side: cuTensorMapEncodeTiled is reached through the runtime's driver
// entry point, so the library does not link against the driver library.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace psb {
namespace tma {

// Polls of an mbarrier before a wait gives up (about a second of spinning).
constexpr uint32_t kWaitPolls = 1u << 24;

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint32_t mbar, int count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar), "r"(count) : "memory");
  // make the initialised barrier visible to the asynchronous (TMA) proxy
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// This thread's arrival, announcing `bytes` of transactions still to land.
__device__ __forceinline__ void mbar_arrive_expect(uint32_t mbar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mbar), "r"(bytes) : "memory");
}

// Wait for phase `parity` to complete, giving up after `limit` polls.
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity, uint32_t limit) {
  for (uint32_t i = 0; i < limit; ++i) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred P1;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t"
        "}\n"
        : "=r"(done)
        : "r"(mbar), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// 4-D tiled bulk copy global -> this CTA's shared memory, completing on mbar.
// Coordinates are element indices (innermost first); the innermost one times
// the element size is a multiple of 16 bytes (the caller keeps it so).
__device__ __forceinline__ void load4d(uint32_t dst, const CUtensorMap* map, int c0, int c1, int c2, int c3,
                                       uint32_t mbar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
      "[%6];" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(mbar)
      : "memory");
}

}  // namespace tma
}  // namespace psb

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
namespace psbh {
namespace tma {

using EncodeFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                              const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                              CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

// cuTensorMapEncodeTiled through the runtime (null when the driver lacks it).
inline EncodeFn encoder() {
  static EncodeFn fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeFn>(p);
    else
      (void)cudaGetLastError();
  }
  return fn;
}

// A 4-D view of complex elements (size esz = 8 or 16 bytes, moved as pairs or
// quadruples of 32-bit words): dims innermost first with element strides of
// the outer three; box sizes in elements.  Returns false when the view breaks
// a TMA rule (base or a stride not a multiple of 16 bytes, a box side above
// 256, an inner box side not a multiple of 16 bytes); the caller then keeps
// the plain loads.
inline bool encode4d(CUtensorMap* m, const void* base, int esz, const long long dims[4], const long long strides[3],
                     const int box[4]) {
  EncodeFn fn = encoder();
  if (!fn) return false;
  if ((reinterpret_cast<uintptr_t>(base) & 15) != 0) return false;
  if (((long long)box[0] * esz) % 16 != 0) return false;
  for (int i = 0; i < 4; ++i)
    if (box[i] < 1 || box[i] > 256 || dims[i] < 1) return false;
  // complex elements as 32-bit words: the innermost dimension counts words
  const int wpe = esz / 4;
  cuuint64_t gd[4] = {(cuuint64_t)dims[0] * wpe, (cuuint64_t)dims[1], (cuuint64_t)dims[2], (cuuint64_t)dims[3]};
  cuuint64_t gs[3];
  for (int i = 0; i < 3; ++i) {
    const long long b = strides[i] * esz;
    if (b % 16 != 0 || b <= 0) return false;
    gs[i] = (cuuint64_t)b;
  }
  cuuint32_t bx[4] = {(cuuint32_t)(box[0] * wpe), (cuuint32_t)box[1], (cuuint32_t)box[2], (cuuint32_t)box[3]};
  if (bx[0] > 256) return false;
  cuuint32_t es[4] = {1, 1, 1, 1};
  const CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, const_cast<void*>(base), gd, gs, bx, es,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                        CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

}  // namespace tma
}  // namespace psbh
