// nb_common.cuh -- shared constants, status codes and sm_100a helpers (TMA bulk
// copies, bulk reductions, mbarriers) for the nipet_b200 kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/nipet_b200.h"

// ---- mMR geometry (reference include/def.h:55-123) ----
#define NB_AW 68516
#define NB_NSBINS 344
#define NB_NSANGLES 252
#define NB_NSBINANG 86688
#define NB_NRINGS 64
#define NB_NLI2R 2074
#define NB_NOBLQ (NB_NLI2R - NB_NRINGS) // 2010 oblique ring pairs
#define NB_NRAYS (NB_NRINGS + 2 * NB_NOBLQ) // 4084 rays per LOR (= span-1 sinograms)
#define NB_NSN1 4084
#define NB_NSN11 837
#define NB_SEG0 127
#define NB_NCRS 504
#define NB_IMX 320
#define NB_IMY 320
#define NB_IMZ 127
#define NB_NCOL (NB_IMX * NB_IMY)
#define NB_NVOX (NB_IMX * NB_IMY * NB_IMZ)
#define NB_N_TT 10
#define NB_N_TV 1807

// Internal image layout ("col128"): a transaxial voxel column (v, u) is 128 floats,
// 512-byte aligned so it moves with one TMA bulk copy; z is de-interleaved
// (even z at [0,64), odd z at [64,127), slot 127 is padding) so that rays whose
// z differ by 2 voxels (neighbouring rings) hit neighbouring shared-memory banks.
#define NB_COLW 128
#define NB_IMG_COL128 ((size_t)NB_NCOL * NB_COLW)

// Per-LOR step lists: fixed stride, multiple of 4 so each list starts 16-byte aligned.
#define NB_STEP_STRIDE 416

// Mask of reference constants used by the Siddon arithmetic (def.h:106-118).
#define NB_TFOV2 890.0f
#define NB_VOXY 0.208626f
#define NB_VOXZ 0.203125f
#define NB_VOXZi 4.923077f
#define NB_RING 0.40625f
#define NB_L21 0.001f
#define NB_TA1 0.7885139f
#define NB_TA2 -0.7822831f

static __host__ __device__ __forceinline__ int nb_zi(int w) { return (w >> 1) + ((w & 1) << 6); }

// -------------------------------------------------------------------------------------------
// sm_90+/sm_100a bulk-copy primitives (PTX ISA: cp.async.bulk, cp.reduce.async.bulk, mbarrier)
// -------------------------------------------------------------------------------------------
static __device__ __forceinline__ uint32_t nb_smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

static __device__ __forceinline__ void nb_mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(nb_smem_u32(bar)), "r"(count)
               : "memory");
}

static __device__ __forceinline__ void nb_fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

static __device__ __forceinline__ void nb_mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(nb_smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

// Bounded wait on an mbarrier phase.  Returns false if the phase did not complete
// within `limit` polls; each poll suspends the thread for at most ~1 us, so the bound
// is about limit microseconds.
static __device__ __forceinline__ bool nb_mbar_wait(uint64_t *bar, uint32_t parity,
                                                    uint32_t limit) {
  uint32_t addr = nb_smem_u32(bar);
  for (uint32_t it = 0; it < limit; ++it) {
    uint32_t done;
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(done)
                 : "r"(addr), "r"(parity), "r"(1000u)
                 : "memory");
    if (done) return true;
  }
  return false;
}

// global -> shared bulk copy, completion counted on `bar` (bytes multiple of 16, both
// addresses 16-byte aligned)
static __device__ __forceinline__ void nb_bulk_g2s(void *dst_smem, const void *src_gmem,
                                                   uint32_t bytes, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(nb_smem_u32(dst_smem)),
      "l"(src_gmem), "r"(bytes), "r"(nb_smem_u32(bar))
      : "memory");
}

// shared -> global bulk reduction (element-wise fp32 add performed at L2)
static __device__ __forceinline__ void nb_bulk_reduce_add_f32(float *dst_gmem,
                                                              const float *src_smem,
                                                              uint32_t bytes) {
  asm volatile("cp.reduce.async.bulk.global.shared::cta.bulk_group.add.f32 [%0], [%1], %2;" ::"l"(
                   dst_gmem),
               "r"(nb_smem_u32(src_smem)), "r"(bytes)
               : "memory");
}

// shared -> global bulk reduction (element-wise uint32 add performed at L2, wrapping)
static __device__ __forceinline__ void nb_bulk_reduce_add_u32(uint32_t *dst_gmem,
                                                              const uint32_t *src_smem,
                                                              uint32_t bytes) {
  asm volatile("cp.reduce.async.bulk.global.shared::cta.bulk_group.add.u32 [%0], [%1], %2;" ::"l"(
                   dst_gmem),
               "r"(nb_smem_u32(src_smem)), "r"(bytes)
               : "memory");
}

static __device__ __forceinline__ void nb_bulk_commit() {
  asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}

// wait until at most N committed bulk groups of this thread still read shared memory
template <int N> static __device__ __forceinline__ void nb_bulk_wait_read() {
  asm volatile("cp.async.bulk.wait_group.read %0;" ::"n"(N) : "memory");
}
template <int N> static __device__ __forceinline__ void nb_bulk_wait_all() {
  asm volatile("cp.async.bulk.wait_group %0;" ::"n"(N) : "memory");
}

// order this thread's generic-proxy shared-memory writes before later async-proxy reads
static __device__ __forceinline__ void nb_fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// device-side error reporting: the first error code wins
static __device__ __forceinline__ void nb_set_error(int *flag, int code) {
  if (flag) atomicCAS(flag, 0, code);
}

// Error codes a kernel can raise through its device flag.
#define NB_DEVERR_MBAR_TIMEOUT 101
#define NB_DEVERR_BAD_LOR 102
#define NB_DEVERR_STEP_OVERFLOW 103
