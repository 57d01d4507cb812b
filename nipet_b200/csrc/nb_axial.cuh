// nb_axial.cuh -- per-ray axial set-up of the Siddon walk.
//
// The voxel a ray visits is decided in float32 with the operation order of the
// reference kernels (prj/src/prjf.cu:38-39 direct, :136-160 oblique; prjb.cu has the
// same lines).  Every operation is written with an explicit round-to-nearest intrinsic
// so the compiler cannot contract or reorder it.  Where nvcc contracts the reference's
// expressions the restatement fuses explicitly: `pz + az_atn * t`, and the voxel position
// .5*SZ_IMZ + SZ_VOXZi*z and plane c*SZ_VOXZ - .5*SZ_IMZ*SZ_VOXZ, whose double sums nvcc
// narrows to float (exact for these operands) and then fuses with the product.  This
// decides the start voxel of a ray whose position falls on a plane (checked against the
// reference's own projections on every LOR).
#pragma once
#include "nb_internal.cuh"

struct nb_axial {
  int w;       // start voxel (z)
  int dir;     // +1 / -1 voxel step at an axial crossing (0: direct, never crosses)
  float tzc;   // parameter t of the next axial crossing (+inf for direct rays)
  float dtz;   // increment of tzc per crossing
  float s;     // oblique length factor sqrt(1 + (dz/atn)^2) (1 for direct rays)
};

// .5*SZ_IMZ + SZ_VOXZi*z as one fused multiply-add; c*SZ_VOXZ - .5*SZ_IMZ*SZ_VOXZ likewise
static __device__ __forceinline__ float nb_zpos(float z) {
  return __fmaf_rn(NB_VOXZi, z, (float)(0.5 * NB_IMZ));
}
static __device__ __forceinline__ float nb_zline(float c) {
  return __fmaf_rn(c, NB_VOXZ, (float)(-0.5 * NB_IMZ * (double)NB_VOXZ));
}
static __device__ __forceinline__ int nb_zvox(float z) { return (int)floorf(nb_zpos(z)); }

static __device__ __forceinline__ void nb_axial_setup(const nb_ray &R, float atn, float tp,
                                                      float t2, nb_axial &A) {
  if (R.kind == 0) {
    float z = __double2float_rn(__dadd_rn((double)R.r0z, 0.5 * (double)NB_RING));
    A.w = nb_zvox(z);
    A.dir = 0;
    A.tzc = __int_as_float(0x7f800000); // +inf
    A.dtz = 0.f;
    A.s = 1.f;
    return;
  }
  float az = __fsub_rn(R.r1z, R.r0z);
  float az_atn = __fdiv_rn(az, atn);
  A.s = __fsqrt_rn(__fmaf_rn(az_atn, az_atn, 1.0f));
  int sgnaz = az >= 0.f ? 1 : -1;
  float pz = __double2float_rn(__dadd_rn((double)R.r0z, 0.5 * (double)NB_RING));
  float z = __fmaf_rn(az_atn, tp, pz);
  int w = nb_zvox(z);
  float lz1 = nb_zline(ceilf(nb_zpos(z)));
  float zm = __double2float_rn(__dsub_rn(__dadd_rn((double)R.r1z, 0.5 * (double)NB_RING),
                                         (double)__fmul_rn(az_atn, tp)));
  int w_ = nb_zvox(zm);
  float z2 = __fmaf_rn(az_atn, t2, pz);
  float lz2 = nb_zline(floorf(nb_zpos(z2)));
  int nz = (int)__fdiv_rn(fabsf(__fsub_rn(lz2, lz1)), NB_VOXZ);
  float tz1 = __fdiv_rn(__fsub_rn(lz1, pz), az_atn);
  float tz2 = __fdiv_rn(__fsub_rn(lz2, pz), az_atn);
  A.dtz = __fdiv_rn(__fsub_rn(tz2, tz1), (float)nz);
  A.tzc = tz1;
  if (R.kind == 1) {
    A.w = w;
    A.dir = sgnaz;
  } else {
    A.w = w_;
    A.dir = -sgnaz;
  }
}

static __device__ __forceinline__ int nb_clampz(int w) { return w < 0 ? 0 : (w > 127 ? 127 : w); }
