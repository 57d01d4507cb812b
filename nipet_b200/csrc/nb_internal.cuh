// nb_internal.cuh -- geometry handle layout and host-side helpers shared by the
// translation units of libnipet_b200.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

#include "nb_common.cuh"

// Per-ray description, canonical ray order r in [0, 4084):
//   r <  64           direct plane of ring li = r
//   r <  64 + 2010    oblique +RD ray of ring pair li = r                (ring r0 -> r1)
//   r <  4084         oblique -RD ray of ring pair li = r - 2010         (ring r1 -> r0)
// (the reference's fprj_oblq computes the +RD and -RD rays of a pair in one thread).
struct nb_ray {
  float r0z, r1z;     // li2rng[li] (ring front edges, cm)
  int16_t out11;      // span-11 sinogram of the ray
  int16_t out1;       // span-1 sinogram of the ray
  int8_t kind;        // 0 direct, 1 +RD, 2 -RD
  int8_t nos;         // span-1 planes in its span-11 sinogram (li2nos)
  int16_t li;
};

struct nb_geom {
  int device;
  int nsm;
  int naw;
  // Siddon step lists: [naw][NB_STEP_STRIDE]
  int32_t *d_scol;   // transaxial column (v*320 + u) of each step
  float *d_st;       // exit parameter t of each step (the entry is the previous exit)
  float4 *d_hdr;     // per LOR: (t entry of step 0, atn, t2, nsteps as int bits)
  float *d_tt;       // reference-layout tt [naw][10]
  nb_ray *d_rays;    // [4084]
  int16_t *d_bin11;  // [837][8] rays summed into each span-11 sinogram (-1 padded)
  int16_t *d_bin1;   // [4084] ray of each span-1 sinogram
  float *d_scratch128;   // one col128 image (reference-layout entry points)
  float maxseg;          // longest walk segment of the geometry (cm)
  int fxbits;            // fixed-point headroom of the backward accumulators
  int *d_err;            // device error flag
  float *d_one;          // the constant 1.0f (randoms factor of a single-image batch)
  // host copies of the LUTs (for nb_geom_tables) and of the ray table (for nb_rings_create)
  float h_crs[504 * 4];
  int16_t *h_s2c;
  nb_ray *h_rays;    // [4084], the order of d_rays
};

// The rays of a reduced axial ring range [rs, re) (span 1 only): the reference's
// Cnt.RNG_STRT / RNG_END mode, in which projections cover the ring pairs inside the range,
// sinograms are numbered by the range's own span-1 Michelogram and images hold the axial
// voxel slab [vz0, vz0 + nvz) with nvz = 2 (re - rs) - 1 (prj/src/prjf.cu:209-320,
// prjb.cu:190-308, mmraux.py:566-617).  Every ray is one of the geometry's own rays, so
// the walk checks of nb_geom_create cover it.
struct nb_rings {
  int device;
  int rs, re;
  int nrays;         // rays of the range = its span-1 sinograms
  int vz0, nvz;
  nb_ray *d_rays;    // [nrays], out1 = the range's sinogram of the ray
  int16_t *d_bin1;   // [nrays] ray of each of the range's sinograms
};

// ---- tracing: an NVTX range around a C-ABI call (header-only NVTX3: without a profiler
// attached a push / pop costs a branch) ----
#include <nvtx3/nvToolsExt.h>
struct NbRange {
  explicit NbRange(const char *name) { nvtxRangePushA(name); }
  ~NbRange() { nvtxRangePop(); }
  NbRange(const NbRange &) = delete;
  NbRange &operator=(const NbRange &) = delete;
};
#define NB_RANGE(name) NbRange nb_range_(name)

// ---- host-side error plumbing (nb_capi.cu) ----
void nb_set_error_msg(const char *fmt, ...);
int nb_cuda_fail(cudaError_t e, const char *what, const char *file, int line);

#define NB_CUDA(call)                                                                          \
  do {                                                                                         \
    cudaError_t _e = (call);                                                                   \
    if (_e != cudaSuccess) return nb_cuda_fail(_e, #call, __FILE__, __LINE__);                 \
  } while (0)

#define NB_REQUIRE(cond, msg)                                                                  \
  do {                                                                                         \
    if (!(cond)) {                                                                             \
      nb_set_error_msg("%s", msg);                                                             \
      return NB_ERR_ARG;                                                                       \
    }                                                                                          \
  } while (0)

// Check the device error flag of a handle after synchronising `stream` (debug/validation
// paths only; the hot entry points do not synchronise).
int nb_check_device_flag(nb_geom *g, cudaStream_t stream);
