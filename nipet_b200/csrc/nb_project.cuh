// nb_project.cuh -- the persistent Siddon projector kernel (forward, backward and the
// fused OSEM sub-iteration), used by nb_prj.cu.
//
// Reference semantics: prj/src/prjf.cu:33-206 (fprj_drct, fprj_oblq), prj/src/prjb.cu:33-187
// (bprj_drct, bprj_oblq), prj/src/recon.cu:252-309 and :459-497 (OSEM sub-iteration).
//
// B200 design
//  * Persistent grid, one 1024-thread CTA per SM.  A CTA owns one LOR (a transaxial
//    sinogram bin) at a time and computes all 4084 rays (span-1 ring pairs) of it, or
//    the rays of a reduced ring range (PrjArgs::rays / nrays); thread t handles rays t,
//    t+1024, t+2048, t+3072 of the ray table's order.
//  * The LOR's voxel columns (512 B each in the col128 layout) are streamed into shared
//    memory in chunks of CH columns with TMA bulk copies (cp.async.bulk + mbarrier),
//    double buffered, so every voxel read of the walk is a shared-memory load.
//  * Span-11 sinograms are formed by a deterministic in-CTA sum over the span-1 rays
//    (no global atomics, run-to-run identical); each CTA writes whole sinogram rows.
//  * Back projection accumulates the LOR's columns in shared memory as int32 fixed point
//    (native shared integer atomics; the scale is a power of two chosen per LOR so no
//    column slot can overflow), converts each finished chunk to float in a staging
//    buffer and flushes it with one TMA bulk reduce-add per column
//    (cp.reduce.async.bulk .add.f32) instead of one global atomic per voxel visit.
//  * The OSEM kernel fuses, per LOR: forward projection, the ratio
//    y / (Ax + (r+s)/(an)) and the back projection of the ratio -- the subset
//    sinogram never goes to HBM.
//
// The axial voxel index of every ray is kept in the de-interleaved column slot `zi`
// (even z in [0,64), odd z in [64,127)); a crossing moves it by `dz`, which alternates
// between two values (+64/-63 upwards, +63/-64 downwards).  nb_geom_create verifies
// once that no ray of the geometry leaves z in [0, 127], so the walk needs no clamp.
#pragma once
#include "nb_axial.cuh"
#include "nb_internal.cuh"

namespace nbk {

constexpr int NT = 1024;  // threads per CTA
constexpr int RPT = 4;    // rays per thread (NT * RPT >= 4084)
constexpr uint32_t WAIT_POLLS = 1u << 20;

enum { MODE_FWD = 0, MODE_BWD = 1, MODE_OSEM = 2 };

struct PrjArgs {
  const int32_t *scol;
  const float *st;
  const float4 *hdr;
  const nb_ray *rays;
  const int16_t *bin11;
  const int16_t *bin1;
  const int32_t *subs;
  int nprj;
  int naw;
  int nrays;             // rays of `rays` (4084, or those of a reduced ring range)
  int nout;              // sinograms per row (837, 4084, or a reduced range's count)
  int span;              // 1 or 11
  int att;               // forward: 0 emission, 1 attenuation
  const float *img;      // col128 image read by forward passes
  float *bimg;           // col128 image accumulated by backward passes
  float *sino;           // forward output [nprj][nout]
  const float *sino_in;  // backward input [nprj][nout] (or [naw][nout] if in_by_lor)
  int in_by_lor;         // backward: row of a LOR is its LOR index, not its subset position
  const uint16_t *psng;  // OSEM prompts [naw][nout]
  const float *rs;       // OSEM (r+s)/(an) [naw][nout]
  int fxbits;            // backward fixed point: |value| * 2^fxbits / 2^e fits every slot
  int *err;
};

template <int MODE, int CH> struct Smem {
  static_assert((2ull * CH * sizeof(float)) % 128 == 0, "tn buffers must keep 128-byte alignment");
  static constexpr bool HAS_I = MODE != MODE_FWD;
  static constexpr size_t buf_bytes = 2ull * CH * NB_COLW * sizeof(float);
  static constexpr size_t fbuf_off = 0;                 // forward columns / backward staging
  static constexpr size_t ibuf_off = fbuf_off + buf_bytes;  // backward int32 accumulators
  static constexpr size_t tn_off = ibuf_off + (HAS_I ? buf_bytes : 0);
  static constexpr size_t vals_off = tn_off + 2ull * CH * sizeof(float);
  static constexpr size_t rat_off = vals_off + 4096 * sizeof(float);
  static constexpr size_t misc_off = rat_off + (MODE == MODE_OSEM ? 4096 * sizeof(float) : 0);
  static constexpr size_t total = misc_off + 64;
  static_assert(misc_off % 128 == 0, "mbarriers must be aligned");
  static_assert(total <= 227 * 1024, "too much shared memory");
};

struct Job {
  int p;    // sinogram row
  int lor;  // LOR index (subs[p])
  int n;    // steps of the LOR
  int nch;  // chunks per pass
  int c;    // chunk index in the LOR's job list (OSEM: [0,nch) forward, [nch,2nch) backward)
  int valid;
};

template <int CH>
__device__ __forceinline__ void job_load(const PrjArgs &a, int p, Job &J) {
  J.p = p;
  J.valid = p < a.nprj;
  J.c = 0;
  if (!J.valid) return;
  const int lor = a.subs ? a.subs[p] : p;
  if (lor < 0 || lor >= a.naw) {
    if (threadIdx.x == 0) nb_set_error(a.err, NB_DEVERR_BAD_LOR);
    J.lor = 0;
    J.n = 0;
  } else {
    J.lor = lor;
    J.n = __float_as_int(a.hdr[lor].w);
  }
  J.nch = J.n > 0 ? (J.n + CH - 1) / CH : 1;
}

template <int MODE, int CH> __device__ __forceinline__ void job_next(const PrjArgs &a, Job &J) {
  const int per_lor = (MODE == MODE_OSEM) ? 2 * J.nch : J.nch;
  if (++J.c >= per_lor) job_load<CH>(a, J.p + gridDim.x, J);
}

template <int MODE> __device__ __forceinline__ bool job_is_load(const Job &J) {
  if (MODE == MODE_FWD) return true;
  if (MODE == MODE_BWD) return false;
  return J.c < J.nch;
}

template <int MODE> __device__ __forceinline__ int job_chunk(const Job &J) {
  return (MODE == MODE_OSEM && J.c >= J.nch) ? J.c - J.nch : J.c;
}

// warp 0: TMA loads of one forward chunk (its columns + exit parameters)
template <int CH>
__device__ __forceinline__ void issue_load(const PrjArgs &a, const Job &J, int chunk,
                                           float *cols, float *tnb, uint64_t *bar) {
  const int lane = threadIdx.x & 31;
  const int s0 = chunk * CH;
  const int n = max(0, min(CH, J.n - s0));
  const uint32_t tn_bytes = max(16u, (uint32_t)((n * 4 + 15) & ~15));
  if (lane == 0) nb_mbar_arrive_expect_tx(bar, (uint32_t)n * (NB_COLW * 4) + tn_bytes);
  __syncwarp();
  const int32_t *sc = a.scol + (size_t)J.lor * NB_STEP_STRIDE + s0;
  for (int i = lane; i < n; i += 32)
    nb_bulk_g2s(cols + (size_t)i * NB_COLW, a.img + (size_t)sc[i] * NB_COLW, NB_COLW * 4, bar);
  if (lane == 0) nb_bulk_g2s(tnb, a.st + (size_t)J.lor * NB_STEP_STRIDE + s0, tn_bytes, bar);
}

// warp 0: exit parameters of one backward chunk (plain loads; read after a CTA barrier)
template <int CH>
__device__ __forceinline__ void load_tn(const PrjArgs &a, const Job &J, int chunk, float *tnb) {
  const int lane = threadIdx.x & 31;
  const int s0 = chunk * CH;
  const int n = max(0, min(CH, J.n - s0));
  for (int i = lane; i < n; i += 32) tnb[i] = a.st[(size_t)J.lor * NB_STEP_STRIDE + s0 + i];
}

struct RayState {
  float acc[RPT];  // forward: line integral; backward: value to spread (bin * s * scale)
  float tzc[RPT];  // next axial crossing
  float dtz[RPT];
  int zo[RPT];     // byte offset of the current voxel in its column (4 * slot)
  int dz4[RPT];    // byte change of zo at the next crossing
  int dir4[RPT];   // 4 * (+1 / -1), 0 for direct planes
  float tp;
};

__device__ __forceinline__ void rays_init(const PrjArgs &a, const float4 h, RayState &S) {
  S.tp = h.x;
#pragma unroll
  for (int r = 0; r < RPT; r++) {
    const int ray = threadIdx.x + NT * r;
    S.acc[r] = 0.f;
    if (ray < a.nrays) {
      nb_axial A;
      nb_axial_setup(a.rays[ray], h.y, h.x, h.z, A);
      S.zo[r] = 4 * nb_zi(A.w);
      S.tzc[r] = A.tzc;
      S.dtz[r] = A.dtz;
      S.dir4[r] = 4 * A.dir;
      // slot change of the first crossing: parity of w decides (+64/-63 up, +63/-64 down)
      S.dz4[r] = 4 * (A.dir > 0 ? ((A.w & 1) ? -63 : 64) : (A.dir < 0 ? ((A.w & 1) ? -64 : 63) : 0));
    } else {
      S.zo[r] = 4 * 127;  // padding slot, never crosses
      S.tzc[r] = __int_as_float(0x7f800000);
      S.dtz[r] = 0.f;
      S.dir4[r] = 0;
      S.dz4[r] = 0;
    }
  }
}

// oblique length factor of ray r of this thread for a LOR of length atn
__device__ __forceinline__ float ray_s(const PrjArgs &a, int ray, float atn) {
  const nb_ray R = a.rays[ray];
  if (R.kind == 0) return 1.f;
  const float az_atn = __fdiv_rn(__fsub_rn(R.r1z, R.r0z), atn);
  return __fsqrt_rn(__fmaf_rn(az_atn, az_atn, 1.0f));
}

// Shared-memory accessors on 32-bit shared-window addresses (the per-ray cursors below).
static __device__ __forceinline__ float lds_f32(uint32_t addr) {
  float v;
  asm volatile("ld.shared.f32 %0, [%1];" : "=f"(v) : "r"(addr));
  return v;
}
// round(x * y) to the nearest integer (ties to even) for |x * y| < 2^22 on the FMA pipe:
// adding 1.5 * 2^23 inside the fused multiply-add leaves the integer in the low mantissa
// bits (the classic magic-constant rounding), instead of a multiply and a conversion on the
// much narrower conversion pipe.  The geometry keeps every back-projection contribution
// below 2^22 (nb_geom_create's choice of fxbits).
static __device__ __forceinline__ int nb_fx_round(float x, float y) {
  return __float_as_int(__fmaf_rn(x, y, 12582912.0f)) - 0x4B400000;
}

static __device__ __forceinline__ void reds_add_s32(uint32_t addr, int v) {
  asm volatile("red.shared.add.s32 [%0], %1;" ::"r"(addr), "r"(v) : "memory");
}

// One step of a ray covers [tp, tn] (prjf.cu:76-86 / :164-190 forward, prjb.cu:70-77 /
// :153-178 backward).  A ray that crosses a z plane at tzc inside the step (at most one per
// step, as in the reference) spends [tp, tzc] in its current voxel v0 and [tzc, tn] in the
// next voxel v1.  `cur` is the ray's shared-memory cursor: the address of its voxel in the
// chunk's first column; step u of the chunk adds u*512 bytes.
//
// Forward: lt*v0 + (tn - tzc)*(v1 - v0), one step per call.
static __device__ __forceinline__ void step_fwd(float &acc, uint32_t &cur, int &dz4, float &tzc,
                                                const int dir4, const float dtz, float tn, float lt,
                                                uint32_t off) {
  const float v0 = lds_f32(cur + off);
  acc = fmaf(lt, v0, acc);
  if (tn > tzc) {
    cur += dz4;
    dz4 = dir4 - dz4;
    const float v1 = lds_f32(cur + off);
    acc = fmaf(__fsub_rn(tn, tzc), v1 - v0, acc);
    tzc = __fadd_rn(tzc, dtz);
  }
}

// Backward: the same segments spread as int32 fixed point (acc holds the ray's value times
// the per-LOR scale), in two phases so that the rays of a thread run as straight-line
// code: phase 1 (every ray) adds the part in the current voxel -- weight lt, or
// (tzc - tp) on a crossing -- and phase 2 (crossing rays only) moves the cursor and adds
// (tn - tzc) to the new voxel.  (Measured on the forward walk the split was slower, so the
// forward keeps the one-call step.)
static __device__ __forceinline__ void step_bwd1(const float acc, const uint32_t cur,
                                                 const float tzc, float tn, float tp, float lt,
                                                 uint32_t off) {
  const float w = (tn > tzc) ? __fsub_rn(tzc, tp) : lt;
  reds_add_s32(cur + off, nb_fx_round(w, acc));
}

static __device__ __forceinline__ void step_bwd2(const float acc, uint32_t &cur, int &dz4,
                                                 float &tzc, const int dir4, const float dtz,
                                                 float tn, uint32_t off) {
  if (tn > tzc) {
    cur += dz4;
    dz4 = dir4 - dz4;
    reds_add_s32(cur + off, nb_fx_round(__fsub_rn(tn, tzc), acc));
    tzc = __fadd_rn(tzc, dtz);
  }
}

// Walk n steps of one shared-memory chunk (column i at chunk + i*512 bytes).  Steps are
// processed 8 at a time with immediate column offsets (the exit parameters come as two
// 16-byte loads), then one at a time for the tail.
template <bool BWD>
__device__ __forceinline__ void walk_chunk(RayState &S, const void *chunk, const float *tnb,
                                           int n) {
  const uint32_t sb = nb_smem_u32(chunk);
  uint32_t cur[RPT];
#pragma unroll
  for (int r = 0; r < RPT; r++) cur[r] = sb + (uint32_t)S.zo[r];
  float tp = S.tp;
  int i = 0;
  for (; i + 8 <= n; i += 8) {
    const float4 ta = *reinterpret_cast<const float4 *>(tnb + i);
    const float4 tb = *reinterpret_cast<const float4 *>(tnb + i + 4);
    const float t8[8] = {ta.x, ta.y, ta.z, ta.w, tb.x, tb.y, tb.z, tb.w};
#pragma unroll
    for (int u = 0; u < 8; u++) {
      const float tn = t8[u];
      const float lt = __fsub_rn(tn, tp);
      if (BWD) {
#pragma unroll
        for (int r = 0; r < RPT; r++) step_bwd1(S.acc[r], cur[r], S.tzc[r], tn, tp, lt, u * 512u);
#pragma unroll
        for (int r = 0; r < RPT; r++)
          step_bwd2(S.acc[r], cur[r], S.dz4[r], S.tzc[r], S.dir4[r], S.dtz[r], tn, u * 512u);
      } else {
#pragma unroll
        for (int r = 0; r < RPT; r++)
          step_fwd(S.acc[r], cur[r], S.dz4[r], S.tzc[r], S.dir4[r], S.dtz[r], tn, lt, u * 512u);
      }
      tp = tn;
    }
#pragma unroll
    for (int r = 0; r < RPT; r++) cur[r] += 8 * 512;
  }
  for (; i < n; i++) {
    const float tn = tnb[i];
    const float lt = __fsub_rn(tn, tp);
    if (BWD) {
#pragma unroll
      for (int r = 0; r < RPT; r++) step_bwd1(S.acc[r], cur[r], S.tzc[r], tn, tp, lt, 0u);
#pragma unroll
      for (int r = 0; r < RPT; r++)
        step_bwd2(S.acc[r], cur[r], S.dz4[r], S.tzc[r], S.dir4[r], S.dtz[r], tn, 0u);
    } else {
#pragma unroll
      for (int r = 0; r < RPT; r++)
        step_fwd(S.acc[r], cur[r], S.dz4[r], S.tzc[r], S.dir4[r], S.dtz[r], tn, lt, 0u);
    }
#pragma unroll
    for (int r = 0; r < RPT; r++) cur[r] += 512;
    tp = tn;
  }
  S.tp = tp;
#pragma unroll
  for (int r = 0; r < RPT; r++) S.zo[r] = (int)(cur[r] - sb) - n * (NB_COLW * 4);
}

template <int MODE, int CH>
__global__ void __launch_bounds__(NT, 1) k_project(const PrjArgs a) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  using L = Smem<MODE, CH>;
  float *fbuf = reinterpret_cast<float *>(smem_raw + L::fbuf_off);
  int *ibuf = reinterpret_cast<int *>(smem_raw + L::ibuf_off);
  float *tnbuf = reinterpret_cast<float *>(smem_raw + L::tn_off);
  float *vals = reinterpret_cast<float *>(smem_raw + L::vals_off);
  float *rat = reinterpret_cast<float *>(smem_raw + L::rat_off);
  uint64_t *bars = reinterpret_cast<uint64_t *>(smem_raw + L::misc_off);
  int *sflag = reinterpret_cast<int *>(smem_raw + L::misc_off + 16);
  unsigned *smax = reinterpret_cast<unsigned *>(smem_raw + L::misc_off + 24);  // [2]

  const int tid = threadIdx.x;
  const bool warp0 = tid < 32;
  const int nout = a.nout;

  if (tid == 0) {
    nb_mbar_init(&bars[0], 1);
    nb_mbar_init(&bars[1], 1);
    *sflag = 0;
    smax[0] = 0u;
    smax[1] = 0u;
    nb_fence_mbar_init();
  }
  if (L::HAS_I)
    for (int i = tid; i < 2 * CH * NB_COLW; i += NT) ibuf[i] = 0;
  __syncthreads();

  Job J, P;  // consumer cursor (all threads), producer cursor (warp 0)
  job_load<CH>(a, blockIdx.x, J);
  if (warp0) {
    P = J;
    for (int k = 0; k < 2 && P.valid; k++) {
      if (job_is_load<MODE>(P))
        issue_load<CH>(a, P, job_chunk<MODE>(P), fbuf + (size_t)k * CH * NB_COLW, tnbuf + k * CH,
                       &bars[k]);
      else
        load_tn<CH>(a, P, job_chunk<MODE>(P), tnbuf + k * CH);
      job_next<MODE, CH>(a, P);
    }
  }
  __syncthreads();

  RayState S;
  float inv_scale = 0.f;
  uint32_t phase = 0;  // bit b: parity of the next completion of bars[b]
  int j = 0, nlor = 0;
  while (J.valid) {
    const int b = j & 1;
    float *fb = fbuf + (size_t)b * CH * NB_COLW;
    int *ib = ibuf + (size_t)b * CH * NB_COLW;
    float *tb = tnbuf + b * CH;
    const bool load = job_is_load<MODE>(J);
    const int chunk = job_chunk<MODE>(J);
    const int n = max(0, min(CH, J.n - chunk * CH));
    const float4 h = a.hdr[J.lor];

    if (chunk == 0) {
      rays_init(a, h, S);
      if (!load) {
        // values to spread and the per-LOR fixed-point scale: a power of two such that
        // the largest slot sum (<= 242 rays x the longest segment x max|value|) stays
        // below 2^31 (fxbits is derived from the geometry's longest segment)
        float m = 0.f;
#pragma unroll
        for (int r = 0; r < RPT; r++) {
          const int ray = tid + NT * r;
          float v = 0.f;
          if (ray < a.nrays) {
            const nb_ray R = a.rays[ray];
            const int o = a.span == 11 ? R.out11 : R.out1;
            const size_t row = a.in_by_lor ? (size_t)J.lor : (size_t)J.p;
            const float bin = (MODE == MODE_BWD) ? a.sino_in[row * nout + o] : rat[o];
            v = bin * ray_s(a, ray, h.y);
          }
          S.acc[r] = v;
          m = fmaxf(m, fabsf(v));
        }
        for (int o = 16; o; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
        const int par = nlor & 1;
        if ((tid & 31) == 0 && m > 0.f) atomicMax(&smax[par], __float_as_uint(m));
        __syncthreads();
        const unsigned mb = smax[par];
        if (tid == 0) smax[par ^ 1] = 0u;
        float scale = 0.f;
        inv_scale = 0.f;
        if (mb != 0u && (mb >> 23) < 255u) {
          const int e = (int)(mb >> 23) - 126;  // max < 2^e
          scale = ldexpf(1.f, a.fxbits - e);
          inv_scale = ldexpf(1.f, e - a.fxbits);
        }
#pragma unroll
        for (int r = 0; r < RPT; r++) S.acc[r] *= scale;
        ++nlor;
      }
    }

    if (load) {
      if (!nb_mbar_wait(&bars[b], (phase >> b) & 1u, WAIT_POLLS)) atomicExch(sflag, 1);
      phase ^= 1u << b;
      walk_chunk<false>(S, fb, tb, n);
    } else {
      // the bulk reduce that last read staging buffer b must be done before we refill it
      if (warp0) nb_bulk_wait_read<1>();
      walk_chunk<true>(S, ib, tb, n);
      __syncthreads();
      // int32 accumulators -> float staging (and back to zero for their next use)
      const int nv = n * NB_COLW / 4;
      int4 *i4 = reinterpret_cast<int4 *>(ib);
      float4 *f4 = reinterpret_cast<float4 *>(fb);
      for (int x = tid; x < nv; x += NT) {
        const int4 q = i4[x];
        // slot 127 (the padding slice) is never written back
        const float w4 = (x & 31) == 31 ? 0.f : (float)q.w * inv_scale;
        f4[x] = make_float4((float)q.x * inv_scale, (float)q.y * inv_scale,
                            (float)q.z * inv_scale, w4);
        i4[x] = make_int4(0, 0, 0, 0);
      }
      nb_fence_proxy_async_smem();
    }

    // forward epilogue at the end of the LOR's forward pass
    if (load && chunk == J.nch - 1) {
#pragma unroll
      for (int r = 0; r < RPT; r++) {
        const int ray = tid + NT * r;
        if (ray < a.nrays) {
          float v = S.acc[r] * ray_s(a, ray, h.y);
          if (MODE == MODE_FWD && a.att == 1) {
            v = expf(-v);
            if (a.span == 11) v = v / (float)a.rays[ray].nos;
          }
          vals[ray] = v;
        }
      }
      __syncthreads();
      for (int o = tid; o < nout; o += NT) {
        float v;
        if (a.span == 11) {
          v = 0.f;
          const int16_t *lst = a.bin11 + o * 8;
#pragma unroll
          for (int q = 0; q < 8; q++) {
            const int ray = lst[q];
            if (ray >= 0) v += vals[ray];
          }
        } else {
          v = vals[a.bin1[o]];
        }
        if (MODE == MODE_FWD) {
          a.sino[(size_t)J.p * nout + o] = v;
        } else {
          const size_t g = (size_t)J.lor * nout + o;
          const float e = v + a.rs[g];
          const float y = (float)a.psng[g];
          rat[o] = (e > -0.000001f && e < 0.000001f) ? 0.f : __fdiv_rn(y, e);
        }
      }
    }

    __syncthreads();  // buffer b, the staging data and rat are complete / free
    if (*sflag) break;

    if (warp0) {
      if (MODE != MODE_FWD) {
        if (!load) {
          const int32_t *sc = a.scol + (size_t)J.lor * NB_STEP_STRIDE + chunk * CH;
          for (int i = tid; i < n; i += 32)
            nb_bulk_reduce_add_f32(a.bimg + (size_t)sc[i] * NB_COLW, fb + (size_t)i * NB_COLW,
                                   NB_COLW * 4);
        }
        nb_bulk_commit();  // one group per job and lane (empty for forward jobs)
      }
      // producer: job j+2 reuses buffer b
      if (P.valid) {
        if (job_is_load<MODE>(P)) {
          if (MODE == MODE_OSEM) nb_bulk_wait_read<0>();
          issue_load<CH>(a, P, job_chunk<MODE>(P), fb, tb, &bars[b]);
        } else {
          load_tn<CH>(a, P, job_chunk<MODE>(P), tb);
        }
        job_next<MODE, CH>(a, P);
      }
    }
    job_next<MODE, CH>(a, J);
    ++j;
  }
  if (*sflag && tid == 0) nb_set_error(a.err, NB_DEVERR_MBAR_TIMEOUT);
  if (warp0 && MODE != MODE_FWD) nb_bulk_wait_all<0>();
}

// Verifies that every ray of every LOR keeps its axial voxel in [0, 127]: the walk
// kernels index shared memory by it without clamping.  z = 127 is one slice above the
// image; it maps to the column's zero padding slot (reads 0, back projections into it
// are discarded).  In the mMR geometry exactly one ray step reaches it (the last step of
// rings 59->63 on LOR 24839).  One block per LOR.
// Walks every ray of every LOR once at geometry creation: counts axial positions outside
// [0, 127] into *bad, and raises *wbits (float bits, positive) to the largest weight a ray
// gives its current voxel at a crossing, |tzc - tp| -- which the back projection's
// fixed-point headroom has to cover besides the longest step.  (A crossing the reference
// takes a step late, when a ray passes two z planes in one step, makes it negative.)
static __global__ void k_check_walk(const float4 *__restrict__ hdr, const float *__restrict__ st,
                                    const nb_ray *__restrict__ rays, int naw, int *bad,
                                    unsigned *wbits) {
  const int lor = blockIdx.x;
  if (lor >= naw) return;
  const float4 h = hdr[lor];
  const int n = __float_as_int(h.w);
  int nbad = 0;
  float wmax = 0.f;
  for (int ray = threadIdx.x; ray < NB_NRAYS; ray += blockDim.x) {
    nb_axial A;
    nb_axial_setup(rays[ray], h.y, h.x, h.z, A);
    int w = A.w;
    float tzc = A.tzc, tp = h.x;
    if (w < 0 || w > NB_IMZ) nbad++;
    for (int k = 0; k < n; k++) {
      const float tn = st[(size_t)lor * NB_STEP_STRIDE + k];
      if (tn > tzc) {
        wmax = fmaxf(wmax, fabsf(__fsub_rn(tzc, tp)));
        w += A.dir;
        tzc = __fadd_rn(tzc, A.dtz);
        if (w < 0 || w > NB_IMZ) nbad++;
      }
      tp = tn;
    }
  }
  if (nbad) atomicAdd(bad, nbad);
  if (wmax > 0.f) atomicMax(wbits, __float_as_uint(wmax));
}

}  // namespace nbk
