// nb_batch.cu -- OSEM for many images at once: bootstrap replicates or dynamic frames that
// share the scanner geometry, attenuation, normalisation and sensitivity, each with its
// own prompts and image (the batched configuration of the reference's osem(),
// prj/src/recon.cu:318-497, run for all replicates in one launch per sub-iteration).
//
// Layout: "col128 x Bs" -- images grouped Bs at a time, group g at
// img + g * [320*320][128][Bs]; inside a column the Bs replicate values of a voxel are
// contiguous, so one 16-byte shared load (Bs = 4) feeds four replicates and every
// geometric decision of the Siddon walk (crossing test, cursor update, segment lengths)
// is shared by the Bs replicates of a ray.  A persistent CTA takes (LOR, group) jobs; per
// job it runs the forward pass of the LOR for the Bs images, forms the Bs ratio rows
// y_b / (Ax_b + c_b (r+s)/(an)) and back projects them, exactly as the single-image
// kernel (nb_project.cuh) does for one image.  The same kernel in forward-only and
// backward-only mode is the batched projector pair (nb_fprj_batch / nb_bprj_batch).
#include <math.h>

#include <atomic>

#include "nb_axial.cuh"
#include "nb_internal.cuh"
#include "nb_project.cuh"

namespace nbb {

using nbk::WAIT_POLLS;
using nbk::lds_f32;
using nbk::nb_fx_round;
using nbk::reds_add_s32;

constexpr int NB_MAXREP = 1024;

struct BatchArgs {
  const int32_t *scol;
  const float *st;
  const float4 *hdr;
  const nb_ray *rays;
  const int16_t *bin11;
  const int16_t *bin1;
  const int32_t *subs;
  int nprj, naw, span, ngroups, nrep;
  const float *img;        // [ngroups][NCOL][128][Bs]
  float *bimg;             // same layout, accumulated
  const uint16_t *psng;    // [nrep][naw][nout]
  const float *rs;         // [naw][nout] (r+s)/(an), scaled per replicate by rscale
  const float *rscale;     // [nrep]
  float *sino_out;         // forward mode: [nrep][nprj][nout]
  const float *sino_in;    // backward mode: [nrep][nprj][nout]
  int fxbits;
  int *err;
};

// kernel modes: the fused OSEM sub-iteration (forward, ratio, backward), a forward
// projection only (sinogram rows out) and a back projection only (sinogram rows in)
enum { BMODE_OSEM = 0, BMODE_FWD = 1, BMODE_BWD = 2 };

// a job (LOR, image group) runs nch chunks of the LOR's columns per pass: two passes
// (forward, then backward) in OSEM mode, one otherwise
template <int MODE> __device__ __forceinline__ bool bphase_load(int c, int nch) {
  return MODE == BMODE_OSEM ? c < nch : MODE == BMODE_FWD;
}
template <int MODE> __device__ __forceinline__ int bphase_chunk(int c, int nch) {
  return (MODE == BMODE_OSEM && c >= nch) ? c - nch : c;
}

// shared-memory layout; every region starts on a 128-byte boundary (the mbarriers in the
// misc region need 8-byte, the vector/TMA accesses 16-byte alignment)
__host__ __device__ constexpr size_t align128(size_t x) { return (x + 127) & ~(size_t)127; }

template <int BS, int CH> struct BSmem {
  static constexpr size_t col_bytes = (size_t)NB_COLW * BS * sizeof(float);
  static constexpr size_t buf_bytes = 2ull * CH * col_bytes;
  static constexpr size_t fbuf_off = 0;
  static constexpr size_t ibuf_off = align128(buf_bytes);
  static constexpr size_t tn_off = align128(ibuf_off + buf_bytes);
  static constexpr size_t vals_off = align128(tn_off + 2ull * CH * sizeof(float));
  static constexpr size_t rat_off = align128(vals_off + 4096ull * BS * sizeof(float));
  template <int NOUT> __host__ __device__ static constexpr size_t misc_off() {
    return align128(rat_off + (size_t)NOUT * BS * sizeof(float));
  }
  template <int NOUT> __host__ __device__ static constexpr size_t total() {
    return misc_off<NOUT>() + 128;  // barriers, flag, maxima, inverse scales, prefetch cursor
  }
};

struct BJob {
  int p, g, lor, n, nch, c, valid;
};
static_assert(sizeof(BJob) <= 32, "prefetch cursor slot in the misc region");

template <int CH>
__device__ __forceinline__ void bjob_load(const BatchArgs &a, int q, BJob &J) {
  J.valid = q < a.nprj * a.ngroups;
  J.c = 0;
  if (!J.valid) return;
  J.p = q / a.ngroups;
  J.g = q - J.p * a.ngroups;
  const int lor = a.subs ? a.subs[J.p] : J.p;
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

template <int CH, int MODE>
__device__ __forceinline__ void bjob_next(const BatchArgs &a, BJob &J, int &q) {
  if (++J.c >= (MODE == BMODE_OSEM ? 2 : 1) * J.nch) {
    q += gridDim.x;
    bjob_load<CH>(a, q, J);
  }
}

template <int BS, int CH>
__device__ __forceinline__ void bissue_load(const BatchArgs &a, const BJob &J, int chunk,
                                            float *cols, float *tnb, uint64_t *bar) {
  constexpr uint32_t colb = NB_COLW * BS * 4;
  const int lane = threadIdx.x & 31;
  const int s0 = chunk * CH;
  const int n = max(0, min(CH, J.n - s0));
  const uint32_t tn_bytes = max(16u, (uint32_t)((n * 4 + 15) & ~15));
  if (lane == 0) nb_mbar_arrive_expect_tx(bar, (uint32_t)n * colb + tn_bytes);
  __syncwarp();
  const int32_t *sc = a.scol + (size_t)J.lor * NB_STEP_STRIDE + s0;
  const float *gimg = a.img + (size_t)J.g * NB_NCOL * NB_COLW * BS;
  for (int i = lane; i < n; i += 32)
    nb_bulk_g2s(cols + (size_t)i * NB_COLW * BS, gimg + (size_t)sc[i] * NB_COLW * BS, colb, bar);
  if (lane == 0) nb_bulk_g2s(tnb, a.st + (size_t)J.lor * NB_STEP_STRIDE + s0, tn_bytes, bar);
}

template <int CH>
__device__ __forceinline__ void bload_tn(const BatchArgs &a, const BJob &J, int chunk, float *tnb) {
  const int lane = threadIdx.x & 31;
  const int s0 = chunk * CH;
  const int n = max(0, min(CH, J.n - s0));
  for (int i = lane; i < n; i += 32) tnb[i] = a.st[(size_t)J.lor * NB_STEP_STRIDE + s0 + i];
}

// rays of one thread: ray index = threadIdx.x + NT * r, r < RPT (NT * RPT >= 4084)
template <int BS, int RPT> struct BRay {
  float acc[RPT][BS];
  float tzc[RPT], dtz[RPT];
  int zo[RPT], dz4[RPT], dir4[RPT];  // byte offsets in units of 4*BS bytes per slot
  float tp;
};

template <int BS, int NT, int RPT>
__device__ __forceinline__ void brays_init(const BatchArgs &a, const float4 h, BRay<BS, RPT> &S) {
  S.tp = h.x;
#pragma unroll
  for (int r = 0; r < RPT; r++) {
    const int ray = threadIdx.x + NT * r;
#pragma unroll
    for (int k = 0; k < BS; k++) S.acc[r][k] = 0.f;
    if (ray < NB_NRAYS) {
      nb_axial A;
      nb_axial_setup(a.rays[ray], h.y, h.x, h.z, A);
      S.zo[r] = 4 * BS * nb_zi(A.w);
      S.tzc[r] = A.tzc;
      S.dtz[r] = A.dtz;
      S.dir4[r] = 4 * BS * A.dir;
      S.dz4[r] = 4 * BS *
                 (A.dir > 0 ? ((A.w & 1) ? -63 : 64) : (A.dir < 0 ? ((A.w & 1) ? -64 : 63) : 0));
    } else {
      S.zo[r] = 4 * BS * 127;
      S.tzc[r] = __int_as_float(0x7f800000);
      S.dtz[r] = 0.f;
      S.dir4[r] = 0;
      S.dz4[r] = 0;
    }
  }
}

// oblique length factor sqrt(1 + (dz/atn)^2) of a ray (1 for direct planes)
__device__ __forceinline__ float oblique_s(const nb_ray &R, float atn) {
  if (R.kind == 0) return 1.f;
  const float az_atn = __fdiv_rn(__fsub_rn(R.r1z, R.r0z), atn);
  return __fsqrt_rn(__fmaf_rn(az_atn, az_atn, 1.0f));
}

// BS floats as one vector type (16-, 8- or 4-byte accesses)
template <int BS> struct VecF;
template <> struct VecF<1> { using T = float; };
template <> struct VecF<2> { using T = float2; };
template <> struct VecF<4> { using T = float4; };

template <int BS> struct VecT;
template <> struct VecT<1> { static __device__ __forceinline__ void ld(uint32_t a, float *v) { v[0] = lds_f32(a); } };
template <> struct VecT<2> {
  static __device__ __forceinline__ void ld(uint32_t a, float *v) {
    asm volatile("ld.shared.v2.f32 {%0,%1}, [%2];" : "=f"(v[0]), "=f"(v[1]) : "r"(a));
  }
};
template <> struct VecT<4> {
  static __device__ __forceinline__ void ld(uint32_t a, float *v) {
    asm volatile("ld.shared.v4.f32 {%0,%1,%2,%3}, [%4];"
                 : "=f"(v[0]), "=f"(v[1]), "=f"(v[2]), "=f"(v[3])
                 : "r"(a));
  }
};

// One column step of ray r, split in two phases so that the rays of a thread run as
// straight-line code: phase 1 (every ray) covers the segment in the current z slot -- the
// whole column, or up to the z crossing -- and phase 2 (only the rays whose z crossing
// falls inside this column) moves the cursor and covers the rest in the new slot.
//   forward:  (tzc - tp) v0 + (tn - tzc) v1   on a crossing, lt v0 otherwise
//   backward: the same weights times the ray's ratio, added to the two voxels
template <int BS, int RPT, bool BWD>
__device__ __forceinline__ void bstep1(BRay<BS, RPT> &S, int r, uint32_t cur, float tn, float tp,
                                       float lt, uint32_t off) {
  const float w = (tn > S.tzc[r]) ? __fsub_rn(S.tzc[r], tp) : lt;
  if (!BWD) {
    float v0[BS];
    VecT<BS>::ld(cur + off, v0);
#pragma unroll
    for (int k = 0; k < BS; k++) S.acc[r][k] = fmaf(w, v0[k], S.acc[r][k]);
  } else {
    // backward accumulators are replicate-major inside a column ([BS][128] ints): the
    // cursor is in units of 4 bytes per slot and replicate k adds k * 512 bytes, so the
    // lanes of a warp (neighbouring slots) hit neighbouring banks
#pragma unroll
    for (int k = 0; k < BS; k++)
      reds_add_s32(cur + off + 512u * k, nb_fx_round(w, S.acc[r][k]));
  }
}

template <int BS, int RPT, bool BWD>
__device__ __forceinline__ void bstep2(BRay<BS, RPT> &S, int r, uint32_t &cur, float tn,
                                       uint32_t off) {
  if (tn > S.tzc[r]) {
    constexpr int LG = BWD ? (BS == 4 ? 2 : (BS == 2 ? 1 : 0)) : 0;
    cur += S.dz4[r] >> LG;
    S.dz4[r] = S.dir4[r] - S.dz4[r];
    const float fb = __fsub_rn(tn, S.tzc[r]);
    if (!BWD) {
      float v1[BS];
      VecT<BS>::ld(cur + off, v1);
#pragma unroll
      for (int k = 0; k < BS; k++) S.acc[r][k] = fmaf(fb, v1[k], S.acc[r][k]);
    } else {
#pragma unroll
      for (int k = 0; k < BS; k++)
        reds_add_s32(cur + off + 512u * k, nb_fx_round(fb, S.acc[r][k]));
    }
    S.tzc[r] = __fadd_rn(S.tzc[r], S.dtz[r]);
  }
}

template <int BS, int RPT, bool BWD>
__device__ __forceinline__ void bwalk(BRay<BS, RPT> &S, const void *chunk, const float *tnb, int n) {
  constexpr uint32_t colb = NB_COLW * BS * 4;
  constexpr int LG = BWD ? (BS == 4 ? 2 : (BS == 2 ? 1 : 0)) : 0;  // see bstep1
  const uint32_t sb = nb_smem_u32(chunk);
  uint32_t cur[RPT];
#pragma unroll
  for (int r = 0; r < RPT; r++) cur[r] = sb + (uint32_t)(S.zo[r] >> LG);
  float tp = S.tp;
  int i = 0;
  for (; i + 4 <= n; i += 4) {
    const float4 t4 = *reinterpret_cast<const float4 *>(tnb + i);
    const float tv[4] = {t4.x, t4.y, t4.z, t4.w};
#pragma unroll
    for (int u = 0; u < 4; u++) {
      const float tn = tv[u];
      const float lt = __fsub_rn(tn, tp);
#pragma unroll
      for (int r = 0; r < RPT; r++) bstep1<BS, RPT, BWD>(S, r, cur[r], tn, tp, lt, u * colb);
#pragma unroll
      for (int r = 0; r < RPT; r++) bstep2<BS, RPT, BWD>(S, r, cur[r], tn, u * colb);
      tp = tn;
    }
#pragma unroll
    for (int r = 0; r < RPT; r++) cur[r] += 4 * colb;
  }
  for (; i < n; i++) {
    const float tn = tnb[i];
    const float lt = __fsub_rn(tn, tp);
#pragma unroll
    for (int r = 0; r < RPT; r++) bstep1<BS, RPT, BWD>(S, r, cur[r], tn, tp, lt, 0u);
#pragma unroll
    for (int r = 0; r < RPT; r++) {
      bstep2<BS, RPT, BWD>(S, r, cur[r], tn, 0u);
      cur[r] += colb;
    }
    tp = tn;
  }
  S.tp = tp;
#pragma unroll
  for (int r = 0; r < RPT; r++) S.zo[r] = ((int)(cur[r] - sb) - n * (int)colb) << LG;
}

template <int BS, int CH, int NOUT, int NT, int RPT, int MODE>
__global__ void __launch_bounds__(NT, 1) k_osem_batch(const BatchArgs a) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  using L = BSmem<BS, CH>;
  constexpr int COLF = NB_COLW * BS;  // floats per column
  float *fbuf = reinterpret_cast<float *>(smem_raw + L::fbuf_off);
  int *ibuf = reinterpret_cast<int *>(smem_raw + L::ibuf_off);
  float *tnbuf = reinterpret_cast<float *>(smem_raw + L::tn_off);
  float *vals = reinterpret_cast<float *>(smem_raw + L::vals_off);   // [4096][BS]
  float *rat = reinterpret_cast<float *>(smem_raw + L::rat_off);     // [NOUT][BS]
  unsigned char *misc = smem_raw + L::template misc_off<NOUT>();
  uint64_t *bars = reinterpret_cast<uint64_t *>(misc);
  int *sflag = reinterpret_cast<int *>(misc + 16);
  // per-image maxima of the back-projected ray values, double-buffered by LOR parity
  unsigned *smax = reinterpret_cast<unsigned *>(misc + 24);  // [2][BS]
  float *sinv = reinterpret_cast<float *>(misc + 64);         // [BS] inverse scales
  // warp 0's prefetch cursor (the job whose chunks it loads ahead) lives in shared memory
  // so that it takes no registers in the other warps
  BJob *sP = reinterpret_cast<BJob *>(misc + 80);
  int *sqP = reinterpret_cast<int *>(misc + 112);

  const int tid = threadIdx.x;
  const bool warp0 = tid < 32;
  if (tid == 0) {
    nb_mbar_init(&bars[0], 1);
    nb_mbar_init(&bars[1], 1);
    *sflag = 0;
    for (int k = 0; k < 2 * BS; k++) smax[k] = 0u;
    nb_fence_mbar_init();
  }
  for (int i = tid; i < 2 * CH * COLF; i += NT) ibuf[i] = 0;
  __syncthreads();

  BJob J;
  int qJ = blockIdx.x;
  bjob_load<CH>(a, qJ, J);
  if (warp0) {
    BJob P = J;
    int qP = blockIdx.x;
    for (int k = 0; k < 2 && P.valid; k++) {
      const bool ld = bphase_load<MODE>(P.c, P.nch);
      const int chunk = bphase_chunk<MODE>(P.c, P.nch);
      if (ld)
        bissue_load<BS, CH>(a, P, chunk, fbuf + (size_t)k * CH * COLF, tnbuf + k * CH, &bars[k]);
      else
        bload_tn<CH>(a, P, chunk, tnbuf + k * CH);
      bjob_next<CH, MODE>(a, P, qP);
    }
    __syncwarp();
    if (tid == 0) {
      *sP = P;
      *sqP = qP;
    }
  }
  __syncthreads();

  BRay<BS, RPT> S;
  uint32_t phase = 0;
  int j = 0, nlor = 0;
  while (J.valid) {
    const int b = j & 1;
    float *fb = fbuf + (size_t)b * CH * COLF;
    int *ib = ibuf + (size_t)b * CH * COLF;
    float *tb = tnbuf + b * CH;
    const bool load = bphase_load<MODE>(J.c, J.nch);
    const int chunk = bphase_chunk<MODE>(J.c, J.nch);
    const int n = max(0, min(CH, J.n - chunk * CH));

    if (chunk == 0) {
      const float4 h = a.hdr[J.lor];
      brays_init<BS, NT, RPT>(a, h, S);
      if (MODE == BMODE_BWD) {  // the rows to back project take the place of the ratio
        for (int x = tid; x < NOUT * BS; x += NT) {
          const int o = x / BS, k = x - o * BS;
          const int rep = J.g * BS + k;
          rat[x] = rep < a.nrep ? a.sino_in[((size_t)rep * a.nprj + J.p) * NOUT + o] : 0.f;
        }
        __syncthreads();
      }
      if (!load) {
        // one fixed-point scale per image: images of one group can differ in count level
        // by orders of magnitude, and a shared scale would quantise the quieter ones'
        // neighbours on the loudest one's grid
        float m[BS];
#pragma unroll
        for (int k = 0; k < BS; k++) m[k] = 0.f;
#pragma unroll
        for (int r = 0; r < RPT; r++) {
          const int ray = tid + NT * r;
          float s = 0.f;
          int o = 0;
          if (ray < NB_NRAYS) {
            const nb_ray R = a.rays[ray];
            o = (NOUT == NB_NSN11) ? R.out11 : R.out1;
            s = oblique_s(R, h.y);
          }
#pragma unroll
          for (int k = 0; k < BS; k++) {
            const float v = (ray < NB_NRAYS) ? rat[o * BS + k] * s : 0.f;
            S.acc[r][k] = v;
            m[k] = fmaxf(m[k], fabsf(v));
          }
        }
        const int par = nlor & 1;
#pragma unroll
        for (int k = 0; k < BS; k++) {
          for (int o = 16; o; o >>= 1) m[k] = fmaxf(m[k], __shfl_xor_sync(0xffffffffu, m[k], o));
          if ((tid & 31) == 0 && m[k] > 0.f) atomicMax(&smax[par * BS + k], __float_as_uint(m[k]));
        }
        __syncthreads();
        float scale[BS];
#pragma unroll
        for (int k = 0; k < BS; k++) {
          const unsigned mb = smax[par * BS + k];
          scale[k] = 0.f;
          float inv = 0.f;
          if (mb != 0u && (mb >> 23) < 255u) {
            const int e = (int)(mb >> 23) - 126;
            scale[k] = ldexpf(1.f, a.fxbits - e);
            inv = ldexpf(1.f, e - a.fxbits);
          }
          if (tid == k) sinv[k] = inv;  // read by this LOR's conversions, after a barrier
        }
        if (tid < BS) smax[(par ^ 1) * BS + tid] = 0u;
#pragma unroll
        for (int r = 0; r < RPT; r++)
#pragma unroll
          for (int k = 0; k < BS; k++) S.acc[r][k] *= scale[k];
        ++nlor;
      }
    }

    if (load) {
      if (!nb_mbar_wait(&bars[b], (phase >> b) & 1u, WAIT_POLLS)) atomicExch(sflag, 1);
      phase ^= 1u << b;
      bwalk<BS, RPT, false>(S, fb, tb, n);
    } else {
      if (warp0) nb_bulk_wait_read<1>();
      bwalk<BS, RPT, true>(S, ib, tb, n);
      __syncthreads();
      // int32 [col][BS][128] -> float staging [col][128][BS] (the image layout the bulk
      // reduce adds into), zeroing the accumulators; slot 127 (padding) is not written back
      const int nv = n * NB_COLW;
      float inv[BS];
#pragma unroll
      for (int k = 0; k < BS; k++) inv[k] = sinv[k];
      for (int x = tid; x < nv; x += NT) {
        const int c = x >> 7, slot = x & 127;
        typename VecF<BS>::T vout;  // the slot's BS values, one vector store
        float *vo = reinterpret_cast<float *>(&vout);
#pragma unroll
        for (int k = 0; k < BS; k++) {
          const int src = c * COLF + k * NB_COLW + slot;
          vo[k] = slot == 127 ? 0.f : (float)ib[src] * inv[k];
          ib[src] = 0;
        }
        *reinterpret_cast<typename VecF<BS>::T *>(fb + c * COLF + slot * BS) = vout;
      }
      nb_fence_proxy_async_smem();
    }

    if (load && chunk == J.nch - 1) {
      const float atn = a.hdr[J.lor].y;
#pragma unroll
      for (int r = 0; r < RPT; r++) {
        const int ray = tid + NT * r;
        if (ray < NB_NRAYS) {
          const float s = oblique_s(a.rays[ray], atn);
#pragma unroll
          for (int k = 0; k < BS; k++) vals[ray * BS + k] = S.acc[r][k] * s;
        }
      }
      __syncthreads();
      for (int x = tid; x < NOUT * BS; x += NT) {
        const int o = x / BS, k = x - o * BS;
        float v;
        if (NOUT == NB_NSN11) {
          v = 0.f;
          const int16_t *lst = a.bin11 + o * 8;
#pragma unroll
          for (int qq = 0; qq < 8; qq++) {
            const int ray = lst[qq];
            if (ray >= 0) v += vals[ray * BS + k];
          }
        } else {
          v = vals[a.bin1[o] * BS + k];
        }
        const int rep = J.g * BS + k;
        if (MODE == BMODE_FWD) {
          if (rep < a.nrep) a.sino_out[((size_t)rep * a.nprj + J.p) * NOUT + o] = v;
          continue;
        }
        float rr = 0.f;
        if (rep < a.nrep) {
          const size_t gi = (size_t)J.lor * NOUT + o;
          const float e = v + a.rscale[rep] * a.rs[gi];
          const float y = (float)a.psng[(size_t)rep * a.naw * NOUT + gi];
          rr = (e > -0.000001f && e < 0.000001f) ? 0.f : __fdiv_rn(y, e);
        }
        rat[x] = rr;
      }
    }

    __syncthreads();
    if (*sflag) break;

    if (warp0) {
      if (!load) {
        const int32_t *sc = a.scol + (size_t)J.lor * NB_STEP_STRIDE + chunk * CH;
        float *gb = a.bimg + (size_t)J.g * NB_NCOL * COLF;
        for (int i = tid; i < n; i += 32)
          nb_bulk_reduce_add_f32(gb + (size_t)sc[i] * COLF, fb + (size_t)i * COLF, COLF * 4);
      }
      nb_bulk_commit();
      BJob P = *sP;
      int qP = *sqP;
      if (P.valid) {
        const bool ld = bphase_load<MODE>(P.c, P.nch);
        const int pch = bphase_chunk<MODE>(P.c, P.nch);
        if (ld) {
          nb_bulk_wait_read<0>();
          bissue_load<BS, CH>(a, P, pch, fb, tb, &bars[b]);
        } else {
          bload_tn<CH>(a, P, pch, tb);
        }
        bjob_next<CH, MODE>(a, P, qP);
      }
      __syncwarp();
      if (tid == 0) {
        *sP = P;
        *sqP = qP;
      }
    }
    bjob_next<CH, MODE>(a, J, qJ);
    ++j;
  }
  if (*sflag && tid == 0) nb_set_error(a.err, NB_DEVERR_MBAR_TIMEOUT);
  if (warp0) nb_bulk_wait_all<0>();
}

}  // namespace nbb

// ---------------------------------------------------------------------------------------
// layout conversion and the batched image update
// ---------------------------------------------------------------------------------------
namespace {

// [nrep][320*320][127] (reference layout) <-> [ngroups][320*320][128][BS]
__global__ void k_to_batch(float *__restrict__ dst, const float *__restrict__ src, int nrep,
                           int bs) {
  const size_t n = (size_t)nrep * NB_NCOL * NB_COLW;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n;
       t += (size_t)gridDim.x * blockDim.x) {
    const int z = (int)(t % NB_COLW);
    const size_t rc = t / NB_COLW;
    const int col = (int)(rc % NB_NCOL);
    const int rep = (int)(rc / NB_NCOL);
    const int g = rep / bs, k = rep - g * bs;
    const float v = z < NB_IMZ ? src[((size_t)rep * NB_NCOL + col) * NB_IMZ + z] : 0.f;
    dst[(((size_t)g * NB_NCOL + col) * NB_COLW + nb_zi(z)) * bs + k] = v;
  }
}

// every voxel of the nrep images of the batched layout set to `value`; the padding slot of
// each column (slot 127) and the images padding the last group set to zero
__global__ void k_fill_batch(float *__restrict__ dst, float value, int nrep, int bs,
                             size_t n) {
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n;
       t += (size_t)gridDim.x * blockDim.x) {
    const int k = (int)(t % bs);
    const int slot = (int)((t / bs) % NB_COLW);
    const int g = (int)(t / ((size_t)bs * NB_COLW * NB_NCOL));
    dst[t] = (g * bs + k < nrep && slot != NB_COLW - 1) ? value : 0.f;
  }
}

__global__ void k_from_batch(float *__restrict__ dst, const float *__restrict__ src, int nrep,
                             int bs) {
  const size_t n = (size_t)nrep * NB_NCOL * NB_IMZ;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n;
       t += (size_t)gridDim.x * blockDim.x) {
    const int z = (int)(t % NB_IMZ);
    const size_t rc = t / NB_IMZ;
    const int col = (int)(rc % NB_NCOL);
    const int rep = (int)(rc / NB_NCOL);
    const int g = rep / bs, k = rep - g * bs;
    dst[t] = src[(((size_t)g * NB_NCOL + col) * NB_COLW + nb_zi(z)) * bs + k];
  }
}

// img = msk ? img * (|sens| < 1e-6 ? 0 : bimg / sens) : 0; bimg = 0  (recon.cu:493-496),
// sens and msk shared by the BS images of a group: one thread per voxel of a group moves
// the group's BS values with one vector access (blockIdx.y strides over the groups)

template <int BS>
__global__ void k_update_batch(float *__restrict__ img, float *__restrict__ bimg,
                               const float *__restrict__ sens, const uint8_t *__restrict__ msk,
                               int ngroups) {
  using V = typename nbb::VecF<BS>::T;
  const size_t nvox = (size_t)NB_NCOL * NB_COLW;
  for (int grp = blockIdx.y; grp < ngroups; grp += gridDim.y) {
    V *gi = reinterpret_cast<V *>(img + (size_t)grp * nvox * BS);
    V *gb = reinterpret_cast<V *>(bimg + (size_t)grp * nvox * BS);
    for (size_t v = blockIdx.x * (size_t)blockDim.x + threadIdx.x; v < nvox;
         v += (size_t)gridDim.x * blockDim.x) {
      const float s = sens[v];
      const bool keep = msk[v] != 0;
      const bool zero_s = s > -0.000001f && s < 0.000001f;
      V x = gi[v];
      const V b = gb[v];
      float *xp = reinterpret_cast<float *>(&x);
      const float *bp = reinterpret_cast<const float *>(&b);
#pragma unroll
      for (int k = 0; k < BS; k++) {
        const float q = zero_s ? 0.f : __fdiv_rn(bp[k], s);
        xp[k] = keep ? xp[k] * q : 0.f;
      }
      gi[v] = x;
      V z;
      float *zp = reinterpret_cast<float *>(&z);
#pragma unroll
      for (int k = 0; k < BS; k++) zp[k] = 0.f;
      gb[v] = z;
    }
  }
}

template <int BS, int CH, int NOUT, int NT, int RPT, int MODE = nbb::BMODE_OSEM>
int launch_batch(nb_geom *g, const nbb::BatchArgs &a, cudaStream_t s) {
  static_assert(NT * RPT >= NB_NRAYS, "not enough ray slots");
  static_assert(nbb::BSmem<BS, CH>::template misc_off<NOUT>() % 128 == 0, "misaligned barriers");
  static_assert(nbb::BSmem<BS, CH>::template total<NOUT>() <= 227 * 1024, "too much shared memory");
  const size_t smem = nbb::BSmem<BS, CH>::template total<NOUT>();
  // the shared-memory opt-in is set once per device and kernel shape; host threads may
  // launch concurrently, so the flags are atomics (setting the attribute twice is harmless)
  static std::atomic<bool> set[64];
  if (!set[g->device & 63].load(std::memory_order_acquire)) {
    NB_CUDA(cudaFuncSetAttribute(nbb::k_osem_batch<BS, CH, NOUT, NT, RPT, MODE>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    set[g->device & 63].store(true, std::memory_order_release);
  }
  const long jobs = (long)a.nprj * a.ngroups;
  const int grid = jobs < g->nsm ? (int)jobs : g->nsm;
  if (grid <= 0) return NB_OK;
  nbb::k_osem_batch<BS, CH, NOUT, NT, RPT, MODE><<<grid, NT, smem, s>>>(a);
  NB_CUDA(cudaGetLastError());
  return NB_OK;
}

// geometry fields of the batched kernels' arguments
void batch_geometry(nb_geom *g, nbb::BatchArgs &a, int nrep, int bs, int span,
                    const int32_t *subs, int nprj) {
  a.scol = g->d_scol;
  a.st = g->d_st;
  a.hdr = g->d_hdr;
  a.rays = g->d_rays;
  a.bin11 = g->d_bin11;
  a.bin1 = g->d_bin1;
  a.subs = subs;
  a.nprj = nprj;
  a.naw = g->naw;
  a.span = span;
  a.ngroups = (nrep + bs - 1) / bs;
  a.nrep = nrep;
  a.fxbits = g->fxbits;
  a.err = g->d_err;
}

// forward (MODE_FWD) or back (MODE_BWD) projection of nrep batched images, default tile
template <int MODE> int launch_batch_prj(nb_geom *g, const nbb::BatchArgs &a, int bs, int span,
                                         cudaStream_t s) {
  if (span == 11) {
    if (bs == 4) return launch_batch<4, 16, NB_NSN11, 1024, 4, MODE>(g, a, s);
    if (bs == 2) return launch_batch<2, 32, NB_NSN11, 1024, 4, MODE>(g, a, s);
    return launch_batch<1, 64, NB_NSN11, 1024, 4, MODE>(g, a, s);
  }
  if (bs == 4) return launch_batch<4, 8, NB_NSN1, 1024, 4, MODE>(g, a, s);
  if (bs == 2) return launch_batch<2, 32, NB_NSN1, 1024, 4, MODE>(g, a, s);
  return launch_batch<1, 64, NB_NSN1, 1024, 4, MODE>(g, a, s);
}

}  // namespace

extern "C" int nb_to_batch(float *dst, const float *src, int nrep, int bs, void *stream) {
  NB_REQUIRE(dst && src && nrep > 0 && (bs == 1 || bs == 2 || bs == 4),
             "nb_to_batch: bad arguments");
  NB_CUDA(cudaMemsetAsync(dst, 0,
                          sizeof(float) * (size_t)((nrep + bs - 1) / bs) * bs * NB_NCOL * NB_COLW,
                          (cudaStream_t)stream));
  k_to_batch<<<4096, 256, 0, (cudaStream_t)stream>>>(dst, src, nrep, bs);
  NB_CUDA(cudaGetLastError());
  return NB_OK;
}

extern "C" int nb_fill_batch(float *dst, float value, int nrep, int bs, void *stream) {
  NB_REQUIRE(dst && nrep > 0 && (bs == 1 || bs == 2 || bs == 4), "nb_fill_batch: bad arguments");
  const size_t n = (size_t)((nrep + bs - 1) / bs) * bs * NB_NCOL * NB_COLW;
  k_fill_batch<<<4096, 256, 0, (cudaStream_t)stream>>>(dst, value, nrep, bs, n);
  NB_CUDA(cudaGetLastError());
  return NB_OK;
}

extern "C" int nb_from_batch(float *dst, const float *src, int nrep, int bs, void *stream) {
  NB_REQUIRE(dst && src && nrep > 0 && (bs == 1 || bs == 2 || bs == 4),
             "nb_from_batch: bad arguments");
  k_from_batch<<<4096, 256, 0, (cudaStream_t)stream>>>(dst, src, nrep, bs);
  NB_CUDA(cudaGetLastError());
  return NB_OK;
}

extern "C" int nb_osem_batch_subset(nb_geom *g, float *img, float *bimg, const float *sens128,
                                    const uint8_t *msk128, const uint16_t *psng, const float *rs,
                                    const float *rscale, int nrep, int bs, int tile,
                                    int span, const int32_t *subs, int nprj, void *stream) {
  NB_RANGE("nb_osem_batch_subset");
  NB_REQUIRE(g != nullptr, "nb_osem_batch_subset: NULL geometry handle");
  NB_REQUIRE(img && bimg && sens128 && msk128 && psng && rs && rscale && subs,
             "nb_osem_batch_subset: NULL argument");
  NB_REQUIRE(nrep > 0 && nrep <= nbb::NB_MAXREP, "nb_osem_batch_subset: nrep out of range");
  NB_REQUIRE(span == 11 || span == 1, "nb_osem_batch_subset: span must be 1 or 11");
  NB_REQUIRE(bs == 1 || bs == 2 || bs == 4, "nb_osem_batch_subset: bs must be 1, 2 or 4");
  NB_REQUIRE(tile >= 0 && tile <= 2, "nb_osem_batch_subset: tile must be 0, 1 or 2");
  NB_REQUIRE(nprj > 0, "nb_osem_batch_subset: empty subset");
  NB_CUDA(cudaSetDevice(g->device));
  cudaStream_t s = (cudaStream_t)stream;
  const int ngroups = (nrep + bs - 1) / bs;
  nbb::BatchArgs a{};
  batch_geometry(g, a, nrep, bs, span, subs, nprj);
  a.img = img;
  a.bimg = bimg;
  a.psng = psng;
  a.rs = rs;
  a.rscale = rscale;
  // kernel shape per (span, bs, tile): columns per staged chunk (CH), threads (NT) and
  // rays per thread (RPT); CH * 128 * bs floats per chunk buffer
#define NB_TILES(BS, CH, NOUT)                                                            \
  (tile == 0   ? launch_batch<BS, CH, NOUT, 1024, 4>(g, a, s)                             \
   : tile == 1 ? launch_batch<BS, CH / 2, NOUT, 1024, 4>(g, a, s)                         \
               : launch_batch<BS, CH, NOUT, 512, 8>(g, a, s))
  int st;
  if (span == 11) {
    if (bs == 4)
      st = NB_TILES(4, 16, NB_NSN11);
    else if (bs == 2)
      st = NB_TILES(2, 32, NB_NSN11);
    else
      st = NB_TILES(1, 64, NB_NSN11);
  } else {
    // span 1: a LOR's ratio rows are 4084 x bs floats, so 4 images stage 8 columns per
    // chunk (16 would need 257 KB of shared memory)
    if (bs == 4)
      st = NB_TILES(4, 8, NB_NSN1);
    else if (bs == 2)
      st = NB_TILES(2, 32, NB_NSN1);
    else
      st = NB_TILES(1, 64, NB_NSN1);
  }
#undef NB_TILES
  if (st) return st;
  const dim3 ugrid(g->nsm * 4, ngroups < 16 ? ngroups : 16);
  if (bs == 4)
    k_update_batch<4><<<ugrid, 256, 0, s>>>(img, bimg, sens128, msk128, ngroups);
  else if (bs == 2)
    k_update_batch<2><<<ugrid, 256, 0, s>>>(img, bimg, sens128, msk128, ngroups);
  else
    k_update_batch<1><<<ugrid, 256, 0, s>>>(img, bimg, sens128, msk128, ngroups);
  NB_CUDA(cudaGetLastError());
  return NB_OK;
}

extern "C" int nb_psf_col128(float *dst128, const float *src128, const float *krnl,
                             float *tmp128, void *stream);

// One span-1 OSEM sub-iteration of one image (the reference's osem() with Cnt.SPN == 1,
// recon.cu:318-497): the batched kernel with one image per walk, whose layout is the col128
// image itself, then the update; with a PSF kernel (krnl, [3][17], may be NULL) the forward
// projection sees the convolved image and the back projection is convolved before the
// update, as nb_osem_subset_psf does at span 11.  work128: two col128 images (PSF only).
extern "C" int nb_osem_subset_span1(nb_geom *g, float *img128, float *bimg128,
                                    const float *sens128, const uint8_t *msk128,
                                    const uint16_t *psng, const float *rs, const int32_t *subs,
                                    int nprj, const float *krnl, float *work128, void *stream) {
  NB_RANGE("nb_osem_subset_span1");
  NB_REQUIRE(g != nullptr, "nb_osem_subset_span1: NULL geometry handle");
  NB_REQUIRE(img128 && bimg128 && sens128 && msk128 && psng && rs && subs,
             "nb_osem_subset_span1: NULL argument");
  NB_REQUIRE(!krnl || work128, "nb_osem_subset_span1: the PSF needs work128");
  NB_REQUIRE(nprj > 0 && nprj <= g->naw, "nb_osem_subset_span1: bad subset size");
  NB_CUDA(cudaSetDevice(g->device));
  cudaStream_t s = (cudaStream_t)stream;
  float *rm = krnl ? work128 : nullptr, *tmp = krnl ? work128 + NB_IMG_COL128 : nullptr;
  if (krnl) {
    const int st = nb_psf_col128(rm, img128, krnl, tmp, stream);
    if (st) return st;
  }
  NB_CUDA(cudaMemsetAsync(bimg128, 0, sizeof(float) * NB_IMG_COL128, s));
  int st = NB_OK;
  cudaError_t e = cudaSuccess;
  {
    nbb::BatchArgs a{};
    batch_geometry(g, a, 1, 1, 1, subs, nprj);
    a.img = krnl ? rm : img128;
    a.bimg = bimg128;
    a.psng = psng;
    a.rs = rs;
    a.rscale = g->d_one;  // the randoms factor of the single image
    st = launch_batch<1, 64, NB_NSN1, 1024, 4>(g, a, s);
    if (!st && krnl) st = nb_psf_col128(rm, bimg128, krnl, tmp, stream);
    if (!st) {
      k_update_batch<1><<<dim3(g->nsm * 4, 1), 256, 0, s>>>(img128, krnl ? rm : bimg128,
                                                            sens128, msk128, 1);
      e = cudaGetLastError();
    }
  }
  if (e != cudaSuccess) return nb_cuda_fail(e, "nb_osem_subset_span1", __FILE__, __LINE__);
  return st;
}

extern "C" int nb_fprj_batch(nb_geom *g, float *sino, const float *img, int nrep, int bs,
                             int span, const int32_t *subs, int nprj, void *stream) {
  NB_RANGE("nb_fprj_batch");
  NB_REQUIRE(g != nullptr, "nb_fprj_batch: NULL geometry handle");
  NB_REQUIRE(sino && img, "nb_fprj_batch: NULL argument");
  NB_REQUIRE(nrep > 0 && nrep <= nbb::NB_MAXREP, "nb_fprj_batch: nrep out of range");
  NB_REQUIRE(span == 11 || span == 1, "nb_fprj_batch: span must be 1 or 11");
  NB_REQUIRE(bs == 1 || bs == 2 || bs == 4, "nb_fprj_batch: bs must be 1, 2 or 4");
  NB_REQUIRE(nprj > 0 && (subs != nullptr || nprj == g->naw), "nb_fprj_batch: bad subset");
  NB_CUDA(cudaSetDevice(g->device));
  nbb::BatchArgs a{};
  batch_geometry(g, a, nrep, bs, span, subs, nprj);
  a.img = img;
  a.sino_out = sino;
  return launch_batch_prj<nbb::BMODE_FWD>(g, a, bs, span, (cudaStream_t)stream);
}

extern "C" int nb_bprj_batch(nb_geom *g, float *bimg, const float *sino, int nrep, int bs,
                             int span, const int32_t *subs, int nprj, void *stream) {
  NB_RANGE("nb_bprj_batch");
  NB_REQUIRE(g != nullptr, "nb_bprj_batch: NULL geometry handle");
  NB_REQUIRE(sino && bimg, "nb_bprj_batch: NULL argument");
  NB_REQUIRE(nrep > 0 && nrep <= nbb::NB_MAXREP, "nb_bprj_batch: nrep out of range");
  NB_REQUIRE(span == 11 || span == 1, "nb_bprj_batch: span must be 1 or 11");
  NB_REQUIRE(bs == 1 || bs == 2 || bs == 4, "nb_bprj_batch: bs must be 1, 2 or 4");
  NB_REQUIRE(nprj > 0 && (subs != nullptr || nprj == g->naw), "nb_bprj_batch: bad subset");
  NB_CUDA(cudaSetDevice(g->device));
  nbb::BatchArgs a{};
  batch_geometry(g, a, nrep, bs, span, subs, nprj);
  a.bimg = bimg;
  a.sino_in = sino;
  return launch_batch_prj<nbb::BMODE_BWD>(g, a, bs, span, (cudaStream_t)stream);
}
