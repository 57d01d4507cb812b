// nb_prj.cu -- Siddon forward / back projectors and the fused OSEM sub-iteration.
//
// Reference semantics: prj/src/prjf.cu:33-206 (fprj_drct, fprj_oblq), prj/src/prjb.cu:33-187
// (bprj_drct, bprj_oblq), prj/src/recon.cu:220-316 and :459-497 (OSEM sub-iteration).
//
// B200 design
//  * Persistent grid, one 1024-thread CTA per SM.  A CTA owns one LOR (a transaxial
//    sinogram bin) at a time and computes all 4084 rays (span-1 ring pairs) of it;
//    thread t handles rays t, t+1024, t+2048, t+3072.
//  * The LOR's voxel columns (512 B each in the col128 layout) are streamed into shared
//    memory in chunks of CH columns with TMA bulk copies (cp.async.bulk + mbarrier),
//    double buffered, so every voxel read of the walk is a shared-memory load.
//  * Span-11 sinograms are formed by a deterministic in-CTA sum over the span-1 rays
//    (no global atomics, run-to-run identical); each CTA writes whole sinogram rows.
//  * Back projection accumulates the LOR's columns in shared memory (shared atomics)
//    and flushes each finished chunk to the image with one TMA bulk reduce-add per
//    column (cp.reduce.async.bulk .add.f32), instead of one global atomic per voxel
//    visit as in the reference.
//  * The OSEM kernel fuses, per LOR: forward projection, ratio y / (Ax + (r+s)/(an)),
//    and the back projection of the ratio -- the subset sinogram never touches HBM.
#include <math.h>

#include "nb_axial.cuh"
#include "nb_internal.cuh"

namespace {

constexpr int NT = 1024;   // threads per CTA
constexpr int RPT = 4;     // rays per thread (NT * RPT >= 4084)
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
  int span;        // 1 or 11
  int att;         // forward: 0 emission, 1 attenuation
  const float *img;      // col128 image read by forward passes
  float *bimg;           // col128 image accumulated by backward passes
  float *sino;           // forward output [nprj][nout]
  const float *sino_in;  // backward input [nprj][nout]
  const uint16_t *psng;  // OSEM prompts [naw][nout]
  const float *rs;       // OSEM (r+s)/(an) [naw][nout]
  int *err;
};

template <int CH> struct Smem {
  static constexpr size_t cols_off = 0;
  static constexpr size_t cols_bytes = 2ull * CH * NB_COLW * sizeof(float);
  static constexpr size_t tn_off = cols_off + cols_bytes;
  static constexpr size_t tn_bytes = 2ull * CH * sizeof(float);
  static constexpr size_t vals_off = tn_off + tn_bytes;
  static constexpr size_t vals_bytes = 4096 * sizeof(float);
  static constexpr size_t rat_off = vals_off + vals_bytes;
  static constexpr size_t rat_bytes = 4096 * sizeof(float);
  static constexpr size_t bar_off = rat_off + rat_bytes;
  static constexpr size_t total = bar_off + 64;
};

struct Job {
  int p;       // sinogram row
  int lor;     // LOR index (subs[p])
  int n;       // steps of the LOR
  int nch;     // chunks per pass
  int c;       // chunk index within the LOR's job list (OSEM: [0,nch) fwd, [nch,2nch) bwd)
  int valid;
};

template <int MODE, int CH>
__device__ __forceinline__ void job_load(const PrjArgs &a, int p, Job &J) {
  J.p = p;
  J.valid = p < a.nprj;
  J.c = 0;
  if (!J.valid) return;
  int lor = a.subs ? a.subs[p] : p;
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
  if (++J.c >= per_lor) job_load<MODE, CH>(a, J.p + gridDim.x, J);
}

template <int MODE, int CH> __device__ __forceinline__ bool job_is_load(const Job &J) {
  if (MODE == MODE_FWD) return true;
  if (MODE == MODE_BWD) return false;
  return J.c < J.nch;
}

// Warp 0: enqueue the TMA loads of one forward chunk (its columns + exit parameters).
template <int CH>
__device__ __forceinline__ void issue_load(const PrjArgs &a, const Job &J, int chunk, float *cols,
                                           float *tnb, uint64_t *bar) {
  const int lane = threadIdx.x & 31;
  const int s0 = chunk * CH;
  const int n = max(0, min(CH, J.n - s0));
  const uint32_t tn_bytes = max(16u, (uint32_t)((n * 4 + 15) & ~15));
  if (lane == 0) nb_mbar_arrive_expect_tx(bar, (uint32_t)n * (NB_COLW * 4) + tn_bytes);
  __syncwarp();
  const int32_t *sc = a.scol + (size_t)J.lor * NB_STEP_STRIDE + s0;
  for (int i = lane; i < n; i += 32) {
    int col = sc[i];
    nb_bulk_g2s(cols + (size_t)i * NB_COLW, a.img + (size_t)col * NB_COLW, NB_COLW * 4, bar);
  }
  if (lane == 0) nb_bulk_g2s(tnb, a.st + (size_t)J.lor * NB_STEP_STRIDE + s0, tn_bytes, bar);
}

struct RayState {
  float acc[RPT];  // forward: running line integral; backward: value to spread (bin * s)
  float tzc[RPT];
  float dtz[RPT];
  float s[RPT];
  int w[RPT];
  int zi[RPT];
  int dir[RPT];
  float tp;
};

__device__ __forceinline__ void rays_init(const PrjArgs &a, const Job &J, RayState &S) {
  const float4 h = a.hdr[J.lor];
  S.tp = h.x;
#pragma unroll
  for (int r = 0; r < RPT; r++) {
    const int ray = threadIdx.x + NT * r;
    S.acc[r] = 0.f;
    if (ray < NB_NRAYS) {
      nb_ray R = a.rays[ray];
      nb_axial A;
      nb_axial_setup(R, h.y, h.x, h.z, A);
      S.w[r] = nb_clampz(A.w);
      S.zi[r] = nb_zi(S.w[r]);
      S.tzc[r] = A.tzc;
      S.dtz[r] = A.dtz;
      S.dir[r] = A.dir;
      S.s[r] = A.s;
    } else {
      S.w[r] = 127;
      S.zi[r] = 127;
      S.tzc[r] = __int_as_float(0x7f800000);
      S.dtz[r] = 0.f;
      S.dir[r] = 0;
      S.s[r] = 0.f;
    }
  }
}

// The walk over n steps of one shared-memory chunk (prjf.cu:76-86 / :164-190 and the
// transposed prjb.cu:70-77 / :153-178).  A ray crosses at most one z plane per step.
template <bool BWD>
__device__ __forceinline__ void walk_chunk(RayState &S, float *col0, const float *tnb, int n) {
  float tp = S.tp;
  for (int i = 0; i < n; ++i) {
    const float tn = tnb[i];
    const float lt = __fsub_rn(tn, tp);
    float *col = col0 + i * NB_COLW;
#pragma unroll
    for (int r = 0; r < RPT; r++) {
      if (__fsub_rn(tn, S.tzc[r]) > 0.f) {
        const float fa = __fsub_rn(S.tzc[r], tp);
        const float fb = __fsub_rn(tn, S.tzc[r]);
        if (BWD) {
          atomicAdd(col + S.zi[r], fa * S.acc[r]);
        } else {
          S.acc[r] = fmaf(fa, col[S.zi[r]], S.acc[r]);
        }
        S.w[r] = nb_clampz(S.w[r] + S.dir[r]);
        S.zi[r] = nb_zi(S.w[r]);
        if (BWD) {
          atomicAdd(col + S.zi[r], fb * S.acc[r]);
        } else {
          S.acc[r] = fmaf(fb, col[S.zi[r]], S.acc[r]);
        }
        S.tzc[r] = __fadd_rn(S.tzc[r], S.dtz[r]);
      } else {
        if (BWD) {
          atomicAdd(col + S.zi[r], lt * S.acc[r]);
        } else {
          S.acc[r] = fmaf(lt, col[S.zi[r]], S.acc[r]);
        }
      }
    }
    tp = tn;
  }
  S.tp = tp;
}

template <int MODE, int CH>
__global__ void __launch_bounds__(NT, 1) k_project(const PrjArgs a) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  using L = Smem<CH>;
  float *cols = reinterpret_cast<float *>(smem_raw + L::cols_off);
  float *tnbuf = reinterpret_cast<float *>(smem_raw + L::tn_off);
  float *vals = reinterpret_cast<float *>(smem_raw + L::vals_off);
  float *rat = reinterpret_cast<float *>(smem_raw + L::rat_off);
  uint64_t *bars = reinterpret_cast<uint64_t *>(smem_raw + L::bar_off);
  int *sflag = reinterpret_cast<int *>(smem_raw + L::bar_off + 16);

  const int tid = threadIdx.x;
  const bool warp0 = tid < 32;
  const int nout = a.span == 11 ? NB_NSN11 : NB_NSN1;

  if (tid == 0) {
    nb_mbar_init(&bars[0], 1);
    nb_mbar_init(&bars[1], 1);
    *sflag = 0;
    nb_fence_mbar_init();
  }
  __syncthreads();

  Job J, P;  // consumer cursor, producer cursor
  job_load<MODE, CH>(a, blockIdx.x, J);
  P = J;
  // prologue: the first two jobs
  if (MODE != MODE_BWD) {
    for (int k = 0; k < 2; k++) {
      if (!P.valid) break;
      if (job_is_load<MODE, CH>(P) && warp0)
        issue_load<CH>(a, P, P.c, cols + (size_t)k * CH * NB_COLW, tnbuf + k * CH, &bars[k]);
      job_next<MODE, CH>(a, P);
    }
  }

  RayState S;
  uint32_t phase = 0;  // bit b: parity of the next completion of bars[b]
  int j = 0;
  while (J.valid) {
    const int b = j & 1;
    float *cb = cols + (size_t)b * CH * NB_COLW;
    float *tb = tnbuf + b * CH;
    const bool load = job_is_load<MODE, CH>(J);
    const int chunk = (MODE == MODE_OSEM && !load) ? J.c - J.nch : J.c;
    const int n = max(0, min(CH, J.n - chunk * CH));

    if (chunk == 0) {
      rays_init(a, J, S);
      if (MODE == MODE_BWD) {
#pragma unroll
        for (int r = 0; r < RPT; r++) {
          const int ray = tid + NT * r;
          float v = 0.f;
          if (ray < NB_NRAYS) {
            const nb_ray R = a.rays[ray];
            v = a.sino_in[(size_t)J.p * nout + (a.span == 11 ? R.out11 : R.out1)] * S.s[r];
          }
          S.acc[r] = v;
        }
      } else if (MODE == MODE_OSEM && !load) {
#pragma unroll
        for (int r = 0; r < RPT; r++) {
          const int ray = tid + NT * r;
          float v = 0.f;
          if (ray < NB_NRAYS) {
            const nb_ray R = a.rays[ray];
            v = rat[a.span == 11 ? R.out11 : R.out1] * S.s[r];
          }
          S.acc[r] = v;
        }
      }
    }

    if (load) {
      if (!nb_mbar_wait(&bars[b], (phase >> b) & 1u, WAIT_POLLS)) atomicExch(sflag, 1);
      phase ^= 1u << b;
      walk_chunk<false>(S, cb, tb, n);
    } else {
      // backward chunk: make sure the bulk reduce that last read this buffer is done
      if (warp0) nb_bulk_wait_read<1>();
      __syncthreads();
      for (int i = tid; i < n * NB_COLW; i += NT) cb[i] = 0.f;
      if (tid < n) tb[tid] = a.st[(size_t)J.lor * NB_STEP_STRIDE + chunk * CH + tid];
      __syncthreads();
      walk_chunk<true>(S, cb, tb, n);
      nb_fence_proxy_async_smem();
    }

    // forward epilogue at the end of the LOR's forward pass
    if (load && chunk == J.nch - 1) {
#pragma unroll
      for (int r = 0; r < RPT; r++) {
        const int ray = tid + NT * r;
        if (ray < NB_NRAYS) {
          float v = S.acc[r] * S.s[r];
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

    __syncthreads();  // everyone is done with buffer b (and rat is complete)
    if (*sflag) break;

    if (warp0) {
      if (MODE != MODE_FWD) {
        // flush a finished backward chunk: one bulk reduce-add per column
        if (!load) {
          const int32_t *sc = a.scol + (size_t)J.lor * NB_STEP_STRIDE + chunk * CH;
          for (int i = tid; i < n; i += 32)
            nb_bulk_reduce_add_f32(a.bimg + (size_t)sc[i] * NB_COLW, cb + (size_t)i * NB_COLW,
                                   NB_COLW * 4);
        }
        nb_bulk_commit();  // one group per job and lane (empty for forward jobs)
      }
      // producer: job j+2 reuses buffer b
      if (MODE != MODE_BWD && P.valid) {
        if (job_is_load<MODE, CH>(P)) {
          if (MODE == MODE_OSEM) nb_bulk_wait_read<0>();
          issue_load<CH>(a, P, P.c, cb, tb, &bars[b]);
        }
        job_next<MODE, CH>(a, P);
      } else if (MODE == MODE_BWD && P.valid) {
        job_next<MODE, CH>(a, P);
      }
    }
    job_next<MODE, CH>(a, J);
    ++j;
  }
  if (*sflag && tid == 0) nb_set_error(a.err, NB_DEVERR_MBAR_TIMEOUT);
  if (warp0 && MODE != MODE_FWD) nb_bulk_wait_all<0>();
}

// ---------------------------------------------------------------------------------------
// layout conversion and element-wise kernels
// ---------------------------------------------------------------------------------------
// reference [320][320][127] -> col128 (one warp per column)
__global__ void k_to_col128(float *__restrict__ dst, const float *__restrict__ src, int ncols) {
  const int wid = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (wid >= ncols) return;
  const float *s = src + (size_t)wid * NB_IMZ;
  float *d = dst + (size_t)wid * NB_COLW;
  for (int z = lane; z < NB_COLW; z += 32) {
    float v = z < NB_IMZ ? s[z] : 0.f;
    d[nb_zi(z)] = z < NB_IMZ ? v : 0.f;
  }
}

__global__ void k_from_col128(float *__restrict__ dst, const float *__restrict__ src, int ncols) {
  const int wid = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (wid >= ncols) return;
  const float *s = src + (size_t)wid * NB_COLW;
  float *d = dst + (size_t)wid * NB_IMZ;
  for (int z = lane; z < NB_IMZ; z += 32) d[z] = s[nb_zi(z)];
}

__global__ void k_osem_rs(float *__restrict__ rs, const float *__restrict__ r,
                          const float *__restrict__ s, const float *__restrict__ an_a,
                          const float *__restrict__ an_n, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    // recon.cu:381-398: rsng += ssng; ansng = asng * nsng; rsng = eldiv0(rsng, ansng)
    const float num = s ? __fadd_rn(r[i], s[i]) : r[i];
    const float an = __fmul_rn(an_a[i], an_n[i]);
    rs[i] = (an > -0.000001f && an < 0.000001f) ? 0.f : __fdiv_rn(num, an);
  }
}

// img = msk ? img * (|sens| < 1e-6 ? 0 : bimg / sens) : 0;  bimg = 0   (recon.cu:493-496)
__global__ void k_osem_update(float4 *__restrict__ img, float4 *__restrict__ bimg,
                              const float4 *__restrict__ sens, const uchar4 *__restrict__ msk,
                              size_t n4) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n4;
       i += (size_t)gridDim.x * blockDim.x) {
    float4 x = img[i], b = bimg[i], s = sens[i];
    uchar4 m = msk[i];
#define UPD(c)                                                                                 \
  {                                                                                            \
    float q = (s.c > -0.000001f && s.c < 0.000001f) ? 0.f : __fdiv_rn(b.c, s.c);               \
    x.c = m.c ? x.c * q : 0.f;                                                                 \
  }
    UPD(x) UPD(y) UPD(z) UPD(w)
#undef UPD
    img[i] = x;
    bimg[i] = make_float4(0.f, 0.f, 0.f, 0.f);
  }
}

// V: voxel reads of a full forward projection, one thread per (LOR, oblique pair)
__global__ void k_count_reads(const float4 *__restrict__ hdr, const float *__restrict__ st,
                              const nb_ray *__restrict__ rays, int naw,
                              unsigned long long *out) {
  const int lor = blockIdx.x;
  if (lor >= naw) return;
  const float4 h = hdr[lor];
  const int n = __float_as_int(h.w);
  unsigned long long tot = 0;
  for (int li = NB_NRINGS + threadIdx.x; li < NB_NLI2R; li += blockDim.x) {
    nb_axial A;
    nb_axial_setup(rays[li], h.y, h.x, h.z, A);
    float tzc = A.tzc;
    for (int k = 0; k < n; k++) {
      float tn = st[(size_t)lor * NB_STEP_STRIDE + k];
      if (__fsub_rn(tn, tzc) > 0.f) {
        tot += 4;
        tzc = __fadd_rn(tzc, A.dtz);
      } else
        tot += 2;
    }
  }
  if (threadIdx.x == 0) tot += (unsigned long long)NB_NRINGS * n;
  atomicAdd(out, tot);
}

template <int MODE, int CH>
int launch_project(nb_geom *g, const PrjArgs &a, cudaStream_t stream) {
  const size_t smem = Smem<CH>::total;
  static bool attr_set[64] = {false};
  if (!attr_set[g->device & 63]) {
    NB_CUDA(cudaFuncSetAttribute(k_project<MODE, CH>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem));
    attr_set[g->device & 63] = true;
  }
  if (a.nprj <= 0) return NB_OK;
  const int grid = a.nprj < g->nsm ? a.nprj : g->nsm;
  k_project<MODE, CH><<<grid, NT, smem, stream>>>(a);
  NB_CUDA(cudaGetLastError());
  return NB_OK;
}

constexpr int CH_DEFAULT = 64;

PrjArgs base_args(nb_geom *g, const int32_t *subs, int nprj, int span) {
  PrjArgs a{};
  a.scol = g->d_scol;
  a.st = g->d_st;
  a.hdr = g->d_hdr;
  a.rays = g->d_rays;
  a.bin11 = g->d_bin11;
  a.bin1 = g->d_bin1;
  a.subs = subs;
  a.nprj = subs ? nprj : g->naw;
  a.naw = g->naw;
  a.span = span;
  a.err = g->d_err;
  return a;
}

int check_common(nb_geom *g, int nprj, const int32_t *subs, int span) {
  NB_REQUIRE(g != nullptr, "NULL geometry handle");
  NB_REQUIRE(span == 1 || span == 11, "span must be 1 or 11");
  NB_REQUIRE(subs == nullptr || nprj >= 0, "nprj must be >= 0");
  NB_CUDA(cudaSetDevice(g->device));
  return NB_OK;
}

}  // namespace

// ---------------------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------------------
extern "C" int nb_im_to_col128(float *im128, const float *im, int nimg, void *stream) {
  NB_REQUIRE(im128 && im && nimg > 0, "nb_im_to_col128: bad arguments");
  const int ncols = NB_NCOL * nimg;
  k_to_col128<<<(ncols * 32 + 255) / 256, 256, 0, (cudaStream_t)stream>>>(im128, im, ncols);
  NB_CUDA(cudaGetLastError());
  return NB_OK;
}

extern "C" int nb_col128_to_im(float *im, const float *im128, int nimg, void *stream) {
  NB_REQUIRE(im128 && im && nimg > 0, "nb_col128_to_im: bad arguments");
  const int ncols = NB_NCOL * nimg;
  k_from_col128<<<(ncols * 32 + 255) / 256, 256, 0, (cudaStream_t)stream>>>(im, im128, ncols);
  NB_CUDA(cudaGetLastError());
  return NB_OK;
}

extern "C" int nb_fprj_col128(nb_geom *g, float *sino, const float *im128, const int32_t *subs,
                              int nprj, int span, int att, void *stream) {
  int st = check_common(g, nprj, subs, span);
  if (st) return st;
  NB_REQUIRE(sino && im128, "nb_fprj_col128: NULL sino or image");
  NB_REQUIRE(att == 0 || att == 1, "att must be 0 or 1");
  PrjArgs a = base_args(g, subs, nprj, span);
  a.att = att;
  a.img = im128;
  a.sino = sino;
  return launch_project<MODE_FWD, CH_DEFAULT>(g, a, (cudaStream_t)stream);
}

extern "C" int nb_bprj_col128(nb_geom *g, float *im128, const float *sino, const int32_t *subs,
                              int nprj, int span, void *stream) {
  int st = check_common(g, nprj, subs, span);
  if (st) return st;
  NB_REQUIRE(sino && im128, "nb_bprj_col128: NULL sino or image");
  PrjArgs a = base_args(g, subs, nprj, span);
  a.bimg = im128;
  a.sino_in = sino;
  return launch_project<MODE_BWD, CH_DEFAULT>(g, a, (cudaStream_t)stream);
}

extern "C" int nb_fprj(nb_geom *g, float *sino, const float *im, const int32_t *subs, int nprj,
                       int span, int att, void *stream) {
  int st = check_common(g, nprj, subs, span);
  if (st) return st;
  NB_REQUIRE(sino && im, "nb_fprj: NULL sino or image");
  st = nb_im_to_col128(g->d_scratch128, im, 1, stream);
  if (st) return st;
  return nb_fprj_col128(g, sino, g->d_scratch128, subs, nprj, span, att, stream);
}

extern "C" int nb_bprj(nb_geom *g, float *im, const float *sino, const int32_t *subs, int nprj,
                       int span, void *stream) {
  int st = check_common(g, nprj, subs, span);
  if (st) return st;
  NB_REQUIRE(sino && im, "nb_bprj: NULL sino or image");
  NB_CUDA(cudaMemsetAsync(g->d_scratch128, 0, sizeof(float) * NB_IMG_COL128,
                          (cudaStream_t)stream));
  st = nb_bprj_col128(g, g->d_scratch128, sino, subs, nprj, span, stream);
  if (st) return st;
  return nb_col128_to_im(im, g->d_scratch128, 1, stream);
}

extern "C" int nb_osem_rs(float *rs, const float *rsng, const float *ssng, const float *asng,
                          const float *nsng, size_t n, void *stream) {
  NB_REQUIRE(rs && rsng && asng && nsng, "nb_osem_rs: NULL argument");
  if (n == 0) return NB_OK;
  k_osem_rs<<<1184, 256, 0, (cudaStream_t)stream>>>(rs, rsng, ssng, asng, nsng, n);
  NB_CUDA(cudaGetLastError());
  return NB_OK;
}

extern "C" int nb_osem_subset(nb_geom *g, float *img128, float *bimg128, const float *sens128,
                              const uint8_t *msk128, const uint16_t *psng, const float *rs,
                              const int32_t *subs, int nprj, void *stream) {
  int st = check_common(g, nprj, subs, 11);
  if (st) return st;
  NB_REQUIRE(img128 && bimg128 && sens128 && msk128 && psng && rs && subs,
             "nb_osem_subset: NULL argument");
  cudaStream_t s = (cudaStream_t)stream;
  NB_CUDA(cudaMemsetAsync(bimg128, 0, sizeof(float) * NB_IMG_COL128, s));
  PrjArgs a = base_args(g, subs, nprj, 11);
  a.img = img128;
  a.bimg = bimg128;
  a.psng = psng;
  a.rs = rs;
  st = launch_project<MODE_OSEM, CH_DEFAULT>(g, a, s);
  if (st) return st;
  const size_t n4 = NB_IMG_COL128 / 4;
  k_osem_update<<<g->nsm * 8, 256, 0, s>>>((float4 *)img128, (float4 *)bimg128,
                                           (const float4 *)sens128, (const uchar4 *)msk128, n4);
  NB_CUDA(cudaGetLastError());
  return NB_OK;
}

extern "C" int nb_geom_count_reads(nb_geom *g, long long *reads) {
  NB_REQUIRE(g && reads, "nb_geom_count_reads: NULL argument");
  NB_CUDA(cudaSetDevice(g->device));
  unsigned long long *d = nullptr;
  NB_CUDA(cudaMalloc(&d, sizeof(unsigned long long)));
  cudaMemset(d, 0, sizeof(unsigned long long));
  k_count_reads<<<g->naw, 128>>>(g->d_hdr, g->d_st, g->d_rays, g->naw, d);
  unsigned long long h = 0;
  cudaError_t e = cudaMemcpy(&h, d, sizeof(h), cudaMemcpyDeviceToHost);
  cudaFree(d);
  if (e != cudaSuccess) return nb_cuda_fail(e, "nb_geom_count_reads", __FILE__, __LINE__);
  *reads = (long long)h;
  return NB_OK;
}

// ---------------------------------------------------------------------------------------
// gap removal / insertion (scanner_0.cu:94-105, 158-166)
// ---------------------------------------------------------------------------------------
template <typename T>
__global__ void k_remgaps(T *__restrict__ sng, const T *__restrict__ sino, int snno,
                          const int32_t *__restrict__ aw2ali) {
  const size_t n = (size_t)NB_AW * snno;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n;
       k += (size_t)gridDim.x * blockDim.x) {
    const int aw = (int)(k / snno), i = (int)(k - (size_t)aw * snno);
    sng[k] = sino[(size_t)i * NB_NSBINANG + aw2ali[aw]];
  }
}

__global__ void k_putgaps(float *__restrict__ sino, const float *__restrict__ sng, int snno,
                          const int32_t *__restrict__ aw2ali) {
  const size_t n = (size_t)NB_AW * snno;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n;
       k += (size_t)gridDim.x * blockDim.x) {
    const int aw = (int)(k / snno), i = (int)(k - (size_t)aw * snno);
    sino[(size_t)i * NB_NSBINANG + aw2ali[aw]] = sng[k];
  }
}

extern "C" int nb_remgaps(float *sng, const float *sino, int snno, const int32_t *aw2ali,
                          void *stream) {
  NB_REQUIRE(sng && sino && aw2ali && snno > 0, "nb_remgaps: bad arguments");
  k_remgaps<float><<<2048, 256, 0, (cudaStream_t)stream>>>(sng, sino, snno, aw2ali);
  NB_CUDA(cudaGetLastError());
  return NB_OK;
}

extern "C" int nb_remgaps_u16(uint16_t *sng, const uint16_t *sino, int snno,
                              const int32_t *aw2ali, void *stream) {
  NB_REQUIRE(sng && sino && aw2ali && snno > 0, "nb_remgaps_u16: bad arguments");
  k_remgaps<uint16_t><<<2048, 256, 0, (cudaStream_t)stream>>>(sng, sino, snno, aw2ali);
  NB_CUDA(cudaGetLastError());
  return NB_OK;
}

extern "C" int nb_putgaps(float *sino, const float *sng, int snno, const int32_t *aw2ali,
                          void *stream) {
  NB_REQUIRE(sng && sino && aw2ali && snno > 0, "nb_putgaps: bad arguments");
  NB_CUDA(cudaMemsetAsync(sino, 0, sizeof(float) * (size_t)snno * NB_NSBINANG,
                          (cudaStream_t)stream));
  k_putgaps<<<2048, 256, 0, (cudaStream_t)stream>>>(sino, sng, snno, aw2ali);
  NB_CUDA(cudaGetLastError());
  return NB_OK;
}

extern "C" int nb_geom_check(nb_geom *g, void *stream) {
  NB_REQUIRE(g != nullptr, "nb_geom_check: NULL handle");
  NB_CUDA(cudaSetDevice(g->device));
  return nb_check_device_flag(g, (cudaStream_t)stream);
}

int nb_check_device_flag(nb_geom *g, cudaStream_t stream) {
  NB_CUDA(cudaStreamSynchronize(stream));
  int h = 0;
  NB_CUDA(cudaMemcpy(&h, g->d_err, sizeof(int), cudaMemcpyDeviceToHost));
  if (h) {
    cudaMemset(g->d_err, 0, sizeof(int));
    nb_set_error_msg("device-side error %d", h);
    return NB_ERR_DEVICE;
  }
  return NB_OK;
}
