// nb_prj.cu -- projector entry points, layout conversion, OSEM element-wise kernels and
// the sinogram gap kernels.  The projector kernel itself is in nb_project.cuh.
#include <math.h>

#include <atomic>

#include "nb_axial.cuh"
#include "nb_internal.cuh"
#include "nb_project.cuh"

namespace {

using namespace nbk;

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

// Images of a reduced ring range hold the axial slab [vz0, vz0 + nvz) only
// ([320][320][nvz], z fastest).  Expand: the slab into a full col128 image, zero elsewhere
// (prjf.cu:19-29 imExpand); reduce: the slab out of a col128 image (prjb.cu:19-29
// imReduce).  One warp per column.
__global__ void k_slab_to_col128(float *__restrict__ dst, const float *__restrict__ src,
                                 int nvz, int vz0) {
  const int wid = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (wid >= NB_NCOL) return;
  const float *s = src + (size_t)wid * nvz;
  float *d = dst + (size_t)wid * NB_COLW;
  for (int z = lane; z < NB_COLW; z += 32) {
    const int zr = z - vz0;
    d[nb_zi(z)] = (z < NB_IMZ && zr >= 0 && zr < nvz) ? s[zr] : 0.f;
  }
}

__global__ void k_col128_to_slab(float *__restrict__ dst, const float *__restrict__ src,
                                 int nvz, int vz0) {
  const int wid = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (wid >= NB_NCOL) return;
  const float *s = src + (size_t)wid * NB_COLW;
  float *d = dst + (size_t)wid * nvz;
  for (int z = lane; z < nvz; z += 32) d[z] = s[nb_zi(vz0 + z)];
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

// V: voxel reads of a full forward projection, one block per LOR
__global__ void k_count_reads(const float4 *__restrict__ hdr, const float *__restrict__ st,
                              const nb_ray *__restrict__ rays, int naw,
                              unsigned long long *out, unsigned long long *per_lor) {
  const int lor = blockIdx.x;
  if (lor >= naw) return;
  const float4 h = hdr[lor];
  const int n = __float_as_int(h.w);
  // per ray: one read per step, one more at each axial crossing (a +RD/-RD pair of the
  // reference: 2 per step, 4 at a crossing); direct rays never cross
  unsigned long long tot = 0;
  for (int ray = threadIdx.x; ray < NB_NRAYS; ray += blockDim.x) {
    nb_axial A;
    nb_axial_setup(rays[ray], h.y, h.x, h.z, A);
    float tzc = A.tzc;
    tot += n;
    for (int k = 0; k < n; k++) {
      const float tn = st[(size_t)lor * NB_STEP_STRIDE + k];
      if (tn > tzc) {
        tot += 1;
        tzc = __fadd_rn(tzc, A.dtz);
      }
    }
  }
  atomicAdd(out, tot);
  atomicAdd(per_lor + lor, tot);
}

template <int MODE, int CH>
int launch_project(nb_geom *g, const PrjArgs &a, cudaStream_t stream) {
  const size_t smem = Smem<MODE, CH>::total;
  // set once per device and kernel shape; atomics, since host threads may launch at once
  static std::atomic<bool> attr_set[64];
  if (!attr_set[g->device & 63].load(std::memory_order_acquire)) {
    NB_CUDA(cudaFuncSetAttribute(k_project<MODE, CH>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem));
    attr_set[g->device & 63].store(true, std::memory_order_release);
  }
  if (a.nprj <= 0) return NB_OK;
  const int grid = a.nprj < g->nsm ? a.nprj : g->nsm;
  k_project<MODE, CH><<<grid, NT, smem, stream>>>(a);
  NB_CUDA(cudaGetLastError());
  return NB_OK;
}

// columns per shared-memory chunk: the forward kernel double-buffers 2 x 64 KB of
// columns; the backward/OSEM kernels also hold the int32 accumulators
constexpr int CH_FWD = 128;
constexpr int CH_BWD = 64;

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
  a.nrays = NB_NRAYS;
  a.nout = span == 11 ? NB_NSN11 : NB_NSN1;
  a.span = span;
  a.fxbits = g->fxbits;
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
  NB_RANGE("nb_fprj");
  int st = check_common(g, nprj, subs, span);
  if (st) return st;
  NB_REQUIRE(sino && im128, "nb_fprj_col128: NULL sino or image");
  NB_REQUIRE(att == 0 || att == 1, "att must be 0 or 1");
  PrjArgs a = base_args(g, subs, nprj, span);
  a.att = att;
  a.img = im128;
  a.sino = sino;
  return launch_project<MODE_FWD, CH_FWD>(g, a, (cudaStream_t)stream);
}

extern "C" int nb_bprj_col128(nb_geom *g, float *im128, const float *sino, const int32_t *subs,
                              int nprj, int span, void *stream) {
  NB_RANGE("nb_bprj");
  int st = check_common(g, nprj, subs, span);
  if (st) return st;
  NB_REQUIRE(sino && im128, "nb_bprj_col128: NULL sino or image");
  PrjArgs a = base_args(g, subs, nprj, span);
  a.bimg = im128;
  a.sino_in = sino;
  return launch_project<MODE_BWD, CH_BWD>(g, a, (cudaStream_t)stream);
}

extern "C" int nb_sens_col128(nb_geom *g, float *sens128, const float *an, const int32_t *subs,
                              int nprj, int span, void *stream) {
  NB_RANGE("nb_sens");
  int st = check_common(g, nprj, subs, span);
  if (st) return st;
  NB_REQUIRE(sens128 && an, "nb_sens_col128: NULL image or sinogram");
  NB_CUDA(cudaMemsetAsync(sens128, 0, sizeof(float) * NB_IMG_COL128, (cudaStream_t)stream));
  PrjArgs a = base_args(g, subs, nprj, span);
  a.bimg = sens128;
  a.sino_in = an;
  a.in_by_lor = 1;
  return launch_project<MODE_BWD, CH_BWD>(g, a, (cudaStream_t)stream);
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

// Span-1 projections over a reduced ring range (gpu_fprj / gpu_bprj with Cnt.RNG_STRT /
// RNG_END, prjf.cu:209-320, prjb.cu:190-308): images are the range's axial slab
// [320][320][nvz], sinograms [nprj][nsino] numbered by the range's Michelogram.  The slab
// is expanded into the handle's col128 scratch with zeros elsewhere (as the reference's
// imExpand) and the persistent projector walks only the range's rays.
static int check_rings(nb_geom *g, const nb_rings *rr) {
  NB_REQUIRE(rr != nullptr, "NULL ring-range handle");
  NB_REQUIRE(rr->device == g->device, "ring-range handle and geometry on different devices");
  NB_REQUIRE(rr->vz0 >= 0 && rr->nvz > 0 && rr->vz0 + rr->nvz <= NB_IMZ,
             "ring-range handle with a bad axial slab");
  return NB_OK;
}

extern "C" int nb_fprj_rings(nb_geom *g, const nb_rings *rr, float *sino, const float *im,
                             const int32_t *subs, int nprj, int att, void *stream) {
  NB_RANGE("nb_fprj_rings");
  int st = check_common(g, nprj, subs, 1);
  if (st) return st;
  st = check_rings(g, rr);
  if (st) return st;
  NB_REQUIRE(sino && im, "nb_fprj_rings: NULL sino or image");
  NB_REQUIRE(att == 0 || att == 1, "att must be 0 or 1");
  cudaStream_t s = (cudaStream_t)stream;
  k_slab_to_col128<<<(NB_NCOL * 32 + 255) / 256, 256, 0, s>>>(g->d_scratch128, im, rr->nvz,
                                                               rr->vz0);
  NB_CUDA(cudaGetLastError());
  PrjArgs a = base_args(g, subs, nprj, 1);
  a.rays = rr->d_rays;
  a.bin1 = rr->d_bin1;
  a.nrays = rr->nrays;
  a.nout = rr->nrays;
  a.att = att;
  a.img = g->d_scratch128;
  a.sino = sino;
  return launch_project<MODE_FWD, CH_FWD>(g, a, s);
}

extern "C" int nb_bprj_rings(nb_geom *g, const nb_rings *rr, float *im, const float *sino,
                             const int32_t *subs, int nprj, void *stream) {
  NB_RANGE("nb_bprj_rings");
  int st = check_common(g, nprj, subs, 1);
  if (st) return st;
  st = check_rings(g, rr);
  if (st) return st;
  NB_REQUIRE(sino && im, "nb_bprj_rings: NULL sino or image");
  cudaStream_t s = (cudaStream_t)stream;
  NB_CUDA(cudaMemsetAsync(g->d_scratch128, 0, sizeof(float) * NB_IMG_COL128, s));
  PrjArgs a = base_args(g, subs, nprj, 1);
  a.rays = rr->d_rays;
  a.bin1 = rr->d_bin1;
  a.nrays = rr->nrays;
  a.nout = rr->nrays;
  a.bimg = g->d_scratch128;
  a.sino_in = sino;
  st = launch_project<MODE_BWD, CH_BWD>(g, a, s);
  if (st) return st;
  k_col128_to_slab<<<(NB_NCOL * 32 + 255) / 256, 256, 0, s>>>(im, g->d_scratch128, rr->nvz,
                                                               rr->vz0);
  NB_CUDA(cudaGetLastError());
  return NB_OK;
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
  NB_RANGE("nb_osem_subset");
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
  st = launch_project<MODE_OSEM, CH_BWD>(g, a, s);
  if (st) return st;
  const size_t n4 = NB_IMG_COL128 / 4;
  k_osem_update<<<g->nsm * 8, 256, 0, s>>>((float4 *)img128, (float4 *)bimg128,
                                           (const float4 *)sens128, (const uchar4 *)msk128, n4);
  NB_CUDA(cudaGetLastError());
  return NB_OK;
}

extern "C" int nb_psf_col128(float *dst128, const float *src128, const float *krnl,
                             float *tmp128, void *stream);

// One OSEM sub-iteration with resolution modelling (recon.cu:459-497 with krnl[0] >= 0):
// the forward projection sees the PSF-convolved image, the back-projected ratio is
// convolved before the division by the (already convolved) sensitivity.  work128 holds two
// col128 images of scratch.
extern "C" int nb_osem_subset_psf(nb_geom *g, float *img128, float *bimg128,
                                  const float *sens128, const uint8_t *msk128,
                                  const uint16_t *psng, const float *rs, const int32_t *subs,
                                  int nprj, const float *krnl, float *work128, void *stream) {
  NB_RANGE("nb_osem_subset_psf");
  int st = check_common(g, nprj, subs, 11);
  if (st) return st;
  NB_REQUIRE(img128 && bimg128 && sens128 && msk128 && psng && rs && subs && krnl && work128,
             "nb_osem_subset_psf: NULL argument");
  cudaStream_t s = (cudaStream_t)stream;
  float *rm = work128, *tmp = work128 + NB_IMG_COL128;
  st = nb_psf_col128(rm, img128, krnl, tmp, stream);
  if (st) return st;
  NB_CUDA(cudaMemsetAsync(bimg128, 0, sizeof(float) * NB_IMG_COL128, s));
  PrjArgs a = base_args(g, subs, nprj, 11);
  a.img = rm;
  a.bimg = bimg128;
  a.psng = psng;
  a.rs = rs;
  st = launch_project<MODE_OSEM, CH_BWD>(g, a, s);
  if (st) return st;
  st = nb_psf_col128(rm, bimg128, krnl, tmp, stream);  // rm: the convolved back projection
  if (st) return st;
  NB_CUDA(cudaMemsetAsync(bimg128, 0, sizeof(float) * NB_IMG_COL128, s));
  const size_t n4 = NB_IMG_COL128 / 4;
  k_osem_update<<<g->nsm * 8, 256, 0, s>>>((float4 *)img128, (float4 *)rm,
                                           (const float4 *)sens128, (const uchar4 *)msk128, n4);
  NB_CUDA(cudaGetLastError());
  return NB_OK;
}

extern "C" int nb_geom_count_reads(nb_geom *g, long long *per_lor, long long *reads) {
  NB_REQUIRE(g && reads, "nb_geom_count_reads: NULL argument");
  NB_CUDA(cudaSetDevice(g->device));
  unsigned long long *d = nullptr;
  NB_CUDA(cudaMalloc(&d, sizeof(unsigned long long) * (1 + (size_t)g->naw)));
  cudaMemset(d, 0, sizeof(unsigned long long) * (1 + (size_t)g->naw));
  k_count_reads<<<g->naw, 128>>>(g->d_hdr, g->d_st, g->d_rays, g->naw, d, d + 1);
  unsigned long long h = 0;
  cudaError_t e = cudaMemcpy(&h, d, sizeof(h), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess && per_lor)
    e = cudaMemcpy(per_lor, d + 1, sizeof(long long) * g->naw, cudaMemcpyDeviceToHost);
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
  NB_RANGE("nb_remgaps");
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
  NB_RANGE("nb_putgaps");
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
