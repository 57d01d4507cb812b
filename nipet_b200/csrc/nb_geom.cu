// nb_geom.cu -- geometry handle: transaxial Siddon tables and per-LOR step lists.
//
// Compiled with -fmad=false: the float arithmetic that decides the crossing order is
// written out operation by operation (reference prj/src/tprj.cu:13-172, sddn_tx), and
// the multiply-adds nvcc contracts in the reference by default are explicit
// __fmaf_rn calls here.  Tables are computed once per handle instead of on every
// projector call (reference prjf.cu:284, prjb.cu:256, recon.cu:349).
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <map>
#include <tuple>
#include <vector>

#include "nb_axial.cuh"
#include "nb_internal.cuh"
#include "nb_project.cuh"

// ---------------------------------------------------------------------------------------
// One thread per LOR: tt[10] and the crossing sequence tv[1807] (reference layout).
// ---------------------------------------------------------------------------------------
__global__ void k_siddon_tx(const float4 *__restrict__ crs, const short2 *__restrict__ s2c,
                            int naw, float *__restrict__ tt, unsigned char *__restrict__ tv) {
  int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= naw) return;
  short c1 = s2c[idx].x, c2 = s2c[idx].y;
  float4 C1 = crs[c1], C2 = crs[c2];
  // crystal-face centres: float sum, double half, rounded to float (tprj.cu:26-30)
  float cc1x = __double2float_rn(0.5 * (double)__fadd_rn(C1.x, C1.z));
  float cc2x = __double2float_rn(0.5 * (double)__fadd_rn(C2.x, C2.z));
  float cc1y = __double2float_rn(0.5 * (double)__fadd_rn(C1.y, C1.w));
  float cc2y = __double2float_rn(0.5 * (double)__fadd_rn(C2.y, C2.w));
  float ex = __fsub_rn(C1.z, C1.x), ey = __fsub_rn(C1.w, C1.y);
  float px = __double2float_rn(__dadd_rn((double)C1.x, 0.5 * (double)ex));
  float py = __double2float_rn(__dadd_rn((double)C1.y, 0.5 * (double)ey));
  float atx = __fsub_rn(cc2x, cc1x), aty = __fsub_rn(cc2y, cc1y);
  float atn = __fsqrt_rn(__fmaf_rn(atx, atx, __fmul_rn(aty, aty)));
  atx = __fdiv_rn(atx, atn);
  aty = __fdiv_rn(aty, atn);
  // chord through the transaxial FOV circle r^2 = TFOV2 (tprj.cu:53-56)
  float Br = __fmul_rn(2.f, __fmaf_rn(px, atx, __fmul_rn(py, aty)));
  float Cr = __fmul_rn(4.f, __fmaf_rn(py, py, __fmaf_rn(px, px, -NB_TFOV2)));
  float sq = __fsqrt_rn(__fmaf_rn(Br, Br, -Cr));
  float t1 = __double2float_rn(0.5 * (double)__fsub_rn(-Br, sq));
  float t2 = __double2float_rn(0.5 * (double)__fadd_rn(-Br, sq));
  // rows (tprj.cu:60-77)
  float y1 = __fmaf_rn(aty, t1, py);
  float sgy = signbit(aty) ? 1.f : 0.f;
  float cy1 = ceilf(__fdiv_rn(y1, NB_VOXY));
  float lr1 = __fmul_rn(NB_VOXY, __fsub_rn(cy1, sgy));
  int v = (int)__dsub_rn(0.5 * NB_IMY, (double)cy1);
  float y2 = __fmaf_rn(aty, t2, py);
  float lr2 = __fmul_rn(NB_VOXY, __fadd_rn(floorf(__fdiv_rn(y2, NB_VOXY)), sgy));
  // the compiled reference fuses the boundary line into the offset (lr - py becomes
  // fma(SZ_VOXY, c, -py)); lr1/lr2 keep the rounded product in their other uses
  float tr1 = __fdiv_rn(__fmaf_rn(NB_VOXY, __fsub_rn(cy1, sgy), -py), aty);
  float cy2 = __fadd_rn(floorf(__fdiv_rn(y2, NB_VOXY)), sgy);
  float tr2 = __fdiv_rn(__fmaf_rn(NB_VOXY, cy2, -py), aty);
  bool y21 = fabsf(__fsub_rn(y2, y1)) >= NB_VOXY;
  bool lr21 = fabsf(__fsub_rn(lr1, lr2)) < NB_L21;
  int nr = (int)__fadd_rn(__fmul_rn((float)y21, roundf(__fdiv_rn(fabsf(__fsub_rn(lr2, lr1)),
                                                                 NB_VOXY))),
                          (float)lr21);
  float dtr;
  if (nr > 0)
    dtr = __fadd_rn(__fdiv_rn(__fsub_rn(tr2, tr1), (float)nr), __fmul_rn((float)lr21, t2));
  else
    dtr = t2;
  // columns (tprj.cu:80-97); x1 is a double holding a float value
  double x1 = (double)__fmaf_rn(atx, t1, px);
  double sgx = signbit(atx) ? 1.0 : 0.0;
  float lc1 = __double2float_rn(
      __dmul_rn((double)NB_VOXY, __dsub_rn(ceil(__ddiv_rn(x1, (double)NB_VOXY)), sgx)));
  int u = (int)__dadd_rn(0.5 * NB_IMX, floor(__ddiv_rn(x1, (double)NB_VOXY)));
  float x2 = __fmaf_rn(atx, t2, px);
  float lc2 = __fmul_rn(NB_VOXY, __fadd_rn(floorf(__fdiv_rn(x2, NB_VOXY)), (float)sgx));
  float tc1 = __fdiv_rn(__fsub_rn(lc1, px), atx);
  float tc2 = __fdiv_rn(
      __fmaf_rn(NB_VOXY, __fadd_rn(floorf(__fdiv_rn(x2, NB_VOXY)), (float)sgx), -px), atx);
  bool x21 = fabsf(__double2float_rn(__dsub_rn((double)x2, x1))) >= NB_VOXY;
  bool lc21 = fabsf(__fsub_rn(lc1, lc2)) < NB_L21;
  int nc = (int)__fadd_rn(__fmul_rn((float)x21, roundf(__fdiv_rn(fabsf(__fsub_rn(lc2, lc1)),
                                                                 NB_VOXY))),
                          (float)lc21);
  float dtc;
  if (nc > 0)
    dtc = __fadd_rn(__fdiv_rn(__fsub_rn(tc2, tc1), (float)nc), __fmul_rn((float)lc21, t2));
  else
    dtc = t2;

  // crossing sequence (tprj.cu:105-157): 1 = row step, 0 = column step
  float ang = atanf(__fdiv_rn(aty, atx));
  unsigned char *T = tv + (size_t)NB_N_TV * idx;
  T[0] = atx >= 0 ? 2 : 0;
  T[1] = aty >= 0 ? 2 : 0;
  int k = 2;
  if ((ang < NB_TA1) & (ang > NB_TA2)) {
    float tf = tc1, ts = tr1;
    for (int i = 0; i <= nc; i++) {
      int tsin = __fsub_rn(tf, ts) > 0.f;
      if (k < NB_N_TV) T[k] = 1;
      k += tsin;
      ts = __fadd_rn(ts, __fmul_rn(dtr, (float)tsin));
      if (k < NB_N_TV) T[k] = 0;
      k += 1;
      tf = __fadd_rn(tf, dtc);
    }
    if (tr2 > tc2) {
      if (k < NB_N_TV) T[k] = 1;
      k += 1;
    }
  } else {
    float tf = tr1, ts = tc1;
    for (int i = 0; i <= nr; i++) {
      int tsin = __fsub_rn(tf, ts) > 0.f;
      if (k < NB_N_TV) T[k] = 0;
      k += tsin;
      ts = __fadd_rn(ts, __fmul_rn(dtc, (float)tsin));
      if (k < NB_N_TV) T[k] = 1;
      k += 1;
      tf = __fadd_rn(tf, dtr);
    }
    if (tc2 > tr2) {
      if (k < NB_N_TV) T[k] = 0;
      k += 1;
    }
  }
  float *t = tt + (size_t)NB_N_TT * idx;
  t[0] = tr1;
  t[1] = tc1;
  t[2] = dtr;
  t[3] = dtc;
  t[4] = t1;
  t[5] = fminf(tr1, tc1);
  t[6] = t2;
  t[7] = atn;
  t[8] = (float)(u + (v << 9));
  t[9] = (float)k;
}

// ---------------------------------------------------------------------------------------
// One thread per LOR: expand the crossing sequence into the step list the projectors
// stream (the walk of prjf.cu:49-86, done once per geometry instead of per ray).
// ---------------------------------------------------------------------------------------
__global__ void k_expand_steps(const float *__restrict__ tt, const unsigned char *__restrict__ tv,
                               int naw, int32_t *__restrict__ scol, float *__restrict__ st,
                               float4 *__restrict__ hdr, int *err) {
  int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= naw) return;
  const float *t = tt + (size_t)NB_N_TT * idx;
  const unsigned char *T = tv + (size_t)NB_N_TV * idx;
  int sgna0 = T[0] - 1, sgna1 = T[1] - 1;
  int rbit = T[2] & 1;
  int uvp = (int)t[8];
  int v = uvp >> 9;
  int col = (uvp & 0x1ff) + NB_IMX * v;
  col += !rbit * sgna0;
  col -= rbit * sgna1 * NB_IMX;
  float dtr = t[2], dtc = t[3];
  float trc = __fadd_rn(t[0], __fmul_rn((float)rbit, dtr));
  float tcc = __fadd_rn(t[1], __fmul_rn(dtc, (float)!rbit));
  rbit = T[3] & 1;
  float tn = __fadd_rn(__fmul_rn(trc, (float)rbit), __fmul_rn(tcc, (float)!rbit));
  int K = (int)t[9];
  int n = 0;
  int32_t *sc = scol + (size_t)idx * NB_STEP_STRIDE;
  float *sv = st + (size_t)idx * NB_STEP_STRIDE;
  for (int k = 3; k < K; k++) {
    if (n < NB_STEP_STRIDE) {
      sc[n] = (col >= 0 && col < NB_NCOL) ? col : 0;
      sv[n] = tn;
      if (col < 0 || col >= NB_NCOL) nb_set_error(err, NB_DEVERR_BAD_LOR);
    }
    n++;
    trc = __fadd_rn(trc, __fmul_rn(dtr, (float)rbit));
    tcc = __fadd_rn(tcc, __fmul_rn(dtc, (float)!rbit));
    col += !rbit * sgna0;
    col -= rbit * sgna1 * NB_IMX;
    rbit = (k + 1 < NB_N_TV) ? (T[k + 1] & 1) : 0;
    tn = __fadd_rn(__fmul_rn(trc, (float)rbit), __fmul_rn(tcc, (float)!rbit));
  }
  if (n > NB_STEP_STRIDE) {
    nb_set_error(err, NB_DEVERR_STEP_OVERFLOW);
    n = NB_STEP_STRIDE;
  }
  // pad the tail so that 16-byte bulk copies never read uninitialised entries
  for (int i = n; i < ((n + 3) & ~3) && i < NB_STEP_STRIDE; i++) {
    sc[i] = 0;
    sv[i] = 0.f;
  }
  hdr[idx] = make_float4(t[5], t[7], t[6], __int_as_float(n));
}

// longest walk segment (tn - tp) of every LOR, as float bits (segments are >= 0)
__global__ void k_maxseg(const float4 *__restrict__ hdr, const float *__restrict__ st, int naw,
                         unsigned *out) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= naw) return;
  const float4 h = hdr[idx];
  const int n = __float_as_int(h.w);
  float tp = h.x, m = 0.f;
  for (int k = 0; k < n; k++) {
    const float tn = st[(size_t)idx * NB_STEP_STRIDE + k];
    m = fmaxf(m, fabsf(__fsub_rn(tn, tp)));
    tp = tn;
  }
  atomicMax(out, __float_as_uint(m));
}

// ---------------------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------------------
static void nb_geom_free(nb_geom *g) {
  if (!g) return;
  cudaFree(g->d_scol);
  cudaFree(g->d_st);
  cudaFree(g->d_hdr);
  cudaFree(g->d_tt);
  cudaFree(g->d_rays);
  cudaFree(g->d_bin11);
  cudaFree(g->d_bin1);
  cudaFree(g->d_scratch128);
  cudaFree(g->d_err);
  cudaFree(g->d_one);
  free(g->h_s2c);
  free(g->h_rays);
  free(g);
}

static int run_tables(nb_geom *g, const float *crs_h, const int16_t *s2c_h, float *d_tt,
                      unsigned char *d_tv) {
  float4 *d_crs = nullptr;
  short2 *d_s2c = nullptr;
  int st = NB_OK;
  cudaError_t e = cudaMalloc(&d_crs, 504 * sizeof(float4));
  if (e == cudaSuccess) e = cudaMalloc(&d_s2c, (size_t)g->naw * sizeof(short2));
  if (e == cudaSuccess)
    e = cudaMemcpy(d_crs, crs_h, 504 * sizeof(float4), cudaMemcpyHostToDevice);
  if (e == cudaSuccess)
    e = cudaMemcpy(d_s2c, s2c_h, (size_t)g->naw * sizeof(short2), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(d_tv, 0, (size_t)g->naw * NB_N_TV);
  if (e == cudaSuccess) {
    k_siddon_tx<<<(g->naw + 255) / 256, 256>>>(d_crs, d_s2c, g->naw, d_tt, d_tv);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e != cudaSuccess) st = nb_cuda_fail(e, "siddon tables", __FILE__, __LINE__);
  cudaFree(d_crs);
  cudaFree(d_s2c);
  return st;
}

extern "C" int nb_geom_create(int device, const float *crs, int ncrs, const int16_t *s2c,
                              int naw, const float *li2rng, const int16_t *li2sn,
                              const int16_t *li2sn1, const int8_t *li2nos, int nli2r,
                              nb_geom **out) {
  NB_RANGE("nb_geom_create (Siddon tables, walk checks)");
  NB_REQUIRE(out != nullptr, "nb_geom_create: out is NULL");
  *out = nullptr;
  NB_REQUIRE(crs && s2c && li2rng && li2sn && li2sn1 && li2nos, "nb_geom_create: NULL LUT");
  NB_REQUIRE(ncrs == NB_NCRS, "nb_geom_create: crs must have 504 crystals");
  NB_REQUIRE(naw == NB_AW, "nb_geom_create: s2c must have 68516 LORs");
  NB_REQUIRE(nli2r == NB_NLI2R, "nb_geom_create: li2rng must have 2074 ring pairs");
  int ndev = 0;
  NB_CUDA(cudaGetDeviceCount(&ndev));
  NB_REQUIRE(device >= 0 && device < ndev, "nb_geom_create: invalid device");
  NB_CUDA(cudaSetDevice(device));
  for (int i = 0; i < naw; i++) {
    if (s2c[2 * i] < 0 || s2c[2 * i] >= NB_NCRS || s2c[2 * i + 1] < 0 ||
        s2c[2 * i + 1] >= NB_NCRS) {
      nb_set_error_msg("nb_geom_create: s2c[%d] crystal index out of range", i);
      return NB_ERR_ARG;
    }
  }

  nb_geom *g = (nb_geom *)calloc(1, sizeof(nb_geom));
  if (!g) return NB_ERR_NOMEM;
  g->device = device;
  g->naw = naw;
  cudaDeviceGetAttribute(&g->nsm, cudaDevAttrMultiProcessorCount, device);
  memcpy(g->h_crs, crs, sizeof(g->h_crs));
  g->h_s2c = (int16_t *)malloc(sizeof(int16_t) * 2 * naw);
  memcpy(g->h_s2c, s2c, sizeof(int16_t) * 2 * naw);

  // ray tables (host) -------------------------------------------------------------
  std::vector<nb_ray> rays(NB_NRAYS);
  for (int r = 0; r < NB_NRAYS; r++) {
    int li, kind;
    if (r < NB_NRINGS) {
      li = r;
      kind = 0;
    } else if (r < NB_NRINGS + NB_NOBLQ) {
      li = r;
      kind = 1;
    } else {
      li = r - NB_NOBLQ;
      kind = 2;
    }
    nb_ray R;
    R.r0z = li2rng[2 * li];
    R.r1z = li2rng[2 * li + 1];
    R.out11 = kind == 2 ? li2sn[2 * li + 1] : li2sn[2 * li];
    R.out1 = kind == 2 ? li2sn1[2 * li + 1] : li2sn1[2 * li];
    R.kind = (int8_t)kind;
    R.nos = li2nos[li];
    R.li = (int16_t)li;
    if (R.out11 < 0 || R.out11 >= NB_NSN11 || R.out1 < 0 || R.out1 >= NB_NSN1 || R.nos <= 0) {
      free(g->h_s2c);
      free(g);
      nb_set_error_msg("nb_geom_create: axial LUT entry %d out of range", li);
      return NB_ERR_ARG;
    }
    rays[r] = R;
  }
  // Warp-friendly ray order: the kernels give thread t the rays t, t+NT, ... so every
  // 32-aligned block of ray indices is the lane set of one warp.  Rays of one ring
  // difference d and direction (a "group", 64-|d| rays) sit 2 voxels apart and cross z
  // planes at the same steps; a warp drawn from one group reads consecutive shared-memory
  // banks and takes its crossings together.  Order: every group's first 32 rays (groups
  // of 32 or more), then warps that pair the rest of group d (32-d rays) with all of group
  // 64-d (d rays) -- exactly 32, at most two groups per warp -- and last the rest of
  // groups 1..3, which have no partner.  Any ray not placed by these rules (none for the
  // mMR's 64 rings and maximum ring difference 60) is appended at the end.
  {
    const std::vector<nb_ray> canon = rays;
    std::map<int, std::vector<int>> grp;  // (kind, d) -> canonical rays in ring order
    auto key = [&](int r) {
      return canon[r].kind * 1000 + (int)lrintf((canon[r].r1z - canon[r].r0z) / NB_RING);
    };
    for (int r = 0; r < NB_NRAYS; r++) grp[key(r)].push_back(r);
    std::vector<int> order;
    std::vector<char> used(NB_NRAYS, 0);
    auto take = [&](int k, size_t from, size_t to) {
      auto it = grp.find(k);
      if (it == grp.end()) return;
      for (size_t i = from; i < to && i < it->second.size(); i++) {
        const int r = it->second[i];
        if (!used[r]) {
          used[r] = 1;
          order.push_back(r);
        }
      }
    };
    auto size_of = [&](int k) -> size_t {
      auto it = grp.find(k);
      return it == grp.end() ? 0 : it->second.size();
    };
    for (auto &kv : grp)  // full first blocks (direct planes: both of theirs)
      for (size_t f = 0; f + 32 <= kv.second.size(); f += 32)
        if (kv.first / 1000 == 0 || f == 0) take(kv.first, f, f + 32);
    for (int kind = 1; kind <= 2; kind++)
      for (int d = 4; d <= 31; d++) {
        const int ka = kind * 1000 + d, kb = kind * 1000 + (64 - d);
        if (size_of(ka) == (size_t)(64 - d) && size_of(kb) == (size_t)d) {
          take(ka, 32, size_of(ka));
          take(kb, 0, size_of(kb));
        }
      }
    for (int kind = 1; kind <= 2; kind++)
      for (int d = 1; d <= 3; d++) take(kind * 1000 + d, 32, size_of(kind * 1000 + d));
    for (int r = 0; r < NB_NRAYS; r++)
      if (!used[r]) order.push_back(r);
    for (int r = 0; r < NB_NRAYS; r++) rays[r] = canon[order[r]];
  }
  std::vector<int16_t> bin11(NB_NSN11 * 8, -1), bin1(NB_NSN1, -1);
  std::vector<int> cnt11(NB_NSN11, 0);
  for (int r = 0; r < NB_NRAYS; r++) {
    int o = rays[r].out11;
    if (cnt11[o] >= 8) {
      free(g->h_s2c);
      free(g);
      nb_set_error_msg("nb_geom_create: more than 8 span-1 planes in span-11 sinogram %d", o);
      return NB_ERR_ARG;
    }
    bin11[o * 8 + cnt11[o]++] = (int16_t)r;
    if (bin1[rays[r].out1] != -1) {
      free(g->h_s2c);
      free(g);
      nb_set_error_msg("nb_geom_create: span-1 sinogram %d mapped twice", rays[r].out1);
      return NB_ERR_ARG;
    }
    bin1[rays[r].out1] = (int16_t)r;
  }

  int st = NB_OK;
  unsigned char *d_tv = nullptr;
  g->h_rays = (nb_ray *)malloc(sizeof(nb_ray) * NB_NRAYS);
  if (!g->h_rays) {
    free(g->h_s2c);
    free(g);
    return NB_ERR_NOMEM;
  }
  memcpy(g->h_rays, rays.data(), sizeof(nb_ray) * NB_NRAYS);
#define ALLOC(p, bytes)                                                                        \
  do {                                                                                         \
    if (cudaMalloc((void **)&(p), (bytes)) != cudaSuccess) {                                   \
      cudaGetLastError();                                                                      \
      nb_set_error_msg("nb_geom_create: cudaMalloc of %zu bytes failed", (size_t)(bytes));      \
      st = NB_ERR_NOMEM;                                                                       \
      goto fail;                                                                               \
    }                                                                                          \
  } while (0)
  ALLOC(g->d_scol, sizeof(int32_t) * (size_t)naw * NB_STEP_STRIDE);
  ALLOC(g->d_st, sizeof(float) * (size_t)naw * NB_STEP_STRIDE);
  ALLOC(g->d_hdr, sizeof(float4) * naw);
  ALLOC(g->d_tt, sizeof(float) * NB_N_TT * (size_t)naw);
  ALLOC(g->d_rays, sizeof(nb_ray) * NB_NRAYS);
  ALLOC(g->d_bin11, sizeof(int16_t) * NB_NSN11 * 8);
  ALLOC(g->d_bin1, sizeof(int16_t) * NB_NSN1);
  ALLOC(g->d_scratch128, sizeof(float) * NB_IMG_COL128);
  ALLOC(g->d_err, sizeof(int));
  ALLOC(g->d_one, sizeof(float));
  ALLOC(d_tv, (size_t)naw * NB_N_TV);
#undef ALLOC
  {
    const float one = 1.f;
    if (cudaMemcpy(g->d_one, &one, sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess) {
      cudaGetLastError();
      nb_set_error_msg("nb_geom_create: upload of a constant failed");
      st = NB_ERR_CUDA;
      goto fail;
    }
  }
  if (cudaMemset(g->d_err, 0, sizeof(int)) != cudaSuccess ||
      cudaMemset(g->d_scol, 0, sizeof(int32_t) * (size_t)naw * NB_STEP_STRIDE) != cudaSuccess ||
      cudaMemset(g->d_st, 0, sizeof(float) * (size_t)naw * NB_STEP_STRIDE) != cudaSuccess ||
      cudaMemcpy(g->d_rays, rays.data(), sizeof(nb_ray) * NB_NRAYS, cudaMemcpyHostToDevice) !=
          cudaSuccess ||
      cudaMemcpy(g->d_bin11, bin11.data(), sizeof(int16_t) * NB_NSN11 * 8,
                 cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(g->d_bin1, bin1.data(), sizeof(int16_t) * NB_NSN1, cudaMemcpyHostToDevice) !=
          cudaSuccess) {
    st = nb_cuda_fail(cudaGetLastError(), "nb_geom_create upload", __FILE__, __LINE__);
    goto fail;
  }
  st = run_tables(g, crs, s2c, g->d_tt, d_tv);
  if (st != NB_OK) goto fail;
  k_expand_steps<<<(naw + 255) / 256, 256>>>(g->d_tt, d_tv, naw, g->d_scol, g->d_st, g->d_hdr,
                                             g->d_err);
  if (cudaDeviceSynchronize() != cudaSuccess) {
    st = nb_cuda_fail(cudaGetLastError(), "k_expand_steps", __FILE__, __LINE__);
    goto fail;
  }
  {
    int herr = 0;
    cudaMemcpy(&herr, g->d_err, sizeof(int), cudaMemcpyDeviceToHost);
    if (herr) {
      nb_set_error_msg("nb_geom_create: step expansion reported device error %d", herr);
      st = NB_ERR_DEVICE;
      goto fail;
    }
    // Walk checks: every ray stays inside z in [0, 127) (the projector kernels index
    // shared memory by it) and the longest segment sets the fixed-point headroom of the
    // back projector (242 overlapping rays per column slot at most).
    cudaMemset(g->d_err, 0, sizeof(int));
    unsigned *d_seg = (unsigned *)d_tv;  // reuse the table buffer
    cudaMemset(d_seg, 0, sizeof(unsigned));
    nbk::k_check_walk<<<naw, 256>>>(g->d_hdr, g->d_st, g->d_rays, naw, g->d_err, d_seg);
    k_maxseg<<<(naw + 255) / 256, 256>>>(g->d_hdr, g->d_st, naw, d_seg);
    unsigned segbits = 0;
    int nbad = 0;
    cudaError_t e = cudaMemcpy(&nbad, g->d_err, sizeof(int), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(&segbits, d_seg, sizeof(unsigned), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) {
      st = nb_cuda_fail(e, "nb_geom_create walk check", __FILE__, __LINE__);
      goto fail;
    }
    cudaMemset(g->d_err, 0, sizeof(int));
    if (nbad) {
      nb_set_error_msg("nb_geom_create: %d ray positions leave the axial FOV", nbad);
      st = NB_ERR_DATA;
      goto fail;
    }
    memcpy(&g->maxseg, &segbits, sizeof(float));
    // maxseg: the largest weight one ray gives one voxel in one step (the longest step, or
    // a late crossing's |tzc - tp|).  Slot sums stay below 2^31 (242 rays per slot at
    // most), and every contribution below 2^22, the range in which the back projectors
    // round w * value to an integer with one fused multiply-add (nb_fx_round).
    const double seg = g->maxseg > 0.f ? (double)g->maxseg : 1.0;
    int lb = (int)ceil(log2(242.0 * seg));
    g->fxbits = 31 - lb;
    int fm = (int)floor(log2(4194304.0 / seg));
    while (fm > 0 && ldexp(seg, fm) >= 4194304.0) fm--;
    if (fm < g->fxbits) g->fxbits = fm;
    if (g->fxbits < 16) {
      nb_set_error_msg("nb_geom_create: walk segments too long (%g cm)", (double)g->maxseg);
      st = NB_ERR_DATA;
      goto fail;
    }
  }
  cudaFree(d_tv);
  *out = g;
  return NB_OK;
fail:
  cudaFree(d_tv);
  nb_geom_free(g);
  return st;
}

// Ring of a ring front edge z (cm): ring i starts at (i - 32) * AXR (mmraux.py:365-370)
static int ring_of(float z) {
  const double r = (double)z / (double)NB_RING + 0.5 * NB_NRINGS;
  const long i = lrint(r);
  return fabs(r - (double)i) < 1e-4 ? (int)i : -1;
}

// Rays of the ring range [rs, re) from the range's axial LUTs, as mmraux.axial_lut builds
// them after mmraux.reduce_rings: li2rng / li2sn1 [nli2r][2], the first re - rs entries
// the direct planes (prjf.cu:33-95 runs them as fprj_drct), the others the oblique pairs,
// whose ring r0 -> r1 ray feeds sinogram li2sn1[.][0] and r1 -> r0 li2sn1[.][1]
// (prjf.cu:98-206).  Each ray must be one of the geometry's rays with both rings in the
// range, and the rays must fill the range's (re - rs)^2 sinograms (4084 for all 64 rings)
// once each; anything else is NB_ERR_ARG (the reference's LUTs of 62- and 63-ring ranges,
// whose ring differences exceed the maximum of 60 without the full-ring correction, end in
// zero entries and fail this check).  The rays keep the geometry's warp-friendly order.
extern "C" int nb_rings_create(nb_geom *g, int rs, int re, const float *li2rng,
                               const int16_t *li2sn1, int nli2r, nb_rings **out) {
  NB_REQUIRE(out != nullptr, "nb_rings_create: out is NULL");
  *out = nullptr;
  NB_REQUIRE(g && li2rng && li2sn1, "nb_rings_create: NULL argument");
  NB_REQUIRE(g->h_rays != nullptr, "nb_rings_create: geometry without a ray table");
  NB_REQUIRE(rs >= 0 && rs < re && re <= NB_NRINGS, "nb_rings_create: need 0 <= rs < re <= 64");
  const int n = re - rs;
  const int want_li = n * (n + 1) / 2 - (n == NB_NRINGS ? 6 : 0);
  const int nsino = n * n - (n == NB_NRINGS ? 12 : 0);
  if (nli2r != want_li) {
    nb_set_error_msg("nb_rings_create: %d ring pairs given, the range [%d, %d) has %d", nli2r,
                     rs, re, want_li);
    return NB_ERR_ARG;
  }
  // the geometry's rays by (kind, ring front edges)
  std::map<std::tuple<int, uint32_t, uint32_t>, int> pos;
  for (int r = 0; r < NB_NRAYS; r++) {
    const nb_ray &R = g->h_rays[r];
    uint32_t a, b;
    memcpy(&a, &R.r0z, 4);
    memcpy(&b, &R.r1z, 4);
    pos[std::make_tuple((int)R.kind, a, b)] = r;
  }
  std::vector<std::pair<int, nb_ray>> sel;  // (position in the geometry's order, ray)
  sel.reserve(nsino);
  for (int li = 0; li < nli2r; li++) {
    const float z0 = li2rng[2 * li], z1 = li2rng[2 * li + 1];
    const int r0 = ring_of(z0), r1 = ring_of(z1);
    if (r0 < rs || r0 >= re || r1 < rs || r1 >= re) {
      nb_set_error_msg("nb_rings_create: ring pair %d (z %g, %g cm) is outside rings [%d, %d)",
                       li, (double)z0, (double)z1, rs, re);
      return NB_ERR_ARG;
    }
    const int nk = li < n ? 1 : 2;
    for (int k = 0; k < nk; k++) {
      const int kind = li < n ? 0 : 1 + k;
      uint32_t a, b;
      memcpy(&a, &z0, 4);
      memcpy(&b, &z1, 4);
      auto it = pos.find(std::make_tuple(kind, a, b));
      if (it == pos.end()) {
        nb_set_error_msg("nb_rings_create: ring pair %d (rings %d, %d) is not a %s ray of the "
                         "geometry", li, r0, r1, kind == 0 ? "direct" : "oblique");
        return NB_ERR_ARG;
      }
      nb_ray R = g->h_rays[it->second];
      R.out1 = li2sn1[2 * li + k];
      R.out11 = 0;  // span 11 does not exist for a reduced range
      sel.emplace_back(it->second, R);
    }
  }
  if ((int)sel.size() != nsino) {
    nb_set_error_msg("nb_rings_create: %zu rays for %d sinograms", sel.size(), nsino);
    return NB_ERR_ARG;
  }
  std::sort(sel.begin(), sel.end(),
            [](const std::pair<int, nb_ray> &x, const std::pair<int, nb_ray> &y) {
              return x.first < y.first;
            });
  std::vector<nb_ray> rays(nsino);
  std::vector<int16_t> bin1(nsino, -1);
  for (int r = 0; r < nsino; r++) {
    rays[r] = sel[r].second;
    const int o = rays[r].out1;
    if (o < 0 || o >= nsino || bin1[o] != -1) {
      nb_set_error_msg("nb_rings_create: sinogram %d of the range is out of [0, %d) or mapped "
                       "twice", o, nsino);
      return NB_ERR_ARG;
    }
    bin1[o] = (int16_t)r;
  }
  NB_CUDA(cudaSetDevice(g->device));
  nb_rings *rr = (nb_rings *)calloc(1, sizeof(nb_rings));
  if (!rr) return NB_ERR_NOMEM;
  rr->device = g->device;
  rr->rs = rs;
  rr->re = re;
  rr->nrays = nsino;
  rr->vz0 = 2 * rs;
  rr->nvz = 2 * n - 1;
  cudaError_t e = cudaMalloc(&rr->d_rays, sizeof(nb_ray) * nsino);
  if (e == cudaSuccess) e = cudaMalloc(&rr->d_bin1, sizeof(int16_t) * nsino);
  if (e == cudaSuccess)
    e = cudaMemcpy(rr->d_rays, rays.data(), sizeof(nb_ray) * nsino, cudaMemcpyHostToDevice);
  if (e == cudaSuccess)
    e = cudaMemcpy(rr->d_bin1, bin1.data(), sizeof(int16_t) * nsino, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    cudaFree(rr->d_rays);
    cudaFree(rr->d_bin1);
    free(rr);
    return nb_cuda_fail(e, "nb_rings_create upload", __FILE__, __LINE__);
  }
  *out = rr;
  return NB_OK;
}

extern "C" int nb_rings_destroy(nb_rings *rr) {
  if (!rr) return NB_OK;
  cudaSetDevice(rr->device);
  cudaFree(rr->d_rays);
  cudaFree(rr->d_bin1);
  free(rr);
  return NB_OK;
}

extern "C" int nb_rings_info(const nb_rings *rr, int *nsino, int *vz0, int *nvz) {
  NB_REQUIRE(rr != nullptr, "nb_rings_info: NULL handle");
  if (nsino) *nsino = rr->nrays;
  if (vz0) *vz0 = rr->vz0;
  if (nvz) *nvz = rr->nvz;
  return NB_OK;
}

extern "C" int nb_geom_destroy(nb_geom *g) {
  if (!g) return NB_OK;
  cudaSetDevice(g->device);
  nb_geom_free(g);
  return NB_OK;
}

extern "C" int nb_geom_tables(nb_geom *g, float *tt, uint8_t *tv) {
  NB_REQUIRE(g && tt && tv, "nb_geom_tables: NULL argument");
  NB_CUDA(cudaSetDevice(g->device));
  float *d_tt = nullptr;
  unsigned char *d_tv = nullptr;
  if (cudaMalloc(&d_tt, sizeof(float) * NB_N_TT * (size_t)g->naw) != cudaSuccess ||
      cudaMalloc(&d_tv, (size_t)g->naw * NB_N_TV) != cudaSuccess) {
    cudaGetLastError();
    cudaFree(d_tt);
    cudaFree(d_tv);
    nb_set_error_msg("nb_geom_tables: cudaMalloc failed");
    return NB_ERR_NOMEM;
  }
  int st = run_tables(g, g->h_crs, g->h_s2c, d_tt, d_tv);
  if (st == NB_OK) {
    cudaError_t e = cudaMemcpy(tt, d_tt, sizeof(float) * NB_N_TT * (size_t)g->naw,
                               cudaMemcpyDeviceToHost);
    if (e == cudaSuccess)
      e = cudaMemcpy(tv, d_tv, (size_t)g->naw * NB_N_TV, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) st = nb_cuda_fail(e, "nb_geom_tables copy", __FILE__, __LINE__);
  }
  cudaFree(d_tt);
  cudaFree(d_tv);
  return st;
}
