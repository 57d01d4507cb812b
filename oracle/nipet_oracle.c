/* nipet_oracle.c -- CPU oracle for the mMR reconstruction hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker the CUDA path is compared
 * against; nothing in the product links or calls it.  It restates, statement by
 * statement, the reference algorithms it is named after:
 *
 *   orc_siddon_tables  <- niftypet/nipet/prj/src/tprj.cu:13-172   (sddn_tx)
 *   orc_fprj           <- niftypet/nipet/prj/src/prjf.cu:33-206   (fprj_drct, fprj_oblq)
 *   orc_bprj           <- niftypet/nipet/prj/src/prjb.cu:33-187   (bprj_drct, bprj_oblq)
 *   orc_osem_iter      <- niftypet/nipet/prj/src/recon.cu:318-497 (osem, no PSF)
 *   orc_osem_batch_iter   the same iteration for several images per walk of a LOR
 *   orc_lm_plan        <- niftypet/nipet/lm/src/lmaux.cu:17-270   (getLMinfo, modifyLMinfo)
 *   orc_hist           <- niftypet/nipet/lm/src/hst.cu:37-244     (hst) + lmproc.cu:156-193
 *   orc_philox4x32     <- Philox4x32-10, Salmon et al., SC'11 ("Parallel random numbers:
 *                         as easy as 1, 2, 3"); the bootstrap stream definition is this
 *                         project's own (the reference uses clock()-seeded curand).
 *
 * Numerics: every quantity that decides WHICH voxel a ray visits (crossing order,
 * start voxel, axial crossing test) is computed in float32 with the reference's
 * operation order; nvcc's default multiply-add contraction is modelled with explicit
 * fmaf() where the reference writes a*b+c in one float expression (switchable with
 * orc_set_contract).  Segment lengths, weights and all accumulation are double.
 *
 * Build: see oracle/Makefile (gcc -O2 -fopenmp -ffp-contract=off -shared -fPIC).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ---- scanner constants (include/def.h:55-123) ---- */
#define AW 68516
#define N_TV 1807
#define N_TT 10
#define SZ_IMX 320
#define SZ_IMY 320
#define SZ_IMZ 127
#define NVOX (SZ_IMX * SZ_IMY * SZ_IMZ)
#define TFOV2 890.0f
#define SZ_VOXY 0.208626f
#define SZ_VOXZ 0.203125f
#define SZ_VOXZi 4.923077f
#define SZ_RING 0.40625f
#define L21 0.001f
#define TA1 0.7885139f
#define TA2 -0.7822831f
#define UV_SHFT 9
#define NRINGS 64
#define NLI2R 2074
#define NSBINS 344
#define NSANGLES 252
#define NSBINANG 86688
#define NSINOS 4084
#define NSINOS11 837
#define SEG0 127
#define nCRS 504
#define NBUCKTS 224
#define ITIME 1000
#define BTPTIME 100
#define VTIME 2
#define MXNITAG 5400
#define TOTHRDS 2560
#define ELECHNK (402653184 / 32)

static int g_contract = 1;
void orc_set_contract(int on) { g_contract = on; }
int orc_get_contract(void) { return g_contract; }

/* a*b + c in float, either fused (nvcc -fmad=true) or as two rounded operations */
static inline float mad(float a, float b, float c) {
  if (g_contract) return fmaf(a, b, c);
  volatile float p = a * b;
  return p + c;
}

int orc_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
void orc_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

/* ========================================================================
 * Transaxial Siddon tables: tprj.cu:13-172.  One LOR per iteration.
 * crs: [ncrs][4] float (x0, y0, x1, y1 of each crystal face); s2c: [naw][2] short.
 * tt: [naw][10] float; tv: [naw][1807] uint8 (caller zero-fills).
 * ====================================================================== */
static void siddon_one(const float *crs, const short *s2c, int idx, float *tt, unsigned char *tv) {
  short c1 = s2c[2 * idx], c2 = s2c[2 * idx + 1];
  const float *C1 = crs + 4 * c1, *C2 = crs + 4 * c2;
  float cc1x = (float)(.5 * (double)(C1[0] + C1[2]));
  float cc2x = (float)(.5 * (double)(C2[0] + C2[2]));
  float cc1y = (float)(.5 * (double)(C1[1] + C1[3]));
  float cc2y = (float)(.5 * (double)(C2[1] + C2[3]));
  float ex = C1[2] - C1[0];
  float ey = C1[3] - C1[1];
  float px = (float)((double)C1[0] + 0.5 * (double)ex);
  float py = (float)((double)C1[1] + 0.5 * (double)ey);
  float atx = cc2x - cc1x, aty = cc2y - cc1y;
  float atn = mad(atx, atx, aty * aty);
  atn = sqrtf(atn);
  atx = atx / atn;
  aty = aty / atn;
  /* ring tfov */
  float Br = 2 * mad(px, atx, py * aty);
  float Cr = 4 * mad(py, py, mad(px, px, -TFOV2));
  float sq = sqrtf(mad(Br, Br, -Cr));
  float t1 = (float)(.5 * (double)(-Br - sq));
  float t2 = (float)(.5 * (double)(-Br + sq));
  /* rows */
  float y1 = mad(aty, t1, py);
  int sgy = signbit(aty) ? 1 : 0;
  float cr1 = ceilf(y1 / SZ_VOXY) - (float)sgy;
  float lr1 = SZ_VOXY * cr1;
  int v = (int)(0.5 * SZ_IMY - (double)ceilf(y1 / SZ_VOXY));
  float y2 = mad(aty, t2, py);
  float cr2 = floorf(y2 / SZ_VOXY) + (float)sgy;
  float lr2 = SZ_VOXY * cr2;
  /* the compiled reference fuses the boundary line into the offset: lr - py is
   * fma(SZ_VOXY, c, -py), the product left unrounded (checked bit for bit against the
   * reference's own tables on all 68516 LORs); lr1/lr2 keep the rounded product in
   * their other uses */
  float tr1 = fmaf(SZ_VOXY, cr1, -py) / aty;
  float tr2 = fmaf(SZ_VOXY, cr2, -py) / aty;
  int y21 = fabsf(y2 - y1) >= SZ_VOXY;
  int lr21 = fabsf(lr1 - lr2) < L21;
  int nr = (int)((float)y21 * roundf(fabsf(lr2 - lr1) / SZ_VOXY) + (float)lr21);
  float dtr;
  if (nr > 0)
    dtr = (tr2 - tr1) / (float)nr + (float)lr21 * t2;
  else
    dtr = t2;
  /* columns */
  double x1 = (double)mad(atx, t1, px);
  int sgx = signbit(atx) ? 1 : 0;
  float lc1 = (float)((double)SZ_VOXY * (ceil(x1 / (double)SZ_VOXY) - sgx));
  int u = (int)(0.5 * SZ_IMX + floor(x1 / (double)SZ_VOXY));
  float x2 = mad(atx, t2, px);
  float cc2 = floorf(x2 / SZ_VOXY) + (float)sgx;
  float lc2 = SZ_VOXY * cc2;
  float tc1 = (lc1 - px) / atx;
  float tc2 = fmaf(SZ_VOXY, cc2, -px) / atx; /* as tr1/tr2 (lc1 is a double: no fusion) */
  int x21 = fabsf((float)((double)x2 - x1)) >= SZ_VOXY;
  int lc21 = fabsf(lc1 - lc2) < L21;
  int nc = (int)((float)x21 * roundf(fabsf(lc2 - lc1) / SZ_VOXY) + (float)lc21);
  float dtc;
  if (nc > 0)
    dtc = (tc2 - tc1) / (float)nc + (float)lc21 * t2;
  else
    dtc = t2;

  float ang = atanf(aty / atx);
  unsigned char *T = tv + (size_t)N_TV * idx;
  T[0] = atx >= 0 ? 2 : 0;
  T[1] = aty >= 0 ? 2 : 0;
  int k = 2;
  if ((ang < TA1) & (ang > TA2)) {
    float tf = tc1, ts = tr1;
    for (int i = 0; i <= nc; i++) {
      int tsin = (tf - ts) > 0;
      if (k < N_TV) T[k] = 1;
      k += tsin;
      ts += dtr * (float)tsin;
      if (k < N_TV) T[k] = 0;
      k += 1;
      tf += dtc;
    }
    if (tr2 > tc2) {
      if (k < N_TV) T[k] = 1;
      k += 1;
    }
  } else {
    float tf = tr1, ts = tc1;
    for (int i = 0; i <= nr; i++) {
      int tsin = (tf - ts) > 0;
      if (k < N_TV) T[k] = 0;
      k += tsin;
      ts += dtc * (float)tsin;
      if (k < N_TV) T[k] = 1;
      k += 1;
      tf += dtr;
    }
    if (tc2 > tr2) {
      if (k < N_TV) T[k] = 0;
      k += 1;
    }
  }
  float *t = tt + (size_t)N_TT * idx;
  t[0] = tr1;
  t[1] = tc1;
  t[2] = dtr;
  t[3] = dtc;
  t[4] = t1;
  t[5] = fminf(tr1, tc1);
  t[6] = t2;
  t[7] = atn;
  t[8] = (float)(u + (v << UV_SHFT));
  t[9] = (float)k;
}

void orc_siddon_tables(const float *crs, const short *s2c, int naw, float *tt,
                       unsigned char *tv) {
  memset(tv, 0, (size_t)N_TV * naw);
#pragma omp parallel for schedule(static)
  for (int i = 0; i < naw; i++) siddon_one(crs, s2c, i, tt, tv);
}

/* ========================================================================
 * The transaxial walk shared by every ray of one LOR (prjf.cu:49-86).
 * Expands the LOR into its step list: voxel column offset uv (image index
 * z + 127*(x + 320*y) with z = 0) and the float entry/exit parameters tp, tn.
 * Returns the number of steps.
 * ====================================================================== */
static int expand_lor(const float *tt, const unsigned char *tv, int ixt, int *uvs, float *tps,
                      float *tns, int cap) {
  const float *t = tt + (size_t)N_TT * ixt;
  const unsigned char *T = tv + (size_t)N_TV * ixt;
  int sgna0 = T[0] - 1, sgna1 = T[1] - 1;
  int rbit = T[2] & 1;
  int u = (int)t[8];
  int v = u >> UV_SHFT;
  int uv = SZ_IMZ * ((u & 0x1ff) + SZ_IMX * v);
  uv += !rbit * sgna0 * SZ_IMZ;
  uv -= rbit * sgna1 * SZ_IMZ * SZ_IMX;
  float dtr = t[2], dtc = t[3];
  float trc = mad((float)rbit, dtr, t[0]);
  float tcc = mad(dtc, (float)!rbit, t[1]);
  rbit = T[3] & 1;
  float tn = mad(trc, (float)rbit, tcc * (float)!rbit);
  float tp = t[5];
  int K = (int)t[9], n = 0;
  for (int k = 3; k < K; k++) {
    if (n < cap) {
      uvs[n] = uv;
      tps[n] = tp;
      tns[n] = tn;
    }
    n++;
    trc = mad(dtr, (float)rbit, trc);
    tcc = mad(dtc, (float)!rbit, tcc);
    uv += !rbit * sgna0 * SZ_IMZ;
    uv -= rbit * sgna1 * SZ_IMZ * SZ_IMX;
    tp = tn;
    rbit = (k + 1 < N_TV) ? (T[k + 1] & 1) : 0;
    tn = mad(trc, (float)rbit, tcc * (float)!rbit);
  }
  return n;
}

#define STEP_CAP 1024

/* Axial set-up of one oblique ring pair (prjf.cu:136-160). */
typedef struct {
  double s;      /* sqrt(1 + (dz/atn)^2), the oblique path-length factor */
  int w, w_;     /* start voxel (z) of the +RD and -RD rays */
  int sgnaz;
  float tzc, dtz; /* next axial crossing and its increment (float, as the reference) */
} axial_t;

/* z position in voxels, .5*SZ_IMZ + SZ_VOXZi*z, and a z plane, c*SZ_VOXZ - .5*SZ_IMZ*SZ_VOXZ,
 * as the compiled reference evaluates them (prjf.cu:39, 148-155, prjb.cu alike): the double
 * sums are narrowed to float (exact for these operands) and the multiply-add fused, so the
 * product is not rounded.  This decides which voxel a ray whose position falls on a plane
 * starts in; checked against the reference's own projections on every LOR. */
static inline float zpos(float z) { return fmaf(SZ_VOXZi, z, (float)(.5 * SZ_IMZ)); }
static inline float zline(float c) { return fmaf(c, SZ_VOXZ, (float)(-.5 * SZ_IMZ * SZ_VOXZ)); }
static inline int zvox(float z) { return (int)floorf(zpos(z)); }

static void axial_setup(const float *li2rng, int ixz, float atn, float tp, float t2,
                        axial_t *A) {
  float r0 = li2rng[2 * ixz], r1 = li2rng[2 * ixz + 1];
  float az = r1 - r0;
  float az_atn = az / atn;
  A->s = sqrt((double)az_atn * (double)az_atn + 1.0);
  A->sgnaz = az >= 0 ? 1 : -1;
  float pz = (float)((double)r0 + .5 * SZ_RING);
  float z = mad(az_atn, tp, pz);
  A->w = zvox(z);
  float lz1 = zline(ceilf(zpos(z)));
  z = (float)((double)r1 + .5 * SZ_RING - (double)(az_atn * tp));
  A->w_ = zvox(z);
  z = mad(az_atn, t2, pz);
  float lz2 = zline(floorf(zpos(z)));
  int nz = (int)(fabsf(lz2 - lz1) / SZ_VOXZ);
  float tz1 = (lz1 - pz) / az_atn;
  float tz2 = (lz2 - pz) / az_atn;
  A->dtz = (tz2 - tz1) / (float)nz;
  A->tzc = tz1;
}

static long long g_oob = 0; /* voxel reads/writes whose z left [0,127) (counted, skipped) */
long long orc_oob_count(void) { return g_oob; }

static inline double img_get(const float *im, int uv, int w, long long *oob) {
  if (w < 0 || w >= SZ_IMZ) {
    (*oob)++;
    return 0.0;
  }
  return (double)im[uv + w];
}

/* ========================================================================
 * Forward projection (prjf.cu:33-206).  sino: [nprj][snno] double, zeroed here.
 * li2sn: span-11 (li2sn) or span-1 (li2sn1) pairs; att: 0 emission, 1 attenuation.
 * ====================================================================== */
void orc_fprj(const float *tt, const unsigned char *tv, const float *li2rng, const short *li2sn,
              const signed char *li2nos, int span, int snno, const float *im, const int *subs,
              int nprj, int att, double *sino) {
  long long oob = 0;
  memset(sino, 0, sizeof(double) * (size_t)nprj * snno);
#pragma omp parallel reduction(+ : oob)
  {
    int *uvs = malloc(sizeof(int) * STEP_CAP);
    float *tps = malloc(sizeof(float) * STEP_CAP), *tns = malloc(sizeof(float) * STEP_CAP);
#pragma omp for schedule(dynamic, 16)
    for (int p = 0; p < nprj; p++) {
      int ixt = subs ? subs[p] : p;
      int n = expand_lor(tt, tv, ixt, uvs, tps, tns, STEP_CAP);
      const float *t = tt + (size_t)N_TT * ixt;
      double *row = sino + (size_t)p * snno;
      /* direct planes: one ray per ring */
      for (int ixz = 0; ixz < NRINGS; ixz++) {
        float z = (float)((double)li2rng[2 * ixz] + .5 * SZ_RING);
        int w = zvox(z);
        double acc = 0;
        for (int k = 0; k < n; k++) acc += ((double)tns[k] - tps[k]) * img_get(im, uvs[k], w, &oob);
        int o = li2sn[2 * ixz];
        if (att == 1) {
          if (span == 1)
            row[o] = exp(-acc);
          else
            row[o] += exp(-acc) / (double)li2nos[ixz];
        } else
          row[o] += acc;
      }
      /* oblique ring pairs: the +RD and -RD rays share the transaxial walk */
      for (int ixz = NRINGS; ixz < NLI2R; ixz++) {
        axial_t A;
        axial_setup(li2rng, ixz, t[7], t[5], t[6], &A);
        int w = A.w, w_ = A.w_;
        float tzc = A.tzc;
        double acc = 0, acc_ = 0;
        for (int k = 0; k < n; k++) {
          float tn = tns[k], tp = tps[k];
          if ((tn - tzc) > 0) {
            double a = (double)tzc - tp, b = (double)tn - tzc;
            acc += a * img_get(im, uvs[k], w, &oob);
            acc_ += a * img_get(im, uvs[k], w_, &oob);
            w += A.sgnaz;
            w_ -= A.sgnaz;
            acc += b * img_get(im, uvs[k], w, &oob);
            acc_ += b * img_get(im, uvs[k], w_, &oob);
            tzc += A.dtz;
          } else {
            double l = (double)tn - tp;
            acc += l * img_get(im, uvs[k], w, &oob);
            acc_ += l * img_get(im, uvs[k], w_, &oob);
          }
        }
        acc *= A.s;
        acc_ *= A.s;
        int o0 = li2sn[2 * ixz], o1 = li2sn[2 * ixz + 1];
        if (att == 1) {
          if (span == 1) {
            row[o0] = exp(-acc);
            row[o1] = exp(-acc_);
          } else {
            row[o0] += exp(-acc) / (double)li2nos[ixz];
            row[o1] += exp(-acc_) / (double)li2nos[ixz];
          }
        } else {
          row[o0] += acc;
          row[o1] += acc_;
        }
      }
    }
    free(uvs);
    free(tps);
    free(tns);
  }
  g_oob += oob;
}

/* ========================================================================
 * Back projection (prjb.cu:33-187), the exact transpose of orc_fprj (att=0).
 * sino: [nprj][snno] float; im: [320*320*127] double, zeroed here.
 * ====================================================================== */
void orc_bprj(const float *tt, const unsigned char *tv, const float *li2rng, const short *li2sn,
              int snno, const float *sino, const int *subs, int nprj, double *im) {
  long long oob = 0;
  memset(im, 0, sizeof(double) * NVOX);
  int nth = orc_num_threads();
  double **priv = calloc(nth, sizeof(double *));
#pragma omp parallel reduction(+ : oob)
  {
    int tid = 0;
#ifdef _OPENMP
    tid = omp_get_thread_num();
#endif
    double *acc = calloc(NVOX, sizeof(double));
    priv[tid] = acc;
    int *uvs = malloc(sizeof(int) * STEP_CAP);
    float *tps = malloc(sizeof(float) * STEP_CAP), *tns = malloc(sizeof(float) * STEP_CAP);
#define PUT(uv, w, val)                                                                         \
  do {                                                                                          \
    int _w = (w);                                                                               \
    if (_w < 0 || _w >= SZ_IMZ)                                                                 \
      oob++;                                                                                    \
    else                                                                                        \
      acc[(uv) + _w] += (val);                                                                  \
  } while (0)
#pragma omp for schedule(dynamic, 16)
    for (int p = 0; p < nprj; p++) {
      int ixt = subs ? subs[p] : p;
      int n = expand_lor(tt, tv, ixt, uvs, tps, tns, STEP_CAP);
      const float *t = tt + (size_t)N_TT * ixt;
      const float *row = sino + (size_t)p * snno;
      for (int ixz = 0; ixz < NRINGS; ixz++) {
        double bin = row[li2sn[2 * ixz]];
        float z = (float)((double)li2rng[2 * ixz] + .5 * SZ_RING);
        int w = zvox(z);
        for (int k = 0; k < n; k++) PUT(uvs[k], w, ((double)tns[k] - tps[k]) * bin);
      }
      for (int ixz = NRINGS; ixz < NLI2R; ixz++) {
        double bin = row[li2sn[2 * ixz]], bin_ = row[li2sn[2 * ixz + 1]];
        axial_t A;
        axial_setup(li2rng, ixz, t[7], t[5], t[6], &A);
        int w = A.w, w_ = A.w_;
        float tzc = A.tzc;
        for (int k = 0; k < n; k++) {
          float tn = tns[k], tp = tps[k];
          if ((tn - tzc) > 0) {
            double a = ((double)tzc - tp) * A.s, b = ((double)tn - tzc) * A.s;
            PUT(uvs[k], w, a * bin);
            PUT(uvs[k], w_, a * bin_);
            w += A.sgnaz;
            w_ -= A.sgnaz;
            PUT(uvs[k], w, b * bin);
            PUT(uvs[k], w_, b * bin_);
            tzc += A.dtz;
          } else {
            double l = ((double)tn - tp) * A.s;
            PUT(uvs[k], w, l * bin);
            PUT(uvs[k], w_, l * bin_);
          }
        }
      }
    }
#undef PUT
    free(uvs);
    free(tps);
    free(tns);
  }
  /* deterministic reduction of the per-thread images */
#pragma omp parallel for schedule(static)
  for (int i = 0; i < NVOX; i++) {
    double s = 0;
    for (int t = 0; t < nth; t++)
      if (priv[t]) s += priv[t][i];
    im[i] = s;
  }
  for (int t = 0; t < nth; t++) free(priv[t]);
  free(priv);
  g_oob += oob;
}

/* Number of Siddon voxel reads of a forward projection over `nprj` LORs
 * (direct: one per step; oblique: two per step, four at an axial crossing). */
long long orc_count_reads(const float *tt, const unsigned char *tv, const float *li2rng,
                          const int *subs, int nprj) {
  long long tot = 0;
#pragma omp parallel reduction(+ : tot)
  {
    int *uvs = malloc(sizeof(int) * STEP_CAP);
    float *tps = malloc(sizeof(float) * STEP_CAP), *tns = malloc(sizeof(float) * STEP_CAP);
#pragma omp for schedule(dynamic, 16)
    for (int p = 0; p < nprj; p++) {
      int ixt = subs ? subs[p] : p;
      int n = expand_lor(tt, tv, ixt, uvs, tps, tns, STEP_CAP);
      const float *t = tt + (size_t)N_TT * ixt;
      tot += (long long)NRINGS * n;
      for (int ixz = NRINGS; ixz < NLI2R; ixz++) {
        axial_t A;
        axial_setup(li2rng, ixz, t[7], t[5], t[6], &A);
        float tzc = A.tzc;
        for (int k = 0; k < n; k++) {
          if ((tns[k] - tzc) > 0) {
            tot += 4;
            tzc += A.dtz;
          } else
            tot += 2;
        }
      }
    }
    free(uvs);
    free(tps);
    free(tns);
  }
  return tot;
}

/* Every (LOR, ring pair, sign, step) at which a ray's axial voxel leaves [0, 127):
 * writes up to `cap` records (lor, li, sign(+1/-1/0 direct), step, w); returns the count. */
int orc_scan_oob(const float *tt, const unsigned char *tv, const float *li2rng, int naw,
                 int *rec, int cap) {
  int cnt = 0;
  int *uvs = malloc(sizeof(int) * STEP_CAP);
  float *tps = malloc(sizeof(float) * STEP_CAP), *tns = malloc(sizeof(float) * STEP_CAP);
  for (int p = 0; p < naw; p++) {
    int n = expand_lor(tt, tv, p, uvs, tps, tns, STEP_CAP);
    const float *t = tt + (size_t)N_TT * p;
    for (int ixz = NRINGS; ixz < NLI2R; ixz++) {
      axial_t A;
      axial_setup(li2rng, ixz, t[7], t[5], t[6], &A);
      int w = A.w, w_ = A.w_;
      float tzc = A.tzc;
      for (int k = -1; k < n; k++) {
        if (k >= 0 && (tns[k] - tzc) > 0) {
          w += A.sgnaz;
          w_ -= A.sgnaz;
          tzc += A.dtz;
        }
        int ws[2] = {w, w_};
        for (int q = 0; q < 2; q++)
          if (ws[q] < 0 || ws[q] >= SZ_IMZ) {
            if (cnt < cap) {
              int *r = rec + 5 * cnt;
              r[0] = p;
              r[1] = ixz;
              r[2] = q ? -1 : 1;
              r[3] = k;
              r[4] = ws[q];
            }
            cnt++;
          }
      }
    }
  }
  free(uvs);
  free(tps);
  free(tns);
  return cnt;
}

/* Step count of every LOR (prjf.cu loop trip count, tt[9]-3). */
void orc_step_counts(const float *tt, int naw, int *nsteps) {
  for (int i = 0; i < naw; i++) nsteps[i] = (int)tt[(size_t)N_TT * i + 9] - 3;
}

/* ========================================================================
 * One OSEM iteration over all subsets (recon.cu:318-497, PSF off).
 * img: [NVOX] double in/out.  psng: [AW][snno] uint16 prompts.  rsng, ssng, nsng,
 * asng: [AW][snno] float.  subs: [nsub][nprj].  sens: [nsub][NVOX] double.
 * msk: [NVOX] uint8.
 * ====================================================================== */
#define WITHIN_EPS(x) (-0.000001 < (x) && (x) < 0.000001)
void orc_osem_iter(double *img, const unsigned short *psng, const float *rsng, const float *ssng,
                   const float *nsng, const float *asng, const int *subs, int nsub, int nprj,
                   const double *sens, const unsigned char *msk, const float *tt,
                   const unsigned char *tv, const float *li2rng, const short *li2sn, int snno) {
  size_t nb = (size_t)AW * snno;
  /* (r+s)/(a*n) with the eldiv0 epsilon rule, recon.cu:381-398 */
  double *rs = malloc(sizeof(double) * nb);
#pragma omp parallel for schedule(static)
  for (size_t i = 0; i < nb; i++) {
    double an = (double)asng[i] * (double)nsng[i];
    double r = (double)rsng[i] + (double)ssng[i];
    rs[i] = WITHIN_EPS(an) ? 0.0 : r / an;
  }
  float *imf = malloc(sizeof(float) * NVOX);
  double *esng = malloc(sizeof(double) * (size_t)nprj * snno);
  float *ratio = malloc(sizeof(float) * (size_t)nprj * snno);
  double *bimg = malloc(sizeof(double) * NVOX);
  for (int s = 0; s < nsub; s++) {
    const int *sub = subs + (size_t)s * nprj;
    for (int i = 0; i < NVOX; i++) imf[i] = (float)img[i];
    orc_fprj(tt, tv, li2rng, li2sn, NULL, 11, snno, imf, sub, nprj, 0, esng);
#pragma omp parallel for schedule(static)
    for (int p = 0; p < nprj; p++)
      for (int j = 0; j < snno; j++) {
        size_t g = (size_t)sub[p] * snno + j;
        double e = esng[(size_t)p * snno + j] + rs[g];
        ratio[(size_t)p * snno + j] = WITHIN_EPS(e) ? 0.0f : (float)((double)psng[g] / e);
      }
    orc_bprj(tt, tv, li2rng, li2sn, snno, ratio, sub, nprj, bimg);
    const double *sn = sens + (size_t)s * NVOX;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < NVOX; i++) {
      double b = WITHIN_EPS(sn[i]) ? 0.0 : bimg[i] / sn[i];
      img[i] = msk[i] ? img[i] * b : 0.0;
    }
  }
  free(rs);
  free(imf);
  free(esng);
  free(ratio);
  free(bimg);
}

/* ========================================================================
 * One OSEM iteration over all subsets for B images at once (recon.cu:318-497 applied to
 * every image, PSF off), as orc_osem_iter does for one: image b has its own prompts
 * psng[b] and randoms + scatter scaled by rscale[b]; attenuation, normalisation, the
 * sensitivity images and the mask are shared.  For each LOR of a subset the forward
 * projection of all its rays (every sum in orc_fprj's order), the ratio y / (Ax + rscale
 * (r+s)/(an)) with the 1e-6 rules, and the back projection (orc_bprj's terms) are done for
 * all B images; the back projection is gathered per image column and added to the image
 * under a per-column lock, so its additions reach a voxel in a different
 * (double) order than orc_bprj's.
 * img: [B][NVOX] double in/out.  psng: [B][AW][snno] uint16.  rscale: [B] double.
 * rsng, ssng, nsng, asng: [AW][snno] float.  subs: [nsub][nprj].  sens: [nsub][NVOX]
 * double.  msk: [NVOX] uint8.  Span 11 (li2sn, snno 837) or span 1 (li2sn1, 4084).
 * ====================================================================== */
#define RBLK 128 /* rays whose forward sums are swept together */
void orc_osem_batch_iter(double *img, int B, const unsigned short *psng, const double *rscale,
                         const float *rsng, const float *ssng, const float *nsng,
                         const float *asng, const int *subs, int nsub, int nprj,
                         const double *sens, const unsigned char *msk, const float *tt,
                         const unsigned char *tv, const float *li2rng, const short *li2sn,
                         int snno) {
  const size_t nb = (size_t)AW * snno;
  const int NCOL = SZ_IMX * SZ_IMY;
  double *rs = malloc(sizeof(double) * nb);
#pragma omp parallel for schedule(static)
  for (size_t i = 0; i < nb; i++) {
    double an = (double)asng[i] * (double)nsng[i];
    double r = (double)rsng[i] + (ssng ? (double)ssng[i] : 0.0);
    rs[i] = WITHIN_EPS(an) ? 0.0 : r / an;
  }
  float *imf = malloc(sizeof(float) * (size_t)NVOX * B);    /* [NVOX][B] */
  double *bimg = malloc(sizeof(double) * (size_t)NVOX * B); /* [NVOX][B] */
#ifdef _OPENMP
  omp_lock_t *lk = malloc(sizeof(omp_lock_t) * NCOL);
  for (int c = 0; c < NCOL; c++) omp_init_lock(&lk[c]);
#endif
  long long oob = 0;
  for (int s = 0; s < nsub; s++) {
    const int *sub = subs + (size_t)s * nprj;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < NVOX; i++)
      for (int b = 0; b < B; b++) {
        imf[(size_t)i * B + b] = (float)img[(size_t)b * NVOX + i];
        bimg[(size_t)i * B + b] = 0.0;
      }
#pragma omp parallel reduction(+ : oob)
    {
      int *uvs = malloc(sizeof(int) * STEP_CAP);
      float *tps = malloc(sizeof(float) * STEP_CAP), *tns = malloc(sizeof(float) * STEP_CAP);
      axial_t *ax = malloc(sizeof(axial_t) * NLI2R);
      int *w0 = malloc(sizeof(int) * NLI2R), *w1 = malloc(sizeof(int) * NLI2R);
      float *tz = malloc(sizeof(float) * NLI2R);
      double *acc = malloc(sizeof(double) * 2 * RBLK * B); /* [ray pair][+/-][B] */
      double *fwd = malloc(sizeof(double) * snno * B);
      float *rat = malloc(sizeof(float) * snno * B);
      double *col = malloc(sizeof(double) * SZ_IMZ * B);
      float *zf = calloc(B, sizeof(float));
      double *sink = calloc(B, sizeof(double));
/* the B values of voxel w of the current column, or zeros (counted) outside [0, 127) */
#define VOX(w) (((w) >= 0 && (w) < SZ_IMZ) ? c + (size_t)(w) * B : (oob += B, zf))
/* the B accumulators of voxel w of the current column, or a discarded sink (counted)
 * outside [0, 127) */
#define SLOT(w) (((w) >= 0 && (w) < SZ_IMZ) ? col + (size_t)(w) * B : (oob += B, sink))
#pragma omp for schedule(dynamic, 4)
      for (int p = 0; p < nprj; p++) {
        const int ixt = sub[p];
        const int n = expand_lor(tt, tv, ixt, uvs, tps, tns, STEP_CAP);
        const float *t = tt + (size_t)N_TT * ixt;
        for (int ixz = 0; ixz < NRINGS; ixz++)
          w0[ixz] = zvox((float)((double)li2rng[2 * ixz] + .5 * SZ_RING));
        for (int ixz = NRINGS; ixz < NLI2R; ixz++) {
          axial_setup(li2rng, ixz, t[7], t[5], t[6], &ax[ixz]);
          w0[ixz] = ax[ixz].w;
          w1[ixz] = ax[ixz].w_;
          tz[ixz] = ax[ixz].tzc;
        }
        /* forward projection of every ray of the LOR, in blocks of RBLK rays: each ray's
         * sum runs over the steps in order (orc_fprj's sums); the block's accumulators stay
         * in cache while the steps are swept */
        memset(fwd, 0, sizeof(double) * snno * B);
        for (int r0 = 0; r0 < NLI2R; r0 += RBLK) {
          const int r1 = r0 + RBLK < NLI2R ? r0 + RBLK : NLI2R;
          memset(acc, 0, sizeof(double) * 2 * RBLK * B);
          for (int k = 0; k < n; k++) {
            const float *c = imf + (size_t)uvs[k] * B;
            const float tn = tns[k], tp = tps[k];
            const double l = (double)tn - tp;
            for (int ixz = r0; ixz < r1; ixz++) {
              double *A0 = acc + (size_t)2 * (ixz - r0) * B, *A1 = A0 + B;
              if (ixz < NRINGS) {
                const float *v0 = VOX(w0[ixz]);
                for (int b = 0; b < B; b++) A0[b] += l * (double)v0[b];
              } else if ((tn - tz[ixz]) > 0) {
                const double a = (double)tz[ixz] - tp, bb = (double)tn - tz[ixz];
                const float *v0 = VOX(w0[ixz]), *v1 = VOX(w1[ixz]);
                for (int b = 0; b < B; b++) {
                  A0[b] += a * (double)v0[b];
                  A1[b] += a * (double)v1[b];
                }
                w0[ixz] += ax[ixz].sgnaz;
                w1[ixz] -= ax[ixz].sgnaz;
                v0 = VOX(w0[ixz]);
                v1 = VOX(w1[ixz]);
                for (int b = 0; b < B; b++) {
                  A0[b] += bb * (double)v0[b];
                  A1[b] += bb * (double)v1[b];
                }
                tz[ixz] += ax[ixz].dtz;
              } else {
                const float *v0 = VOX(w0[ixz]), *v1 = VOX(w1[ixz]);
                for (int b = 0; b < B; b++) {
                  A0[b] += l * (double)v0[b];
                  A1[b] += l * (double)v1[b];
                }
              }
            }
          }
          for (int ixz = r0; ixz < r1; ixz++) {
            const double *A0 = acc + (size_t)2 * (ixz - r0) * B, *A1 = A0 + B;
            if (ixz < NRINGS) {
              for (int b = 0; b < B; b++) fwd[(size_t)li2sn[2 * ixz] * B + b] += A0[b];
            } else {
              const int o0 = li2sn[2 * ixz], o1 = li2sn[2 * ixz + 1];
              for (int b = 0; b < B; b++) {
                fwd[(size_t)o0 * B + b] += A0[b] * ax[ixz].s;
                fwd[(size_t)o1 * B + b] += A1[b] * ax[ixz].s;
              }
            }
          }
        }
        /* ratio, recon.cu:459-470 (sneladd, sneldiv) */
        for (int j = 0; j < snno; j++) {
          const size_t g = (size_t)ixt * snno + j;
          for (int b = 0; b < B; b++) {
            const double e = fwd[(size_t)j * B + b] + rscale[b] * rs[g];
            rat[(size_t)j * B + b] =
                WITHIN_EPS(e) ? 0.0f : (float)((double)psng[(size_t)b * nb + g] / e);
          }
        }
        /* back projection of the ratio (orc_bprj's terms), one image column at a time */
        for (int ixz = 0; ixz < NRINGS; ixz++)
          w0[ixz] = zvox((float)((double)li2rng[2 * ixz] + .5 * SZ_RING));
        for (int ixz = NRINGS; ixz < NLI2R; ixz++) {
          w0[ixz] = ax[ixz].w;
          w1[ixz] = ax[ixz].w_;
          tz[ixz] = ax[ixz].tzc;
        }
        for (int k = 0; k < n; k++) {
          const float tn = tns[k], tp = tps[k];
          memset(col, 0, sizeof(double) * SZ_IMZ * B);
          for (int ixz = 0; ixz < NRINGS; ixz++) {
            const float *bin = rat + (size_t)li2sn[2 * ixz] * B;
            const double l = (double)tn - tp;
            double *d0 = SLOT(w0[ixz]);
            for (int b = 0; b < B; b++) d0[b] += l * (double)bin[b];
          }
          for (int ixz = NRINGS; ixz < NLI2R; ixz++) {
            const float *bin = rat + (size_t)li2sn[2 * ixz] * B;
            const float *bin_ = rat + (size_t)li2sn[2 * ixz + 1] * B;
            if ((tn - tz[ixz]) > 0) {
              const double a = ((double)tz[ixz] - tp) * ax[ixz].s;
              const double bb = ((double)tn - tz[ixz]) * ax[ixz].s;
              double *d0 = SLOT(w0[ixz]), *d1 = SLOT(w1[ixz]);
              for (int b = 0; b < B; b++) {
                d0[b] += a * (double)bin[b];
                d1[b] += a * (double)bin_[b];
              }
              w0[ixz] += ax[ixz].sgnaz;
              w1[ixz] -= ax[ixz].sgnaz;
              d0 = SLOT(w0[ixz]);
              d1 = SLOT(w1[ixz]);
              for (int b = 0; b < B; b++) {
                d0[b] += bb * (double)bin[b];
                d1[b] += bb * (double)bin_[b];
              }
              tz[ixz] += ax[ixz].dtz;
            } else {
              const double l = ((double)tn - tp) * ax[ixz].s;
              double *d0 = SLOT(w0[ixz]), *d1 = SLOT(w1[ixz]);
              for (int b = 0; b < B; b++) {
                d0[b] += l * (double)bin[b];
                d1[b] += l * (double)bin_[b];
              }
            }
          }
          double *dst = bimg + (size_t)uvs[k] * B;
#ifdef _OPENMP
          omp_set_lock(&lk[uvs[k] / SZ_IMZ]);
#endif
          for (int i = 0; i < SZ_IMZ * B; i++) dst[i] += col[i];
#ifdef _OPENMP
          omp_unset_lock(&lk[uvs[k] / SZ_IMZ]);
#endif
        }
      }
#undef VOX
#undef SLOT
      free(uvs);
      free(tps);
      free(tns);
      free(ax);
      free(w0);
      free(w1);
      free(tz);
      free(acc);
      free(fwd);
      free(rat);
      free(col);
      free(zf);
      free(sink);
    }
    const double *sn = sens + (size_t)s * NVOX;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < NVOX; i++)
      for (int b = 0; b < B; b++) {
        const double q = WITHIN_EPS(sn[i]) ? 0.0 : bimg[(size_t)i * B + b] / sn[i];
        double *x = img + (size_t)b * NVOX + i;
        *x = msk[i] ? *x * q : 0.0;
      }
  }
  g_oob += oob;
#ifdef _OPENMP
  for (int c = 0; c < NCOL; c++) omp_destroy_lock(&lk[c]);
  free(lk);
#endif
  free(rs);
  free(imf);
  free(bimg);
}

/* ========================================================================
 * Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11).
 * ====================================================================== */
void orc_philox4x32(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
  uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
  uint32_t k0 = key[0], k1 = key[1];
  for (int r = 0; r < 10; r++) {
    uint64_t p0 = (uint64_t)0xD2511F53u * c0;
    uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
    uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    c0 = hi1 ^ c1 ^ k0;
    c1 = lo1;
    c2 = hi0 ^ c3 ^ k1;
    c3 = lo0;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  out[0] = c0;
  out[1] = c1;
  out[2] = c2;
  out[3] = c3;
}

/* Integer inverse-CDF thresholds for Poisson(lam), n = 0..31:
 * thr[n] = ceil(2^32 * P(X <= n)), saturated at 2^32. */
void orc_poisson_thresholds(double lam, uint64_t thr[32]) {
  double pmf = exp(-lam), cdf = 0;
  for (int n = 0; n < 32; n++) {
    if (n > 0) pmf = pmf * lam / (double)n;
    cdf += pmf;
    double t = ceil(cdf * 4294967296.0);
    thr[n] = t >= 4294967296.0 ? 4294967296ull : (uint64_t)t;
  }
}

static inline uint32_t boot_draw(uint64_t seed, int rep, uint64_t gidx, uint32_t stream) {
  uint32_t ctr[4] = {(uint32_t)gidx, (uint32_t)(gidx >> 32), (uint32_t)rep, stream};
  uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
  uint32_t o[4];
  orc_philox4x32(ctr, key, o);
  return o[0];
}

/* Poisson bootstrap uniform of replicate `rep` for word `gidx`: output rep % 4 of the
 * Philox block with counter (gidx, rep / 4, 0) -- one block serves four replicates. */
static inline uint32_t boot_draw_pois(uint64_t seed, int rep, uint64_t gidx) {
  uint32_t ctr[4] = {(uint32_t)gidx, (uint32_t)(gidx >> 32), (uint32_t)rep >> 2, 0u};
  uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
  uint32_t o[4];
  orc_philox4x32(ctr, key, o);
  return o[rep & 3];
}

/* ========================================================================
 * List-mode chunk plan (lmaux.cu:17-226) and time-window selection
 * (lmaux.cu:229-270).  Arrays are caller-allocated with capacity `cap`.
 * Returns the number of chunks kept (>= 0) or a negative error.
 * ====================================================================== */
int orc_lm_plan(const int32_t *lm, int64_t ele, int tstart, int tstop, int cap, int64_t *atag,
                int64_t *btag, int *ele4chnk, int *ele4thrd, int *out_toff, int *out_nitag,
                int *out_last_ttag, int *out_tstart, int *out_tstop) {
  int64_t i0 = -1, i1 = -1;
  for (int64_t i = 0; i < ele; i++)
    if ((lm[i] >> 29) == -4) {
      i0 = i;
      break;
    }
  for (int64_t i = ele - 1; i >= 0; i--)
    if ((lm[i] >> 29) == -4) {
      i1 = i;
      break;
    }
  if (i0 < 0) return -1;
  int first = lm[i0] & 0x1fffffff, last = lm[i1] & 0x1fffffff;
  if (!(first < last)) return -2;
  int toff = first;
  int nitag = ((last - toff) + ITIME - 1) / ITIME;
  int nchnk_max = 10 + (int)((ele + ELECHNK - 1) / ELECHNK);
  if (nchnk_max + 1 > cap) return -3;
  int64_t *A = malloc(sizeof(int64_t) * (nchnk_max + 1));
  int64_t *Bt = malloc(sizeof(int64_t) * (nchnk_max + 1));
  int *E = malloc(sizeof(int) * nchnk_max), *ET = malloc(sizeof(int) * nchnk_max);
  A[0] = 0;
  Bt[0] = 0;
  int i = 0;
  while ((ele - A[i]) > (int64_t)ELECHNK) {
    i += 1;
    if (i >= nchnk_max) {
      free(A); free(Bt); free(E); free(ET);
      return -4;
    }
    int64_t pos = A[i - 1] + ELECHNK - 1, found = -1;
    for (; pos > A[i - 1]; pos--) {
      int wd = lm[pos];
      if ((wd >> 29) == -4 && ((wd & 0x1fffffff) % BTPTIME) == 0) {
        found = pos;
        break;
      }
    }
    if (found < 0) { /* the reference would loop forever here */
      free(A); free(Bt); free(E); free(ET);
      return -5;
    }
    Bt[i] = (lm[found] & 0x1fffffff) - toff;
    A[i] = found;
    E[i - 1] = (int)(A[i] - A[i - 1]);
    ET[i - 1] = (int)((A[i] - A[i - 1] + (TOTHRDS - 1)) / TOTHRDS);
  }
  i += 1;
  Bt[i] = last - toff + 1;
  A[i] = ele;
  ET[i - 1] = (int)((ele - A[i - 1] + (TOTHRDS - 1)) / TOTHRDS);
  E[i - 1] = (int)(ele - A[i - 1]);
  int nchnk = i;
  if (tstart == tstop) {
    tstart = 0;
    tstop = nitag;
  }
  int n0 = -1, n1 = -1, newn = 0;
  for (int n = 0; n < nchnk; n++)
    if (tstart <= (Bt[n + 1] / ITIME) && (Bt[n] / ITIME) < tstop) {
      if (n0 == -1) n0 = n;
      n1 = n;
      newn++;
    }
  int nn = 0;
  if (newn > 0) {
    atag[0] = A[n0];
    btag[0] = Bt[n0];
    for (int n = n0; n <= n1; n++) {
      atag[nn + 1] = A[n + 1];
      btag[nn + 1] = Bt[n + 1];
      ele4thrd[nn] = ET[n];
      ele4chnk[nn] = E[n];
      nn++;
    }
  }
  free(A); free(Bt); free(E); free(ET);
  *out_toff = toff;
  *out_nitag = nitag;
  *out_last_ttag = last;
  *out_tstart = tstart;
  *out_tstop = tstop;
  return newn;
}

/* ========================================================================
 * Histogram (hst.cu:37-244), one pass of the reference kernel over every
 * chunk of the plan, thread slice by thread slice, in file order.
 * btp: 0 none, 1 non-parametric, 2 parametric (Poisson(btprt)) bootstrap.
 * Outputs are caller-allocated and zeroed by the caller; all counters are
 * uint32 with wrap-around, like the reference.  Words past a chunk's end are
 * never read (the reference's last thread slices may read stale buffer words
 * there; see the design notes).
 * ====================================================================== */
void orc_hist(const int32_t *lm, int nchnk, const int64_t *atag, const int *ele4chnk,
              const int *ele4thrd, int toff, int nitag, int span, int btp, double btprt,
              uint64_t seed, int rep, int tstart, int tstop, const short *sn1_sn11,
              const short *sn1_ssrb, const short *sn1_rno, const short *s2cF,
              uint32_t *psino, uint32_t *ssrb, uint32_t *rprmt, uint32_t *rdlyd, int32_t *zR,
              int32_t *zM, uint32_t *snview, uint32_t *fansums, uint32_t *bucks) {
  uint64_t thr[32];
  orc_poisson_thresholds(btprt, thr);
  for (int n = 0; n < nchnk; n++) {
    int64_t off = atag[n];
    int elm = ele4chnk[n], e4t = ele4thrd[n];
    int64_t cend = off + elm;
    for (int idx = 0; idx < TOTHRDS; idx++) {
      int64_t i_start, i_stop;
      if (idx == TOTHRDS - 1) {
        i_stop = off + elm;
        i_start = off + (int64_t)(TOTHRDS - 1) * e4t;
      } else {
        i_stop = off + (int64_t)(idx + 1) * e4t;
        i_start = off + (int64_t)idx * e4t;
      }
      if (i_stop > cend) i_stop = cend;
      if (i_start >= i_stop) continue;
      /* the first time tag of the slice (a tag in its last word does not count) */
      int itag = nitag, itagu = 0;
      for (int64_t i = i_start; i < i_stop - 1; i++)
        if ((lm[i] >> 29) == -4) {
          int tv = (lm[i] & 0x1fffffff) - toff;
          itag = tv / ITIME;
          itagu = tv - itag * ITIME;
          break;
        }
      for (int64_t i = i_start; i < i_stop; i++) {
        int word = lm[i];
        uint32_t N = 1;
        if (btp == 1) {
          if (word > 0) {
            int64_t len = i_stop - i_start;
            int got = 0;
            for (uint32_t j = 0; j < 64 && !got; j++) {
              uint32_t x = boot_draw(seed, rep, (uint64_t)i, 1 + j);
              int64_t bi = (int64_t)(((uint64_t)x * (uint64_t)len) >> 32);
              if (lm[i_start + bi] > 0) {
                word = lm[i_start + bi];
                got = 1;
              }
            }
            if (!got) N = 0;
          }
        } else if (btp == 2) {
          uint32_t x = boot_draw_pois(seed, rep, (uint64_t)i);
          uint32_t k = 0;
          while (k < 32 && (uint64_t)x >= thr[k]) k++;
          N = k;
        }
        int val = word & 0x3fffffff;
        if (!((itag >= tstart) && (itag < tstop))) continue;
        if (word > 0) {
          if (N > 0 && N < 32) {
            int si = val / NSBINANG;
            if (si >= NSINOS) continue; /* malformed address: skipped */
            int aw = val - si * NSBINANG;
            int a = aw / NSBINS;
            int w = aw - a * NSBINS;
            int si11 = sn1_sn11[si];
            int si_ssrb = sn1_ssrb[si];
            int64_t addr;
            if (span == 1)
              addr = val;
            else if (span == 11)
              addr = (int64_t)si11 * NSBINANG + aw;
            else
              addr = (int64_t)si_ssrb * NSBINANG + aw;
            int P = (word >> 30);
            if (P == 1) {
              rprmt[itag] += N;
              ssrb[(int64_t)si_ssrb * NSBINANG + aw] += N;
              psino[addr] += N;
              zR[itag] = (int32_t)((uint32_t)zR[itag] + (uint32_t)si_ssrb);
              zM[itag] = (int32_t)((uint32_t)zM[itag] + N);
              int a0 = a == 0, a126 = a == 126;
              if ((a0 || a126) && itag < MXNITAG)
                snview[(int64_t)(itag >> VTIME) * SEG0 * NSBINS + si_ssrb * NSBINS + w] +=
                    N << (a126 * 8);
            } else {
              psino[addr] += N << 16;
              rdlyd[itag] += N;
              const short *rr = sn1_rno + 2 * si;
              const short *cc = s2cF + 2 * (a + NSANGLES * w);
              fansums[nCRS * rr[0] + cc[0]] += N;
              fansums[nCRS * rr[1] + cc[1]] += N;
            }
          }
        } else {
          if ((word >> 29) == -4) {
            itag = (val - toff) / ITIME;
            itagu = (val - toff) - itag * ITIME;
          } else if ((word >> 29) == -3) {
            unsigned ibck = (unsigned)((word & 0x1fffffff) >> 19);
            if (ibck < NBUCKTS) {
              int64_t b0 = ibck + (int64_t)NBUCKTS * itag;
              int64_t b1 = b0 + (int64_t)NBUCKTS * nitag;
              bucks[b0] += (uint32_t)(word & 0x0007ffff) << 3;
              bucks[b1] += (uint32_t)((word & 0x0007ffff) > 0) << 30;
              if (bucks[b1] == 0)
                bucks[b1] += (uint32_t)itagu;
              else
                bucks[b1] += (uint32_t)itagu << 10;
            }
          }
        }
      }
    }
  }
}
