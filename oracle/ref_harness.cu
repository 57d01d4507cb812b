// Test-only harness around the reference's own CUDA projectors, OSEM and list-mode
// histogrammer, randoms and normalisation.
//
// Built by oracle/build_ref.sh together with the reference sources
// (niftypet/nipet/prj/src/{prjf,prjb,tprj,recon}.cu, lm/src/{lmproc,hst,lmaux}.cu and
// src/scanner_0.cu, compiled in place from the reference tree, nothing copied) into
// oracle/_ref/, and used only by tests/ and bench.py's reference arm to check the oracle
// and time the reference.  The reference's Python glue (prj/src/prj_module.cu,
// lm/src/lm_module.cu) needs the un-vendored `cuvec` package, so these wrappers stand in
// for its argument handling: host arrays in, device buffers allocated and filled the way
// prj_module.cu:232-425 (fprj), :430-608 (bprj), :613-839 (osem) and
// lm_module.cu:174-391 (hist) do, the reference routine called, results copied back.
// Kernel time is measured with CUDA events around the reference call.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>

#include "lmproc.h"
#include "norm.h"
#include "rnd.h"
#include "prjb.h"
#include "prjf.h"
#include "recon.h"
#include "sct.h"

// resolution-modelling routines of prj/src/recon.cu (defined there, not in its header)
void setConvolutionKernel(float *krnl);
void d_pad(float *dst, float *src, const int z);
void d_unpad(float *dst, float *src, const int z);
void d_conv(float *d_buff, float *d_imgout, float *d_imgint, int Nvk, int Nvj, int Nvi);

namespace {

Cnst make_cnst(int span) {
  Cnst c;
  std::memset(&c, 0, sizeof(c));
  c.SPN = (char)span;
  c.RNG_STRT = 0;
  c.RNG_END = NRINGS;
  c.NRNG = NRINGS;
  c.NSN1 = NSINOS;
  c.NSN11 = NSINOS11;
  c.LOG = LOGWARNING;
  c.DEVID = 0;
  return c;
}

int nsinos(int span) { return span == 11 ? NSINOS11 : NSINOS; }

struct Tx {
  float4 *crs = nullptr;
  short2 *s2c = nullptr;
  float *tt = nullptr;
  unsigned char *tv = nullptr;
  int *subs = nullptr;
  cudaError_t err = cudaSuccess;

  Tx(const float *crs_h, int ncrs, const int16_t *s2c_h, const int *subs_h, int nprj) {
    chk(cudaMalloc(&crs, ncrs * sizeof(float4)));
    chk(cudaMemcpy(crs, crs_h, ncrs * sizeof(float4), cudaMemcpyHostToDevice));
    chk(cudaMalloc(&s2c, AW * sizeof(short2)));
    chk(cudaMemcpy(s2c, s2c_h, AW * sizeof(short2), cudaMemcpyHostToDevice));
    chk(cudaMalloc(&tt, (size_t)N_TT * AW * sizeof(float)));
    chk(cudaMalloc(&tv, (size_t)N_TV * AW));
    chk(cudaMemset(tv, 0, (size_t)N_TV * AW));
    chk(cudaMalloc(&subs, (size_t)nprj * sizeof(int)));
    if (subs_h) {
      chk(cudaMemcpy(subs, subs_h, (size_t)nprj * sizeof(int), cudaMemcpyHostToDevice));
    } else {
      int *all = new int[nprj];
      for (int i = 0; i < nprj; i++) all[i] = i;
      chk(cudaMemcpy(subs, all, (size_t)nprj * sizeof(int), cudaMemcpyHostToDevice));
      delete[] all;
    }
  }
  ~Tx() {
    cudaFree(crs);
    cudaFree(s2c);
    cudaFree(tt);
    cudaFree(tv);
    cudaFree(subs);
  }
  void chk(cudaError_t e) {
    if (err == cudaSuccess && e != cudaSuccess) err = e;
  }
};

}  // namespace

extern "C" {

// Forward projection of `im` ([320][320][127] float, host) into `sino` ([nprj][nsinos]
// float, host) by the reference's gpu_fprj; subs (host [nprj]) or NULL with nprj = 68516.
// *ms: device time of the gpu_fprj call (tables + projection kernels).  Returns a
// cudaError_t code (0 = success).
int ref_fprj(float *sino, const float *im, const int *subs, int nprj, int span, int att,
             const float *li2rng, const int16_t *li2sn, const int8_t *li2nos,
             const int16_t *s2c, const int *aw2ali, const float *crs, int ncrs, float *ms) {
  const int nsn = nsinos(span);
  Tx tx(crs, ncrs, s2c, subs, nprj);
  float *d_im = nullptr, *d_sn = nullptr;
  tx.chk(cudaMalloc(&d_im, (size_t)SZ_IMX * SZ_IMY * SZ_IMZ * sizeof(float)));
  tx.chk(cudaMemcpy(d_im, im, (size_t)SZ_IMX * SZ_IMY * SZ_IMZ * sizeof(float),
                    cudaMemcpyHostToDevice));
  tx.chk(cudaMalloc(&d_sn, (size_t)nprj * nsn * sizeof(float)));
  if (tx.err != cudaSuccess) return (int)tx.err;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, 0);
  gpu_fprj(d_sn, d_im, const_cast<float *>(li2rng), const_cast<short *>(li2sn),
           reinterpret_cast<char *>(const_cast<int8_t *>(li2nos)), tx.s2c,
           const_cast<int *>(aw2ali), tx.crs, tx.subs, tx.tt, tx.tv, nprj, AW, make_cnst(span),
           (char)att, false);
  cudaEventRecord(e1, 0);
  tx.chk(cudaEventSynchronize(e1));
  tx.chk(cudaGetLastError());
  float t = 0.f;
  cudaEventElapsedTime(&t, e0, e1);
  if (ms) *ms = t;
  tx.chk(cudaMemcpy(sino, d_sn, (size_t)nprj * nsn * sizeof(float), cudaMemcpyDeviceToHost));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(d_im);
  cudaFree(d_sn);
  return (int)tx.err;
}

// Back projection of `sino` ([nprj][nsinos], host) into `im` ([320][320][127], host,
// overwritten) by the reference's gpu_bprj.  Arguments as ref_fprj.
int ref_bprj(float *im, const float *sino, const int *subs, int nprj, int span,
             const float *li2rng, const int16_t *li2sn, const int8_t *li2nos,
             const int16_t *s2c, const float *crs, int ncrs, float *ms) {
  const int nsn = nsinos(span);
  Tx tx(crs, ncrs, s2c, subs, nprj);
  float *d_im = nullptr, *d_sn = nullptr;
  tx.chk(cudaMalloc(&d_im, (size_t)SZ_IMX * SZ_IMY * SZ_IMZ * sizeof(float)));
  tx.chk(cudaMalloc(&d_sn, (size_t)nprj * nsn * sizeof(float)));
  tx.chk(cudaMemcpy(d_sn, sino, (size_t)nprj * nsn * sizeof(float), cudaMemcpyHostToDevice));
  if (tx.err != cudaSuccess) return (int)tx.err;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, 0);
  gpu_bprj(d_im, d_sn, const_cast<float *>(li2rng), const_cast<short *>(li2sn),
           reinterpret_cast<char *>(const_cast<int8_t *>(li2nos)), tx.s2c, tx.crs, tx.subs,
           tx.tt, tx.tv, nprj, make_cnst(span), false);
  cudaEventRecord(e1, 0);
  tx.chk(cudaEventSynchronize(e1));
  tx.chk(cudaGetLastError());
  float t = 0.f;
  cudaEventElapsedTime(&t, e0, e1);
  if (ms) *ms = t;
  tx.chk(cudaMemcpy(im, d_im, (size_t)SZ_IMX * SZ_IMY * SZ_IMZ * sizeof(float),
                    cudaMemcpyDeviceToHost));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(d_im);
  cudaFree(d_sn);
  return (int)tx.err;
}

// The reduced-rings mode of the same routines (span 1, Cnt.RNG_STRT = rs, Cnt.RNG_END = re,
// with the range's axial LUTs from mmraux.reduce_rings): the image is the range's axial
// slab [320][320][nvz], nvz = 2 (re - rs) - 1, the sinogram [nprj][nsino] with
// nsino = (re - rs)^2 (less 12 for 64 rings).  gpu_fprj / gpu_bprj expand and reduce the
// slab themselves (prjf.cu:19-29, :255-266; prjb.cu:19-29, :286-296).
int ref_fprj_rng(float *sino, const float *im, const int *subs, int nprj, int rs, int re,
                 int att, const float *li2rng, const int16_t *li2sn1, const int8_t *li2nos,
                 const int16_t *s2c, const int *aw2ali, const float *crs, int ncrs, float *ms) {
  const int n = re - rs;
  const int nsn = n * n - (n == NRINGS ? 12 : 0);
  const size_t nvox = (size_t)SZ_IMX * SZ_IMY * (2 * n - 1);
  Cnst c = make_cnst(1);
  c.RNG_STRT = (char)rs;
  c.RNG_END = (char)re;
  Tx tx(crs, ncrs, s2c, subs, nprj);
  float *d_im = nullptr, *d_sn = nullptr;
  tx.chk(cudaMalloc(&d_im, nvox * sizeof(float)));
  tx.chk(cudaMemcpy(d_im, im, nvox * sizeof(float), cudaMemcpyHostToDevice));
  tx.chk(cudaMalloc(&d_sn, (size_t)nprj * nsn * sizeof(float)));
  if (tx.err != cudaSuccess) return (int)tx.err;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, 0);
  gpu_fprj(d_sn, d_im, const_cast<float *>(li2rng), const_cast<short *>(li2sn1),
           reinterpret_cast<char *>(const_cast<int8_t *>(li2nos)), tx.s2c,
           const_cast<int *>(aw2ali), tx.crs, tx.subs, tx.tt, tx.tv, nprj, AW, c, (char)att,
           false);
  cudaEventRecord(e1, 0);
  tx.chk(cudaEventSynchronize(e1));
  tx.chk(cudaGetLastError());
  float t = 0.f;
  cudaEventElapsedTime(&t, e0, e1);
  if (ms) *ms = t;
  tx.chk(cudaMemcpy(sino, d_sn, (size_t)nprj * nsn * sizeof(float), cudaMemcpyDeviceToHost));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(d_im);
  cudaFree(d_sn);
  return (int)tx.err;
}

int ref_bprj_rng(float *im, const float *sino, const int *subs, int nprj, int rs, int re,
                 const float *li2rng, const int16_t *li2sn1, const int8_t *li2nos,
                 const int16_t *s2c, const float *crs, int ncrs, float *ms) {
  const int n = re - rs;
  const int nsn = n * n - (n == NRINGS ? 12 : 0);
  const size_t nvox = (size_t)SZ_IMX * SZ_IMY * (2 * n - 1);
  Cnst c = make_cnst(1);
  c.RNG_STRT = (char)rs;
  c.RNG_END = (char)re;
  Tx tx(crs, ncrs, s2c, subs, nprj);
  float *d_im = nullptr, *d_sn = nullptr;
  // gpu_bprj back-projects into a full-size image of its own and copies the slab into d_im
  tx.chk(cudaMalloc(&d_im, (n == NRINGS ? (size_t)SZ_IMX * SZ_IMY * SZ_IMZ : nvox) *
                               sizeof(float)));
  tx.chk(cudaMalloc(&d_sn, (size_t)nprj * nsn * sizeof(float)));
  tx.chk(cudaMemcpy(d_sn, sino, (size_t)nprj * nsn * sizeof(float), cudaMemcpyHostToDevice));
  if (tx.err != cudaSuccess) return (int)tx.err;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, 0);
  gpu_bprj(d_im, d_sn, const_cast<float *>(li2rng), const_cast<short *>(li2sn1),
           reinterpret_cast<char *>(const_cast<int8_t *>(li2nos)), tx.s2c, tx.crs, tx.subs,
           tx.tt, tx.tv, nprj, c, false);
  cudaEventRecord(e1, 0);
  tx.chk(cudaEventSynchronize(e1));
  tx.chk(cudaGetLastError());
  float t = 0.f;
  cudaEventElapsedTime(&t, e0, e1);
  if (ms) *ms = t;
  tx.chk(cudaMemcpy(im, d_im, nvox * sizeof(float), cudaMemcpyDeviceToHost));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(d_im);
  cudaFree(d_sn);
  return (int)tx.err;
}

// One OSEM iteration over all subsets by the reference's osem(), updating `img`
// ([320][320][127], host) in place, as petprj.osem does; psf: the [3][17] resolution
// kernel, or NULL for none.  subs is the
// [nsub][nprj1] table (column 0 = projections in the subset, then the LOR indices), sens
// the [nsub][320][320][127] sensitivity images, msk a [320][320][127] byte mask (0/1),
// psng [68516][nsinos] uint16, rsng/ssng/nsng/asng [68516][nsinos] float.  *ms: time of
// the call including the reference's own host<->device transfers.
int ref_osem(float *img, const uint8_t *msk, const uint16_t *psng, const float *rsng,
             const float *ssng, const float *nsng, const float *asng, const int *subs, int nsub,
             int nprj1, const float *sens, const float *li2rng, const int16_t *li2sn,
             const int8_t *li2nos, const int16_t *s2c, const float *crs, int ncrs, int span,
             const float *psf, float *ms) {
  float krnl[3 * KERNEL_LENGTH];
  for (int i = 0; i < 3 * KERNEL_LENGTH; i++) krnl[i] = psf ? psf[i] : -1.f;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, 0);
  osem(img, reinterpret_cast<bool *>(const_cast<uint8_t *>(msk)),
       const_cast<unsigned short *>(psng), const_cast<float *>(rsng), const_cast<float *>(ssng),
       const_cast<float *>(nsng), const_cast<float *>(asng), const_cast<int *>(subs),
       const_cast<float *>(sens), krnl, const_cast<float *>(li2rng), const_cast<short *>(li2sn),
       reinterpret_cast<char *>(const_cast<int8_t *>(li2nos)), const_cast<short *>(s2c),
       const_cast<float *>(crs), nsub, nprj1, ncrs, make_cnst(span));
  cudaEventRecord(e1, 0);
  cudaError_t err = cudaEventSynchronize(e1);
  if (err == cudaSuccess) err = cudaGetLastError();
  float t = 0.f;
  cudaEventElapsedTime(&t, e0, e1);
  if (ms) *ms = t;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return (int)err;
}

// Transaxial Siddon tables of the reference's gpu_siddon_tx (prj/src/tprj.cu): tt
// [68516][N_TT] float and tv [68516][N_TV] bytes, host.  Returns a cudaError_t code.
int ref_tables(float *tt, uint8_t *tv, const int16_t *s2c, const float *crs, int ncrs) {
  Tx tx(crs, ncrs, s2c, nullptr, 1);
  if (tx.err != cudaSuccess) return (int)tx.err;
  gpu_siddon_tx(tx.crs, tx.s2c, tx.tt, tx.tv);
  tx.chk(cudaDeviceSynchronize());
  tx.chk(cudaGetLastError());
  tx.chk(cudaMemcpy(tt, tx.tt, (size_t)N_TT * AW * sizeof(float), cudaMemcpyDeviceToHost));
  tx.chk(cudaMemcpy(tv, tx.tv, (size_t)N_TV * AW, cudaMemcpyDeviceToHost));
  return (int)tx.err;
}

// List-mode file summary by the reference's getLMinfo (lm/src/lmaux.cu): number of
// one-second time tags.  bpe = bytes per event (4 for the mMR).
int ref_lminfo(const char *fname, int bpe, int *nitag) {
  Cnst c = make_cnst(11);
  c.BPE = bpe;
  c.LMOFF = 0;
  getLMinfo(const_cast<char *>(fname), c);
  *nitag = lmprop.nitag;
  free(lmprop.atag);
  free(lmprop.btag);
  free(lmprop.ele4chnk);
  free(lmprop.ele4thrd);
  return (int)cudaGetLastError();
}

// Histogram of a list-mode file by the reference's lmproc (lm/src/lmproc.cu), as
// mmr_lmproc.hist calls it (lm_module.cu:174-391); btp 0 (none), 1 or 2 (bootstrap with
// the reference's clock-seeded curand, btprt the Poisson mean): outputs sized by the
// caller for nitag time tags -- psn/dsn [tot_bins] uint16, ssr [127*86688], snv [sne],
// hcp/hcd/mss [nitag], fan [64*504], bck [2*224*nitag].  s2cF [86688][2], sn1_rno
// [4084][2], sn1_sn11 [4084], sn1_ssrb [4084] (txLUT / axLUT arrays).  *ms: time of
// the call (file reading included).
int ref_hist(const char *fname, int tstart, int tstop, int span, int btp, float btprt,
             const int16_t *s2cF,
             const int16_t *sn1_rno, const int16_t *sn1_sn11, const int16_t *sn1_ssrb,
             uint16_t *psn, uint16_t *dsn, uint32_t *ssr, uint32_t *snv, uint32_t *hcp,
             uint32_t *hcd, float *mss, uint32_t *fan, uint32_t *bck,
             unsigned long long *psm, unsigned long long *dsm, float *ms) {
  Cnst c = make_cnst(span);
  c.BPE = 4;
  c.LMOFF = 0;
  c.BTP = (char)btp;
  c.BTPRT = btprt;
  c.W = NSBINS;
  c.A = NSANGLES;
  c.NSN1 = NSINOS;
  axialLUT ax;
  std::memset(&ax, 0, sizeof(ax));
  ax.sn1_rno = const_cast<short *>(sn1_rno);
  ax.sn1_sn11 = const_cast<short *>(sn1_sn11);
  ax.sn1_ssrb = const_cast<short *>(sn1_ssrb);
  hstout out;
  std::memset(&out, 0, sizeof(out));
  out.psn = psn;
  out.dsn = dsn;
  out.ssr = ssr;
  out.snv = snv;
  out.hcp = hcp;
  out.hcd = hcd;
  out.mss = mss;
  out.fan = fan;
  out.bck = bck;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, 0);
  lmproc(out, const_cast<char *>(fname), tstart, tstop,
         reinterpret_cast<LORcc *>(const_cast<int16_t *>(s2cF)), ax, c);
  cudaEventRecord(e1, 0);
  cudaError_t err = cudaEventSynchronize(e1);
  if (err == cudaSuccess) err = cudaGetLastError();
  float t = 0.f;
  cudaEventElapsedTime(&t, e0, e1);
  if (ms) *ms = t;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  // lmproc fills the counts of its (by-value) output struct only in its own copy: sum here
  unsigned long long sp = 0, sd = 0;
  const size_t nb = span == 11 ? (size_t)TOT_BINS : (span == 1 ? (size_t)TOT_BINS_S1
                                                                 : (size_t)SEG0 * NSBINANG);
  for (size_t i = 0; i < nb; i++) {
    sp += psn[i];
    sd += dsn[i];
  }
  if (psm) *psm = sp;
  if (dsm) *dsm = sd;
  return (int)err;
}

// The reference's PSF convolution of one image (recon.cu: d_pad, d_conv, d_unpad with the
// kernel krnl [3][17]), host [320][320][127] in and out.
int ref_psf(float *out, const float *in, const float *krnl) {
  const size_t n = (size_t)SZ_IMX * SZ_IMY * SZ_IMZ, np = (size_t)SZ_IMX * SZ_IMY * (SZ_IMZ + 1);
  float *d_in = nullptr, *d_src = nullptr, *d_dst = nullptr, *d_tmp = nullptr;
  cudaError_t e = cudaMalloc(&d_in, n * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&d_src, np * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&d_dst, np * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&d_tmp, np * sizeof(float));
  if (e == cudaSuccess) e = cudaMemcpy(d_in, in, n * sizeof(float), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    setConvolutionKernel(const_cast<float *>(krnl));
    d_pad(d_src, d_in, 1);
    d_conv(d_tmp, d_dst, d_src, SZ_IMX, SZ_IMY, SZ_IMZ + 1);
    d_unpad(d_in, d_dst, 1);
    e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpy(out, d_in, n * sizeof(float), cudaMemcpyDeviceToHost);
  }
  cudaFree(d_in);
  cudaFree(d_src);
  cudaFree(d_dst);
  cudaFree(d_tmp);
  return (int)e;
}

// Randoms from the delayed fan sums by the reference's gpu_randoms (lm/src/rnd.cu:169-386),
// as mmr_lmproc.rand calls it (lm_module.cu:396-560): host arrays in and out -- rsn
// [nsinos][252][344], cmap [504][64], fansums [64][504]; txLUT crsri/cij/s2cr/aw2sn and
// axLUT sn1_rno/sn1_sn11.
int ref_randoms(float *rsn, float *cmap, const uint32_t *fansums, const int16_t *crsr,
                const int8_t *cij, const int16_t *s2cr, const int16_t *aw2sn,
                const int16_t *sn1_rno, const int16_t *sn1_sn11, int span) {
  Cnst c = make_cnst(span);
  c.A = NSANGLES;
  c.W = NSBINS;
  c.NCRS = nCRS;
  c.NCRSR = nCRSR;
  c.MRD = mxRD;
  txLUTs tx;
  std::memset(&tx, 0, sizeof(tx));
  tx.s2cr = reinterpret_cast<LORcc *>(const_cast<int16_t *>(s2cr));
  tx.aw2sn = reinterpret_cast<LORaw *>(const_cast<int16_t *>(aw2sn));
  tx.cij = reinterpret_cast<char *>(const_cast<int8_t *>(cij));
  tx.crsr = const_cast<short *>(crsr);
  tx.naw = AW;
  gpu_randoms(rsn, cmap, const_cast<unsigned int *>(fansums), tx,
              const_cast<short *>(sn1_rno), const_cast<short *>(sn1_sn11), c);
  cudaError_t e = cudaDeviceSynchronize();
  if (e == cudaSuccess) e = cudaGetLastError();
  return (int)e;
}

// Normalisation sinogram from its components by the reference's norm_from_components
// (src/norm.cu:54-210), as mmr_auxe.norm passes them (src/aux_module.cu:150-268): host
// arrays in, gap-free sino [68516][nsinos] out.  geo [ngeo0][344], cinf [344][9], ceff
// [64][504], axe1 [837], axf1 [4084] (read for both spans), dtp/dtnp [64], buckets [224];
// axLUT sn1_rno/sn1_sn11/sn1_sn11no; txLUT aw2ali.
int ref_norm(float *sino, const float *geo, int ngeo0, const float *cinf, const float *ceff,
             const float *axe1, const float *axf1, const float *dtp, const float *dtnp,
             const int *buckets, const int16_t *sn1_rno, const int16_t *sn1_sn11,
             const int8_t *sn1_sn11no, const int *aw2ali, int span) {
  Cnst c = make_cnst(span);
  NormCmp n;
  std::memset(&n, 0, sizeof(n));
  n.geo = const_cast<float *>(geo);
  n.cinf = const_cast<float *>(cinf);
  n.ceff = const_cast<float *>(ceff);
  n.axe1 = const_cast<float *>(axe1);
  n.axf1 = const_cast<float *>(axf1);
  n.dtp = const_cast<float *>(dtp);
  n.dtnp = const_cast<float *>(dtnp);
  n.ngeo[0] = ngeo0;
  n.ngeo[1] = NSBINS;
  n.ncinf[0] = NSBINS;
  n.ncinf[1] = 9;
  n.nceff[0] = NRINGS;
  n.nceff[1] = nCRS;
  n.naxe = NSINOS11;
  n.nrdt = NRINGS;
  axialLUT ax;
  std::memset(&ax, 0, sizeof(ax));
  ax.sn1_rno = const_cast<short *>(sn1_rno);
  ax.sn1_sn11 = const_cast<short *>(sn1_sn11);
  ax.sn1_sn11no = reinterpret_cast<char *>(const_cast<int8_t *>(sn1_sn11no));
  ax.Nli2rno[1] = 2;
  norm_from_components(sino, n, ax, const_cast<int *>(aw2ali), const_cast<int *>(buckets), c);
  cudaError_t e = cudaDeviceSynchronize();
  if (e == cudaSuccess) e = cudaGetLastError();
  return (int)e;
}

// Gap removal by the reference's remove_gaps (src/scanner_0.cu:107-156) as mmr_auxe.rgaps
// calls it (src/aux_module.cu:389-440): Siemens sino [snno][252*344] float (host) ->
// gap-free [68516][snno] float (host).
int ref_remgaps(float *sng, const float *sino, int snno, const int *aw2ali) {
  Cnst c = make_cnst(11);
  remove_gaps(sng, const_cast<float *>(sino), snno, const_cast<int *>(aw2ali), c);
  cudaError_t e = cudaDeviceSynchronize();
  if (e == cudaSuccess) e = cudaGetLastError();
  return (int)e;
}

// Gap insertion by the reference's put_gaps (src/scanner_0.cu:169-241) as mmr_auxe.pgaps
// calls it (src/aux_module.cu:299-387): gap-free [68516][snno] float (host) -> [252*344][snno]
// float (host, bin-major as put_gaps writes it; mmraux.putgaps transposes it to
// [snno][252][344]).  sino_no 0 takes snno from the span (837 or 4084), as pgaps does.
int ref_putgaps(float *sino, const float *sng, const int *aw2ali, int sino_no, int span) {
  Cnst c = make_cnst(span);
  put_gaps(sino, const_cast<float *>(sng), const_cast<int *>(aw2ali), sino_no, c);
  cudaError_t e = cudaDeviceSynchronize();
  if (e == cudaSuccess) e = cudaGetLastError();
  return (int)e;
}

// The reference's voxel-driven scatter model, prob_scatt (sct/src/sct.cu:338-582: raysLUT,
// Psct, srslt2sino), called as nifty_scatter.vsm does (sct/src/sct_module.cu:60-335): host
// mu-map [63][172][172] with its mask, emission image [43][114][114], the scatter LUTs and
// constants; non-TOF (TOFBINN 1).  Outputs on the host: sval [8][64][8][64] and s3d
// [nsn][64][64] (nsn 4096 at span 1, 837 at span 11).
int ref_sct(float *sval, float *s3d, float *mu, int8_t *mumsk, float *em, float *knlut,
            float cosupsmx, float ethrld, int *sctaxR, float *sctaxW, int16_t *offseg,
            float *scrs, int16_t *isrng, float *srng, int8_t *xsxu, int16_t *sn1_rno,
            int16_t *sn1_sn11, int span) {
  Cnst c = make_cnst(span);
  c.NSN64 = NRINGS * NRINGS;
  c.NSEG0 = SEG0;
  c.NSCRS = 64;
  c.NSRNG = 8;
  c.TOFBINN = 1;
  c.TOFBINS = 0.f;
  c.TOFBIND = 0.f;
  c.ITOFBIND = 0.f;
  c.COSUPSMX = cosupsmx;
  c.ETHRLD = ethrld;
  // image statistics as sct_module.cu:277-306 computes them
  auto stats = [](float *im, size_t n) {
    IMflt r;
    r.im = im;
    r.nvx = n;
    float mx = -1e12f, mn = 1e12f;
    for (size_t i = 0; i < n; i++) {
      if (im[i] > mx) mx = im[i];
      if (im[i] < mn) mn = im[i];
    }
    r.max = mx;
    r.min = mn;
    r.n10mx = 0;
    for (size_t i = 0; i < n; i++)
      if (im[i] > 0.1 * mx) r.n10mx += 1;
    return r;
  };
  IMflt muI = stats(mu, (size_t)SS_IMX * SS_IMY * SS_IMZ);
  IMflt emI = stats(em, (size_t)SSE_IMX * SSE_IMY * SSE_IMZ);
  scatOUT o;
  o.sval = sval;
  o.s3d = s3d;
  prob_scatt(o, knlut, reinterpret_cast<char *>(mumsk), muI, emI, sctaxR, sctaxW, offseg, scrs,
             isrng, srng, reinterpret_cast<char *>(xsxu), sn1_rno, sn1_sn11, c);
  cudaError_t e = cudaDeviceSynchronize();
  if (e == cudaSuccess) e = cudaGetLastError();
  return (int)e;
}

}  // extern "C"
