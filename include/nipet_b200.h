/* nipet_b200.h -- C ABI of the B200 reconstruction hot path for the Siemens mMR.
 *
 * Plain pointers and sizes only.  "dev" pointers are CUDA device (or managed)
 * memory on the handle's device; "host" pointers are ordinary host memory.
 * Every entry point returns an nb_status (0 = success) and never exits the
 * process; nb_last_error() gives a message for the calling thread's last failure.
 * Work is enqueued on the given CUDA stream (NULL = legacy default stream);
 * nothing synchronises unless the entry point says so.
 *
 * Each declaration names the reference interface it replaces
 * (paths inside the NiftyPET/NIPET tree).
 */
#ifndef NIPET_B200_H
#define NIPET_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  NB_OK = 0,
  NB_ERR_ARG = 1,         /* invalid argument (null pointer, size, span, index range) */
  NB_ERR_CUDA = 2,        /* a CUDA runtime call failed */
  NB_ERR_NOMEM = 3,       /* device allocation failed */
  NB_ERR_DEVICE = 4,      /* a kernel reported a device-side error (see nb_last_error) */
  NB_ERR_UNSUPPORTED = 5, /* valid in the reference but not provided here */
  NB_ERR_DATA = 6         /* malformed input data (e.g. list-mode stream without time tags) */
} nb_status;

/* Opaque geometry handle: device-resident LUTs, Siddon step lists and scratch. */
typedef struct nb_geom nb_geom;

int nb_version(void);
const char *nb_strerror(int status);
const char *nb_last_error(void);

/* ---- geometry -------------------------------------------------------------------------
 * Replaces the per-call LUT upload and transaxial table computation of
 * prj/src/prj_module.cu:380-398 (fprj), :560-585 (bprj), prj/src/recon.cu:334-349 (osem)
 * and prj/src/tprj.cu:174-200 (gpu_siddon_tx): tables are computed once per handle.
 *   crs    host [ncrs][4] float   (txLUT['crs'])
 *   s2c    host [naw][2] int16    (txLUT['s2c'])
 *   li2rng host [nli2r][2] float  (axLUT['li2rng'])
 *   li2sn  host [nli2r][2] int16  (axLUT['li2sn'], span-11)
 *   li2sn1 host [nli2r][2] int16  (axLUT['li2sn1'], span-1)
 *   li2nos host [nli2r] int8      (axLUT['li2nos'])
 * Only the full mMR geometry is accepted (ncrs 504, naw 68516, nli2r 2074). */
int nb_geom_create(int device, const float *crs, int ncrs, const int16_t *s2c, int naw,
                   const float *li2rng, const int16_t *li2sn, const int16_t *li2sn1,
                   const int8_t *li2nos, int nli2r, nb_geom **out);
int nb_geom_destroy(nb_geom *g);

/* Transaxial Siddon tables in the reference layout: tt host [naw][10] float, tv host
 * [naw][1807] uint8.  Replaces petprj.tprj (prj/src/prj_module.cu:70-224).  Synchronous. */
int nb_geom_tables(nb_geom *g, float *tt, uint8_t *tv);

/* Voxel-read count V of a forward projection (direct: 1 per step, oblique: 2 per step,
 * 4 at an axial crossing), computed on the device: the total over all LORs in *reads and,
 * if per_lor (host [naw] int64) is not NULL, the count of every LOR.  Synchronous. */
int nb_geom_count_reads(nb_geom *g, long long *per_lor, long long *reads);

/* ---- projectors on the reference image layout [320][320][127] (y, x, z) ---------------
 * nb_fprj replaces petprj.fprj (prj/src/prj_module.cu:232-425 -> gpu_fprj, prjf.cu:209-320).
 *   sino dev [nprj][nsinos] float, overwritten; nsinos 837 (span 11) or 4084 (span 1)
 *   im   dev [320*320*127] float
 *   subs dev [nprj] int32 LOR indices into [0, 68516), or NULL for all 68516 LORs in order
 *   att  0 emission (line integrals), 1 attenuation factors exp(-integral)
 * nb_bprj replaces petprj.bprj (prj_module.cu:430-608 -> gpu_bprj, prjb.cu:190-308).
 *   im   dev [320*320*127] float, overwritten with the back projection of sino. */
int nb_fprj(nb_geom *g, float *sino, const float *im, const int32_t *subs, int nprj, int span,
            int att, void *stream);
int nb_bprj(nb_geom *g, float *im, const float *sino, const int32_t *subs, int nprj, int span,
            void *stream);

/* ---- span-1 projectors over a reduced axial ring range ---------------------------------
 * The reference's reduced-rings mode (Cnt.RNG_STRT = rs, Cnt.RNG_END = re, set by
 * mmraux.reduce_rings, mmraux.py:566-617): petprj.fprj / petprj.bprj in span 1 with the
 * range's axial LUTs run gpu_fprj / gpu_bprj over the ring pairs inside [rs, re) only, on
 * an image of the axial slab [2 rs, 2 re - 1) (prj/src/prjf.cu:19-29 imExpand, :209-320;
 * prjb.cu:19-29 imReduce, :190-308).
 * nb_rings_create builds the range's ray set once from the range's LUTs:
 *   li2rng host [nli2r][2] float  (reduced axLUT['li2rng'])
 *   li2sn1 host [nli2r][2] int16  (reduced axLUT['li2sn1'])
 *   nli2r  (re-rs)(re-rs+1)/2, less 6 for all 64 rings
 * Every pair must be a ray of the geometry with both rings in the range, and the rays
 * must fill the range's nsino = (re-rs)^2 sinograms (4084 for 64 rings) once each.
 * nb_rings_info: nsino, the slab's first voxel vz0 = 2 rs and its size nvz = 2 (re-rs) - 1.
 * nb_fprj_rings: sino dev [nprj][nsino] float, overwritten; im dev [320*320*nvz] float.
 * nb_bprj_rings: im dev [320*320*nvz] float, overwritten; sino dev [nprj][nsino] float.
 * subs, nprj, att as for nb_fprj. */
typedef struct nb_rings nb_rings;
int nb_rings_create(nb_geom *g, int rs, int re, const float *li2rng, const int16_t *li2sn1,
                    int nli2r, nb_rings **out);
int nb_rings_destroy(nb_rings *rr);
int nb_rings_info(const nb_rings *rr, int *nsino, int *vz0, int *nvz);
int nb_fprj_rings(nb_geom *g, const nb_rings *rr, float *sino, const float *im,
                  const int32_t *subs, int nprj, int att, void *stream);
int nb_bprj_rings(nb_geom *g, const nb_rings *rr, float *im, const float *sino,
                  const int32_t *subs, int nprj, void *stream);

/* ---- the same projectors on the internal "col128" layout -------------------------------
 * col128: nimg images of [320*320][128] float, column-major in z with even z in slots
 * [0,64), odd z in [64,127) and slot 127 zero.  nb_bprj_col128 ADDS into im128.
 * These are the forms the OSEM and batched paths use (no layout conversion). */
int nb_fprj_col128(nb_geom *g, float *sino, const float *im128, const int32_t *subs, int nprj,
                   int span, int att, void *stream);
int nb_bprj_col128(nb_geom *g, float *im128, const float *sino, const int32_t *subs, int nprj,
                   int span, void *stream);
/* Sensitivity image of a subset: sens128 = back projection of the rows subs[] of the
 * full gap-free sinogram an (dev [68516][nsinos], e.g. attenuation x normalisation),
 * i.e. what the reference computes with petprj.bprj(ansng[subs], subs)
 * (prj/mmrrec.py:289-299).  sens128 is overwritten. */
int nb_sens_col128(nb_geom *g, float *sens128, const float *an, const int32_t *subs, int nprj,
                   int span, void *stream);
int nb_im_to_col128(float *im128, const float *im, int nimg, void *stream);
int nb_col128_to_im(float *im, const float *im128, int nimg, void *stream);

/* Synchronise `stream` and report (then clear) any device-side error a kernel of this
 * handle raised.  Synchronous. */
int nb_geom_check(nb_geom *g, void *stream);

/* ---- sinogram layout (src/scanner_0.cu:94-241, mmr_auxe.rgaps / pgaps) -----------------
 * nb_remgaps: Siemens [snno][252*344] -> gap-free [68516][snno] (d_remgaps);
 * nb_putgaps: gap-free [68516][snno] -> Siemens [snno][252*344], gaps set to 0 (d_putgaps).
 *   aw2ali dev [68516] int32 (txLUT['aw2ali']).  The _u16 forms move uint16 counts. */
int nb_remgaps(float *sng, const float *sino, int snno, const int32_t *aw2ali, void *stream);
int nb_remgaps_u16(uint16_t *sng, const uint16_t *sino, int snno, const int32_t *aw2ali,
                   void *stream);
int nb_putgaps(float *sino, const float *sng, int snno, const int32_t *aw2ali, void *stream);

/* ---- OSEM (prj/src/recon.cu:318-521, petprj.osem prj_module.cu:613-839) --------------
 * nb_osem_rs: rs = (rsng + ssng) / (asng * nsng), 0 where |asng*nsng| < 1e-6
 *   (recon.cu:381-398), all dev [n] float; ssng may be NULL (zero scatter).
 * nb_osem_subset: one fused OSEM sub-iteration on col128 images, replacing the
 *   per-subset rec_fprj / sneladd / sneldiv / rec_bprj / eldiv0 / elmsk sequence
 *   (recon.cu:459-497):
 *     img128 dev col128 image, updated in place: img = msk ? img * (bimg/sens) : 0
 *     bimg128 dev col128 scratch image (zeroed by the call)
 *     sens128 dev col128 sensitivity image of this subset
 *     msk128 dev col128 uint8 mask (0 outside the reconstruction cylinder)
 *     psng dev [68516][837] uint16 prompts; rs dev [68516][837] float from nb_osem_rs
 *     subs dev [nprj] int32 LORs of the subset. */
int nb_osem_rs(float *rs, const float *rsng, const float *ssng, const float *asng,
               const float *nsng, size_t n, void *stream);
int nb_osem_subset(nb_geom *g, float *img128, float *bimg128, const float *sens128,
                   const uint8_t *msk128, const uint16_t *psng, const float *rs,
                   const int32_t *subs, int nprj, void *stream);

/* nb_osem_subset_span1: one span-1 OSEM sub-iteration of one image, the reference's
 * osem() with Cnt.SPN == 1 (recon.cu:318-497): psng [68516][4084] uint16 prompts, rs
 * [68516][4084] float from nb_osem_rs, the other arguments as nb_osem_subset; krnl
 * (host [3][17], NULL for none) applies the resolution kernel as nb_osem_subset_psf, with
 * work128 two col128 images of scratch. */
int nb_osem_subset_span1(nb_geom *g, float *img128, float *bimg128, const float *sens128,
                         const uint8_t *msk128, const uint16_t *psng, const float *rs,
                         const int32_t *subs, int nprj, const float *krnl, float *work128,
                         void *stream);

/* Resolution modelling (recon.cu:49-216, the PSF of petprj.osem when krnl[0][0] >= 0).
 * nb_psf_col128: the reference's separable convolution of one col128 image -- along z
 *   with krnl row 0, then x with row 1, then y with row 2 (the row order psf_config,
 *   prj/mmrrec.py:96-155, produces), 17 taps, zeros outside the volume; bit-identical to
 *   the reference's d_conv.  krnl host [3][17]; dst may equal src; tmp128 dev col128
 *   scratch distinct from both.
 * nb_osem_subset_psf: nb_osem_subset with the PSF inside the sub-iteration
 *   (recon.cu:459-497): forward projection of the convolved image, convolution of the
 *   back projection before the division by sens128 (which the caller has convolved once,
 *   recon.cu:437-445).  work128 dev 2 x col128 scratch. */
int nb_psf_col128(float *dst128, const float *src128, const float *krnl, float *tmp128,
                  void *stream);
int nb_osem_subset_psf(nb_geom *g, float *img128, float *bimg128, const float *sens128,
                       const uint8_t *msk128, const uint16_t *psng, const float *rs,
                       const int32_t *subs, int nprj, const float *krnl, float *work128,
                       void *stream);

/* ---- batched OSEM: many images (bootstrap replicates, dynamic frames) per launch --------
 * The reference reconstructs one image per osem() call (recon.cu:318-521); these entry
 * points run one sub-iteration for nrep images that share geometry, attenuation,
 * normalisation and sensitivity, each with its own prompts:
 *   img, bimg  dev [ceil(nrep/bs)][320*320][128][bs] float ("col128 x bs" layout: the bs
 *              images of a group interleaved per voxel); img updated in place, bimg scratch
 *              (left zeroed)
 *   sens128    dev col128 sensitivity image of this subset; msk128 dev col128 uint8 mask
 *   psng       dev [nrep][68516][nsinos] uint16 prompts; rs dev [68516][nsinos] float
 *              (r+s)/(an) from nb_osem_rs; rscale dev [nrep] per-image randoms factor
 *   bs         1, 2 or 4; span 11 (837 sinograms) or 1 (4084)
 *   tile       kernel shape: 0 = 1024 threads x 4 rays each, 64/bs columns of the LOR
 *              staged per shared-memory chunk; 1 = the same threads, 32/bs columns per
 *              chunk; 2 = 512 threads x 8 rays, 64/bs columns.  Results agree to rounding;
 *              batch.autotune picks (bs, tile) by timing them.
 * nb_to_batch / nb_from_batch convert nrep reference-layout images [nrep][320][320][127]
 * to and from that layout; nb_fill_batch sets every voxel of the nrep images in that layout
 * to `value` (the OSEM start image) without a reference-layout source, zeroing the padding
 * slot of each column and the images that pad the last group. */
int nb_to_batch(float *dst, const float *src, int nrep, int bs, void *stream);
int nb_from_batch(float *dst, const float *src, int nrep, int bs, void *stream);
int nb_fill_batch(float *dst, float value, int nrep, int bs, void *stream);

/* Forward and back projection of nrep images in the batched layout, one walk of the
 * geometry per bs images -- what gpu_fprj / gpu_bprj (prjf.cu:209-320, prjb.cu:190-308) do
 * for one image per call.  Used by the differentiable projector for image batches.
 *   nb_fprj_batch: sino dev [nrep][nprj][nsinos] float, overwritten (att = 0: emission)
 *   nb_bprj_batch: bimg dev batched layout, the back projection of sino is ADDED (zero it
 *                  first); sino dev [nrep][nprj][nsinos]
 *   subs dev [nprj] LOR indices, or NULL with nprj = 68516. */
int nb_fprj_batch(nb_geom *g, float *sino, const float *img, int nrep, int bs, int span,
                  const int32_t *subs, int nprj, void *stream);
int nb_bprj_batch(nb_geom *g, float *bimg, const float *sino, int nrep, int bs, int span,
                  const int32_t *subs, int nprj, void *stream);
int nb_osem_batch_subset(nb_geom *g, float *img, float *bimg, const float *sens128,
                         const uint8_t *msk128, const uint16_t *psng, const float *rs,
                         const float *rscale, int nrep, int bs, int tile, int span,
                         const int32_t *subs, int nprj, void *stream);

/* ---- normalisation sinogram (src/norm.cu:13-210 norm_from_components, driven by
 * mmrnorm.get_norm_sino, mmrnorm.py:155-195) --------------------------------------------
 * nb_norm replaces norm_from_components: the norm sinogram from the Siemens components
 * (read from the norm file by the caller) and the average bucket singles.
 *   sng  dev [68516][nsinos] float (gap-free), overwritten
 *   geo [>=344] (first segment row of the geometric effects), cinf [344][9] crystal
 *   interference, ceff [64][504] crystal efficiencies, axe1 [837] axial effects, axf1
 *   [4084] span-1 axial factors (span 1 only, else may be NULL), dtp/dtnp [64]
 *   dead-time parameters, buckets [224] int32 average singles (mmrhist's `buckets`),
 *   sn1_rno [4084][2], sn1_sn11 [4084], sn1_sn11no [4084], aw2ali [68516]; all host.
 *   span 1 or 11. */
int nb_norm(float *sng, const float *geo, int ngeo, const float *cinf, const float *ceff,
            const float *axe1, const float *axf1, const float *dtp, const float *dtnp,
            const int32_t *buckets, const int16_t *sn1_rno, const int16_t *sn1_sn11,
            const int8_t *sn1_sn11no, const int32_t *aw2ali, int span, void *stream);

/* ---- randoms from the delayed fan sums (lm/src/rnd.cu:169-386 gpu_randoms, driven by
 * mmrhist.randoms / rand, lm/mmrhist.py:188-221) ---------------------------------------
 * nb_randoms replaces gpu_randoms: crystal singles fitted to the delayed fan sums (ten
 * damped fixed-point steps) and the randoms sinogram they imply.
 *   rsn      dev [nsinos][252][344] float (Siemens layout with gaps, gaps 0), overwritten
 *   cmap     dev [504][64] float singles per crystal (with gaps) and ring, overwritten
 *   fansums  [64][504] uint32 (mmr_lmproc.hist's `fan`), host or device memory
 *   crsr [504], cij [448][448], s2cr [68516][2], aw2sn [68516][2], sn1_rno [4084][2],
 *   sn1_sn11 [4084] (txLUT crsri/cij/s2cr/aw2sn, axLUT sn1_rno/sn1_sn11), host int16/int8
 *   span 1 or 11; mrd the maximum ring difference (60).
 * Waits on `stream` for the fan sums, then runs asynchronously. */
int nb_randoms(float *rsn, float *cmap, const uint32_t *fansums, const int16_t *crsr,
               const int8_t *cij, const int16_t *s2cr, const int16_t *aw2sn,
               const int16_t *sn1_rno, const int16_t *sn1_sn11, int span, int mrd,
               void *stream);

/* ---- list-mode histogramming (lm/src/lmproc.cu:12-230, hst.cu:37-528, lmaux.cu:17-270) -
 * nb_lm_plan replaces getLMinfo + modifyLMinfo: the chunk plan of a list-mode stream
 * (host [ele] int32 words), chunks cut at time tags with t % 100 ms == 0, and the time
 * window [t0, t1) in seconds (t0 == t1: whole stream).  Arrays have capacity `cap`.
 * Returns the number of chunks in *nchnk. */
int nb_lm_plan(const int32_t *lm, int64_t ele, int t0, int t1, int cap, int64_t *atag,
               int *ele4chnk, int *ele4thrd, int *nchnk, int *toff, int *nitag, int *tstart,
               int *tstop);

/* nb_hist replaces gpu_hst (hst.cu:347-528) + the lmproc unpack (lmproc.cu:156-193):
 * histograms the dev stream `lm` (the whole file, word 0 = file word 0) with the plan
 * from nb_lm_plan (host arrays), for `nrep` bootstrap replicates rep0..rep0+nrep-1.
 *   span 1, 11 or 0 (SSRB); btp 0 none, 1 non-parametric, 2 parametric (Poisson(btprt))
 *   seed: bootstrap stream key (Philox4x32-10; counter = (word index, replicate, draw))
 * Outputs (dev, ZEROED BY THE CALLER, accumulated):
 *   psino [nrep][nbins] uint32 packed prompts (low 16 bits) / delayeds (high 16 bits)
 *   ssrb [nrep][127*86688] uint32, phc/dhc [nrep][nitag] uint32, zR/zM [nrep][nitag] int32,
 *   pvs [nrep][sne] uint32, fan [nrep][64*504] uint32, bck [nrep][2*224*nitag] uint32
 *   (nbins: 354033792 span 1, 72557856 span 11, 11009376 span 0;
 *    sne = ceil(min(nitag,5400)/4)*127*344 as lmproc.cu:60-63)
 *   sn1_sn11, sn1_ssrb, sn1_rno, s2cF: host LUTs (axLUT/txLUT, int16).
 * Device scratch comes stream-ordered from the histogrammer's own memory pool, which keeps
 * it for the next call (nb_hist_trim releases it).  With nrep > 1 the replicates go through
 * in equal launches of at most 16, each counting into an unpacked scratch of
 * nbins * 8 * r bytes (r: the launch's replicates rounded up to a multiple of 4; 7.0 GB for
 * 10 replicates at span 11); one span-1 histogram without bootstrap takes 4 bytes per
 * stream word of slab records. */
int nb_hist(const int32_t *lm, int64_t ele, int nchnk, const int64_t *atag, const int *ele4chnk,
            const int *ele4thrd, int toff, int nitag, int tstart, int tstop, int span, int btp,
            double btprt, uint64_t seed, int rep0, int nrep, const int16_t *sn1_sn11,
            const int16_t *sn1_ssrb, const int16_t *sn1_rno, const int16_t *s2cF,
            uint32_t *psino, uint32_t *ssrb, uint32_t *phc, uint32_t *dhc, int32_t *zR,
            int32_t *zM, uint32_t *pvs, uint32_t *fan, uint32_t *bck, void *stream);

/* nb_hist_static has no counterpart in the reference.  It is nb_hist for callers that
 * cannot allocate device memory: for example an acquisition loop that histograms each
 * incoming list-mode buffer while the scan runs, where a device allocation could fail or
 * stall the stream mid-acquisition, or a host process whose device memory is entirely
 * owned by another allocator.  Same arguments, semantics and outputs as nb_hist; it makes
 * no allocation: the look-up tables and chunk plan are staged in a file-scope static
 * device array of 512 KiB that every GPU loading this library keeps until exit.
 * Limits: at most 4096 chunks in the plan (about 5e10 words); larger plans are rejected
 * with NB_ERR_ARG.  The first call on a device looks up that array's device address
 * (cudaGetSymbolAddress, with the device current) and caches it, so make that first call
 * before any stream capture; the cached address belongs to that device's context, so it is
 * stale after a cudaDeviceReset (do not call this after one).  The host arrays (LUTs and
 * plan) are gathered into one host buffer and staged before the call returns, so the caller
 * may reuse or free them at once, pinned or not.  All calls on a device share the array
 * and it keeps the last call's tables; calls that overlap on the GPU race on it and must be
 * serialised. */
int nb_hist_static(const int32_t *lm, int64_t ele, int nchnk, const int64_t *atag,
                   const int *ele4chnk, const int *ele4thrd, int toff, int nitag, int tstart,
                   int tstop, int span, int btp, double btprt, uint64_t seed, int rep0, int nrep,
                   const int16_t *sn1_sn11, const int16_t *sn1_ssrb, const int16_t *sn1_rno,
                   const int16_t *s2cF, uint32_t *psino, uint32_t *ssrb, uint32_t *phc,
                   uint32_t *dhc, int32_t *zR, int32_t *zM, uint32_t *pvs, uint32_t *fan,
                   uint32_t *bck, void *stream);

/* Split packed sinograms: psn = w & 0xFFFF, dsn = w >> 16 (lmproc.cu:162-168), and the
 * prompt/delayed totals (host, may be NULL).  Synchronous. */
int nb_hist_unpack(const uint32_t *psino, size_t nbins, uint16_t *psn, uint16_t *dsn,
                   unsigned long long *psum, unsigned long long *dsum, void *stream);

/* nb_hist_trim has no counterpart in the reference.  nb_hist takes its stream-ordered
 * scratch (tables, and for bootstrap replicates the unpacked counters: 8 x nbins x rblk
 * bytes, rblk = nrep rounded up to 4 -- about 7 GB for 10 span-11 replicates) from a
 * memory pool of its own per device that keeps freed memory for the next call.  This
 * returns the current device's unused pool memory to the system (cudaMemPoolTrimTo 0);
 * memory of calls still in flight on a stream stays until they finish. */
int nb_hist_trim(void);

/* ---- scatter (sct/src/sct.cu prob_scatt, ray.cu raysLUT, sctaux.cu srslt2sino) ----------
 * nb_sct_vsm replaces nifty_scatter.vsm (sct/src/sct_module.cu:60-335 -> prob_scatt,
 * sct.cu:338-582): the voxel-driven single-scatter model for the mMR's 64 scatter crystals
 * x 8 scatter rings, non-TOF.
 *   mu     host [63][172][172] float: the down-sampled mu-map (1/cm)
 *   mumsk  host [63][172][172] int8: attenuating voxels (> 0) for which paths are summed
 *   em     host [43][114][114] float: the down-sampled emission image
 *   scrs   host [64][3] float (crystal, x, y cm), srng host [8][2] float (ring, z cm),
 *   isrng  host [8] int16 scatter rings; knlut host [256][2] float Klein-Nishina LUT;
 *   cosupsmx cos of the largest scatter angle; ethrld emitting-voxel threshold / maximum;
 *   xsxu   host [64][64] int8; offseg host [nseg0+1] int16; sctaxR host [4096][4] int32,
 *   sctaxW host [4096][4] float (axial interpolation); sn1_sn11 host [4084] int16
 *   sval   dev [8][64][8][64] float, overwritten: the raw results (sct_val)
 *   s3d    dev [nsn][64][64] float, overwritten: the pre-sinograms, nsn 4096 at span 1
 *          (sinograms past 4083 zero) or 837 at span 11 (sct_3d)
 *   nvx    host [2] int, may be NULL: attenuating and emitting voxels used.
 * Synchronous (the mu-map texture lives for the call). */
int nb_sct_vsm(const float *mu, const int8_t *mumsk, const float *em, const float *scrs,
               int nscrs, const float *srng, const int16_t *isrng, int nsrng,
               const float *knlut, float cosupsmx, float ethrld, const int8_t *xsxu,
               const int16_t *offseg, int nseg0, const int32_t *sctaxR, const float *sctaxW,
               int nsn64, const int16_t *sn1_sn11, int nsn1, int span, float *sval, float *s3d,
               int *nvx, void *stream);

/* ---- host -> device transfer ----------------------------------------------------------
 * nb_copy_h2d replaces the per-call pageable cudaMemcpy of the host arrays petprj.osem,
 * fprj and bprj receive (prj/src/prj_module.cu:613-839 -> recon.cu:334-419, and the
 * sinogram/image uploads of prj_module.cu:232-608): `bytes` from pageable host memory `src`
 * to device memory `dst`, through a ring of pinned staging buffers (allocated on the first
 * call on a device, kept until exit) filled by several host threads while the DMA of the
 * previous chunk runs.  Returns once `src` has been read entirely (the caller may reuse it);
 * the copies are ordered on `stream`.  Calls on one device are serialised. */
int nb_copy_h2d(void *dst, const void *src, size_t bytes, void *stream);
/* nb_copy_d2h: the reverse, for the results petprj.osem and bprj copy back into the caller's
 * host arrays (prj_module.cu:595-600, :826-832): `bytes` from device memory `src`, after the
 * work queued on `stream`, into pageable host memory `dst`, the DMA of one chunk overlapping
 * the host threads' unpacking of the previous.  Returns when `dst` holds the data. */
int nb_copy_d2h(void *dst, const void *src, size_t bytes, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* NIPET_B200_H */
