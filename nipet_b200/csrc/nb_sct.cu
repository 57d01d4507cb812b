// nb_sct.cu -- voxel-driven single-scatter model (VSM) of the Siemens mMR.
//
// Reference: niftypet/nipet/sct/src/ray.cu:22-105 (satt: attenuation path sums from every
// attenuating voxel to every scatter crystal), sct.cu:43-335 (Psct: the scatter
// probabilities) and :338-582 (prob_scatt), sctaux.cu:18-74 (d_sct2sn1, d_sct_axinterp) and
// :78-197 (srslt2sino), :200-340 (the voxel masks).
//
// The model: an emitting voxel of the down-sampled emission image sends an unscattered
// photon to a crystal of a 64-crystal x 8-ring subset of the scanner; the partner photon
// is followed along the opposite direction, and at every patch of 4 path samples it
// scatters, with Klein-Nishina probability, towards each of the 32 scatter crystals facing
// it, attenuated on the way by the path sums of the mu-map.  The results, one value per
// (unscattered ring, unscattered crystal, scatter ring, scatter crystal), become span-1
// pre-sinograms of 64 x 64 bins and are interpolated axially to every span-1 (and summed
// into every span-11) sinogram.
//
// B200 design.  The mu-map is sampled through a 3D texture with hardware trilinear
// filtering, as the reference does, so a sample at a given position is the same value;
// positions are computed with the reference's expressions because float rounding decides
// where a ray samples.  The reference launches one block per (emitting voxel, unscattered
// ring, unscattered crystal) and adds every (scatter patch, scatter crystal) term to the
// result with a global float atomic; here a block owns one (unscattered ring, unscattered
// crystal) pair and walks a strided share of the emitting voxels, each warp (one scatter
// ring) keeping the terms of a voxel in registers, summing a crystal's 8 patches with
// shuffles and the voxels in shared memory, so a block issues 512 global atomics in all.
// The pre-sinogram steps are gathers: the span-1 pre-sinogram is written by plain stores
// (every result has its own bin) and a span-11 bin sums its span-1 sinograms in ascending
// order, deterministic, where the reference adds them with float atomics.
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include <vector>

#include "nb_internal.cuh"

namespace nbs {

// grids of the down-sampled mu-map (SS) and emission image (SSE) and the geometry the
// model is defined with (sct/src/sct.h:17-67); the images are made on these grids by the
// caller
constexpr int SS_IMX = 172, SS_IMY = 172, SS_IMZ = 63;
constexpr int SSE_IMX = 114, SSE_IMY = 114, SSE_IMZ = 43;
constexpr int NCOS = 256;
constexpr int NSCRS = 64, NSRNG = 8;
constexpr int SS_WRP = 32, LSCT2 = 2;
constexpr float SS_VXY = 0.417252f, SS_VXZ = 0.409474f, IS_VXZ = 2.442157f;
constexpr float SSE_VXY = 0.629538f, SSE_VXZ = 0.599927f;
constexpr float R_2 = 1120.2409f, IR_RING = 0.029878f, SRFCRS = 0.1695112f;
constexpr float ASTP = SS_VXZ, SSTP = SS_VXZ;
constexpr float RES_SUM = 0.000091552734375f;
constexpr float PI_F = 3.1415926535f;

struct PsctArgs {
  cudaTextureObject_t tex;
  const int16_t *rays;   // [nvx_mu][NSCRS][NSRNG] path sums / RES_SUM
  const int *mu_v2i;     // [SS grid] index into rays, -1 outside the mu mask
  const int *em_i2v;     // [nvx_em] SSE grid voxel of each emitting voxel
  const float *em;       // [SSE grid]
  const float *scrs;     // [NSCRS][3]: crystal number, x, y (cm)
  const float *srng;     // [NSRNG][2]: ring number, z (cm)
  const float2 *kn;      // [NCOS] Klein-Nishina value and attenuation factor per angle
  float cos0, cosstp_inv;  // cos of the largest scatter angle, (NCOS - 1) / (1 - cos0)
  int nvx_em;
  float *rslt;           // [NSRNG][NSCRS][NSRNG][NSCRS] (unscattered ring, crystal, ...)
};

__device__ __forceinline__ signed char sgn(float x) { return x > 0 ? 1 : (x < 0 ? -1 : 0); }

// ---------------------------------------------------------------------------------------
// attenuation path sums (ray.cu:22-105): one warp per (attenuating voxel, scatter crystal,
// scatter ring); the 32 lanes sample 32 consecutive steps of the path, summed by a
// shuffle tree per step group, as the reference sums them
// ---------------------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_sct_rays(int16_t *out, cudaTextureObject_t tex,
                                                  const int *i2v, const float *scrs,
                                                  const float *srng) {
  const int vxi = blockIdx.x, icrs = blockIdx.y;
  const int irng = threadIdx.y, idx = threadIdx.x;
  const int im_idx = i2v[vxi];
  const int w = im_idx / (SS_IMX * SS_IMY);
  const int v = (im_idx - w * SS_IMY * SS_IMX) / SS_IMX;
  const int u = im_idx - (w * SS_IMY * SS_IMX + v * SS_IMX);
  // voxel centre (cm): the reference's mixed float/double expressions
  const float x = (u + 0.5 * (1 - SS_IMY)) * SS_VXY;
  const float y = ((SS_IMY - 1) * 0.5 - v) * SS_VXY;
  const float z = w * SS_VXZ - .5 * SS_VXZ * (SS_IMZ - 1);
  float ax = scrs[3 * icrs + 1] - x;
  float ay = scrs[3 * icrs + 2] - y;
  float az = srng[2 * irng + 1] - z;
  const float a_lgth = powf(ax * ax + ay * ay + az * az, 0.5f);
  ax /= a_lgth;
  ay /= a_lgth;
  az /= a_lgth;
  float ray_sum = 0;
  for (int k = 0; k <= (int)(a_lgth / (SS_WRP * ASTP)); k++) {
    const float t = (idx + k * SS_WRP) * ASTP;
    const float sx = .5 * SS_IMX + (x + ax * t) / SS_VXY;
    const float sy = .5 * SS_IMY - (y + ay * t) / SS_VXY;
    const float sz = .5 * SS_IMZ + (z + az * t) / SS_VXZ;
    float uval = tex3D<float>(tex, sx, sy, sz);
    for (int off = 16; off > 0; off /= 2) uval += __shfl_down_sync(0xffffffffu, uval, off);
    if (idx == 0) ray_sum += uval;
  }
  if (idx == 0)
    out[(size_t)vxi * NSCRS * NSRNG + icrs * NSRNG + irng] = (short)(ray_sum * ASTP / RES_SUM);
}

__device__ __forceinline__ float warpsum_xor(float val) {
  for (int mask = SS_WRP / 2; mask > 0; mask /= 2)
    val += __shfl_xor_sync(0xffffffffu, val, mask);
  return val;
}

__device__ __forceinline__ float wcumsum(int idx, float val) {
  for (int off = 1; off < SS_WRP; off *= 2)
    val += __shfl_sync(0xffffffffu, val, idx - off) * ((idx - off) >= 0);
  return val;
}

// ---------------------------------------------------------------------------------------
// scatter probabilities (sct.cu:43-335, non-TOF): block (32 lanes, 8 scatter rings) per
// (unscattered crystal iuc = blockIdx.x, unscattered ring iur = blockIdx.y), emitting
// voxels blockIdx.z, blockIdx.z + gridDim.z, ...
// ---------------------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_sct_psct(const PsctArgs a) {
  __shared__ float2 s_kn[NCOS];
  __shared__ float s_acc[NSRNG][NSCRS];
  const int idx = threadIdx.x, isr = threadIdx.y;
  const int iuc = blockIdx.x, iur = blockIdx.y;
  const int tid = isr * 32 + idx;
  for (int i = tid; i < NCOS; i += 256) s_kn[i] = a.kn[i];
  for (int i = tid; i < NSRNG * NSCRS; i += 256) (&s_acc[0][0])[i] = 0.f;
  __syncthreads();

  // the unscattered photon's crystal, and the opposing crystal pair used for the offset
  const float ucx = a.scrs[3 * iuc + 1], ucy = a.scrs[3 * iuc + 2];
  const int isuc = (iuc + NSCRS / 2) & (NSCRS - 1);
  const float oscx = a.scrs[3 * isuc + 1], oscy = a.scrs[3 * isuc + 2];
  const float nscx = a.scrs[3 * ((isuc + 1) & (NSCRS - 1)) + 1];
  const float nscy = a.scrs[3 * ((isuc + 1) & (NSCRS - 1)) + 2];
  const float ucz = a.srng[2 * iur + 1];
  const float scz = a.srng[2 * isr + 1];

  for (int evxi = blockIdx.z; evxi < a.nvx_em; evxi += gridDim.z) {
    const int im_idx = a.em_i2v[evxi];
    const float em_vox = a.em[im_idx];
    int w = im_idx / (SSE_IMX * SSE_IMY);
    int v = (im_idx - w * SSE_IMY * SSE_IMX) / SSE_IMX;
    int u = im_idx - (w * SSE_IMY * SSE_IMX + v * SSE_IMX);
    const float x = (u + 0.5 * (1 - SSE_IMX)) * SSE_VXY;
    const float y = ((SSE_IMY - 1) * 0.5 - v) * SSE_VXY;
    const float z = w * SSE_VXZ - .5 * SSE_VXZ * (SSE_IMZ - 1);
    // the mu-map voxel of the emitting point; outside the mu mask it emits nothing here
    u = .5 * SS_IMX + floorf(x / SS_VXY);
    v = (.5 * SS_IMY - ceilf(y / SS_VXY));
    w = floorf(.5 * SS_IMZ + z * IS_VXZ);
    const int mvxi = a.mu_v2i[(int)(u + SS_IMX * v + SS_IMX * SS_IMY * w)];
    if (mvxi < 0) continue;  // uniform over the block

    float3 av;
    av.x = ucx - x;
    av.y = ucy - y;
    av.z = ucz - z;
    const float an = powf(av.x * av.x + av.y * av.y + av.z * av.z, 0.5f);
    float2 aux;
    aux.x = av.x;
    aux.y = av.y;
    float a_lgth = powf(aux.x * aux.x + aux.y * aux.y, 0.5f);
    av.x /= an;
    av.y /= an;
    av.z /= an;
    aux.x /= a_lgth;
    aux.y /= a_lgth;
    // solid angle and survival of the unscattered photon
    const float uomg =
        (SRFCRS * (av.x * ucx * IR_RING + av.y * ucy * IR_RING) / (2 * PI_F * an * an)) *
        expf(-a.rays[(size_t)mvxi * NSCRS * NSRNG + iuc * NSRNG + iur] * RES_SUM);
    // the scattering photon goes the other way
    av.x *= -1;
    av.y *= -1;
    av.z *= -1;
    aux.x *= -1;
    aux.y *= -1;
    const float Br = 2 * (x * aux.x + y * aux.y);
    const float t0 = .5 * (-Br + sqrtf(Br * Br - 4 * (-R_2 + x * x + y * y)));
    float2 ms;
    ms.x = aux.x * t0 + x;
    ms.y = aux.y * t0 + y;
    // the crystal nearest to where the scattering photon meets the ring, as an offset
    // from the opposing crystal
    const signed char imsc =
        isuc + (signed char)(sgn((ms.x - oscx) * (nscx - oscx) + (ms.y - oscy) * (nscy - oscy)) *
                             NSCRS *
                             acosf((ms.x * oscx + ms.y * oscy) /
                                   (sqrtf(oscx * oscx + oscy * oscy) *
                                    sqrtf(ms.x * ms.x + ms.y * ms.y))) /
                             (2 * PI_F));
    a_lgth = t0 / (a_lgth / an);
    // this lane's scatter crystal (the 32 crystals facing the scattering photon)
    const signed char isc = (imsc - (NSCRS / 4) + idx) & (NSCRS - 1);

    // how many 32-sample groups of the path meet attenuating matter
    int Nw = 0;
    for (int k = 0; k <= (int)(a_lgth / (SS_WRP * SSTP)); k++) {
      const float t = (idx + 0.5 + k * SS_WRP) * SSTP;
      const int su = .5 * SS_IMX + floorf((x + av.x * t) / SS_VXY);
      const int sv = .5 * SS_IMX - ceilf((y + av.y * t) / SS_VXY);
      const int sw = floorf(.5 * SS_IMZ + (z + av.z * t) * IS_VXZ);
      float uval = tex3D<float>(a.tex, su, sv, sw);
      uval = warpsum_xor(uval);
      if (uval > 0) Nw = k;
    }

    float3 sc;
    sc.x = a.scrs[3 * isc + 1];
    sc.y = a.scrs[3 * isc + 2];
    sc.z = scz;
    float acc[SS_WRP >> LSCT2];
#pragma unroll
    for (int j = 0; j < (SS_WRP >> LSCT2); j++) acc[j] = 0.f;
    float rcsum = 0;
    for (int k = 0; k <= Nw; k++) {
      const float t = (idx + k * SS_WRP + 0.5) * SSTP;
      const float sval =
          tex3D<float>(a.tex, .5 * SS_IMX + (x + av.x * t) / SS_VXY,
                       .5 * SS_IMY - (y + av.y * t) / SS_VXY, .5 * SS_IMZ + (z + av.z * t) * IS_VXZ);
      float cumum = wcumsum(idx, sval);
      const float sumWarp = __shfl_sync(0xffffffffu, cumum, SS_WRP - 1);
      // mu summed over the 4-sample patch ending at this sample
      const float smu = cumum - __shfl_sync(0xffffffffu, cumum, idx - (1 << LSCT2)) *
                                    ((idx - (1 << LSCT2)) >= 0);
      float p_scatter = (1 - expf(-smu * SSTP));
      cumum -= sval;
      p_scatter *= uomg * expf(-(__shfl_sync(0xffffffffu, cumum, idx & ~((1 << LSCT2) - 1)) +
                                 rcsum) * SSTP);
      rcsum += sumWarp;
      const float tt = t - ((1 << (LSCT2 - 1)) - 0.5) * SSTP;
      // lane idx handles scatter point sct_id (its patch) and crystals aid + 4 j
      const int sct_id = (idx & (-((1 << LSCT2)))) + (1 << LSCT2) - 1;
      const int aid = idx & ((1 << LSCT2) - 1);
      const float ttp = __shfl_sync(0xffffffffu, tt, sct_id);
      const float psp = __shfl_sync(0xffffffffu, p_scatter, sct_id);
#pragma unroll
      for (int j = 0; j < (SS_WRP >> LSCT2); j++) {
        const int crs_shft = aid + j * (1 << LSCT2);
        float3 s;
        s.x = (x + av.x * ttp);
        s.y = (y + av.y * ttp);
        s.z = (z + av.z * ttp);
        int i_smsk;
        char infov = 1;
        if ((fabsf(s.z) < (SS_VXZ * SS_IMZ / 2 - 0.01 * SS_VXZ)) &&
            (fabsf(s.x) < (SS_VXY * SS_IMX / 2 - 0.01 * SS_VXY)) &&
            (fabsf(s.y) < (SS_VXY * SS_IMY / 2 - 0.01 * SS_VXY))) {
          i_smsk = a.mu_v2i[(int)(.5 * SS_IMX + floorf(s.x / SS_VXY) +
                                  SS_IMX * (.5 * SS_IMY - ceilf(s.y / SS_VXY)) +
                                  SS_IMX * SS_IMY * floorf(.5 * SS_IMZ + s.z * IS_VXZ))];
        } else {
          infov = 0;
          i_smsk = 0;
        }
        if (i_smsk < 0) {
          infov = 0;
          i_smsk = 0;
        }
        const float scx = __shfl_sync(0xffffffffu, sc.x, crs_shft);
        const float scy = __shfl_sync(0xffffffffu, sc.y, crs_shft);
        const float scz_ = __shfl_sync(0xffffffffu, sc.z, crs_shft);
        const int iscj = __shfl_sync(0xffffffffu, (int)isc, crs_shft);
        s.x = scx - s.x;
        s.y = scy - s.y;
        s.z = scz_ - s.z;
        const float s_l = powf(s.x * s.x + s.y * s.y + s.z * s.z, 0.5f);
        const float _s_lgth = 1 / s_l;
        s.x *= _s_lgth;
        s.y *= _s_lgth;
        s.z *= _s_lgth;
        const float cosups = s.x * av.x + s.y * av.y + s.z * av.z;
        unsigned short icos =
            (unsigned short)(a.cosstp_inv * (cosups - a.cos0)) * (cosups >= a.cos0);
        if (icos > NCOS - 1) icos = NCOS - 1;  // a dot product of unit vectors above 1
        acc[j] += infov * s_kn[icos].x * em_vox *
                  (SRFCRS * (s.x * scx * IR_RING + s.y * scy * IR_RING) * (_s_lgth * _s_lgth)) *
                  expf(-s_kn[icos].y * a.rays[(size_t)i_smsk * NSCRS * NSRNG + iscj * NSRNG + isr] *
                       RES_SUM) *
                  psp;
      }
    }
    // the 8 patches of a crystal: lanes with equal idx & 3
#pragma unroll
    for (int j = 0; j < (SS_WRP >> LSCT2); j++) {
      float vsum = acc[j];
      vsum += __shfl_xor_sync(0xffffffffu, vsum, 4);
      vsum += __shfl_xor_sync(0xffffffffu, vsum, 8);
      vsum += __shfl_xor_sync(0xffffffffu, vsum, 16);
      const int crs = __shfl_sync(0xffffffffu, (int)isc, (idx & 3) + j * (1 << LSCT2));
      if (idx < 4) s_acc[isr][crs] += vsum;
    }
  }
  __syncthreads();
  for (int i = tid; i < NSRNG * NSCRS; i += 256) {
    const int sr = i / NSCRS, scr = i - sr * NSCRS;
    const float vv = s_acc[sr][scr];
    if (vv != 0.f) atomicAdd(a.rslt + scr + sr * NSCRS + (iuc + iur * NSCRS) * (NSRNG * NSCRS), vv);
  }
}

// raw results -> span-1 pre-sinogram [NSN64][NSCRS * NSCRS] (sctaux.cu:18-43): block
// (scatter crystal, scatter ring), grid (unscattered crystal, unscattered ring); every
// result has a bin of its own
__global__ void k_sct2sn1(float *scts1, const float *srslt, const int8_t *xsxu,
                          const int16_t *offseg, const int16_t *isrng) {
  const int ics = threadIdx.x, irs = threadIdx.y, icu = blockIdx.x, iru = blockIdx.y;
  const int ssi = NSCRS * icu + ics;
  const bool pos = ((2 * xsxu[ssi] - 1) * (irs - iru)) > 0;
  const int rd = abs(isrng[irs] - isrng[iru]);
  const int rdi = 2 * rd - 1 * pos;
  const int sni = offseg[rdi] + min(isrng[irs], isrng[iru]);
  scts1[(size_t)sni * NSCRS * NSCRS + ssi] =
      srslt[iru * NSCRS * NSRNG * NSCRS + icu * NSRNG * NSCRS + irs * NSCRS + ics];
}

// axial interpolation of the pre-sinogram bin b of span-1 sinogram sni (sctaux.cu:46-72)
__device__ __forceinline__ float axinterp(const float *scts1, const int4 *R, const float4 *W,
                                          int sni, int b) {
  constexpr int NBIN = NSCRS * NSCRS;
  return W[sni].x * scts1[NBIN * R[sni].x + b] + W[sni].y * scts1[NBIN * R[sni].y + b] +
         W[sni].z * scts1[NBIN * R[sni].z + b] + W[sni].w * scts1[NBIN * R[sni].w + b];
}

// span 1: out [NSN64][NBIN], rows >= nsn1 left zero
__global__ void k_sct_ax1(float *out, const float *scts1, const int4 *R, const float4 *W,
                          int nsn1) {
  constexpr int NBIN = NSCRS * NSCRS;
  const size_t n = (size_t)nsn1 * NBIN;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const int sni = (int)(i / NBIN), b = (int)(i - (size_t)sni * NBIN);
    out[i] = axinterp(scts1, R, W, sni, b);
  }
}

// span 11: out [NSN11][NBIN]; sinogram s sums its span-1 sinograms lst[off[s] .. off[s+1])
// in ascending order
__global__ void k_sct_ax11(float *out, const float *scts1, const int4 *R, const float4 *W,
                           const int *off, const int16_t *lst, int nsn11) {
  constexpr int NBIN = NSCRS * NSCRS;
  const size_t n = (size_t)nsn11 * NBIN;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const int s = (int)(i / NBIN), b = (int)(i - (size_t)s * NBIN);
    float acc = 0.f;
    for (int q = off[s]; q < off[s + 1]; q++) acc += axinterp(scts1, R, W, lst[q], b);
    out[i] = acc;
  }
}

}  // namespace nbs

using namespace nbs;

extern "C" int nb_sct_vsm(const float *mu, const int8_t *mumsk, const float *em,
                          const float *scrs, int nscrs, const float *srng,
                          const int16_t *isrng, int nsrng, const float *knlut, float cosupsmx,
                          float ethrld, const int8_t *xsxu, const int16_t *offseg, int nseg0,
                          const int32_t *sctaxR, const float *sctaxW, int nsn64,
                          const int16_t *sn1_sn11, int nsn1, int span, float *sval,
                          float *s3d, int *nvx, void *stream) {
  NB_RANGE("nb_sct_vsm");
  NB_REQUIRE(mu && mumsk && em && scrs && srng && isrng && knlut && xsxu && offseg && sctaxR &&
                 sctaxW && sn1_sn11 && sval && s3d,
             "nb_sct_vsm: NULL argument");
  NB_REQUIRE(nscrs == NSCRS && nsrng == NSRNG,
             "nb_sct_vsm: the mMR scatter model uses 64 scatter crystals and 8 scatter rings");
  NB_REQUIRE(span == 1 || span == 11, "nb_sct_vsm: span must be 1 or 11");
  NB_REQUIRE(nsn64 == NB_NRINGS * NB_NRINGS && nsn1 == NB_NSN1 && nseg0 >= 1,
             "nb_sct_vsm: unexpected sinogram counts");
  NB_REQUIRE(cosupsmx > -1.f && cosupsmx < 1.f, "nb_sct_vsm: COSUPSMX out of (-1, 1)");
  constexpr int NBIN = NSCRS * NSCRS;
  constexpr size_t NMU = (size_t)SS_IMX * SS_IMY * SS_IMZ;
  constexpr size_t NEM = (size_t)SSE_IMX * SSE_IMY * SSE_IMZ;
  for (int i = 0; i < NSRNG; i++)
    NB_REQUIRE(isrng[i] >= 0 && isrng[i] < NB_NRINGS, "nb_sct_vsm: scatter ring out of range");
  for (int i = 0; i < nsn64; i++)
    for (int q = 0; q < 4; q++)
      NB_REQUIRE(sctaxR[4 * i + q] >= 0 && sctaxR[4 * i + q] < nsn64,
                 "nb_sct_vsm: axial interpolation index out of range");
  // every (scatter ring, unscattered ring) pair must land in the span-1 pre-sinogram
  for (int r0 = 0; r0 < NSRNG; r0++)
    for (int r1 = 0; r1 < NSRNG; r1++)
      for (int pos = 0; pos < 2; pos++) {
        const int rd = abs(isrng[r0] - isrng[r1]);
        if (rd == 0 && pos) continue;
        const int rdi = 2 * rd - pos;
        NB_REQUIRE(rdi >= 0 && rdi <= nseg0, "nb_sct_vsm: segment index out of range");
        const int sni = offseg[rdi] + (isrng[r0] < isrng[r1] ? isrng[r0] : isrng[r1]);
        NB_REQUIRE(sni >= 0 && sni < nsn64, "nb_sct_vsm: segment offset out of range");
      }
  cudaStream_t s = (cudaStream_t)stream;

  // voxel masks (sctaux.cu:200-340): attenuating voxels from the mask, emitting voxels
  // above ethrld x the emission maximum
  std::vector<int> mu_v2i(NMU), mu_i2v;
  mu_i2v.reserve(NMU / 2);
  for (size_t i = 0; i < NMU; i++) {
    mu_v2i[i] = -1;
    if (mumsk[i] > 0) {
      mu_v2i[i] = (int)mu_i2v.size();
      mu_i2v.push_back((int)i);
    }
  }
  float emmx = -1e12f;
  for (size_t i = 0; i < NEM; i++)
    if (em[i] > emmx) emmx = em[i];
  const float thr = ethrld * emmx;
  std::vector<int> em_i2v;
  for (size_t i = 0; i < NEM; i++)
    if (em[i] > thr) em_i2v.push_back((int)i);
  const int nmu = (int)mu_i2v.size(), nem = (int)em_i2v.size();
  if (nvx) {
    nvx[0] = nmu;
    nvx[1] = nem;
  }
  // span-11 sums: the span-1 sinograms of each span-11 sinogram, ascending
  std::vector<int> off11(NB_NSN11 + 1, 0);
  std::vector<int16_t> lst11;
  for (int k = 0; k < NB_NSN11; k++) {
    for (int i = 0; i < nsn1; i++)
      if (sn1_sn11[i] == k) lst11.push_back((int16_t)i);
    off11[k + 1] = (int)lst11.size();
  }
  NB_REQUIRE((int)lst11.size() == nsn1, "nb_sct_vsm: sn1_sn11 out of range");
  float sctcnt[2] = {cosupsmx, (NCOS - 1) / (1 - cosupsmx)};

  // device scratch, one block: masks, emission image, LUTs, rays, span-1 pre-sinogram
  const size_t rays_n = (size_t)(nmu > 0 ? nmu : 1) * NSCRS * NSRNG;
  size_t o = 0;
  auto take = [&o](size_t bytes) {
    const size_t at = o;
    o = (o + bytes + 255) & ~(size_t)255;
    return at;
  };
  const size_t o_v2i = take(sizeof(int) * NMU), o_mi2v = take(sizeof(int) * (nmu + 1));
  const size_t o_ei2v = take(sizeof(int) * (nem + 1)), o_em = take(sizeof(float) * NEM);
  const size_t o_scrs = take(sizeof(float) * 3 * NSCRS), o_srng = take(sizeof(float) * 2 * NSRNG);
  const size_t o_kn = take(sizeof(float2) * NCOS), o_xsxu = take(NSCRS * NSCRS);
  const size_t o_off = take(sizeof(int16_t) * (nseg0 + 1)), o_isr = take(sizeof(int16_t) * NSRNG);
  const size_t o_R = take(sizeof(int4) * nsn64), o_W = take(sizeof(float4) * nsn64);
  const size_t o_o11 = take(sizeof(int) * off11.size()), o_l11 = take(sizeof(int16_t) * nsn1);
  const size_t o_rays = take(sizeof(int16_t) * rays_n);
  const size_t o_s1 = take(sizeof(float) * (size_t)nsn64 * NBIN);
  const size_t host_end = o_rays;  // everything before the rays comes from the host
  unsigned char *d = nullptr;
  NB_CUDA(cudaMallocAsync((void **)&d, o, s));
  std::vector<unsigned char> h(host_end, 0);
  memcpy(&h[o_v2i], mu_v2i.data(), sizeof(int) * NMU);
  memcpy(&h[o_mi2v], mu_i2v.data(), sizeof(int) * nmu);
  memcpy(&h[o_ei2v], em_i2v.data(), sizeof(int) * nem);
  memcpy(&h[o_em], em, sizeof(float) * NEM);
  memcpy(&h[o_scrs], scrs, sizeof(float) * 3 * NSCRS);
  memcpy(&h[o_srng], srng, sizeof(float) * 2 * NSRNG);
  memcpy(&h[o_kn], knlut, sizeof(float2) * NCOS);
  memcpy(&h[o_xsxu], xsxu, NSCRS * NSCRS);
  memcpy(&h[o_off], offseg, sizeof(int16_t) * (nseg0 + 1));
  memcpy(&h[o_isr], isrng, sizeof(int16_t) * NSRNG);
  memcpy(&h[o_R], sctaxR, sizeof(int4) * nsn64);
  memcpy(&h[o_W], sctaxW, sizeof(float4) * nsn64);
  memcpy(&h[o_o11], off11.data(), sizeof(int) * off11.size());
  memcpy(&h[o_l11], lst11.data(), sizeof(int16_t) * nsn1);
  cudaError_t e = cudaMemcpyAsync(d, h.data(), host_end, cudaMemcpyHostToDevice, s);

  // the mu-map as a 3D texture: trilinear filtering, zero outside (ray.cu / sct.cu set-up)
  cudaArray_t arr = nullptr;
  cudaTextureObject_t tex = 0;
  const cudaExtent ext = make_cudaExtent(SS_IMX, SS_IMY, SS_IMZ);
  if (e == cudaSuccess) {
    cudaChannelFormatDesc cd = cudaCreateChannelDesc(32, 0, 0, 0, cudaChannelFormatKindFloat);
    e = cudaMalloc3DArray(&arr, &cd, ext);
  }
  if (e == cudaSuccess) {
    cudaMemcpy3DParms cp = {};
    cp.srcPtr = make_cudaPitchedPtr((void *)mu, SS_IMX * sizeof(float), SS_IMX, SS_IMY);
    cp.dstArray = arr;
    cp.extent = ext;
    cp.kind = cudaMemcpyHostToDevice;
    e = cudaMemcpy3DAsync(&cp, s);
  }
  if (e == cudaSuccess) {
    cudaResourceDesc rd = {};
    rd.resType = cudaResourceTypeArray;
    rd.res.array.array = arr;
    cudaTextureDesc td = {};
    td.addressMode[0] = td.addressMode[1] = td.addressMode[2] = cudaAddressModeBorder;
    td.filterMode = cudaFilterModeLinear;
    td.readMode = cudaReadModeElementType;
    td.normalizedCoords = 0;
    e = cudaCreateTextureObject(&tex, &rd, &td, nullptr);
  }
  int16_t *rays = (int16_t *)(d + o_rays);
  float *scts1 = (float *)(d + o_s1);
  if (e == cudaSuccess) e = cudaMemsetAsync(sval, 0, sizeof(float) * NSRNG * NSCRS * NSRNG * NSCRS, s);
  if (e == cudaSuccess && nmu > 0 && nem > 0) {
    k_sct_rays<<<dim3(nmu, NSCRS), dim3(SS_WRP, NSRNG), 0, s>>>(
        rays, tex, (const int *)(d + o_mi2v), (const float *)(d + o_scrs),
        (const float *)(d + o_srng));
    e = cudaGetLastError();
    if (e == cudaSuccess) {
      PsctArgs pa;
      pa.tex = tex;
      pa.rays = rays;
      pa.mu_v2i = (const int *)(d + o_v2i);
      pa.em_i2v = (const int *)(d + o_ei2v);
      pa.em = (const float *)(d + o_em);
      pa.scrs = (const float *)(d + o_scrs);
      pa.srng = (const float *)(d + o_srng);
      pa.kn = (const float2 *)(d + o_kn);
      pa.cos0 = sctcnt[0];
      pa.cosstp_inv = sctcnt[1];
      pa.nvx_em = nem;
      pa.rslt = sval;
      int dev = 0, nsm = 148;
      cudaGetDevice(&dev);
      cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
      // about 16 blocks per SM over the (crystal, ring) pairs and voxel shares
      int nz = (nsm * 16 + NSCRS * NSRNG - 1) / (NSCRS * NSRNG);
      if (nz > nem) nz = nem;
      k_sct_psct<<<dim3(NSCRS, NSRNG, nz), dim3(SS_WRP, NSRNG), 0, s>>>(pa);
      e = cudaGetLastError();
    }
  }
  if (e == cudaSuccess) e = cudaMemsetAsync(scts1, 0, sizeof(float) * (size_t)nsn64 * NBIN, s);
  if (e == cudaSuccess) {
    k_sct2sn1<<<dim3(NSCRS, NSRNG), dim3(NSCRS, NSRNG), 0, s>>>(
        scts1, sval, (const int8_t *)(d + o_xsxu), (const int16_t *)(d + o_off),
        (const int16_t *)(d + o_isr));
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) {
    const int4 *R = (const int4 *)(d + o_R);
    const float4 *W = (const float4 *)(d + o_W);
    if (span == 1) {
      e = cudaMemsetAsync(s3d, 0, sizeof(float) * (size_t)nsn64 * NBIN, s);
      if (e == cudaSuccess) k_sct_ax1<<<2048, 256, 0, s>>>(s3d, scts1, R, W, nsn1);
    } else {
      k_sct_ax11<<<2048, 256, 0, s>>>(s3d, scts1, R, W, (const int *)(d + o_o11),
                                      (const int16_t *)(d + o_l11), NB_NSN11);
    }
    if (e == cudaSuccess) e = cudaGetLastError();
  }
  // the texture and its array are released once the kernels that sample them are done
  const cudaError_t es = cudaStreamSynchronize(s);
  if (e == cudaSuccess) e = es;
  if (tex) cudaDestroyTextureObject(tex);
  if (arr) cudaFreeArray(arr);
  cudaFreeAsync(d, s);
  if (e != cudaSuccess) return nb_cuda_fail(e, "nb_sct_vsm", __FILE__, __LINE__);
  return NB_OK;
}
