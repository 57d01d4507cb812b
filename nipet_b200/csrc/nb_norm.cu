// nb_norm.cu -- the normalisation sinogram from its components (the reference's
// norm_from_components, src/norm.cu:13-210, driven by mmrnorm.get_norm_sino,
// mmrnorm.py:155-195).
//
// For a LOR (sinogram bin w, angle a; crystals c1, c2 of the two detectors) and a span-1
// plane (rings r0, r1) the factor is
//   geo[w] * cinf[w][a % 9] * ceff[r0][c1] * ceff[r1][c2] * d(b1, r0) * d(b2, r1),
//   d(b, r) = exp(x dtp[r] / (1 + x dtnp[r])) / (1 + x dtnp[r]),  x = buckets[b] / 2,
// with b the singles bucket of the crystal (28 x 18 crystals transaxially, 8 rings
// axially); span 1 scales it by axf1[plane] / axe1[span-11 sinogram], span 11 sums
// factor / (axe1 * planes of the sinogram) over its planes (norm.cu:13-48).
//
// B200 form: the dead-time part depends only on (ring, crystal): a [64][504] table of
// {ceff, exp term, denominator} is made once on the device with the reference's own
// mixed float/double expression, so a bin costs one 16-byte read per crystal and the
// float products in the reference's left-to-right order; span 11 is a gather over each
// sinogram's planes in ascending plane order -- the order in which the reference's one
// thread per LOR adds its atomics -- so the sinogram is deterministic and bit-exact with
// the reference's.
#include <cuda_runtime.h>

#include <vector>

#include "nb_internal.cuh"

namespace {

constexpr int NR = 64, NCF = 504, MAXPL = 16, NB_BUCKETS = 224;
constexpr int BT = 28, CBT = 18, CBA = 8;  // buckets transaxially, crystals per bucket
                                          // transaxially and axially (norm.cu:176-178)

// crystal pair of a gap-free LOR, as norm.cu:18-23 computes it from the full linear index
__device__ __forceinline__ void norm_crystals(int ali, int &wi, int &ai, int &c1, int &c2) {
  wi = ali % NB_NSBINS;
  ai = (ali - wi) / NB_NSBINS;
  const float h1 = (float)ai + 0.5f * (float)(NCF - 2 + NB_NSBINS / 2 - wi);
  const float h2 = (float)ai + 0.5f * (float)(2 * NCF - 2 - NB_NSBINS / 2 + wi);
  c1 = (int)floorf(fmodf(h1, (float)NCF));
  c2 = (int)floorf(fmodf(h2, (float)NCF));
}

// per (ring, crystal): {efficiency, dead-time exponential, dead-time denominator}, as
// norm.cu:36-40 evaluates them (double products, float conversions)
__global__ void k_norm_crystal(float4 *__restrict__ tab, const float *__restrict__ ceff,
                               const float *__restrict__ dtp, const float *__restrict__ dtnp,
                               const int32_t *__restrict__ bck) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= NR * NCF) return;
  const int r = i / NCF, c = i - r * NCF;
  const int b = c / CBT + BT * (r / CBA);
  const float den = (float)(1 + 0.5 * bck[b] * dtnp[r]);
  const float e = expf(0.5 * (float)bck[b] * dtp[r] / den);
  tab[i] = make_float4(ceff[i], e, den, 0.f);
}

// out [68516][nout]: thread per (LOR, output sinogram)
__global__ void k_norm(float *__restrict__ out, const float *__restrict__ geo,
                       const float *__restrict__ cinf, const float4 *__restrict__ tab,
                       const float *__restrict__ axe1, const float *__restrict__ axf1,
                       const short2 *__restrict__ sn1_rno, const int16_t *__restrict__ sn1_sn11,
                       const int16_t *__restrict__ planes, const int8_t *__restrict__ nos,
                       const int32_t *__restrict__ aw2ali, int nout, int span) {
  const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i >= (size_t)NB_AW * nout) return;
  const int aw = (int)(i / nout), so = (int)(i - (size_t)aw * nout);
  int wi, ai, c1, c2;
  norm_crystals(aw2ali[aw], wi, ai, c1, c2);
  const float gc = geo[wi] * cinf[ai % 9 + 9 * wi];
  float v = 0.f;
  for (int p = 0; p < MAXPL; p++) {
    const int si = planes[so * MAXPL + p];
    if (si < 0) break;
    const short2 rr = sn1_rno[si];
    const float4 t1 = tab[rr.x * NCF + c1], t2 = tab[rr.y * NCF + c2];
    // geo * cinf * ceff1 * ceff2 * e1 / den1 * e2 / den2, left to right (norm.cu:36-40)
    float f = __fmul_rn(__fmul_rn(gc, t1.x), t2.x);
    f = __fdiv_rn(__fmul_rn(f, t1.y), t1.z);
    f = __fdiv_rn(__fmul_rn(f, t2.y), t2.z);
    v += span == 1 ? __fdiv_rn(__fmul_rn(f, axf1[si]), axe1[sn1_sn11[si]])
                   : __fdiv_rn(f, __fmul_rn(axe1[so], (float)nos[si]));
  }
  out[i] = v;
}

}  // namespace

extern "C" int nb_norm(float *sng, const float *geo, int ngeo, const float *cinf,
                       const float *ceff, const float *axe1, const float *axf1,
                       const float *dtp, const float *dtnp, const int32_t *buckets,
                       const int16_t *sn1_rno, const int16_t *sn1_sn11, const int8_t *sn1_sn11no,
                       const int32_t *aw2ali, int span, void *stream) {
  NB_RANGE("nb_norm");
  NB_REQUIRE(sng && geo && cinf && ceff && axe1 && dtp && dtnp && buckets && sn1_rno &&
                 sn1_sn11 && sn1_sn11no && aw2ali,
             "nb_norm: NULL argument");
  NB_REQUIRE(span == 11 || (span == 1 && axf1), "nb_norm: span must be 11, or 1 with axf1");
  NB_REQUIRE(ngeo >= NB_NSBINS, "nb_norm: geo must hold at least 344 values");
  cudaStream_t st = (cudaStream_t)stream;
  const int nout = span == 11 ? NB_NSN11 : NB_NSN1;
  std::vector<int16_t> planes((size_t)nout * MAXPL, -1);
  std::vector<int> npl(nout, 0);
  for (int si = 0; si < NB_NSN1; si++) {
    const int so = span == 11 ? sn1_sn11[si] : si;
    NB_REQUIRE(so >= 0 && so < nout && npl[so] < MAXPL, "nb_norm: bad span-1 to span-11 map");
    planes[(size_t)so * MAXPL + npl[so]++] = (int16_t)si;
  }
  char *buf = nullptr;
  const size_t bytes = sizeof(float4) * (size_t)NR * NCF +
                       sizeof(float) * (2 * (size_t)NR * NCF + NB_NSBINS + 9 * NB_NSBINS +
                                        NB_NSN11 + NB_NSN1 + 2 * NR) +
                       sizeof(int32_t) * NB_BUCKETS +
                       sizeof(short2) * NB_NSN1 + sizeof(int16_t) * (planes.size() + NB_NSN1) +
                       sizeof(int32_t) * NB_AW + NB_NSN1 + 64;
  NB_CUDA(cudaMallocAsync((void **)&buf, bytes, st));
  float4 *d_tab = (float4 *)buf;
  float *d_ceff = (float *)(d_tab + NR * NCF), *d_geo = d_ceff + NR * NCF;
  float *d_cinf = d_geo + NB_NSBINS, *d_dtp = d_cinf + 9 * NB_NSBINS, *d_dtnp = d_dtp + NR;
  float *d_axe1 = d_dtnp + NR, *d_axf1 = d_axe1 + NB_NSN11;
  int32_t *d_bck = (int32_t *)(d_axf1 + NB_NSN1), *d_aw = d_bck + NB_BUCKETS;
  short2 *d_rno = (short2 *)(d_aw + NB_AW);
  int16_t *d_s11 = (int16_t *)(d_rno + NB_NSN1), *d_pl = d_s11 + NB_NSN1;
  int8_t *d_nos = (int8_t *)(d_pl + planes.size());
  int st_ = NB_OK;
  auto cp = [&](void *dst, const void *src, size_t n) {
    if (st_ == NB_OK && cudaMemcpyAsync(dst, src, n, cudaMemcpyHostToDevice, st) != cudaSuccess)
      st_ = nb_cuda_fail(cudaGetLastError(), "nb_norm upload", __FILE__, __LINE__);
  };
  cp(d_ceff, ceff, sizeof(float) * NR * NCF);
  cp(d_dtp, dtp, sizeof(float) * NR);
  cp(d_dtnp, dtnp, sizeof(float) * NR);
  cp(d_bck, buckets, sizeof(int32_t) * NB_BUCKETS);
  cp(d_geo, geo, sizeof(float) * NB_NSBINS);
  cp(d_cinf, cinf, sizeof(float) * 9 * NB_NSBINS);
  cp(d_axe1, axe1, sizeof(float) * NB_NSN11);
  if (span == 1) cp(d_axf1, axf1, sizeof(float) * NB_NSN1);
  cp(d_aw, aw2ali, sizeof(int32_t) * NB_AW);
  cp(d_rno, sn1_rno, sizeof(short2) * NB_NSN1);
  cp(d_s11, sn1_sn11, sizeof(int16_t) * NB_NSN1);
  cp(d_pl, planes.data(), sizeof(int16_t) * planes.size());
  cp(d_nos, sn1_sn11no, NB_NSN1);
  if (st_ == NB_OK) {
    k_norm_crystal<<<(NR * NCF + 255) / 256, 256, 0, st>>>(d_tab, d_ceff, d_dtp, d_dtnp, d_bck);
    const size_t n = (size_t)NB_AW * nout;
    k_norm<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(sng, d_geo, d_cinf, d_tab, d_axe1, d_axf1,
                                                        d_rno, d_s11, d_pl, d_nos, d_aw, nout,
                                                        span);
    if (cudaGetLastError() != cudaSuccess)
      st_ = nb_cuda_fail(cudaGetLastError(), "nb_norm launch", __FILE__, __LINE__);
  }
  cudaFreeAsync(buf, st);
  return st_;
}
