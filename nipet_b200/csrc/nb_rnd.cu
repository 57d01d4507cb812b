// nb_rnd.cu -- randoms from the delayed fan sums (the reference's gpu_randoms,
// lm/src/rnd.cu:169-386, driven by mmrhist.randoms/rand, lm/mmrhist.py:188-221).
//
// Crystal singles s[r][c] (64 rings x 448 active crystals) are fitted to the delayed fan
// sums F[r][c] with F ~ s[r][c] * fan(s)[r][c], where fan(s)[r][c] sums s over the rings
// within the maximum ring difference of r and the crystals in coincidence with c (one
// circular range per crystal, from the cij table): s0 = sqrt(F / fan(1)), then ten steps
// s <- s/2 + F / (2 fan(s)) (rnd.cu:238-262).  The randoms sinogram is s[r0][c0] s[r1][c1]
// per LOR and span-1 plane, summed over the planes of a span-11 sinogram.
//
// B200 form: the fan sum is separable -- a crystal-range sum per ring, then a ring-range
// sum -- so each pass is a plain per-element loop instead of the reference's block-wide
// tree reductions; the span-11 sum is a gather over each sinogram's planes in plane order
// instead of float atomics, so the sinogram is deterministic.  Sums are float32 like the
// reference's; results agree to rounding (relative 1e-5 in the tests).
#include <cuda_runtime.h>

#include <vector>

#include "nb_internal.cuh"

namespace {

constexpr int NR = 64;    // rings
constexpr int NC = 448;   // active crystals per ring
constexpr int NCF = 504;  // crystals per ring with gaps
constexpr int NITER = 10;
constexpr int MAXPL = 16;  // span-1 planes per span-11 sinogram (at most 6 for the mMR)

// T[r][c] = sum over the crystals in coincidence with c of s[r][.]
__global__ void k_fan_crystals(float *__restrict__ T, const float *__restrict__ s,
                               const short2 *__restrict__ crange) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= NR * NC) return;
  const int r = i / NC, c = i - r * NC;
  const short2 cr = crange[c];  // (first crystal, count), circular
  float acc = 0.f;
  for (int k = 0; k < cr.y; k++) {
    int cc = cr.x + k;
    cc -= cc >= NC ? NC : 0;
    acc += s[r * NC + cc];
  }
  T[i] = acc;
}

// U[r][c] = sum over the rings within the maximum ring difference of r of T[.][c]
__global__ void k_fan_rings(float *__restrict__ U, const float *__restrict__ T,
                            const short2 *__restrict__ rrange) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= NR * NC) return;
  const int r = i / NC, c = i - r * NC;
  const short2 rr = rrange[r];  // (first ring, last ring)
  float acc = 0.f;
  for (int q = rr.x; q <= rr.y; q++) acc += T[q * NC + c];
  U[i] = acc;
}

__global__ void k_fill_ones(float *__restrict__ s) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < NR * NC) s[i] = 1.f;
}

// init (s = sqrt(F / n)) or one damped step (s = s/2 + F/(2 U))
__global__ void k_singles_step(float *__restrict__ s, const float *__restrict__ U,
                               const uint32_t *__restrict__ F, int init) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= NR * NC) return;
  const float f = (float)F[i];
  s[i] = init ? sqrtf(f / U[i]) : 0.5f * s[i] + 0.5f * (f / U[i]);
}

// randoms sinogram: thread per (output sinogram, LOR); gapped layout [nout][252][344]
__global__ void k_singles_to_sino(float *__restrict__ rsn, const float *__restrict__ s,
                                  const short2 *__restrict__ s2cr, const short2 *__restrict__ aw2sn,
                                  const short2 *__restrict__ sn1_rno,
                                  const int16_t *__restrict__ planes, int nout, int naw) {
  const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i >= (size_t)nout * naw) return;
  const int so = (int)(i / naw), aw = (int)(i - (size_t)so * naw);
  const short2 cc = s2cr[aw], a = aw2sn[aw];
  float v = 0.f;
  for (int p = 0; p < MAXPL; p++) {
    const int si = planes[so * MAXPL + p];
    if (si < 0) break;
    const short2 rr = sn1_rno[si];
    v += s[rr.x * NC + cc.x] * s[rr.y * NC + cc.y];
  }
  rsn[(size_t)so * NB_NSBINANG + a.x * NB_NSBINS + a.y] = v;
}

// singles map [504][64] (crystal with gaps, ring), zero at gap crystals
__global__ void k_singles_map(float *__restrict__ cmap, const float *__restrict__ s,
                              const int16_t *__restrict__ crsr) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= NCF * NR) return;
  const int c = i / NR, r = i - c * NR;
  const int cr = crsr[c];
  cmap[i] = cr >= 0 ? s[r * NC + cr] : 0.f;
}

}  // namespace

extern "C" int nb_randoms(float *rsn, float *cmap, const uint32_t *fansums, const int16_t *crsr,
                          const int8_t *cij, const int16_t *s2cr, const int16_t *aw2sn,
                          const int16_t *sn1_rno, const int16_t *sn1_sn11, int span, int mrd,
                          void *stream) {
  NB_RANGE("nb_randoms");
  NB_REQUIRE(rsn && cmap && fansums && crsr && cij && s2cr && aw2sn && sn1_rno,
             "nb_randoms: NULL argument");
  NB_REQUIRE(span == 1 || (span == 11 && sn1_sn11), "nb_randoms: span must be 1 or 11");
  NB_REQUIRE(mrd >= 0 && mrd < NR, "nb_randoms: bad maximum ring difference");
  cudaStream_t st = (cudaStream_t)stream;
  const int naw = NB_AW, nout = span == 11 ? NB_NSN11 : NB_NSN1;
  // host tables: crystal fan ranges (circular runs of cij), ring ranges, planes per output
  std::vector<short2> crange(NC), rrange(NR);
  for (int c1 = 0; c1 < NC; c1++) {
    const int8_t *row = cij + (size_t)c1 * NC;
    int first = -1, cnt = 0;
    for (int c2 = 0; c2 < NC; c2++) {
      cnt += row[c2] != 0;
      const int prv = row[(c2 + NC - 1) % NC];
      if (row[c2] != 0 && prv == 0) {
        NB_REQUIRE(first < 0, "nb_randoms: cij row is not one circular run");
        first = c2;
      }
    }
    if (first < 0) first = 0;  // empty row, or a full ring
    crange[c1] = make_short2((short)first, (short)cnt);
  }
  for (int r = 0; r < NR; r++)
    rrange[r] = make_short2((short)(r - mrd < 0 ? 0 : r - mrd),
                            (short)(r + mrd > NR - 1 ? NR - 1 : r + mrd));
  std::vector<int16_t> planes((size_t)nout * MAXPL, -1);
  std::vector<int> npl(nout, 0);
  for (int si = 0; si < NB_NSN1; si++) {
    const int so = span == 11 ? sn1_sn11[si] : si;
    NB_REQUIRE(so >= 0 && so < nout && npl[so] < MAXPL, "nb_randoms: bad span-1 to span-11 map");
    planes[(size_t)so * MAXPL + npl[so]++] = (int16_t)si;
  }
  std::vector<uint32_t> fr((size_t)NR * NC);  // fan sums [ring][active crystal]
  std::vector<uint32_t> fh((size_t)NR * NCF);
  // fansums may live on the device (the histogram's output) or on the host
  cudaPointerAttributes pa{};
  const bool on_dev = cudaPointerGetAttributes(&pa, fansums) == cudaSuccess &&
                      pa.type == cudaMemoryTypeDevice;
  cudaGetLastError();
  if (on_dev)
    NB_CUDA(cudaMemcpyAsync(fh.data(), fansums, sizeof(uint32_t) * fh.size(),
                            cudaMemcpyDeviceToHost, st));
  NB_CUDA(cudaStreamSynchronize(st));
  const uint32_t *fsrc = on_dev ? fh.data() : fansums;
  for (int c = 0; c < NCF; c++)
    if (crsr[c] >= 0) {
      NB_REQUIRE(crsr[c] < NC, "nb_randoms: bad reduced crystal index");
      for (int r = 0; r < NR; r++) fr[(size_t)r * NC + crsr[c]] = fsrc[(size_t)r * NCF + c];
    }
  // device buffers (freed on the stream once the kernels are done)
  char *buf = nullptr;
  const size_t nsz = sizeof(float) * NR * NC;
  const size_t bytes = 4 * nsz + sizeof(short2) * (NC + NR) + sizeof(int16_t) * planes.size() +
                       sizeof(short2) * (2 * (size_t)naw + NB_NSN1) + sizeof(int16_t) * NCF;
  NB_CUDA(cudaMallocAsync((void **)&buf, bytes, st));
  float *s = (float *)buf, *T = s + NR * NC, *U = T + NR * NC;
  uint32_t *F = (uint32_t *)(U + NR * NC);
  short2 *d_cr = (short2 *)(F + NR * NC), *d_rr = d_cr + NC;
  int16_t *d_pl = (int16_t *)(d_rr + NR);
  short2 *d_s2cr = (short2 *)(d_pl + planes.size());
  short2 *d_aw2sn = d_s2cr + naw, *d_rno = d_aw2sn + naw;
  int16_t *d_crsr = (int16_t *)(d_rno + NB_NSN1);
  int st_ = NB_OK;
  auto cp = [&](void *dst, const void *src, size_t n) {
    if (st_ == NB_OK && cudaMemcpyAsync(dst, src, n, cudaMemcpyHostToDevice, st) != cudaSuccess)
      st_ = nb_cuda_fail(cudaGetLastError(), "nb_randoms upload", __FILE__, __LINE__);
  };
  cp(F, fr.data(), nsz);
  cp(d_cr, crange.data(), sizeof(short2) * NC);
  cp(d_rr, rrange.data(), sizeof(short2) * NR);
  cp(d_pl, planes.data(), sizeof(int16_t) * planes.size());
  cp(d_s2cr, s2cr, sizeof(short2) * naw);
  cp(d_aw2sn, aw2sn, sizeof(short2) * naw);
  cp(d_rno, sn1_rno, sizeof(short2) * NB_NSN1);
  cp(d_crsr, crsr, sizeof(int16_t) * NCF);
  if (st_ == NB_OK) {
    const int nb = (NR * NC + 255) / 256;
    k_fill_ones<<<nb, 256, 0, st>>>(s);
    // fan(1): the number of partners of each crystal; s0 = sqrt(F / fan(1))
    k_fan_crystals<<<nb, 256, 0, st>>>(T, s, d_cr);
    k_fan_rings<<<nb, 256, 0, st>>>(U, T, d_rr);
    k_singles_step<<<nb, 256, 0, st>>>(s, U, F, 1);
    for (int it = 0; it < NITER; it++) {
      k_fan_crystals<<<nb, 256, 0, st>>>(T, s, d_cr);
      k_fan_rings<<<nb, 256, 0, st>>>(U, T, d_rr);
      k_singles_step<<<nb, 256, 0, st>>>(s, U, F, 0);
    }
    if (cudaMemsetAsync(rsn, 0, sizeof(float) * (size_t)nout * NB_NSBINANG, st) != cudaSuccess)
      st_ = nb_cuda_fail(cudaGetLastError(), "nb_randoms", __FILE__, __LINE__);
    const size_t nt = (size_t)nout * naw;
    k_singles_to_sino<<<(unsigned)((nt + 255) / 256), 256, 0, st>>>(rsn, s, d_s2cr, d_aw2sn,
                                                                   d_rno, d_pl, nout, naw);
    k_singles_map<<<(NCF * NR + 255) / 256, 256, 0, st>>>(cmap, s, d_crsr);
    if (st_ == NB_OK && cudaGetLastError() != cudaSuccess)
      st_ = nb_cuda_fail(cudaGetLastError(), "nb_randoms launch", __FILE__, __LINE__);
  }
  cudaFreeAsync(buf, st);
  return st_;
}
