// nb_psf.cu -- resolution modelling: the separable 3-D convolution the reference applies
// inside OSEM when a PSF kernel is given (prj/src/recon.cu:49-216, used at :437-445 on the
// sensitivity images, :463-467 on the current image before the forward projection and
// :487-491 on the back projection), on the col128 image layout.
//
// The reference pads the image to [320][320][128] (z fastest), convolves along z with
// kernel row 0, then along the second image axis (x) with row 1, then along the first (y)
// with row 2, each a 17-tap sum with zeros outside the volume, accumulated tap by tap
// from offset -8 to +8 with fused multiply-adds.  The passes here do the same, in the
// same order and with the same rounding, so the results agree bit for bit; z slot 127
// (the padding) stays zero.
#include <cuda_runtime.h>

#include "nb_internal.cuh"

namespace {

constexpr int R = 8;               // kernel radius (RSZ_PSF_KRNL)
constexpr int KL = 2 * R + 1;      // taps per axis
constexpr int TILE = 32;           // output columns per block in the x / y passes

struct PsfKernel {
  float k[3][KL];  // [0] z, [1] second axis (x), [2] first axis (y)
};

// z pass: one block per transaxial column, thread = output z
__global__ void k_psf_z(float *__restrict__ dst, const float *__restrict__ src,
                        const PsfKernel K) {
  __shared__ float s[NB_COLW + 2 * R];  // natural z order, zero halo
  const int t = threadIdx.x;            // 0..127
  for (int col = blockIdx.x; col < NB_NCOL; col += gridDim.x) {
    const float *c = src + (size_t)col * NB_COLW;
    __syncthreads();
    if (t < R) {
      s[t] = 0.f;
      s[R + NB_COLW + t] = 0.f;
    }
    // slot of z: even z at z/2, odd z at 64 + z/2; z = 127 is the zero padding slot
    s[R + t] = t < 127 ? c[(t >> 1) + ((t & 1) << 6)] : 0.f;
    __syncthreads();
    float sum = 0.f;
#pragma unroll
    for (int j = -R; j <= R; j++) sum = __fmaf_rn(K.k[0][R - j], s[R + t + j], sum);
    const int slot = (t >> 1) + ((t & 1) << 6);
    dst[(size_t)col * NB_COLW + slot] = t < 127 ? sum : 0.f;
  }
}

// x / y pass: block = TILE consecutive output columns along the axis (stride `step`
// columns between neighbours) x 128 slots; the tile and its halo are staged in shared
// memory.  AXIS 1: neighbours along x (step 1), AXIS 2: along y (step 320).
template <int AXIS>
__global__ void k_psf_xy(float *__restrict__ dst, const float *__restrict__ src,
                         const PsfKernel K) {
  extern __shared__ float tile[];  // [TILE + 2R][128]
  constexpr int step = AXIS == 1 ? 1 : NB_IMX;
  const int ntile = NB_IMX / TILE;  // tiles per line
  const int slot = threadIdx.x;    // 0..127
  for (int b = blockIdx.x; b < NB_IMY * ntile; b += gridDim.x) {
    const int line = b / ntile, seg = b - line * ntile;
    // first output column of the tile and the column index of its position 0
    const int p0 = seg * TILE;
    const int base = AXIS == 1 ? line * NB_IMX : line;  // column of position 0 on the line
    __syncthreads();
    for (int q = threadIdx.y; q < TILE + 2 * R; q += blockDim.y) {
      const int p = p0 - R + q;  // position along the line
      tile[q * NB_COLW + slot] =
          (p >= 0 && p < NB_IMX) ? src[((size_t)base + (size_t)p * step) * NB_COLW + slot] : 0.f;
    }
    __syncthreads();
    for (int q = threadIdx.y; q < TILE; q += blockDim.y) {
      float sum = 0.f;
#pragma unroll
      for (int j = -R; j <= R; j++)
        sum = __fmaf_rn(K.k[AXIS][R - j], tile[(q + R + j) * NB_COLW + slot], sum);
      const int p = p0 + q;
      dst[((size_t)base + (size_t)p * step) * NB_COLW + slot] = slot == 127 ? 0.f : sum;
    }
  }
}

}  // namespace

extern "C" int nb_psf_col128(float *dst128, const float *src128, const float *krnl,
                             float *tmp128, void *stream) {
  NB_RANGE("nb_psf");
  NB_REQUIRE(dst128 && src128 && krnl && tmp128, "nb_psf_col128: NULL argument");
  NB_REQUIRE(dst128 != tmp128 && src128 != tmp128, "nb_psf_col128: tmp must be its own buffer");
  PsfKernel K;
  for (int a = 0; a < 3; a++)
    for (int i = 0; i < KL; i++) K.k[a][i] = krnl[a * KL + i];
  cudaStream_t s = (cudaStream_t)stream;
  int dev = 0, nsm = 148;
  NB_CUDA(cudaGetDevice(&dev));
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  const size_t smem = (size_t)(TILE + 2 * R) * NB_COLW * sizeof(float);
  static_assert(NB_IMX % TILE == 0, "tiles must cover a line");
  // z: src -> tmp, x: tmp -> dst, y: dst -> tmp, copy back: the passes of the reference
  // in its order; dst may alias src
  k_psf_z<<<nsm * 16, NB_COLW, 0, s>>>(tmp128, src128, K);
  k_psf_xy<1><<<nsm * 8, dim3(NB_COLW, 8), smem, s>>>(dst128, tmp128, K);
  k_psf_xy<2><<<nsm * 8, dim3(NB_COLW, 8), smem, s>>>(tmp128, dst128, K);
  NB_CUDA(cudaMemcpyAsync(dst128, tmp128, sizeof(float) * NB_IMG_COL128,
                          cudaMemcpyDeviceToDevice, s));
  NB_CUDA(cudaGetLastError());
  return NB_OK;
}
