// nb_hist.cu -- list-mode histogramming of Siemens mMR 32-bit event words.
//
// Reference semantics: lm/src/hst.cu:37-244 (kernel hst), lm/src/lmaux.cu:17-270
// (chunk plan getLMinfo / modifyLMinfo), lm/src/lmproc.cu:156-193 (unpack).
//
// Bit-exactness with the reference comes from reproducing its work decomposition, not
// its launch shape: the reference cuts the stream into chunks ending at 100-ms time
// tags and each chunk into 2560 thread slices; a slice's events before its first time
// tag are attributed to that tag's second, and time tags are honoured only while the
// slice's current second is inside the frame window.  Here one warp processes one slice
// (32 consecutive words per step, coalesced), carrying the slice's current second
// across steps, so head curves, centre of mass and projection views match bit for bit.
// All counters are uint32 sums (order independent, wrap-around like the reference);
// per-second counters are warp-aggregated before their atomic.
//
// Bootstrap: the reference draws from clock()-seeded curand states; here every draw is
// Philox4x32-10 (Salmon et al., SC'11) keyed by the 64-bit seed, so replicates are
// reproducible and independent of the launch shape.  btp=2 draws N ~ Poisson(btprt) per
// word by integer inverse CDF (events with N = 0 or N >= 32 are dropped as in the
// reference) from output rep % 4 of the block with counter (word index, rep / 4, 0);
// btp=1 replaces each event word by a uniformly drawn event word of the same slice (at
// most 64 draws, counter (word index, replicate, 1 + draw)).
//
// Performance: persistent warps pull slices from a counter; per-second sums stay in
// shared memory until the warp's second changes.  With bootstrap replicates nb_hist counts
// the sinogram unpacked in a scratch ([bin][2][rblk]: prompts and delayeds apart, a bin's
// replicates side by side, so one event's replicate updates share one or two L2
// sectors), then packs it into the caller's sinograms (prompts + 65536 x delayeds, the
// reference's uint32 sum) and sums the SSRB counters from the prompts (every output
// sinogram lies in one SSRB sinogram) in the same pass, so the SSRB counters take no
// atomics; an event's replicate weights are staged in shared memory and added to its
// bin's replicate block by one bulk reduce-add (cp.reduce.async.bulk .add.u32) instead of
// one atomic per replicate.  More than 16 replicates go through in chunks of at most 16,
// one launch and one scratch fill each.
// A single span-1 histogram (1.4 GB of counters, ten times L2) writes 4-byte slab records
// instead of its sinogram atomics and then counts them one 64 MB slab of counters at a
// time, every update an L2 hit; a single span-11 or SSRB histogram, and nb_hist_static
// (which may not allocate), count both directly.
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <vector>

#include "nb_internal.cuh"

#define NB_TOTHRDS 2560
#define NB_ELECHNK (402653184 / 32)
#define NB_ITIME 1000
#define NB_BTPTIME 100
#define NB_MXNITAG 5400
#define NB_NBUCKTS 224

struct HistLUT {
  int16_t sn1_sn11[NB_NSN1];
  int16_t sn1_ssrb[NB_NSN1];
  int16_t sn1_rno[2 * NB_NSN1];
};

struct HistArgs {
  const int32_t *lm;
  const int64_t *atag;   // chunk starts [nchnk]
  const int *e4c;        // words per chunk
  const int *e4t;        // words per thread slice
  int nchnk;
  int toff, nitag, tstart, tstop, span, btp;
  uint64_t seed;
  int rep0, nrep;
  const HistLUT *lut;
  const short2 *s2cF;
  uint64_t thr[32];      // Poisson inverse-CDF thresholds (2^32 scaled)
  size_t nbins, sne;
  uint32_t *psino, *ssrb, *phc, *dhc, *pvs, *fan, *bck;
  int32_t *zR, *zM;
  int unp;                  // 1: psino is an unpacked scratch [bin][2][rblk] (prompts,
                            // delayeds) and SSRB is derived afterwards; 0: packed
                            // [nrep][bin] with SSRB counted here
  int rblk;                 // unpacked scratch: replicate block length (nrep rounded up to 4)
  int bulk;                 // unpacked scratch: one bulk reduce-add per event for all replicates
  unsigned *next_slice;     // work counter, 0 at launch
  // slab records (one histogram without bootstrap, counters larger than L2): instead of
  // its sinogram atomic, an event appends a record -- bin within its slab | delayed << 31
  // -- to its warp's region of its slab in `rec`; k_slab_add then counts one slab at a
  // time.  Warp w of the nwst launched takes slices w, w + nwst, ... (a fixed assignment,
  // so that k_slab_count can size every warp's regions beforehand).
  uint32_t *rec;            // NULL: count the sinogram directly
  const unsigned *roff;     // [nslab * nwst + 1] region starts, slab-major
  int nslab, nwst;
};

#define NB_SLAB_SHIFT 24   // bins per slab: 2^24 uint32 counters = 64 MB, well inside L2
#define NB_SLAB_CW 32      // records a warp stages per slab before it writes them out
#define NB_HIST_ROWS 2     // bulk-reduce staging rows per thread, used in turn

// Words between two threads' staging rows: the rows' length rounded up to an odd multiple
// of four words, so that every row stays 16-byte aligned for the bulk copy and a warp's
// stores of one replicate's weights spread over 8 banks (4-way, the least any 16-byte
// stride allows) instead of 1 or 2.
static __host__ __device__ __forceinline__ int hist_row_stride(int rblk) {
  const int w = NB_HIST_ROWS * rblk;
  return ((w >> 2) & 1) ? w : w + 4;
}
#define NB_HIST_REPCHUNK 16  // bootstrap replicates per histogram launch, at most

static __device__ __forceinline__ void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1) {
#pragma unroll
  for (int r = 0; r < 10; r++) {
    const uint32_t hi0 = __umulhi(0xD2511F53u, c[0]), lo0 = 0xD2511F53u * c[0];
    const uint32_t hi1 = __umulhi(0xCD9E8D57u, c[2]), lo1 = 0xCD9E8D57u * c[2];
    const uint32_t n0 = hi1 ^ c[1] ^ k0, n2 = hi0 ^ c[3] ^ k1;
    c[0] = n0;
    c[1] = lo1;
    c[2] = n2;
    c[3] = lo0;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
}

static __device__ __forceinline__ uint32_t boot_draw(uint64_t seed, int rep, uint64_t gidx,
                                                     uint32_t stream) {
  uint32_t c[4] = {(uint32_t)gidx, (uint32_t)(gidx >> 32), (uint32_t)rep, stream};
  philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
  return c[0];
}

// one event word decoded: span-1 address parts and the histogram addresses
struct EvDec {
  size_t addr;   // bin of the output sinogram
  int aw, an, w, si, sis;
  bool valid, prompt;
};

static __device__ __forceinline__ EvDec decode_event(int word, const HistLUT &slut, int span) {
  EvDec e;
  const int val = word & 0x3fffffff;
  e.si = val / NB_NSBINANG;
  e.valid = word > 0 && e.si < NB_NSN1;
  e.prompt = (word >> 30) == 1;
  e.aw = e.an = e.w = e.sis = 0;
  e.addr = 0;
  if (e.valid) {
    e.aw = val - e.si * NB_NSBINANG;
    e.an = e.aw / NB_NSBINS;
    e.w = e.aw - e.an * NB_NSBINS;
    e.sis = slut.sn1_ssrb[e.si];
    if (span == 1)
      e.addr = (size_t)val;
    else if (span == 11)
      e.addr = (size_t)slut.sn1_sn11[e.si] * NB_NSBINANG + e.aw;
    else
      e.addr = (size_t)e.sis * NB_NSBINANG + e.aw;
  }
  return e;
}

// Add a warp's per-second sums (held per replicate in shared memory) to the global
// per-second counters and clear them.  Lane l handles replicates l, l + 32, ...
static __device__ __forceinline__ void flush_seconds(const HistArgs &a, uint32_t *acc, int sec,
                                                     int lane) {
  __syncwarp();
  if (sec >= 0) {
    for (int r = lane; r < a.nrep; r += 32) {
      uint32_t *q = acc + 3 * r;
      const uint32_t pd = q[0], sz = q[1], sd = q[2];
      const uint32_t sp = pd;
      const size_t o = (size_t)r * a.nitag + sec;
      if (sp) {
        atomicAdd(a.phc + o, sp);
        atomicAdd((uint32_t *)a.zM + o, sp);
        atomicAdd((uint32_t *)a.zR + o, sz);
      }
      if (sd) atomicAdd(a.dhc + o, sd);
      q[0] = q[1] = q[2] = 0;
    }
  }
  __syncwarp();
}

// A step's per-second sums of replicate r: into the warp's accumulators when the step lies
// in one second (`uni`), else one global atomic per distinct second of the step.
static __device__ __forceinline__ void second_sums(const HistArgs &a, uint32_t *acc, int r,
                                                   bool uni, bool ok, int itag, uint32_t p_n,
                                                   uint32_t d_n, uint32_t zr, int lane) {
  if (uni) {
    // the step's prompts and delayeds (each <= 31 x 32 < 2^10) and ring sums (SSRB index
    // <= 126, <= 126 x 32 < 2^12) share one 32-bit reduction
    const uint32_t s = __reduce_add_sync(0xffffffffu, p_n | (d_n << 10) | (zr << 20));
    if (lane == 0) {
      acc[3 * r] += s & 0x3FFu;
      acc[3 * r + 1] += s >> 20;
      acc[3 * r + 2] += (s >> 10) & 0x3FFu;
    }
    return;
  }
  const unsigned grp = __match_any_sync(0xffffffffu, ok ? itag : -1);
  if (ok) {
    const uint32_t sp = __reduce_add_sync(grp, p_n);
    const uint32_t sd = __reduce_add_sync(grp, d_n);
    const uint32_t sz = __reduce_add_sync(grp, zr);
    if (lane == __ffs(grp) - 1) {
      const size_t o = (size_t)r * a.nitag + itag;
      if (sp) {
        atomicAdd(a.phc + o, sp);
        atomicAdd((uint32_t *)a.zM + o, sp);
        atomicAdd((uint32_t *)a.zR + o, sz);
      }
      if (sd) atomicAdd(a.dhc + o, sd);
    }
  }
}

// Slab records: a warp keeps, per slab, up to NB_SLAB_CW records in shared memory (wcnt[s]
// of them in wbuf[s][.]) and writes a slab's records out as one coalesced store at its
// write position wpos[s] in its own region of the slab.  Whole-warp calls; `lim` is the
// region's end (the regions are sized by a count of every event word of the warp's
// slices, so the records always fit; the bound only guards the store).
static __device__ __forceinline__ void slab_flush(const HistArgs &a, unsigned *wcnt,
                                                  unsigned *wpos, const uint32_t *wbuf, int s,
                                                  int lane, int gw) {
  __syncwarp();
  const unsigned c = wcnt[s];
  if (c) {
    const unsigned base = wpos[s];
    const unsigned lim = a.roff[(size_t)s * a.nwst + gw + 1];
    // streaming store: the records are read once, by k_slab_add, and should not push the
    // SSRB counters this launch updates out of L2
    if ((unsigned)lane < c && base + lane < lim) __stcs(a.rec + base + lane, wbuf[s * NB_SLAB_CW + lane]);
    __syncwarp();
    if (lane == 0) {
      wcnt[s] = 0;
      wpos[s] = base + c;
    }
  }
  __syncwarp();
}

static __device__ __forceinline__ void slab_stage(const HistArgs &a, unsigned *wcnt,
                                                  unsigned *wpos, uint32_t *wbuf, bool has,
                                                  size_t addr, bool prompt, int lane, int gw) {
  if (__ballot_sync(0xffffffffu, has) == 0) return;
  const int s = has ? (int)(addr >> NB_SLAB_SHIFT) : -1;
  const unsigned grp = __match_any_sync(0xffffffffu, s);
  const unsigned gsz = __popc(grp);
  const bool leader = has && lane == __ffs(grp) - 1;
  // slabs whose staged records and this step's would not fit are written out first
  unsigned fm = __ballot_sync(0xffffffffu, leader && wcnt[s] + gsz > NB_SLAB_CW);
  while (fm) {
    const int l = __ffs(fm) - 1;
    fm &= fm - 1;
    slab_flush(a, wcnt, wpos, wbuf, __shfl_sync(0xffffffffu, s, l), lane, gw);
  }
  if (has) {
    const unsigned c = wcnt[s];
    const unsigned rank = __popc(grp & ((1u << lane) - 1u));
    wbuf[s * NB_SLAB_CW + c + rank] =
        (uint32_t)(addr & ((1ull << NB_SLAB_SHIFT) - 1)) | (prompt ? 0u : 0x80000000u);
  }
  __syncwarp();
  if (leader) wcnt[s] += gsz;
  __syncwarp();
}

// Persistent: every warp takes the next thread slice from a.next_slice until none is left.
// Dynamic shared memory: 3 x nrep uint32 per warp (per-second prompt, ring-sum and
// delayed accumulators of the second the warp is in).
// (Held to 64 registers for a fourth block per SM it ran 1.7% slower: 4.20 vs 4.13 ms at
// span 11, 6% more instructions.  A copy specialised for one histogram without bootstrap
// -- 32 registers, 6 blocks per SM, 28% fewer instructions -- was slower too, 4.23 ms: the
// launch waits on its L2 atomics, not on issue.)
__global__ void __launch_bounds__(256) k_hist(const HistArgs a) {
  __shared__ HistLUT slut;
  __shared__ uint64_t s_thr[32];
  extern __shared__ uint32_t s_acc[];
  for (int i = threadIdx.x; i < (int)(sizeof(HistLUT) / 4); i += blockDim.x)
    reinterpret_cast<int *>(&slut)[i] = reinterpret_cast<const int *>(a.lut)[i];
  if (threadIdx.x < 32) s_thr[threadIdx.x] = a.thr[threadIdx.x];
  // the first eight Poisson thresholds in registers, less one: x >= thr  <=>  x > thr - 1,
  // and a threshold saturated at 2^32 becomes 0xFFFFFFFF, which no 32-bit uniform exceeds
  // (thresholds are ceilings of positive CDF values, so at least 1; the loop over the
  // shared copy handles a zero).  The first four decide almost every draw, the next four
  // nearly all the rest.
  const bool fast = a.thr[0] >= 1;
  const uint4 t4 = make_uint4((uint32_t)(a.thr[0] - 1), (uint32_t)(a.thr[1] - 1),
                              (uint32_t)(a.thr[2] - 1), (uint32_t)(a.thr[3] - 1));
  const uint4 t8 = make_uint4((uint32_t)(a.thr[4] - 1), (uint32_t)(a.thr[5] - 1),
                              (uint32_t)(a.thr[6] - 1), (uint32_t)(a.thr[7] - 1));
  const int lane = threadIdx.x & 31;
  uint32_t *acc = s_acc + (size_t)(threadIdx.x >> 5) * 3 * a.nrep;
  for (int r = lane; r < 3 * a.nrep; r += 32) acc[r] = 0;
  // bulk mode: NB_HIST_ROWS staging rows of rblk weights per thread, after the
  // accumulators (both offsets are multiples of 16 bytes, as the bulk copy needs)
  uint32_t *const stg =
      s_acc + (size_t)8 * 3 * a.nrep + (size_t)threadIdx.x * hist_row_stride(a.rblk);
  // slab records (no bulk staging then): per warp nslab counts, nslab write positions and
  // nslab x CW records
  unsigned *const wcnt =
      s_acc + (size_t)8 * 3 * a.nrep + (size_t)(threadIdx.x >> 5) * a.nslab * (NB_SLAB_CW + 2);
  unsigned *const wpos = wcnt + a.nslab;
  uint32_t *const wbuf = wpos + a.nslab;
  const int gw = (int)(blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5));
  int sl_next = gw;  // fixed slice assignment in slab mode
  if (a.rec)
    for (int s = lane; s < a.nslab; s += 32) {
      wcnt[s] = 0;
      wpos[s] = a.roff[(size_t)s * a.nwst + gw];
    }
  int par = 0;  // bulk mode: the staging row of the step
  __syncthreads();

  const int nslices = a.nchnk * NB_TOTHRDS;
  // replicate / bin strides of the two large counter arrays
  // replicate / bin strides of the sinogram counters, the delayed slot offset and shift
  const size_t pstr_r = a.unp ? 1 : a.nbins, pstr_b = a.unp ? 2 * (size_t)a.rblk : 1;
  const size_t doff = a.unp ? (size_t)a.rblk : 0;
  const int dshift = a.unp ? 0 : 16;
  const size_t sstr_r = (size_t)NB_SEG0 * NB_NSBINANG;
  for (;;) {
    int sl = 0;
    if (a.rec) {
      sl = sl_next;
      sl_next += a.nwst;
    } else {
      if (lane == 0) sl = (int)atomicAdd(a.next_slice, 1u);
      sl = __shfl_sync(0xffffffffu, sl, 0);
    }
    if (sl >= nslices) break;
    const int n = sl / NB_TOTHRDS, idx = sl - n * NB_TOTHRDS;
    const int64_t off = a.atag[n];
    const int elm = a.e4c[n], e4t = a.e4t[n];
    int64_t s0, s1;
    if (idx == NB_TOTHRDS - 1) {
      s1 = off + elm;
      s0 = off + (int64_t)(NB_TOTHRDS - 1) * e4t;
    } else {
      s1 = off + (int64_t)(idx + 1) * e4t;
      s0 = off + (int64_t)idx * e4t;
    }
    if (s1 > off + elm) s1 = off + elm;
    if (s0 >= s1) continue;

    // initial second: first time tag in [s0, s1-1) (hst.cu:84-100)
    int cur = a.nitag, curu = 0;
    for (int64_t base = s0; base < s1 - 1; base += 32) {
      const int64_t i = base + lane;
      const int wd = (i < s1 - 1) ? a.lm[i] : 0;
      const unsigned m = __ballot_sync(0xffffffffu, (wd >> 29) == -4);
      if (m) {
        const int src = __ffs(m) - 1;
        const int tv = (__shfl_sync(0xffffffffu, wd, src) & 0x1fffffff) - a.toff;
        cur = tv / NB_ITIME;
        curu = tv - cur * NB_ITIME;
        break;
      }
    }
    const int64_t slen = s1 - s0;
    int acc_sec = -1;  // the second whose sums `acc` holds (warp-uniform)

    // the next step's words are loaded one step ahead (streaming loads: the stream is read
    // once and should not displace the counters from L2)
    int nxt = s0 + lane < s1 ? __ldcs(a.lm + s0 + lane) : 0;
    for (int64_t base = s0; base < s1; base += 32) {
      // a slice is dead once its current second leaves the window (hst.cu:135)
      if (!(cur >= a.tstart && cur < a.tstop)) break;
      const int64_t i = base + lane;
      const bool inb = i < s1;
      const int word0 = nxt;  // 0 past the slice end
      nxt = i + 32 < s1 ? __ldcs(a.lm + i + 32) : 0;
      const bool istag = inb && (word0 >> 29) == -4;
      const unsigned tmask = __ballot_sync(0xffffffffu, istag);
      const int tval = istag ? (word0 & 0x3fffffff) - a.toff : 0;
      const int titag = tval / NB_ITIME;
      // the second in force when this word is processed
      const unsigned before = tmask & ((1u << lane) - 1u);
      const int srcl = before ? 31 - __clz(before) : -1;
      const int my_itag_t = __shfl_sync(0xffffffffu, titag, srcl < 0 ? 0 : srcl);
      const int my_itagu_t = __shfl_sync(0xffffffffu, tval - titag * NB_ITIME, srcl < 0 ? 0 : srcl);
      const int itag = srcl < 0 ? cur : my_itag_t;
      const int itagu = srcl < 0 ? curu : my_itagu_t;
      const bool okw = itag >= a.tstart && itag < a.tstop;
      const unsigned bad = __ballot_sync(0xffffffffu, inb && !okw);
      const bool live = inb && (bad == 0 || lane < __ffs(bad) - 1);
      // carry the second to the next step
      const unsigned livetags = tmask & __ballot_sync(0xffffffffu, live);
      if (livetags) {
        const int last = 31 - __clz(livetags);
        cur = __shfl_sync(0xffffffffu, titag, last);
        curu = __shfl_sync(0xffffffffu, tval - titag * NB_ITIME, last);
      }
      if (bad) cur = -2147483647;  // dead from the first out-of-window word on

      // ---- singles (hst.cu:215-235), in word order within the warp ----
      {
        const bool issgl = live && (word0 >> 29) == -3;
        unsigned sm = __ballot_sync(0xffffffffu, issgl);
        while (sm) {
          const int L = __ffs(sm) - 1;
          sm &= sm - 1;
          if (lane == L) {
            const unsigned ibck = (unsigned)((word0 & 0x1fffffff) >> 19);
            if (ibck < NB_NBUCKTS) {
              for (int r = 0; r < a.nrep; r++) {
                uint32_t *bk = a.bck + (size_t)r * 2 * NB_NBUCKTS * a.nitag;
                const size_t b0 = ibck + (size_t)NB_NBUCKTS * itag;
                const size_t b1 = b0 + (size_t)NB_NBUCKTS * a.nitag;
                atomicAdd(bk + b0, (uint32_t)(word0 & 0x0007ffff) << 3);
                const uint32_t prev =
                    atomicAdd(bk + b1, (uint32_t)((word0 & 0x0007ffff) > 0) << 30);
                const uint32_t now = prev + ((uint32_t)((word0 & 0x0007ffff) > 0) << 30);
                atomicAdd(bk + b1, now == 0 ? (uint32_t)itagu : (uint32_t)itagu << 10);
              }
            }
          }
          __syncwarp();
        }
      }

      // ---- events ----
      const bool evw = live && word0 > 0;
      const unsigned evm = __ballot_sync(0xffffffffu, evw);
      if (evm == 0) continue;
      // the step's second, if all its event words share one (almost every step: a
      // second spans ~1e5 words); the per-second sums then go to the warp's accumulators
      const int sec0 = __shfl_sync(0xffffffffu, itag, __ffs(evm) - 1);
      const bool uni = __all_sync(0xffffffffu, !evw || itag == sec0);
      if (uni && sec0 != acc_sec) {
        flush_seconds(a, acc, acc_sec, lane);
        acc_sec = sec0;
      }
      if (a.btp != 1) {
        // one decode per word; per replicate only its weight N and the counter updates
        const EvDec e = decode_event(word0, slut, a.span);
        const bool okb = evw && e.valid;
        const size_t pbin = e.addr * pstr_b + (e.prompt ? 0 : doff);
        const size_t sbin = (size_t)e.sis * NB_NSBINANG + e.aw;
        const bool pv = okb && e.prompt && (e.an == 0 || e.an == 126) && itag < NB_MXNITAG;
        const size_t pvo = (size_t)(itag >> 2) * NB_SEG0 * NB_NSBINS + e.sis * NB_NSBINS + e.w;
        int f0 = 0, f1 = 0;
        if (okb && !e.prompt) {
          const short2 cc = a.s2cF[e.an + NB_NSANGLES * e.w];
          f0 = NB_NCRS * slut.sn1_rno[2 * e.si] + cc.x;
          f1 = NB_NCRS * slut.sn1_rno[2 * e.si + 1] + cc.y;
        }
        // the sinogram update of either kind, and the per-kind extra counters
        const int pshift = e.prompt ? 0 : dshift;
        uint32_t *const ps0 = a.psino + pbin;
        uint32_t *const ss0 = a.ssrb + sbin;
        uint32_t blk[4] = {0u, 0u, 0u, 0u};
        int qblk = -1;
        // the row's previous bulk add (two steps back) must have read it.  (Four rows with
        // one bulk group per two steps, waiting half as often, ran 22% slower.)
        uint32_t *const row = stg + (par & 1) * a.rblk;
        if (a.bulk) nb_bulk_wait_read<1>();
        bool any = false;
        for (int r = 0; r < a.nrep; r++) {
          const int rep = a.rep0 + r;
          uint32_t N = 1;
          if (a.btp == 2) {
            // N ~ Poisson: the number of inverse-CDF thresholds at or below the uniform,
            // output rep % 4 of the Philox block (word index, rep / 4)
            if ((rep >> 2) != qblk) {
              qblk = rep >> 2;
              blk[0] = (uint32_t)i;
              blk[1] = (uint32_t)((uint64_t)i >> 32);
              blk[2] = (uint32_t)qblk;
              blk[3] = 0u;
              philox4x32_10(blk, (uint32_t)a.seed, (uint32_t)(a.seed >> 32));
            }
            const int j = rep & 3;
            const uint32_t x = j == 0 ? blk[0] : j == 1 ? blk[1] : j == 2 ? blk[2] : blk[3];
            uint32_t k;
            if (fast) {
              k = (uint32_t)(x > t4.x) + (uint32_t)(x > t4.y) + (uint32_t)(x > t4.z) +
                  (uint32_t)(x > t4.w);
              if (k == 4) {
                k += (uint32_t)(x > t8.x) + (uint32_t)(x > t8.y) + (uint32_t)(x > t8.z) +
                     (uint32_t)(x > t8.w);
                if (k == 8)
                  while (k < 32 && (uint64_t)x >= s_thr[k]) k++;
              }
            } else {
              k = 0;
              while (k < 32 && (uint64_t)x >= s_thr[k]) k++;
            }
            N = k;
          }
          const bool ok = okb && N > 0 && N < 32;
          if (a.bulk) {
            row[r] = ok ? N : 0u;
            any |= ok;
          }
          if (ok) {
            if (!a.bulk && !a.rec) atomicAdd(ps0 + (size_t)r * pstr_r, N << pshift);
            if (e.prompt) {
              if (!a.unp) atomicAdd(ss0 + (size_t)r * sstr_r, N);
              if (pv) atomicAdd(a.pvs + (size_t)r * a.sne + pvo, N << ((e.an == 126) * 8));
            } else {
              uint32_t *fn = a.fan + (size_t)r * NB_NRINGS * NB_NCRS;
              atomicAdd(fn + f0, N);
              atomicAdd(fn + f1, N);
            }
          }
          // centre of mass: zR adds the prompt's SSRB index once, zM its weight (hst.cu:176-178)
          const uint32_t nn = ok ? N : 0u;
          second_sums(a, acc, r, uni, ok, itag, e.prompt ? nn : 0u, e.prompt ? 0u : nn,
                      (ok && e.prompt) ? (uint32_t)e.sis : 0u, lane);
        }
        if (a.bulk) {
          // all replicates of the event in one L2 reduction of the bin's replicate block
          for (int r = a.nrep; r < a.rblk; r++) row[r] = 0u;
          if (any) {
            nb_fence_proxy_async_smem();
            nb_bulk_reduce_add_u32(ps0, row, 4u * (uint32_t)a.rblk);
          }
          nb_bulk_commit();  // one group per step, empty or not: groups alternate rows
          par ^= 1;
        }
        // slab records: one histogram, weight 1 (nb_hist sets rec only then)
        if (a.rec) slab_stage(a, wcnt, wpos, wbuf, okb, e.addr, e.prompt, lane, gw);
        continue;
      }
      // btp = 1: each replicate replaces the word by a draw from the slice
      for (int r = 0; r < a.nrep; r++) {
        const int rep = a.rep0 + r;
        int word = word0;
        uint32_t N = 1;
        if (evw) {
          bool got = false;
          for (uint32_t jd = 0; jd < 64 && !got; jd++) {
            const uint32_t x = boot_draw(a.seed, rep, (uint64_t)i, 1 + jd);
            const int64_t bi = (int64_t)(((uint64_t)x * (uint64_t)slen) >> 32);
            const int cand = a.lm[s0 + bi];
            if (cand > 0) {
              word = cand;
              got = true;
            }
          }
          if (!got) N = 0;
        }
        const EvDec e = decode_event(word, slut, a.span);
        const bool ok = evw && e.valid && N > 0;
        uint32_t p_n = 0, d_n = 0, zr = 0;
        if (ok) {
          uint32_t *ps = a.psino + (size_t)r * pstr_r + e.addr * pstr_b;
          if (e.prompt) {
            p_n = N;
            zr = (uint32_t)e.sis;
            if (!a.unp)
              atomicAdd(a.ssrb + (size_t)r * sstr_r + (size_t)e.sis * NB_NSBINANG + e.aw, N);
            atomicAdd(ps, N);
            if ((e.an == 0 || e.an == 126) && itag < NB_MXNITAG)
              atomicAdd(a.pvs + (size_t)r * a.sne + (size_t)(itag >> 2) * NB_SEG0 * NB_NSBINS +
                            e.sis * NB_NSBINS + e.w,
                        N << ((e.an == 126) * 8));
          } else {
            d_n = N;
            atomicAdd(ps + doff, N << dshift);
            const short2 cc = a.s2cF[e.an + NB_NSANGLES * e.w];
            uint32_t *fn = a.fan + (size_t)r * NB_NRINGS * NB_NCRS;
            atomicAdd(fn + NB_NCRS * slut.sn1_rno[2 * e.si] + cc.x, N);
            atomicAdd(fn + NB_NCRS * slut.sn1_rno[2 * e.si + 1] + cc.y, N);
          }
        }
        second_sums(a, acc, r, uni, ok, itag, p_n, d_n, zr, lane);
      }
    }
    flush_seconds(a, acc, acc_sec, lane);
  }
  if (a.rec)
    for (int s = 0; s < a.nslab; s++) slab_flush(a, wcnt, wpos, wbuf, s, lane, gw);
  if (a.bulk) nb_bulk_wait_all<0>();
}

// Unpacked scratch [bin][2][rblk] (prompts, delayeds) added into the caller's packed
// [nrep][bin] counters -- prompts + 65536 x delayeds, the reference's packed uint32 sum
// (hst.cu:167,192), wrap-around included -- and the SSRB counters summed from the prompts
// in the same pass.  Every output sinogram belongs to one SSRB sinogram (its rings' sum),
// so SSRB bin (k, aw) of replicate r adds the prompts of bin aw of the sinograms listed in
// lst[off[k] .. off[k+1]); the lists partition the output sinograms, so walking them visits
// every scratch bin once.  A warp takes 32 consecutive SSRB bins and one group of four
// replicates, 4g .. 4g+3 (rblk = 4 ngrp), the ngrp warps of the other groups of the same
// bins next to it: the sinogram stores of a warp are whole 128-byte lines, and the
// 16-byte pieces of a bin's block that one warp skips are read by its neighbours while the
// lines are still in L1 (cached loads; streaming loads, or one thread per bin and group,
// measured 1.2 and 0.9 ms slower at 10 replicates x 72.6M bins).
__global__ void k_pack_ssrb(uint32_t *__restrict__ dst, uint32_t *__restrict__ ssrb,
                            const uint32_t *__restrict__ src, const int *__restrict__ off,
                            const int16_t *__restrict__ lst, size_t nbins, int nrep, int rblk) {
  const int ngrp = rblk >> 2;
  const size_t nss = (size_t)NB_SEG0 * NB_NSBINANG;
  const size_t nt = ((nss + 31) / 32) * 32 * ngrp;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < nt;
       t += (size_t)gridDim.x * blockDim.x) {
    const size_t wid = t >> 5;
    const size_t i = (wid / ngrp) * 32 + (t & 31);
    const int g = (int)(wid % ngrp);
    if (i >= nss) continue;
    const int k = (int)(i / NB_NSBINANG), aw = (int)(i - (size_t)k * NB_NSBINANG);
    const int r0 = 4 * g;
    uint32_t s0 = 0, s1 = 0, s2 = 0, s3 = 0;
    for (int j = off[k]; j < off[k + 1]; j++) {
      const size_t b = (size_t)lst[j] * NB_NSBINANG + aw;
      const uint32_t *q = src + b * 2 * rblk + r0;
      const uint4 p = __ldg(reinterpret_cast<const uint4 *>(q));
      const uint4 d = __ldg(reinterpret_cast<const uint4 *>(q + rblk));
      uint32_t *o = dst + (size_t)r0 * nbins + b;
      o[0] += p.x + (d.x << 16);
      if (r0 + 1 < nrep) o[nbins] += p.y + (d.y << 16);
      if (r0 + 2 < nrep) o[2 * nbins] += p.z + (d.z << 16);
      if (r0 + 3 < nrep) o[3 * nbins] += p.w + (d.w << 16);
      s0 += p.x;
      s1 += p.y;
      s2 += p.z;
      s3 += p.w;
    }
    uint32_t *o = ssrb + (size_t)r0 * nss + i;
    o[0] += s0;
    if (r0 + 1 < nrep) o[nss] += s1;
    if (r0 + 2 < nrep) o[2 * nss] += s2;
    if (r0 + 3 < nrep) o[3 * nss] += s3;
  }
}

// Slab regions: warp w of the nwst that k_hist launches counts, per slab, the event words
// of the slices k_hist gives it (w, w + nwst, ...) -- every event word with a valid
// address, whatever its time, so that its records always fit -- into cnt[slab][w].
__global__ void __launch_bounds__(256) k_slab_count(const HistArgs a, unsigned *__restrict__ cnt) {
  __shared__ unsigned h[8][64];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int gw = (int)(blockIdx.x * 8 + warp);
  for (int s = lane; s < 64; s += 32) h[warp][s] = 0;
  __syncwarp();
  const int nslices = a.nchnk * NB_TOTHRDS;
  for (int sl = gw; sl < nslices; sl += a.nwst) {
    const int n = sl / NB_TOTHRDS, idx = sl - n * NB_TOTHRDS;
    const int64_t off = a.atag[n];
    const int elm = a.e4c[n], e4t = a.e4t[n];
    int64_t s0 = off + (int64_t)idx * e4t, s1;
    if (idx == NB_TOTHRDS - 1) {
      s1 = off + elm;
      s0 = off + (int64_t)(NB_TOTHRDS - 1) * e4t;
    } else {
      s1 = off + (int64_t)(idx + 1) * e4t;
    }
    if (s1 > off + elm) s1 = off + elm;
    // eight steps of 32 words per iteration, their loads issued together
    for (int64_t base = s0; base < s1; base += 256) {
      int w[8];
#pragma unroll
      for (int k = 0; k < 8; k++) {
        const int64_t i = base + 32 * k + lane;
        w[k] = i < s1 ? __ldcs(a.lm + i) : 0;
      }
#pragma unroll
      for (int k = 0; k < 8; k++) {
        int s = -1;
        if (w[k] > 0) {
          const int val = w[k] & 0x3fffffff;
          const int si = val / NB_NSBINANG;
          if (si < NB_NSN1) {
            const size_t addr = a.span == 1 ? (size_t)val
                                            : (size_t)a.lut->sn1_sn11[si] * NB_NSBINANG +
                                                  (val - si * NB_NSBINANG);
            s = (int)(addr >> NB_SLAB_SHIFT);
          }
        }
        const unsigned grp = __match_any_sync(0xffffffffu, s);
        if (s >= 0 && lane == __ffs(grp) - 1) atomicAdd(&h[warp][s], (unsigned)__popc(grp));
      }
    }
  }
  __syncwarp();
  for (int s = lane; s < a.nslab; s += 32) cnt[(size_t)s * a.nwst + gw] = h[warp][s];
}

// Region starts: the exclusive prefix sum of cnt[n] into off[n], off[n] = the total; one
// block of 1024 threads, each over a contiguous share.
__global__ void k_slab_scan(const unsigned *__restrict__ cnt, unsigned *__restrict__ off,
                            int n) {
  __shared__ unsigned part[1024];
  const int t = threadIdx.x;
  const int per = (n + 1023) / 1024, lo = min(n, t * per), hi = min(n, lo + per);
  unsigned sum = 0;
  for (int i = lo; i < hi; i++) sum += cnt[i];
  part[t] = sum;
  __syncthreads();
  if (t == 0) {
    unsigned acc = 0;
    for (int k = 0; k < 1024; k++) {
      const unsigned v = part[k];
      part[k] = acc;
      acc += v;
    }
    off[n] = acc;
  }
  __syncthreads();
  unsigned acc = part[t];
  for (int i = lo; i < hi; i++) {
    off[i] = acc;
    acc += cnt[i];
  }
}

// Count slab s's records into the packed sinogram: prompt +1, delayed +65536 (the
// reference's packed uint32 sum, hst.cu:167,192).  One slab per launch, so the counters
// being updated stay in L2.  The slab's records lie in [off[s nwst], off[(s+1) nwst]); the
// unused tail of each warp's region holds 0xFFFFFFFF (no record has all bits set).
__global__ void k_slab_add(uint32_t *__restrict__ psino, const uint32_t *__restrict__ rec,
                           const unsigned *__restrict__ off, int s, int nwst) {
  const unsigned b0 = off[(size_t)s * nwst], b1 = off[(size_t)(s + 1) * nwst];
  uint32_t *const ps = psino + ((size_t)s << NB_SLAB_SHIFT);
  for (unsigned i = b0 + blockIdx.x * blockDim.x + threadIdx.x; i < b1;
       i += gridDim.x * blockDim.x) {
    const uint32_t r = __ldcs(rec + i);
    if (r != 0xFFFFFFFFu)
      atomicAdd(ps + (r & ((1u << NB_SLAB_SHIFT) - 1)), (r >> 31) ? 65536u : 1u);
  }
}

// ---------------------------------------------------------------------------------------
// host: chunk plan (lmaux.cu:17-270)
// ---------------------------------------------------------------------------------------
extern "C" int nb_lm_plan(const int32_t *lm, int64_t ele, int t0, int t1, int cap, int64_t *atag,
                          int *ele4chnk, int *ele4thrd, int *nchnk, int *toff, int *nitag,
                          int *tstart, int *tstop) {
  NB_REQUIRE(lm && atag && ele4chnk && ele4thrd && nchnk && toff && nitag && tstart && tstop,
             "nb_lm_plan: NULL argument");
  NB_REQUIRE(ele > 0, "nb_lm_plan: empty stream");
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
  if (i0 < 0) {
    nb_set_error_msg("nb_lm_plan: no time tag in the list-mode stream");
    return NB_ERR_DATA;
  }
  const int first = lm[i0] & 0x1fffffff, last = lm[i1] & 0x1fffffff;
  if (!(first < last)) {
    nb_set_error_msg("nb_lm_plan: first time tag %d is not before the last %d", first, last);
    return NB_ERR_DATA;
  }
  const int tof = first;
  const int nit = ((last - tof) + NB_ITIME - 1) / NB_ITIME;
  std::vector<int64_t> A(1, 0), Bt(1, 0);
  std::vector<int> E, ET;
  while ((ele - A.back()) > (int64_t)NB_ELECHNK) {
    const int64_t prev = A.back();
    int64_t found = -1;
    for (int64_t pos = prev + NB_ELECHNK - 1; pos > prev; pos--) {
      const int wd = lm[pos];
      if ((wd >> 29) == -4 && ((wd & 0x1fffffff) % NB_BTPTIME) == 0) {
        found = pos;
        break;
      }
    }
    if (found < 0) {
      nb_set_error_msg("nb_lm_plan: no 100-ms time tag within %d words after word %lld",
                       NB_ELECHNK, (long long)prev);
      return NB_ERR_DATA;
    }
    Bt.push_back((int64_t)((lm[found] & 0x1fffffff) - tof));
    A.push_back(found);
    E.push_back((int)(found - prev));
    ET.push_back((int)((found - prev + NB_TOTHRDS - 1) / NB_TOTHRDS));
  }
  Bt.push_back((int64_t)(last - tof + 1));
  const int64_t prev = A.back();
  A.push_back(ele);
  E.push_back((int)(ele - prev));
  ET.push_back((int)((ele - prev + NB_TOTHRDS - 1) / NB_TOTHRDS));
  const int nch = (int)E.size();
  int ts = t0, te = t1;
  if (ts == te) {
    ts = 0;
    te = nit;
  }
  int n0 = -1, n1 = -1, newn = 0;
  for (int n = 0; n < nch; n++)
    if (ts <= (Bt[n + 1] / NB_ITIME) && (Bt[n] / NB_ITIME) < te) {
      if (n0 == -1) n0 = n;
      n1 = n;
      newn++;
    }
  if (newn + 1 > cap) {
    nb_set_error_msg("nb_lm_plan: capacity %d too small for %d chunks", cap, newn);
    return NB_ERR_ARG;
  }
  int nn = 0;
  if (newn > 0) {
    for (int n = n0; n <= n1; n++) {
      atag[nn] = A[n];
      ele4chnk[nn] = E[n];
      ele4thrd[nn] = ET[n];
      nn++;
    }
    atag[nn] = A[n1 + 1];
  }
  *nchnk = newn;
  *toff = tof;
  *nitag = nit;
  *tstart = ts;
  *tstop = te;
  return NB_OK;
}

static void poisson_thresholds(double lam, uint64_t thr[32]) {
  double pmf = exp(-lam), cdf = 0;
  for (int n = 0; n < 32; n++) {
    if (n > 0) pmf = pmf * lam / (double)n;
    cdf += pmf;
    const double t = ceil(cdf * 4294967296.0);
    thr[n] = t >= 4294967296.0 ? 4294967296ull : (uint64_t)t;
  }
}

// Stream-ordered scratch of the histogrammer comes from its own memory pool per device,
// which keeps freed memory for the next call (the replicate-interleaved counters of a
// bootstrap run are gigabytes; re-mapping them on every call would cost more than the
// histogram).  The pool is created on first use and lives until the process exits.
#include <mutex>
static std::mutex g_pool_mu;
static cudaMemPool_t g_pool[64] = {};

static cudaError_t hist_pool(cudaMemPool_t *out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lk(g_pool_mu);
  if (!g_pool[dev]) {
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t p = nullptr;
    e = cudaMemPoolCreate(&p, &props);
    if (e != cudaSuccess) return e;
    uint64_t keep = ~0ull;
    e = cudaMemPoolSetAttribute(p, cudaMemPoolAttrReleaseThreshold, &keep);
    if (e != cudaSuccess) return e;
    g_pool[dev] = p;
  }
  *out = g_pool[dev];
  return cudaSuccess;
}

extern "C" int nb_hist_trim(void) {
  cudaMemPool_t pool = nullptr;
  NB_CUDA(hist_pool(&pool));
  NB_CUDA(cudaMemPoolTrimTo(pool, 0));
  return NB_OK;
}

// dynamic shared memory of a k_hist launch: per-second sums, bulk staging rows, slab records
static size_t hist_dyn(const HistArgs &a, bool slab) {
  return (size_t)8 * 3 * a.nrep * sizeof(uint32_t) +
         (a.bulk ? (size_t)256 * hist_row_stride(a.rblk) * sizeof(uint32_t) : 0) +
         (slab ? (size_t)8 * a.nslab * (NB_SLAB_CW + 2) * sizeof(uint32_t) : 0);
}

// 256-thread blocks of k_hist that fit on the current device at once
static cudaError_t hist_blocks(size_t dyn, int *blocks) {
  int dev = 0, nsm = 148, per_sm = 1;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  // static plus dynamic shared memory above 48 KB needs the kernel's opt-in
  if (dyn + sizeof(HistLUT) + 32 * sizeof(uint64_t) > 48 * 1024) {
    cudaError_t e =
        cudaFuncSetAttribute(k_hist, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn);
    if (e != cudaSuccess) return e;
  }
  cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_hist, 256, dyn);
  if (e != cudaSuccess) return e;
  *blocks = nsm * (per_sm > 0 ? per_sm : 1);
  return cudaSuccess;
}

// Launch the persistent histogram kernel: as many 256-thread blocks as fit on the device at
// once, each warp pulling thread slices from the counter `ctr` (zeroed here) -- or, with
// slab records, exactly a.nwst / 8 blocks taking their slices in the fixed order the
// regions were sized for.
static cudaError_t launch_hist(HistArgs &a, unsigned *ctr, cudaStream_t s) {
  cudaError_t e = cudaMemsetAsync(ctr, 0, sizeof(unsigned), s);
  if (e != cudaSuccess) return e;
  a.next_slice = ctr;
  const size_t dyn = hist_dyn(a, a.rec != nullptr);
  int blocks = 1;
  e = hist_blocks(dyn, &blocks);
  if (e != cudaSuccess) return e;
  const int nslices = a.nchnk * NB_TOTHRDS;
  if (a.rec)
    blocks = a.nwst / 8;
  else if (blocks > (nslices + 7) / 8)
    blocks = (nslices + 7) / 8;
  k_hist<<<blocks, 256, dyn, s>>>(a);
  return cudaGetLastError();
}

extern "C" int nb_hist(const int32_t *lm, int64_t ele, int nchnk, const int64_t *atag,
                       const int *ele4chnk, const int *ele4thrd, int toff, int nitag, int tstart,
                       int tstop, int span, int btp, double btprt, uint64_t seed, int rep0,
                       int nrep, const int16_t *sn1_sn11, const int16_t *sn1_ssrb,
                       const int16_t *sn1_rno, const int16_t *s2cF, uint32_t *psino,
                       uint32_t *ssrb, uint32_t *phc, uint32_t *dhc, int32_t *zR, int32_t *zM,
                       uint32_t *pvs, uint32_t *fan, uint32_t *bck, void *stream) {
  NB_RANGE("nb_hist");
  NB_REQUIRE(lm && atag && ele4chnk && ele4thrd, "nb_hist: NULL stream or plan");
  NB_REQUIRE(sn1_sn11 && sn1_ssrb && sn1_rno && s2cF, "nb_hist: NULL LUT");
  NB_REQUIRE(psino && ssrb && phc && dhc && zR && zM && pvs && fan && bck,
             "nb_hist: NULL output");
  NB_REQUIRE(span == 0 || span == 1 || span == 11, "nb_hist: span must be 0, 1 or 11");
  NB_REQUIRE(btp >= 0 && btp <= 2, "nb_hist: btp must be 0, 1 or 2");
  NB_REQUIRE(nrep >= 1 && nrep <= 1024 && nitag > 0 && nchnk >= 0, "nb_hist: bad sizes");
  NB_REQUIRE(!(btp == 2 && !(btprt > 0)), "nb_hist: btprt must be > 0");
  for (int n = 0; n < nchnk; n++) {
    NB_REQUIRE(atag[n] >= 0 && ele4chnk[n] >= 0 && atag[n] + ele4chnk[n] <= ele,
               "nb_hist: chunk outside the stream");
    NB_REQUIRE(ele4thrd[n] >= 0, "nb_hist: bad slice length");
  }
  for (int i = 0; i < NB_NSN1; i++)
    NB_REQUIRE(sn1_sn11[i] >= 0 && sn1_sn11[i] < NB_NSN11 && sn1_ssrb[i] >= 0 &&
                   sn1_ssrb[i] < NB_SEG0 && sn1_rno[2 * i] >= 0 && sn1_rno[2 * i] < NB_NRINGS &&
                   sn1_rno[2 * i + 1] >= 0 && sn1_rno[2 * i + 1] < NB_NRINGS,
               "nb_hist: axial LUT out of range");
  if (nchnk == 0) return NB_OK;
  cudaStream_t s = (cudaStream_t)stream;

  HistArgs a{};
  a.lm = lm;
  a.nchnk = nchnk;
  a.toff = toff;
  a.nitag = nitag;
  a.tstart = tstart;
  a.tstop = tstop;
  a.span = span;
  a.btp = btp;
  a.seed = seed;
  a.rep0 = rep0;
  a.nrep = nrep;
  poisson_thresholds(btp == 2 ? btprt : 1.0, a.thr);
  a.nbins = span == 1 ? 354033792ull : (span == 11 ? 72557856ull : (size_t)NB_SEG0 * NB_NSBINANG);
  const int tn = nitag > NB_MXNITAG ? NB_MXNITAG : nitag;
  a.sne = (size_t)((tn + 3) / 4) * NB_SEG0 * NB_NSBINS;
  a.psino = psino;
  a.ssrb = ssrb;
  a.phc = phc;
  a.dhc = dhc;
  a.zR = zR;
  a.zM = zM;
  a.pvs = pvs;
  a.fan = fan;
  a.bck = bck;

  // small device-side tables, the SSRB source lists and the work counter, stream-ordered
  HistLUT hl;
  memcpy(hl.sn1_sn11, sn1_sn11, sizeof(hl.sn1_sn11));
  memcpy(hl.sn1_ssrb, sn1_ssrb, sizeof(hl.sn1_ssrb));
  memcpy(hl.sn1_rno, sn1_rno, sizeof(hl.sn1_rno));
  // SSRB sinogram k gathers the output sinograms listed in lst[off[k] .. off[k+1]): span 11
  // its span-11 sinograms (each has one SSRB index), span 1 its span-1 sinograms, SSRB
  // mode itself
  const int nout = span == 11 ? NB_NSN11 : (span == 1 ? NB_NSN1 : NB_SEG0);
  std::vector<int> ssrb_of(nout, -1);
  for (int si = 0; si < NB_NSN1; si++) {
    const int so = span == 11 ? sn1_sn11[si] : (span == 1 ? si : sn1_ssrb[si]);
    const int k = span == 0 ? so : sn1_ssrb[si];
    NB_REQUIRE(ssrb_of[so] < 0 || ssrb_of[so] == k,
               "nb_hist: an output sinogram spans two SSRB sinograms");
    ssrb_of[so] = k;
  }
  // replicates are packed by walking these lists, which must then reach every sinogram
  if (nrep > 1)
    for (int so = 0; so < nout; so++)
      NB_REQUIRE(ssrb_of[so] >= 0, "nb_hist: an output sinogram lies in no SSRB sinogram");
  std::vector<int> soff(NB_SEG0 + 1, 0);
  std::vector<int16_t> slst;
  for (int k = 0; k < NB_SEG0; k++) {
    for (int so = 0; so < nout; so++)
      if (ssrb_of[so] == k) slst.push_back((int16_t)so);
    soff[k + 1] = (int)slst.size();
  }
  const size_t plan_bytes = (size_t)nchnk * (sizeof(int64_t) + 2 * sizeof(int));
  const size_t s2c_bytes = (size_t)NB_NSBINANG * sizeof(short2);
  const size_t ssl_bytes = sizeof(int) * soff.size() + sizeof(int16_t) * slst.size();
  const size_t tot = sizeof(HistLUT) + s2c_bytes + plan_bytes + ssl_bytes + 96;
  unsigned char *d = nullptr;
  cudaMemPool_t pool = nullptr;
  NB_CUDA(hist_pool(&pool));
  NB_CUDA(cudaMallocFromPoolAsync((void **)&d, tot, pool, s));
  std::vector<unsigned char> h(tot);
  size_t o = 0;
  memcpy(&h[o], &hl, sizeof(HistLUT));
  a.lut = (const HistLUT *)(d + o);
  o += sizeof(HistLUT);
  memcpy(&h[o], s2cF, s2c_bytes);
  a.s2cF = (const short2 *)(d + o);
  o += s2c_bytes;
  o = (o + 15) & ~(size_t)15;
  memcpy(&h[o], atag, sizeof(int64_t) * nchnk);
  a.atag = (const int64_t *)(d + o);
  o += sizeof(int64_t) * nchnk;
  memcpy(&h[o], ele4chnk, sizeof(int) * nchnk);
  a.e4c = (const int *)(d + o);
  o += sizeof(int) * nchnk;
  memcpy(&h[o], ele4thrd, sizeof(int) * nchnk);
  a.e4t = (const int *)(d + o);
  o += sizeof(int) * nchnk;
  o = (o + 15) & ~(size_t)15;
  memcpy(&h[o], soff.data(), sizeof(int) * soff.size());
  const int *d_soff = (const int *)(d + o);
  o += sizeof(int) * soff.size();
  memcpy(&h[o], slst.data(), sizeof(int16_t) * slst.size());
  const int16_t *d_slst = (const int16_t *)(d + o);
  o += sizeof(int16_t) * slst.size();
  o = (o + 15) & ~(size_t)15;
  unsigned *ctr = (unsigned *)(d + o);
  cudaError_t e = cudaMemcpyAsync(d, h.data(), o, cudaMemcpyHostToDevice, s);
  // replicates: the sinogram counters are histogrammed unpacked -- prompts and delayeds
  // of a bin in separate uint32s, the replicates of a bin side by side ([bin][2][nrep], so
  // one event's replicate updates share one or two 32-byte sectors) -- in a stream-ordered
  // scratch, then packed into the caller's sinograms, and the SSRB counters are summed
  // from the prompts instead of counted per event.  One histogram counts both directly
  // (an unpacked scratch would double its L2 footprint for less than it saves).
  // Replicates go through in chunks of at most NB_HIST_REPCHUNK, as equal as possible (the
  // staging rows of a chunk must fit in shared memory, and the scratch is sized for one).
  uint32_t *scr = nullptr;
  const int nrch = (nrep + NB_HIST_REPCHUNK - 1) / NB_HIST_REPCHUNK;
  const int rchunk = (nrep + nrch - 1) / nrch;
  const size_t scr_bytes = sizeof(uint32_t) * a.nbins * 2 * (size_t)((rchunk + 3) & ~3);
  if (e == cudaSuccess && nrep > 1) {
    e = cudaMallocFromPoolAsync((void **)&scr, scr_bytes, pool, s);
    if (e == cudaSuccess) {
      a.unp = 1;
      a.bulk = 1;
    }
  }
  // One histogram without bootstrap whose sinogram counters are larger than L2: its events
  // become slab records (sinogram bin and kind, 4 bytes each) and the counters are then
  // added one 64 MB slab at a time, so that every counter update hits L2 (random updates
  // of counters larger than L2 run at a sixth of the rate of L2-resident ones).  The
  // sums are integers, so the result is the same bit for bit.  Every warp of the
  // histogram launch writes its records into regions of its own, sized beforehand by a
  // count of the event words of the slices it will take.
  uint32_t *rec = nullptr;
  unsigned *rmeta = nullptr;
  const int nslab = (int)((a.nbins + (1ull << NB_SLAB_SHIFT) - 1) >> NB_SLAB_SHIFT);
  int64_t nwords = 0;
  for (int n = 0; n < nchnk; n++) nwords += ele4chnk[n];
  int dev = 0, nsm = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  // (Span 1 only: at span 11 the 290 MB of counters keep enough L2 hits that the direct
  // count, 4.5 ms for 2e8 events, beats count + records + slab passes, 6.3 ms.)
  if (e == cudaSuccess && nrep == 1 && btp == 0 && span == 1 && nslab > 1 && nslab <= 64 &&
      nwords > 0 && nwords < (int64_t)UINT32_MAX) {
    a.nslab = nslab;
    int blocks = 1;
    e = hist_blocks(hist_dyn(a, true), &blocks);
    a.nwst = blocks * 8;
    const size_t nreg = (size_t)nslab * a.nwst;
    if (e == cudaSuccess)
      e = cudaMallocFromPoolAsync((void **)&rmeta, sizeof(unsigned) * (2 * nreg + 1), pool, s);
    if (e == cudaSuccess)
      e = cudaMallocFromPoolAsync((void **)&rec, sizeof(uint32_t) * (size_t)nwords, pool, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(rec, 0xFF, sizeof(uint32_t) * (size_t)nwords, s);
    if (e == cudaSuccess) {
      unsigned *cnt = rmeta, *roff = rmeta + nreg;
      k_slab_count<<<blocks, 256, 0, s>>>(a, cnt);
      k_slab_scan<<<1, 1024, 0, s>>>(cnt, roff, (int)nreg);
      e = cudaGetLastError();
      a.rec = rec;
      a.roff = roff;
    }
  }
  if (a.unp) {
    // one launch per replicate chunk, its outputs at the chunk's first replicate, its
    // replicate numbers (the random streams) from rep0 + c0
    const size_t nss = (size_t)NB_SEG0 * NB_NSBINANG;
    for (int c0 = 0; c0 < nrep && e == cudaSuccess; c0 += rchunk) {
      const int nc = nrep - c0 < rchunk ? nrep - c0 : rchunk;
      const int rblk = (nc + 3) & ~3;
      HistArgs ac = a;
      ac.rep0 = rep0 + c0;
      ac.nrep = nc;
      ac.rblk = rblk;
      ac.psino = scr;
      ac.ssrb = ssrb + c0 * nss;
      ac.phc = phc + (size_t)c0 * nitag;
      ac.dhc = dhc + (size_t)c0 * nitag;
      ac.zR = zR + (size_t)c0 * nitag;
      ac.zM = zM + (size_t)c0 * nitag;
      ac.pvs = pvs + c0 * a.sne;
      ac.fan = fan + (size_t)c0 * NB_NRINGS * NB_NCRS;
      ac.bck = bck + (size_t)c0 * 2 * NB_NBUCKTS * nitag;
      e = cudaMemsetAsync(scr, 0, sizeof(uint32_t) * a.nbins * 2 * (size_t)rblk, s);
      if (e == cudaSuccess) e = launch_hist(ac, ctr, s);
      if (e == cudaSuccess) {
        k_pack_ssrb<<<nsm * 8, 256, 0, s>>>(psino + c0 * a.nbins, ac.ssrb, scr, d_soff, d_slst,
                                            a.nbins, nc, rblk);
        e = cudaGetLastError();
      }
    }
  } else {
    if (e == cudaSuccess) e = launch_hist(a, ctr, s);
    if (e == cudaSuccess && a.rec) {
      for (int sl = 0; sl < nslab; sl++)
        k_slab_add<<<nsm * 8, 256, 0, s>>>(psino, rec, a.roff, sl, a.nwst);
      e = cudaGetLastError();
    }
  }
  // a pageable-source cudaMemcpyAsync has staged `h` before returning, so `h` may go
  if (rec) cudaFreeAsync(rec, s);
  if (rmeta) cudaFreeAsync(rmeta, s);
  if (scr) cudaFreeAsync(scr, s);
  cudaFreeAsync(d, s);
  if (e != cudaSuccess) return nb_cuda_fail(e, "nb_hist", __FILE__, __LINE__);
  return NB_OK;
}

__global__ void k_unpack(const uint32_t *__restrict__ p, size_t n, uint16_t *__restrict__ psn,
                         uint16_t *__restrict__ dsn, unsigned long long *sums) {
  unsigned long long ps = 0, ds = 0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const uint32_t w = p[i];
    const uint16_t a = (uint16_t)(w & 0xFFFF), b = (uint16_t)(w >> 16);
    if (psn) psn[i] = a;
    if (dsn) dsn[i] = b;
    ps += a;
    ds += b;
  }
  for (int o = 16; o; o >>= 1) {
    ps += __shfl_down_sync(0xffffffffu, ps, o);
    ds += __shfl_down_sync(0xffffffffu, ds, o);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(&sums[0], ps);
    atomicAdd(&sums[1], ds);
  }
}

extern "C" int nb_hist_unpack(const uint32_t *psino, size_t nbins, uint16_t *psn, uint16_t *dsn,
                              unsigned long long *psum, unsigned long long *dsum, void *stream) {
  NB_RANGE("nb_hist_unpack");
  NB_REQUIRE(psino != nullptr, "nb_hist_unpack: NULL input");
  cudaStream_t s = (cudaStream_t)stream;
  unsigned long long *d = nullptr;
  NB_CUDA(cudaMallocAsync((void **)&d, 2 * sizeof(unsigned long long), s));
  cudaMemsetAsync(d, 0, 2 * sizeof(unsigned long long), s);
  k_unpack<<<1184, 256, 0, s>>>(psino, nbins, psn, dsn, d);
  unsigned long long h[2] = {0, 0};
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(h, d, sizeof(h), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  cudaFreeAsync(d, s);
  if (e != cudaSuccess) return nb_cuda_fail(e, "nb_hist_unpack", __FILE__, __LINE__);
  if (psum) *psum = h[0];
  if (dsum) *dsum = h[1];
  return NB_OK;
}

// ---------------------------------------------------------------------------------------
// nb_hist_static: nb_hist for callers that cannot allocate device memory.
//
// nb_hist stages its look-up tables and chunk plan in a stream-ordered device allocation
// made on every call.  This variant stages them instead in one file-scope static device
// array (NB_HIST_STATIC_BYTES, holding at most NB_HIST_STATIC_MAX_CHUNKS chunks), so a call
// makes no allocation of any kind: only cudaMemcpyAsync copies from the caller's host
// arrays into that array and the kernel launch.  The array belongs to every GPU that loads
// this library until the process exits; all calls on a device share it and it keeps the
// last call's tables, which every call overwrites before its kernel reads them (nothing in
// it has to start at zero).  Calls that overlap on the GPU (different streams, or other
// host threads) race on the array and must be serialised by the caller.
// ---------------------------------------------------------------------------------------
#include <mutex>

#define NB_HIST_STATIC_MAX_CHUNKS 4096
#define NB_HIST_STATIC_BYTES (512u * 1024u)

static __device__ __align__(256) unsigned char g_hist_static_scratch[NB_HIST_STATIC_BYTES];

namespace {
constexpr size_t kLutOff = 0;
constexpr size_t kS2cOff = (sizeof(HistLUT) + 255) & ~(size_t)255;
constexpr size_t kAtagOff = (kS2cOff + (size_t)NB_NSBINANG * sizeof(short2) + 255) & ~(size_t)255;
constexpr size_t kE4cOff = kAtagOff + sizeof(int64_t) * NB_HIST_STATIC_MAX_CHUNKS;
constexpr size_t kE4tOff = kE4cOff + sizeof(int) * NB_HIST_STATIC_MAX_CHUNKS;
constexpr size_t kCtrOff = (kE4tOff + sizeof(int) * NB_HIST_STATIC_MAX_CHUNKS + 15) & ~(size_t)15;
constexpr size_t kStaticEnd = kCtrOff + 16;
static_assert(kStaticEnd <= NB_HIST_STATIC_BYTES, "static histogram scratch too small");

std::mutex g_static_mu;
unsigned char *g_static_addr[64] = {};

// Device address of the static array on the current device.  The host-side name of a
// __device__ variable is only a stand-in, so the address is looked up once per device
// (on the first call there, with that device current) and cached.
int static_scratch(unsigned char **out) {
  int dev = 0;
  NB_CUDA(cudaGetDevice(&dev));
  NB_REQUIRE(dev >= 0 && dev < 64, "nb_hist_static: device index above 63");
  std::lock_guard<std::mutex> lk(g_static_mu);
  if (!g_static_addr[dev]) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_hist_static_scratch);
    if (e != cudaSuccess)
      return nb_cuda_fail(e, "cudaGetSymbolAddress(histogram static scratch)", __FILE__,
                          __LINE__);
    g_static_addr[dev] = static_cast<unsigned char *>(p);
  }
  *out = g_static_addr[dev];
  return NB_OK;
}
}  // namespace

extern "C" int nb_hist_static(const int32_t *lm, int64_t ele, int nchnk, const int64_t *atag,
                              const int *ele4chnk, const int *ele4thrd, int toff, int nitag,
                              int tstart, int tstop, int span, int btp, double btprt,
                              uint64_t seed, int rep0, int nrep, const int16_t *sn1_sn11,
                              const int16_t *sn1_ssrb, const int16_t *sn1_rno,
                              const int16_t *s2cF, uint32_t *psino, uint32_t *ssrb,
                              uint32_t *phc, uint32_t *dhc, int32_t *zR, int32_t *zM,
                              uint32_t *pvs, uint32_t *fan, uint32_t *bck, void *stream) {
  NB_REQUIRE(lm && atag && ele4chnk && ele4thrd, "nb_hist_static: NULL stream or plan");
  NB_REQUIRE(sn1_sn11 && sn1_ssrb && sn1_rno && s2cF, "nb_hist_static: NULL LUT");
  NB_REQUIRE(psino && ssrb && phc && dhc && zR && zM && pvs && fan && bck,
             "nb_hist_static: NULL output");
  NB_REQUIRE(span == 0 || span == 1 || span == 11, "nb_hist_static: span must be 0, 1 or 11");
  NB_REQUIRE(btp >= 0 && btp <= 2, "nb_hist_static: btp must be 0, 1 or 2");
  NB_REQUIRE(nrep >= 1 && nrep <= 1024 && nitag > 0 && nchnk >= 0,
             "nb_hist_static: bad sizes");
  NB_REQUIRE(!(btp == 2 && !(btprt > 0)), "nb_hist_static: btprt must be > 0");
  if (nchnk > NB_HIST_STATIC_MAX_CHUNKS) {
    nb_set_error_msg("nb_hist_static: the chunk plan has %d chunks, but the static scratch holds "
                     "at most %d (use nb_hist)", nchnk, NB_HIST_STATIC_MAX_CHUNKS);
    return NB_ERR_ARG;
  }
  for (int n = 0; n < nchnk; n++) {
    NB_REQUIRE(atag[n] >= 0 && ele4chnk[n] >= 0 && atag[n] + ele4chnk[n] <= ele,
               "nb_hist_static: chunk outside the stream");
    NB_REQUIRE(ele4thrd[n] >= 0, "nb_hist_static: bad slice length");
  }
  for (int i = 0; i < NB_NSN1; i++)
    NB_REQUIRE(sn1_sn11[i] >= 0 && sn1_sn11[i] < NB_NSN11 && sn1_ssrb[i] >= 0 &&
                   sn1_ssrb[i] < NB_SEG0 && sn1_rno[2 * i] >= 0 && sn1_rno[2 * i] < NB_NRINGS &&
                   sn1_rno[2 * i + 1] >= 0 && sn1_rno[2 * i + 1] < NB_NRINGS,
               "nb_hist_static: axial LUT out of range");
  if (nchnk == 0) return NB_OK;
  unsigned char *base = nullptr;
  int st = static_scratch(&base);
  if (st) return st;
  cudaStream_t s = (cudaStream_t)stream;

  HistArgs a{};
  a.lm = lm;
  a.nchnk = nchnk;
  a.toff = toff;
  a.nitag = nitag;
  a.tstart = tstart;
  a.tstop = tstop;
  a.span = span;
  a.btp = btp;
  a.seed = seed;
  a.rep0 = rep0;
  a.nrep = nrep;
  poisson_thresholds(btp == 2 ? btprt : 1.0, a.thr);
  a.nbins = span == 1 ? 354033792ull : (span == 11 ? 72557856ull : (size_t)NB_SEG0 * NB_NSBINANG);
  const int tn = nitag > NB_MXNITAG ? NB_MXNITAG : nitag;
  a.sne = (size_t)((tn + 3) / 4) * NB_SEG0 * NB_NSBINS;
  a.psino = psino;
  a.ssrb = ssrb;
  a.phc = phc;
  a.dhc = dhc;
  a.zR = zR;
  a.zM = zM;
  a.pvs = pvs;
  a.fan = fan;
  a.bck = bck;
  a.lut = reinterpret_cast<const HistLUT *>(base + kLutOff);
  a.s2cF = reinterpret_cast<const short2 *>(base + kS2cOff);
  a.atag = reinterpret_cast<const int64_t *>(base + kAtagOff);
  a.e4c = reinterpret_cast<const int *>(base + kE4cOff);
  a.e4t = reinterpret_cast<const int *>(base + kE4tOff);
  // The caller's host arrays are first gathered into one pageable host buffer, laid out as
  // the static array, and moved with one copy: a cudaMemcpyAsync from pageable memory has
  // staged its source before it returns, so the caller may reuse or free its arrays (pinned
  // ones included) as soon as this call returns, as with nb_hist.  Only host memory is
  // allocated here.
  const size_t used = kE4tOff + sizeof(int) * (size_t)nchnk;
  std::vector<unsigned char> h(used, 0);
  HistLUT hl;
  memcpy(hl.sn1_sn11, sn1_sn11, sizeof(hl.sn1_sn11));
  memcpy(hl.sn1_ssrb, sn1_ssrb, sizeof(hl.sn1_ssrb));
  memcpy(hl.sn1_rno, sn1_rno, sizeof(hl.sn1_rno));
  memcpy(&h[kLutOff], &hl, sizeof(HistLUT));
  memcpy(&h[kS2cOff], s2cF, (size_t)NB_NSBINANG * sizeof(short2));
  memcpy(&h[kAtagOff], atag, sizeof(int64_t) * nchnk);
  memcpy(&h[kE4cOff], ele4chnk, sizeof(int) * nchnk);
  memcpy(&h[kE4tOff], ele4thrd, sizeof(int) * nchnk);
  cudaError_t e = cudaMemcpyAsync(base, h.data(), used, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = launch_hist(a, reinterpret_cast<unsigned *>(base + kCtrOff), s);
  if (e != cudaSuccess) return nb_cuda_fail(e, "nb_hist_static", __FILE__, __LINE__);
  return NB_OK;
}
