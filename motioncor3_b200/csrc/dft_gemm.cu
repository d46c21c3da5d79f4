// Split-precision BF16 DFT-GEMMs on the Blackwell tensor cores.
//
// The row pass of the patch transforms (CTransformStack on the patch
// buffer, Align/CMeasurePatches.cpp:55 -> Util/CCufft2D.cpp:65-78, patches
// not normalised) as a GEMM: every patch row of K reals times the K x 2C
// real DFT matrix (C = K/2+1 frequencies, columns interleaved as re, im)
// gives the row's half spectrum directly in the [row][C] complex layout.
//
// Precision: each FP32 operand x is split as hi = bf16(x), lo = bf16(x - hi)
// and the product is hi*hi + hi*lo + lo*hi (the lo*lo term, ~2^-16 of the
// product, is dropped), accumulated in FP32 in tensor memory: about 2^-16
// relative error per product instead of BF16's 2^-8.
//
// Kernel: one CTA computes a 128-row x 208-column tile of the output with
// tcgen05.mma (kind::f16, BF16 inputs, FP32 accumulator in TMEM, M = 128,
// N = 208, K = 16 per instruction), one thread issuing.  K runs in chunks
// of 32 through a two-stage shared-memory pipeline:
//  * the B chunk (DFT matrix, hi and lo, precomputed in the UMMA operand
//    layout) arrives by one cp.async.bulk copy completing on an mbarrier;
//  * the A chunk is loaded from the patch rows by the CTA's threads one
//    chunk ahead (the loads of chunk c+1 are in flight while chunk c is
//    converted and its MMAs run), split into hi/lo and stored in the operand
//    layout (patch rows start at arbitrary float offsets, which a tensor
//    copy cannot address);
//  * tcgen05.commit signals an mbarrier when the chunk's MMAs have read the
//    stage, which frees it for the chunk after next.
// The epilogue reads the accumulator with tcgen05.ld and stores the
// interleaved spectrum.  Every mbarrier wait gives up after a fixed number
// of polls, records an error flag and lets the CTA release its tensor
// memory and return.
//
// Operand layout (K-major, no swizzle): 8-row x 16-byte core matrices;
// byte offset of element (r, k) in an R-row, 32-column chunk =
// (k / 8) * (R * 16) + (r / 8) * 128 + (r % 8) * 16 + (k % 8) * 2, so the
// descriptor's leading-dimension offset (between the two 8-element K
// halves of one instruction) is R * 16 bytes and its stride offset
// (between 8-row groups) 128 bytes.
#include <cuda_bf16.h>

#include <cmath>
#include <mutex>
#include <vector>

#include "kernels.cuh"
#include "dft_gemm.cuh"

namespace mc3 {

namespace {

constexpr int kDgM = 128;       // output rows per CTA (UMMA M)
constexpr int kDgN = 208;       // output columns per CTA (UMMA N)
constexpr int kDgK = 32;        // K per pipeline stage
constexpr int kDgStages = 2;
constexpr int kDgThreads = 256;      // 8 warps: 2 A rows per thread per chunk
constexpr int kDgRowsPerThread = kDgM * 4 / kDgThreads;
constexpr int kDgTmemCols = 256;
constexpr int kATile = kDgM * kDgK * 2;          // one BF16 A tile (bytes)
constexpr int kBTile = kDgN * kDgK * 2;          // one BF16 B tile
constexpr int kBBlob = 2 * kBTile;               // hi + lo
constexpr int kStageBytes = 2 * kATile + kBBlob; // A hi, A lo, B hi, B lo
constexpr int kDgSmem = kDgStages * kStageBytes + 128;
// Longest wait on one mbarrier (about 1 s at the B200's clock).
constexpr long long kWaitCycles = 2000000000ll;
static_assert(kDgN % 16 == 0 && kDgN <= 256, "UMMA N for M = 128");
static_assert(kBBlob % 16 == 0, "bulk copies move multiples of 16 bytes");
// two CTAs per SM at most: their tensor memory (2 x 256 columns) fits
static_assert(3 * kDgSmem > 227 * 1024, "a third CTA must not fit");

__host__ __device__ constexpr int op_off(int r, int k, int R) {
  return (k >> 3) * (R * 16) + (r >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2;
}

// Instruction descriptor: FP32 accumulator, BF16 A and B, both K-major,
// N >> 3 at bit 17, M >> 4 at bit 24.
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) |
                            ((uint32_t)(kDgN >> 3) << 17) | ((uint32_t)(kDgM >> 4) << 24);

__device__ int g_dft_gemm_error;  // set by a CTA whose wait gave up

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// Shared-memory operand descriptor (no swizzle, Blackwell version bit 46).
__device__ __forceinline__ uint64_t op_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

// Polls the mbarrier phase with the given parity.  Gives up (false) after
// kWaitCycles, or, when `abortable`, as soon as another CTA has recorded an
// error, so that a failing launch ends quickly.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, bool abortable = true) {
  const long long t0 = clock64();
  for (unsigned i = 0;; ++i) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
    if ((i & 255u) == 255u) {
      if (abortable && *reinterpret_cast<volatile int*>(&g_dft_gemm_error)) return false;
      if (clock64() - t0 > kWaitCycles) return false;
    }
  }
}

__device__ __forceinline__ void bulk_load(uint32_t dst, const void* src, uint32_t bytes,
                                          uint32_t bar) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
               : "memory");
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
      "l"(src), "r"(bytes), "r"(bar)
      : "memory");
}

__device__ __forceinline__ void umma(uint32_t tmem, uint64_t a, uint64_t b, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
      "l"(a), "l"(b), "r"(kIdesc), "r"(accumulate));
}

__device__ __forceinline__ void umma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
               : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ uint32_t pack_bf16(float a, float b) {
  __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
  return *reinterpret_cast<uint32_t*>(&h);
}

// Patch rows (K reals each) times the DFT matrix -> half spectra.  Rows:
// global row g = item * H + y reads in + batch_in_off(bt, item) + y * in_pitch;
// writes out + item * bt.out_stride + y * out_pitch (complex), C = K/2+1
// values per row, times `scale`.
__global__ void __launch_bounds__(kDgThreads, 2)
    k_dft_rows_bf16x3(const float* __restrict__ in, long in_pitch, float2* out, long out_pitch,
                      int K, int H, Batch bt, const uint8_t* __restrict__ bmat, int nchunks,
                      float scale) {
  extern __shared__ __align__(1024) uint8_t sm[];
  uint8_t* stage0 = sm;
  uint64_t* bars = reinterpret_cast<uint64_t*>(sm + kDgStages * kStageBytes);
  // bars[0..1]: B chunk arrived; bars[2..3]: MMAs of the stage done
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * kDgStages);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int mt = blockIdx.x >> 1, nt = blockIdx.x & 1;
  const long rows_total = (long)bt.items * H;
  const long m0 = (long)mt * kDgM;

  if (tid == 0) {
    for (int i = 0; i < 2 * kDgStages; ++i) mbar_init(smem_u32(&bars[i]), 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(tmem_slot)),
                 "r"(kDgTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;

  // This thread's A rows (2 of the tile's 128) and 8-element K group.
  const int kc = tid & 3;
  const float* rowp[kDgRowsPerThread];
  int rloc[kDgRowsPerThread];
#pragma unroll
  for (int i = 0; i < kDgRowsPerThread; ++i) {
    rloc[i] = (tid >> 2) + (kDgThreads / 4) * i;
    const long g = m0 + rloc[i];
    rowp[i] = nullptr;
    if (g < rows_total) {
      const int item = (int)(g / H), y = (int)(g % H);
      rowp[i] = in + batch_in_off(bt, item) + (long)y * in_pitch;
    }
  }
  // A values of the current chunk; the next chunk's are loaded ahead
  float va[kDgRowsPerThread][8], vn[kDgRowsPerThread][8];
  auto load_chunk = [&](int c, float (&v)[kDgRowsPerThread][8]) {
    const int k0 = c * kDgK + kc * 8;
#pragma unroll
    for (int i = 0; i < kDgRowsPerThread; ++i)
#pragma unroll
      for (int j = 0; j < 8; ++j) v[i][j] = (rowp[i] && k0 + j < K) ? rowp[i][k0 + j] : 0.0f;
  };
  load_chunk(0, va);
  const uint8_t* bsrc = bmat + (size_t)nt * nchunks * kBBlob;
  bool ok = true;
  int last_commit = -1;  // thread 0: the last chunk whose MMAs were committed

  for (int c = 0; c < nchunks && ok; ++c) {
    const int s = c & 1;
    const uint32_t use = (uint32_t)(c >> 1);
    uint8_t* st = stage0 + s * kStageBytes;
    const uint32_t bar_b = smem_u32(&bars[s]), bar_m = smem_u32(&bars[kDgStages + s]);
    // the MMAs of chunk c-2 must have read this stage
    bool good = c < 2 || mbar_wait(bar_m, (use - 1) & 1);
    if (c + 1 < nchunks) load_chunk(c + 1, vn);  // in flight during this chunk
    good = __syncthreads_and(good);
    if (good) {
      if (tid == 0) bulk_load(smem_u32(st + 2 * kATile), bsrc + (size_t)c * kBBlob, kBBlob, bar_b);
      // A chunk: split into hi / lo and stored in the operand layout
#pragma unroll
      for (int i = 0; i < kDgRowsPerThread; ++i) {
        uint32_t hi[4], lo[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const __nv_bfloat162 h = __floats2bfloat162_rn(va[i][2 * j], va[i][2 * j + 1]);
          const float2 hf = __bfloat1622float2(h);
          hi[j] = *reinterpret_cast<const uint32_t*>(&h);
          lo[j] = pack_bf16(va[i][2 * j] - hf.x, va[i][2 * j + 1] - hf.y);
        }
        const int off = op_off(rloc[i], kc * 8, kDgM);
        *reinterpret_cast<uint4*>(st + off) = make_uint4(hi[0], hi[1], hi[2], hi[3]);
        *reinterpret_cast<uint4*>(st + kATile + off) = make_uint4(lo[0], lo[1], lo[2], lo[3]);
      }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    __syncthreads();
    if (good && tid == 0) {
      if (!mbar_wait(bar_b, use & 1)) {
        good = false;
      } else {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t a_hi = smem_u32(st), a_lo = a_hi + kATile;
        const uint32_t b_hi = a_hi + 2 * kATile, b_lo = b_hi + kBTile;
#pragma unroll
        for (int ks = 0; ks < kDgK / 16; ++ks) {
          const uint32_t ao = ks * 2 * kDgM * 16, bo = ks * 2 * kDgN * 16;
          const uint64_t dah = op_desc(a_hi + ao, kDgM * 16, 128);
          const uint64_t dal = op_desc(a_lo + ao, kDgM * 16, 128);
          const uint64_t dbh = op_desc(b_hi + bo, kDgN * 16, 128);
          const uint64_t dbl = op_desc(b_lo + bo, kDgN * 16, 128);
          umma(tmem, dah, dbh, (c | ks) ? 1u : 0u);
          umma(tmem, dah, dbl, 1u);
          umma(tmem, dal, dbh, 1u);
        }
        umma_commit(bar_m);
        last_commit = c;
      }
    }
    ok = __syncthreads_and(good);
#pragma unroll
    for (int i = 0; i < kDgRowsPerThread; ++i)
#pragma unroll
      for (int j = 0; j < 8; ++j) va[i][j] = vn[i][j];
  }
  // the last chunk's commit covers every MMA this CTA issued
  if (ok) {
    const int cl = nchunks - 1;
    ok = mbar_wait(smem_u32(&bars[kDgStages + (cl & 1)]), (uint32_t)(cl >> 1) & 1);
  }
  ok = __syncthreads_and(ok);
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (ok) {
    // warps w and w + 4 share TMEM lanes 32 (w % 4) ..; they split the
    // 13 column chunks of 16 (7 and 6)
    const int r = (warp & 3) * 32 + lane;
    const long g = m0 + r;
    float* orow = nullptr;
    if (g < rows_total) {
      const int item = (int)(g / H), y = (int)(g % H);
      orow = reinterpret_cast<float*>(out + (long)item * bt.out_stride + (long)y * out_pitch);
    }
    const int nvalid = 2 * (K / 2 + 1), n0 = nt * kDgN;
    const uint32_t tl = tmem + ((uint32_t)((warp & 3) * 32) << 16);
    const int jbeg = warp < 4 ? 0 : 112, jend = warp < 4 ? 112 : kDgN;
#pragma unroll 1
    for (int j0 = jbeg; j0 < jend; j0 += 16) {
      float v[16];
      tmem_ld16(tl + (uint32_t)j0, v);
      if (orow) {
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          const int n = n0 + j0 + 2 * q;
          if (n + 1 < nvalid)
            *reinterpret_cast<float2*>(orow + n) = make_float2(v[2 * q] * scale, v[2 * q + 1] * scale);
        }
      }
    }
  } else if (tid == 0) {
    atomicOr(&g_dft_gemm_error, 1);
    __threadfence();
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (!ok && tid == 0 && last_commit >= 0) {
    // MMAs may still be in flight after a failed wait: give the last
    // committed chunk a bounded time to finish before the tensor memory is
    // released
    mbar_wait(smem_u32(&bars[kDgStages + (last_commit & 1)]), (uint32_t)(last_commit >> 1) & 1,
              false);
  }
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(kDgTmemCols)
                 : "memory");
}

// DFT matrix of a K-point real transform in the B operand layout: for each
// column tile (208 outputs) and K chunk (32 inputs), hi then lo.  Output n
// = 2c + t: t = 0 -> cos(2 pi c k / K), t = 1 -> -sin(2 pi c k / K).
std::vector<uint8_t> dft_matrix_blobs(int K, int nchunks) {
  const int C = K / 2 + 1;
  std::vector<uint8_t> blob((size_t)2 * nchunks * kBBlob, 0);
  for (int nt = 0; nt < 2; ++nt)
    for (int c = 0; c < nchunks; ++c) {
      uint8_t* b = blob.data() + ((size_t)nt * nchunks + c) * kBBlob;
      for (int r = 0; r < kDgN; ++r)
        for (int kk = 0; kk < kDgK; ++kk) {
          const int n = nt * kDgN + r, k = c * kDgK + kk;
          double v = 0.0;
          if (n / 2 < C && k < K) {
            const long m = ((long)(n / 2) * k) % K;
            const double a = 2.0 * 3.14159265358979323846 * (double)m / K;
            v = (n & 1) ? -std::sin(a) : std::cos(a);
          }
          const __nv_bfloat16 h = __float2bfloat16_rn((float)v);
          const __nv_bfloat16 l = __float2bfloat16_rn((float)(v - (double)__bfloat162float(h)));
          const int off = op_off(r, kk, kDgN);
          *reinterpret_cast<__nv_bfloat16*>(b + off) = h;
          *reinterpret_cast<__nv_bfloat16*>(b + kBTile + off) = l;
        }
    }
  return blob;
}

struct BCache {
  int dev, K;
  uint8_t* d;
};
std::mutex g_bmu;
std::vector<BCache> g_bcache;

int b_operand(int K, int nchunks, const uint8_t** out) {
  int dev = 0;
  MC3_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(g_bmu);
  for (const BCache& b : g_bcache)
    if (b.dev == dev && b.K == K) {
      *out = b.d;
      return kOk;
    }
  std::vector<uint8_t> h = dft_matrix_blobs(K, nchunks);
  uint8_t* d = nullptr;
  MC3_CUDA(cudaMalloc(&d, h.size()));
  MC3_CUDA(cudaMemcpy(d, h.data(), h.size(), cudaMemcpyHostToDevice));
  g_bcache.push_back(BCache{dev, K, d});
  *out = d;
  return kOk;
}

}  // namespace

bool dft_rows_supported(int K) { return K >= 16 && K % 2 == 0 && 2 * (K / 2 + 1) <= 2 * kDgN; }

int dft_rows_r2c(const float* in, long in_pitch, float2* out, long out_pitch, int K, int H,
                 const Batch& b, float scale, cudaStream_t st) {
  if (!dft_rows_supported(K) || H < 1 || b.items < 1) return kEUnsupported;
  const int nchunks = (K + kDgK - 1) / kDgK;
  const uint8_t* bmat = nullptr;
  MC3_TRY(b_operand(K, nchunks, &bmat));
  MC3_TRY(set_smem_attr(k_dft_rows_bf16x3, kDgSmem));
  const long rows = (long)b.items * H;
  const long mtiles = (rows + kDgM - 1) / kDgM;
  if (2 * mtiles > 0x7fffffffl) return kEUnsupported;
  // algorithmic bytes: the FP32 rows read once, the spectra written once
  prof::Scope ps("k_dft_rows_bf16x3", (double)rows * (K * 4.0 + (K / 2 + 1) * 8.0), st);
  k_dft_rows_bf16x3<<<(unsigned)(2 * mtiles), kDgThreads, kDgSmem, st>>>(
      in, in_pitch, out, out_pitch, K, H, b, bmat, nchunks, scale);
  MC3_CHECK_LAUNCH("k_dft_rows_bf16x3");
  return kOk;
}

int dft_gemm_error(bool reset, int* flag) {
  int v = 0;
  MC3_CUDA(cudaMemcpyFromSymbol(&v, g_dft_gemm_error, sizeof(int)));
  if (reset && v) {
    const int z = 0;
    MC3_CUDA(cudaMemcpyToSymbol(g_dft_gemm_error, &z, sizeof(int)));
  }
  *flag = v;
  return kOk;
}

}  // namespace mc3
