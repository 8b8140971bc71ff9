// BF16 3x3x3 convolutions on the 5th-generation tensor cores (tcgen05) for
// the learned multigrid warm start (a small 3D U-Net). No reference
// counterpart: WARP has no learned components.
//
// Forward / data-gradient (k_conv3_mma): implicit GEMM
//   Y[v][co] = sum_{t<27} sum_ci X[v + off_t][ci] * Wt[t][co][ci]   (+bias, ReLU)
// with X and Y in NDHWC bf16 (channels fastest), zero padding at the box
// edges. A CTA computes M = 128 consecutive output voxels by N = Cout
// channels; the K loop runs over taps and 16-channel slices. Operand tiles
// are staged in shared memory in the canonical K-major no-swizzle layout of
// UMMA (8x16-byte core matrices), one elected thread issues
// tcgen05.mma.cta_group::1.kind::f16 with FP32 accumulation in tensor memory,
// completion is tracked with tcgen05.commit on mbarriers (bounded waits),
// and the epilogue reads the accumulator back with tcgen05.ld. The data
// gradient is the same kernel with the taps mirrored and Cin/Cout swapped in
// the weights.
//
// Weight gradient (k_conv3_wgrad_mma): per tap t,
//   dW[t][co][ci] = sum_v dY[v][co] * X[v + off_t][ci]
// a GEMM with K = voxels, from channel-major (CDHW) copies of dY and X so
// both operands are K-major; CTAs take voxel chunks and add their FP32
// partial sums to dW atomically.

#include <cuda_bf16.h>

#include <cstdint>

#include "wg_internal.h"

namespace wg {
namespace {

constexpr int CM = 128;      // output voxels per CTA (UMMA M)
constexpr int CNT = 128;     // threads per CTA
constexpr int CSTAGES = 4;   // shared-memory pipeline stages
constexpr long long kSpinLimit = 1LL << 26;  // mbarrier poll limit before giving up

__device__ inline uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor: K-major, no swizzle, 8x16 B core matrices;
// lbo = byte distance between the two core matrices along K, sbo = between
// 8-row groups along M/N; version 1 (tcgen05).
__device__ inline uint64_t make_sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}

// Instruction descriptor of kind::f16: BF16 A and B, FP32 D, both K-major.
__host__ __device__ constexpr uint32_t make_idesc(int m, int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

__device__ inline void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

// Waits for completion of phase `parity` with an iteration limit; returns
// false (and leaves the error flag to the caller) when the limit is hit.
__device__ inline bool mbar_wait(uint64_t* bar, uint32_t parity) {
  const uint32_t a = smem_u32(bar);
  for (long long it = 0; it < kSpinLimit; ++it) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(a), "r"(parity)
        : "memory");
    if (ok) return true;
  }
  return false;
}

__device__ inline void umma_f16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t accum) {
  const uint32_t z = 0;  // disable-output-lane mask: all lanes written
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t}" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accum), "r"(z)
      : "memory");
}

__device__ inline void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ inline void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ inline void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ inline void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }

// 16 FP32 columns of this warp's 32 TMEM lanes.
__device__ inline void tmem_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// Byte offset of element (row, k) (k < 16) in a K-major no-swizzle tile:
// 8-row groups 256 B apart, the two 8-element K halves 128 B apart.
__device__ inline uint32_t kmaj_off(int row, int k) {
  return (uint32_t)((row >> 3) * 256 + (k >> 3) * 128 + (row & 7) * 16 + (k & 7) * 2);
}

struct ConvArgs {
  const __nv_bfloat16* x;   // [D][H][W][cin]
  const __nv_bfloat16* w;   // [27][cout][cin]
  const float* bias;        // [cout] or null
  __nv_bfloat16* y;         // [D][H][W][ystride], channels yoff..yoff+cout-1 written
  const __nv_bfloat16* mask;  // optional [D][H][W][mstride] activation: y *= (mask > 0)
  int D, H, W, cin, cout, ystride, yoff, mstride, relu;
  int* err;
};

// Forward / data-gradient implicit GEMM, N = cout (16..256, multiple of 16).
__global__ void __launch_bounds__(CNT) k_conv3_mma(ConvArgs a) {
  extern __shared__ __align__(1024) unsigned char sm[];
  const int N = a.cout;
  const int a_bytes = CM * 32;   // 128 rows x 16 bf16
  const int b_bytes = N * 32;
  const int stage_bytes = a_bytes + b_bytes;
  __shared__ __align__(8) uint64_t bars[CSTAGES + 1];
  __shared__ uint32_t tmem_base_s;
  __shared__ int fail_s;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const long long nvox = (long long)a.D * a.H * a.W;
  const long long v0 = (long long)blockIdx.x * CM;
  uint32_t ncols = 32;
  while ((int)ncols < N) ncols <<= 1;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base_s)),
                 "r"(ncols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    for (int s = 0; s <= CSTAGES; ++s) mbar_init(&bars[s], 1);
    fail_s = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_base_s;

  // this thread's A row: output voxel v0 + tid
  const long long vr = v0 + tid;
  const bool row_ok = vr < nvox;
  int rx = 0, ry = 0, rz = 0;
  if (row_ok) {
    rx = (int)(vr % a.W);
    ry = (int)((vr / a.W) % a.H);
    rz = (int)(vr / ((long long)a.W * a.H));
  }
  const int kslices = a.cin >> 4;
  const int nsteps = 27 * kslices;
  const uint32_t idesc = make_idesc(CM, N);
  bool ok = true;
  for (int j = 0; j < nsteps; ++j) {
    const int s = j % CSTAGES;
    unsigned char* st = sm + s * stage_bytes;
    if (j >= CSTAGES) {
      // the MMA that last read this stage must be done
      if (!mbar_wait(&bars[s], (uint32_t)(((j / CSTAGES) - 1) & 1))) ok = false;
    }
    const int t = j / kslices, ks = j % kslices;
    const int dz = t / 9 - 1, dy = (t / 3) % 3 - 1, dx = t % 3 - 1;
    // A: 16 channels of the shifted input voxel (zero outside the box)
    {
      uint4 lo = make_uint4(0, 0, 0, 0), hi = make_uint4(0, 0, 0, 0);
      const int xx = rx + dx, yy = ry + dy, zz = rz + dz;
      if (row_ok && xx >= 0 && xx < a.W && yy >= 0 && yy < a.H && zz >= 0 && zz < a.D) {
        const uint4* src = reinterpret_cast<const uint4*>(
            a.x + (((long long)zz * a.H + yy) * a.W + xx) * a.cin + ks * 16);
        lo = src[0];
        hi = src[1];
      }
      *reinterpret_cast<uint4*>(st + kmaj_off(tid, 0)) = lo;
      *reinterpret_cast<uint4*>(st + kmaj_off(tid, 8)) = hi;
    }
    // B: weights of tap t, channels ks*16.., all N output channels
    for (int i = tid; i < 2 * N; i += CNT) {
      const int n = i >> 1, h = i & 1;
      const uint4 v = *reinterpret_cast<const uint4*>(a.w + ((long long)t * N + n) * a.cin + ks * 16 + h * 8);
      *reinterpret_cast<uint4*>(st + a_bytes + kmaj_off(n, h * 8)) = v;
    }
    fence_async_smem();
    __syncthreads();
    if (tid == 0) {
      tc_fence_after();
      const uint32_t sa = smem_u32(st), sb = smem_u32(st + a_bytes);
      umma_f16(tmem, make_sdesc(sa, 128, 256), make_sdesc(sb, 128, 256), idesc, j > 0 ? 1u : 0u);
      umma_commit(&bars[s]);
    }
  }
  // all MMAs done: the last commit covers every earlier MMA of this thread
  if (tid == 0) umma_commit(&bars[CSTAGES]);
  if (!mbar_wait(&bars[CSTAGES], 0)) ok = false;
  tc_fence_after();
  if (!ok) atomicOr(&fail_s, 1);
  __syncthreads();
  if (!fail_s) {
    // epilogue: row m = 32*warp + lane, 16 columns at a time
    const long long v = v0 + 32 * warp + lane;
    for (int c0 = 0; c0 < N; c0 += 16) {
      float f[16];
      tmem_ld16(tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)c0, f);
      if (v < nvox) {
        __nv_bfloat16 out[16];
#pragma unroll
        for (int i = 0; i < 16; ++i) {
          float r = f[i] + (a.bias ? a.bias[c0 + i] : 0.f);
          if (a.relu) r = fmaxf(r, 0.f);
          if (a.mask && !(__bfloat162float(a.mask[v * a.mstride + c0 + i]) > 0.f)) r = 0.f;
          out[i] = __float2bfloat16_rn(r);
        }
        __nv_bfloat16* dst = a.y + v * a.ystride + a.yoff + c0;
        *reinterpret_cast<uint4*>(dst) = *reinterpret_cast<uint4*>(&out[0]);
        *reinterpret_cast<uint4*>(dst + 8) = *reinterpret_cast<uint4*>(&out[8]);
      }
    }
  } else if (tid == 0) {
    atomicOr(a.err, 1);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols));
}

struct WgradArgs {
  const __nv_bfloat16* xT;   // [cin][D][H][W]
  const __nv_bfloat16* dyT;  // [cout][D][H][W]
  float* dw;                 // [27][cout][cin], accumulated
  int D, H, W, cin, cout, mpad;
  long long chunk;           // voxels per CTA (multiple of 16)
  int* err;
};

// Weight gradient of one tap (blockIdx.y) over one voxel chunk (blockIdx.x):
// D[co][ci] = sum_v dY[co][v] * X[ci][v + off_t]; M = cout padded to 64/128,
// N = cin.
__global__ void __launch_bounds__(CNT) k_conv3_wgrad_mma(WgradArgs a) {
  extern __shared__ __align__(1024) unsigned char sm[];
  const int M = a.mpad, N = a.cin;
  const int a_bytes = M * 32, b_bytes = N * 32, stage_bytes = a_bytes + b_bytes;
  __shared__ __align__(8) uint64_t bars[CSTAGES + 1];
  __shared__ uint32_t tmem_base_s;
  __shared__ int fail_s;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int t = blockIdx.y;
  const int dz = t / 9 - 1, dy = (t / 3) % 3 - 1, dx = t % 3 - 1;
  const long long nvox = (long long)a.D * a.H * a.W;
  const long long k0 = (long long)blockIdx.x * a.chunk;
  const long long k1 = min(nvox, k0 + a.chunk);
  uint32_t ncols = 32;
  while ((int)ncols < N) ncols <<= 1;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base_s)),
                 "r"(ncols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    for (int s = 0; s <= CSTAGES; ++s) mbar_init(&bars[s], 1);
    fail_s = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_base_s;
  const uint32_t idesc = make_idesc(M, N);
  const int nsteps = (int)((k1 - k0 + 15) / 16);
  bool ok = true;
  for (int j = 0; j < nsteps; ++j) {
    const int s = j % CSTAGES;
    unsigned char* st = sm + s * stage_bytes;
    if (j >= CSTAGES && !mbar_wait(&bars[s], (uint32_t)(((j / CSTAGES) - 1) & 1))) ok = false;
    const long long kb = k0 + 16LL * j;
    // A: dY rows (output channels, zero above cout), 16 voxels each
    for (int i = tid; i < M * 16; i += CNT) {
      const int row = i >> 4, k = i & 15;
      const long long v = kb + k;
      __nv_bfloat16 e = __float2bfloat16_rn(0.f);
      if (row < a.cout && v < k1) e = a.dyT[(long long)row * nvox + v];
      *reinterpret_cast<__nv_bfloat16*>(st + kmaj_off(row, k)) = e;
    }
    // B: X rows (input channels) at the voxel shifted by the tap offset
    for (int i = tid; i < N * 16; i += CNT) {
      const int row = i >> 4, k = i & 15;
      const long long v = kb + k;
      __nv_bfloat16 e = __float2bfloat16_rn(0.f);
      if (v < k1) {
        const int x = (int)(v % a.W) + dx, y = (int)((v / a.W) % a.H) + dy, z = (int)(v / ((long long)a.W * a.H)) + dz;
        if (x >= 0 && x < a.W && y >= 0 && y < a.H && z >= 0 && z < a.D)
          e = a.xT[(long long)row * nvox + ((long long)z * a.H + y) * a.W + x];
      }
      *reinterpret_cast<__nv_bfloat16*>(st + a_bytes + kmaj_off(row, k)) = e;
    }
    fence_async_smem();
    __syncthreads();
    if (tid == 0) {
      tc_fence_after();
      umma_f16(tmem, make_sdesc(smem_u32(st), 128, 256), make_sdesc(smem_u32(st + a_bytes), 128, 256), idesc,
               j > 0 ? 1u : 0u);
      umma_commit(&bars[s]);
    }
  }
  if (tid == 0) umma_commit(&bars[CSTAGES]);
  if (nsteps > 0 && !mbar_wait(&bars[CSTAGES], 0)) ok = false;
  tc_fence_after();
  if (!ok) atomicOr(&fail_s, 1);
  __syncthreads();
  if (!fail_s && nsteps > 0) {
    // rows 0..M-1 live in TMEM lanes 0..M-1; warps 0..M/32-1 read them
    if (32 * warp < M) {
      const int row = 32 * warp + lane;
      for (int c0 = 0; c0 < N; c0 += 16) {
        float f[16];
        tmem_ld16(tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)c0, f);
        if (row < a.cout)
          for (int i = 0; i < 16; ++i) atomicAdd(&a.dw[((long long)t * a.cout + row) * a.cin + c0 + i], f[i]);
      }
    }
  } else if (fail_s && tid == 0) {
    atomicOr(a.err, 1);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols));
}

}  // namespace
}  // namespace wg

using namespace wg;

extern "C" {

int wg_conv3_fwd(const void* x, int D, int H, int W, int cin, const void* w, const float* bias, int cout, void* y,
                 int ystride, int yoff, const void* mask, int mstride, int relu, int* err, void* stream) {
  if (!x || !w || !y || !err || D < 1 || H < 1 || W < 1 || cin < 16 || cin % 16 || cout < 16 || cout > 256 ||
      cout % 16 || ystride < yoff + cout || (yoff % 8) || (ystride % 8) || (mask && mstride < cout)) {
    set_error("wg_conv3_fwd: bad arguments (cin, cout multiples of 16, cout <= 256, 16-byte aligned rows)");
    return WG_EINVAL;
  }
  ConvArgs a{(const __nv_bfloat16*)x, (const __nv_bfloat16*)w, bias, (__nv_bfloat16*)y,
             (const __nv_bfloat16*)mask, D, H, W, cin, cout, ystride, yoff, mstride, relu, err};
  const long long nvox = (long long)D * H * W;
  const int smem = CSTAGES * (CM * 32 + cout * 32);
  static bool attr = false;
  if (!attr) {
    WG_TRY_CUDA(cudaFuncSetAttribute(k_conv3_mma, cudaFuncAttributeMaxDynamicSharedMemorySize, 64 * 1024));
    attr = true;
  }
  k_conv3_mma<<<(unsigned)((nvox + CM - 1) / CM), CNT, smem, (cudaStream_t)stream>>>(a);
  WG_TRY_CUDA(cudaGetLastError());
  return WG_OK;
}

int wg_conv3_wgrad(const void* xT, const void* dyT, int D, int H, int W, int cin, int cout, float* dw, int* err,
                   void* stream) {
  if (!xT || !dyT || !dw || !err || D < 1 || H < 1 || W < 1 || cin < 16 || cin % 16 || cin > 256 || cout < 1 ||
      cout > 128) {
    set_error("wg_conv3_wgrad: bad arguments (cin multiple of 16 up to 256, cout <= 128)");
    return WG_EINVAL;
  }
  // M = 128 keeps accumulator row m in TMEM lane m (output channels padded with zeros)
  const int mpad = 128;
  const long long nvox = (long long)D * H * W;
  const long long chunk = 4096;
  WgradArgs a{(const __nv_bfloat16*)xT, (const __nv_bfloat16*)dyT, dw, D, H, W, cin, cout, mpad, chunk, err};
  const int smem = CSTAGES * (mpad * 32 + cin * 32);
  static bool attr = false;
  if (!attr) {
    WG_TRY_CUDA(cudaFuncSetAttribute(k_conv3_wgrad_mma, cudaFuncAttributeMaxDynamicSharedMemorySize, 64 * 1024));
    attr = true;
  }
  dim3 grid((unsigned)((nvox + chunk - 1) / chunk), 27);
  k_conv3_wgrad_mma<<<grid, CNT, smem, (cudaStream_t)stream>>>(a);
  WG_TRY_CUDA(cudaGetLastError());
  return WG_OK;
}

}  // extern "C"
