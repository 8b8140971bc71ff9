// BF16 3x3x3 convolutions on the 5th-generation tensor cores (tcgen05) for
// the learned multigrid warm start (a small 3D U-Net). No reference
// counterpart: WARP has no learned components.
//
// Forward / data gradient (k_conv3_tile): implicit GEMM
//   Y[v][co] = sum_{t<27} sum_ci X[v + off_t][ci] * Wt[t][co][ci]   (+bias, ReLU)
// with X and Y in NDHWC bf16 (channels fastest) and zero padding at the box
// edges, over output tiles whose input halo stays in shared memory for all
// 27 taps. The data gradient is the same kernel with the taps mirrored and
// Cin/Cout swapped in the weights.
// Weight gradient (k_conv3_wgrad_tile + k_wgrad_reduce): per tap
//   dW[t][co][ci] = sum_v dY[v][co] * X[v + off_t][ci]
// over the same halo tiles, with fixed-order partial sums.
// One elected thread issues tcgen05.mma.cta_group::1.kind::f16 (BF16 in,
// FP32 accumulators in tensor memory); completion is tracked with
// tcgen05.commit on mbarriers; every wait is bounded.

#include <cuda_bf16.h>

#include <algorithm>
#include <cstdint>

#include "wg_internal.h"

namespace wg {
namespace {

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

// ---- forward / data gradient: halo tiles, warp-specialised -----------------
//
// A tile is TX x TY output voxels of one z plane (M = 128 GEMM rows, row m =
// voxel (x0 + m % TX, y0 + m / TX, z0)). Its input halo, (TX+2) x (TY+2) x 3
// voxels of KC channels, sits in shared memory as [KC/8][z][y][x][8 channels]
// (16 bytes per voxel and channel group). In that layout the A operand of
// every tap (dx, dy, dz) is the same K-major, no-swizzle matrix shifted by
// 16 * (dx + HX * (dy + HY * dz)) bytes: eight rows of a core matrix are eight
// x-consecutive voxels (16 bytes apart), 8-row groups are HX voxels apart
// (SBO = 16 * HX) and the two 8-channel halves of a 16-channel slice are one
// channel-group plane apart (LBO = 16 * HVOX). So one halo load serves all 27
// taps. The weights come pre-packed as [27][cin/8][cout][8]: the block of
// one tap and one channel chunk is contiguous and is a K-major B operand
// (SBO = 128, LBO = 16 * cout) as it lands, so it is brought in by one bulk
// copy. Roles (320 threads):
//   warps 0-3  halo loads (16-byte cp.async with zero fill outside the box),
//   warp 4     one thread issues the tcgen05.mma of every tap and slice,
//   warp 5     one thread streams the weight blocks (cp.async.bulk),
//   warps 6-9  epilogue: tcgen05.ld of their TMEM lane quarter, bias, ReLU,
//              mask, bf16 stores.
// The CTA is persistent over tiles; the accumulator is double-buffered in
// TMEM so the epilogue of one tile overlaps the MMAs of the next. Every wait
// is bounded: on a time-out the role stops, sets the error flag, and the CTA
// still frees its TMEM after its last MMA has completed.
constexpr int TX = 8, TY = 16;
constexpr int HX = TX + 2, HY = TY + 2;
constexpr int FT = 320;
constexpr int NLOAD = 128;
constexpr int MAXHS = 4, MAXWS = 12;
constexpr int kConvSmem = 227 * 1024;

struct FwdArgs {
  const __nv_bfloat16* x;     // [D][H][W][cin]
  const __nv_bfloat16* w;     // [27][cin/8][cout][8]
  const float* bias;          // [cout] or null
  __nv_bfloat16* y;           // [D][H][W][ystride], channels yoff..yoff+cout-1 written
  float* yf;                  // or, when set, the same in FP32 (y unused)
  const __nv_bfloat16* mask;  // optional [D][H][W][mstride]: y *= (mask > 0)
  int D, H, W, cin, cout, ystride, yoff, mstride, relu;
  int kc, nchunk, hs, ws;     // channels per chunk, chunks, halo stages, weight stages
  int zg, hvox;               // z planes per work item, halo voxels (HX * HY * (zg + 2))
  int ntx, nty, ntz;
  long long ntiles;           // work items: ntx * nty * ntz
  uint32_t tmem_cols;
  int* err;
};

__device__ inline void cp_async16(uint32_t dst, const void* src, int src_bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(src_bytes) : "memory");
}
__device__ inline void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
}
__device__ inline void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ inline void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
// Untiled bulk copy global -> this CTA's shared memory, completing on bar.
__device__ inline void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}

__device__ inline void tile_origin(const FwdArgs& a, long long t, int& x0, int& y0, int& z0) {
  x0 = (int)(t % a.ntx) * TX;
  y0 = (int)((t / a.ntx) % a.nty) * TY;
  z0 = (int)(t / ((long long)a.ntx * a.nty)) * a.zg;
}

__global__ void __launch_bounds__(FT, 1) k_conv3_tile(FwdArgs a) {
  extern __shared__ __align__(1024) unsigned char sm[];
  __shared__ __align__(8) uint64_t hfull[MAXHS], hempty[MAXHS], wfull[MAXWS], wempty[MAXWS], afull[2], aempty[2],
      fin;
  __shared__ uint32_t tmem_s;
  __shared__ int fail_s;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int HVOX = a.hvox;
  const uint32_t halo_bytes = (uint32_t)HVOX * a.kc * 2, w_bytes = (uint32_t)a.cout * a.kc * 2;
  unsigned char* halo = sm;
  unsigned char* wring = sm + (size_t)a.hs * halo_bytes;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_s)),
                 "r"(a.tmem_cols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    for (int i = 0; i < a.hs; ++i) {
      mbar_init(&hfull[i], NLOAD);
      mbar_init(&hempty[i], 1);
    }
    for (int i = 0; i < a.ws; ++i) {
      mbar_init(&wfull[i], 1);
      mbar_init(&wempty[i], 1);
    }
    for (int i = 0; i < 2; ++i) {
      mbar_init(&afull[i], 1);
      mbar_init(&aempty[i], 128);
    }
    mbar_init(&fin, 1);
    fail_s = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_s;
  bool ok = true;
  if (warp < 4) {
    // halo loads
    const int cg8 = a.kc >> 3;
    long long j = 0;
    for (long long t = blockIdx.x; t < a.ntiles && ok; t += gridDim.x) {
      int x0, y0, z0;
      tile_origin(a, t, x0, y0, z0);
      for (int c = 0; c < a.nchunk; ++c, ++j) {
        const int hb = (int)(j % a.hs);
        const long long r = j / a.hs;
        if (r >= 1 && !mbar_wait(&hempty[hb], (uint32_t)((r - 1) & 1))) {
          ok = false;
          break;
        }
        const uint32_t dst = smem_u32(halo + (size_t)hb * halo_bytes);
        for (int p = tid; p < HVOX * cg8; p += NLOAD) {
          const int cg = p % cg8, v = p / cg8;
          const int gx = x0 - 1 + v % HX, gy = y0 - 1 + (v / HX) % HY, gz = z0 - 1 + v / (HX * HY);
          const bool in = gx >= 0 && gx < a.W && gy >= 0 && gy < a.H && gz >= 0 && gz < a.D;
          const __nv_bfloat16* src =
              in ? a.x + (((long long)gz * a.H + gy) * a.W + gx) * a.cin + c * a.kc + cg * 8 : a.x;
          cp_async16(dst + (uint32_t)(cg * HVOX + v) * 16u, src, in ? 16 : 0);
        }
        cp_async_wait_all();
        fence_async_smem();
        mbar_arrive(&hfull[hb]);
      }
    }
  } else if (warp == 5) {
    // weight blocks
    if (lane == 0) {
      long long q = 0;
      for (long long t = blockIdx.x; t < a.ntiles && ok; t += gridDim.x) {
        for (int c = 0; c < a.nchunk && ok; ++c) {
          for (int tap = 0; tap < 27; ++tap, ++q) {
            const int ws = (int)(q % a.ws);
            const long long r = q / a.ws;
            if (r >= 1 && !mbar_wait(&wempty[ws], (uint32_t)((r - 1) & 1))) {
              ok = false;
              break;
            }
            mbar_expect_tx(&wfull[ws], w_bytes);
            const __nv_bfloat16* src = a.w + ((size_t)tap * (a.cin >> 3) + (size_t)c * (a.kc >> 3)) * a.cout * 8;
            bulk_g2s(smem_u32(wring + (size_t)ws * w_bytes), src, w_bytes, &wfull[ws]);
          }
        }
      }
    }
  } else if (warp == 4) {
    // MMA issue
    if (lane == 0) {
      const uint32_t idesc = make_idesc(128, a.cout);
      long long j = 0, q = 0, li = 0;
      for (long long t = blockIdx.x; t < a.ntiles && ok; t += gridDim.x, ++li) {
        const int ab = (int)(li & 1);
        const long long ar = li >> 1;
        if (ar >= 1 && !mbar_wait(&aempty[ab], (uint32_t)((ar - 1) & 1))) {
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t dcol = tmem + (uint32_t)(ab * a.zg * a.cout);
        for (int c = 0; c < a.nchunk && ok; ++c, ++j) {
          const int hb = (int)(j % a.hs);
          if (!mbar_wait(&hfull[hb], (uint32_t)((j / a.hs) & 1))) {
            ok = false;
            break;
          }
          tc_fence_after();
          // Descriptors are built once per halo and weight slot; the start
          // address field (bits 0-13, 16-byte units) is then advanced by plain
          // adds (every shared address here is below 256 KB, so the field
          // never carries into the next one).
          const uint64_t ad0 = make_sdesc(smem_u32(halo + (size_t)hb * halo_bytes), (uint32_t)HVOX * 16u, HX * 16);
          const int nsl = a.kc >> 4;
          for (int tap = 0; tap < 27; ++tap, ++q) {
            const int ws = (int)(q % a.ws);
            if (!mbar_wait(&wfull[ws], (uint32_t)((q / a.ws) & 1))) {
              ok = false;
              break;
            }
            tc_fence_after();
            const int dz = tap / 9, dy = (tap / 3) % 3, dx = tap % 3;  // offsets + 1
            const uint64_t bd0 = make_sdesc(smem_u32(wring + (size_t)ws * w_bytes), (uint32_t)a.cout * 16u, 128u);
            // one weight block feeds the zg planes of the work item
            uint64_t adp = ad0 + (uint64_t)(dx + HX * (dy + HY * dz));
            uint32_t dc = dcol;
            for (int i = 0; i < a.zg; ++i, adp += HX * HY, dc += (uint32_t)a.cout) {
              uint64_t ad = adp, bd = bd0;
              for (int sl = 0; sl < nsl; ++sl, ad += 2 * HVOX, bd += 2 * a.cout)
                umma_f16(dc, ad, bd, idesc, (c | tap | sl) ? 1u : 0u);
            }
            umma_commit(&wempty[ws]);
          }
          umma_commit(&hempty[hb]);
        }
        umma_commit(&afull[ab]);
      }
      // no MMA may still run when the TMEM is freed
      umma_commit(&fin);
      if (!mbar_wait(&fin, 0)) ok = false;
    }
  } else if (warp >= 6) {
    // epilogue
    const int qtr = warp & 3;
    const int m = 32 * qtr + lane;
    long long li = 0;
    for (long long t = blockIdx.x; t < a.ntiles && ok; t += gridDim.x, ++li) {
      const int ab = (int)(li & 1);
      if (!mbar_wait(&afull[ab], (uint32_t)((li >> 1) & 1))) {
        ok = false;
        break;
      }
      tc_fence_after();
      int x0, y0, z0;
      tile_origin(a, t, x0, y0, z0);
      const int ox = x0 + (m % TX), oy = y0 + m / TX;
      for (int i = 0; i < a.zg; ++i)
      for (int c0 = 0; c0 < a.cout; c0 += 16) {
        const bool valid = ox < a.W && oy < a.H && z0 + i < a.D;
        const long long v = ((long long)(z0 + i) * a.H + oy) * a.W + ox;
        float f[16];
        tmem_ld16(tmem + ((uint32_t)(32 * qtr) << 16) + (uint32_t)((ab * a.zg + i) * a.cout + c0), f);
        if (valid) {
#pragma unroll
          for (int i = 0; i < 16; ++i) {
            float r = f[i] + (a.bias ? a.bias[c0 + i] : 0.f);
            if (a.relu) r = fmaxf(r, 0.f);
            if (a.mask && !(__bfloat162float(a.mask[v * a.mstride + c0 + i]) > 0.f)) r = 0.f;
            f[i] = r;
          }
          if (a.yf) {
            float* dst = a.yf + v * a.ystride + a.yoff + c0;
#pragma unroll
            for (int q = 0; q < 4; ++q) reinterpret_cast<float4*>(dst)[q] = reinterpret_cast<float4*>(f)[q];
          } else {
            __nv_bfloat16 out[16];
#pragma unroll
            for (int i = 0; i < 16; ++i) out[i] = __float2bfloat16_rn(f[i]);
            __nv_bfloat16* dst = a.y + v * a.ystride + a.yoff + c0;
            *reinterpret_cast<uint4*>(dst) = *reinterpret_cast<uint4*>(&out[0]);
            *reinterpret_cast<uint4*>(dst + 8) = *reinterpret_cast<uint4*>(&out[8]);
          }
        }
      }
      tc_fence_before();
      mbar_arrive(&aempty[ab]);
    }
  }
  if (!ok) atomicOr(&fail_s, 1);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (tid == 0 && fail_s) atomicOr(a.err, 1);
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(a.tmem_cols));
}

// ---- weight gradient: halo tiles, MN-major operands, fixed-order partials --
//
// dW[t][co][ci] = sum_v dY[v][co] * X[v + off_t][ci]: per tap a GEMM with
// M = co (padded to 128 rows), N = ci and K = voxels. Both operands are read
// in the NDHWC layout as MN-major UMMA matrices (a 16-byte row holds 8
// channels of one voxel; eight K rows are eight voxels): the dY tile as
// [co/8][128 voxels][8] (row groups SBO = 2048 B apart, K groups LBO = 128 B),
// the X halo as in the forward kernel, [ci/8][z][y][x][8] (SBO = 16 * HVOX,
// and the K groups of the tile's voxel order, one y row of 8 voxels each, are
// LBO = 16 * HX apart), shifted per tap by the same byte offsets. A CTA takes
// a group of TG taps (TG * cin TMEM columns of accumulators) and a fixed
// share of the tiles, accumulates over them in TMEM, and writes its partial
// sums to its own slice of a scratch array; k_wgrad_reduce then adds the
// slices in a fixed order, so dW is the same bits on every run.
struct WgArgs {
  const __nv_bfloat16* x;   // [D][H][W][cin]
  const __nv_bfloat16* dy;  // [D][H][W][cout]
  float* part;              // [nsplit][27][cout][cin]
  int D, H, W, cin, cout;
  int kc, nchunk, tg, ntg, nsplit, hvox;
  int ntx, nty;
  long long ntiles;
  uint32_t tmem_cols;
  int* err;
};

constexpr int WG_ABYTES = 128 * 128 * 2;  // dY tile: 128 voxels x 128 (padded) channels

__global__ void __launch_bounds__(FT, 1) k_conv3_wgrad_tile(WgArgs a) {
  extern __shared__ __align__(1024) unsigned char sm[];
  __shared__ __align__(8) uint64_t sfull[2], sempty[2], fin;
  __shared__ uint32_t tmem_s;
  __shared__ int fail_s;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int HVOX = a.hvox;
  const uint32_t halo_bytes = (uint32_t)HVOX * a.kc * 2, stage_bytes = WG_ABYTES + halo_bytes;
  const int tg0 = (blockIdx.x % a.ntg) * a.tg;                 // first tap of this CTA's group
  const int ntap = min(a.tg, 27 - tg0);
  const int split = blockIdx.x / a.ntg;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_s)),
                 "r"(a.tmem_cols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    for (int i = 0; i < 2; ++i) {
      mbar_init(&sfull[i], NLOAD);
      mbar_init(&sempty[i], 1);
    }
    mbar_init(&fin, 1);
    fail_s = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_s;
  bool ok = true;
  if (warp < 4) {
    // loads: the dY tile (all channels, zero above cout and outside the box)
    // and the X halo of one channel chunk, per stage
    const int cg8 = a.kc >> 3;
    long long j = 0;
    for (long long t = split; t < a.ntiles && ok; t += a.nsplit) {
      const int x0 = (int)(t % a.ntx) * TX, y0 = (int)((t / a.ntx) % a.nty) * TY;
      const int z0 = (int)(t / ((long long)a.ntx * a.nty));
      for (int c = 0; c < a.nchunk; ++c, ++j) {
        const int sb = (int)(j & 1);
        const long long r = j >> 1;
        if (r >= 1 && !mbar_wait(&sempty[sb], (uint32_t)((r - 1) & 1))) {
          ok = false;
          break;
        }
        const uint32_t sa = smem_u32(sm + (size_t)sb * stage_bytes), sh = sa + WG_ABYTES;
        for (int p = tid; p < 16 * 128; p += NLOAD) {
          const int cog = p >> 7, m = p & 127;
          const int gx = x0 + (m % TX), gy = y0 + m / TX;
          const bool in = gx < a.W && gy < a.H && 8 * cog < a.cout;
          const __nv_bfloat16* src = in ? a.dy + (((long long)z0 * a.H + gy) * a.W + gx) * a.cout + 8 * cog : a.dy;
          cp_async16(sa + (uint32_t)(cog * 128 + m) * 16u, src, in ? 16 : 0);
        }
        for (int p = tid; p < HVOX * cg8; p += NLOAD) {
          const int cg = p % cg8, v = p / cg8;
          const int gx = x0 - 1 + v % HX, gy = y0 - 1 + (v / HX) % HY, gz = z0 - 1 + v / (HX * HY);
          const bool in = gx >= 0 && gx < a.W && gy >= 0 && gy < a.H && gz >= 0 && gz < a.D;
          const __nv_bfloat16* src =
              in ? a.x + (((long long)gz * a.H + gy) * a.W + gx) * a.cin + c * a.kc + cg * 8 : a.x;
          cp_async16(sh + (uint32_t)(cg * HVOX + v) * 16u, src, in ? 16 : 0);
        }
        cp_async_wait_all();
        fence_async_smem();
        mbar_arrive(&sfull[sb]);
      }
    }
  } else if (warp == 4) {
    if (lane == 0) {
      // M = 128 (co), N = kc (ci of the chunk), both operands MN-major
      const uint32_t idesc = make_idesc(128, a.kc) | (1u << 15) | (1u << 16);
      long long j = 0;
      bool first = true;
      for (long long t = split; t < a.ntiles && ok; t += a.nsplit) {
        for (int c = 0; c < a.nchunk && ok; ++c, ++j) {
          const int sb = (int)(j & 1);
          if (!mbar_wait(&sfull[sb], (uint32_t)((j >> 1) & 1))) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t sa = smem_u32(sm + (size_t)sb * stage_bytes), sh = sa + WG_ABYTES;
          const uint64_t ad0 = make_sdesc(sa, 128u, 2048u);
          const uint64_t bd0 = make_sdesc(sh, (uint32_t)HX * 16u, (uint32_t)HVOX * 16u);
          for (int i = 0; i < ntap; ++i) {
            const int tap = tg0 + i;
            const int dz = tap / 9, dy = (tap / 3) % 3, dx = tap % 3;
            const uint64_t bt = bd0 + (uint64_t)(dx + HX * (dy + HY * dz));
            const uint32_t dcol = tmem + (uint32_t)(i * a.cin + c * a.kc);
            // K = 128 voxels of the tile in 8 steps of two y rows
            for (int k = 0; k < 8; ++k)
              umma_f16(dcol, ad0 + (uint64_t)(16 * k), bt + (uint64_t)(2 * k * HX), idesc,
                       (first && k == 0) ? 0u : 1u);
          }
          umma_commit(&sempty[sb]);
          // the first MMA of every accumulator column block overwrites it
          if (c == a.nchunk - 1) first = false;
        }
      }
      umma_commit(&fin);
      if (!mbar_wait(&fin, 0)) ok = false;
    }
  } else if (warp >= 6) {
    // wait for the last MMA (fin is committed after it), then write the
    // partial sums of rows co < cout
    const int qtr = warp & 3;
    const int co = 32 * qtr + lane;
    if (!mbar_wait(&fin, 0)) ok = false;
    tc_fence_after();
    const bool any = split < a.ntiles;
    for (int i = 0; i < ntap && ok; ++i)
      for (int c0 = 0; c0 < a.cin; c0 += 16) {
        float f[16];
        tmem_ld16(tmem + ((uint32_t)(32 * qtr) << 16) + (uint32_t)(i * a.cin + c0), f);
        if (co < a.cout) {
          float* dst = a.part + (((size_t)split * 27 + tg0 + i) * a.cout + co) * a.cin + c0;
#pragma unroll
          for (int q = 0; q < 16; ++q) dst[q] = any ? f[q] : 0.f;
        }
      }
  }
  if (!ok) atomicOr(&fail_s, 1);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (tid == 0 && fail_s) atomicOr(a.err, 1);
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(a.tmem_cols));
}

// dw[i] = sum over the splits of part[s][i], in split order.
__global__ void k_wgrad_reduce(const float* __restrict__ part, float* __restrict__ dw, size_t n, int nsplit) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    float acc = 0.f;
    for (int s = 0; s < nsplit; ++s) acc += part[(size_t)s * n + i];
    dw[i] = acc;
  }
}

// Work split of the weight gradient: taps per CTA group (their accumulators
// fill at most 512 TMEM columns), tap groups, and tile splits per group.
void wgrad_plan(int cin, int nsm, int* tg, int* ntg, int* nsplit) {
  *tg = std::min(27, 512 / cin);
  *ntg = (27 + *tg - 1) / *tg;
  *nsplit = std::max(1, (nsm + *ntg - 1) / *ntg);
}

}  // namespace
}  // namespace wg

using namespace wg;

namespace {
// wg_conv3_fwd and wg_conv3_fwd_f32: y is bf16 or, with f32, float.
int conv3_fwd(const void* x, int D, int H, int W, int cin, const void* w, const float* bias, int cout, void* y,
              int ystride, int yoff, const void* mask, int mstride, int relu, int* err, void* stream, bool f32) {
  // a row of y starts 16-byte aligned: 8 bf16 or 4 float channels
  const int ya = f32 ? 4 : 8;
  if (!x || !w || !y || !err || D < 1 || H < 1 || W < 1 || cin < 16 || cin % 16 || cout < 16 || cout > 256 ||
      cout % 16 || ystride < yoff + cout || (yoff % ya) || (ystride % ya) || (mask && mstride < cout)) {
    set_error("wg_conv3_fwd: bad arguments (cin, cout multiples of 16, cout <= 256, 16-byte aligned rows)");
    return WG_EINVAL;
  }
  if (((uintptr_t)x | (uintptr_t)w | (uintptr_t)y) & 15) {
    set_error("wg_conv3_fwd: x, w and y must be 16-byte aligned");
    return WG_EINVAL;
  }
  // dynamic shared memory: the opt-in limit less the kernel's static part
  int dev = 0, nsm = 0, optin = 0;
  WG_TRY_CUDA(cudaGetDevice(&dev));
  WG_TRY_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  WG_TRY_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  cudaFuncAttributes fa{};
  WG_TRY_CUDA(cudaFuncGetAttributes(&fa, k_conv3_tile));
  const int smem_max = std::min(kConvSmem, optin - (int)fa.sharedSizeBytes);
  FwdArgs a{};
  a.x = (const __nv_bfloat16*)x;
  a.w = (const __nv_bfloat16*)w;
  a.bias = bias;
  a.y = f32 ? nullptr : (__nv_bfloat16*)y;
  a.yf = f32 ? (float*)y : nullptr;
  a.mask = (const __nv_bfloat16*)mask;
  a.D = D;
  a.H = H;
  a.W = W;
  a.cin = cin;
  a.cout = cout;
  a.ystride = ystride;
  a.yoff = yoff;
  a.mstride = mstride;
  a.relu = relu;
  a.err = err;
  // channels per halo chunk: the largest of 64, 48, 32, 16 that divides cin
  a.kc = cin % 64 == 0 ? 64 : cin % 48 == 0 ? 48 : cin % 32 == 0 ? 32 : 16;
  a.nchunk = cin / a.kc;
  // z planes per work item: each weight block then feeds zg accumulators
  // (2 * zg * cout TMEM columns, double-buffered). Take the largest zg <= 4
  // whose two halo stages leave room for at least four weight stages; zg = 1
  // with the fewest stages that fit otherwise.
  const int w_bytes = cout * a.kc * 2;
  a.zg = 0;
  for (int zg = 4; zg >= 1 && !a.zg; --zg) {
    const int hb = HX * HY * (zg + 2) * a.kc * 2;
    if (2 * zg * cout <= 512 && 2 * hb + 4 * w_bytes <= smem_max && zg <= D) a.zg = zg;
  }
  if (!a.zg) a.zg = 1;
  a.hvox = HX * HY * (a.zg + 2);
  const int halo_bytes = a.hvox * a.kc * 2;
  a.hs = 2;
  while (a.hs < MAXHS && (a.hs + 1) * halo_bytes + 4 * w_bytes <= smem_max / 2) ++a.hs;
  a.ws = std::min(MAXWS, (smem_max - a.hs * halo_bytes) / w_bytes);
  if (a.ws < 2) {
    set_error("wg_conv3_fwd: cout too large for the shared-memory stages");
    return WG_EINVAL;
  }
  uint32_t cols = 32;
  while ((int)cols < 2 * a.zg * cout) cols <<= 1;
  a.tmem_cols = cols;
  a.ntx = (W + TX - 1) / TX;
  a.nty = (H + TY - 1) / TY;
  a.ntz = (D + a.zg - 1) / a.zg;
  a.ntiles = (long long)a.ntx * a.nty * a.ntz;
  const int smem = a.hs * halo_bytes + a.ws * w_bytes;
  WG_TRY_CUDA(cudaFuncSetAttribute(k_conv3_tile, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  const long long grid = std::min<long long>(a.ntiles, nsm);
  k_conv3_tile<<<(unsigned)grid, FT, smem, (cudaStream_t)stream>>>(a);
  WG_TRY_CUDA(cudaGetLastError());
  return WG_OK;
}
}  // namespace

extern "C" {


int wg_conv3_fwd(const void* x, int D, int H, int W, int cin, const void* w, const float* bias, int cout, void* y,
                 int ystride, int yoff, const void* mask, int mstride, int relu, int* err, void* stream) {
  return conv3_fwd(x, D, H, W, cin, w, bias, cout, y, ystride, yoff, mask, mstride, relu, err, stream, false);
}

int wg_conv3_fwd_f32(const void* x, int D, int H, int W, int cin, const void* w, const float* bias, int cout,
                     float* y, int ystride, int yoff, const void* mask, int mstride, int relu, int* err,
                     void* stream) {
  return conv3_fwd(x, D, H, W, cin, w, bias, cout, y, ystride, yoff, mask, mstride, relu, err, stream, true);
}

int wg_conv3_wgrad_scratch(int cin, int cout, int64_t* nfloats) {
  if (!nfloats || cin < 16 || cin % 16 || cin > 256 || cout < 16 || cout % 16 || cout > 128) {
    set_error("wg_conv3_wgrad_scratch: bad arguments (cin multiple of 16 up to 256, cout multiple of 16 up to 128)");
    return WG_EINVAL;
  }
  int dev = 0, nsm = 0, tg, ntg, nsplit;
  WG_TRY_CUDA(cudaGetDevice(&dev));
  WG_TRY_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  wgrad_plan(cin, nsm, &tg, &ntg, &nsplit);
  *nfloats = (int64_t)nsplit * 27 * cout * cin;
  return WG_OK;
}

int wg_conv3_wgrad(const void* x, const void* dy, int D, int H, int W, int cin, int cout, float* dw, float* scratch,
                   int64_t scratch_floats, int* err, void* stream) {
  if (!x || !dy || !dw || !scratch || !err || D < 1 || H < 1 || W < 1 || cin < 16 || cin % 16 || cin > 256 ||
      cout < 16 || cout % 16 || cout > 128) {
    set_error("wg_conv3_wgrad: bad arguments (cin multiple of 16 up to 256, cout multiple of 16 up to 128)");
    return WG_EINVAL;
  }
  if (((uintptr_t)x | (uintptr_t)dy) & 15) {
    set_error("wg_conv3_wgrad: x and dy must be 16-byte aligned");
    return WG_EINVAL;
  }
  int dev = 0, nsm = 0, optin = 0;
  WG_TRY_CUDA(cudaGetDevice(&dev));
  WG_TRY_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  WG_TRY_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  WgArgs a{};
  a.x = (const __nv_bfloat16*)x;
  a.dy = (const __nv_bfloat16*)dy;
  a.part = scratch;
  a.D = D;
  a.H = H;
  a.W = W;
  a.cin = cin;
  a.cout = cout;
  a.err = err;
  a.kc = cin % 64 == 0 ? 64 : cin % 48 == 0 ? 48 : cin % 32 == 0 ? 32 : 16;
  a.nchunk = cin / a.kc;
  a.hvox = HX * HY * 3;
  wgrad_plan(cin, nsm, &a.tg, &a.ntg, &a.nsplit);
  if (scratch_floats < (int64_t)a.nsplit * 27 * cout * cin) {
    set_error("wg_conv3_wgrad: scratch smaller than wg_conv3_wgrad_scratch reports");
    return WG_EINVAL;
  }
  uint32_t cols = 32;
  while ((int)cols < a.tg * cin) cols <<= 1;
  a.tmem_cols = cols;
  a.ntx = (W + TX - 1) / TX;
  a.nty = (H + TY - 1) / TY;
  a.ntiles = (long long)a.ntx * a.nty * D;
  const int smem = 2 * (WG_ABYTES + a.hvox * a.kc * 2);
  cudaFuncAttributes fa{};
  WG_TRY_CUDA(cudaFuncGetAttributes(&fa, k_conv3_wgrad_tile));
  if (smem > optin - (int)fa.sharedSizeBytes) {
    set_error("wg_conv3_wgrad: shared-memory stages do not fit");
    return WG_EINVAL;
  }
  WG_TRY_CUDA(cudaFuncSetAttribute(k_conv3_wgrad_tile, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  k_conv3_wgrad_tile<<<(unsigned)(a.ntg * a.nsplit), FT, smem, (cudaStream_t)stream>>>(a);
  WG_TRY_CUDA(cudaGetLastError());
  const size_t n = (size_t)27 * cout * cin;
  k_wgrad_reduce<<<(unsigned)std::min<size_t>((n + 255) / 256, 1024), 256, 0, (cudaStream_t)stream>>>(scratch, dw, n,
                                                                                                     a.nsplit);
  WG_TRY_CUDA(cudaGetLastError());
  return WG_OK;
}

}  // extern "C"
