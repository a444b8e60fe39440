// BF16 tensor-core MLP kernels for the learned corrector: one GEMM kernel on
// the 5th-generation tensor cores (tcgen05.mma, accumulator in tensor
// memory) with fused epilogues, and the elementwise kernels of training
// (loss gradient, bias gradient, Adam).  Declarations: include/hexmlp.h.
//
// GEMM: C[M][N] = A[M][K] . B[N][K]^T with A and B bf16, both K-contiguous
// ("K-major"), FP32 accumulation.  Every product of the network is cast in
// this form by keeping transposed copies where needed (W^T for the input
// gradient, H^T and dZ^T for the weight gradient), so one kernel serves the
// forward pass and both backward products.
//
// Tiling: a CTA of 256 threads owns a 128 x BN output tile (BN = 128 or
// 256) whose FP32 accumulator lives in BN columns of tensor memory (128
// lanes = 128 rows).  K advances in 64-element slabs through NSTAGE shared
// memory stages filled by asynchronous 16-byte copies (cp.async) in the
// canonical K-major no-swizzle layout (8-row x 16-byte core matrices; the
// descriptor's leading offset steps along K, the stride offset along rows):
// the copies of the next NSTAGE-1 slabs are in flight while the tensor core
// works on the current one.  One thread issues four K=16 MMAs per slab and
// commits them to the stage's mbarrier; a stage is refilled once that
// mbarrier completes.  The epilogue reads the accumulator with tcgen05.ld
// (warp w may read lanes 32(w%4)..32(w%4)+31, so warps w and w+4 split that
// lane quarter's columns in halves), applies bias / GELU / GELU' and stores.
//
// GELU is the tanh form, 0.5 x (1 + tanh(sqrt(2/pi) (x + 0.044715 x^3))),
// evaluated with the hardware tanh approximation (tanh.approx.f32).
//
// Every wait on an mbarrier is bounded: past the limit the kernel records
// an error in *err, stops issuing work, waits (bounded again) for its own
// MMAs, frees its tensor memory and returns.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

#include "../../include/hexmlp.h"

namespace {

constexpr int BM = 128;
constexpr int BK = 64;
constexpr int THREADS = 256;
constexpr int NSTAGE = 3;
constexpr uint32_t WAIT_LIMIT = 1u << 20;  // try_wait polls before an mbarrier wait gives up

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor, K-major, no swizzle (layout type 0),
// version 1; offsets in 16-byte units.
__device__ __forceinline__ uint64_t umma_desc(uint32_t addr, uint32_t lbo_bytes, uint32_t sbo_bytes) {
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo_bytes >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo_bytes >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}

// Instruction descriptor of kind::f16: BF16 A and B, FP32 D, both K-major.
__host__ __device__ constexpr uint32_t umma_idesc(int m, int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0));
}

__device__ __forceinline__ void mma_commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
               : "memory");
}

__device__ __forceinline__ void mbar_init(uint32_t mbar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar), "r"(count));
}

__device__ __forceinline__ bool mbar_try(uint32_t mbar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(done)
      : "r"(mbar), "r"(parity)
      : "memory");
  return done != 0;
}

// Bounded wait for the completion of phase `parity`; false when it gave up.
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity) {
  for (uint32_t i = 0; i < WAIT_LIMIT; ++i)
    if (mbar_try(mbar, parity)) return true;
  return false;
}

// As mbar_wait with at most `limit` polls, giving up early once another
// role of the CTA has raised its abort word (checked every 64 polls).
__device__ __forceinline__ bool mbar_wait_or_abort(uint32_t mbar, uint32_t parity, volatile int* abort_word,
                                                   uint32_t limit) {
  for (uint32_t i = 0; i < limit; ++i) {
    if (mbar_try(mbar, parity)) return true;
    if ((i & 63u) == 63u && *abort_word) return false;
  }
  return false;
}

// 32 consecutive accumulator columns of this thread's lane
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float* v) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ float tanh_hw(float x) {
  float y;
  asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
constexpr float GELU_C = 0.7978845608028654f;  // sqrt(2/pi)
constexpr float GELU_CA = 0.7978845608028654f * 0.044715f;
// tanh argument sqrt(2/pi) (x + 0.044715 x^3) written as x (C + C A x^2)
__device__ __forceinline__ float gelu(float x) {
  const float hx = 0.5f * x;
  return __fmaf_rn(hx, tanh_hw(x * __fmaf_rn(GELU_CA, x * x, GELU_C)), hx);
}
__device__ __forceinline__ float gelu_grad(float x) {
  const float x2 = x * x;
  const float t = tanh_hw(x * __fmaf_rn(GELU_CA, x2, GELU_C));
  // 0.5 (1 + t) + 0.5 x (1 - t^2) (C + 3 C A x^2)
  return __fmaf_rn(0.5f * x * __fmaf_rn(-t, t, 1.0f), __fmaf_rn(3.0f * GELU_CA, x2, GELU_C), __fmaf_rn(0.5f, t, 0.5f));
}

// Asynchronous copy of a rows x 64 slab (K-contiguous rows of length ld)
// into the canonical layout: chunk (r, kc) of 8 elements at
// (r/8)*1024 + kc*128 + (r%8)*16.
__device__ __forceinline__ void load_slab(uint8_t* dst, const __nv_bfloat16* src, int rows, int ld, int k0) {
  const int chunks = rows * (BK / 8);
  for (int i = threadIdx.x; i < chunks; i += THREADS) {
    const int r = i >> 3, kc = i & 7;
    const void* g = src + (size_t)r * ld + k0 + kc * 8;
    const uint32_t d = smem_u32(dst + (r >> 3) * 1024 + kc * 128 + (r & 7) * 16);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(g) : "memory");
  }
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

using bf16 = __nv_bfloat16;

// Kernel-side view of HexMlpGemm with typed pointers.
struct Gemm {
  const bf16* A;
  const bf16* B;
  int M, N, K, bn, epilogue;
  const float* bias;
  bf16* C;
  bf16* Ct;
  bf16* Z;
  const bf16* Zin;
  float* Cf;
  int* err;
  uint32_t mma_wait_polls;  // polls of the MMA issuer's wait for a loaded stage (WAIT_LIMIT normally)
};

// Epilogue of 8 accumulator columns of one row: bias, then the selected
// epilogue, stores of C / C^T / Z / Cf (shared by both GEMM kernels).
__device__ __forceinline__ void epilogue8(const Gemm& p, int row, int col, float* v, uint4* c_out = nullptr,
                                          float4* f_out = nullptr) {
  if (p.bias) {
    // the same 8 bias words for every lane of the warp: two broadcast 128-bit loads
    const float4 b0 = __ldg(reinterpret_cast<const float4*>(p.bias + col));
    const float4 b1 = __ldg(reinterpret_cast<const float4*>(p.bias + col + 4));
    v[0] += b0.x;
    v[1] += b0.y;
    v[2] += b0.z;
    v[3] += b0.w;
    v[4] += b1.x;
    v[5] += b1.y;
    v[6] += b1.z;
    v[7] += b1.w;
  }
  if (p.epilogue == HEXMLP_EPI_GELU) {
    __nv_bfloat16 z[8], h[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      z[i] = __float2bfloat16_rn(v[i]);
      h[i] = __float2bfloat16_rn(gelu(v[i]));
    }
    if (p.Z) *reinterpret_cast<uint4*>(p.Z + (size_t)row * p.N + col) = *reinterpret_cast<uint4*>(z);
    if (c_out)
      *c_out = *reinterpret_cast<uint4*>(h);  // the caller stores C
    else if (p.C)
      *reinterpret_cast<uint4*>(p.C + (size_t)row * p.N + col) = *reinterpret_cast<uint4*>(h);
    if (p.Ct) {
#pragma unroll
      for (int i = 0; i < 8; ++i) p.Ct[(size_t)(col + i) * p.M + row] = h[i];
    }
  } else if (p.epilogue == HEXMLP_EPI_GELU_GRAD) {
    __nv_bfloat16 d[8];
    const uint4 zr = *reinterpret_cast<const uint4*>(p.Zin + (size_t)row * p.N + col);
    const __nv_bfloat16* zz = reinterpret_cast<const __nv_bfloat16*>(&zr);
#pragma unroll
    for (int i = 0; i < 8; ++i) d[i] = __float2bfloat16_rn(v[i] * gelu_grad(__bfloat162float(zz[i])));
    if (p.C) *reinterpret_cast<uint4*>(p.C + (size_t)row * p.N + col) = *reinterpret_cast<uint4*>(d);
    if (p.Ct) {
#pragma unroll
      for (int i = 0; i < 8; ++i) p.Ct[(size_t)(col + i) * p.M + row] = d[i];
    }
  } else {
    float4* dst = f_out ? f_out : reinterpret_cast<float4*>(p.Cf + (size_t)row * p.N + col);  // f_out: caller stores
    dst[0] = make_float4(v[0], v[1], v[2], v[3]);
    dst[1] = make_float4(v[4], v[5], v[6], v[7]);
    if (p.C) {
      __nv_bfloat16 b[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) b[i] = __float2bfloat16_rn(v[i]);
      *reinterpret_cast<uint4*>(p.C + (size_t)row * p.N + col) = *reinterpret_cast<uint4*>(b);
    }
  }
}

__global__ void __launch_bounds__(THREADS, 2) k_gemm_bf16(Gemm p) {
  extern __shared__ __align__(1024) uint8_t smem[];
  const int BN = p.bn;
  const int m0 = blockIdx.x * BM, n0 = blockIdx.y * BN;
  const int nk = p.K / BK;
  const int stage_bytes = (BM + BN) * BK * 2;
  auto stage_a = [&](int s) { return smem + s * stage_bytes; };
  auto stage_b = [&](int s) { return smem + s * stage_bytes + BM * BK * 2; };
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + NSTAGE * stage_bytes);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + NSTAGE);
  int& s_failed = *reinterpret_cast<int*>(tmem_slot + 1);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  if (threadIdx.x == 0) {
    for (int s = 0; s < NSTAGE; ++s) mbar_init(smem_u32(&bars[s]), 1);
    s_failed = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    // BN columns of tensor memory (128 or 256, a power of two as required)
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(BN));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;
  const uint32_t idesc = umma_idesc(BM, BN);

  const __nv_bfloat16* A = p.A + (size_t)m0 * p.K;
  const __nv_bfloat16* B = p.B + (size_t)n0 * p.K;
  int issued = 0;  // slabs whose MMAs were issued
  // prologue: the first NSTAGE-1 slabs in flight (one commit group each)
  for (int q = 0; q < NSTAGE - 1; ++q) {
    if (q < nk) {
      load_slab(stage_a(q), A, BM, p.K, q * BK);
      load_slab(stage_b(q), B, BN, p.K, q * BK);
    }
    cp_commit();
  }
  for (int kt = 0; kt < nk; ++kt) {
    const int s = kt % NSTAGE;
    cp_wait<NSTAGE - 2>();  // this thread's copies of slab kt have landed
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (threadIdx.x == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t a0 = smem_u32(stage_a(s)), b0 = smem_u32(stage_b(s));
#pragma unroll
      for (int j = 0; j < BK / 16; ++j) {
        // K = 16 per MMA: two 8-element core-matrix columns, 256 bytes apart
        const uint64_t ad = umma_desc(a0 + j * 256, 128, 1024);
        const uint64_t bd = umma_desc(b0 + j * 256, 128, 1024);
        mma_bf16(tmem, ad, bd, idesc, (kt > 0 || j > 0) ? 1u : 0u);
      }
      mma_commit(smem_u32(&bars[s]));
    }
    issued = kt + 1;
    // refill the stage of slab kt-1 with slab kt+NSTAGE-1 once slab kt-1's
    // MMAs (committed one iteration ago) are complete
    const int nxt = kt + NSTAGE - 1;
    if (nxt < nk) {
      const int sn = nxt % NSTAGE;
      if (kt >= 1 && threadIdx.x == 0 && !mbar_wait(smem_u32(&bars[sn]), ((kt - 1) / NSTAGE) & 1)) s_failed = 1;
      __syncthreads();
      if (s_failed) break;
      load_slab(stage_a(sn), A, BM, p.K, nxt * BK);
      load_slab(stage_b(sn), B, BN, p.K, nxt * BK);
    }
    cp_commit();
  }
  cp_wait<0>();
  // wait for the last commit: every MMA issued before it is then complete
  __syncthreads();
  if (threadIdx.x == 0 && issued > 0) {
    const int last = issued - 1;
    if (!mbar_wait(smem_u32(&bars[last % NSTAGE]), (last / NSTAGE) & 1)) s_failed = 1;
  }
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const bool ok = s_failed == 0 && issued == nk;
  if (!ok && threadIdx.x == 0) atomicOr(p.err, 1);

  if (ok) {
    const int quarter = warp & 3, half = warp >> 2;
    const int row = m0 + quarter * 32 + lane;
    const uint32_t lane_base = tmem + ((uint32_t)(quarter * 32) << 16);
    for (int c32 = half * (BN / 2); c32 < (half + 1) * (BN / 2); c32 += 32) {
      float v32[32];
      tmem_ld32(lane_base + (uint32_t)c32, v32);
#pragma unroll
      for (int g8 = 0; g8 < 4; ++g8) {
      float* v = v32 + 8 * g8;
      const int col = n0 + c32 + 8 * g8;
      epilogue8(p, row, col, v);
      }
    }
  } else if (threadIdx.x == 0 && issued > 0) {
    // gave up: a last bounded wait for this CTA's own MMAs before freeing
    const int last = issued - 1;
    mbar_wait(smem_u32(&bars[last % NSTAGE]), (last / NSTAGE) & 1);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(BN));
  }
}

// ---------------------------------------------------------------------------
// Persistent warp-specialised GEMM.  One CTA per SM loops over output tiles
// (128 x BN, n fastest so that consecutive tiles reuse the same A rows from
// L2).  Warp 0 (one lane) loads 64-element K slabs of A and B with TMA
// (128-byte swizzle, completion counted in bytes on the stage's "full"
// mbarrier) into an NS-stage ring; warp 1 (one lane) issues four K=16
// tcgen05.mma per slab into one of two tensor-memory accumulators and
// commits each slab to the stage's "empty" mbarrier and each finished tile
// to the accumulator's "full" mbarrier; warps 2..9 drain the other
// accumulator (warp w reads lanes 32(w%4).. and one half of the columns),
// apply the epilogue and store, then release the accumulator.  The
// epilogue of tile i thus overlaps the loads and MMAs of tile i+1.  Every
// wait is bounded; a role that gives up raises the CTA's abort word and
// all roles stop.  Before the CTA frees its tensor memory and exits, the
// producer waits for every TMA load it issued to land and the MMA issuer
// commits a drain barrier and waits for every MMA it issued, so no
// asynchronous copy or MMA is in flight at exit on either path.
constexpr int WS_THREADS = 320;
constexpr int WS_STAGES = 4;
constexpr int STAGE_ROW = 80;  // bytes between rows of an epilogue warp's staging tile

__device__ __forceinline__ void mbar_expect_tx(uint32_t mbar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mbar), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t mbar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(mbar) : "memory");
}
__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, int x, int y, uint32_t mbar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
      "[%4];" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(mbar)
      : "memory");
}
// K-major, 128-byte swizzle: 8-row groups 1024 bytes apart (stride offset),
// leading offset unused (1), layout type 2.
__device__ __forceinline__ uint64_t umma_desc_sw128(uint32_t addr) {
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3FFFu);
  d |= (uint64_t)1 << 16;
  d |= (uint64_t)(1024 >> 4) << 32;
  d |= (uint64_t)1 << 46;
  d |= (uint64_t)2 << 61;
  return d;
}

template <int BN>
__global__ void __launch_bounds__(WS_THREADS, 1)
    k_gemm_ws(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, Gemm p) {
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  // stage buffers on a 1024-byte boundary (the swizzle atom)
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
  constexpr int A_BYTES = BM * BK * 2, B_BYTES = BN * BK * 2, STAGE = A_BYTES + B_BYTES;
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + WS_STAGES * STAGE);
  uint64_t* empty = full + WS_STAGES;
  uint64_t* acc_full = empty + WS_STAGES;
  uint64_t* acc_empty = acc_full + 2;
  uint64_t* drain = acc_empty + 2;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(drain + 1);
  volatile int* abort_word = reinterpret_cast<volatile int*>(tmem_slot + 1);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int n_n = p.N / BN, tiles = (p.M / BM) * n_n, nk = p.K / BK;

  if (threadIdx.x == 0) {
    for (int i = 0; i < WS_STAGES; ++i) {
      mbar_init(smem_u32(&full[i]), 1);
      mbar_init(smem_u32(&empty[i]), 1);
    }
    for (int i = 0; i < 2; ++i) {
      mbar_init(smem_u32(&acc_full[i]), 1);
      mbar_init(smem_u32(&acc_empty[i]), 8);  // one arrival per epilogue warp
    }
    mbar_init(smem_u32(drain), 1);
    *abort_word = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(2 * BN));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;

  if (warp == 0) {
    // TMA producer
    if (lane == 0) {
      int it = 0;
      int last_it[WS_STAGES];  // last iteration whose loads went to each stage
#pragma unroll
      for (int s = 0; s < WS_STAGES; ++s) last_it[s] = -1;
      for (int t = blockIdx.x; t < tiles && !*abort_word; t += gridDim.x) {
        const int m0 = (t / n_n) * BM, n0 = (t % n_n) * BN;
        for (int kt = 0; kt < nk; ++kt, ++it) {
          const int s = it % WS_STAGES;
          if (!mbar_wait_or_abort(smem_u32(&empty[s]), ((it / WS_STAGES) & 1) ^ 1, abort_word, WAIT_LIMIT)) {
            *abort_word = 1;
            break;
          }
          uint8_t* a = smem + s * STAGE;
          mbar_expect_tx(smem_u32(&full[s]), STAGE);
          tma_load_2d(smem_u32(a), &tmA, kt * BK, m0, smem_u32(&full[s]));
          tma_load_2d(smem_u32(a + A_BYTES), &tmB, kt * BK, n0, smem_u32(&full[s]));
          last_it[s] = it;
        }
      }
      // Every load issued has landed before the stage memory may go away:
      // the last load into stage s completes phase last_it[s] / WS_STAGES of
      // full[s], and no later load can move that barrier on.
#pragma unroll
      for (int s = 0; s < WS_STAGES; ++s)
        if (last_it[s] >= 0 && !mbar_wait(smem_u32(&full[s]), (last_it[s] / WS_STAGES) & 1)) *abort_word = 1;
    }
  } else if (warp == 1) {
    // MMA issuer
    if (lane == 0) {
      const uint32_t idesc = umma_idesc(BM, BN);
      int it = 0, tc = 0;
      for (int t = blockIdx.x; t < tiles && !*abort_word; t += gridDim.x, ++tc) {
        const int b = tc & 1;
        if (!mbar_wait_or_abort(smem_u32(&acc_empty[b]), ((tc >> 1) & 1) ^ 1, abort_word, WAIT_LIMIT)) {
          *abort_word = 1;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t acc = tmem + (uint32_t)(b * BN);
        for (int kt = 0; kt < nk; ++kt, ++it) {
          const int s = it % WS_STAGES;
          if (!mbar_wait_or_abort(smem_u32(&full[s]), (it / WS_STAGES) & 1, abort_word, p.mma_wait_polls)) {
            *abort_word = 1;
            break;
          }
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          const uint32_t a0 = smem_u32(smem + s * STAGE), b0 = a0 + A_BYTES;
#pragma unroll
          for (int j = 0; j < BK / 16; ++j)
            mma_bf16(acc, umma_desc_sw128(a0 + 32 * j), umma_desc_sw128(b0 + 32 * j), idesc,
                     (kt > 0 || j > 0) ? 1u : 0u);
          mma_commit(smem_u32(&empty[s]));
        }
        if (*abort_word) break;
        mma_commit(smem_u32(&acc_full[b]));
      }
      // Every MMA issued by this thread completes before the tensor memory
      // and the stage buffers it reads may be released.
      mma_commit(smem_u32(drain));
      if (!mbar_wait(smem_u32(drain), 0)) *abort_word = 1;
    }
  } else {
    // epilogue warps 2..9: lane quarter warp % 4, column half (warp - 2) / 4
    const int quarter = warp & 3, half = (warp - 2) >> 2;
    // bf16 activations leave through a per-warp staging tile (32 rows of 64
    // bytes, rows 80 bytes apart) so that the global stores are row-contiguous
    const bool staged = p.epilogue == HEXMLP_EPI_GELU && p.C != nullptr;
    const bool staged_f32 = p.epilogue == HEXMLP_EPI_F32 && p.C == nullptr;
    uint8_t* stage_tile = smem + WS_STAGES * STAGE + 256 + (warp - 2) * 32 * STAGE_ROW;
    int tc = 0;
    for (int t = blockIdx.x; t < tiles; t += gridDim.x, ++tc) {
      const int b = tc & 1;
      bool ok = true;
      if (lane == 0) ok = mbar_wait_or_abort(smem_u32(&acc_full[b]), (tc >> 1) & 1, abort_word, WAIT_LIMIT);
      ok = __shfl_sync(0xffffffffu, ok ? 1 : 0, 0) != 0;
      if (!ok) {
        if (lane == 0) *abort_word = 1;
        break;
      }
      if (*abort_word) break;
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const int m0 = (t / n_n) * BM, n0 = (t % n_n) * BN;
      const int row = m0 + quarter * 32 + lane;
      const uint32_t base = tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(b * BN);
      for (int c32 = half * (BN / 2); c32 < (half + 1) * (BN / 2); c32 += 32) {
        float v32[32];
        tmem_ld32(base + (uint32_t)c32, v32);
        if (staged) {
          // this lane's row of 32 activations into the warp's staging tile,
          // then out row by row: 4 lanes write a row's 64 contiguous bytes
#pragma unroll
          for (int g8 = 0; g8 < 4; ++g8) {
            uint4 h;
            epilogue8(p, row, n0 + c32 + 8 * g8, v32 + 8 * g8, &h);
            *reinterpret_cast<uint4*>(stage_tile + lane * STAGE_ROW + 16 * g8) = h;
          }
          __syncwarp();
#pragma unroll
          for (int j = 0; j < 4; ++j) {
            const int r = 8 * j + (lane >> 2), piece = lane & 3;
            const uint4 h = *reinterpret_cast<const uint4*>(stage_tile + r * STAGE_ROW + 16 * piece);
            *reinterpret_cast<uint4*>(p.C + (size_t)(m0 + quarter * 32 + r) * p.N + n0 + c32 + 8 * piece) = h;
          }
          __syncwarp();
        } else if (staged_f32) {
          // FP32 out: two halves of 16 columns (64 bytes a row) through the tile
#pragma unroll
          for (int hh = 0; hh < 2; ++hh) {
#pragma unroll
            for (int g = 0; g < 2; ++g) {
              const int g8 = 2 * hh + g;
              epilogue8(p, row, n0 + c32 + 8 * g8, v32 + 8 * g8, nullptr,
                        reinterpret_cast<float4*>(stage_tile + lane * STAGE_ROW + 32 * g));
            }
            __syncwarp();
#pragma unroll
            for (int j = 0; j < 4; ++j) {
              const int r = 8 * j + (lane >> 2), piece = lane & 3;
              const float4 f = *reinterpret_cast<const float4*>(stage_tile + r * STAGE_ROW + 16 * piece);
              *reinterpret_cast<float4*>(p.Cf + (size_t)(m0 + quarter * 32 + r) * p.N + n0 + c32 + 16 * hh +
                                         4 * piece) = f;
            }
            __syncwarp();
          }
        } else {
#pragma unroll
          for (int g8 = 0; g8 < 4; ++g8) epilogue8(p, row, n0 + c32 + 8 * g8, v32 + 8 * g8);
        }
      }
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      __syncwarp();
      if (lane == 0) mbar_arrive(smem_u32(&acc_empty[b]));
    }
  }
  __syncthreads();
  if (*abort_word && threadIdx.x == 0) atomicOr(p.err, 1);
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2 * BN));
  }
}

// dY = 2 (Y - T) / count over the valid rows and columns (zero elsewhere),
// in bf16 and transposed bf16; the squared error summed into *loss.
__global__ void k_mse_grad(const float* __restrict__ Y, const float* __restrict__ T, int M, int N, int m_valid,
                           int n_valid, float scale, __nv_bfloat16* __restrict__ dY,
                           __nv_bfloat16* __restrict__ dYt, float* loss) {
  const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  float sq = 0.0f;
  if (i < (size_t)M * N) {
    const int m = (int)(i / N), n = (int)(i % N);
    float g = 0.0f;
    if (m < m_valid && n < n_valid) {
      const float d = Y[i] - T[i];
      sq = d * d;
      g = 2.0f * d * scale;
    }
    const __nv_bfloat16 b = __float2bfloat16_rn(g);
    dY[i] = b;
    if (dYt) dYt[(size_t)n * M + m] = b;
  }
  for (int o = 16; o > 0; o >>= 1) sq += __shfl_down_sync(0xffffffffu, sq, o);
  if ((threadIdx.x & 31) == 0 && loss) atomicAdd(loss, sq);
}

// db[n] = sum over m of dZ^T[n][m]
__global__ void k_bias_grad(const __nv_bfloat16* __restrict__ dZt, int N, int M, float* __restrict__ db) {
  const int n = blockIdx.x;
  float acc = 0.0f;
  for (int m = threadIdx.x; m < M; m += blockDim.x) acc += __bfloat162float(dZt[(size_t)n * M + m]);
  __shared__ float red[32];
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x < 32) {
    acc = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0f;
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if (threadIdx.x == 0) db[n] = acc;
  }
}

// Adam on FP32 master weights [rows][cols] (bias when rows == 1); refreshes
// the bf16 copy and, when given, its transpose.
__global__ void k_adam(float* __restrict__ w, float* __restrict__ m1, float* __restrict__ m2,
                       const float* __restrict__ g, int rows, int cols, float lr, float b1, float b2, float eps,
                       float c1, float c2, float decay, __nv_bfloat16* __restrict__ wb, __nv_bfloat16* __restrict__ wbt) {
  const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i >= (size_t)rows * cols) return;
  const float gi = g[i] + decay * w[i];
  const float a = b1 * m1[i] + (1.0f - b1) * gi;
  const float b = b2 * m2[i] + (1.0f - b2) * gi * gi;
  m1[i] = a;
  m2[i] = b;
  const float wi = w[i] - lr * (a / c1) / (sqrtf(b / c2) + eps);
  w[i] = wi;
  const __nv_bfloat16 h = __float2bfloat16_rn(wi);
  if (wb) wb[i] = h;
  if (wbt) {
    const int r = (int)(i / cols), c = (int)(i % cols);
    wbt[(size_t)c * rows + r] = h;
  }
}

// out[r][f] = bf16((raw[r][f] - mean[f]) * inv_std[f]) for r < rows and
// f < n_feat, zero elsewhere in [rows_pad][ld_out]; the transpose too if given.
__global__ void k_pack(const float* __restrict__ raw, int rows, int n_feat, int ld_raw,
                       const float* __restrict__ mean, const float* __restrict__ inv_std, int rows_pad, int ld_out,
                       bf16* __restrict__ out, bf16* __restrict__ out_t) {
  const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i >= (size_t)rows_pad * ld_out) return;
  const int r = (int)(i / ld_out), f = (int)(i % ld_out);
  float v = 0.0f;
  if (r < rows && f < n_feat) v = (raw[(size_t)r * ld_raw + f] - mean[f]) * inv_std[f];
  const bf16 b = __float2bfloat16_rn(v);
  out[i] = b;
  if (out_t) out_t[(size_t)f * rows_pad + r] = b;
}

}  // namespace

extern "C" {

int hexmlp_pack(const float* raw, int rows, int n_feat, int ld_raw, const float* mean, const float* inv_std,
                int rows_pad, int ld_out, void* out, void* out_t, void* stream) {
  if (!raw || !mean || !inv_std || !out || rows < 0 || rows > rows_pad || n_feat > ld_out || n_feat > ld_raw)
    return HEXMLP_E_ARG;
  const size_t n = (size_t)rows_pad * ld_out;
  if (n == 0) return 0;
  k_pack<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(raw, rows, n_feat, ld_raw, mean, inv_std,
                                                                       rows_pad, ld_out, (bf16*)out, (bf16*)out_t);
  return (int)cudaGetLastError();
}

size_t hexmlp_gemm_smem_bytes(int bn) { return (size_t)NSTAGE * (BM + bn) * BK * 2 + 64; }

int hexmlp_gemm_tile_rows(void) { return BM; }
int hexmlp_gemm_tile_k(void) { return BK; }

}  // extern "C"

namespace {

using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                 const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiled encode_fn() {
  static EncodeTiled fn = nullptr;
  if (!fn) {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (EncodeTiled)f;
  }
  return fn;
}

// [rows][K] bf16 row-major, boxes of 64 K-elements x box_rows rows, 128-byte swizzle
bool make_map(CUtensorMap* m, const void* base, int rows, int K, int box_rows) {
  EncodeTiled fn = encode_fn();
  if (!fn) return false;
  const cuuint64_t dims[2] = {(cuuint64_t)K, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)K * 2};
  const cuuint32_t box[2] = {(cuuint32_t)BK, (cuuint32_t)box_rows};
  const cuuint32_t es[2] = {1, 1};
  return fn(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims, strides, box, es,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <int BN>
size_t ws_smem_bytes() {
  return (size_t)WS_STAGES * (BM + BN) * BK * 2 + 1024 + 256 + 8 * 32 * STAGE_ROW;
}

template <int BN>
int launch_ws(const Gemm& g, cudaStream_t st) {
  CUtensorMap ta, tb;
  if (!make_map(&ta, g.A, g.M, g.K, BM) || !make_map(&tb, g.B, g.N, g.K, BN)) return HEXMLP_E_ARG;
  static int sms = 0;
  if (!sms) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, 0);
  const size_t smem = ws_smem_bytes<BN>();
  cudaError_t e = cudaFuncSetAttribute(k_gemm_ws<BN>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return (int)e;
  const int tiles = (g.M / BM) * (g.N / BN);
  k_gemm_ws<BN><<<tiles < sms ? tiles : sms, WS_THREADS, smem, st>>>(ta, tb, g);
  return (int)cudaGetLastError();
}

}  // namespace

namespace {

int gemm_impl(const HexMlpGemm* p, uint32_t mma_wait_polls, void* stream) {
  if (!p || !p->A || !p->B || !p->err) return HEXMLP_E_ARG;
  if (p->M <= 0 || p->N <= 0 || p->K <= 0 || p->M % BM || p->K % BK) return HEXMLP_E_ARG;
  if (!(p->bn == 128 || p->bn == 256) || p->N % p->bn) return HEXMLP_E_ARG;
  if (p->epilogue == HEXMLP_EPI_F32 && !p->Cf) return HEXMLP_E_ARG;
  if (p->epilogue == HEXMLP_EPI_GELU_GRAD && !p->Zin) return HEXMLP_E_ARG;
  if (p->epilogue < HEXMLP_EPI_F32 || p->epilogue > HEXMLP_EPI_GELU_GRAD) return HEXMLP_E_ARG;
  // 16-byte alignment of every row: K and N multiples of 8 hold by the checks
  // above; the base pointers must be 16-byte aligned
  const void* ptrs[] = {p->A, p->B, p->C, p->Z, p->Zin, p->Cf, p->bias};
  for (const void* q : ptrs)
    if (q && ((uintptr_t)q & 15u)) return HEXMLP_E_ARG;
  const size_t smem = hexmlp_gemm_smem_bytes(p->bn);
  cudaError_t e = cudaFuncSetAttribute(k_gemm_bf16, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return (int)e;
  const Gemm g{(const bf16*)p->A, (const bf16*)p->B, p->M, p->N, p->K, p->bn, p->epilogue, p->bias, (bf16*)p->C,
               (bf16*)p->Ct, (bf16*)p->Z, (const bf16*)p->Zin, p->Cf, p->err, mma_wait_polls};
  if (p->kernel == HEXMLP_GEMM_PERSISTENT)
    return p->bn == 256 ? launch_ws<256>(g, (cudaStream_t)stream) : launch_ws<128>(g, (cudaStream_t)stream);
  if (p->kernel != HEXMLP_GEMM_STAGED || mma_wait_polls != WAIT_LIMIT) return HEXMLP_E_ARG;
  dim3 grid(p->M / BM, p->N / p->bn);
  k_gemm_bf16<<<grid, THREADS, smem, (cudaStream_t)stream>>>(g);
  return (int)cudaGetLastError();
}

}  // namespace

extern "C" {

int hexmlp_gemm(const HexMlpGemm* p, void* stream) { return gemm_impl(p, WAIT_LIMIT, stream); }

int hexmlp_gemm_wait_limit(const HexMlpGemm* p, uint32_t mma_wait_polls, void* stream) {
  if (!p || p->kernel != HEXMLP_GEMM_PERSISTENT) return HEXMLP_E_ARG;
  return gemm_impl(p, mma_wait_polls, stream);
}

int hexmlp_mse_grad(const float* Y, const float* T, int M, int N, int m_valid, int n_valid, float scale,
                    void* dY_, void* dYt_, float* loss, void* stream) {
  bf16* dY = (bf16*)dY_;
  bf16* dYt = (bf16*)dYt_;
  if (!Y || !T || !dY || M <= 0 || N <= 0) return HEXMLP_E_ARG;
  const size_t n = (size_t)M * N;
  k_mse_grad<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(Y, T, M, N, m_valid, n_valid, scale,
                                                                          dY, dYt, loss);
  return (int)cudaGetLastError();
}

int hexmlp_bias_grad(const void* dZt_, int N, int M, float* db, void* stream) {
  const bf16* dZt = (const bf16*)dZt_;
  if (!dZt || !db || N <= 0 || M <= 0) return HEXMLP_E_ARG;
  k_bias_grad<<<N, 256, 0, (cudaStream_t)stream>>>(dZt, N, M, db);
  return (int)cudaGetLastError();
}

int hexmlp_adam(float* w, float* m1, float* m2, const float* g, int rows, int cols, float lr, float b1, float b2,
                float eps, int t, float decay, void* wb_, void* wbt_, void* stream) {
  bf16* wb = (bf16*)wb_;
  bf16* wbt = (bf16*)wbt_;
  if (!w || !m1 || !m2 || !g || rows <= 0 || cols <= 0 || t < 1) return HEXMLP_E_ARG;
  const float c1 = 1.0f - powf(b1, (float)t), c2 = 1.0f - powf(b2, (float)t);
  const size_t n = (size_t)rows * cols;
  k_adam<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(w, m1, m2, g, rows, cols, lr, b1, b2, eps,
                                                                      c1, c2, decay, wb, wbt);
  return (int)cudaGetLastError();
}

}  // extern "C"
