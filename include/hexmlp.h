/*
 * hexmlp: BF16 tensor-core MLP kernels of the learned corrector, C ABI.
 *
 * No counterpart in the reference's dycore path: the learned corrector (a
 * per-column network that corrects a step taken with fewer acoustic
 * substeps, trained on pairs of full and reduced steps) is this library's
 * own.  The kernels run on the 5th-generation tensor cores (tcgen05.mma,
 * FP32 accumulation in tensor memory).  bf16 arrays are passed as void*
 * (IEEE bfloat16 words); every call returns 0, HEXMLP_E_ARG for a refused
 * argument, or a positive CUDA error code, and runs on `stream` (a
 * cudaStream_t).
 */
#ifndef HEXMLP_H
#define HEXMLP_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define HEXMLP_E_ARG (-1)

/* GEMM epilogues. */
#define HEXMLP_EPI_F32 0        /* Cf = A.B^T (+ bias); optional bf16 copy in C */
#define HEXMLP_EPI_GELU 1       /* Z = A.B^T + bias (bf16), C = GELU(Z), Ct = C^T; GELU in
                                   its tanh form with the hardware tanh approximation */
#define HEXMLP_EPI_GELU_GRAD 2  /* C = (A.B^T) * GELU'(Zin), Ct = C^T (bf16) */

/* C[M][N] = A[M][K] . B[N][K]^T; A and B bf16 with K contiguous.  M a
 * multiple of 128, K of 64, N of bn (128 or 256); base pointers 16-byte
 * aligned.  Output arrays are [M][N] row-major, Ct is [N][M].  *err
 * (device int) is OR-ed with 1 if a CTA gave up waiting on the tensor core
 * (the results are then invalid). */
typedef struct HexMlpGemm {
  const void* A;
  const void* B;
  int32_t M, N, K, bn, epilogue;
  const float* bias;   /* [N] or NULL */
  void* C;             /* bf16 [M][N] or NULL */
  void* Ct;            /* bf16 [N][M] or NULL */
  void* Z;             /* bf16 [M][N] pre-activation (HEXMLP_EPI_GELU) or NULL */
  const void* Zin;     /* bf16 [M][N] (HEXMLP_EPI_GELU_GRAD) */
  float* Cf;           /* float [M][N] (HEXMLP_EPI_F32) */
  int* err;            /* device int */
  int32_t kernel;      /* HEXMLP_GEMM_PERSISTENT (default) or HEXMLP_GEMM_STAGED */
} HexMlpGemm;

/* GEMM kernels: persistent and warp-specialised (TMA loads, one MMA thread,
 * epilogue warps on a double-buffered tensor-memory accumulator), or one CTA
 * per tile with cp.async staging. */
#define HEXMLP_GEMM_PERSISTENT 0
#define HEXMLP_GEMM_STAGED 1

int hexmlp_gemm(const HexMlpGemm* p, void* stream);
/* Check of the persistent GEMM's failure path: hexmlp_gemm with the MMA
 * issuer's wait for each loaded stage bounded by `mma_wait_polls` mbarrier
 * polls instead of 2^20.  With 0 that wait gives up before the first stage
 * lands: the kernel sets *err, its producer waits for every TMA load it
 * issued, its MMA issuer for every MMA it issued, it frees its tensor memory
 * and returns (outputs invalid).  Only HEXMLP_GEMM_PERSISTENT. */
int hexmlp_gemm_wait_limit(const HexMlpGemm* p, uint32_t mma_wait_polls, void* stream);
size_t hexmlp_gemm_smem_bytes(int bn);
int hexmlp_gemm_tile_rows(void);
int hexmlp_gemm_tile_k(void);

/* Mean-squared-error gradient: dY = 2 (Y - T) * scale on rows < m_valid
 * and columns < n_valid, 0 elsewhere (bf16 [M][N] and, if dYt, [N][M]);
 * the summed squared error is added to *loss (device float) if loss. */
int hexmlp_mse_grad(const float* Y, const float* T, int M, int N, int m_valid, int n_valid, float scale,
                    void* dY, void* dYt, float* loss, void* stream);

/* db[n] = sum over m of dZt[n][m] (bf16 [N][M]). */
int hexmlp_bias_grad(const void* dZt, int N, int M, float* db, void* stream);

/* Adam step t (1-based) on FP32 weights w [rows][cols] with moments m1, m2
 * and gradient g (L2 decay `decay`); refreshes the bf16 copy wb and, if
 * given, its transpose wbt [cols][rows]. */
int hexmlp_adam(float* w, float* m1, float* m2, const float* g, int rows, int cols, float lr, float b1, float b2,
                float eps, int t, float decay, void* wb, void* wbt, void* stream);

/* Normalise and pack network inputs: out[r][f] = bf16((raw[r][f] -
 * mean[f]) * inv_std[f]) for r < rows, f < n_feat; zero in the padding of
 * out [rows_pad][ld_out] (and of its transpose out_t [ld_out][rows_pad] if
 * given). */
int hexmlp_pack(const float* raw, int rows, int n_feat, int ld_raw, const float* mean, const float* inv_std,
                int rows_pad, int ld_out, void* out, void* out_t, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* HEXMLP_H */
