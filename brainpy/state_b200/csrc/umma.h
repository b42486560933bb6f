// umma.h -- the tensor-core contraction of umma_gemm.cu (C = X^T Y over rows
// k of row-major X [K][M] and Y [K][N], FP32 results from bf16 parts).
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace bspk {
// elements of one packed bf16 part of an operand with R columns and K rows
size_t umma_part_elems(int R, int64_t K);
// src [K][R] FP32 into `parts` bf16 parts (out: parts x umma_part_elems)
cudaError_t umma_pack_f32(const float *src, int R, int64_t K, int parts, __nv_bfloat16 *out,
                          cudaStream_t st);
// src [K][R] uint8 counts into one bf16 part (exact)
cudaError_t umma_pack_u8(const uint8_t *src, int R, int64_t K, __nv_bfloat16 *out, cudaStream_t st);
// row splits: enough 128 x 128 tiles x splits for one CTA per SM
int umma_splits(int sms, int M, int N, int64_t K);
// part[z][m][n] = sum over split z's rows k of X[k][m] Y[k][n] (ny: Y parts)
cudaError_t umma_gemm(const __nv_bfloat16 *x, int M, const __nv_bfloat16 *y, int ny, int N, int64_t K,
                      int splits, float *part, int *err, cudaStream_t st);
}  // namespace bspk
