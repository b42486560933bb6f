// umma_gemm.cu -- the FP32 BPTT weight-gradient contractions on the 5th-
// generation tensor cores: C[m][n] = sum_k X[k][m] Y[k][n] over K = steps x
// trials rows, X the input adjoints (FP32) and Y the shifted spikes (FP32)
// or the input counts (uint8).
//
// bf16 carries 8 mantissa bits, so each FP32 operand value is split into
// bf16 parts whose sum restates it: X = X0 + X1 + X2 (24 bits, FP32's own
// precision) and Y = Y0 + Y1 (Y1 = 0 for spikes and counts, which bf16
// holds exactly; the relaxed forward's surrogate spikes need it).  The
// products X0 Y0 + X1 Y0 + X2 Y0 + X0 Y1 accumulate in FP32 in tensor memory
// (the dropped X1 Y1 etc. are below 2^-16 of the product).
//
// k_umma_pack writes the parts in the order the MMA reads them: tile
// (rows r0..r0+127, k0..k0+63) is one contiguous 16 KB block laid out as
// 16 groups of 8 rows x 8 chunks of 16 bytes (8 bf16 along k), each chunk a
// "core matrix" of 8 rows x 16 bytes -- the K-major, unswizzled canonical
// layout of a tcgen05 shared-memory descriptor (leading byte offset 128 B
// between the two K-adjacent core matrices of one instruction, stride byte
// offset 1024 B between 8-row groups).
//
// k_umma_gemm: one 128-thread CTA per 128 x 128 output tile and row split;
// per 64-deep K chunk the warps copy the chunk's tiles (one 16 KB block per
// part) into shared memory with cp.async, one thread issues the chunk's
// tcgen05.mma (M = 128, N = 128, K = 16, kind::f16 with bf16 inputs) into a
// 128-column FP32 accumulator in tensor memory and commits them to the
// stage's mbarrier; with three stages (two when the relaxed spikes' second
// part does not leave room) the copies of the next two chunks are in flight
// while a chunk's MMAs run.  Each warp then reads its 32 accumulator lanes with tcgen05.ld and
// writes the tile's partial sums.  Every mbarrier wait is bounded: past the
// limit the kernel raises the error flag, stops issuing, waits (bounded) for
// what it issued, frees its tensor memory and returns.
#include <cuda_bf16.h>
#include <cuda_pipeline.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "../../../include/bspk.h"
#include "device_types.h"

namespace bspk {

namespace {

constexpr int kUT = 128;            // output tile rows / columns
constexpr int kUK = 64;             // K chunk (elements)
constexpr int kUTileBytes = kUT * kUK * 2;  // one part's tile: 16 KB
constexpr int kUXParts = 3;
constexpr int kUMaxStages = 3;       // shared-memory stages of the K loop
constexpr uint32_t kUTmemCols = 128;
constexpr long long kUSpinLimit = 1ll << 26;

// Element (r, k) of a packed operand with nkc K chunks: tile (r / 128,
// k / 64), then group (r % 128) / 8, chunk (k % 64) / 8, row r % 8, k % 8.
__device__ __forceinline__ size_t upack_index(int r, int64_t k, int64_t nkc) {
    const int64_t tile = (static_cast<int64_t>(r / kUT) * nkc + k / kUK);
    const int g = (r % kUT) >> 3, rr = r & 7;
    const int c = static_cast<int>((k % kUK) >> 3), e = static_cast<int>(k & 7);
    return static_cast<size_t>(tile) * (kUT * kUK) + ((g * 8 + c) * 8 + rr) * 8 + e;
}

// The bf16 parts of x: p[0] = bf16(x), p[i] = bf16(x - p[0] - ... - p[i-1]).
template <int P>
__device__ __forceinline__ void split_bf16(float x, __nv_bfloat16 (&p)[P]) {
    float rem = x;
#pragma unroll
    for (int i = 0; i < P; ++i) {
        p[i] = __float2bfloat16_rn(rem);
        rem = rem - __bfloat162float(p[i]);
    }
}

// Packs src[k][r] (row-major over k, R columns) for rows r < R_pad and
// k < K_pad (zero outside R x K) into P bf16 parts, each at out + part *
// part_elems.  One thread per (k, r) pair of a 32 x 32 block, through shared
// memory so that reads run along r and writes along k.
template <typename TS, int P>
__global__ void __launch_bounds__(256) k_umma_pack(const TS *src, int R, int64_t K, int R_pad,
                                                   int64_t nkc, __nv_bfloat16 *out, size_t part_elems) {
    __shared__ float tile[32][33];
    const int r0 = blockIdx.x * 32;
    const int64_t k0 = static_cast<int64_t>(blockIdx.y) * 32;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 32 x 8 threads
    for (int j = ty; j < 32; j += 8) {
        const int64_t k = k0 + j;
        const int r = r0 + tx;
        tile[j][tx] = (k < K && r < R) ? static_cast<float>(src[k * R + r]) : 0.f;
    }
    __syncthreads();
    for (int j = ty; j < 32; j += 8) {
        const int r = r0 + j;
        const int64_t k = k0 + tx;
        if (r >= R_pad || k >= nkc * kUK) continue;
        __nv_bfloat16 p[P];
        split_bf16<P>(tile[tx][j], p);
        const size_t o = upack_index(r, k, nkc);
#pragma unroll
        for (int i = 0; i < P; ++i) out[static_cast<size_t>(i) * part_elems + o] = p[i];
    }
}


__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// shared-memory matrix descriptor of a K-major, unswizzled tile at saddr:
// leading byte offset 128 B (K-adjacent core matrices), stride byte offset
// 1024 B (8-row groups), descriptor version 1
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr) {
    return static_cast<uint64_t>((saddr >> 4) & 0x3FFFu) | (static_cast<uint64_t>(128 >> 4) << 16) |
           (static_cast<uint64_t>(1024 >> 4) << 32) | (1ull << 46);
}

// instruction descriptor: FP32 accumulator, bf16 A and B, both K-major,
// N = 128 (bits 17-22: N / 8), M = 128 (bits 24-28: M / 16)
constexpr uint32_t kUIdesc = (1u << 4) | (1u << 7) | (1u << 10) |
                             (static_cast<uint32_t>(kUT >> 3) << 17) |
                             (static_cast<uint32_t>(kUT >> 4) << 24);

__device__ __forceinline__ void umma_bf16(uint32_t tmem, uint64_t adesc, uint64_t bdesc, uint32_t acc) {
    asm volatile(
        "{\n\t"
        ".reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t"
        "}\n"
        :
        : "r"(tmem), "l"(adesc), "l"(bdesc), "r"(kUIdesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u),
          "r"(0u)
        : "memory");
}

// bounded wait for the completion of phase `parity` of an mbarrier
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
    for (long long i = 0; i < kUSpinLimit; ++i) {
        uint32_t done;
        asm volatile(
            "{\n\t"
            ".reg .pred P1;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, P1;\n\t"
            "}"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

struct UmmaArgs {
    const __nv_bfloat16 *x, *y;  // packed parts of X (kUXParts) and Y (ny)
    size_t x_part, y_part;       // elements per part
    int ny;
    int M, N;                    // valid output rows and columns
    int64_t nkc;                 // K chunks of the packing
    int64_t kc_split;            // K chunks per row split
    int stages;                  // shared-memory stages (2 or 3)
    float *part;                 // [splits][M][N] partial sums
    int *err;
};

__global__ void __launch_bounds__(128, 1) k_umma_gemm(const UmmaArgs a) {
    extern __shared__ __align__(1024) unsigned char u_smem[];
    __shared__ __align__(8) unsigned long long s_bar[kUMaxStages];
    __shared__ uint32_t s_tmem;
    __shared__ int s_fail;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int nt = blockIdx.x, mt = blockIdx.y, z = blockIdx.z;
    const int64_t c0 = static_cast<int64_t>(z) * a.kc_split;
    const int64_t c1 = c0 + a.kc_split < a.nkc ? c0 + a.kc_split : a.nkc;
    const int nparts = kUXParts + a.ny;
    unsigned char *base = reinterpret_cast<unsigned char *>(
        (reinterpret_cast<uintptr_t>(u_smem) + 1023) & ~static_cast<uintptr_t>(1023));
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     :
                     : "r"(smem_u32(&s_tmem)), "r"(kUTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        for (int b = 0; b < kUMaxStages; ++b)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&s_bar[b])) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        s_fail = 0;
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = s_tmem;
    // NB stages: the copies of chunk c + NB - 1 are issued while the MMAs of
    // chunk c run (a stage is refilled once the MMAs that read it are done)
    const int NB = a.stages;
    uint32_t parity[kUMaxStages] = {0u, 0u, 0u};
    bool pending[kUMaxStages] = {false, false, false};
    const size_t tile_elems = static_cast<size_t>(kUT) * kUK;
    auto issue = [&](int64_t c, int b) {
        unsigned char *buf = base + static_cast<size_t>(b) * nparts * kUTileBytes;
        for (int p = 0; p < nparts; ++p) {
            const __nv_bfloat16 *src =
                p < kUXParts ? a.x + p * a.x_part + (static_cast<size_t>(mt) * a.nkc + c) * tile_elems
                             : a.y + (p - kUXParts) * a.y_part + (static_cast<size_t>(nt) * a.nkc + c) * tile_elems;
            unsigned char *dst = buf + static_cast<size_t>(p) * kUTileBytes;
            for (int q = tid; q < kUTileBytes / 16; q += blockDim.x)
                __pipeline_memcpy_async(dst + q * 16, reinterpret_cast<const unsigned char *>(src) + q * 16, 16);
        }
    };
    for (int st = 0; st < NB - 1; ++st) {
        if (c0 + st < c1) issue(c0 + st, st);
        __pipeline_commit();
    }
    for (int64_t c = c0; c < c1; ++c) {
        const int i = static_cast<int>(c - c0);
        const int b = i % NB;
        const int64_t cn = c + NB - 1;
        const int bn = (i + NB - 1) % NB;
        if (cn < c1) {
            // the MMAs that last read stage bn are complete before it is refilled
            if (pending[bn]) {
                if (!mbar_wait(smem_u32(&s_bar[bn]), parity[bn])) s_fail = 1;
                parity[bn] ^= 1u;
                pending[bn] = false;
            }
            issue(cn, bn);
        }
        __pipeline_commit();
        __pipeline_wait_prior(NB - 1);
        // the copies (generic proxy) become visible to the tensor cores
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (s_fail) break;
        unsigned char *buf = base + static_cast<size_t>(b) * nparts * kUTileBytes;
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t xb = smem_u32(buf), yb = xb + kUXParts * kUTileBytes;
#pragma unroll
            for (int ks = 0; ks < kUK / 16; ++ks) {
                // 16 elements of K: two 16-byte core-matrix columns, 256 B
                const uint32_t off = static_cast<uint32_t>(ks) * 256u;
                for (int q = 0; q < kUXParts + a.ny - 1; ++q) {
                    const int px = q < kUXParts ? q : 0, py = q < kUXParts ? 0 : 1;
                    const uint32_t acc = (c == c0 && ks == 0 && q == 0) ? 0u : 1u;
                    umma_bf16(tmem, umma_desc(xb + px * kUTileBytes + off),
                              umma_desc(yb + py * kUTileBytes + off), acc);
                }
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                         ::"r"(smem_u32(&s_bar[b]))
                         : "memory");
        }
        pending[b] = true;
    }
    __pipeline_wait_prior(0);  // no copy left in flight
    // the last MMAs (a second bounded wait after a failure, before the
    // accumulator's memory is released)
    for (int b = 0; b < NB; ++b)
        if (pending[b] && !mbar_wait(smem_u32(&s_bar[b]), parity[b])) s_fail = 1;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    __syncthreads();
    const bool ok = s_fail == 0;
    if (!ok && tid == 0) atomicExch(a.err, BSPK_DEV_ERR_TIMEOUT);
    if (ok) {
        const int m = mt * kUT + warp * 32 + lane;
        float *row = a.part + (static_cast<size_t>(z) * a.M + (m < a.M ? m : 0)) * a.N;
        for (int col = 0; col < kUT; col += 8) {
            uint32_t v[8] = {0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u};
            if (c1 > c0) {
                const uint32_t addr = tmem + (static_cast<uint32_t>(warp * 32) << 16) + static_cast<uint32_t>(col);
                asm volatile(
                    "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                    : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]),
                      "=r"(v[6]), "=r"(v[7])
                    : "r"(addr));
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            }
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                const int n = nt * kUT + col + i;
                if (m < a.M && n < a.N) row[n] = __uint_as_float(v[i]);
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kUTmemCols)
                     : "memory");
}

}  // namespace

size_t umma_part_elems(int R, int64_t K) {
    const int64_t rp = (R + kUT - 1) / kUT * kUT, kp = (K + kUK - 1) / kUK * kUK;
    return static_cast<size_t>(rp) * static_cast<size_t>(kp);
}

cudaError_t umma_pack_f32(const float *src, int R, int64_t K, int parts, __nv_bfloat16 *out,
                          cudaStream_t st) {
    const int rp = (R + kUT - 1) / kUT * kUT;
    const int64_t nkc = (K + kUK - 1) / kUK;
    const dim3 grid(static_cast<unsigned>((rp + 31) / 32), static_cast<unsigned>((nkc * kUK + 31) / 32));
    const size_t pe = umma_part_elems(R, K);
    if (parts == 3) k_umma_pack<float, 3><<<grid, 256, 0, st>>>(src, R, K, rp, nkc, out, pe);
    else if (parts == 2) k_umma_pack<float, 2><<<grid, 256, 0, st>>>(src, R, K, rp, nkc, out, pe);
    else k_umma_pack<float, 1><<<grid, 256, 0, st>>>(src, R, K, rp, nkc, out, pe);
    return cudaGetLastError();
}

cudaError_t umma_pack_u8(const uint8_t *src, int R, int64_t K, __nv_bfloat16 *out, cudaStream_t st) {
    const int rp = (R + kUT - 1) / kUT * kUT;
    const int64_t nkc = (K + kUK - 1) / kUK;
    const dim3 grid(static_cast<unsigned>((rp + 31) / 32), static_cast<unsigned>((nkc * kUK + 31) / 32));
    k_umma_pack<uint8_t, 1><<<grid, 256, 0, st>>>(src, R, K, rp, nkc, out, umma_part_elems(R, K));
    return cudaGetLastError();
}

int umma_splits(int sms, int M, int N, int64_t K) {
    const int64_t tiles = static_cast<int64_t>((M + kUT - 1) / kUT) * ((N + kUT - 1) / kUT);
    const int64_t nkc = (K + kUK - 1) / kUK;
    int64_t s = (static_cast<int64_t>(sms > 0 ? sms : 1) + tiles - 1) / tiles;
    s = s < nkc ? s : nkc;
    return static_cast<int>(s < 1 ? 1 : (s > 64 ? 64 : s));
}

cudaError_t umma_gemm(const __nv_bfloat16 *x, int M, const __nv_bfloat16 *y, int ny, int N, int64_t K,
                      int splits, float *part, int *err, cudaStream_t st) {
    UmmaArgs a{};
    a.x = x;
    a.y = y;
    a.x_part = umma_part_elems(M, K);
    a.y_part = umma_part_elems(N, K);
    a.ny = ny;
    a.M = M;
    a.N = N;
    a.nkc = (K + kUK - 1) / kUK;
    a.kc_split = (a.nkc + splits - 1) / splits;
    a.part = part;
    a.err = err;
    // three stages when they fit in the 227 KB of a CTA, else two
    a.stages = 3 * (kUXParts + ny) * kUTileBytes + 1024 <= 227 * 1024 ? 3 : 2;
    const int smem = a.stages * (kUXParts + ny) * kUTileBytes + 1024;
    cudaError_t e = cudaFuncSetAttribute(k_umma_gemm, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    const dim3 grid(static_cast<unsigned>((N + kUT - 1) / kUT), static_cast<unsigned>((M + kUT - 1) / kUT),
                    static_cast<unsigned>(splits));
    k_umma_gemm<<<grid, 128, smem, st>>>(a);
    return cudaGetLastError();
}

}  // namespace bspk
