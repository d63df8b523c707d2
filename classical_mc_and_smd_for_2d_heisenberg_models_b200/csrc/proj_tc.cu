// proj_tc.cu -- list-q projection on the 5th-generation tensor cores.
//
// S(q_l) = scale sum_k S_k exp(-i q_l . r_k) (get_qct_SqData,
// Codes_Folder/subrouts.cpp:8460-8525) for every snapshot row (sample,
// record, component) is the GEMM
//
//     C[m][2l + 0/1] = sum_k A[m][k] B[2l + 0/1][k]
//     A = snapshot rows (FP32),  B = (scale cos(q.r_k), -scale sin(q.r_k))
//
// run in split-BF16 form: A = Ah + Al, B = Bh + Bl (bf16 each) and
// C = Ah Bh + Ah Bl + Al Bh, accumulated in FP32 in tensor memory.  The
// dropped Al Bl term is 2^-16 of the product.  The three products are three
// K segments of one tcgen05 accumulation.
//
// Tile 128 x 256, K blocks of 64 bf16 (one 128-byte swizzle row).  Warp 0
// loads A and B K-blocks with TMA (128B swizzle) into a 4-stage ring, warp 1
// issues tcgen05.mma (M=128, N=256, K=16) from one thread, and all four warps
// drain the accumulator with tcgen05.ld, apply the record's window weight and
// store complex64 values straight into the q-blocked time series.  Every mbarrier wait is bounded: after the limit the
// kernel records an error, stops issuing work, waits (bounded) for its
// copies in flight, frees its tensor memory and returns.
#include "smd_device.cuh"

#include <cuda.h>
#include <cuda_bf16.h>
#include <cudaTypedefs.h>

#include <mutex>

namespace smd {

namespace tc {

constexpr int BM = 128, BN = 256, BK = 64, STAGES = 4;
constexpr int A_BYTES = BM * BK * 2, B_BYTES = BN * BK * 2;
constexpr int STAGE_BYTES = A_BYTES + B_BYTES;
constexpr int SMEM = STAGES * STAGE_BYTES + 1024 /* alignment */ + 256 /* barriers */;
constexpr unsigned kSpinLimit = 1u << 26;   // about a second of polling

__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *b, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(count));
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *b, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(b)),
                 "r"(bytes)
                 : "memory");
}

// Bounded wait for phase `parity` of barrier b; false after the limit.
__device__ __forceinline__ bool mbar_wait(uint64_t *b, unsigned parity)
{
    const uint32_t a = smem_u32(b);
    for (unsigned it = 0; it < kSpinLimit; it++) {
        uint32_t ok;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
            " selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(ok)
            : "r"(a), "r"(parity)
            : "memory");
        if (ok) return true;
    }
    return false;
}

__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, uint64_t *bar, int x,
                                            int y)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, "
        "{%3, %4}], [%2];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(x), "r"(y)
        : "memory");
}

// Shared-memory matrix descriptor: K-major operand, 128-byte swizzle, rows of
// 128 bytes, 8-row core groups 1024 bytes apart.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr)
{
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFFu);          // start address
    d |= (uint64_t)1 << 16;                          // leading byte offset (unused with swizzle)
    d |= (uint64_t)((1024 >> 4) & 0x3FFFu) << 32;    // stride byte offset
    d |= (uint64_t)1 << 46;                          // descriptor version
    d |= (uint64_t)2 << 61;                          // 128-byte swizzle
    return d;
}

// Instruction descriptor: kind::f16 with bf16 A and B, FP32 accumulator,
// both operands K-major, M = 128, N = 256.
__host__ __device__ constexpr uint32_t instr_desc()
{
    return (1u << 4)              // D format F32
           | (1u << 7)            // A format BF16
           | (1u << 10)           // B format BF16
           | ((uint32_t)(BN >> 3) << 17) | ((uint32_t)(BM >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem, uint64_t da, uint64_t db, uint32_t idesc,
                                         uint32_t accumulate)
{
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem),
        "l"(da), "l"(db), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void mma_commit(uint64_t *bar)
{
    asm volatile(
        "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
            smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16])
{
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
        "%12, %13, %14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
          "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

// grid: (column tiles, row tiles).  Rows are snapshot rows of the chunk,
// m = (s * R + slot) * 3 + c; rows whose slot >= nrec_chunk are skipped.
__global__ void __launch_bounds__(128, 1) list_proj_tc_kernel(
    const __grid_constant__ CUtensorMap mAh, const __grid_constant__ CUtensorMap mAl,
    const __grid_constant__ CUtensorMap mBh, const __grid_constant__ CUtensorMap mBl, int M,
    int nkb, int R, int nrec_chunk, int rec_begin, int n_rec_total, int Lq,
    const double *__restrict__ win, cplx<float> *__restrict__ series, int nqb, int qoff,
    int *status)
{
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    unsigned char *sm = reinterpret_cast<unsigned char *>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    unsigned char *sA = sm;
    unsigned char *sB = sm + STAGES * A_BYTES;
    uint64_t *full = reinterpret_cast<uint64_t *>(sm + STAGES * STAGE_BYTES);
    uint64_t *empty = full + STAGES;
    uint64_t *acc_full = empty + STAGES;
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(acc_full + 1);
    volatile int *abort_flag = reinterpret_cast<volatile int *>(tmem_slot + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // column tiles vary fastest, so the tiles sharing a row tile of A run
    // together and read it once from HBM
    const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
    const int total_kb = 3 * nkb;

    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        mbar_init(acc_full, 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(tmem_slot)),
                     "r"(256));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;

    int issued = 0;   // TMA stages issued by the producer
    if (warp == 0 && lane == 0) {
        // ---------------- producer
        for (int kb = 0; kb < total_kb; kb++) {
            const int s = kb % STAGES;
            if (kb >= STAGES && !mbar_wait(&empty[s], ((kb / STAGES) - 1) & 1)) {
                atomicOr(status, 4);
                *abort_flag = 1;
                break;
            }
            if (*abort_flag) break;
            const int seg = kb / nkb, kk = (kb % nkb) * BK;
            const CUtensorMap *ma = seg < 2 ? &mAh : &mAl;
            const CUtensorMap *mb = seg == 1 ? &mBl : &mBh;
            mbar_expect_tx(&full[s], STAGE_BYTES);
            tma_load_2d(sA + s * A_BYTES, ma, &full[s], kk, m0);
            tma_load_2d(sB + s * B_BYTES, mb, &full[s], kk, n0);
            issued++;
        }
    } else if (warp == 1 && lane == 0) {
        // ---------------- MMA issuer
        const uint32_t idesc = instr_desc();
        for (int kb = 0; kb < total_kb; kb++) {
            const int s = kb % STAGES;
            if (!mbar_wait(&full[s], (kb / STAGES) & 1)) {
                atomicOr(status, 4);
                *abort_flag = 1;
                break;
            }
            if (*abort_flag) break;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t a_addr = smem_u32(sA + s * A_BYTES);
            const uint32_t b_addr = smem_u32(sB + s * B_BYTES);
#pragma unroll
            for (int k4 = 0; k4 < BK / 16; k4++) {
                const uint64_t da = smem_desc(a_addr + k4 * 32);
                const uint64_t db = smem_desc(b_addr + k4 * 32);
                mma_bf16(tmem, da, db, idesc, (kb > 0 || k4 > 0) ? 1u : 0u);
            }
            mma_commit(&empty[s]);
        }
        // also after an abort: the barrier then tracks the MMAs still in
        // flight, so tensor memory is released only after they finish
        mma_commit(acc_full);
    }
    __syncwarp();

    // ---------------- epilogue: TMEM lane = tile row
    bool have = mbar_wait(acc_full, 0);
    if (!have && threadIdx.x == 0) atomicOr(status, 4);
    have = have && !*abort_flag;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const int row = m0 + warp * 32 + lane;
    const int c = row % 3, slot = row / 3 % R, s = row / (3 * R);
    const bool row_ok = have && row < M && slot < nrec_chunk;
    // windowed series: record t of this row, q = qoff + l in blocks of two
    const int t = rec_begin + slot;
    const float w = row_ok ? (float)win[t] : 0.f;
    cplx<float> *out = series + series_off<float>(s, c, 0, t, nqb, n_rec_total);
    const size_t bstride = (size_t)n_rec_total * 2;   // elements between q blocks
    if (have) {
#pragma unroll 1
        for (int c0 = 0; c0 < BN; c0 += 16) {
            float v[16];
            tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + c0, v);
            if (row_ok) {
                const int l0 = (n0 + c0) / 2;
                if ((qoff & 1) == 0 && l0 + 8 <= Lq) {
                    // whole blocks: one 16-byte store per pair of q
#pragma unroll
                    for (int p = 0; p < 4; p++) {
                        const int q = qoff + l0 + 2 * p;
                        *reinterpret_cast<float4 *>(out + (q >> 1) * bstride) =
                            make_float4(w * v[4 * p], w * v[4 * p + 1], w * v[4 * p + 2],
                                        w * v[4 * p + 3]);
                    }
                } else {
#pragma unroll
                    for (int p = 0; p < 8; p++) {
                        const int l = l0 + p, q = qoff + l;
                        if (l < Lq) out[(q >> 1) * bstride + (q & 1)] = {w * v[2 * p], w * v[2 * p + 1]};
                    }
                }
            }
        }
    }
    // copies still in flight after an abort complete before the buffers go away
    if (warp == 0 && lane == 0 && *abort_flag) {
        for (int kb = (issued > STAGES ? issued - STAGES : 0); kb < issued; kb++)
            mbar_wait(&full[kb % STAGES], (kb / STAGES) & 1);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(256));
    }
}

// FP32 snapshot rows -> bf16 high and low parts, row pitch kp (zero pad)
__global__ void split_bf16_kernel(const float *__restrict__ x, int rows, int N, int kp,
                                  __nv_bfloat16 *__restrict__ hi, __nv_bfloat16 *__restrict__ lo)
{
    const size_t total = (size_t)rows * kp;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total;
         e += (size_t)gridDim.x * blockDim.x) {
        const size_t r = e / kp;
        const int k = (int)(e - r * kp);
        const float v = k < N ? x[r * N + k] : 0.f;
        const __nv_bfloat16 h = __float2bfloat16_rn(v);
        hi[e] = h;
        lo[e] = __float2bfloat16_rn(v - __bfloat162float(h));
    }
}

PFN_cuTensorMapEncodeTiled_v12000 encode_fn()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    return fn;
}

}  // namespace tc

// 2D bf16 tensor map over a row-major [rows][kp] matrix, box box_rows x 64.
bool make_bf16_map(CUtensorMap *map, const void *base, int rows, int kp, int box_rows)
{
    auto fn = tc::encode_fn();
    if (!fn) return false;
    cuuint64_t dims[2] = {(cuuint64_t)kp, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)kp * 2};
    cuuint32_t box[2] = {(cuuint32_t)tc::BK, (cuuint32_t)box_rows};
    cuuint32_t estr[2] = {1, 1};
    return fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void *>(base), dims, strides, box,
              estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
              CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

int tc_kpitch(int N) { return (N + 63) / 64 * 64; }
int tc_bn() { return tc::BN; }
int tc_bm() { return tc::BM; }

cudaError_t launch_split_bf16(const float *x, int rows, int N, int kp, void *hi, void *lo,
                              cudaStream_t st)
{
    tc::split_bf16_kernel<<<1184, 256, 0, st>>>(x, rows, N, kp, (__nv_bfloat16 *)hi,
                                               (__nv_bfloat16 *)lo);
    return cudaGetLastError();
}

cudaError_t launch_list_proj_tc(const CUtensorMap &Ah, const CUtensorMap &Al, const CUtensorMap &Bh,
                                const CUtensorMap &Bl, int M, int kp, int R, int nrec_chunk,
                                int rec_begin, int n_rec_total, int Lq, const double *win,
                                void *series, int nqb, int qoff, int *status, cudaStream_t st)
{
    auto k = tc::list_proj_tc_kernel;
    cudaError_t e = allow_dynamic_smem(k);
    if (e != cudaSuccess) return e;
    dim3 grid((2 * Lq + tc::BN - 1) / tc::BN, (M + tc::BM - 1) / tc::BM);
    k<<<grid, 128, tc::SMEM, st>>>(Ah, Al, Bh, Bl, M, kp / tc::BK, R, nrec_chunk, rec_begin,
                                   n_rec_total, Lq, win, (cplx<float> *)series, nqb, qoff, status);
    return cudaGetLastError();
}

}  // namespace smd
