// Mixed-precision triple-product lag accumulation on the int8 tensor cores:
// 3-digit fixed point (an Ozaki-style split), exact int32 accumulation in
// TMEM, FP64 recombination and lag reduction.  Replaces the float loop of
// 4_fbe/amber.c:247-279 / amber_v2.c:243-283.
//
// Why not FP32 accumulation: on the B200 tensor cores a long FP32 accumulation
// chain of coherent (same-sign) products loses ~2^-24 of the running sum per
// step, which breaks the 1e-6-of-Σ|products| bound on the v2 sampling-mask
// sums; integer accumulation has no rounding at all, so chunks can be long.
//
// Representation.  Every map row r (ring slot, channel) has an exponent E_r
// with max|D_r| < 2^E_r and three signed int8 digits in base 254
//     D_r(x) = 2^E_r/127 · (d0 + d1/254 + d2/254²) + O(2^E_r·2^−24),
// d0, d1, d2 ∈ [−127, 127] (quantize_kernel, maps.cu).
// For one anchor p1 the GEMM is, as in the reference's loop,
//     T_p1[p2, p3] = Σ_x D2[p2,x] · (D1[p1,x]·D3[p3,x])
// with M = p2 (128 TMEM lanes), N = p3 (BN ∈ {32, 64}), K = pixels:
//   A = the D2 digit planes, staged by TMA in 64B-swizzled shared memory and
//       moved into TMEM with tcgen05.st (the "TS" MMA form) — no per-anchor
//       arithmetic on the 128 A rows;
//   B = D1[p1]·D3[p3] formed in FP32 on the CUDA cores (packed FP32x2) from
//       TMA-staged fp32 tiles, scaled by 127·2^−(E1+E3) and cut into FOUR
//       int8 digits written into 128B-swizzled shared memory — only BN rows
//       of per-anchor work per n-tile;
//   acc_k += Σ_{i+j=k} A_i·B_jᵀ for k = 0..3 — nine kind::i8 MMAs per 32
//       pixels into four int32 TMEM accumulators (terms with i+j ≥ 4 are
//       below 2^−31 of the leading one).  Per pixel |Σ_{i+j=k}| ≤ 3·127² <
//       2^15.6, so a chunk of up to 2^15 pixels cannot overflow.
// Why four digits for the product: its digits are scaled to the bound
// max|D1|·max|D3|, so three digits leave an error of ~6e-8 of that bound on
// every pixel, whatever the product's own size.  On sampling-mask maps (a
// peak at the origin, noise-like sidelobes far below it) those errors add up
// over the 10^5-10^6 pixels to ~4e-6 of Σ|products|; the fourth digit cuts
// them by 254.  The plain D2 operand keeps three digits: its error scales
// with the product it multiplies, which is small wherever D2's own bound is
// loose.  The k = 3 class matters for the same reason.  Four accumulators of
// 64 columns plus two 128-pixel A stages (2 × 96 columns) fill TMEM.
// Epilogue: T = 2^(E1+E2+E3)/127² · Σ_k acc_k·254^−k in FP64,
// weighted by the channel multiplicities, written to the partial buffer
// [anchor][chunk][lag2][lag3]; lag_reduce then sums it per lag cell with a
// compensated FP64 accumulator in a fixed order (deterministic).
//
// Issue rate.  An M=128, N=64 int8 MMA runs ~32 tensor cycles, and the pipe
// buffers only about two of them, so any latency in a single issuing thread
// (a barrier test, a commit) leaves it idle.  Two issuing warps, one owning
// accumulators 0 and 2 and one owning 1 and 3, each issuing its MMAs grouped
// by accumulator, keep it ~85% busy (measured 37 cycles per MMA against 54
// for one thread issuing in digit-class order).
//
// Warp roles (768 threads): warps 0-3 move the D2 digits from shared memory
// into TMEM (one warp per 32 TMEM lanes), warps 4-19 form the B digits, warp
// 20 streams the fp32 D3 tiles and the D1 row by TMA (128B-swizzled, so the
// row reads are conflict-free), warp 22 streams the D2 digit tiles by TMA,
// warps 21 and 23 issue the MMAs from one lane each (warp 21 also owns
// TMEM); warps 0-15 read the accumulators out.
// Every mbarrier wait is bounded; on expiry the CTA raises an error flag the
// host turns into AMBER_ERR_TIMEOUT, drains its own copies and MMAs, frees TMEM.
#include <algorithm>
#include <cmath>
#include <vector>

#include "common.cuh"
#include "tc_ptx.cuh"

namespace amber {

namespace {

using namespace tc;

constexpr int BM = 128;           // p2 rows per tile = TMEM lanes
constexpr int KB_B = 128;         // pixels per pipeline stage: one 128-byte swizzle row of int8
constexpr int KB_A = 64;          // pixels per D2 digit tile in shared memory
constexpr int NACC = 4;           // int32 accumulators, one per digit class i+j = 0..3
constexpr int A_STAGE_COLS = 96;  // 3 digits × 32 columns (128 int8 per lane per digit)
constexpr int NSTAGE = 2;         // pipeline stages in flight: A in TMEM, B digits in shared memory
constexpr int NWARP_A = 4;        // D2-digit movers: one warp per 32 TMEM lanes
constexpr int NWARP_B = 16;       // B formers
constexpr int WARP_TMA = 20;      // fp32 B inputs
constexpr int WARP_MMA = 21;      // owns TMEM; MMA issuer 0 (accumulators 0 and 2)
constexpr int WARP_TMA_A = 22;    // D2 digit tiles
constexpr int WARP_MMA2 = 23;     // MMA issuer 1 (accumulators 1 and 3)
constexpr int NEPI = 16;          // epilogue warps (movers and the first formers): 4 warpgroups
constexpr int NISSUE = 2;
constexpr int NTHREADS = 24 * 32;
constexpr int TMEM_COLS = 512;
constexpr int NAS = 4;            // D2 digit tiles in shared memory
constexpr int NBI = 2;            // fp32 input stages (D3 tile + D1 row)
constexpr int NDB = 4;            // int8 digits of the per-anchor product (B)
constexpr int A_BOX = KB_A * BM;  // one digit plane of one D2 tile: 128 rows × 64 bytes, 64B-swizzled

struct ParamsI8 {
    const int *e1, *e2, *e3;  // row exponents [nc]
    long k, kp;
    int nc, nc10, nclen;
    int mt_count, nt_count, nchunk, nanchors;
    long chunk;  // pixels per chunk (multiple of KB_B)
    const int *anchors;
    const int *weight;
    double *partial;  // [anchor][chunk][nclen²]
    int *err;
};

// Four base-254 digits of two products u·v at once (packed FP32x2): every
// step is one fused op on a pair, the product enters the first rounding
// unrounded (y0 = fma(u, v, M)), and round-to-nearest through the 1.5·2^23
// magic number leaves each digit's two's-complement byte in the low mantissa
// bits (as in quantize_kernel, maps.cu).  M − y = −digit exactly, and each
// residual 254·s − d is exact in FP32 (its lowest bit is at most 2^−22 and
// it is at most 1/2 in magnitude).
__device__ __forceinline__ void digits254x2(float2 u, float2 v, float2 &y0, float2 &y1, float2 &y2, float2 &y3)
{
    const float2 M = make_float2(12582912.0f, 12582912.0f);
    const float2 K254 = make_float2(254.f, 254.f);
    const float2 NEG1 = make_float2(-1.f, -1.f);
    y0 = __ffma2_rn(u, v, M);                     // M + d0
    const float2 nq0 = __ffma2_rn(y0, NEG1, M);   // −d0
    const float2 r0 = __ffma2_rn(u, v, nq0);      // u·v − d0
    y1 = __ffma2_rn(r0, K254, M);                 // M + d1
    const float2 nq1 = __ffma2_rn(y1, NEG1, M);   // −d1
    const float2 s1 = __ffma2_rn(r0, K254, nq1);  // 254·r0 − d1
    y2 = __ffma2_rn(s1, K254, M);                 // M + d2
    const float2 nq2 = __ffma2_rn(y2, NEG1, M);   // −d2
    const float2 s2 = __ffma2_rn(s1, K254, nq2);  // 254·s1 − d2
    y3 = __ffma2_rn(s2, K254, M);                 // M + d3
}

__device__ __forceinline__ uint32_t pack_low_bytes(float a, float b, float c, float d)
{
    return __byte_perm(__byte_perm(__float_as_uint(a), __float_as_uint(b), 0x0040),
                       __byte_perm(__float_as_uint(c), __float_as_uint(d), 0x0040), 0x5410);
}

__device__ __forceinline__ void tmem_ld8(uint32_t taddr, uint32_t (&v)[8])
{
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7])
                 : "r"(taddr)
                 : "memory");
}

// kind::i8 MMA, A from TMEM, always accumulating (no predicate set-up on the issue path)
__device__ __forceinline__ void umma_ts_i8_acc(uint32_t d_tmem, uint32_t a_tmem, uint64_t b_desc, uint32_t idesc)
{
    asm volatile("tcgen05.mma.cta_group::1.kind::i8 [%0], [%1], %2, %3, 1;" ::"r"(d_tmem), "r"(a_tmem), "l"(b_desc),
                 "r"(idesc)
                 : "memory");
}

// One issuer's share of a 128-pixel stage: accumulators k = q and q + 2, each fed
// Σ_{i+j=k} A_i·B_jᵀ (A: 3 digits, B: 4) over the four 32-pixel slices, grouped by accumulator
// (back-to-back MMAs into one accumulator keep the tensor pipe fullest).
// The stage's first MMA into each accumulator overwrites it when `fresh`.
template <int BN>
__device__ __forceinline__ void issue_stage(uint32_t tmem, uint32_t a_stage, uint64_t b_stage, uint32_t idesc, int q,
                                            bool fresh)
{
    constexpr uint32_t TILE16 = (uint32_t)(BN * KB_B) >> 4;
#pragma unroll
    for (int kc = 0; kc < 2; ++kc) {
        const int k = q + 2 * kc;
        const uint32_t acc = tmem + (uint32_t)(k * BN);
        bool first = true;
#pragma unroll
        for (int kk = 0; kk < 4; ++kk)
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                const int j = k - i;
                if (j < 0 || j >= NDB) continue;
                const uint32_t a = a_stage + (uint32_t)(i * 32 + kk * 8);
                const uint64_t bd = b_stage + (uint64_t)(j * TILE16 + kk * 2);
                if (first) umma_ts_i8(acc, a, bd, idesc, fresh ? 0u : 1u);
                else umma_ts_i8_acc(acc, a, bd, idesc);
                first = false;
            }
    }
}

__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

template <int BN>
__global__ void __launch_bounds__(NTHREADS, 1)
    contract_i8_kernel(const __grid_constant__ CUtensorMap tm_a0, const __grid_constant__ CUtensorMap tm_a1,
                       const __grid_constant__ CUtensorMap tm_a2, const __grid_constant__ CUtensorMap tm_d3,
                       const __grid_constant__ CUtensorMap tm_d1, const ParamsI8 prm)
{
    constexpr int STAGE_BI = BN * KB_B * 4;         // four 32-pixel fp32 boxes of BN rows (the D1 rows sit apart)
    constexpr int TILE = BN * KB_B;                 // one B digit tile (BN rows × 128 bytes)
    constexpr int STAGE_BD = NDB * TILE;
    constexpr int A_COL0 = NACC * BN;
    constexpr int PT = BN * KB_B / (NWARP_B * 32);  // pixels per B-former thread per stage (16 or 8)
    static_assert(BN == 32 || BN == 64, "BN");
    static_assert(A_COL0 + NSTAGE * A_STAGE_COLS <= TMEM_COLS, "A stages must fit in TMEM");
    static_assert(PT == 16 || PT == 8, "former pixels per thread");
    static_assert(NWARP_A == 4 && NEPI <= NWARP_A + NWARP_B, "warp roles");

    extern __shared__ __align__(1024) unsigned char smem_raw[];
    unsigned char *smem = (unsigned char *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    unsigned char *bin = smem;                       // NBI × STAGE_BI
    unsigned char *bdig = smem + NBI * STAGE_BI;     // NSTAGE × STAGE_BD
    unsigned char *atile = bdig + NSTAGE * STAGE_BD;  // NAS × 3 × A_BOX
    float *d1rows = reinterpret_cast<float *>(atile + NAS * 3 * A_BOX);  // NBI × KB_B fp32: the D1 row of each input stage
    uint64_t *bars = reinterpret_cast<uint64_t *>(d1rows + NBI * KB_B);
    uint64_t *as_full = bars, *as_empty = as_full + NAS;
    uint64_t *bin_full = as_empty + NAS, *bin_empty = bin_full + NBI;
    uint64_t *st_full = bin_empty + NBI, *st_empty = st_full + NSTAGE;
    uint64_t *acc_full = st_empty + NSTAGE;
    uint64_t *drain = acc_full + 1;  // one per issuer
    volatile uint32_t *tmem_slot = reinterpret_cast<volatile uint32_t *>(drain + NISSUE);
    volatile int *abort_flag = reinterpret_cast<volatile int *>(tmem_slot + 1);

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

    // Chunk-major order: the CTAs resident at one time share a pixel chunk, so
    // that chunk of every map row stays in L2 while all anchors read it.
    long item = blockIdx.x;
    const int nt = (int)(item % prm.nt_count);
    item /= prm.nt_count;
    const int mt = (int)(item % prm.mt_count);
    item /= prm.mt_count;
    const int aidx = (int)(item % prm.nanchors);
    const int chunk = (int)(item / prm.nanchors);
    const int p1 = prm.anchors[aidx];
    const long x_begin = (long)chunk * prm.chunk;
    const long x_end = min(prm.k, x_begin + prm.chunk);
    const int nb = (int)((x_end - x_begin + KB_B - 1) / KB_B);  // 128-pixel stages
    const int na = 2 * nb;                                      // 64-pixel D2 tiles
    const int bbase = p1 - prm.nc10 + nt * BN;                  // first p3 row of the B tile
    const int rbase = p1 - prm.nc10 + mt * BM;                  // first p2 row of the A tile
    const int E1 = prm.e1[p1];

    if (tid == 0) {
        for (int s = 0; s < NAS; ++s) { mbar_init(&as_full[s], 1); mbar_init(&as_empty[s], NWARP_A); }
        for (int s = 0; s < NBI; ++s) { mbar_init(&bin_full[s], 1); mbar_init(&bin_empty[s], NWARP_B); }
        for (int s = 0; s < NSTAGE; ++s) { mbar_init(&st_full[s], NWARP_A + NWARP_B); mbar_init(&st_empty[s], NISSUE); }
        mbar_init(acc_full, NISSUE);
        for (int q = 0; q < NISSUE; ++q) mbar_init(&drain[q], 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == WARP_MMA) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32((const void *)tmem_slot)),
                     "r"(TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem = *tmem_slot;
    bool ok = true;

    if (warp == WARP_TMA) {
        // fp32 inputs of the B formers: D3 rows [bbase, bbase+BN) as four 32-pixel swizzled boxes, D1 row p1.
        // Pixels past the end of the map and rows outside [0, nc) come back as zeros.
        if (lane == 0) {
            int issued = 0;
            for (int it = 0; it < nb; ++it) {
                const int s = it % NBI;
                if (!mbar_wait(&bin_empty[s], ((it / NBI) & 1) ^ 1, abort_flag, prm.err, 1)) break;
                unsigned char *t = bin + s * STAGE_BI;
                mbar_expect_tx(&bin_full[s], BN * KB_B * 4 + KB_B * 4);
                const int x = (int)(x_begin + (long)it * KB_B);
#pragma unroll
                for (int j = 0; j < 4; ++j) tma_load_2d(t + j * (BN * 128), &tm_d3, &bin_full[s], x + 32 * j, bbase);
                tma_load_2d(d1rows + s * KB_B, &tm_d1, &bin_full[s], x, p1);
                ++issued;
            }
            if (*abort_flag)
                for (int it = max(0, issued - NBI); it < issued; ++it)
                    for (long long i = 0; i < WAIT_LIMIT && !mbar_try_wait(&bin_full[it % NBI], (it / NBI) & 1); ++i)
                        __nanosleep(100);
        }
    } else if (warp == WARP_TMA_A) {
        // D2 digit planes, rows [rbase, rbase+128) × 64 pixels per tile; rows outside [0, nc) and
        // pixels past the end of the map come back as zeros.
        if (lane == 0) {
            int issued = 0;
            for (int ia = 0; ia < na; ++ia) {
                const int s = ia % NAS;
                if (!mbar_wait(&as_empty[s], ((ia / NAS) & 1) ^ 1, abort_flag, prm.err, 8)) break;
                unsigned char *t = atile + s * 3 * A_BOX;
                mbar_expect_tx(&as_full[s], 3 * A_BOX);
                const int x = (int)(x_begin + (long)ia * KB_A);
                tma_load_2d(t, &tm_a0, &as_full[s], x, rbase);
                tma_load_2d(t + A_BOX, &tm_a1, &as_full[s], x, rbase);
                tma_load_2d(t + 2 * A_BOX, &tm_a2, &as_full[s], x, rbase);
                ++issued;
            }
            if (*abort_flag)
                for (int ia = max(0, issued - NAS); ia < issued; ++ia)
                    for (long long i = 0; i < WAIT_LIMIT && !mbar_try_wait(&as_full[ia % NAS], (ia / NAS) & 1); ++i)
                        __nanosleep(100);
        }
    } else if (warp == WARP_MMA || warp == WARP_MMA2) {
        if (lane == 0) {
            const int q = warp == WARP_MMA ? 0 : 1;
            // S32 accumulate, signed int8 A and B, both K-major, M = 128, N = BN
            const uint32_t idesc = (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) |
                                   ((uint32_t)(BM >> 4) << 24);
            // descriptors are linear in the start address (bits 0-13, 16-byte units)
            const uint64_t desc0 = smem_desc_sw128(smem_u32(bdig));
            for (int it = 0; it < nb; ++it) {
                const int s = it & 1;
                if (!mbar_wait(&st_full[s], (it >> 1) & 1, abort_flag, prm.err, 2)) { ok = false; break; }
                fence_after();
                issue_stage<BN>(tmem, tmem + A_COL0 + s * A_STAGE_COLS, desc0 + (uint64_t)((s * STAGE_BD) >> 4), idesc,
                                q, it == 0);
                umma_commit(&st_empty[s]);
            }
            if (ok) {
                umma_commit(acc_full);
            } else {
                umma_commit(&drain[q]);
                for (long long i = 0; i < WAIT_LIMIT && !mbar_try_wait(&drain[q], 0); ++i) __nanosleep(100);
            }
        }
    } else if (warp < NWARP_A) {
        // ---- D2 digits → TMEM: warp w moves TMEM lanes [32w, 32w+32), all 64 pixels of each tile ----
        // Row m of a 64B-swizzled box holds its 16-byte chunk c at position c ^ ((m >> 1) & 3), so
        // eight consecutive rows reading the same chunk hit eight different bank groups.
        // tcgen05.st reads its source registers asynchronously: they are not reused before
        // tcgen05.wait::st, and a tile's shared memory is released only after that wait.
        const int m = (warp << 5) + lane;
        const uint32_t lane_field = (uint32_t)(warp << 5) << 16;
        const int sw = (m >> 1) & 3;
        for (int it = 0; it < nb && ok; ++it) {
            const int s = it & 1;
#pragma unroll 1
            for (int h = 0; h < 2; ++h) {
                const int ia = 2 * it + h, sa = ia % NAS;
                if (!mbar_wait_warp(&as_full[sa], (ia / NAS) & 1, abort_flag, prm.err, 9)) { ok = false; break; }
                const unsigned char *t = atile + sa * 3 * A_BOX + m * KB_A;
                uint32_t v[3][16];
#pragma unroll
                for (int d = 0; d < 3; ++d)
#pragma unroll
                    for (int c = 0; c < 4; ++c) {
                        const uint4 x = *reinterpret_cast<const uint4 *>(t + d * A_BOX + ((c ^ sw) << 4));
                        v[d][4 * c] = x.x; v[d][4 * c + 1] = x.y; v[d][4 * c + 2] = x.z; v[d][4 * c + 3] = x.w;
                    }
                if (h == 0) {
                    if (!mbar_wait_warp(&st_empty[s], ((it >> 1) & 1) ^ 1, abort_flag, prm.err, 4)) { ok = false; break; }
                    fence_after();
                }
                // pixels 64h .. 64h+63 of the stage = 32-pixel slices 2h, 2h+1: columns 16h .. 16h+15 of each digit
                const uint32_t col = tmem + lane_field + A_COL0 + s * A_STAGE_COLS + 16 * h;
#pragma unroll
                for (int d = 0; d < 3; ++d) tmem_st16(col + 32 * d, v[d]);
                asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
                __syncwarp();
                if (lane == 0) mbar_arrive(&as_empty[sa]);
            }
            if (!ok) break;
            fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(&st_full[s]);
        }
    } else if (warp < NWARP_A + NWARP_B) {
        // ---- B formers: thread (row n, segment sg) forms PT pixels of D1[p1]·D3[bbase+n] per stage ----
        const int tb = tid - NWARP_A * 32;  // 0 .. 32·NWARP_B − 1
        const int n = tb % BN, sg = tb / BN;
        const int px0 = sg * PT;  // first pixel of this thread inside the 128-pixel stage
        const int p3 = bbase + n;
        const bool col_ok = p3 >= 0 && p3 < prm.nc;
        const float scale = col_ok ? ldexpf(127.f, -(E1 + prm.e3[p3])) : 0.f;
        const float2 sc2 = make_float2(scale, scale);
        const int box = px0 / 32, c0 = (px0 % 32) / 4;  // input box and first 16-byte chunk in it
        // destination: 16-byte chunk px0/16 of each 128-byte digit row, at its swizzled position; PT = 8
        // fills one half of it
        const int dst_off = n * 128 + (((px0 / 16) ^ (n & 7)) << 4) + (px0 % 16);
        for (int it = 0; it < nb; ++it) {
            const int si = it % NBI, s = it & 1;
            if (!mbar_wait_warp(&bin_full[si], (it / NBI) & 1, abort_flag, prm.err, 6)) { ok = false; break; }
            const unsigned char *rowp = bin + si * STAGE_BI + box * (BN * 128) + n * 128;
            const float *d1p = d1rows + si * KB_B + px0;
            uint32_t w[NDB][PT / 4];
#pragma unroll
            for (int q = 0; q < PT / 4; ++q) {
                const float4 v = *reinterpret_cast<const float4 *>(rowp + (((c0 + q) ^ (n & 7)) << 4));
                const float4 u = *reinterpret_cast<const float4 *>(d1p + 4 * q);
                float2 ya0, ya1, ya2, ya3, yb0, yb1, yb2, yb3;
                digits254x2(__fmul2_rn(make_float2(u.x, u.y), sc2), make_float2(v.x, v.y), ya0, ya1, ya2, ya3);
                digits254x2(__fmul2_rn(make_float2(u.z, u.w), sc2), make_float2(v.z, v.w), yb0, yb1, yb2, yb3);
                w[0][q] = pack_low_bytes(ya0.x, ya0.y, yb0.x, yb0.y);
                w[1][q] = pack_low_bytes(ya1.x, ya1.y, yb1.x, yb1.y);
                w[2][q] = pack_low_bytes(ya2.x, ya2.y, yb2.x, yb2.y);
                w[3][q] = pack_low_bytes(ya3.x, ya3.y, yb3.x, yb3.y);
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(&bin_empty[si]);
            if (!mbar_wait_warp(&st_empty[s], ((it >> 1) & 1) ^ 1, abort_flag, prm.err, 7)) { ok = false; break; }
            unsigned char *dst = bdig + s * STAGE_BD + dst_off;
#pragma unroll
            for (int d = 0; d < NDB; ++d) {
                if constexpr (PT == 16)
                    *reinterpret_cast<uint4 *>(dst + d * TILE) = make_uint4(w[d][0], w[d][1], w[d][2], w[d][3]);
                else
                    *reinterpret_cast<uint2 *>(dst + d * TILE) = make_uint2(w[d][0], w[d][1]);
            }
            fence_proxy_async_smem();
            __syncwarp();
            if (lane == 0) mbar_arrive(&st_full[s]);
        }
    }

    // ---- epilogue (warps 0-15): int32 digit accumulators → FP64 partial tile; warpgroup wg reads BN/4 columns ----
    if (warp < NEPI) {
        const int wg = warp >> 2;
        const int m = ((warp & 3) << 5) + lane;
        const uint32_t lane_field = (uint32_t)((warp & 3) << 5) << 16;
        const bool good = __all_sync(0xffffffffu, ok) && mbar_wait_warp(acc_full, 0, abort_flag, prm.err, 5);
        if (good) {
            fence_after();
            const int d2 = mt * BM + m;
            const int p2 = rbase + m;
            const bool row_ok = d2 < prm.nclen && p2 >= 0 && p2 < prm.nc && prm.weight[p2] > 0;
            const int E12 = E1 + (row_ok ? prm.e2[p2] : 0);
            const double wr = row_ok ? (double)prm.weight[p1] * (double)prm.weight[p2] : 0.0;
            double *dst = nullptr;
            if (d2 < prm.nclen)
                dst = prm.partial + ((long)aidx * prm.nchunk + chunk) * prm.nclen * prm.nclen + (long)d2 * prm.nclen;
            const int c_begin = wg * (BN / 4), c_end = c_begin + BN / 4;
            const double i254 = 1.0 / 254.0, i254_2 = i254 * i254, i254_3 = i254_2 * i254;
            for (int c0 = c_begin; c0 < c_end; c0 += 8) {
                uint32_t v0[8], v1[8], v2[8], v3[8];
                tmem_ld8(tmem + lane_field + c0, v0);
                tmem_ld8(tmem + lane_field + BN + c0, v1);
                tmem_ld8(tmem + lane_field + 2 * BN + c0, v2);
                tmem_ld8(tmem + lane_field + 3 * BN + c0, v3);
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                if (dst) {
#pragma unroll
                    for (int j = 0; j < 8; ++j) {
                        const int nn = c0 + j;
                        const int d3 = nt * BN + nn;
                        if (d3 >= prm.nclen) continue;
                        const int p3 = bbase + nn;
                        double val = 0.0;
                        if (wr != 0.0 && p3 >= 0 && p3 < prm.nc && prm.weight[p3] > 0) {
                            const double s = (double)(int)v0[j] + (double)(int)v1[j] * i254 +
                                             (double)(int)v2[j] * i254_2 + (double)(int)v3[j] * i254_3;
                            val = ldexp(s * (1.0 / 16129.0), E12 + prm.e3[p3]) * wr * (double)prm.weight[p3];
                        }
                        dst[d3] = val;
                    }
                }
            }
        }
    }

    fence_before();
    __syncthreads();
    if (warp == WARP_MMA) {
        fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS));
    }
}

template <int BN>
size_t smem_bytes()
{
    return 1024 + (size_t)NBI * BN * KB_B * 4 + (size_t)NSTAGE * NDB * BN * KB_B + (size_t)NAS * 3 * A_BOX +
           (size_t)NBI * KB_B * 4 + 256;
}

typedef CUresult (*EncodeTiled)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

int encode(amber_cuda_ctx *c, CUtensorMap *m, CUtensorMapDataType dt, const void *plane, long k, long row_bytes,
           long rows, int box_x, int box_rows, CUtensorMapSwizzle sw)
{
    static EncodeTiled enc = nullptr;
    if (!enc) {
        void *fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess || !fn)
            return fail(c, AMBER_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
        enc = (EncodeTiled)fn;
    }
    cuuint64_t dims[2] = {(cuuint64_t)k, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)row_bytes};
    cuuint32_t box[2] = {(cuuint32_t)box_x, (cuuint32_t)box_rows};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = enc(m, dt, 2, (void *)plane, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, sw,
                     CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(c, AMBER_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
    return AMBER_OK;
}

template <int BN>
int launch(amber_cuda_ctx *c, const CUtensorMap (&ta)[3], const CUtensorMap &td3, const CUtensorMap &td1,
           const ParamsI8 &prm, long items)
{
    const size_t sm = smem_bytes<BN>();
    cudaFuncSetAttribute(contract_i8_kernel<BN>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    phase_begin(c, 1);
    contract_i8_kernel<BN><<<(unsigned)items, NTHREADS, sm, c->stream>>>(ta[0], ta[1], ta[2], td3, td1, prm);
    phase_end(c);
    c->launches += 1;
    c->contractions += 1;
    return cuda_check(c, cudaGetLastError(), "contract_i8_kernel launch");
}

// Pixel chunks per (anchor, tile) pair.  One CTA runs per SM, so the launch
// takes ceil(items / SMs) rounds of one chunk each; more chunks shorten a
// round but add a fixed cost per CTA (pipeline fill, epilogue) and partial
// tiles for lag_reduce to read.  Picks the count with the least modelled time.
long choose_chunks(long k, long pairs, int sms, long ncsize, long max_chunk)
{
    const long nch_min = std::max<long>(1, (k + max_chunk - 1) / max_chunk);
    const long nch_max = std::max<long>(nch_min, std::min<long>(4 * nch_min + 16, (k + 1023) / 1024));
    const double stage_s = 0.65e-6;     // one 128-pixel stage of one CTA
    const double fixed_s = 6 * stage_s;  // fill, drain and epilogue of one CTA
    const double reduce_bw = 5e12;      // bytes/s for lag_reduce reading the partial tiles
    long best = nch_min;
    double best_t = 1e300;
    for (long nch = nch_min; nch <= nch_max; ++nch) {
        const long chunk = ((k + nch - 1) / nch + KB_B - 1) / KB_B * KB_B;
        const long n = (k + chunk - 1) / chunk;
        if (n != nch) continue;
        const double rounds = std::ceil((double)(pairs * n) / sms);
        const double t = rounds * ((double)(chunk / KB_B) * stage_s + fixed_s) + 8.0 * pairs * n * ncsize / reduce_bw;
        if (t < best_t) { best_t = t; best = n; }
    }
    return best;
}

}  // namespace

int contract_i8(amber_cuda_ctx *c, const DigitMaps &m1, const DigitMaps &m2, const DigitMaps &m3, long k, long kp,
                double *lag_out)
{
    const int nc10 = c->nc10, nclen = 2 * nc10 + 1;
    const long ncsize = (long)nclen * nclen;
    const int nA = (int)c->anchors.size();
    if (nA == 0) return cuda_check(c, cudaMemsetAsync(lag_out, 0, sizeof(double) * ncsize, c->stream), "zero lag");
    const int MT = (nclen + BM - 1) / BM;
    const int BN = nclen <= 32 ? 32 : 64;
    const int NT = (nclen + BN - 1) / BN;
    const long base_items = (long)nA * MT * NT;
    long max_chunk = c->chunk_px > 0 ? std::min<long>(c->chunk_px, 32768) : 32768;
    max_chunk = std::max<long>(KB_B, max_chunk / KB_B * KB_B);
    long nch = choose_chunks(k, base_items, c->num_sms, ncsize, max_chunk);
    const long chunk = ((k + nch - 1) / nch + KB_B - 1) / KB_B * KB_B;
    nch = (k + chunk - 1) / chunk;

    int rc;
    const size_t pbytes = sizeof(double) * (size_t)nA * nch * ncsize;
    if ((rc = ensure(c, c->partial, pbytes, "partial lag tiles"))) return rc;
    if ((rc = ensure(c, c->misc, 256, "error flag"))) return rc;
    int *d_err = (int *)c->misc.p;
    if ((rc = cuda_check(c, cudaMemsetAsync(d_err, 0, sizeof(int), c->stream), "error flag"))) return rc;

    CUtensorMap ta[3], td3, td1;
    const CUtensorMapDataType u8 = CU_TENSOR_MAP_DATA_TYPE_UINT8, f32 = CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
    const int8_t *planes[3] = {m2.d0, m2.d1, m2.d2};
    for (int d = 0; d < 3; ++d)
        if ((rc = encode(c, &ta[d], u8, planes[d], k, kp, c->nc, KB_A, BM, CU_TENSOR_MAP_SWIZZLE_64B))) return rc;
    if ((rc = encode(c, &td3, f32, m3.f32, k, kp * 4, c->nc, 32, BN, CU_TENSOR_MAP_SWIZZLE_128B))) return rc;
    if ((rc = encode(c, &td1, f32, m1.f32, k, kp * 4, c->nc, KB_B, 1, CU_TENSOR_MAP_SWIZZLE_NONE))) return rc;
    ParamsI8 prm{};
    prm.nanchors = nA;
    prm.e1 = m1.expo; prm.e2 = m2.expo; prm.e3 = m3.expo;
    prm.k = k; prm.kp = kp;
    prm.nc = (int)c->nc; prm.nc10 = nc10; prm.nclen = nclen;
    prm.mt_count = MT; prm.nt_count = NT; prm.nchunk = (int)nch; prm.chunk = chunk;
    prm.anchors = (const int *)c->d_anchors.p;
    prm.weight = (const int *)c->d_weight.p;
    prm.partial = (double *)c->partial.p;
    prm.err = d_err;
    const long items = base_items * nch;
    switch (BN) {
        case 32: rc = launch<32>(c, ta, td3, td1, prm, items); break;
        case 64: rc = launch<64>(c, ta, td3, td1, prm, items); break;
        default: rc = fail(c, AMBER_ERR_ARG, "no int8 tile configuration for nclen=%d (BN=%d)", nclen, BN);
    }
    if (rc) return rc;
    if ((rc = lag_reduce(c, (const double *)c->partial.p, (long)nA * nch, ncsize, lag_out))) return rc;
    int herr = 0;
    if ((rc = cuda_check(c, cudaMemcpyAsync(&herr, d_err, sizeof(int), cudaMemcpyDeviceToHost, c->stream),
                         "error flag read")))
        return rc;
    if ((rc = cuda_check(c, cudaStreamSynchronize(c->stream), "contract_i8"))) return rc;
    if (herr) return fail(c, AMBER_ERR_TIMEOUT, "int8 tensor-core contraction: a pipeline wait gave up (site %d)", herr);
    return AMBER_OK;
}

}  // namespace amber
