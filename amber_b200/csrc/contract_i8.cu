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
//     T_p1[p2, p3] = Σ_x (D1[p1,x]·D2[p2,x]) · D3[p3,x]
// with M = p2 (128 TMEM lanes), N = p3 (BN ≤ 128), K = pixels:
//   A = D1[p1]·D2[p2] formed in FP32 on the CUDA cores from the maps' FP32
//       planes, scaled by 127·2^−(E1+E2) and cut into three int8 digits
//       written straight into TMEM (tcgen05.st; the "TS" MMA form);
//   B = the D3 digit planes, streamed by TMA into 128-byte-swizzled smem;
//   acc_k += Σ_{i+j=k} A_i·B_jᵀ for k = 0..3 — eight kind::i8 MMAs per 32
//       pixels into four int32 TMEM accumulators (the i+j = 4 term is below
//       2^−31 of the leading one).  Per pixel |Σ_{i+j=k}| ≤ 3·127² < 2^15.6,
//       so a chunk of up to 2^15 pixels cannot overflow.
// The k = 3 class matters: dropping it leaves ~2e-6 of Σ|products| on sharply
// peaked sampling-mask maps, keeping it gives ≤ 3e-7; four accumulators cap
// the p3 tile at 96 columns (TMEM holds 512).
// Epilogue: T = 2^(E1+E2+E3)/127² · Σ_k acc_k·254^−k in FP64,
// weighted by the channel multiplicities, written to the partial buffer
// [anchor][chunk][lag2][lag3]; lag_reduce then sums it per lag cell with a
// compensated FP64 accumulator in a fixed order (deterministic).
//
// Warp roles (608 threads): warps 0-15 form A from fp32 D1/D2 tiles that warp
// 17 stages in shared memory by TMA (3-deep ring, 128B-swizzled so the row
// reads are conflict-free), and later read the accumulators out; warp 16
// streams the D3 digit tiles by TMA; warp 18 owns TMEM and issues the MMAs
// from one lane.
// Every mbarrier wait is bounded; on expiry the CTA raises an error flag the
// host turns into AMBER_ERR_TIMEOUT, drains its own copies and MMAs, frees TMEM.
#include <algorithm>
#include <vector>

#include "common.cuh"
#include "tc_ptx.cuh"

namespace amber {

namespace {

using namespace tc;

constexpr int BM = 128;        // p2 rows per tile = TMEM lanes
constexpr int KB_B = 128;      // pixels per B stage: one 128-byte swizzle row of int8
constexpr int KB_A = 64;       // pixels per A stage in TMEM (two 32-pixel fp32 input boxes)
constexpr int NSI = 3;         // fp32 input stages in shared memory
constexpr int NACC = 4;        // int32 accumulators, one per digit class i+j = 0..3
constexpr int A_STAGE_COLS = 48;  // 3 digits × 16 columns (64 int8 per lane per digit)
constexpr int NWARP_A = 16;    // A-forming / epilogue warps: 4 warpgroups, 16 pixels each per A stage
constexpr int WARP_TMA_B = 16;
constexpr int WARP_TMA_A = 17;
constexpr int WARP_MMA = 18;
constexpr int NTHREADS = 19 * 32;
constexpr int TMEM_COLS = 512;
constexpr int IN_D2 = BM * KB_A * 4;  // bytes of one D2 input stage (two swizzled 32-pixel boxes)
constexpr int IN_D1 = KB_A * 4;       // bytes of the D1 row of one input stage
constexpr int IN_STAGE = IN_D2 + 1024;  // D1 row padded to keep 1024-byte alignment

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

// Three base-254 digits of t ∈ [−127, 127] (see quantize_kernel in maps.cu):
// round-to-nearest via the 1.5·2^23 magic number leaves each digit's
// two's-complement byte in the low mantissa bits.
__device__ __forceinline__ void digits254(float t, uint32_t &b0, uint32_t &b1, uint32_t &b2)
{
    const float M = 12582912.0f;
    float y0 = t + M;
    float r0 = (t - (y0 - M)) * 254.f;
    float y1 = r0 + M;
    float r1 = (r0 - (y1 - M)) * 254.f;
    float y2 = r1 + M;
    b0 = __float_as_uint(y0);
    b1 = __float_as_uint(y1);
    b2 = __float_as_uint(y2);
}

// The same three digits for two products u·v at once, with packed FP32x2
// arithmetic: every step is one fused op on a pair and the product u·v enters
// the first rounding unrounded (y0 = fma(u, v, M)).  M − y = −digit exactly.
__device__ __forceinline__ void digits254x2(float2 u, float2 v, float2 &y0, float2 &y1, float2 &y2)
{
    const float2 M = make_float2(12582912.0f, 12582912.0f);
    const float2 K254 = make_float2(254.f, 254.f);
    const float2 NEG1 = make_float2(-1.f, -1.f);
    y0 = __ffma2_rn(u, v, M);                   // M + d0
    const float2 nq0 = __ffma2_rn(y0, NEG1, M); // −d0
    const float2 r0 = __ffma2_rn(u, v, nq0);    // u·v − d0
    y1 = __ffma2_rn(r0, K254, M);               // M + d1
    const float2 nq1 = __ffma2_rn(y1, NEG1, M); // −d1
    const float2 s1 = __ffma2_rn(r0, K254, nq1); // 254·r0 − d1
    y2 = __ffma2_rn(s1, K254, M);               // M + d2
}

__device__ __forceinline__ uint32_t pack_low_bytes(uint32_t a, uint32_t b, uint32_t c, uint32_t d)
{
    return __byte_perm(__byte_perm(a, b, 0x0040), __byte_perm(c, d, 0x0040), 0x5410);
}

__device__ __forceinline__ void tmem_st4(uint32_t taddr, uint32_t a, uint32_t b, uint32_t c, uint32_t d)
{
    asm volatile("tcgen05.st.sync.aligned.32x32b.x4.b32 [%0], {%1, %2, %3, %4};" ::"r"(taddr), "r"(a), "r"(b),
                 "r"(c), "r"(d)
                 : "memory");
}

__device__ __forceinline__ void tmem_ld8(uint32_t taddr, uint32_t (&v)[8])
{
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7])
                 : "r"(taddr)
                 : "memory");
}

template <int BN>
__global__ void __launch_bounds__(NTHREADS, 1)
    contract_i8_kernel(const __grid_constant__ CUtensorMap tm0, const __grid_constant__ CUtensorMap tm1,
                       const __grid_constant__ CUtensorMap tm2, const __grid_constant__ CUtensorMap tmd2,
                       const __grid_constant__ CUtensorMap tmd1, const ParamsI8 prm)
{
    constexpr int TILE = BN * KB_B;  // bytes of one digit tile
    constexpr int STAGE_B = 3 * TILE;
    // TMEM: the four accumulators take 4·BN columns, the A stages the rest (≤ 4 stages)
    constexpr int A_COL0 = NACC * BN;
    constexpr int NSA = (TMEM_COLS - A_COL0) / A_STAGE_COLS < 4 ? (TMEM_COLS - A_COL0) / A_STAGE_COLS : 4;
    constexpr int NSB = ((200 * 1024 - NSI * IN_STAGE) / STAGE_B) < 4 ? ((200 * 1024 - NSI * IN_STAGE) / STAGE_B) : 4;
    static_assert(NSB >= 2, "shared memory too small for the B stages");
    static_assert(NSA >= 2, "TMEM must hold at least two A stages");
    static_assert(A_COL0 + NSA * A_STAGE_COLS <= TMEM_COLS, "A stages must fit in TMEM");
    static_assert(BN % 32 == 0 && BN >= 32 && BN <= 96, "BN");

    extern __shared__ __align__(1024) unsigned char smem_raw[];
    unsigned char *smem = (unsigned char *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    unsigned char *in_tiles = smem;                        // NSI × {D2 box 0, D2 box 1, D1 row}
    unsigned char *b_tiles = smem + NSI * IN_STAGE;        // NSB × {d0, d1, d2}
    uint64_t *bars = reinterpret_cast<uint64_t *>(b_tiles + NSB * STAGE_B);
    uint64_t *b_full = bars, *b_empty = bars + NSB;
    uint64_t *a_full = bars + 2 * NSB, *a_empty = a_full + NSA;
    uint64_t *in_full = a_empty + NSA, *in_empty = in_full + NSI;
    uint64_t *acc_full = in_empty + NSI;
    uint64_t *drain = acc_full + 1;
    volatile uint32_t *tmem_slot = reinterpret_cast<volatile uint32_t *>(drain + 1);
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
    const int nb = (int)((x_end - x_begin + KB_B - 1) / KB_B);  // B stages; 2 A stages each
    const int na = 2 * nb;
    const int bbase = p1 - prm.nc10 + nt * BN;                  // first p3 row of the B tile
    const int rbase = p1 - prm.nc10 + mt * BM;                  // first p2 row of the A tile

    if (tid == 0) {
        for (int s = 0; s < NSB; ++s) { mbar_init(&b_full[s], 1); mbar_init(&b_empty[s], 1); }
        for (int s = 0; s < NSA; ++s) { mbar_init(&a_full[s], NWARP_A); mbar_init(&a_empty[s], 1); }
        for (int s = 0; s < NSI; ++s) { mbar_init(&in_full[s], 1); mbar_init(&in_empty[s], NWARP_A); }
        mbar_init(acc_full, 1);
        mbar_init(drain, 1);
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

    if (warp == WARP_TMA_B) {
        // B operand: the D3 digit planes, 128 pixels × BN rows per stage
        if (lane == 0) {
            int issued = 0;
            for (int it = 0; it < nb; ++it) {
                const int s = it % NSB;
                if (!mbar_wait(&b_empty[s], ((it / NSB) & 1) ^ 1, abort_flag, prm.err, 1)) break;
                unsigned char *t0 = b_tiles + s * STAGE_B;
                mbar_expect_tx(&b_full[s], STAGE_B);
                const int x = (int)(x_begin + (long)it * KB_B);
                tma_load_2d(t0, &tm0, &b_full[s], x, bbase);
                tma_load_2d(t0 + TILE, &tm1, &b_full[s], x, bbase);
                tma_load_2d(t0 + 2 * TILE, &tm2, &b_full[s], x, bbase);
                ++issued;
            }
            if (*abort_flag)
                for (int it = max(0, issued - NSB); it < issued; ++it)
                    for (long long i = 0; i < WAIT_LIMIT && !mbar_try_wait(&b_full[it % NSB], (it / NSB) & 1); ++i)
                        __nanosleep(100);
        }
    } else if (warp == WARP_TMA_A) {
        // A inputs: 64 pixels of the 128 D2 rows (two swizzled 32-pixel boxes) and of the D1 row.
        // Pixels past the end of the map come back as zeros, rows outside [0, nc) too.
        if (lane == 0) {
            int issued = 0;
            for (int ia = 0; ia < na; ++ia) {
                const int s = ia % NSI;
                if (!mbar_wait(&in_empty[s], ((ia / NSI) & 1) ^ 1, abort_flag, prm.err, 6)) break;
                unsigned char *t = in_tiles + s * IN_STAGE;
                mbar_expect_tx(&in_full[s], IN_D2 + IN_D1);
                const int x = (int)(x_begin + (long)ia * KB_A);
                tma_load_2d(t, &tmd2, &in_full[s], x, rbase);
                tma_load_2d(t + IN_D2 / 2, &tmd2, &in_full[s], x + 32, rbase);
                tma_load_2d(t + IN_D2, &tmd1, &in_full[s], x, p1);
                ++issued;
            }
            if (*abort_flag)
                for (int ia = max(0, issued - NSI); ia < issued; ++ia)
                    for (long long i = 0; i < WAIT_LIMIT && !mbar_try_wait(&in_full[ia % NSI], (ia / NSI) & 1); ++i)
                        __nanosleep(100);
        }
    } else if (warp == WARP_MMA) {
        if (lane == 0) {
            // S32 accumulate, signed int8 A and B, both K-major, M = 128, N = BN
            const uint32_t idesc = (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) |
                                   ((uint32_t)(BM >> 4) << 24);
            const uint32_t acc0 = tmem, acc1 = tmem + BN, acc2 = tmem + 2 * BN, acc3 = tmem + 3 * BN;
            // descriptors are linear in the start address (bits 0-13, 16-byte units): build the
            // first one once and advance it by (byte offset >> 4)
            const uint64_t desc0 = smem_desc_sw128(smem_u32(b_tiles));
            bool ok = true;
            uint32_t started = 0;
            for (int it = 0; it < nb && ok; ++it) {
                const int sb = it % NSB;
                if (!mbar_wait(&b_full[sb], (it / NSB) & 1, abort_flag, prm.err, 2)) { ok = false; break; }
                const uint64_t dstage = desc0 + (uint64_t)((sb * STAGE_B) >> 4);
                for (int h = 0; h < 2; ++h) {
                    const int ia = 2 * it + h, sa = ia % NSA;
                    if (!mbar_wait(&a_full[sa], (ia / NSA) & 1, abort_flag, prm.err, 3)) { ok = false; break; }
                    fence_after();
#pragma unroll
                    for (int kk = 0; kk < 2; ++kk) {
                        const uint64_t B0 = dstage + (uint64_t)((2 * h + kk) * 2), B1 = B0 + (TILE >> 4),
                                       B2 = B0 + (2 * TILE >> 4);
                        const uint32_t a = tmem + A_COL0 + sa * A_STAGE_COLS + kk * 8;
                        const uint32_t A0 = a, A1 = a + 16, A2 = a + 32;
                        umma_ts_i8(acc0, A0, B0, idesc, started);  // i+j = 0
                        umma_ts_i8(acc1, A0, B1, idesc, started);  // i+j = 1
                        umma_ts_i8(acc1, A1, B0, idesc, 1u);
                        umma_ts_i8(acc2, A0, B2, idesc, started);  // i+j = 2
                        umma_ts_i8(acc2, A1, B1, idesc, 1u);
                        umma_ts_i8(acc2, A2, B0, idesc, 1u);
                        umma_ts_i8(acc3, A1, B2, idesc, started);  // i+j = 3
                        umma_ts_i8(acc3, A2, B1, idesc, 1u);
                        started = 1u;
                    }
                    umma_commit(&a_empty[sa]);
                }
                if (ok) umma_commit(&b_empty[sb]);
            }
            if (ok) {
                umma_commit(acc_full);
            } else {
                umma_commit(drain);
                for (long long i = 0; i < WAIT_LIMIT && !mbar_try_wait(drain, 0); ++i) __nanosleep(100);
            }
        }
    } else {
        // ---- A formation: warps 0-15; warpgroup g covers pixels [16g, 16g + 16) of each A stage ----
        const int g = warp >> 2;
        const int m = ((warp & 3) << 5) + lane;
        const uint32_t lane_field = (uint32_t)((warp & 3) << 5) << 16;
        const int d2 = mt * BM + m;
        const int p2 = rbase + m;
        const bool row_ok = d2 < prm.nclen && p2 >= 0 && p2 < prm.nc && prm.weight[p2] > 0;
        const int E1 = prm.e1[p1];
        const int E2 = row_ok ? prm.e2[p2] : 0;
        const float scale = row_ok ? ldexpf(127.f, -(E1 + E2)) : 0.f;  // A·127·2^−(E1+E2) ∈ [−127, 127]
        // this thread's 16 pixels: 16-byte chunks j0..j0+3 of one 32-pixel box, 128B-swizzled by row
        const int box = g >> 1, j0 = (g & 1) * 4;
        const int px0 = g * 16;
        bool ok = true;
        for (int ia = 0; ia < na; ++ia) {
            const int si = ia % NSI, sa = ia % NSA;
            if (!mbar_wait_warp(&in_full[si], (ia / NSI) & 1, abort_flag, prm.err, 7)) { ok = false; break; }
            const unsigned char *t = in_tiles + si * IN_STAGE;
            const float *rowp = reinterpret_cast<const float *>(t + box * (IN_D2 / 2) + m * 128);
            const float *d1p = reinterpret_cast<const float *>(t + IN_D2) + px0;
            uint32_t w[3][4];
            const float2 sc2 = make_float2(scale, scale);
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const float4 v = *reinterpret_cast<const float4 *>(rowp + (((j0 + q) ^ (m & 7)) << 2));
                const float4 u = *reinterpret_cast<const float4 *>(d1p + 4 * q);
                float2 ya0, ya1, ya2, yb0, yb1, yb2;
                digits254x2(__fmul2_rn(make_float2(u.x, u.y), sc2), make_float2(v.x, v.y), ya0, ya1, ya2);
                digits254x2(__fmul2_rn(make_float2(u.z, u.w), sc2), make_float2(v.z, v.w), yb0, yb1, yb2);
                w[0][q] = pack_low_bytes(__float_as_uint(ya0.x), __float_as_uint(ya0.y), __float_as_uint(yb0.x),
                                         __float_as_uint(yb0.y));
                w[1][q] = pack_low_bytes(__float_as_uint(ya1.x), __float_as_uint(ya1.y), __float_as_uint(yb1.x),
                                         __float_as_uint(yb1.y));
                w[2][q] = pack_low_bytes(__float_as_uint(ya2.x), __float_as_uint(ya2.y), __float_as_uint(yb2.x),
                                         __float_as_uint(yb2.y));
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(&in_empty[si]);
            if (!mbar_wait_warp(&a_empty[sa], ((ia / NSA) & 1) ^ 1, abort_flag, prm.err, 4)) { ok = false; break; }
            fence_after();
            const uint32_t col = tmem + lane_field + A_COL0 + sa * A_STAGE_COLS + g * 4;
            tmem_st4(col, w[0][0], w[0][1], w[0][2], w[0][3]);
            tmem_st4(col + 16, w[1][0], w[1][1], w[1][2], w[1][3]);
            tmem_st4(col + 32, w[2][0], w[2][1], w[2][2], w[2][3]);
            asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
            fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(&a_full[sa]);
        }

        // ---- epilogue: int32 digit accumulators → FP64 partial tile; warpgroup g reads BN/4 columns ----
        if (ok && mbar_wait_warp(acc_full, 0, abort_flag, prm.err, 5)) {
            fence_after();
            const double wr = row_ok ? (double)prm.weight[p1] * (double)prm.weight[p2] : 0.0;
            double *dst = nullptr;
            if (d2 < prm.nclen)
                dst = prm.partial + ((long)aidx * prm.nchunk + chunk) * prm.nclen * prm.nclen + (long)d2 * prm.nclen;
            const int c_begin = g * (BN / 4), c_end = c_begin + BN / 4;
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
                        const int n = c0 + j;
                        const int d3 = nt * BN + n;
                        if (d3 >= prm.nclen) continue;
                        const int p3 = bbase + n;
                        double val = 0.0;
                        if (wr != 0.0 && p3 >= 0 && p3 < prm.nc && prm.weight[p3] > 0) {
                            const double s = (double)(int)v0[j] + (double)(int)v1[j] * i254 +
                                             (double)(int)v2[j] * i254_2 + (double)(int)v3[j] * i254_3;
                            val = ldexp(s * (1.0 / 16129.0), E1 + E2 + prm.e3[p3]) * wr * (double)prm.weight[p3];
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
size_t smem_bytes()  // NSB as in the kernel
{
    constexpr int STAGE_B = 3 * BN * KB_B;
    constexpr int NSB = ((200 * 1024 - NSI * IN_STAGE) / STAGE_B) < 4 ? ((200 * 1024 - NSI * IN_STAGE) / STAGE_B) : 4;
    return 1024 + (size_t)NSI * IN_STAGE + (size_t)NSB * STAGE_B + 256;
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
int launch(amber_cuda_ctx *c, const CUtensorMap &t0, const CUtensorMap &t1, const CUtensorMap &t2,
           const CUtensorMap &td2, const CUtensorMap &td1, const ParamsI8 &prm, long items)
{
    const size_t sm = smem_bytes<BN>();
    cudaFuncSetAttribute(contract_i8_kernel<BN>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    phase_begin(c, 1);
    contract_i8_kernel<BN><<<(unsigned)items, NTHREADS, sm, c->stream>>>(t0, t1, t2, td2, td1, prm);
    phase_end(c);
    c->launches += 1;
    c->contractions += 1;
    return cuda_check(c, cudaGetLastError(), "contract_i8_kernel launch");
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
    const int NT = (nclen + 95) / 96;
    const int BN = ((nclen + NT - 1) / NT + 31) / 32 * 32;
    const long base_items = (long)nA * MT * NT;
    const long target = 4L * c->num_sms;
    long max_chunk = c->chunk_px > 0 ? std::min<long>(c->chunk_px, 32768) : 32768;
    max_chunk = std::max<long>(KB_B, max_chunk / KB_B * KB_B);
    long nch = std::max<long>((k + max_chunk - 1) / max_chunk,
                              std::min<long>((target + base_items - 1) / base_items, (k + 1023) / 1024));
    nch = std::max<long>(nch, 1);
    long chunk = ((k + nch - 1) / nch + KB_B - 1) / KB_B * KB_B;
    nch = (k + chunk - 1) / chunk;

    int rc;
    const size_t pbytes = sizeof(double) * (size_t)nA * nch * ncsize;
    if ((rc = ensure(c, c->partial, pbytes, "partial lag tiles"))) return rc;
    if ((rc = ensure(c, c->misc, 256, "error flag"))) return rc;
    int *d_err = (int *)c->misc.p;
    if ((rc = cuda_check(c, cudaMemsetAsync(d_err, 0, sizeof(int), c->stream), "error flag"))) return rc;

    CUtensorMap t0, t1, t2, td2, td1;
    const CUtensorMapDataType u8 = CU_TENSOR_MAP_DATA_TYPE_UINT8, f32 = CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
    if ((rc = encode(c, &t0, u8, m3.d0, k, kp, c->nc, KB_B, BN, CU_TENSOR_MAP_SWIZZLE_128B))) return rc;
    if ((rc = encode(c, &t1, u8, m3.d1, k, kp, c->nc, KB_B, BN, CU_TENSOR_MAP_SWIZZLE_128B))) return rc;
    if ((rc = encode(c, &t2, u8, m3.d2, k, kp, c->nc, KB_B, BN, CU_TENSOR_MAP_SWIZZLE_128B))) return rc;
    if ((rc = encode(c, &td2, f32, m2.f32, k, kp * 4, c->nc, 32, BM, CU_TENSOR_MAP_SWIZZLE_128B))) return rc;
    if ((rc = encode(c, &td1, f32, m1.f32, k, kp * 4, c->nc, KB_A, 1, CU_TENSOR_MAP_SWIZZLE_NONE))) return rc;
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
        case 32: rc = launch<32>(c, t0, t1, t2, td2, td1, prm, items); break;
        case 64: rc = launch<64>(c, t0, t1, t2, td2, td1, prm, items); break;
        case 96: rc = launch<96>(c, t0, t1, t2, td2, td1, prm, items); break;
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
