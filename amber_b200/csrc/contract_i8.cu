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
//
// contract_i8_ss_kernel (below) is the 128-wide variant with both MMA operands in
// shared memory (tile_n = 128); it computes bit-identical results and is chosen
// only on request.
#include <algorithm>
#include <cmath>
#include <deque>
#include <map>
#include <mutex>
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

// One contraction job (one triangle's D or mask pass) as the kernel sees it.
// Lives in device memory; the tensor maps are read from there by TMA.
struct alignas(64) JobDesc {
    CUtensorMap ta[3];  // D2 digit planes: box {64 px, 128 rows}, 64B swizzle
    CUtensorMap td3;    // D3 fp32: box {32 px, BN rows}, 128B swizzle
    CUtensorMap td1;    // D1 fp32: box {128 px, 1 row}
    const int *e1, *e2, *e3;  // row exponents [nc]
    const int *anchors;       // channels with weight > 0
    const int *weight;        // channel multiplicities [nc]
    double *partial;          // [anchor][chunk][nclen²]
    long k, kp;
    long chunk;               // pixels per chunk (multiple of KB_B)
    int nc, nc10, nclen;
    int mt_count, nt_count, nchunk, nanchors;
};

// Work item: job index and the item's index inside the job (chunk-major).
struct Item {
    int job;
    int local;
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

// Decoded work item: everything a role needs to run one (anchor, tile, chunk).
struct ItemView {
    const JobDesc *j;
    int nt, mt, aidx, chunk, p1, nb, bbase, rbase, E1;
    long x_begin;
};

template <int BN>
__device__ __forceinline__ ItemView decode(const JobDesc *jobs, const Item *items, int g)
{
    ItemView v;
    const Item it = items[g];
    v.j = jobs + it.job;
    const JobDesc &j = *v.j;
    long q = it.local;
    v.nt = (int)(q % j.nt_count);
    q /= j.nt_count;
    v.mt = (int)(q % j.mt_count);
    q /= j.mt_count;
    v.aidx = (int)(q % j.nanchors);
    v.chunk = (int)(q / j.nanchors);
    v.p1 = j.anchors[v.aidx];
    v.x_begin = (long)v.chunk * j.chunk;
    const long x_end = min(j.k, v.x_begin + j.chunk);
    v.nb = (int)((x_end - v.x_begin + KB_B - 1) / KB_B);  // 128-pixel stages
    v.bbase = v.p1 - j.nc10 + v.nt * BN;                 // first p3 row of the B tile
    v.rbase = v.p1 - j.nc10 + v.mt * BM;                 // first p2 row of the A tile
    v.E1 = j.e1[v.p1];
    return v;
}

// Persistent: CTA b runs items b, b + gridDim.x, ... of the list (jobs one after the other,
// each chunk-major, so the CTAs resident at one time share a pixel chunk of one job in L2).
// The pipelines run on across items: stage and tile counters are global to the CTA, TMEM
// stays allocated, and the accumulators are handed from the MMA issuers to the epilogue
// warps and back once per item (acc_full / acc_empty).
template <int BN>
__global__ void __launch_bounds__(NTHREADS, 1)
    contract_i8_kernel(const JobDesc *__restrict__ jobs, const Item *__restrict__ items, int nitems, int *err)
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
    unsigned char *bin = smem;                        // NBI × STAGE_BI
    unsigned char *bdig = smem + NBI * STAGE_BI;      // NSTAGE × STAGE_BD
    unsigned char *atile = bdig + NSTAGE * STAGE_BD;  // NAS × 3 × A_BOX
    float *d1rows = reinterpret_cast<float *>(atile + NAS * 3 * A_BOX);  // NBI × KB_B fp32: the D1 row of each input stage
    uint64_t *bars = reinterpret_cast<uint64_t *>(d1rows + NBI * KB_B);
    uint64_t *as_full = bars, *as_empty = as_full + NAS;
    uint64_t *bin_full = as_empty + NAS, *bin_empty = bin_full + NBI;
    uint64_t *st_full = bin_empty + NBI, *st_empty = st_full + NSTAGE;
    uint64_t *acc_full = st_empty + NSTAGE, *acc_empty = acc_full + 1;
    uint64_t *drain = acc_empty + 1;  // one per issuer
    volatile uint32_t *tmem_slot = reinterpret_cast<volatile uint32_t *>(drain + NISSUE);
    volatile int *abort_flag = reinterpret_cast<volatile int *>(tmem_slot + 1);

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

    if (tid == 0) {
        for (int s = 0; s < NAS; ++s) { mbar_init(&as_full[s], 1); mbar_init(&as_empty[s], NWARP_A); }
        for (int s = 0; s < NBI; ++s) { mbar_init(&bin_full[s], 1); mbar_init(&bin_empty[s], NWARP_B); }
        for (int s = 0; s < NSTAGE; ++s) { mbar_init(&st_full[s], NWARP_A + NWARP_B); mbar_init(&st_empty[s], NISSUE); }
        mbar_init(acc_full, NISSUE);
        mbar_init(acc_empty, NEPI);
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
            int gs = 0;  // stages issued so far
            for (int g = blockIdx.x; g < nitems && ok; g += gridDim.x) {
                const ItemView v = decode<BN>(jobs, items, g);
                for (int it = 0; it < v.nb; ++it, ++gs) {
                    const int s = (gs % NBI);
                    if (!mbar_wait(&bin_empty[s], ((gs / NBI) & 1) ^ 1, abort_flag, err, 1)) { ok = false; break; }
                    unsigned char *t = bin + s * STAGE_BI;
                    mbar_expect_tx(&bin_full[s], BN * KB_B * 4 + KB_B * 4);
                    const int x = (int)(v.x_begin + (long)it * KB_B);
#pragma unroll
                    for (int jb = 0; jb < 4; ++jb)
                        tma_load_2d(t + jb * (BN * 128), &v.j->td3, &bin_full[s], x + 32 * jb, v.bbase);
                    tma_load_2d(d1rows + s * KB_B, &v.j->td1, &bin_full[s], x, v.p1);
                }
            }
            if (!ok)
                for (int q = max(0, gs - NBI); q < gs; ++q)
                    for (long long i = 0; i < WAIT_LIMIT && !mbar_try_wait(&bin_full[q % NBI], ((q / NBI) & 1)); ++i)
                        __nanosleep(100);
        }
    } else if (warp == WARP_TMA_A) {
        // D2 digit planes, rows [rbase, rbase+128) × 64 pixels per tile; rows outside [0, nc) and
        // pixels past the end of the map come back as zeros.
        if (lane == 0) {
            int gt = 0;  // tiles issued so far
            for (int g = blockIdx.x; g < nitems && ok; g += gridDim.x) {
                const ItemView v = decode<BN>(jobs, items, g);
                for (int ia = 0; ia < 2 * v.nb; ++ia, ++gt) {
                    const int s = (gt % NAS);
                    if (!mbar_wait(&as_empty[s], ((gt / NAS) & 1) ^ 1, abort_flag, err, 8)) { ok = false; break; }
                    unsigned char *t = atile + s * 3 * A_BOX;
                    mbar_expect_tx(&as_full[s], 3 * A_BOX);
                    const int x = (int)(v.x_begin + (long)ia * KB_A);
                    tma_load_2d(t, &v.j->ta[0], &as_full[s], x, v.rbase);
                    tma_load_2d(t + A_BOX, &v.j->ta[1], &as_full[s], x, v.rbase);
                    tma_load_2d(t + 2 * A_BOX, &v.j->ta[2], &as_full[s], x, v.rbase);
                }
            }
            if (!ok)
                for (int q = max(0, gt - NAS); q < gt; ++q)
                    for (long long i = 0; i < WAIT_LIMIT && !mbar_try_wait(&as_full[q % NAS], ((q / NAS) & 1)); ++i)
                        __nanosleep(100);
        }
    } else if (warp == WARP_MMA || warp == WARP_MMA2) {
        // Two issuers feed the tensor pipe from independent instruction streams, so one
        // thread's barrier wait or commit does not leave the pipe idle.
        if (lane == 0) {
            const int q = warp == WARP_MMA ? 0 : 1;
            // S32 accumulate, signed int8 A and B, both K-major, M = 128, N = BN
            const uint32_t idesc = (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) |
                                   ((uint32_t)(BM >> 4) << 24);
            // descriptors are linear in the start address (bits 0-13, 16-byte units)
            const uint64_t desc0 = smem_desc_sw128(smem_u32(bdig));
            int gs = 0, seq = 0;
            for (int g = blockIdx.x; g < nitems && ok; g += gridDim.x, ++seq) {
                const int nb = decode<BN>(jobs, items, g).nb;
                // the epilogue of the previous item has read the accumulators out
                if (!mbar_wait(acc_empty, (seq & 1) ^ 1, abort_flag, err, 10)) { ok = false; break; }
                for (int it = 0; it < nb; ++it, ++gs) {
                    const int s = (gs & 1);
                    if (!mbar_wait(&st_full[s], ((gs >> 1) & 1), abort_flag, err, 2)) { ok = false; break; }
                    fence_after();
                    issue_stage<BN>(tmem, tmem + A_COL0 + s * A_STAGE_COLS, desc0 + (uint64_t)((s * STAGE_BD) >> 4),
                                    idesc, q, it == 0);
                    umma_commit(&st_empty[s]);
                }
                if (ok) umma_commit(acc_full);
            }
            if (!ok) {
                umma_commit(&drain[q]);
                for (long long i = 0; i < WAIT_LIMIT && !mbar_try_wait(&drain[q], 0); ++i) __nanosleep(100);
            }
        }
    } else {
        // ---- warps 0-19: D2 movers (0-3) and B formers (4-19); warps 0-15 also run each item's epilogue ----
        const bool mover = warp < NWARP_A;
        // mover: TMEM lanes [32w, 32w+32), all 64 pixels of each tile
        const int m = (warp << 5) + lane;
        const uint32_t lane_field = (uint32_t)((warp & 3) << 5) << 16;
        const int sw = (m >> 1) & 3;
        // former: thread (row n, segment sg) forms PT pixels of D1[p1]·D3[bbase+n] per stage
        const int tb = tid - NWARP_A * 32;
        const int n = tb % BN, sg = tb / BN;
        const int px0 = sg * PT;
        const int box = px0 / 32, c0 = (px0 % 32) / 4;  // input box and first 16-byte chunk in it
        // destination: 16-byte chunk px0/16 of each 128-byte digit row, at its swizzled position; PT = 8
        // fills one half of it
        const int dst_off = n * 128 + (((px0 / 16) ^ (n & 7)) << 4) + (px0 % 16);
        int gs = 0, gt = 0, seq = 0;
        // ---- epilogue (warps 0-15): int32 digit accumulators → FP64 partial tile; warpgroup wg reads BN/4 columns ----
        auto epilogue_item = [&](int g) {
            const ItemView v = decode<BN>(jobs, items, g);
            const JobDesc &j = *v.j;
            const int wg = warp >> 2;
            const int me = ((warp & 3) << 5) + lane;
            const bool good = __all_sync(0xffffffffu, ok) && mbar_wait_warp(acc_full, (seq & 1), abort_flag, err, 5);
            if (!good) { ok = false; return; }
            fence_after();
            const int d2 = v.mt * BM + me;
            const int p2 = v.rbase + me;
            const bool row_ok = d2 < j.nclen && p2 >= 0 && p2 < j.nc && j.weight[p2] > 0;
            const int E12 = v.E1 + (row_ok ? j.e2[p2] : 0);
            const double wr = row_ok ? (double)j.weight[v.p1] * (double)j.weight[p2] : 0.0;
            double *dst = nullptr;
            if (d2 < j.nclen)
                dst = j.partial + ((long)v.aidx * j.nchunk + v.chunk) * j.nclen * j.nclen + (long)d2 * j.nclen;
            const int c_begin = wg * (BN / 4), c_end = c_begin + BN / 4;
            const double i254 = 1.0 / 254.0, i254_2 = i254 * i254, i254_3 = i254_2 * i254;
            for (int cb = c_begin; cb < c_end; cb += 8) {
                uint32_t v0[8], v1[8], v2[8], v3[8];
                tmem_ld8(tmem + lane_field + cb, v0);
                tmem_ld8(tmem + lane_field + BN + cb, v1);
                tmem_ld8(tmem + lane_field + 2 * BN + cb, v2);
                tmem_ld8(tmem + lane_field + 3 * BN + cb, v3);
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                if (cb + 8 >= c_end) {
                    // last read of this item: hand the accumulators back to the MMA issuers
                    fence_before();
                    __syncwarp();
                    if (lane == 0) mbar_arrive(acc_empty);
                }
                if (dst) {
#pragma unroll
                    for (int e = 0; e < 8; ++e) {
                        const int nn = cb + e;
                        const int d3 = v.nt * BN + nn;
                        if (d3 >= j.nclen) continue;
                        const int p3 = v.bbase + nn;
                        double val = 0.0;
                        if (wr != 0.0 && p3 >= 0 && p3 < j.nc && j.weight[p3] > 0) {
                            const double sm = (double)(int)v0[e] + (double)(int)v1[e] * i254 +
                                              (double)(int)v2[e] * i254_2 + (double)(int)v3[e] * i254_3;
                            val = ldexp(sm * (1.0 / 16129.0), E12 + j.e3[p3]) * wr * (double)j.weight[p3];
                        }
                        dst[d3] = val;
                    }
                }
            }
        };
        for (int g = blockIdx.x; g < nitems && ok; g += gridDim.x, ++seq) {
            const ItemView v = decode<BN>(jobs, items, g);
            const JobDesc &j = *v.j;
            if (mover) {
                // tcgen05.st reads its source registers asynchronously: they are not reused before
                // tcgen05.wait::st, and a tile's shared memory is released only after that wait.
                for (int it = 0; it < v.nb && ok; ++it, ++gs) {
                    const int s = (gs & 1);
#pragma unroll 1
                    for (int h = 0; h < 2; ++h, ++gt) {
                        const int sa = (gt % NAS);
                        if (!mbar_wait_warp(&as_full[sa], ((gt / NAS) & 1), abort_flag, err, 9)) { ok = false; break; }
                        const unsigned char *t = atile + sa * 3 * A_BOX + m * KB_A;
                        uint32_t r[3][16];
#pragma unroll
                        for (int d = 0; d < 3; ++d)
#pragma unroll
                            for (int c = 0; c < 4; ++c) {
                                const uint4 x = *reinterpret_cast<const uint4 *>(t + d * A_BOX + ((c ^ sw) << 4));
                                r[d][4 * c] = x.x; r[d][4 * c + 1] = x.y; r[d][4 * c + 2] = x.z; r[d][4 * c + 3] = x.w;
                            }
                        if (h == 0) {
                            if (!mbar_wait_warp(&st_empty[s], ((gs >> 1) & 1) ^ 1, abort_flag, err, 4)) { ok = false; break; }
                            fence_after();
                        }
                        // pixels 64h .. 64h+63 of the stage = 32-pixel slices 2h, 2h+1: columns 16h .. 16h+15 of each digit
                        const uint32_t col = tmem + lane_field + A_COL0 + s * A_STAGE_COLS + 16 * h;
#pragma unroll
                        for (int d = 0; d < 3; ++d) tmem_st16(col + 32 * d, r[d]);
                        asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
                        __syncwarp();
                        if (lane == 0) mbar_arrive(&as_empty[sa]);
                    }
                    if (!ok) break;
                    fence_before();
                    __syncwarp();
                    if (lane == 0) mbar_arrive(&st_full[s]);
                }
            } else {
                const int p3 = v.bbase + n;
                const bool col_ok = p3 >= 0 && p3 < j.nc;
                const float scale = col_ok ? ldexpf(127.f, -(v.E1 + j.e3[p3])) : 0.f;
                const float2 sc2 = make_float2(scale, scale);
                for (int it = 0; it < v.nb; ++it, ++gs) {
                    const int si = (gs % NBI), s = (gs & 1);
                    if (!mbar_wait_warp(&bin_full[si], ((gs / NBI) & 1), abort_flag, err, 6)) { ok = false; break; }
                    const unsigned char *rowp = bin + si * STAGE_BI + box * (BN * 128) + n * 128;
                    const float *d1p = d1rows + si * KB_B + px0;
                    uint32_t w[NDB][PT / 4];
#pragma unroll
                    for (int q = 0; q < PT / 4; ++q) {
                        const float4 x3 = *reinterpret_cast<const float4 *>(rowp + (((c0 + q) ^ (n & 7)) << 4));
                        const float4 u = *reinterpret_cast<const float4 *>(d1p + 4 * q);
                        float2 ya0, ya1, ya2, ya3, yb0, yb1, yb2, yb3;
                        digits254x2(__fmul2_rn(make_float2(u.x, u.y), sc2), make_float2(x3.x, x3.y), ya0, ya1, ya2, ya3);
                        digits254x2(__fmul2_rn(make_float2(u.z, u.w), sc2), make_float2(x3.z, x3.w), yb0, yb1, yb2, yb3);
                        w[0][q] = pack_low_bytes(ya0.x, ya0.y, yb0.x, yb0.y);
                        w[1][q] = pack_low_bytes(ya1.x, ya1.y, yb1.x, yb1.y);
                        w[2][q] = pack_low_bytes(ya2.x, ya2.y, yb2.x, yb2.y);
                        w[3][q] = pack_low_bytes(ya3.x, ya3.y, yb3.x, yb3.y);
                    }
                    __syncwarp();
                    if (lane == 0) mbar_arrive(&bin_empty[si]);
                    if (!mbar_wait_warp(&st_empty[s], ((gs >> 1) & 1) ^ 1, abort_flag, err, 7)) { ok = false; break; }
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
            if (warp >= NEPI) continue;
            epilogue_item(g);
        }
    }

    fence_before();
    __syncthreads();
    if (warp == WARP_MMA) {
        fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS));
    }
}

// ---- 128-wide p3 tiles, both operands from shared memory (the SS MMA form) ----
//
// Four 128-column accumulators fill all 512 TMEM columns, so A cannot be staged in TMEM: the
// MMAs read the D2 digit tiles straight from the TMA ring (64B-swizzled, K-major) and the B
// digits from a 64B-swizzled ring the formers fill.  No movers.  A stage is 64 pixels (one D2
// tile, two 32-pixel K slices): nine digit pairs × 2 slices = 18 MMAs of N = 128, each twice
// the work of an N = 64 MMA for little more time.  The MMAs of a stage retire ~700 cycles
// after they are issued, so the B ring needs three stages; to make room the fp32 inputs come in
// 32-pixel half stages (one 128-row TMA box and the D1 row's 32 pixels each) through a ring of
// three: formers of warps 0-7 take the first half of every stage, warps 8-15 the second.  The
// digit arithmetic, the int32 classes and the epilogue are those of contract_i8_kernel, so
// results are bit-identical to it.
//
// Warp roles (640 threads): warps 0-15 form the B digits and run the epilogue, warp 16 streams
// the fp32 half stages, warp 17 owns TMEM and issues MMAs for accumulators 0 and 2, warp 18
// streams the D2 digit tiles, warp 19 issues MMAs for accumulators 1 and 3.
constexpr int SS_BN = 128;
constexpr int SS_KB = 64;                      // pixels per stage
constexpr int SS_HALF = 32;                    // pixels per fp32 half stage
constexpr int SS_NBI = 3;                      // fp32 half stages in shared memory
constexpr int SS_HALF_BYTES = SS_BN * SS_HALF * 4;  // one 128B-swizzled box of 128 rows
constexpr int SS_NSB = 4;                      // B digit stages: two 128-pixel slots, two stages each
constexpr int SS_NAS = 2;                      // D2 digit tiles
// B digits: 128-byte rows (128B swizzle, the fast layout for the MMA's reads), so a slot holds
// two 64-pixel stages side by side in every row: stage gs fills bytes 64(gs & 1) .. +63 of slot
// (gs / 2) % 2.
constexpr int SS_PLANE = SS_BN * 128;           // one B digit plane of a slot: 128 rows × 128 bytes
constexpr int SS_SLOT = NDB * SS_PLANE;         // 64 KB
constexpr int SS_NWARP_B = 16;
constexpr int SS_WARP_TMA = 16, SS_WARP_MMA = 17, SS_WARP_TMA_A = 18, SS_WARP_MMA2 = 19;
constexpr int SS_NTHREADS = 20 * 32;

// Shared-memory matrix descriptor: K-major, 64-byte swizzle, 8-row atoms of 512 B.
__device__ __forceinline__ uint64_t smem_desc_sw64(uint32_t saddr)
{
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFF);        // start address
    d |= (uint64_t)(1) << 16;                       // leading byte offset (unused for swizzled K-major)
    d |= (uint64_t)((512 >> 4) & 0x3FFF) << 32;    // stride byte offset: 8 rows × 64 B
    d |= (uint64_t)1 << 46;                         // descriptor version (sm_100)
    d |= (uint64_t)4 << 61;                         // SWIZZLE_64B
    return d;
}

// kind::i8 MMA, A and B from shared memory
__device__ __forceinline__ void umma_ss_i8(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                           uint32_t accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
        "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate)
        : "memory");
}

// One issuer's share of a 64-pixel stage: accumulators k = q and q + 2, grouped by accumulator.
// b_stage points at the stage's half of its slot (the start address already advanced by 64 bytes
// for the second half).
__device__ __forceinline__ void issue_stage_ss(uint32_t tmem, uint64_t a_stage, uint64_t b_stage, uint32_t idesc,
                                               int q, bool fresh)
{
    constexpr uint32_t A16 = (uint32_t)A_BOX >> 4, B16 = (uint32_t)SS_PLANE >> 4;
#pragma unroll
    for (int kc = 0; kc < 2; ++kc) {
        const int k = q + 2 * kc;
        const uint32_t acc = tmem + (uint32_t)(k * SS_BN);
        bool first = true;
#pragma unroll
        for (int kk = 0; kk < 2; ++kk)
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                const int j = k - i;
                if (j < 0 || j >= NDB) continue;
                // K slice kk = bytes [32kk, 32kk+32) of the stage's 64 bytes of each row: +2 in 16-byte units
                umma_ss_i8(acc, a_stage + (uint64_t)(i * A16 + kk * 2), b_stage + (uint64_t)(j * B16 + kk * 2), idesc,
                           (first && fresh) ? 0u : 1u);
                first = false;
            }
    }
}

__global__ void __launch_bounds__(SS_NTHREADS, 1)
    contract_i8_ss_kernel(const JobDesc *__restrict__ jobs, const Item *__restrict__ items, int nitems, int *err)
{
    constexpr int BN = SS_BN;
    constexpr int PT = BN * SS_KB / (SS_NWARP_B * 32);  // 16 pixels per former thread per stage
    static_assert(PT == 16, "former pixels per thread");
    static_assert(NACC * BN <= TMEM_COLS, "accumulators must fit in TMEM");
    static_assert(NEPI == SS_NWARP_B, "the formers run the epilogue");
    static_assert(SS_NAS <= SS_NSB, "the D2 ring waits on B-stage releases");

    extern __shared__ __align__(1024) unsigned char smem_raw[];
    unsigned char *smem = (unsigned char *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    unsigned char *bin = smem;                               // SS_NBI × SS_HALF_BYTES
    unsigned char *bdig = bin + SS_NBI * SS_HALF_BYTES;      // 2 × SS_SLOT
    unsigned char *atile = bdig + 2 * SS_SLOT;               // SS_NAS × 3 × A_BOX
    float *d1rows = reinterpret_cast<float *>(atile + SS_NAS * 3 * A_BOX);  // SS_NBI × SS_HALF fp32
    uint64_t *bars = reinterpret_cast<uint64_t *>(d1rows + SS_NBI * SS_HALF);
    uint64_t *as_full = bars, *as_empty = as_full + SS_NAS;
    uint64_t *bin_full = as_empty + SS_NAS, *bin_empty = bin_full + SS_NBI;
    uint64_t *st_full = bin_empty + SS_NBI, *st_empty = st_full + SS_NSB;
    uint64_t *acc_full = st_empty + SS_NSB, *acc_empty = acc_full + 1;
    uint64_t *drain = acc_empty + 1;  // one per issuer
    volatile uint32_t *tmem_slot = reinterpret_cast<volatile uint32_t *>(drain + NISSUE);
    volatile int *abort_flag = reinterpret_cast<volatile int *>(tmem_slot + 1);

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

    if (tid == 0) {
        for (int s = 0; s < SS_NAS; ++s) { mbar_init(&as_full[s], 1); mbar_init(&as_empty[s], NISSUE); }
        // a half stage is read by the 8 former warps of its half
        for (int s = 0; s < SS_NBI; ++s) { mbar_init(&bin_full[s], 1); mbar_init(&bin_empty[s], SS_NWARP_B / 2); }
        for (int s = 0; s < SS_NSB; ++s) { mbar_init(&st_full[s], SS_NWARP_B); mbar_init(&st_empty[s], NISSUE); }
        mbar_init(acc_full, NISSUE);
        mbar_init(acc_empty, NEPI);
        for (int q = 0; q < NISSUE; ++q) mbar_init(&drain[q], 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == SS_WARP_MMA) {
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
    // 64-pixel stages of an item
    auto stages_of = [&](const ItemView &v) {
        const long x_end = min(v.j->k, v.x_begin + v.j->chunk);
        return (int)((x_end - v.x_begin + SS_KB - 1) / SS_KB);
    };

    if (warp == SS_WARP_TMA) {
        // fp32 half stages: D3 rows [bbase, bbase+128) × 32 pixels (128B-swizzled) and the D1 row's
        // 32 pixels; pixels past the end of the map and rows outside [0, nc) come back as zeros
        if (lane == 0) {
            int gh = 0;  // half stages issued so far
            for (int g = blockIdx.x; g < nitems && ok; g += gridDim.x) {
                const ItemView v = decode<BN>(jobs, items, g);
                const int nh = 2 * stages_of(v);
                for (int ih = 0; ih < nh; ++ih, ++gh) {
                    const int s = gh % SS_NBI;
                    if (!mbar_wait(&bin_empty[s], ((gh / SS_NBI) & 1) ^ 1, abort_flag, err, 11)) { ok = false; break; }
                    mbar_expect_tx(&bin_full[s], SS_HALF_BYTES + SS_HALF * 4);
                    const int x = (int)(v.x_begin + (long)ih * SS_HALF);
                    tma_load_2d(bin + s * SS_HALF_BYTES, &v.j->td3, &bin_full[s], x, v.bbase);
                    tma_load_2d(d1rows + s * SS_HALF, &v.j->td1, &bin_full[s], x, v.p1);
                }
            }
            if (!ok)
                for (int q = max(0, gh - SS_NBI); q < gh; ++q)
                    for (long long i = 0; i < WAIT_LIMIT && !mbar_try_wait(&bin_full[q % SS_NBI], ((q / SS_NBI) & 1)); ++i)
                        __nanosleep(100);
        }
    } else if (warp == SS_WARP_TMA_A) {
        // D2 digit planes, rows [rbase, rbase+128) × 64 pixels: one tile per stage; rows outside
        // [0, nc) and pixels past the end of the map come back as zeros
        if (lane == 0) {
            int gs = 0;
            for (int g = blockIdx.x; g < nitems && ok; g += gridDim.x) {
                const ItemView v = decode<BN>(jobs, items, g);
                const int nb = stages_of(v);
                for (int it = 0; it < nb; ++it, ++gs) {
                    const int s = gs % SS_NAS;
                    // the tile slot's previous stage (gs − SS_NAS) has retired when its B stage is released:
                    // one commit per stage serves both rings
                    if (gs >= SS_NAS && !mbar_wait(&st_empty[(gs - SS_NAS) % SS_NSB], ((gs - SS_NAS) / SS_NSB) & 1,
                                                   abort_flag, err, 18)) { ok = false; break; }
                    unsigned char *t = atile + s * 3 * A_BOX;
                    mbar_expect_tx(&as_full[s], 3 * A_BOX);
                    const int x = (int)(v.x_begin + (long)it * SS_KB);
                    tma_load_2d(t, &v.j->ta[0], &as_full[s], x, v.rbase);
                    tma_load_2d(t + A_BOX, &v.j->ta[1], &as_full[s], x, v.rbase);
                    tma_load_2d(t + 2 * A_BOX, &v.j->ta[2], &as_full[s], x, v.rbase);
                }
            }
            if (!ok)
                for (int q = max(0, gs - SS_NAS); q < gs; ++q)
                    for (long long i = 0; i < WAIT_LIMIT && !mbar_try_wait(&as_full[q % SS_NAS], ((q / SS_NAS) & 1)); ++i)
                        __nanosleep(100);
        }
    } else if (warp == SS_WARP_MMA || warp == SS_WARP_MMA2) {
        if (lane == 0) {
            const int q = warp == SS_WARP_MMA ? 0 : 1;
            // S32 accumulate, signed int8 A and B, both K-major, M = 128, N = 128
            const uint32_t idesc = (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) |
                                   ((uint32_t)(BM >> 4) << 24);
            // descriptors are linear in the start address (bits 0-13, 16-byte units)
            const uint64_t adesc0 = smem_desc_sw64(smem_u32(atile));
            const uint64_t bdesc0 = smem_desc_sw128(smem_u32(bdig));
            int gs = 0, seq = 0;
            for (int g = blockIdx.x; g < nitems && ok; g += gridDim.x, ++seq) {
                const int nb = stages_of(decode<BN>(jobs, items, g));
                if (!mbar_wait(acc_empty, (seq & 1) ^ 1, abort_flag, err, 20)) { ok = false; break; }
                for (int it = 0; it < nb; ++it, ++gs) {
                    const int s = gs % SS_NSB, sa = gs % SS_NAS;
                    if (!mbar_wait(&st_full[s], ((gs / SS_NSB) & 1), abort_flag, err, 12)) { ok = false; break; }
                    if (!mbar_wait(&as_full[sa], ((gs / SS_NAS) & 1), abort_flag, err, 19)) { ok = false; break; }
                    fence_after();
                    issue_stage_ss(tmem, adesc0 + (uint64_t)((sa * 3 * A_BOX) >> 4),
                                   bdesc0 + (uint64_t)((((gs >> 1) & 1) * SS_SLOT + (gs & 1) * 64) >> 4), idesc, q,
                                   it == 0);
                    umma_commit(&st_empty[s]);
                }
                if (ok) umma_commit(acc_full);
            }
            if (!ok) {
                umma_commit(&drain[q]);
                for (long long i = 0; i < WAIT_LIMIT && !mbar_try_wait(&drain[q], 0); ++i) __nanosleep(100);
            }
        }
    } else {
        // ---- warps 0-15: B formers, then each item's epilogue ----
        const uint32_t lane_field = (uint32_t)((warp & 3) << 5) << 16;
        // thread (row n, segment sg) forms pixels 16sg .. 16sg+15 of D1[p1]·D3[bbase+n] per stage:
        // segments 0-1 (warps 0-7) read the stage's first fp32 half, segments 2-3 the second
        const int n = tid % BN, sg = tid / BN;
        const int half = sg >> 1;
        const int c0 = (sg & 1) * 4;  // first 16-byte chunk of the thread's 16 pixels in the half's 128-byte row
        // destination: 16-byte chunk 4(gs & 1) + sg of the 128-byte digit row n, at its 128B-swizzled
        // position (the chunk index is XORed with the row's low three bits)
        int gs = 0, seq = 0;
        for (int g = blockIdx.x; g < nitems && ok; g += gridDim.x, ++seq) {
            const ItemView v = decode<BN>(jobs, items, g);
            const JobDesc &j = *v.j;
            const int nb = stages_of(v);
            const int p3 = v.bbase + n;
            const bool col_ok = p3 >= 0 && p3 < j.nc;
            const float scale = col_ok ? ldexpf(127.f, -(v.E1 + j.e3[p3])) : 0.f;
            const float2 sc2 = make_float2(scale, scale);
            for (int it = 0; it < nb; ++it, ++gs) {
                const int gh = 2 * gs + half;  // this thread's half stage
                const int si = gh % SS_NBI, s = gs % SS_NSB;
                if (!mbar_wait_warp(&bin_full[si], ((gh / SS_NBI) & 1), abort_flag, err, 16)) { ok = false; break; }
                const unsigned char *rowp = bin + si * SS_HALF_BYTES + n * 128;
                const float *d1p = d1rows + si * SS_HALF + (sg & 1) * 16;
                uint32_t w[NDB][PT / 4];
#pragma unroll
                for (int qq = 0; qq < PT / 4; ++qq) {
                    const float4 x3 = *reinterpret_cast<const float4 *>(rowp + (((c0 + qq) ^ (n & 7)) << 4));
                    const float4 u = *reinterpret_cast<const float4 *>(d1p + 4 * qq);
                    float2 ya0, ya1, ya2, ya3, yb0, yb1, yb2, yb3;
                    digits254x2(__fmul2_rn(make_float2(u.x, u.y), sc2), make_float2(x3.x, x3.y), ya0, ya1, ya2, ya3);
                    digits254x2(__fmul2_rn(make_float2(u.z, u.w), sc2), make_float2(x3.z, x3.w), yb0, yb1, yb2, yb3);
                    w[0][qq] = pack_low_bytes(ya0.x, ya0.y, yb0.x, yb0.y);
                    w[1][qq] = pack_low_bytes(ya1.x, ya1.y, yb1.x, yb1.y);
                    w[2][qq] = pack_low_bytes(ya2.x, ya2.y, yb2.x, yb2.y);
                    w[3][qq] = pack_low_bytes(ya3.x, ya3.y, yb3.x, yb3.y);
                }
                __syncwarp();
                if (lane == 0) mbar_arrive(&bin_empty[si]);
                if (!mbar_wait_warp(&st_empty[s], ((gs / SS_NSB) & 1) ^ 1, abort_flag, err, 17)) { ok = false; break; }
                unsigned char *dst = bdig + ((gs >> 1) & 1) * SS_SLOT + n * 128 + (((4 * (gs & 1) + sg) ^ (n & 7)) << 4);
#pragma unroll
                for (int d = 0; d < NDB; ++d)
                    *reinterpret_cast<uint4 *>(dst + d * SS_PLANE) = make_uint4(w[d][0], w[d][1], w[d][2], w[d][3]);
                fence_proxy_async_smem();
                __syncwarp();
                if (lane == 0) mbar_arrive(&st_full[s]);
            }
            // ---- epilogue: int32 digit accumulators → FP64 partial tile; warpgroup wg reads BN/4 columns ----
            const int wg = warp >> 2;
            const int me = ((warp & 3) << 5) + lane;
            const bool good = __all_sync(0xffffffffu, ok) && mbar_wait_warp(acc_full, (seq & 1), abort_flag, err, 15);
            if (!good) { ok = false; break; }
            fence_after();
            const int d2 = v.mt * BM + me;
            const int p2 = v.rbase + me;
            const bool row_ok = d2 < j.nclen && p2 >= 0 && p2 < j.nc && j.weight[p2] > 0;
            const int E12 = v.E1 + (row_ok ? j.e2[p2] : 0);
            const double wr = row_ok ? (double)j.weight[v.p1] * (double)j.weight[p2] : 0.0;
            double *dst = nullptr;
            if (d2 < j.nclen)
                dst = j.partial + ((long)v.aidx * j.nchunk + v.chunk) * j.nclen * j.nclen + (long)d2 * j.nclen;
            const int c_begin = wg * (BN / 4), c_end = c_begin + BN / 4;
            const double i254 = 1.0 / 254.0, i254_2 = i254 * i254, i254_3 = i254_2 * i254;
            for (int cb = c_begin; cb < c_end; cb += 8) {
                uint32_t v0[8], v1[8], v2[8], v3[8];
                tmem_ld8(tmem + lane_field + cb, v0);
                tmem_ld8(tmem + lane_field + BN + cb, v1);
                tmem_ld8(tmem + lane_field + 2 * BN + cb, v2);
                tmem_ld8(tmem + lane_field + 3 * BN + cb, v3);
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                if (cb + 8 >= c_end) {
                    // last read of this item: hand the accumulators back to the MMA issuers
                    fence_before();
                    __syncwarp();
                    if (lane == 0) mbar_arrive(acc_empty);
                }
                if (dst) {
#pragma unroll
                    for (int e = 0; e < 8; ++e) {
                        const int nn = cb + e;
                        const int d3 = v.nt * BN + nn;
                        if (d3 >= j.nclen) continue;
                        const int q3 = v.bbase + nn;
                        double val = 0.0;
                        if (wr != 0.0 && q3 >= 0 && q3 < j.nc && j.weight[q3] > 0) {
                            const double sm = (double)(int)v0[e] + (double)(int)v1[e] * i254 +
                                              (double)(int)v2[e] * i254_2 + (double)(int)v3[e] * i254_3;
                            val = ldexp(sm * (1.0 / 16129.0), E12 + j.e3[q3]) * wr * (double)j.weight[q3];
                        }
                        dst[d3] = val;
                    }
                }
            }
        }
    }

    fence_before();
    __syncthreads();
    if (warp == SS_WARP_MMA) {
        fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS));
    }
}

size_t smem_bytes_ss()
{
    return 1024 + (size_t)SS_NBI * SS_HALF_BYTES + 2 * (size_t)SS_SLOT + (size_t)SS_NAS * 3 * A_BOX +
           (size_t)SS_NBI * SS_HALF * 4 + 256;
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

// Pixel chunks per (anchor, tile) pair of one job.  One CTA runs per SM; more chunks give
// more, shorter items (a shorter tail when this job runs alone) but add a fixed cost per
// item (pipeline fill, epilogue) and partial tiles for lag_reduce to read.  Picks the count
// with the least modelled time of the job on its own, so the choice (and with it the FP64
// summation grouping) depends on the job only, never on what else shares the launch.
long choose_chunks(long k, long pairs, int sms, long ncsize, long max_chunk)
{
    const long nch_min = std::max<long>(1, (k + max_chunk - 1) / max_chunk);
    const long nch_max = std::max<long>(nch_min, std::min<long>(4 * nch_min + 16, (k + 1023) / 1024));
    const double stage_s = 0.65e-6;      // one 128-pixel stage of one CTA
    const double fixed_s = 6 * stage_s;  // fill, drain and epilogue of one item
    const double reduce_bw = 5e12;       // bytes/s for lag_reduce reading the partial tiles
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

struct Planned {
    const I8Job *job;
    int bn, mt, nt;
    long nch, chunk;
    size_t partial_bytes;
    bool accumulate;  // a later anchor group of a split job: its lag sum adds to the array
};

int launch_ss(amber_cuda_ctx *c, const JobDesc *d_jobs, const Item *d_items, long nitems, long grid_ctas, int *d_err)
{
    const size_t sm = smem_bytes_ss();
    cudaFuncSetAttribute(contract_i8_ss_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    const unsigned grid = (unsigned)std::min<long>(nitems, grid_ctas);
    contract_i8_ss_kernel<<<grid, SS_NTHREADS, sm, c->stream>>>(d_jobs, d_items, (int)nitems, d_err);
    c->launches += 1;
    c->contractions += 1;
    return cuda_check(c, cudaGetLastError(), "contract_i8_ss_kernel launch");
}

template <int BN>
int launch(amber_cuda_ctx *c, const JobDesc *d_jobs, const Item *d_items, long nitems, long grid_ctas, int *d_err)
{
    const size_t sm = smem_bytes<BN>();
    cudaFuncSetAttribute(contract_i8_kernel<BN>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    const unsigned grid = (unsigned)std::min<long>(nitems, grid_ctas);
    contract_i8_kernel<BN><<<grid, NTHREADS, sm, c->stream>>>(d_jobs, d_items, (int)nitems, d_err);
    c->launches += 1;
    c->contractions += 1;
    return cuda_check(c, cudaGetLastError(), "contract_i8_kernel launch");
}

// Host side of one launch: descriptors and items written into the pinned staging area.
struct LaunchPlan {
    std::vector<Planned> jobs;
    size_t desc_off = 0, item_off = 0;  // byte offsets in the staging area / device job list
    long nitems = 0;
    size_t partial_bytes = 0;
    bool persistent = true;  // false: one CTA per item, dispatched by the hardware as SMs free up
};

int fill_launch(amber_cuda_ctx *c, LaunchPlan &lp, char *stage, bool first_chunk_only)
{
    int rc;
    const int BN = lp.jobs[0].bn;
    JobDesc *desc = (JobDesc *)(stage + lp.desc_off);
    Item *items = (Item *)(stage + lp.item_off);
    size_t poff = 0;
    long ni = 0;
    const CUtensorMapDataType u8 = CU_TENSOR_MAP_DATA_TYPE_UINT8, f32 = CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
    for (size_t i = 0; i < lp.jobs.size(); ++i) {
        const Planned &p = lp.jobs[i];
        const I8Job &jb = *p.job;
        JobDesc &d = desc[i];
        memset(&d, 0, sizeof(d));
        const int8_t *planes[3] = {jb.m2.d0, jb.m2.d1, jb.m2.d2};
        for (int q = 0; q < 3; ++q)
            if ((rc = encode(c, &d.ta[q], u8, planes[q], jb.k, jb.kp, jb.nc, KB_A, BM, CU_TENSOR_MAP_SWIZZLE_64B)))
                return rc;
        if ((rc = encode(c, &d.td3, f32, jb.m3.f32, jb.k, jb.kp * 4, jb.nc, 32, BN, CU_TENSOR_MAP_SWIZZLE_128B)))
            return rc;
        // the D1 row: one box per stage (128 pixels; 32 for the 128-wide tiles' half stages)
        if ((rc = encode(c, &d.td1, f32, jb.m1.f32, jb.k, jb.kp * 4, jb.nc, BN == SS_BN ? SS_HALF : KB_B, 1,
                         CU_TENSOR_MAP_SWIZZLE_NONE)))
            return rc;
        d.e1 = jb.m1.expo; d.e2 = jb.m2.expo; d.e3 = jb.m3.expo;
        d.anchors = jb.anchors;
        d.weight = jb.weight;
        d.partial = (double *)((char *)c->partial.p + poff);
        d.k = jb.k; d.kp = jb.kp; d.chunk = p.chunk;
        d.nc = jb.nc; d.nc10 = jb.nc10; d.nclen = 2 * jb.nc10 + 1;
        d.mt_count = p.mt; d.nt_count = p.nt; d.nchunk = (int)p.nch; d.nanchors = jb.nanchors;
        const long n_local = (long)jb.nanchors * p.mt * p.nt * (first_chunk_only ? 1 : p.nch);
        for (long q = 0; q < n_local; ++q) items[ni++] = Item{(int)i, (int)q};
        poff += p.partial_bytes;
    }
    return AMBER_OK;
}

}  // namespace

size_t contract_partial_cap(const amber_cuda_ctx *c)
{
    return std::max<size_t>((size_t)512 << 20, std::min<size_t>((size_t)8 << 30, c->budget / 8));
}

namespace {

// Plans and enqueues the launches of a list of jobs, job i with p3 tile width bn[i].
int execute_jobs(amber_cuda_ctx *c, const std::vector<const I8Job *> &jobs, const std::vector<int> &bn, int *d_err,
                 bool first_chunk_only = false)
{
    int rc;
    long max_chunk = c->chunk_px > 0 ? std::min<long>(c->chunk_px, 32768) : 32768;
    max_chunk = std::max<long>(KB_B, max_chunk / KB_B * KB_B);
    // Launch plan.  A job with many items runs in a launch of its own with one CTA per
    // item: the hardware hands items to SMs as they free up (even with uneven items) and
    // the resident CTAs stay on one pixel chunk of one job (L2 reuse of the maps).  Small
    // jobs share persistent launches (one CTA per SM looping over the list), so a batch
    // of them fills the GPU without a tail per job.  Partial tiles of one launch stay
    // within a slice of the budget.
    const size_t pcap = contract_partial_cap(c);
    const long big_items = 4L * c->num_sms;
    std::vector<LaunchPlan> plans;
    std::deque<I8Job> parts;  // anchor groups of jobs whose partial tiles exceed the cap
    for (int BN : {32, 64, SS_BN}) {
        LaunchPlan shared;
        for (size_t ji = 0; ji < jobs.size(); ++ji) {
            const I8Job &jb = *jobs[ji];
            const int nclen = 2 * jb.nc10 + 1;
            const long ncsize = (long)nclen * nclen;
            if (bn[ji] != BN) continue;
            if (jb.nanchors == 0) {
                if ((rc = cuda_check(c, cudaMemsetAsync(jb.lag_out, 0, sizeof(double) * ncsize, c->stream), "zero lag")))
                    return rc;
                continue;
            }
            Planned p;
            p.job = &jb;
            p.bn = BN;
            p.mt = (nclen + BM - 1) / BM;
            p.nt = (nclen + BN - 1) / BN;
            // the chunk count (and with it the FP64 summation grouping) must not depend on BN, so
            // that the tile width is numerically neutral: it is planned for 64-wide tiles
            p.nch = choose_chunks(jb.k, (long)jb.nanchors * p.mt * ((nclen + 63) / 64), c->num_sms, ncsize, max_chunk);
            p.chunk = ((jb.k + p.nch - 1) / p.nch + KB_B - 1) / KB_B * KB_B;
            p.nch = (jb.k + p.chunk - 1) / p.chunk;
            p.partial_bytes = (sizeof(double) * (size_t)jb.nanchors * p.nch * ncsize + 255) / 256 * 256;
            p.accumulate = false;
            if (p.partial_bytes > pcap) {
                // split the anchors into groups whose partial tiles fit; each group is a launch of
                // its own and adds its sum to the lag array in group order (deterministic)
                const long ng = (long)((p.partial_bytes + pcap - 1) / pcap);
                const long per = (jb.nanchors + ng - 1) / ng;
                for (long a0 = 0; a0 < jb.nanchors; a0 += per) {
                    parts.push_back(jb);
                    I8Job &sj = parts.back();
                    sj.anchors = jb.anchors + a0;
                    sj.nanchors = (int)std::min<long>(per, jb.nanchors - a0);
                    Planned q = p;
                    q.job = &sj;
                    q.accumulate = a0 > 0;
                    q.partial_bytes = (sizeof(double) * (size_t)sj.nanchors * q.nch * ncsize + 255) / 256 * 256;
                    LaunchPlan lp;
                    lp.persistent = false;
                    lp.jobs.push_back(q);
                    lp.nitems = (long)sj.nanchors * q.mt * q.nt * q.nch;
                    lp.partial_bytes = q.partial_bytes;
                    plans.push_back(lp);
                }
                continue;
            }
            const long ni = (long)jb.nanchors * p.mt * p.nt * p.nch;
            if (ni >= big_items) {
                LaunchPlan lp;
                lp.persistent = false;
                lp.jobs.push_back(p);
                lp.nitems = ni;
                lp.partial_bytes = p.partial_bytes;
                plans.push_back(lp);
                continue;
            }
            if (!shared.jobs.empty() && shared.partial_bytes + p.partial_bytes > pcap) {
                plans.push_back(shared);
                shared = LaunchPlan();
            }
            shared.jobs.push_back(p);
            shared.nitems += ni;
            shared.partial_bytes += p.partial_bytes;
        }
        if (!shared.jobs.empty()) plans.push_back(shared);
    }
    if (plans.empty()) return AMBER_OK;
    // staging: every launch's descriptors and items, uploaded once
    size_t stage_bytes = 0, pmax = 0;
    for (LaunchPlan &lp : plans) {
        lp.desc_off = stage_bytes;
        stage_bytes += sizeof(JobDesc) * lp.jobs.size();
        lp.item_off = stage_bytes;
        stage_bytes = (stage_bytes + sizeof(Item) * lp.nitems + 127) / 128 * 128;
        pmax = std::max(pmax, lp.partial_bytes);
    }
    if ((rc = ensure(c, c->partial, pmax, "partial lag tiles"))) return rc;
    if ((rc = ensure(c, c->jobdesc, stage_bytes, "job list"))) return rc;
    if (c->stage_bytes < stage_bytes) {
        if ((rc = cuda_check(c, cudaStreamSynchronize(c->stream), "job staging"))) return rc;
        if (c->stage) cudaFreeHost(c->stage);
        c->stage = nullptr;
        c->stage_bytes = 0;
        if ((rc = cuda_check(c, cudaHostAlloc(&c->stage, stage_bytes, cudaHostAllocDefault), "job staging"))) return rc;
        c->stage_bytes = stage_bytes;
    }
    // the staging area may still feed the previous run's upload
    if ((rc = cuda_check(c, cudaStreamSynchronize(c->stream), "job staging"))) return rc;
    if (first_chunk_only)
        for (LaunchPlan &lp : plans) {
            lp.nitems = 0;
            for (const Planned &p : lp.jobs) lp.nitems += (long)p.job->nanchors * p.mt * p.nt;
        }
    for (LaunchPlan &lp : plans)
        if ((rc = fill_launch(c, lp, (char *)c->stage, first_chunk_only))) return rc;
    if ((rc = cuda_check(c, cudaMemcpyAsync(c->jobdesc.p, c->stage, stage_bytes, cudaMemcpyHostToDevice, c->stream),
                         "job list upload")))
        return rc;
    for (LaunchPlan &lp : plans) {
        const JobDesc *d_jobs = (const JobDesc *)((char *)c->jobdesc.p + lp.desc_off);
        const Item *d_items = (const Item *)((char *)c->jobdesc.p + lp.item_off);
        phase_begin(c, 1);
        const long grid = lp.persistent ? c->num_sms : lp.nitems;
        const int bw = lp.jobs[0].bn;
        rc = bw == 32   ? launch<32>(c, d_jobs, d_items, lp.nitems, grid, d_err)
             : bw == 64 ? launch<64>(c, d_jobs, d_items, lp.nitems, grid, d_err)
                        : launch_ss(c, d_jobs, d_items, lp.nitems, grid, d_err);
        phase_end(c);
        if (rc) return rc;
        if (first_chunk_only) continue;  // a timing trial: its partial tiles are not reduced
        const JobDesc *h_desc = (const JobDesc *)((char *)c->stage + lp.desc_off);
        for (size_t i = 0; i < lp.jobs.size(); ++i) {
            const I8Job &jb = *lp.jobs[i].job;
            const long ncsize = (long)(2 * jb.nc10 + 1) * (2 * jb.nc10 + 1);
            if ((rc = lag_reduce(c, h_desc[i].partial, (long)jb.nanchors * lp.jobs[i].nch, ncsize, jb.lag_out,
                                 lp.jobs[i].accumulate)))
                return rc;
        }
    }
    return AMBER_OK;
}

// Lag-window class of the autotuner: nclen rounded up to 8.
int tile_class(int nclen) { return (nclen + 7) / 8 * 8; }

// The autotuner's decisions, per (device, class), shared by every context of the process:
// the choice never changes a result, only the time.
std::mutex g_tile_mu;
std::map<std::pair<int, int>, int> g_tile_choice;

}  // namespace

int contract_i8_jobs(amber_cuda_ctx *c, const std::vector<I8Job> &jobs)
{
    int rc;
    if ((rc = ensure(c, c->misc, 256, "error flag"))) return rc;
    int *d_err = (int *)c->misc.p;
    if ((rc = cuda_check(c, cudaMemsetAsync(d_err, 0, sizeof(int), c->stream), "error flag"))) return rc;
    // Tile width: 32 for nclen ≤ 32, 64 above 128; in between both are possible (one 64-wide
    // tile with idle columns, or more 32-wide tiles that each reload the A operand) and the
    // autotuner measures the first job of each lag-window class with both, once per context.
    // The int8 digit products accumulate exactly and the chunking does not depend on the tile
    // width, so the choice does not change any result.
    std::vector<const I8Job *> rest;
    std::vector<int> bn;
    for (const I8Job &jb : jobs) {
        const int nclen = 2 * jb.nc10 + 1;
        int w = nclen <= 32 ? 32 : 64;
        if (c->tile_n == SS_BN) w = SS_BN;
        else if (c->tile_n && nclen <= 128) w = nclen <= 32 ? 32 : c->tile_n;
        if (!c->tile_n && nclen > 32 && nclen <= 128 && jb.nanchors > 0) {
            const int cls = tile_class(nclen);
            int known = 0;
            {
                std::lock_guard<std::mutex> lk(g_tile_mu);
                auto it = g_tile_choice.find({c->device, cls});
                if (it != g_tile_choice.end()) known = it->second;
            }
            if (!known) {
                // trial: the first pixel chunk of the job with both widths, each launch alone
                // and timed; the job itself then runs with the winner below
                const long ncsize = (long)nclen * nclen;
                if ((rc = ensure(c, c->lagtrial, sizeof(double) * ncsize, "tile trial lag array"))) return rc;
                I8Job scratch = jb;
                scratch.lag_out = (double *)c->lagtrial.p;
                // Each width alone, alternating, until both have been timed for at least 1.5 ms
                // (at most 8 rounds), so that launch overhead and noise do not decide; 32 wins
                // only when clearly (5 %) faster, otherwise the 64-wide default stays.
                double tot[2] = {0, 0};
                int reps = 0;
                const int widths[2] = {32, 64};
                while (reps < 8 && (reps < 2 || std::min(tot[0], tot[1]) < 1.5)) {
                    for (int q0 = 0; q0 < 2; ++q0) {
                        const int q = (reps & 1) ? 1 - q0 : q0;
                        float ms = 0;
                        cudaEventRecord(c->tev0, c->stream);
                        if ((rc = execute_jobs(c, {&scratch}, {widths[q]}, d_err, true))) return rc;
                        cudaEventRecord(c->tev1, c->stream);
                        if ((rc = cuda_check(c, cudaEventSynchronize(c->tev1), "tile trial"))) return rc;
                        cudaEventElapsedTime(&ms, c->tev0, c->tev1);
                        tot[q] += ms;
                    }
                    ++reps;
                }
                c->tile_trials.push_back({cls * 100 + 32, (float)(tot[0] / reps)});
                c->tile_trials.push_back({cls * 100 + 64, (float)(tot[1] / reps)});
                known = tot[0] < 0.95 * tot[1] ? 32 : 64;
                std::lock_guard<std::mutex> lk(g_tile_mu);
                g_tile_choice[{c->device, cls}] = known;
            }
            c->tile_tuned[cls] = known;
            w = known;
        }
        rest.push_back(&jb);
        bn.push_back(w);
    }
    if (!rest.empty() && (rc = execute_jobs(c, rest, bn, d_err))) return rc;
    int herr = 0;
    if ((rc = cuda_check(c, cudaMemcpyAsync(&herr, d_err, sizeof(int), cudaMemcpyDeviceToHost, c->stream),
                         "error flag read")))
        return rc;
    if ((rc = cuda_check(c, cudaStreamSynchronize(c->stream), "contract_i8"))) return rc;
    if (herr) return fail(c, AMBER_ERR_TIMEOUT, "int8 tensor-core contraction: a pipeline wait gave up (site %d)", herr);
    return AMBER_OK;
}

int contract_i8(amber_cuda_ctx *c, const DigitMaps &m1, const DigitMaps &m2, const DigitMaps &m3, long k, long kp,
                double *lag_out)
{
    std::vector<I8Job> jobs(1);
    I8Job &jb = jobs[0];
    jb.m1 = m1; jb.m2 = m2; jb.m3 = m3;
    jb.k = k; jb.kp = kp;
    jb.nc = (int)c->nc; jb.nc10 = c->nc10;
    jb.anchors = (const int *)c->d_anchors.p;
    jb.weight = (const int *)c->d_weight.p;
    jb.nanchors = (int)c->anchors.size();
    jb.lag_out = lag_out;
    return contract_i8_jobs(c, jobs);
}

}  // namespace amber
