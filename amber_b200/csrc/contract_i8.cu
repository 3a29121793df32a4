// Mixed-precision triple-product lag accumulation on the int8 tensor cores: the
// lag-space GEMM of lagspace.cuh run as tcgen05 kind::i8 MMAs with exact int32
// accumulation in TMEM, FP64 recombination per pixel block and the compensated
// FP64 reduction of ls_reduce.  Replaces the float loop of 4_fbe/amber.c:247-279
// / amber_v2.c:243-283.
//
// Why not FP32 accumulation: on the B200 tensor cores a long FP32 accumulation
// chain of coherent (same-sign) products loses ~2^-24 of the running sum per
// step, which breaks the 1e-6-of-Σ|products| bound on the v2 sampling-mask
// sums; integer accumulation has no rounding at all.
//
// Representation.  Every block of 256 pixels of every ring map has one exponent
// E (maps.cu), shared by all channels.  Within block b the D2 operand is three
// base-254 digits of t = w·D2·127·2^−E2 (quantize_kernel), and the per-anchor
// product w·D1[p1]·w·D3[p3] is formed in FP32 on the CUDA cores (packed FP32x2),
// scaled by 127·2^−(E1+E3) and cut into three digits (the D maps) or four (the
// sampling-mask maps).  With Q_i the D2 digits and P_j the product digits:
//     Σ_x (w1D1)(w2D2)(w3D3) = 2^(E1+E2+E3)/127² · Σ_k 254^−k Σ_{i+j=k} Σ_x Q_i P_j.
// Class k accumulates in its own int32 TMEM accumulator.  Classes 0-2 (six
// MMAs per 32 pixels) bound the D-map error near 1e-7 of Σ|products|; the
// peaked sampling-mask maps also need class 3 (P3·Q0 + P2·Q1 + P1·Q2): the
// three accumulators of classes 0-2 at N = 128 plus the A staging fill TMEM,
// so a mask block runs a second sweep that forms digits 1-3 of the product
// and accumulates class 3 alone.  The numbers behind this choice: a numpy
// emulation of these exact digit operations on the single-realisation
// workload's Ng1 = 354 and 740 maps gave 6–9e-8 (D, classes 0-2) and
// 4.5e-8 (mask, classes 0-3), against 5–8e-7 for the mask maps without class 3.
// A per-block exponent is what lets all anchors share one accumulator: the
// scale of a product no longer depends on its channels.  |class sum| ≤
// 3·127² per pixel and anchor, and a block holds at most 128 anchor groups of
// 256 pixels (32768 terms): the int32 accumulators cannot overflow.
//
// Operands.  A (TMEM, M = 128 rows Δ3, written by the formers with tcgen05.st)
// = the per-anchor product digits; B (shared memory, N ≤ 128 rows Δ2) = the D2
// digits of the anchor's window, read straight from the staged channel rows at
// the window's offset: TMA writes the D2 digits as [digit][16-pixel group]
// [channel][16 bytes], the K-major no-swizzle layout of 8-row core matrices,
// whose rows may start at any channel.  Per 32-pixel slice a unit stages, once,
// the fp32 D3 rows of its span (128B-swizzled, conflict-free row reads), the
// fp32 D1 rows of its anchor block and the D2 digits of its window span, and
// then runs every anchor group of the block against them.
//
// Warp roles (576 threads): warps 0-15 form the A digits (warp w: TMEM lanes
// 32·(w mod 4) .. +31, pixels 8·(w div 4) .. +7 of the slice) and run each
// block's epilogue; warp 16 streams the slices by TMA; warp 17 owns TMEM and
// issues the MMAs from one lane.  Four A buffers let the formers run ahead of
// the tensor pipe.  Every mbarrier wait is bounded; on expiry the CTA raises an
// error flag the host turns into AMBER_ERR_TIMEOUT, drains its own copies and
// MMAs and frees TMEM.  No cluster launch and no multicast.
#include <string.h>

#include <algorithm>
#include <cmath>
#include <type_traits>
#include <vector>

#include "lagspace.cuh"
#include "tc_ptx.cuh"

namespace amber {

namespace {

using namespace tc;

constexpr int SLICE = 32;                    // pixels per K step (one kind::i8 MMA)
constexpr int NSLICE = LS_BLOCK / SLICE;     // slices per block
constexpr int NFORM = 16;                    // former / epilogue warps
constexpr int WARP_TMA = 16, WARP_MMA = 17;
constexpr int NTHREADS = 18 * 32;
constexpr int TMEM_COLS = 512;
constexpr int ACC_STRIDE = 128;              // TMEM columns per class accumulator
constexpr int NABUF = 5;                     // A buffers
constexpr int NSET = 4;                      // former sets: each anchor group is formed by one set of 4 warps
constexpr int ABUF_COLS = 24;                // 3 digits × 8 columns (32 int8 per row per digit)
constexpr int A_COL0 = 3 * ACC_STRIDE;       // first A buffer column
static_assert(A_COL0 + NABUF * ABUF_COLS <= TMEM_COLS, "TMEM");

// One stage (one 32-pixel slice) in shared memory, at fixed offsets sized for the largest boxes:
constexpr int ST_D3 = 0;                     // fp32 D3 rows, 128 B each, 128B swizzle (≤ LS_SPAN rows)
constexpr int ST_D1 = LS_SPAN * 128;         // fp32 D1 rows of the anchor block, 128 B each
constexpr int ST_D2 = ST_D1 + LS_SPAN * 128; // D2 digits [3][2][span2][16]
constexpr int ST_BYTES = ST_D2 + 3 * 2 * LS_SPAN * 16;
constexpr int NSTAGE = 2;
static_assert(ST_BYTES % 1024 == 0, "stages keep the 1024-byte alignment of the 128B swizzle");

struct alignas(64) I8Desc {
    CUtensorMap t3;  // w·D3 fp32 {k, nc}, box {32, span3}, 128B swizzle
    CUtensorMap t1;  // w·D1 fp32 {k, nc}, box {32, AB}
    CUtensorMap t2;  // D2 digits {16, nc, kp/16, 3}, box {16, span2, 2, 3}
    const int *e1, *e2, *e3;        // block exponents
    const int *groups, *group_off;  // anchor groups of every anchor block
    long k;
    int nc, nc10, nclen, ks, AB, T;
    int span3, span2;
    int sweeps;                     // 1: classes 0-2; 2: also class 3 (mask maps)
    uint32_t tx_bytes;              // bytes one slice's three TMA boxes deliver
};

// Three or four base-254 digits of two products u·v at once (packed FP32x2):
// every step is one fused op on a pair, the product enters the first rounding
// unrounded (y0 = fma(u, v, M)), and round-to-nearest through the 1.5·2^23
// magic number leaves each digit's two's-complement byte in the low mantissa
// bits.  M − y = −digit exactly, and each residual 254·s − d is exact in FP32
// (its lowest bit is at most 2^−22 and it is at most 1/2 in magnitude).
template <int ND>
__device__ __forceinline__ void digits254x2(float2 u, float2 v, float2 (&y)[4])
{
    const float2 M = make_float2(12582912.0f, 12582912.0f);
    const float2 K254 = make_float2(254.f, 254.f);
    const float2 NEG1 = make_float2(-1.f, -1.f);
    y[0] = __ffma2_rn(u, v, M);                    // M + d0
    const float2 nq0 = __ffma2_rn(y[0], NEG1, M);  // −d0
    const float2 r0 = __ffma2_rn(u, v, nq0);       // u·v − d0
    y[1] = __ffma2_rn(r0, K254, M);                // M + d1
    const float2 nq1 = __ffma2_rn(y[1], NEG1, M);  // −d1
    const float2 s1 = __ffma2_rn(r0, K254, nq1);   // 254·r0 − d1
    y[2] = __ffma2_rn(s1, K254, M);                // M + d2
    if constexpr (ND == 4) {
        const float2 nq2 = __ffma2_rn(y[2], NEG1, M);  // −d2
        const float2 s2 = __ffma2_rn(s1, K254, nq2);   // 254·s1 − d2
        y[3] = __ffma2_rn(s2, K254, M);                // M + d3
    }
}

__device__ __forceinline__ uint32_t pack_low_bytes(float a, float b, float c, float d)
{
    return __byte_perm(__byte_perm(__float_as_uint(a), __float_as_uint(b), 0x0040),
                       __byte_perm(__float_as_uint(c), __float_as_uint(d), 0x0040), 0x5410);
}

__device__ __forceinline__ void tmem_st4(uint32_t taddr, const uint32_t (&v)[4])
{
    asm volatile("tcgen05.st.sync.aligned.32x32b.x4.b32 [%0], {%1, %2, %3, %4};" ::"r"(taddr), "r"(v[0]), "r"(v[1]),
                 "r"(v[2]), "r"(v[3])
                 : "memory");
}

__device__ __forceinline__ void tmem_ld8(uint32_t taddr, uint32_t (&v)[8])
{
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7])
                 : "r"(taddr)
                 : "memory");
}

__device__ __forceinline__ void tma_load_4d(void *dst, const CUtensorMap *map, uint64_t *bar, int x, int y, int z,
                                            int w)
{
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cta.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
        "[%6];" ::"r"(smem_u32(dst)),
        "l"(map), "r"(x), "r"(y), "r"(z), "r"(w), "r"(smem_u32(bar))
        : "memory");
}

// kind::i8 MMA, A from TMEM, issued by the lane elect.sync picks from the converged MMA warp (every
// operand is warp-uniform, so the issue costs one instruction), with the accumulate operand as an
// immediate: the first MMA into an accumulator overwrites it, the rest add.
__device__ __forceinline__ void umma_i8_set(uint32_t d_tmem, uint32_t a_tmem, uint64_t b_desc, uint32_t idesc)
{
    asm volatile("{\n\t.reg .pred e;\n\telect.sync _|e, 0xffffffff;\n\t"
                 "@e tcgen05.mma.cta_group::1.kind::i8 [%0], [%1], %2, %3, 0;\n\t}" ::"r"(d_tmem), "r"(a_tmem),
                 "l"(b_desc), "r"(idesc)
                 : "memory");
}
__device__ __forceinline__ void umma_i8_add(uint32_t d_tmem, uint32_t a_tmem, uint64_t b_desc, uint32_t idesc)
{
    asm volatile("{\n\t.reg .pred e;\n\telect.sync _|e, 0xffffffff;\n\t"
                 "@e tcgen05.mma.cta_group::1.kind::i8 [%0], [%1], %2, %3, 1;\n\t}" ::"r"(d_tmem), "r"(a_tmem),
                 "l"(b_desc), "r"(idesc)
                 : "memory");
}
// tcgen05.commit from the elected lane of the converged warp
__device__ __forceinline__ void umma_commit_elect(uint64_t *bar)
{
    asm volatile("{\n\t.reg .pred e;\n\telect.sync _|e, 0xffffffff;\n\t"
                 "@e tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n\t}" ::"r"(
                     smem_u32(bar))
                 : "memory");
}

// Shared-memory descriptor of a K-major operand without swizzle: 8-row core matrices of
// 16-byte rows stacked every 128 bytes (SBO), the second 16-byte K chunk `lbo` bytes on.
__device__ __forceinline__ uint64_t smem_desc_plain(uint32_t saddr, uint32_t lbo)
{
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFF);      // start address
    d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;  // leading byte offset: K-adjacent core matrices
    d |= (uint64_t)((128 >> 4) & 0x3FFF) << 32;  // stride byte offset: the next 8 rows
    d |= (uint64_t)1 << 46;                      // descriptor version (sm_100)
    return d;                                    // swizzle mode 0: none
}

__global__ void __launch_bounds__(NTHREADS, 1)
    ls_i8_kernel(const I8Desc *__restrict__ jobs, const LsUnit *__restrict__ units, double *__restrict__ partial,
                 int *err)
{
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    unsigned char *smem = (unsigned char *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem + NSTAGE * ST_BYTES);
    uint64_t *st_full = bars, *st_empty = st_full + NSTAGE;
    uint64_t *ab_full = st_empty + NSTAGE, *ab_empty = ab_full + NABUF;
    uint64_t *acc_full = ab_empty + NABUF, *acc_empty = acc_full + 1, *drain = acc_empty + 1;
    volatile uint32_t *tmem_slot = reinterpret_cast<volatile uint32_t *>(drain + 1);
    volatile int *abort_flag = reinterpret_cast<volatile int *>(tmem_slot + 1);
    int *sgroups = reinterpret_cast<int *>(smem + NSTAGE * ST_BYTES + 256);  // this anchor block's groups
    unsigned char *zero_row = smem + NSTAGE * ST_BYTES + 256 + sizeof(int) * LS_SPAN;  // 128 zero bytes

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const LsUnit u = units[blockIdx.x];
    const I8Desc *jd = jobs + u.job;
    const int g0 = jd->group_off[u.ab], g1 = jd->group_off[u.ab + 1];
    const int ks = jd->ks, nclen = jd->nclen, nc = jd->nc;
    const int c0 = u.ab * jd->AB, c1 = min(nc, c0 + jd->AB);
    const int mrows = ks > 1 ? ks * nclen : min(LS_ROWS, nclen - LS_ROWS * u.t3);
    const int ncols = ks > 1 ? nclen : min(LS_ROWS, nclen - LS_ROWS * u.t2);  // lag columns
    const int nmma = ks > 1 ? ((nclen + ks - 1 + 15) / 16) * 16 : ((ncols + 15) / 16) * 16;  // MMA N
    double *out = partial + u.tile * (long)(LS_ROWS * LS_ROWS);

    if (g1 == g0) {
        // an anchor block without anchors contributes nothing: its partial tile is zero
        for (int e = tid; e < LS_ROWS * LS_ROWS; e += NTHREADS) out[e] = 0.0;
        return;
    }

    for (int i = tid; i < g1 - g0; i += NTHREADS) sgroups[i] = jd->groups[g0 + i];
    if (tid < 32) reinterpret_cast<uint32_t *>(zero_row)[tid] = 0u;
    if (tid == 0) {
        for (int s = 0; s < NSTAGE; ++s) { mbar_init(&st_full[s], 1); mbar_init(&st_empty[s], NFORM + 1); }
        for (int s = 0; s < NABUF; ++s) { mbar_init(&ab_full[s], NFORM / NSET); mbar_init(&ab_empty[s], 1); }
        mbar_init(acc_full, 1);
        mbar_init(acc_empty, NFORM);
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
    bool ok = true;
    const int sweeps = jd->sweeps;
    const long k = jd->k;
    auto nslices = [&](long b) {
        const long n = (k - b * LS_BLOCK + SLICE - 1) / SLICE;
        return (int)(n < NSLICE ? n : NSLICE);
    };

    if (warp == WARP_TMA) {
        if (lane == 0) {
            const int row0_3 = c0 - jd->nc10 + (ks > 1 ? 0 : LS_ROWS * u.t3);
            const int row0_2 = c0 - jd->nc10 + (ks > 1 ? 0 : LS_ROWS * u.t2);
            int ns = 0;
            for (long b = u.b0; b < u.b1 && ok; ++b)
                for (int sw = 0; sw < sweeps && ok; ++sw)
                    for (int sl = 0; sl < nslices(b); ++sl, ++ns) {
                        const int s = ns % NSTAGE;
                        if (!mbar_wait(&st_empty[s], ((ns / NSTAGE) & 1) ^ 1, abort_flag, err, 31)) { ok = false; break; }
                        unsigned char *st = smem + s * ST_BYTES;
                        mbar_expect_tx(&st_full[s], jd->tx_bytes);
                        const int x = (int)(b * LS_BLOCK + sl * SLICE);
                        tma_load_2d(st + ST_D3, &jd->t3, &st_full[s], x, row0_3);
                        tma_load_2d(st + ST_D1, &jd->t1, &st_full[s], x, c0);
                        tma_load_4d(st + ST_D2, &jd->t2, &st_full[s], 0, row0_2, x / 16, 0);
                    }
            if (!ok)
                for (int q = max(0, ns - NSTAGE); q < ns; ++q)
                    for (long long i = 0; i < WAIT_LIMIT && !mbar_try_wait(&st_full[q % NSTAGE], ((q / NSTAGE) & 1)); ++i)
                        __nanosleep(100);
        }
    } else if (warp == WARP_MMA) {
        // The whole warp runs the issue loop and polls the barriers together; one elected lane
        // issues.  The tensor pipe queues only about two MMAs, so the loop is kept to a few
        // instructions per MMA: the B descriptors move with the start address alone (bits 0-13,
        // 16-byte units, no carry out for shared-memory addresses), the first anchor group of a
        // sweep is peeled so that the accumulate flag is an immediate.
        // S32 accumulate, signed int8 A and B, both K-major, M = 128, N = nmma
        const uint32_t idesc = (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(nmma >> 3) << 17) |
                               ((uint32_t)(LS_ROWS >> 4) << 24);
        const uint32_t lbo = (uint32_t)jd->span2 * 16;          // the second 16-pixel group of a digit
        const uint64_t ddig = (uint64_t)((2 * lbo) >> 4);        // the next digit plane
        const uint64_t desc0 = smem_desc_plain(smem_u32(smem + ST_D2), lbo) - (uint64_t)c0;  // row c0 at offset 0
        const uint32_t accA = tmem, accB = tmem + ACC_STRIDE, accC = tmem + 2 * ACC_STRIDE;
        const int ngr = g1 - g0;
        int ns = 0, na = 0, ni = 0;
        for (long b = u.b0; b < u.b1 && ok; ++b)
            for (int sw = 0; sw < sweeps && ok; ++sw, ++ni) {
                // the epilogue of the previous item has read the accumulators out
                if (!mbar_wait_conv(acc_empty, (ni & 1) ^ 1, abort_flag, err, 32)) { ok = false; break; }
                for (int sl = 0; sl < nslices(b) && ok; ++sl, ++ns) {
                    const int s = ns % NSTAGE;
                    if (!mbar_wait_conv(&st_full[s], (ns / NSTAGE) & 1, abort_flag, err, 33)) { ok = false; break; }
                    const uint64_t sdesc = desc0 + (uint64_t)((s * ST_BYTES) >> 4);
                    for (int g = 0; g < ngr; ++g, ++na) {
                        const int ab = na % NABUF;
                        if (!mbar_wait_conv(&ab_full[ab], (na / NABUF) & 1, abort_flag, err, 34)) { ok = false; break; }
                        fence_after();
                        const uint64_t q0 = sdesc + (uint64_t)sgroups[g], q1 = q0 + ddig, q2 = q1 + ddig;
                        const uint32_t a0 = tmem + A_COL0 + ab * ABUF_COLS;
                        if (sw == 0) {
                            // class k = Σ_{i+j=k} Q_i·P_j into accumulator k
                            if (sl == 0 && g == 0) {
                                umma_i8_set(accA, a0, q0, idesc);
                                umma_i8_set(accB, a0 + 8, q0, idesc);
                                umma_i8_set(accC, a0 + 16, q0, idesc);
                            } else {
                                umma_i8_add(accA, a0, q0, idesc);
                                umma_i8_add(accB, a0 + 8, q0, idesc);
                                umma_i8_add(accC, a0 + 16, q0, idesc);
                            }
                            umma_i8_add(accB, a0, q1, idesc);
                            umma_i8_add(accC, a0 + 8, q1, idesc);
                            umma_i8_add(accC, a0, q2, idesc);
                        } else {
                            // class 3: P3·Q0 + P2·Q1 + P1·Q2; the A buffer holds P1, P2, P3
                            if (sl == 0 && g == 0) umma_i8_set(accA, a0 + 16, q0, idesc);
                            else umma_i8_add(accA, a0 + 16, q0, idesc);
                            umma_i8_add(accA, a0 + 8, q1, idesc);
                            umma_i8_add(accA, a0, q2, idesc);
                        }
                        umma_commit_elect(&ab_empty[ab]);
                    }
                    if (ok) umma_commit_elect(&st_empty[s]);
                }
                if (ok) umma_commit_elect(acc_full);
            }
        if (!ok) {
            umma_commit_elect(drain);
            if (lane == 0)
                for (long long i = 0; i < WAIT_LIMIT && !mbar_try_wait(drain, 0); ++i) __nanosleep(100);
            __syncwarp();
        }
    } else {
        // ---- warps 0-15: form the A digits, then each block's epilogue ----
        const int q = warp & 3, ps = warp >> 2;
        const int r = 32 * q + lane;                      // TMEM lane = accumulator row
        const int a = ks > 1 ? r / nclen : 0;             // anchor slot of the row
        const int d3 = ks > 1 ? r % nclen : r;            // lag Δ3 within the tile
        const bool row_ok = r < mrows;
        const uint32_t lane_field = (uint32_t)(32 * q) << 16;
        const int ngr = g1 - g0, nab1 = c1 - c0;
        const int row0_3 = c0 - jd->nc10 + (ks > 1 ? 0 : LS_ROWS * u.t3);  // channel of staged D3 row 0
        int ns = 0, na = 0, ni = 0;
        // The 16 formers are four sets of four: set ps forms anchor groups ps, ps + 4, … of each
        // slice, and within a set warp q fills TMEM lanes 32q .. 32q+31 of the group's A buffer
        // with all 32 pixels (four 8-pixel chunks, one tcgen05.st.x8 per digit plane), so the
        // per-group work (addresses, barrier wait, TMEM hand-off) is spread over 32 pixels.  A
        // lane whose row has no data (past the tile or past the anchor block) reads a zeroed row,
        // so its digits come out zero with no per-digit select; D3 channels outside [0, nc) arrive
        // as zero rows from the TMA bounds fill, and a warp whose rows all lie there stores zero
        // digits without the arithmetic.
        auto form_slice = [&](auto ndc, const unsigned char *st) {
            constexpr int ND = decltype(ndc)::value;
            constexpr int D0 = ND - 3;  // sweep 2 stores product digits 1-3
            for (int g = ps; g < ngr && ok; g += NSET) {
                const int n = na + g;  // the group's place in the MMA warp's order
                if (!mbar_wait_warp(&ab_empty[n % NABUF], ((n / NABUF) & 1) ^ 1, abort_flag, err, 36)) {
                    ok = false;
                    break;
                }
                const int p1 = sgroups[g] + a;
                const int rho = p1 - c0 + d3;  // staged D3 row of this lane
                const bool valid = row_ok && p1 < c1;
                const int p3 = row0_3 + rho;  // D3 channel of this lane's row
                // two halves of 16 pixels: 12 digit words stay live until their tcgen05.wait::st
                // (the 18 warps leave ~96 registers a thread)
                const bool live = __any_sync(0xffffffffu, valid && p3 >= 0 && p3 < nc);
                const unsigned char *row3 = valid ? st + ST_D3 + rho * 128 : zero_row;
                // the D1 row, already scaled by 127·2^−(E1+E3) for this block
                const float4 *row1 = reinterpret_cast<const float4 *>(st + ST_D1 + min(p1 - c0, nab1 - 1) * 128);
                const uint32_t col = tmem + lane_field + A_COL0 + (n % NABUF) * ABUF_COLS;
#pragma unroll
                for (int half = 0; half < 2; ++half) {
                    uint32_t w[3][4];
                    if (live) {
#pragma unroll
                        for (int cc = 0; cc < 2; ++cc) {
                            const int c = 2 * half + cc;
                            const float4 x0 = *reinterpret_cast<const float4 *>(row3 + (((2 * c) ^ (rho & 7)) << 4));
                            const float4 x1 =
                                *reinterpret_cast<const float4 *>(row3 + (((2 * c + 1) ^ (rho & 7)) << 4));
                            const float4 u0 = row1[2 * c], u1 = row1[2 * c + 1];
                            {  // pixels 0-3 of the chunk -> word 2cc of each digit plane
                                float2 ya[4], yb[4];
                                digits254x2<ND>(make_float2(u0.x, u0.y), make_float2(x0.x, x0.y), ya);
                                digits254x2<ND>(make_float2(u0.z, u0.w), make_float2(x0.z, x0.w), yb);
#pragma unroll
                                for (int dd = 0; dd < 3; ++dd)
                                    w[dd][2 * cc] =
                                        pack_low_bytes(ya[dd + D0].x, ya[dd + D0].y, yb[dd + D0].x, yb[dd + D0].y);
                            }
                            {  // pixels 4-7 -> word 2cc + 1
                                float2 yc[4], yd[4];
                                digits254x2<ND>(make_float2(u1.x, u1.y), make_float2(x1.x, x1.y), yc);
                                digits254x2<ND>(make_float2(u1.z, u1.w), make_float2(x1.z, x1.w), yd);
#pragma unroll
                                for (int dd = 0; dd < 3; ++dd)
                                    w[dd][2 * cc + 1] =
                                        pack_low_bytes(yc[dd + D0].x, yc[dd + D0].y, yd[dd + D0].x, yd[dd + D0].y);
                            }
                        }
                    } else {
#pragma unroll
                        for (int dd = 0; dd < 3; ++dd)
#pragma unroll
                            for (int e = 0; e < 4; ++e) w[dd][e] = 0u;
                    }
                    // pixels 16·half .. +15 = columns 4·half .. +3 of each digit plane
#pragma unroll
                    for (int dd = 0; dd < 3; ++dd) tmem_st4(col + 8 * dd + 4 * half, w[dd]);
                    // tcgen05.st reads its source registers asynchronously: wait before they change
                    asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
                }
                fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive(&ab_full[n % NABUF]);
            }
            na += ngr;
        };
        for (long b = u.b0; b < u.b1 && ok; ++b) {
            const int E13 = jd->e1[b] + jd->e3[b];
            const float sc = ldexpf(127.f, -E13);
            for (int sw = 0; sw < sweeps && ok; ++sw, ++ni) {
                for (int sl = 0; sl < nslices(b) && ok; ++sl, ++ns) {
                    const int s = ns % NSTAGE;
                    if (!mbar_wait_warp(&st_full[s], (ns / NSTAGE) & 1, abort_flag, err, 35)) { ok = false; break; }
                    unsigned char *st = smem + s * ST_BYTES;
                    // scale the staged D1 rows once for every row that uses them (the formers alone read them)
                    float *d1 = reinterpret_cast<float *>(st + ST_D1);
                    for (int e = tid; e < nab1 * SLICE; e += NFORM * 32) d1[e] *= sc;
                    asm volatile("bar.sync 1, %0;" ::"n"(NFORM * 32) : "memory");
                    if (sw == 0) form_slice(std::integral_constant<int, 3>(), st);
                    else form_slice(std::integral_constant<int, 4>(), st);
                    __syncwarp();
                    if (ok && lane == 0) mbar_arrive(&st_empty[s]);
                }
                if (!ok) break;
                // ---- epilogue: int32 class accumulators → FP64, added into the unit's partial tile ----
                if (!mbar_wait_warp(acc_full, ni & 1, abort_flag, err, 37)) { ok = false; break; }
                fence_after();
                const int E = E13 + jd->e2[b];
                const double scale = sw == 0 ? ldexp(1.0, E) * (1.0 / (16129.0 * 64516.0))
                                             : ldexp(1.0, E) * (1.0 / (16129.0 * 16387064.0));
                const bool first = b == u.b0 && sw == 0;
                for (int cb = 8 * ps; cb < nmma; cb += 32) {
                    uint32_t v0[8], v1[8], v2[8];
                    tmem_ld8(tmem + lane_field + cb, v0);
                    if (sw == 0) {
                        tmem_ld8(tmem + lane_field + ACC_STRIDE + cb, v1);
                        tmem_ld8(tmem + lane_field + 2 * ACC_STRIDE + cb, v2);
                    }
                    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                    if (!row_ok) continue;
#pragma unroll
                    for (int e = 0; e < 8; ++e) {
                        const int colx = cb + e - a;  // slot a of a packed tile: lag column = column − a
                        if (colx < 0 || colx >= ncols) continue;
                        const long long V = sw == 0 ? (long long)(int)v0[e] * 64516LL + (long long)(int)v1[e] * 254LL +
                                                          (long long)(int)v2[e]
                                                    : (long long)(int)v0[e];
                        double *o = out + (long)colx * LS_ROWS + r;
                        const double val = (double)V * scale;
                        *o = first ? val : *o + val;
                    }
                }
                fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive(acc_empty);
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

constexpr size_t SMEM_BYTES = 1024 + (size_t)NSTAGE * ST_BYTES + 256 + sizeof(int) * LS_SPAN + 128;

typedef CUresult (*EncodeTiled)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

int encode(amber_cuda_ctx *c, CUtensorMap *m, CUtensorMapDataType dt, int rank, const void *base,
           const cuuint64_t *dims, const cuuint64_t *strides, const cuuint32_t *box, CUtensorMapSwizzle sw)
{
    static EncodeTiled enc = nullptr;
    if (!enc) {
        void *fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess || !fn)
            return fail(c, AMBER_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
        enc = (EncodeTiled)fn;
    }
    cuuint32_t estr[4] = {1, 1, 1, 1};
    CUresult r = enc(m, dt, (cuuint32_t)rank, (void *)base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, sw,
                     CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(c, AMBER_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
    return AMBER_OK;
}

}  // namespace

size_t contract_partial_cap(const amber_cuda_ctx *c)
{
    return std::max<size_t>((size_t)512 << 20, std::min<size_t>((size_t)8 << 30, c->budget / 8));
}

int contract_i8_jobs(amber_cuda_ctx *c, const std::vector<I8Job> &jobs)
{
    int rc;
    if (jobs.empty()) return AMBER_OK;
    if ((rc = ensure(c, c->misc, 256, "error flag"))) return rc;
    int *d_err = (int *)c->misc.p;
    if ((rc = cuda_check(c, cudaMemsetAsync(d_err, 0, sizeof(int), c->stream), "error flag"))) return rc;
    constexpr size_t TILE_B = sizeof(double) * LS_ROWS * LS_ROWS;
    const size_t pcap = contract_partial_cap(c);
    const CUtensorMapDataType u8 = CU_TENSOR_MAP_DATA_TYPE_UINT8, f32 = CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
    cudaFuncSetAttribute(ls_i8_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_BYTES);
    size_t j0 = 0;
    while (j0 < jobs.size()) {
        // plan as many jobs as their partial tiles allow in one launch
        std::vector<LsJobPlan> plans;
        long tiles = 0;
        size_t j1 = j0;
        for (; j1 < jobs.size(); ++j1) {
            const I8Job &jb = jobs[j1];
            LsJobPlan p;
            ls_plan_job(p, jb.nc, jb.nc10, jb.k, *jb.weight, c->num_sms, 8, ls_force_bpu(c->chunk_px));
            if (j1 > j0 && (size_t)(tiles + p.s.units()) * TILE_B > pcap) break;
            p.unit_base = tiles;
            tiles += p.s.units();
            plans.push_back(std::move(p));
        }
        std::vector<LsUnit> units;
        for (size_t i = 0; i < plans.size(); ++i) {
            const size_t first = units.size();
            ls_units(plans[i], (int)i, units);
            if (jobs[j0 + i].mask_pass)
                for (size_t q = first; q < units.size(); ++q) units[q].work *= 1.6;  // the class-3 sweep
        }
        // largest units first, so that the small ones fill the tail of the launch
        std::stable_sort(units.begin(), units.end(), [](const LsUnit &a, const LsUnit &b) { return a.work > b.work; });
        size_t ngroups = 0, noff = 0;
        for (const LsJobPlan &p : plans) {
            ngroups += p.groups.size();
            noff += p.group_off.size();
        }
        const size_t desc_b = sizeof(I8Desc) * plans.size(), unit_b = sizeof(LsUnit) * units.size();
        const size_t off_u = (desc_b + 255) / 256 * 256, off_g = off_u + (unit_b + 255) / 256 * 256;
        const size_t off_o = off_g + (sizeof(int) * ngroups + 255) / 256 * 256;
        const size_t stage_b = off_o + sizeof(int) * noff;
        if ((rc = ensure(c, c->partial, (size_t)tiles * TILE_B, "partial lag tiles"))) return rc;
        if ((rc = ensure(c, c->jobdesc, stage_b, "job list"))) return rc;
        // the staging area may still feed the previous launch's upload
        if ((rc = cuda_check(c, cudaStreamSynchronize(c->stream), "job staging"))) return rc;
        if (c->stage_bytes < stage_b) {
            if (c->stage) cudaFreeHost(c->stage);
            c->stage = nullptr;
            c->stage_bytes = 0;
            if ((rc = cuda_check(c, cudaHostAlloc(&c->stage, stage_b, cudaHostAllocDefault), "job staging"))) return rc;
            c->stage_bytes = stage_b;
        }
        char *h = (char *)c->stage, *d = (char *)c->jobdesc.p;
        I8Desc *hd = (I8Desc *)h;
        int *hg = (int *)(h + off_g), *ho = (int *)(h + off_o);
        std::vector<LsReduceJob> red;
        size_t gpos = 0, opos = 0;
        for (size_t i = 0; i < plans.size(); ++i) {
            const I8Job &jb = jobs[j0 + i];
            const LsJobPlan &p = plans[i];
            const LsShape &s = p.s;
            I8Desc &x = hd[i];
            memset(&x, 0, sizeof(x));
            x.span3 = s.AB + (s.k > 1 ? s.nclen : s.rows(0)) - 1;
            x.span2 = s.AB + s.cols(0) - 1;
            const cuuint64_t fdims[2] = {(cuuint64_t)jb.k, (cuuint64_t)jb.nc};
            const cuuint64_t fstr[1] = {(cuuint64_t)jb.kp * 4};
            const cuuint32_t box3[2] = {SLICE, (cuuint32_t)x.span3}, box1[2] = {SLICE, (cuuint32_t)s.AB};
            if ((rc = encode(c, &x.t3, f32, 2, jb.m3.f32, fdims, fstr, box3, CU_TENSOR_MAP_SWIZZLE_128B))) return rc;
            if ((rc = encode(c, &x.t1, f32, 2, jb.m1.f32, fdims, fstr, box1, CU_TENSOR_MAP_SWIZZLE_NONE))) return rc;
            const cuuint64_t ddims[4] = {16, (cuuint64_t)jb.nc, (cuuint64_t)(jb.kp / 16), 3};
            const cuuint64_t dstr[3] = {16, (cuuint64_t)jb.nc * 16, (cuuint64_t)jb.nc * jb.kp};
            const cuuint32_t box2[4] = {16, (cuuint32_t)x.span2, 2, 3};
            if ((rc = encode(c, &x.t2, u8, 4, jb.m2.dig, ddims, dstr, box2, CU_TENSOR_MAP_SWIZZLE_NONE))) return rc;
            x.e1 = jb.m1.bexp;
            x.e2 = jb.m2.bexp;
            x.e3 = jb.m3.bexp;
            x.groups = (const int *)(d + off_g) + gpos;
            x.group_off = (const int *)(d + off_o) + opos;
            x.k = jb.k;
            x.nc = jb.nc;
            x.nc10 = jb.nc10;
            x.nclen = s.nclen;
            x.ks = s.k;
            x.AB = s.AB;
            x.T = s.T;
            x.sweeps = jb.mask_pass ? 2 : 1;
            x.tx_bytes = (uint32_t)(x.span3 * 128 + s.AB * 128 + 3 * 2 * x.span2 * 16);
            std::copy(p.groups.begin(), p.groups.end(), hg + gpos);
            for (size_t q = 0; q < p.group_off.size(); ++q) ho[opos + q] = p.group_off[q];
            gpos += p.groups.size();
            opos += p.group_off.size();
            red.push_back(LsReduceJob{(const double *)c->partial.p + p.unit_base * LS_ROWS * LS_ROWS, jb.lag_out,
                                      s.nclen, s.k, s.T, s.nab, s.V});
        }
        std::copy(units.begin(), units.end(), (LsUnit *)(h + off_u));
        if ((rc = cuda_check(c, cudaMemcpyAsync(d, h, stage_b, cudaMemcpyHostToDevice, c->stream), "job list upload")))
            return rc;
        phase_begin(c, 1);
        ls_i8_kernel<<<(unsigned)units.size(), NTHREADS, SMEM_BYTES, c->stream>>>(
            (const I8Desc *)d, (const LsUnit *)(d + off_u), (double *)c->partial.p, d_err);
        phase_end(c);
        c->launches += 1;
        c->contractions += 1;
        if ((rc = cuda_check(c, cudaGetLastError(), "ls_i8_kernel launch"))) return rc;
        if ((rc = ls_reduce(c, red))) return rc;
        j0 = j1;
    }
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
    jb.m1 = m1;
    jb.m2 = m2;
    jb.m3 = m3;
    jb.k = k;
    jb.kp = kp;
    jb.nc = (int)c->nc;
    jb.nc10 = c->nc10;
    jb.weight = &c->weight;
    jb.nanchors = (int)c->anchors.size();
    jb.mask_pass = false;
    jb.lag_out = lag_out;
    return contract_i8_jobs(c, jobs);
}

}  // namespace amber
