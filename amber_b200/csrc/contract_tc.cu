// Mixed-precision triple-product lag accumulation on the 5th-generation
// tensor cores (tcgen05 + TMEM + TMA), replacing the float loop of
// 4_fbe/amber.c:247-279 / amber_v2.c:243-283.
//
// For one anchor channel p1 the reference's work is the matrix
//     T_p1[p2, p3] = Σ_x (D1[p1,x]·D2[p2,x]) · D3[p3,x]
// over the lag window p2, p3 ∈ [p1−nc10, p1+nc10].  Here that is a GEMM with
// M = p2 (128 rows = the 128 TMEM lanes), N = p3 (BN columns), K = pixels:
//   A[m][x] = D1[p1,x]·D2[p2(m),x]  formed on the CUDA cores in FP32 from the
//             maps' bf16 hi/lo planes, split again into bf16 hi + lo and
//             written straight into TMEM (tcgen05.st) — the "TS" MMA form, so
//             A never touches shared memory;
//   B[n][x] = D3[p3(n),x]           bf16 hi/lo planes streamed by TMA into
//             128-byte-swizzled shared memory;
//   D      += A_hi·B_hiᵀ + A_hi·B_loᵀ + A_lo·B_hiᵀ   (split-BF16×3, FP32 in TMEM).
// Two anchors p1, p1+1 whose windows fit one BN-wide B tile share every B
// tile (halving TMA traffic); each keeps its own accumulator.
//
// Warp roles (320 threads): warps 0-7 form A (and read the accumulators out
// at the end), warp 8 issues TMA, warp 9 owns TMEM and issues the MMAs from
// one thread.  Stages are handed over with mbarriers; every wait is bounded
// and on expiry raises an error flag the host turns into AMBER_ERR_TIMEOUT,
// drains its own in-flight work and frees TMEM before returning.
//
// A CTA covers one pixel chunk; its FP32 tile is converted to FP64 and
// written, weighted by the channel multiplicities, to the partial buffer
// [anchor][chunk][lag2][lag3], which lag_reduce sums per lag cell with a
// compensated FP64 accumulator in a fixed order (deterministic).
#include <cuda.h>
#include <cuda_bf16.h>

#include <algorithm>
#include <vector>

#include "common.cuh"
#include "tc_ptx.cuh"

namespace amber {

namespace {

using namespace tc;

constexpr int BM = 128;       // p2 rows per tile = TMEM lanes
constexpr int KBLK = 64;      // pixels per stage: one 128-byte swizzle row of bf16
constexpr int NWARP_A = 8;    // A-forming / epilogue warps
constexpr int WARP_TMA = 8;
constexpr int WARP_MMA = 9;
constexpr int NTHREADS = 320;
constexpr int TMEM_COLS = 512;
constexpr int A_COL0 = 256;   // TMEM columns [256, 512) hold the A stages

struct Group {
    int p1[2];     // anchor channels (p1[1] valid when count == 2)
    int aidx[2];   // anchor indices (rows of the partial buffer)
    int count;
    int off1;      // p1[1] − p1[0]
};

struct Params {
    const uint16_t *h1, *l1, *h2, *l2;  // D1, D2 hi/lo planes [nc][kp]
    long k, kp;
    int nc, nc10, nclen;
    int mt_count, nt_count, nchunk;
    long chunk;      // pixels per chunk (multiple of KBLK)
    const Group *groups;
    int ngroups;
    const int *weight;
    double *partial;  // [anchor][chunk][nclen²]
    int *err;
};

// ---- the kernel -------------------------------------------------------------------------------

template <int P, int BN>
__global__ void __launch_bounds__(NTHREADS, 1)
    contract_tc_kernel(const __grid_constant__ CUtensorMap tm_hi, const __grid_constant__ CUtensorMap tm_lo,
                       const Params prm)
{
    constexpr int NSA = (P == 2) ? 2 : 4;  // A stages in TMEM
    constexpr int STAGE_B = 2 * BN * KBLK * 2;  // hi + lo tiles
    constexpr int NSB = (200 * 1024 / STAGE_B) < 4 ? (200 * 1024 / STAGE_B) : 4;
    static_assert(P * BN <= A_COL0, "accumulators must fit below the A region");
    static_assert(A_COL0 + NSA * P * 64 <= TMEM_COLS, "A stages must fit in TMEM");
    static_assert(BN % 32 == 0 && BN >= 32 && BN <= 256, "BN");

    extern __shared__ __align__(1024) unsigned char smem_raw[];
    unsigned char *smem = (unsigned char *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    unsigned char *b_tiles = smem;  // NSB × {hi, lo}
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem + NSB * STAGE_B);
    uint64_t *b_full = bars, *b_empty = bars + NSB;
    uint64_t *a_full = bars + 2 * NSB, *a_empty = bars + 2 * NSB + NSA;
    uint64_t *acc_full = bars + 2 * NSB + 2 * NSA;
    uint64_t *drain = acc_full + 1;
    volatile uint32_t *tmem_slot = reinterpret_cast<volatile uint32_t *>(drain + 1);
    volatile int *abort_flag = reinterpret_cast<volatile int *>(tmem_slot + 1);

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

    // work item → (group, m-tile, n-tile, chunk)
    // Chunk-major order (see contract_i8.cu): resident CTAs share a pixel chunk.
    long item = blockIdx.x;
    const int nt = (int)(item % prm.nt_count);
    item /= prm.nt_count;
    const int mt = (int)(item % prm.mt_count);
    item /= prm.mt_count;
    const int g = (int)(item % prm.ngroups);
    const int chunk = (int)(item / prm.ngroups);
    const Group grp = prm.groups[g];
    const long x_begin = (long)chunk * prm.chunk;
    const long x_end = min(prm.k, x_begin + prm.chunk);
    const int nstage = (int)((x_end - x_begin + KBLK - 1) / KBLK);
    const int bbase = grp.p1[0] - prm.nc10 + nt * BN;  // first p3 row of the B tile

    if (tid == 0) {
        for (int s = 0; s < NSB; ++s) { mbar_init(&b_full[s], 1); mbar_init(&b_empty[s], 1); }
        for (int s = 0; s < NSA; ++s) { mbar_init(&a_full[s], NWARP_A); mbar_init(&a_empty[s], 1); }
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

    if (warp == WARP_TMA) {
        if (lane == 0) {
            int issued = 0;
            for (int it = 0; it < nstage; ++it) {
                const int s = it % NSB;
                if (!mbar_wait(&b_empty[s], ((it / NSB) & 1) ^ 1, abort_flag, prm.err, 1)) break;
                unsigned char *hi = b_tiles + s * STAGE_B;
                mbar_expect_tx(&b_full[s], STAGE_B);
                const int x = (int)(x_begin + (long)it * KBLK);
                tma_load_2d(hi, &tm_hi, &b_full[s], x, bbase);
                tma_load_2d(hi + STAGE_B / 2, &tm_lo, &b_full[s], x, bbase);
                ++issued;
            }
            if (*abort_flag) {
                // let our own copies land before the CTA's shared memory goes away
                for (int it = max(0, issued - NSB); it < issued; ++it) {
                    const int s = it % NSB;
                    for (long long i = 0; i < WAIT_LIMIT && !mbar_try_wait(&b_full[s], (it / NSB) & 1); ++i)
                        __nanosleep(100);
                }
            }
        }
    } else if (warp == WARP_MMA) {
        if (lane == 0) {
            // instruction descriptor: F32 accumulate, BF16 A and B, both K-major, M = 128, N = BN
            const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) |
                                   ((uint32_t)(BM >> 4) << 24);
            bool ok = true;
            for (int it = 0; it < nstage && ok; ++it) {
                const int sb = it % NSB, sa = it % NSA;
                if (!mbar_wait(&b_full[sb], (it / NSB) & 1, abort_flag, prm.err, 2)) { ok = false; break; }
                if (!mbar_wait(&a_full[sa], (it / NSA) & 1, abort_flag, prm.err, 3)) { ok = false; break; }
                fence_after();
                const uint32_t bh = smem_u32(b_tiles + sb * STAGE_B), bl = bh + STAGE_B / 2;
#pragma unroll
                for (int a = 0; a < P; ++a) {
                    if (a >= grp.count) break;
                    const uint32_t d = tmem + a * BN;
                    const uint32_t acol = tmem + A_COL0 + (sa * P + a) * 64;
#pragma unroll
                    for (int kk = 0; kk < KBLK / 16; ++kk) {
                        const uint64_t dh = smem_desc_sw128(bh + kk * 32), dl = smem_desc_sw128(bl + kk * 32);
                        const uint32_t ah = acol + kk * 8, al = acol + 32 + kk * 8;
                        umma_ts(d, ah, dh, idesc, (it | kk) ? 1u : 0u);
                        umma_ts(d, ah, dl, idesc, 1u);
                        umma_ts(d, al, dh, idesc, 1u);
                    }
                }
                umma_commit(&b_empty[sb]);
                umma_commit(&a_empty[sa]);
            }
            if (ok) {
                umma_commit(acc_full);
            } else {
                // drain: wait until every MMA we issued has finished before TMEM is freed
                umma_commit(drain);
                for (long long i = 0; i < WAIT_LIMIT && !mbar_try_wait(drain, 0); ++i) __nanosleep(100);
            }
        }
    } else {
        // ---- A formation: warps 0-7 ----
        const int wg = warp >> 2;            // warpgroup 0 or 1
        const int m = ((warp & 3) << 5) + lane;  // TMEM lane = row of the tile
        const uint32_t lane_field = (uint32_t)((warp & 3) << 5) << 16;
        // P == 2: warpgroup wg forms anchor wg over the whole stage (two 32-pixel units).
        // P == 1: warpgroup wg forms pixels [32·wg, 32·wg + 32) of anchor 0.
        const int anchor = (P == 2) ? wg : 0;
        const bool active = anchor < grp.count;
        const int p1 = grp.p1[anchor];
        const int d2 = mt * BM + m;
        const int p2 = p1 - prm.nc10 + d2;
        const bool row_ok = active && d2 < prm.nclen && p2 >= 0 && p2 < prm.nc && prm.weight[p2] > 0;
        const uint16_t *r1h = prm.h1 + (long)p1 * prm.kp, *r1l = prm.l1 + (long)p1 * prm.kp;
        const uint16_t *r2h = prm.h2 + (long)(row_ok ? p2 : 0) * prm.kp;
        const uint16_t *r2l = prm.l2 + (long)(row_ok ? p2 : 0) * prm.kp;
        bool ok = true;
        for (int it = 0; it < nstage; ++it) {
            const int sa = it % NSA;
            if (!mbar_wait_warp(&a_empty[sa], ((it / NSA) & 1) ^ 1, abort_flag, prm.err, 4)) { ok = false; break; }
            fence_after();
            const long xs = x_begin + (long)it * KBLK;
#pragma unroll
            for (int u = 0; u < (P == 2 ? 2 : 1); ++u) {
                const int px0 = (P == 2) ? u * 32 : wg * 32;  // pixel offset inside the stage
                uint32_t hv[16], lv[16];
                if (row_ok && active) {
                    const long x = xs + px0;
                    // 32 pixels of D1 and D2, hi and lo planes: 4 × 16-byte loads each
                    uint4 a_h[4], a_l[4], b_h[4], b_l[4];
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        a_h[q] = __ldg(reinterpret_cast<const uint4 *>(r1h + x) + q);
                        a_l[q] = __ldg(reinterpret_cast<const uint4 *>(r1l + x) + q);
                        b_h[q] = __ldg(reinterpret_cast<const uint4 *>(r2h + x) + q);
                        b_l[q] = __ldg(reinterpret_cast<const uint4 *>(r2l + x) + q);
                    }
                    const uint32_t *ah = reinterpret_cast<const uint32_t *>(a_h);
                    const uint32_t *al = reinterpret_cast<const uint32_t *>(a_l);
                    const uint32_t *bh = reinterpret_cast<const uint32_t *>(b_h);
                    const uint32_t *blw = reinterpret_cast<const uint32_t *>(b_l);
#pragma unroll
                    for (int w2 = 0; w2 < 16; ++w2) {
                        float c0 = (bf_lo(ah[w2]) + bf_lo(al[w2])) * (bf_lo(bh[w2]) + bf_lo(blw[w2]));
                        float c1 = (bf_hi(ah[w2]) + bf_hi(al[w2])) * (bf_hi(bh[w2]) + bf_hi(blw[w2]));
                        const long xx = x + 2 * w2;
                        if (xx >= x_end) c0 = 0.f;
                        if (xx + 1 >= x_end) c1 = 0.f;
                        const uint32_t h0 = bf16_rn_bits(c0), h1 = bf16_rn_bits(c1);
                        const uint32_t l0 = bf16_rn_bits(c0 - __uint_as_float(h0 << 16));
                        const uint32_t l1 = bf16_rn_bits(c1 - __uint_as_float(h1 << 16));
                        hv[w2] = h0 | (h1 << 16);
                        lv[w2] = l0 | (l1 << 16);
                    }
                } else {
#pragma unroll
                    for (int w2 = 0; w2 < 16; ++w2) { hv[w2] = 0u; lv[w2] = 0u; }
                }
                const uint32_t col = A_COL0 + (sa * P + anchor) * 64 + px0 / 2;
                tmem_st16(tmem + lane_field + col, hv);
                tmem_st16(tmem + lane_field + col + 32, lv);
            }
            asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
            fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(&a_full[sa]);
        }

        // ---- epilogue: TMEM accumulators → FP64 partial tiles ----
        if (ok && mbar_wait_warp(acc_full, 0, abort_flag, prm.err, 5)) {
            fence_after();
            const double w1 = active ? (double)prm.weight[p1] : 0.0;
            const double wr = row_ok ? w1 * (double)prm.weight[p2] : 0.0;
            const int off = (P == 2 && anchor == 1) ? grp.off1 : 0;
            const int c_begin = (P == 2) ? 0 : wg * (BN / 2);
            const int c_end = (P == 2) ? BN : c_begin + BN / 2;
            double *dst = nullptr;
            if (active && d2 < prm.nclen)
                dst = prm.partial + ((long)grp.aidx[anchor] * prm.nchunk + chunk) * prm.nclen * prm.nclen +
                      (long)d2 * prm.nclen;
            for (int c0 = c_begin; c0 < c_end; c0 += 16) {
                uint32_t v[16];
                tmem_ld16(tmem + lane_field + anchor * BN + c0, v);
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                if (dst) {
#pragma unroll
                    for (int j = 0; j < 16; ++j) {
                        const int n = c0 + j;
                        const int d3 = nt * BN + n - off;
                        if (d3 < 0 || d3 >= prm.nclen) continue;
                        // columns this n-tile owns for this anchor
                        if (n - off < 0 && nt == 0) continue;
                        const int p3 = bbase + n;
                        double wc = (p3 >= 0 && p3 < prm.nc) ? (double)prm.weight[p3] : 0.0;
                        dst[d3] = (double)__uint_as_float(v[j]) * wr * wc;
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

template <int P, int BN>
size_t smem_bytes()
{
    constexpr int STAGE_B = 2 * BN * KBLK * 2;
    constexpr int NSB = (200 * 1024 / STAGE_B) < 4 ? (200 * 1024 / STAGE_B) : 4;
    return 1024 + (size_t)NSB * STAGE_B + 256;
}

typedef CUresult (*EncodeTiled)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

int make_map(amber_cuda_ctx *c, CUtensorMap *m, const uint16_t *plane, long k, long kp, long rows, int box_rows)
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
    cuuint64_t strides[1] = {(cuuint64_t)kp * 2};
    cuuint32_t box[2] = {(cuuint32_t)KBLK, (cuuint32_t)box_rows};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, (void *)plane, dims, strides, box, estr,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(c, AMBER_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
    return AMBER_OK;
}

template <int P, int BN>
int launch(amber_cuda_ctx *c, const CUtensorMap &th, const CUtensorMap &tl, const Params &prm, long items)
{
    const size_t sm = smem_bytes<P, BN>();
    cudaFuncSetAttribute(contract_tc_kernel<P, BN>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    phase_begin(c, 1);
    contract_tc_kernel<P, BN><<<(unsigned)items, NTHREADS, sm, c->stream>>>(th, tl, prm);
    phase_end(c);
    c->launches += 1;
    c->contractions += 1;
    return cuda_check(c, cudaGetLastError(), "contract_tc_kernel launch");
}

}  // namespace

int contract_bf16x3(amber_cuda_ctx *c, const uint16_t *h1, const uint16_t *l1, const uint16_t *h2, const uint16_t *l2,
                   const uint16_t *h3, const uint16_t *l3, long k, long kp, double *lag_out)
{
    const int nc10 = c->nc10, nclen = 2 * nc10 + 1;
    const long ncsize = (long)nclen * nclen;
    const int nA = (int)c->anchors.size();
    if (nA == 0) return cuda_check(c, cudaMemsetAsync(lag_out, 0, sizeof(double) * ncsize, c->stream), "zero lag");

    // tile plan
    int P, BN, MT, NT;
    if (nclen + 1 <= 128) {
        P = 2;
        BN = std::max(32, (nclen + 1 + 31) / 32 * 32);
        MT = 1;
        NT = 1;
    } else {
        P = 1;
        MT = (nclen + BM - 1) / BM;
        NT = (nclen + 255) / 256;
        BN = ((nclen + NT - 1) / NT + 31) / 32 * 32;
    }
    // anchor groups: consecutive unflagged channels pair up when P == 2
    std::vector<Group> groups;
    for (int i = 0; i < nA;) {
        Group g{};
        g.p1[0] = c->anchors[i];
        g.aidx[0] = i;
        g.count = 1;
        if (P == 2 && i + 1 < nA && c->anchors[i + 1] - c->anchors[i] <= BN - nclen) {
            g.p1[1] = c->anchors[i + 1];
            g.aidx[1] = i + 1;
            g.off1 = g.p1[1] - g.p1[0];
            g.count = 2;
            i += 2;
        } else {
            g.p1[1] = g.p1[0];
            g.aidx[1] = i;
            g.off1 = 0;
            i += 1;
        }
        groups.push_back(g);
    }
    const long base_items = (long)groups.size() * MT * NT;
    const long target = 4L * c->num_sms;
    long max_chunk = c->chunk_px > 0 ? c->chunk_px : 32768;
    max_chunk = std::max<long>(KBLK, max_chunk / KBLK * KBLK);
    long nch = std::max<long>((k + max_chunk - 1) / max_chunk, std::min<long>((target + base_items - 1) / base_items,
                                                                           (k + 1023) / 1024));
    nch = std::max<long>(nch, 1);
    long chunk = ((k + nch - 1) / nch + KBLK - 1) / KBLK * KBLK;
    nch = (k + chunk - 1) / chunk;

    int rc;
    const size_t gbytes = sizeof(Group) * groups.size();
    const size_t pbytes = sizeof(double) * (size_t)nA * nch * ncsize;
    if ((rc = ensure(c, c->partial, pbytes, "partial lag tiles"))) return rc;
    if ((rc = ensure(c, c->misc, 256 + gbytes, "tile plan"))) return rc;
    int *d_err = (int *)c->misc.p;
    Group *d_groups = (Group *)((char *)c->misc.p + 256);
    if ((rc = cuda_check(c, cudaMemcpyAsync(d_groups, groups.data(), gbytes, cudaMemcpyHostToDevice, c->stream),
                         "tile plan upload")))
        return rc;
    if ((rc = cuda_check(c, cudaMemsetAsync(d_err, 0, sizeof(int), c->stream), "error flag"))) return rc;

    CUtensorMap th, tl;
    if ((rc = make_map(c, &th, h3, k, kp, c->nc, BN))) return rc;
    if ((rc = make_map(c, &tl, l3, k, kp, c->nc, BN))) return rc;
    Params prm{};
    prm.h1 = h1; prm.l1 = l1; prm.h2 = h2; prm.l2 = l2;
    prm.k = k; prm.kp = kp;
    prm.nc = (int)c->nc; prm.nc10 = nc10; prm.nclen = nclen;
    prm.mt_count = MT; prm.nt_count = NT; prm.nchunk = (int)nch; prm.chunk = chunk;
    prm.groups = d_groups; prm.ngroups = (int)groups.size();
    prm.weight = (const int *)c->d_weight.p;
    prm.partial = (double *)c->partial.p;
    prm.err = d_err;
    const long items = base_items * nch;

#define CASE(PP, BB)                                                   \
    if (P == PP && BN == BB) rc = launch<PP, BB>(c, th, tl, prm, items); \
    else
    CASE(2, 32) CASE(2, 64) CASE(2, 96) CASE(2, 128)
    CASE(1, 160) CASE(1, 192) CASE(1, 224) CASE(1, 256) CASE(1, 128)
    rc = fail(c, AMBER_ERR_ARG, "no tile configuration for nclen=%d (P=%d BN=%d)", nclen, P, BN);
#undef CASE
    if (rc) return rc;
    if ((rc = lag_reduce(c, (const double *)c->partial.p, (long)nA * nch, ncsize, lag_out))) return rc;
    int herr = 0;
    if ((rc = cuda_check(c, cudaMemcpyAsync(&herr, d_err, sizeof(int), cudaMemcpyDeviceToHost, c->stream),
                         "error flag read")))
        return rc;
    if ((rc = cuda_check(c, cudaStreamSynchronize(c->stream), "contract_tc"))) return rc;
    if (herr) return fail(c, AMBER_ERR_TIMEOUT, "tensor-core contraction: a pipeline wait gave up (site %d)", herr);
    return AMBER_OK;
}

}  // namespace amber
