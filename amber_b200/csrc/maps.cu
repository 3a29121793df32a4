// Ring filter + unnormalised 2D c2r, fused and batched over (ring × channel).
//
// Replaces Dfg/Ifg + fill_s2d_float/fill_s2I (4_fbe/amber_funcs.c:573-621,
// 967-1010, 1109-1131) and the mask transform inside calCR (389-437).  For a
// ring [lo, hi) the reference scatters grid cell (ia mod N1, j) into bin
// (ia mod Ng1, j) of a zeroed Ng1 × (Ng1/2+1) half-plane for ia ∈ (−Ng1/2,
// Ng1/2], j < Ng1/3, lo ≤ √(ia²+j²) < hi, √ > 0, then runs
// fftw_plan_dft_c2r_2d.  Only |ia|, j < hi are ever non-zero, so instead of a
// full FFT of a mostly-empty plane we evaluate the transform directly on the
// non-zero support ("pruned DFT"), which is exact for any Ng1 — the map sides
// here have large prime factors (740 = 4·5·37, 1460 = 4·5·73):
//
//   pass 1 (axis 0, per column j < J):  Y[n0][j] = Σ_ia X[ia][j] · e^{+2πi·ia·n0/Ng1}
//   pass 2 (axis 1, c2r):               D[n0][n1] = Re Y[n0][0] + 2 Σ_{j≥1} Re(Y[n0][j] · e^{+2πi·j·n1/Ng1})
//
// The c2r convention — complex DFT along axis 0, then a 1D c2r along axis 1
// that ignores Im of bin 0 — is what a rank-2 c2r does with the non-Hermitian
// j = 0 column the ring scatter produces; the Nyquist bin j = Ng1/2 is never
// filled because j < Ng1/3.
//
// Both passes stage one column / one row of the spectrum for C channels in
// shared memory together with the twiddle table e^{2πik/Ng1}; lanes of a warp
// walk channels (coalesced loads of the channel-innermost grid and of Y) and
// share one twiddle per step (a shared-memory broadcast).  Twiddle indices
// advance incrementally (k += n mod Ng1), so the inner loop is FP64 FMA work;
// pass 2 evaluates pixels n1 and Ng1 − n1 from the same twiddle (the table is
// exactly conjugate-symmetric).
// All arithmetic is FP64.
#include <cuda_bf16.h>
#include <math.h>

#include <algorithm>
#include <vector>

#include "lagspace.cuh"

namespace amber {

namespace {

constexpr int kThreads = 256;

// Rows of column j that fall inside ring [lo, hi) for an ng-point output grid.
__device__ __forceinline__ bool in_ring(long ia, long j, double lo, double hi)
{
    double uu = sqrt(1.0 * (double)(ia * ia + j * j));
    return uu >= lo && uu < hi && uu > 0.0;
}

// Ring edges and column counts of the slots one launch builds, passed by value: no upload and no
// stream synchronisation before the launch, so the host can queue the next request's maps while
// these run.  A batch with more slots runs as several launches.
constexpr int RING_META_MAX = 96;
struct RingMeta {
    double lo[RING_META_MAX], hi[RING_META_MAX];
    int jc[RING_META_MAX];
};

template <int C>
__global__ void __launch_bounds__(kThreads) ring_cols_kernel(const void *__restrict__ src, int src_complex, long n1,
                                                              long nc, long chan_base, long nch, long ng,
                                                              const RingMeta meta, int jmax,
                                                              const double2 *__restrict__ tw_g,
                                                              double2 *__restrict__ Y, int rowcap)
{
    extern __shared__ double2 smem[];
    double2 *tw = smem;                        // ng
    double2 *xs = tw + ng;                     // rowcap × C
    int *ias = reinterpret_cast<int *>(xs + (size_t)rowcap * C);  // rowcap
    __shared__ int warp_cnt[kThreads / 32];
    __shared__ int nrows_s;

    const int j = blockIdx.x, s = blockIdx.y;
    const long q0 = (long)blockIdx.z * C;
    if (j >= meta.jc[s]) return;
    const double lo = meta.lo[s], hi = meta.hi[s];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const long h1 = n1 / 2 + 1;

    for (long i = tid; i < ng; i += kThreads) tw[i] = tw_g[i];

    // Ordered compaction of the ring's rows in this column.
    const long A = (long)ceil(hi) - 1;
    const long ia_min = max(-A, -ng / 2 + 1), ia_max = min(A, ng / 2);
    if (tid == 0) nrows_s = 0;
    __syncthreads();
    for (long base = ia_min; base <= ia_max; base += kThreads) {
        long ia = base + tid;
        bool hit = ia <= ia_max && in_ring(ia, j, lo, hi);
        unsigned m = __ballot_sync(0xffffffffu, hit);
        if (lane == 0) warp_cnt[warp] = __popc(m);
        __syncthreads();
        int off = nrows_s;
        for (int w = 0; w < warp; ++w) off += warp_cnt[w];
        off += __popc(m & ((1u << lane) - 1u));
        if (hit && off < rowcap) ias[off] = (int)ia;
        __syncthreads();
        if (tid == 0) {
            int tot = 0;
            for (int w = 0; w < kThreads / 32; ++w) tot += warp_cnt[w];
            nrows_s += tot;
        }
        __syncthreads();
    }
    const int nrows = min(nrows_s, rowcap);

    // Gather the ring's cells for C channels (channel-innermost: coalesced).
    for (int e = tid; e < nrows * C; e += kThreads) {
        int r = e / C, q = e % C;
        long ia = ias[r];
        long iN = ia < 0 ? n1 + ia : ia;
        long cell = iN * h1 + j;
        double2 v = make_double2(0.0, 0.0);
        if (q0 + q < nch) {
            long ch = chan_base + q0 + q;
            if (src_complex)
                v = reinterpret_cast<const double2 *>(src)[cell * nc + ch];
            else
                v.x = reinterpret_cast<const double *>(src)[cell * nc + ch];
        }
        xs[r * C + q] = v;
    }
    __syncthreads();

    // Y[n0][j] for this thread's channel q and R rows n0 at a time.
    constexpr int G = 32 / C;  // n0 groups per warp
    constexpr int R = 4;
    const int q = lane % C, g = lane / C;
    const int gid = warp * G + g;
    const int ngroups = (kThreads / 32) * G;
    for (long nb = (long)gid; nb * R < ng; nb += ngroups) {
        long n0[R];
        double2 acc[R];
        int idx[R];
#pragma unroll
        for (int r = 0; r < R; ++r) {
            n0[r] = nb * R + r;
            acc[r] = make_double2(0.0, 0.0);
            idx[r] = 0;
        }
        long prev = LONG_MIN;
        for (int row = 0; row < nrows; ++row) {
            long ia = ias[row];
            if (ia != prev + 1) {
                long iam = ia < 0 ? ia + ng : ia;
#pragma unroll
                for (int r = 0; r < R; ++r) idx[r] = (int)((iam * (n0[r] < ng ? n0[r] : 0)) % ng);
            } else {
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    int t = idx[r] + (int)(n0[r] < ng ? n0[r] : 0);
                    idx[r] = t >= ng ? t - (int)ng : t;
                }
            }
            prev = ia;
            double2 x = xs[row * C + q];
#pragma unroll
            for (int r = 0; r < R; ++r) {
                double2 w = tw[idx[r]];
                acc[r].x = fma(x.x, w.x, acc[r].x);
                acc[r].x = fma(-x.y, w.y, acc[r].x);
                acc[r].y = fma(x.x, w.y, acc[r].y);
                acc[r].y = fma(x.y, w.x, acc[r].y);
            }
        }
        if (q0 + q < nch) {
#pragma unroll
            for (int r = 0; r < R; ++r)
                if (n0[r] < ng) Y[(((long)s * ng + n0[r]) * jmax + j) * nch + q0 + q] = acc[r];
        }
    }
}

__device__ __forceinline__ uint16_t bf16_bits(float f)
{
    __nv_bfloat16 b = __float2bfloat16_rn(f);
    return *reinterpret_cast<uint16_t *>(&b);
}

template <int C>
__global__ void __launch_bounds__(kThreads) ring_rows_kernel(const double2 *__restrict__ Y, long ng, int jmax,
                                                              const RingMeta meta, long nch,
                                                              const double2 *__restrict__ tw_g, long kp,
                                                              double *__restrict__ out_f64,
                                                              uint16_t *__restrict__ out_hi,
                                                              uint16_t *__restrict__ out_lo,
                                                              float *__restrict__ out_f32,
                                                              const int *__restrict__ weight)
{
    extern __shared__ double2 smem[];
    double2 *tw = smem;       // ng
    double2 *ys = tw + ng;    // J × C
    const long n0 = blockIdx.x;
    const int s = blockIdx.y;
    const long q0 = (long)blockIdx.z * C;
    const int J = meta.jc[s];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (long i = tid; i < ng; i += kThreads) tw[i] = tw_g[i];
    for (int e = tid; e < J * C; e += kThreads) {
        int jj = e / C, q = e % C;
        double2 v = make_double2(0.0, 0.0);
        if (q0 + q < nch) v = Y[(((long)s * ng + n0) * jmax + jj) * nch + q0 + q];
        if (jj == 0) v.y = 0.0;  // c2r ignores Im of the DC bin
        else { v.x *= 2.0; v.y *= 2.0; }
        ys[e] = v;
    }
    __syncthreads();

    constexpr int G = 32 / C;
    // A thread evaluates R pixel pairs (x, Ng − x): they share each twiddle, cos and −sin,
    // so one shared-memory load and one index step feed four FMAs.  x runs over [0, Ng/2];
    // for x = 0 and x = Ng/2 the pair is one pixel.
    constexpr int R = 4;
    const int q = lane % C, g = lane / C;
    const int gid = warp * G + g;
    const int ngroups = (kThreads / 32) * G;
    const long npair = ng / 2 + 1;
    const long slot_row = ((long)s * nch + q0 + q) * kp + n0 * ng;
    // the mixed path's fp32 maps carry the channel multiplicity (0 for flagged channels)
    const double wq = (weight && q0 + q < nch) ? (double)weight[q0 + q] : 1.0;
    for (long nb = gid; nb * R < npair; nb += ngroups) {
        double acc[R], accm[R];  // pixel x, pixel Ng − x
        int idx[R], step[R];
#pragma unroll
        for (int r = 0; r < R; ++r) {
            long x = nb * R + r;
            step[r] = (int)(x < npair ? x : 0);
            idx[r] = 0;
            acc[r] = 0.0;
            accm[r] = 0.0;
        }
        for (int jj = 0; jj < J; ++jj) {
            double2 y = ys[jj * C + q];
#pragma unroll
            for (int r = 0; r < R; ++r) {
                double2 w = tw[idx[r]];
                acc[r] = fma(y.x, w.x, acc[r]);
                acc[r] = fma(-y.y, w.y, acc[r]);
                accm[r] = fma(y.x, w.x, accm[r]);
                accm[r] = fma(y.y, w.y, accm[r]);
                int t = idx[r] + step[r];
                idx[r] = t >= ng ? t - (int)ng : t;
            }
        }
        if (q0 + q < nch) {
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const long x = nb * R + r;
                if (x >= npair) continue;
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const long n1 = h == 0 ? x : ng - x;
                    if (h == 1 && (x == 0 || n1 == x)) continue;
                    const long o = slot_row + n1;
                    const double v = h == 0 ? acc[r] : accm[r];
                    if (out_f64) out_f64[o] = v;
                    if (out_f32) out_f32[o] = (float)(v * wq);
                    if (out_hi) {
                        // split: hi = bf16(v), lo = bf16(v − hi) (both round-to-nearest)
                        float f = (float)v;
                        uint16_t hb = bf16_bits(f);
                        float hf = __uint_as_float((uint32_t)hb << 16);
                        out_hi[o] = hb;
                        out_lo[o] = bf16_bits((float)(v - (double)hf));
                    }
                }
            }
        }
    }
}

// Fixed-point digits for the int8 tensor-core contraction.  Every block of
// LS_BLOCK pixels of a ring slot has one exponent E, shared by all channels:
// the smallest with max|v| < 2^E over the block (0 for an all-zero block).
// Then, with base 254,
//     v·2^−E·127 = d0 + d1/254 + d2/254² + r,   d0, d1, d2 ∈ [−127, 127],
// |r| ≤ 1/(2·254²): signed, balanced digits that use the whole int8 range.
// An exponent per pixel block (rather than per channel row) is what lets the
// contraction add every anchor into one accumulator (lagspace.cuh), and it
// follows the maps' spatial dynamic range: the sampling-mask maps are sharply
// peaked at the origin, so blocks far from it get a much finer digit scale.
__device__ __forceinline__ void digits254(float t, uint32_t &b0, uint32_t &b1, uint32_t &b2)
{
    // round-to-nearest via the 1.5·2^23 magic number: the integer sits in the
    // low mantissa bits, so its low byte is the two's-complement int8 digit
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

// bexp[s][b] for block b of slot s (one CTA of LS_BLOCK threads per block: a thread per pixel,
// looping over the channels, so every channel row is read coalesced).
__global__ void __launch_bounds__(LS_BLOCK) block_expo_kernel(const float *__restrict__ f32, long k, long kp,
                                                              long nch, long nblk, int *__restrict__ bexp)
{
    __shared__ float red[LS_BLOCK / 32];
    const long b = blockIdx.x;
    const int s = blockIdx.y;
    const long x = b * LS_BLOCK + threadIdx.x;
    float m = 0.f;
    if (x < k)
        for (long ch = 0; ch < nch; ++ch) m = fmaxf(m, fabsf(f32[((long)s * nch + ch) * kp + x]));
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < LS_BLOCK / 32; ++w) m = fmaxf(m, red[w]);
        bexp[(long)s * nblk + b] = m > 0.f ? ilogbf(m) + 1 : 0;
    }
}

// Three digit planes per slot in the contraction's staging order,
// dig[s][digit][x/16][ch][16 pixels]: a TMA box of consecutive channels and two 16-pixel
// groups then lands in shared memory exactly as the MMA reads a K-major operand without
// swizzle (8-row core matrices of 16 bytes).  Pixels at or past k become zero digits.
__global__ void __launch_bounds__(256) quantize_kernel(const float *__restrict__ f32, const int *__restrict__ bexp,
                                                       long k, long kp, long nch, long nblk,
                                                       int8_t *__restrict__ dig)
{
    const long b = blockIdx.x;
    const int s = blockIdx.y;
    const float sc = ldexpf(127.f, -bexp[(long)s * nblk + b]);
    const long kpg = kp / 16;
    for (long e = threadIdx.x; e < (LS_BLOCK / 16) * nch; e += blockDim.x) {
        const long g = e / nch, ch = e % nch;
        const long x0 = b * LS_BLOCK + g * 16;
        const float *src = f32 + ((long)s * nch + ch) * kp + x0;
        uint32_t w[3][4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            uint32_t a[4], bb[4], cc[4];
#pragma unroll
            for (int t = 0; t < 4; ++t) digits254(x0 + 4 * q + t < k ? src[4 * q + t] * sc : 0.f, a[t], bb[t], cc[t]);
            w[0][q] = __byte_perm(__byte_perm(a[0], a[1], 0x0040), __byte_perm(a[2], a[3], 0x0040), 0x5410);
            w[1][q] = __byte_perm(__byte_perm(bb[0], bb[1], 0x0040), __byte_perm(bb[2], bb[3], 0x0040), 0x5410);
            w[2][q] = __byte_perm(__byte_perm(cc[0], cc[1], 0x0040), __byte_perm(cc[2], cc[3], 0x0040), 0x5410);
        }
#pragma unroll
        for (int d = 0; d < 3; ++d)
            *reinterpret_cast<uint4 *>(dig + (((long)s * 3 + d) * kpg + x0 / 16) * nch * 16 + ch * 16) =
                make_uint4(w[d][0], w[d][1], w[d][2], w[d][3]);
    }
}

// Host: exact per-slot column counts and the largest number of ring rows in
// any column (for the shared-memory staging size).
void ring_shape(long ng, double lo, double hi, int *jcols, int *rows_max)
{
    long J = std::min<long>(ng / 3, (long)ceil(hi));
    long A = (long)ceil(hi) - 1;
    long ia_min = std::max(-A, -ng / 2 + 1), ia_max = std::min(A, ng / 2);
    int best = 0;
    for (long j = 0; j < J; ++j) {
        int n = 0;
        for (long ia = ia_min; ia <= ia_max; ++ia) {
            double uu = sqrt(1.0 * (double)(ia * ia + j * j));
            if (uu >= lo && uu < hi && uu > 0.0) ++n;
        }
        best = std::max(best, n);
    }
    *jcols = (int)std::max<long>(J, 0);
    *rows_max = best;
}

}  // namespace

int build_maps(amber_cuda_ctx *c, const MapJob &job)
{
    const long ng = job.ng;
    std::vector<int> jc(job.nslots);
    int jmax = 1, rows_max = 1;
    for (int s = 0; s < job.nslots; ++s) {
        int rm;
        ring_shape(ng, job.lo[s], job.hi[s], &jc[s], &rm);
        jmax = std::max(jmax, jc[s]);
        rows_max = std::max(rows_max, rm);
    }
    const double2 *tw;
    int rc = twiddle_table(c, ng, &tw);
    if (rc) return rc;
    size_t ybytes = sizeof(double2) * (size_t)job.nslots * ng * jmax * job.nch;
    if ((rc = ensure(c, c->y, ybytes, "map intermediate"))) return rc;
    double2 *Y = reinterpret_cast<double2 *>(c->y.p);

    // pass 1: choose channels per block so the staged column fits
    const size_t smem_cap = 200 * 1024;
    auto p1_smem = [&](int C) { return sizeof(double2) * ng + (sizeof(double2) * C + sizeof(int)) * rows_max; };
    int C1 = 32;
    while (C1 > 1 && p1_smem(C1) > smem_cap) C1 /= 2;
    if (p1_smem(C1) > smem_cap) return fail(c, AMBER_ERR_ARG, "ring too wide for the column stage (%d rows)", rows_max);
    const size_t s1 = p1_smem(C1);
    auto p2_smem = [&](int C) { return sizeof(double2) * ng + sizeof(double2) * C * jmax; };
    int C2 = 32;
    while (C2 > 1 && p2_smem(C2) > smem_cap) C2 /= 2;
    const size_t s2 = p2_smem(C2);
    // up to RING_META_MAX slots per launch pair, each launch's pointers offset to its first slot
    for (int sb = 0; sb < job.nslots; sb += RING_META_MAX) {
        const int ns = std::min(RING_META_MAX, job.nslots - sb);
        RingMeta meta;
        for (int i = 0; i < ns; ++i) {
            meta.lo[i] = job.lo[sb + i];
            meta.hi[i] = job.hi[sb + i];
            meta.jc[i] = jc[sb + i];
        }
        double2 *Ys = Y + (size_t)sb * ng * jmax * job.nch;
        const size_t so = (size_t)sb * job.nch * job.kp;
        double *of64 = job.out_f64 ? job.out_f64 + so : nullptr;
        uint16_t *ohi = job.out_hi ? job.out_hi + so : nullptr, *olo = job.out_lo ? job.out_lo + so : nullptr;
        float *of32 = job.out_f32 ? job.out_f32 + so : nullptr;
        dim3 g1(jmax, ns, (unsigned)((job.nch + C1 - 1) / C1));
#define LAUNCH_COLS(CC)                                                                                        \
    do {                                                                                                        \
        cudaFuncSetAttribute(ring_cols_kernel<CC>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)s1);        \
        ring_cols_kernel<CC><<<g1, kThreads, s1, c->stream>>>(job.src, job.src_complex ? 1 : 0, job.n1, job.nc, \
                                                               job.chan_base, job.nch, ng, meta, jmax, tw, Ys,  \
                                                               rows_max);                                        \
    } while (0)
        switch (C1) {
            case 32: LAUNCH_COLS(32); break;
            case 16: LAUNCH_COLS(16); break;
            case 8: LAUNCH_COLS(8); break;
            case 4: LAUNCH_COLS(4); break;
            case 2: LAUNCH_COLS(2); break;
            default: LAUNCH_COLS(1); break;
        }
#undef LAUNCH_COLS
        c->launches += 1;
        if ((rc = cuda_check(c, cudaGetLastError(), "ring_cols_kernel launch"))) return rc;

        dim3 g2((unsigned)ng, ns, (unsigned)((job.nch + C2 - 1) / C2));
#define LAUNCH_ROWS(CC)                                                                                        \
    do {                                                                                                        \
        cudaFuncSetAttribute(ring_rows_kernel<CC>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)s2);        \
        ring_rows_kernel<CC><<<g2, kThreads, s2, c->stream>>>(Ys, ng, jmax, meta, job.nch, tw, job.kp, of64, ohi, \
                                                               olo, of32, job.weight);                           \
    } while (0)
        switch (C2) {
            case 32: LAUNCH_ROWS(32); break;
            case 16: LAUNCH_ROWS(16); break;
            case 8: LAUNCH_ROWS(8); break;
            case 4: LAUNCH_ROWS(4); break;
            case 2: LAUNCH_ROWS(2); break;
            default: LAUNCH_ROWS(1); break;
        }
#undef LAUNCH_ROWS
        c->launches += 1;
        if ((rc = cuda_check(c, cudaGetLastError(), "ring_rows_kernel launch"))) return rc;
    }
    if (job.dig) {
        const long nblk = job.kp / LS_BLOCK;
        dim3 gq((unsigned)nblk, (unsigned)job.nslots);
        block_expo_kernel<<<gq, LS_BLOCK, 0, c->stream>>>(job.out_f32, ng * ng, job.kp, job.nch, nblk, job.bexp);
        quantize_kernel<<<gq, 256, 0, c->stream>>>(job.out_f32, job.bexp, ng * ng, job.kp, job.nch, nblk, job.dig);
        c->launches += 2;
        rc = cuda_check(c, cudaGetLastError(), "quantize_kernel launch");
    }
    return rc;
}

}  // namespace amber
