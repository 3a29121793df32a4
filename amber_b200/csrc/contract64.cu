// Plain FP64 triple-product lag accumulation (the reference loop of
// 4_fbe/amber.c:247-279 restated for the GPU in FP64), the deterministic lag
// reduction shared with the mixed-precision path, and the FP64 triple sum
// that gives calCR's normaliser (amber_funcs.c:451-457).
//
// For a triangle (r1, r2, r3) with maps D1, D2, D3 [channel][pixel] the
// reference sums, over every admissible channel triplet (p1, p2, p3) with
// |p2−p1|, |p3−p1| ≤ nc10, Σ_x D1[p1,x]·D2[p2,x]·D3[p3,x] into the lag cell
// (p2−p1+nc10, p3−p1+nc10).  For one anchor p1 that is the matrix
// T_p1 = (D2 ∘ D1[p1])·D3ᵀ restricted to the p1 window.  Each CTA here owns a
// 64 × 64 tile of one anchor's window over one pixel range: it stages
// D1[p1]·D2 and D3 for 16 pixels at a time in shared memory and accumulates a
// 4 × 4 register block per thread in FP64.  Channel multiplicities
// (flagging) weight the tile when it is written.  Tiles go to a partial
// buffer [anchor][k-split][lag2][lag3]; lag_reduce sums that buffer per lag
// cell in a fixed grouping and order with compensated (TwoSum) accumulators,
// so results are deterministic.
#include <algorithm>

#include "common.cuh"

namespace amber {

namespace {

constexpr int TT = 64;  // tile edge in channels
constexpr int KB = 16;  // pixels per shared-memory stage

__global__ void __launch_bounds__(256) contract64_kernel(const double *__restrict__ m1, const double *__restrict__ m2,
                                                          const double *__restrict__ m3, long k, long kp,
                                                          const int *__restrict__ anchors,
                                                          const int *__restrict__ weight, int nc, int nc10, int tiles,
                                                          long kchunk, int use_abs, double *__restrict__ partial)
{
    // rows padded by 2 doubles: the transposed stores hit 8 distinct bank pairs
    __shared__ __align__(16) double As[2][KB][TT + 2];
    __shared__ __align__(16) double Bs[2][KB][TT + 2];
    const int tid = threadIdx.x;
    const int a = blockIdx.y, ks = blockIdx.z, KS = gridDim.z;
    const int t2 = blockIdx.x / tiles, t3 = blockIdx.x % tiles;
    const int p1 = anchors[a];
    const int nclen = 2 * nc10 + 1;
    const int d2b = TT * t2, d3b = TT * t3;
    const int tx = tid & 15, ty = tid >> 4;
    double *out = partial + ((size_t)a * KS + ks) * nclen * nclen;

    // rows (p2) and columns (p3) this tile covers; -1 marks an empty row/col
    __shared__ int prow[TT], pcol[TT];
    __shared__ int any_row, any_col;
    if (tid == 0) { any_row = 0; any_col = 0; }
    __syncthreads();
    if (tid < TT) {
        int d = d2b + tid, p = p1 - nc10 + d;
        bool ok = d < nclen && p >= 0 && p < nc && weight[p] > 0;
        prow[tid] = ok ? p : -1;
        if (ok) atomicOr(&any_row, 1);
    } else if (tid < 2 * TT) {
        int d = d3b + tid - TT, p = p1 - nc10 + d;
        bool ok = d < nclen && p >= 0 && p < nc && weight[p] > 0;
        pcol[tid - TT] = ok ? p : -1;
        if (ok) atomicOr(&any_col, 1);
    }
    __syncthreads();

    double acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = 0.0;

    const long x0 = (long)ks * kchunk, x1 = min(k, x0 + kchunk);
    if (any_row && any_col && x0 < x1) {
        const double *c1 = m1 + (long)p1 * kp;
        // each thread loads 4 elements of A and 4 of B per stage
        auto load = [&](int buf, long xs) {
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                int e = tid + i * 256;
                int r = e / KB, xx = e % KB;
                long x = xs + xx;
                double va = 0.0, vb = 0.0;
                if (x < x1) {
                    int pr = prow[r], pc = pcol[r];
                    double s1 = c1[x];
                    if (pr >= 0) va = s1 * m2[(long)pr * kp + x];
                    if (pc >= 0) vb = m3[(long)pc * kp + x];
                    if (use_abs) {
                        va = fabs(va);
                        vb = fabs(vb);
                    }
                }
                As[buf][xx][r] = va;
                Bs[buf][xx][r] = vb;
            }
        };
        int buf = 0;
        load(0, x0);
        __syncthreads();
        for (long xs = x0; xs < x1; xs += KB) {
            if (xs + KB < x1) load(buf ^ 1, xs + KB);
#pragma unroll
            for (int xx = 0; xx < KB; ++xx) {
                double2 a01 = *reinterpret_cast<const double2 *>(&As[buf][xx][ty * 4]);
                double2 a23 = *reinterpret_cast<const double2 *>(&As[buf][xx][ty * 4 + 2]);
                double2 b01 = *reinterpret_cast<const double2 *>(&Bs[buf][xx][tx * 4]);
                double2 b23 = *reinterpret_cast<const double2 *>(&Bs[buf][xx][tx * 4 + 2]);
                double av[4] = {a01.x, a01.y, a23.x, a23.y};
                double bv[4] = {b01.x, b01.y, b23.x, b23.y};
#pragma unroll
                for (int i = 0; i < 4; ++i)
#pragma unroll
                    for (int j = 0; j < 4; ++j) acc[i][j] = fma(av[i], bv[j], acc[i][j]);
            }
            __syncthreads();
            buf ^= 1;
        }
    }
    const double w1 = (double)weight[p1];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        int r = ty * 4 + i, d2 = d2b + r;
        if (d2 >= nclen) continue;
        int pr = prow[r];
        double wr = pr >= 0 ? w1 * (double)weight[pr] : 0.0;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            int cc = tx * 4 + j, d3 = d3b + cc;
            if (d3 >= nclen) continue;
            int pc = pcol[cc];
            double wc = pc >= 0 ? (double)weight[pc] : 0.0;
            out[(long)d2 * nclen + d3] = acc[i][j] * wr * wc;
        }
    }
}

// Pass 1 of the lag reduction: unit group g of cell d sums partial[u][d] for
// u in [g·U/G, (g+1)·U/G) with a TwoSum-compensated accumulator, in order, and
// leaves (sum, compensation) in part[g][d] / part[G + g][d].
__global__ void lag_reduce_groups(const double *__restrict__ partial, long nunits, long ncsize,
                                  double *__restrict__ part)
{
    const long d = (long)blockIdx.x * blockDim.x + threadIdx.x;
    const int g = blockIdx.y, G = gridDim.y;
    if (d >= ncsize) return;
    const long u0 = nunits * g / G, u1 = nunits * (g + 1) / G;
    double s = 0.0, comp = 0.0;
    for (long u = u0; u < u1; ++u) {
        const double v = partial[u * ncsize + d];
        const double t = s + v;
        const double bp = t - s;
        comp += (s - (t - bp)) + (v - bp);
        s = t;
    }
    part[(long)g * ncsize + d] = s;
    part[(long)(G + g) * ncsize + d] = comp;
}

// Pass 2: lag[d] = the groups' sums added in group order (TwoSum again) plus all compensations;
// with accumulate, the sum starts from the lag array's current value (a job split into anchor groups).
__global__ void lag_reduce_final(const double *__restrict__ part, int G, long ncsize, int accumulate,
                                 double *__restrict__ lag)
{
    const long d = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= ncsize) return;
    double s = accumulate ? lag[d] : 0.0, comp = 0.0;
    for (int g = 0; g < G; ++g) {
        const double v = part[(long)g * ncsize + d];
        const double t = s + v;
        const double bp = t - s;
        comp += (s - (t - bp)) + (v - bp);
        s = t;
        comp += part[(long)(G + g) * ncsize + d];
    }
    lag[d] = s + comp;
}

// calCR's Num for every closed triangle at once (amber_funcs.c:451-457):
// Num_t = Σ_x II_r1(x)·II_r2(x)·II_r3(x) over the N1² mask maps.  CTA (chunk,
// t) sums a fixed grid-stride slice of pixels; one thread per triangle then
// adds the slices in order with compensation.  The grouping depends only on
// the map size, so every triangle's Num is deterministic.
constexpr int kNumChunks = 256;

__global__ void triple_sum_partial(const double *__restrict__ maps, long n, const int *__restrict__ tri,
                                   double *__restrict__ part)
{
    __shared__ double red[256];
    const int t = blockIdx.y;
    const double *a = maps + (long)tri[3 * t] * n, *b = maps + (long)tri[3 * t + 1] * n,
                 *c = maps + (long)tri[3 * t + 2] * n;
    double s = 0.0;
    for (long i = (long)blockIdx.x * 256 + threadIdx.x; i < n; i += (long)gridDim.x * 256) s += a[i] * b[i] * c[i];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[(long)t * gridDim.x + blockIdx.x] = red[0];
}

__global__ void sum_fixed(const double *__restrict__ part, int n, int ntri, double *__restrict__ out)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ntri) return;
    const double *p = part + (long)t * n;
    double s = 0.0, comp = 0.0;
    for (int i = 0; i < n; ++i) {
        double u = s + p[i];
        double bp = u - s;
        comp += (s - (u - bp)) + (p[i] - bp);
        s = u;
    }
    out[t] = s + comp;
}

}  // namespace

int lag_reduce(amber_cuda_ctx *c, const double *partial, long nunits, long ncsize, double *lag, bool accumulate)
{
    // enough unit groups to give every SM several blocks; the grouping depends only on
    // (nunits, ncsize, SM count), so the result is deterministic
    const long bx = (ncsize + 255) / 256;
    const long G = std::max<long>(1, std::min<long>({64L, (8L * c->num_sms + bx - 1) / bx, (nunits + 3) / 4}));
    int rc = ensure(c, c->lagred, sizeof(double) * 2 * (size_t)G * ncsize, "lag reduction scratch");
    if (rc) return rc;
    double *part = (double *)c->lagred.p;
    phase_begin(c, 2);
    lag_reduce_groups<<<dim3((unsigned)bx, (unsigned)G), 256, 0, c->stream>>>(partial, nunits, ncsize, part);
    lag_reduce_final<<<(unsigned)bx, 256, 0, c->stream>>>(part, (int)G, ncsize, accumulate ? 1 : 0, lag);
    phase_end(c);
    c->launches += 2;
    return cuda_check(c, cudaGetLastError(), "lag reduction launch");
}

int contract_fp64(amber_cuda_ctx *c, const double *m1, const double *m2, const double *m3, long k, long kp,
                  double *lag_out)
{
    const int nc10 = c->nc10;
    const int nclen = 2 * nc10 + 1;
    const long ncsize = (long)nclen * nclen;
    const int nA = (int)c->anchors.size();
    if (nA == 0) return cuda_check(c, cudaMemsetAsync(lag_out, 0, sizeof(double) * ncsize, c->stream), "zero lag");
    const int tiles = (nclen + TT - 1) / TT;
    long blocks = (long)tiles * tiles * nA;
    long want = 4L * c->num_sms;
    int KS = (int)std::max<long>(1, std::min<long>((want + blocks - 1) / blocks, (k + 1023) / 1024));
    long kchunk = ((k + KS - 1) / KS + KB - 1) / KB * KB;
    KS = (int)((k + kchunk - 1) / kchunk);
    if (KS < 1) KS = 1;
    size_t pbytes = sizeof(double) * (size_t)nA * KS * ncsize;
    int rc = ensure(c, c->partial, pbytes, "partial lag tiles");
    if (rc) return rc;
    dim3 grid((unsigned)(tiles * tiles), (unsigned)nA, (unsigned)KS);
    phase_begin(c, 1);
    contract64_kernel<<<grid, 256, 0, c->stream>>>(m1, m2, m3, k, kp, (const int *)c->d_anchors.p,
                                                   (const int *)c->d_weight.p, (int)c->nc, nc10, tiles, kchunk,
                                                   c->fp64_abs ? 1 : 0, (double *)c->partial.p);
    phase_end(c);
    c->launches += 1;
    c->contractions += 1;
    if ((rc = cuda_check(c, cudaGetLastError(), "contract64_kernel launch"))) return rc;
    return lag_reduce(c, (const double *)c->partial.p, (long)nA * KS, ncsize, lag_out);
}

int triple_sums(amber_cuda_ctx *c, const double *maps, long n, const std::vector<int> &tri, double *out)
{
    const int ntri = (int)tri.size() / 3;
    if (ntri == 0) return AMBER_OK;
    // partial sums [ntri][chunks] (doubles), then the triangle list (ints)
    const size_t part_b = sizeof(double) * (size_t)ntri * kNumChunks;
    int rc = ensure(c, c->misc, part_b + sizeof(int) * tri.size(), "calCR partial sums");
    if (rc) return rc;
    double *part = (double *)c->misc.p;
    int *d_tri = (int *)((char *)c->misc.p + part_b);
    if ((rc = cuda_check(c, cudaMemcpyAsync(d_tri, tri.data(), sizeof(int) * tri.size(), cudaMemcpyHostToDevice,
                                            c->stream), "calCR triangles")))
        return rc;
    for (int t0 = 0; t0 < ntri; t0 += 65535) {  // grid y limit
        const int nt = std::min(65535, ntri - t0);
        triple_sum_partial<<<dim3(kNumChunks, nt), 256, 0, c->stream>>>(maps, n, d_tri + 3 * t0,
                                                                         part + (size_t)t0 * kNumChunks);
        c->launches += 1;
    }
    sum_fixed<<<(ntri + 127) / 128, 128, 0, c->stream>>>(part, kNumChunks, ntri, out);
    c->launches += 1;
    return cuda_check(c, cudaGetLastError(), "calCR sums launch");
}

}  // namespace amber
