// Plain FP64 triple-product lag accumulation (the reference loop of
// 4_fbe/amber.c:247-279 / amber_v2.c:243-270 restated for the GPU in FP64), the
// per-anchor lag reduction still used by the split-BF16 comparison path, and the
// FP64 triple sum that gives calCR's normaliser (amber_funcs.c:451-457).
//
// The contraction is the lag-space GEMM of lagspace.cuh: per unit (a tile pair,
// an anchor block and a run of pixel blocks) one CTA of 8 warps holds a 128 × 128
// FP64 accumulator tile in registers, 16 warps each holding a 32 × 32 block as
// 2 × 4 fragments of the FP64 tensor-core MMA mma.sync m16n8k8 (1024 FMAs per
// instruction; the m8n8k4 shape reaches only about half the FP64 tensor rate).  Per stage of 16
// pixels the CTA copies the channel rows its anchors touch — w·D1 of the anchor
// block, w·D3 and w·D2 of the spans their windows cover — into shared memory
// once (transposed, [pixel][channel]); then, for every anchor group, it forms
// the A operand D1[p1]·D3[p1 − nc10 + Δ3] (one multiply per element, into one
// of two buffers) and runs two k = 8 steps of 8 MMAs per warp, reading B
// straight from the staged D2 rows at the group's window offset.  Row strides
// of the A buffer and the D2 stage are ≡ 4 (mod 16) doubles, so a fragment
// load (4 pixels × 8 rows) hits 16 distinct bank pairs per half warp.  The sums
// stay in registers until the unit's end; its partial tile is then summed per
// lag cell by ls_reduce in a fixed order.
#include <algorithm>

#include "lagspace.cuh"

namespace amber {

namespace {

constexpr int F_KX = 16;   // pixels per stage
constexpr int F_NT = 512;  // threads per CTA (16 warps: 4 along rows × 4 along columns)

struct F64Desc {
    const double *m1, *m2, *m3;  // ring maps of r1, r2, r3 [nc][kp]
    const int *weight;           // channel multiplicities [nc]
    const int *groups;           // anchor groups, concatenated over anchor blocks
    const int *group_off;        // [nab + 1]
    long k, kp;
    int nc, nc10, nclen, ks, AB;
};

constexpr int F_S1 = LS_SPAN + 1;  // D1 rows of an anchor block (≤ 256)
constexpr int F_S3 = LS_SPAN + 1;  // D3 span
constexpr int F_S2 = 260;          // D2 span (≤ 256), ≡ 4 mod 16
constexpr int F_SA = 132;          // A buffer rows (128), ≡ 4 mod 16
constexpr size_t F_SMEM = sizeof(double) * ((size_t)F_KX * (F_S1 + F_S3 + F_S2) + 2 * F_KX * F_SA);

// D(16×8) += A(16×8) · B(8×8), FP64.  Fragments (g = lane / 4, t = lane % 4): A {(g, t), (g+8, t),
// (g, t+4), (g+8, t+4)}, B {(t, g), (t+4, g)}, C {(g, 2t), (g, 2t+1), (g+8, 2t), (g+8, 2t+1)}.
__device__ __forceinline__ void dmma(double (&c)[4], const double (&a)[4], const double (&b)[2])
{
    asm volatile("mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, "
                 "{%0, %1, %2, %3};"
                 : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
                 : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b[0]), "d"(b[1]));
}

__global__ void __launch_bounds__(F_NT, 1) ls_fp64_kernel(const F64Desc *__restrict__ jobs,
                                                          const LsUnit *__restrict__ units,
                                                          double *__restrict__ partial, int use_abs)
{
    extern __shared__ __align__(16) double sm[];
    double *st1 = sm;                    // [F_KX][F_S1]  w·D1 of the anchor block
    double *st3 = st1 + F_KX * F_S1;     // [F_KX][F_S3]  w·D3 of the span
    double *st2 = st3 + F_KX * F_S3;     // [F_KX][F_S2]  w·D2 of the span
    double *As = st2 + F_KX * F_S2;      // [2][F_KX][F_SA] the formed A operand

    const LsUnit u = units[blockIdx.x];
    const F64Desc j = jobs[u.job];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int wm = warp >> 2, wn = warp & 3;   // warp tile: rows 32·wm .., columns 32·wn ..
    const int gq = lane >> 2, tq = lane & 3;   // fragment row / column group, k index
    const int ks = j.ks, nclen = j.nclen, nc = j.nc;
    const int c0 = u.ab * j.AB, c1 = min(nc, c0 + j.AB), nab1 = c1 - c0;
    const int mrows = ks > 1 ? ks * nclen : min(LS_ROWS, nclen - LS_ROWS * u.t3);
    const int ncols = ks > 1 ? nclen + ks - 1 : min(LS_ROWS, nclen - LS_ROWS * u.t2);
    const int row0_3 = c0 - j.nc10 + (ks > 1 ? 0 : LS_ROWS * u.t3);  // channel of staged D3 row 0
    const int row0_2 = c0 - j.nc10 + (ks > 1 ? 0 : LS_ROWS * u.t2);  // channel of staged D2 row 0
    const int span3 = nab1 + (ks > 1 ? nclen : mrows) - 1;
    const int span2 = nab1 + ncols - 1;
    const int g0 = j.group_off[u.ab], g1 = j.group_off[u.ab + 1];
    // the A row this thread forms (pixels tid/128 + 4i), its anchor slot and lag
    const int ar = tid & (LS_ROWS - 1), ax = tid >> 7;
    const int aslot = ks > 1 ? ar / nclen : 0, ad3 = ks > 1 ? ar % nclen : ar;
    const bool arow = ar < mrows;

    double acc[2][4][4];
#pragma unroll
    for (int mt = 0; mt < 2; ++mt)
#pragma unroll
        for (int nt = 0; nt < 4; ++nt)
#pragma unroll
            for (int e = 0; e < 4; ++e) acc[mt][nt][e] = 0.0;

    // stage rows [0, n) of map m starting at channel ch0, weighted, into st[x][row]
    auto stage = [&](double *st, int stride, const double *m, int ch0, int n, long x0) {
        for (int e = tid; e < n * F_KX; e += F_NT) {
            const int row = e / F_KX, xx = e % F_KX;
            const int ch = ch0 + row;
            const long x = x0 + xx;
            double v = 0.0;
            if (ch >= 0 && ch < nc && x < j.k) {
                const int w = j.weight[ch];
                if (w) {
                    v = (double)w * m[(long)ch * j.kp + x];
                    if (use_abs) v = fabs(v);
                }
            }
            st[xx * stride + row] = v;
        }
    };

    int buf = 0;
    for (long b = u.b0; b < u.b1; ++b) {
        const long xb = b * LS_BLOCK;
        for (long x0 = xb; x0 < min(j.k, xb + LS_BLOCK); x0 += F_KX) {
            __syncthreads();  // every reader of the previous stage is done
            stage(st1, F_S1, j.m1, c0, nab1, x0);
            stage(st3, F_S3, j.m3, row0_3, span3, x0);
            stage(st2, F_S2, j.m2, row0_2, span2, x0);
            __syncthreads();
            for (int g = g0; g < g1; ++g) {
                const int pb = j.groups[g];
                // A[x][r] = D1[p1, x] · D3[p1 − nc10 + Δ3, x] for slot a and lag Δ3 of row r.  A[buf] was
                // last read two groups ago, before the barrier that ended the previous formation.
                double *A = As + buf * (F_KX * F_SA);
                const int p1 = pb + aslot;
                const bool ok = arow && p1 < c1;
#pragma unroll
                for (int i = 0; i < F_KX / 4; ++i) {
                    const int xx = ax + 4 * i;
                    A[xx * F_SA + ar] = ok ? st1[xx * F_S1 + (p1 - c0)] * st3[xx * F_S3 + (p1 - c0) + ad3] : 0.0;
                }
                __syncthreads();
                const double *Aw = A + 32 * wm + gq;
                const double *Bw = st2 + (pb - c0) + 32 * wn + gq;
#pragma unroll
                for (int k8 = 0; k8 < F_KX / 8; ++k8) {
                    const int xx = 8 * k8 + tq;
                    double a[2][4], bv[4][2];
#pragma unroll
                    for (int mt = 0; mt < 2; ++mt) {
                        a[mt][0] = Aw[xx * F_SA + 16 * mt];
                        a[mt][1] = Aw[xx * F_SA + 16 * mt + 8];
                        a[mt][2] = Aw[(xx + 4) * F_SA + 16 * mt];
                        a[mt][3] = Aw[(xx + 4) * F_SA + 16 * mt + 8];
                    }
#pragma unroll
                    for (int nt = 0; nt < 4; ++nt) {
                        bv[nt][0] = Bw[xx * F_S2 + 8 * nt];
                        bv[nt][1] = Bw[(xx + 4) * F_S2 + 8 * nt];
                    }
#pragma unroll
                    for (int mt = 0; mt < 2; ++mt)
#pragma unroll
                        for (int nt = 0; nt < 4; ++nt) dmma(acc[mt][nt], a[mt], bv[nt]);
                }
                buf ^= 1;
            }
        }
    }
    // the unit's partial tile [column][row]; slot a of a packed tile lands at lag column c − a
    double *out = partial + u.tile * (long)(LS_ROWS * LS_ROWS);
    const int lagc = ks > 1 ? nclen : ncols;
#pragma unroll
    for (int mt = 0; mt < 2; ++mt)
#pragma unroll
        for (int hr = 0; hr < 2; ++hr) {
            const int r = 32 * wm + 16 * mt + 8 * hr + gq;
            if (r >= mrows) continue;
            const int a = ks > 1 ? r / nclen : 0;
#pragma unroll
            for (int nt = 0; nt < 4; ++nt)
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const int col = 32 * wn + 8 * nt + 2 * tq + h - a;
                    if (col >= 0 && col < lagc) out[(long)col * LS_ROWS + r] = acc[mt][nt][2 * hr + h];
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

int contract_fp64_jobs(amber_cuda_ctx *c, const std::vector<F64Job> &jobs)
{
    int rc;
    if (jobs.empty()) return AMBER_OK;
    const int nclen = 2 * c->nc10 + 1;
    const long ncsize = (long)nclen * nclen;
    const int nA = (int)c->anchors.size();
    if (nA == 0) {
        for (const F64Job &jb : jobs)
            if ((rc = cuda_check(c, cudaMemsetAsync(jb.lag_out, 0, sizeof(double) * ncsize, c->stream), "zero lag")))
                return rc;
        return AMBER_OK;
    }
    constexpr size_t TILE_B = sizeof(double) * LS_ROWS * LS_ROWS;
    const size_t pcap = std::max<size_t>((size_t)256 << 20, contract_partial_cap(c));
    size_t j0 = 0;
    while (j0 < jobs.size()) {
        // plan as many jobs as their partial tiles allow in one launch
        std::vector<LsJobPlan> plans;
        long tiles = 0;
        size_t j1 = j0;
        for (; j1 < jobs.size(); ++j1) {
            LsJobPlan p;
            ls_plan_job(p, (int)c->nc, c->nc10, jobs[j1].k, c->weight, c->num_sms, 8, ls_force_bpu(c->chunk_px));
            if (j1 > j0 && (size_t)(tiles + p.s.units()) * TILE_B > pcap) break;
            p.unit_base = tiles;
            tiles += p.s.units();
            plans.push_back(std::move(p));
        }
        std::vector<LsUnit> units;
        for (size_t i = 0; i < plans.size(); ++i) ls_units(plans[i], (int)i, units);
        // largest units first, so that the small ones fill the tail of the launch
        std::stable_sort(units.begin(), units.end(), [](const LsUnit &a, const LsUnit &b) { return a.work > b.work; });
        // device: descriptors, units and anchor groups, through the pinned staging area
        size_t ngroups = 0, noff = 0;
        for (const LsJobPlan &p : plans) {
            ngroups += p.groups.size();
            noff += p.group_off.size();
        }
        const size_t desc_b = sizeof(F64Desc) * plans.size(), unit_b = sizeof(LsUnit) * units.size();
        const size_t off_u = (desc_b + 255) / 256 * 256, off_g = off_u + (unit_b + 255) / 256 * 256;
        const size_t off_o = off_g + (sizeof(int) * ngroups + 255) / 256 * 256;
        const size_t stage_b = off_o + sizeof(int) * noff;
        if ((rc = ensure(c, c->partial, (size_t)tiles * TILE_B, "partial lag tiles"))) return rc;
        if ((rc = ensure(c, c->jobdesc, stage_b, "job list"))) return rc;
        if ((rc = cuda_check(c, cudaStreamSynchronize(c->stream), "job staging"))) return rc;
        if (c->stage_bytes < stage_b) {
            if (c->stage) cudaFreeHost(c->stage);
            c->stage = nullptr;
            c->stage_bytes = 0;
            if ((rc = cuda_check(c, cudaHostAlloc(&c->stage, stage_b, cudaHostAllocDefault), "job staging"))) return rc;
            c->stage_bytes = stage_b;
        }
        char *h = (char *)c->stage, *d = (char *)c->jobdesc.p;
        F64Desc *hd = (F64Desc *)h;
        int *hg = (int *)(h + off_g), *ho = (int *)(h + off_o);
        std::vector<LsReduceJob> red;
        size_t gpos = 0, opos = 0;
        for (size_t i = 0; i < plans.size(); ++i) {
            const F64Job &jb = jobs[j0 + i];
            const LsJobPlan &p = plans[i];
            F64Desc &x = hd[i];
            x.m1 = jb.m1; x.m2 = jb.m2; x.m3 = jb.m3;
            x.weight = (const int *)c->d_weight.p;
            x.groups = (const int *)(d + off_g) + gpos;
            x.group_off = (const int *)(d + off_o) + opos;
            x.k = jb.k; x.kp = jb.kp;
            x.nc = (int)c->nc; x.nc10 = c->nc10; x.nclen = nclen; x.ks = p.s.k; x.AB = p.s.AB;
            std::copy(p.groups.begin(), p.groups.end(), hg + gpos);
            for (size_t q = 0; q < p.group_off.size(); ++q) ho[opos + q] = p.group_off[q];
            gpos += p.groups.size();
            opos += p.group_off.size();
            red.push_back(LsReduceJob{(const double *)c->partial.p + p.unit_base * LS_ROWS * LS_ROWS, jb.lag_out, nclen,
                                      p.s.k, p.s.T, p.s.nab, p.s.V});
        }
        std::copy(units.begin(), units.end(), (LsUnit *)(h + off_u));
        if ((rc = cuda_check(c, cudaMemcpyAsync(d, h, stage_b, cudaMemcpyHostToDevice, c->stream), "job list upload")))
            return rc;
        cudaFuncSetAttribute(ls_fp64_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)F_SMEM);
        phase_begin(c, 1);
        for (size_t u0 = 0; u0 < units.size(); u0 += 1u << 30) {
            const unsigned n = (unsigned)std::min<size_t>(units.size() - u0, 1u << 30);
            ls_fp64_kernel<<<n, F_NT, F_SMEM, c->stream>>>((const F64Desc *)d, (const LsUnit *)(d + off_u) + u0,
                                                          (double *)c->partial.p, c->fp64_abs ? 1 : 0);
            c->launches += 1;
            c->contractions += 1;
        }
        phase_end(c);
        if ((rc = cuda_check(c, cudaGetLastError(), "ls_fp64_kernel launch"))) return rc;
        if ((rc = ls_reduce(c, red))) return rc;
        j0 = j1;
    }
    return AMBER_OK;
}

int contract_fp64(amber_cuda_ctx *c, const double *m1, const double *m2, const double *m3, long k, long kp,
                  double *lag_out)
{
    return contract_fp64_jobs(c, {F64Job{m1, m2, m3, k, kp, lag_out}});
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
