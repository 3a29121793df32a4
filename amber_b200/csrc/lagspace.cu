// Lag-space contraction plan and the deterministic reduction of the units' partial
// tiles (see lagspace.cuh).
#include <algorithm>

#include "lagspace.cuh"

namespace amber {

namespace {

int round16(int n) { return (n + 15) / 16 * 16; }

// lag[Δ2·nclen + Δ3] = Σ over the job's units (anchor blocks, then units of the block, then
// slots) of the partial tiles, TwoSum-compensated, in that fixed order.  Partial tiles are
// [column][row] so that consecutive Δ3 read consecutive doubles.
__global__ void ls_reduce_kernel(const LsReduceJob *__restrict__ jobs)
{
    const LsReduceJob j = jobs[blockIdx.y];
    const long ncsize = (long)j.nclen * j.nclen;
    const long d = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= ncsize) return;
    const int d2 = (int)(d / j.nclen), d3 = (int)(d % j.nclen);
    constexpr long TILE = (long)LS_ROWS * LS_ROWS;
    double s = 0.0, comp = 0.0;
    auto add = [&](double v) {
        const double t = s + v, bp = t - s;
        comp += (s - (t - bp)) + (v - bp);
        s = t;
    };
    if (j.k > 1) {
        for (int u = 0; u < j.nab * j.V; ++u) {
            const double *p = j.partial + u * TILE + (long)d2 * LS_ROWS;
            for (int a = 0; a < j.k; ++a) add(p[a * j.nclen + d3]);
        }
    } else {
        const int t2 = d2 / LS_ROWS, c = d2 % LS_ROWS, t3 = d3 / LS_ROWS, r = d3 % LS_ROWS;
        const long u0 = (long)(t3 * j.T + t2) * j.nab * j.V;
        for (int u = 0; u < j.nab * j.V; ++u) add(j.partial[(u0 + u) * TILE + (long)c * LS_ROWS + r]);
    }
    j.lag[d] = s + comp;
}

}  // namespace

int LsShape::rows(int t3) const { return k > 1 ? k * nclen : std::min(LS_ROWS, nclen - LS_ROWS * t3); }
int LsShape::cols(int t2) const
{
    return k > 1 ? round16(nclen + k - 1) : round16(std::min(LS_ROWS, nclen - LS_ROWS * t2));
}
int LsShape::lag_cols(int t2) const { return k > 1 ? nclen : std::min(LS_ROWS, nclen - LS_ROWS * t2); }

LsShape ls_shape(int nc, int nc10, long k_px, int sms, long min_bpu, long force_bpu)
{
    LsShape s;
    s.nc = nc;
    s.nc10 = nc10;
    s.nclen = 2 * nc10 + 1;
    s.k = s.nclen <= LS_ROWS / 2 ? LS_ROWS / s.nclen : 1;
    s.T = s.k > 1 ? 1 : (s.nclen + LS_ROWS - 1) / LS_ROWS;
    // Staged rows of one unit: D3 spans AB + rows − 1 channels and the D2 window AB + N − 1;
    // both must fit one TMA box (LS_SPAN rows).  An anchor block also holds at most 128 anchor
    // groups, so that 128 groups × LS_BLOCK pixels of int8 digit products cannot overflow the
    // int32 accumulators (|class sum| ≤ 3·127² per term, 32768 terms < 2^31 / 48387).
    const int span_extra = std::max(s.rows(0), s.cols(0)) - 1;
    s.AB = std::max(1, std::min({nc, LS_SPAN - span_extra, LS_ROWS * s.k}));
    s.nab = (nc + s.AB - 1) / s.AB;
    s.nblk = std::max<long>(1, (k_px + LS_BLOCK - 1) / LS_BLOCK);
    // Units: about six per SM for a large job, so the last wave is short; at least min_bpu blocks
    // each (a unit's partial tile costs a write and a read of 128 KB).
    const long combos = (long)s.T * s.T * s.nab;
    const long target = 6L * std::max(1, sms);
    s.bpu = force_bpu > 0 ? std::min(s.nblk, force_bpu)
                          : std::min(s.nblk, std::max(min_bpu, (s.nblk * combos + target - 1) / target));
    s.V = (int)((s.nblk + s.bpu - 1) / s.bpu);
    return s;
}

void ls_plan_job(LsJobPlan &p, int nc, int nc10, long k_px, const std::vector<int> &weight, int sms, long min_bpu,
                 long force_bpu)
{
    p.s = ls_shape(nc, nc10, k_px, sms, min_bpu, force_bpu);
    p.groups.clear();
    p.group_off.assign(1, 0);
    for (int ab = 0; ab < p.s.nab; ++ab) {
        const int c0 = ab * p.s.AB, c1 = std::min(nc, c0 + p.s.AB);
        for (int pb = c0; pb < c1; pb += p.s.k) {
            bool any = false;
            for (int a = 0; a < p.s.k && pb + a < c1; ++a) any = any || weight[pb + a] > 0;
            if (any) p.groups.push_back(pb);
        }
        p.group_off.push_back((int)p.groups.size());
    }
}

void ls_units(const LsJobPlan &p, int job, std::vector<LsUnit> &out)
{
    const LsShape &s = p.s;
    long local = 0;
    for (int t3 = 0; t3 < s.T; ++t3)
        for (int t2 = 0; t2 < s.T; ++t2)
            for (int ab = 0; ab < s.nab; ++ab)
                for (int v = 0; v < s.V; ++v) {
                    LsUnit u;
                    u.job = job;
                    u.t3 = (short)t3;
                    u.t2 = (short)t2;
                    u.ab = ab;
                    u.b0 = (int)(v * s.bpu);
                    u.b1 = (int)std::min(s.nblk, (v + 1) * s.bpu);
                    u.tile = p.unit_base + local++;
                    u.work = (double)(u.b1 - u.b0) * (p.group_off[ab + 1] - p.group_off[ab]);
                    out.push_back(u);
                }
}

int ls_reduce(amber_cuda_ctx *c, const std::vector<LsReduceJob> &jobs)
{
    if (jobs.empty()) return AMBER_OK;
    int rc;
    const size_t bytes = sizeof(LsReduceJob) * jobs.size();
    if ((rc = ensure(c, c->lsred, bytes, "lag reduction job list"))) return rc;
    if ((rc = cuda_check(c, cudaMemcpyAsync(c->lsred.p, jobs.data(), bytes, cudaMemcpyHostToDevice, c->stream),
                         "lag reduction job list")))
        return rc;
    long cells = 0;
    for (const LsReduceJob &j : jobs) cells = std::max<long>(cells, (long)j.nclen * j.nclen);
    phase_begin(c, 2);
    for (size_t j0 = 0; j0 < jobs.size(); j0 += 65535) {
        const unsigned nj = (unsigned)std::min<size_t>(65535, jobs.size() - j0);
        ls_reduce_kernel<<<dim3((unsigned)((cells + 255) / 256), nj), 256, 0, c->stream>>>(
            (const LsReduceJob *)c->lsred.p + j0);
        c->launches += 1;
    }
    phase_end(c);
    return cuda_check(c, cudaGetLastError(), "ls_reduce launch");
}

}  // namespace amber
