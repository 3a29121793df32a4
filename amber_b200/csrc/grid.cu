// Visibility gridding as a sort-by-cell gather (replaces group_loop_gridding
// and group_loop_gridding_without_flag, 3_vcg/tgefuncs.c:377-505, 511-621).
//
// The reference walks the records in order and adds each one's RR channels
// into its nearest cell.  The FP64 sums of float inputs are order-dependent,
// so to be bit-identical on the GPU every cell must add its records in record
// order:
//   1. cell_kernel: per record, the same float arithmetic as the reference
//      (u1 = ν0·signv·u, |U| = √(float(u1²+v1²)) ≤ Umax, ii = round(u1/dU)
//      wrapped, jj = round(v1/dU)), with explicit _rn intrinsics so nothing is
//      contracted into an FMA; records outside Umax get key = ncell;
//   2. a stable radix sort of (cell, record) pairs (CUB; stable keeps record
//      order inside a cell);
//   3. segment_kernel marks each cell's [begin, end) in the sorted order;
//   4. sum_kernel: one thread per (cell, channel) adds that cell's records in
//      sorted (= record) order in FP64 — deterministic and identical to the
//      sequential loop.  Lanes walk channels, so loads of the channel-major
//      record payload and stores of the channel-innermost grid coalesce.
#include <cub/cub.cuh>

#include <algorithm>

#include "common.cuh"

namespace amber {

namespace {

__global__ void cell_kernel(const float *__restrict__ randpar, long npar, long G, float nu0, double dU, double Umax,
                            long NN, long ncell, unsigned *__restrict__ key, unsigned *__restrict__ val,
                            int *__restrict__ bad)
{
    long g = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= G) return;
    const float *rp = randpar + g * npar;
    float signv = (rp[1] < 0.f) ? -1.f : 1.f;             // tgefuncs.c:400
    float u1 = __fmul_rn(__fmul_rn(nu0, signv), rp[0]);   // 402
    float v1 = __fmul_rn(__fmul_rn(nu0, signv), rp[1]);   // 403
    float s = __fadd_rn(__fmul_rn(u1, u1), __fmul_rn(v1, v1));
    double Uval = __dsqrt_rn((double)s);                  // 405
    unsigned k = (unsigned)ncell;
    if (Uval <= Umax) {
        long ii = (long)(int)round(__ddiv_rn((double)u1, dU));  // 466-468
        ii = (ii < 0) ? NN + ii : ii;
        long jj = (long)(int)round(__ddiv_rn((double)v1, dU));
        const long H = NN / 2 + 1;
        if (ii < 0 || ii >= NN || jj < 0 || jj >= H) {
            atomicExch(bad, 1);
        } else {
            k = (unsigned)(ii * H + jj);  // 483
        }
    }
    key[g] = k;
    val[g] = (unsigned)g;
}

__global__ void segment_kernel(const unsigned *__restrict__ key, long G, long ncell, unsigned *__restrict__ begin,
                               unsigned *__restrict__ end)
{
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= G) return;
    unsigned k = key[i];
    if (k >= (unsigned)ncell) return;
    if (i == 0 || key[i - 1] != k) begin[k] = (unsigned)i;
    if (i == G - 1 || key[i + 1] != k) end[k] = (unsigned)i + 1;
}

__global__ void sum_kernel(const unsigned *__restrict__ begin, const unsigned *__restrict__ end,
                           const unsigned *__restrict__ order, const float *__restrict__ randpar, long npar,
                           const float *__restrict__ data, long nc, long nstokes, int flag_key, long ncell,
                           double *__restrict__ re_im, double *__restrict__ ntig)
{
    long cell = blockIdx.x;
    long ch = (long)blockIdx.y * blockDim.x + threadIdx.x;
    if (cell >= ncell || ch >= nc) return;
    unsigned b = begin[cell], e = end[cell];
    double sr = 0.0, si = 0.0, sn = 0.0;
    for (unsigned i = b; i < e; ++i) {
        long g = order[i];
        float signv = (randpar[g * npar + 1] < 0.f) ? -1.f : 1.f;
        const float *rr = data + ((g * nc + ch) * nstokes) * 3;  // Stokes 0 = RR
        if (flag_key == 1) {
            if (rr[2] > 0.f) {  // tgefuncs.c:418-431
                sr += (double)rr[0];
                si += (double)__fmul_rn(signv, rr[1]);
                sn += 1.0;
            }
        } else {  // 564-566, 608
            sr += (double)rr[0];
            si += (double)__fmul_rn(signv, rr[1]);
            sn += 1.0;
        }
    }
    long o = cell * nc + ch;
    re_im[2 * o] = sr;
    re_im[2 * o + 1] = si;
    ntig[o] = sn;
}

// Channel collapse (tgefuncs.c:816-838): output channel col of a cell is the sum of input
// channels col·n .. col·n + n − 1, added in that order from 0.0 as the reference's loop does.
__global__ void collapse_kernel(const double *__restrict__ re_im, const double *__restrict__ ntig, long ncell, long nc,
                                long n, long ncoll, double *__restrict__ re_im_c, double *__restrict__ ntig_c)
{
    const long total = ncell * ncoll;
    for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x) {
        const long cell = e / ncoll, col = e % ncoll;
        const long base = cell * nc + col * n;
        double sr = 0.0, si = 0.0, sn = 0.0;
        for (long k = 0; k < n; ++k) {
            sr = __dadd_rn(sr, re_im[2 * (base + k)]);
            si = __dadd_rn(si, re_im[2 * (base + k) + 1]);
            sn = __dadd_rn(sn, ntig[base + k]);
        }
        re_im_c[2 * e] = sr;
        re_im_c[2 * e + 1] = si;
        ntig_c[e] = sn;
    }
}

}  // namespace

}  // namespace amber

using namespace amber;

extern "C" int amber_cuda_grid_vis_collapsed(amber_cuda_ctx *c, long NN, long nc, double dU, double Umax,
                                             float nu_chan0, int flag_key, long ngroups, long npar, long nstokes,
                                             const float *randpar, const float *data, long n_collapse,
                                             double *re_im_out, double *ntig_out)
{
    if (!c) return AMBER_ERR_ARG;
    if (NN <= 0 || NN % 2 || nc <= 0 || !(dU > 0) || ngroups < 0 || npar < 2 || nstokes < 1 ||
        (ngroups > 0 && (!randpar || !data)) || !re_im_out || !ntig_out)
        return fail(c, AMBER_ERR_ARG, "bad gridding arguments");
    if (n_collapse < 1 || nc / n_collapse < 1)
        return fail(c, AMBER_ERR_ARG, "n_collapse %ld must be in 1..nc (%ld)", n_collapse, nc);
    const long ncoll = nc / n_collapse;
    if (flag_key != 0 && flag_key != 1) return fail(c, AMBER_ERR_ARG, "flag_key must be 0 or 1");
    const long H = NN / 2 + 1, ncell = NN * H;
    if (ncell >= (long)UINT32_MAX || ngroups >= (long)UINT32_MAX)
        return fail(c, AMBER_ERR_ARG, "grid or record count too large for 32-bit sort keys");
    cudaSetDevice(c->device);
    const long G = ngroups;
    const size_t rp_b = sizeof(float) * G * npar, dt_b = sizeof(float) * G * nc * nstokes * 3;
    const size_t kv_b = sizeof(unsigned) * std::max<long>(G, 1);
    const size_t out_b = sizeof(double) * ncell * nc * 3, seg_b = sizeof(unsigned) * ncell * 2;
    const size_t coll_b = n_collapse > 1 ? sizeof(double) * ncell * ncoll * 3 : 0;
    size_t cub_b = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, cub_b, (unsigned *)nullptr, (unsigned *)nullptr, (unsigned *)nullptr,
                                    (unsigned *)nullptr, (int)std::max<long>(G, 1));
    auto al = [](size_t b) { return (b + 255) / 256 * 256; };
    size_t total = al(rp_b) + al(dt_b) + 4 * al(kv_b) + al(out_b) + al(coll_b) + al(seg_b) + al(cub_b) + 256;
    int rc = ensure(c, c->mixed_scratch, total, "gridding scratch");
    if (rc) return rc;
    char *p = (char *)c->mixed_scratch.p;
    float *d_rp = (float *)p; p += al(rp_b);
    float *d_dt = (float *)p; p += al(dt_b);
    unsigned *k0 = (unsigned *)p; p += al(kv_b);
    unsigned *v0 = (unsigned *)p; p += al(kv_b);
    unsigned *k1 = (unsigned *)p; p += al(kv_b);
    unsigned *v1 = (unsigned *)p; p += al(kv_b);
    double *d_out = (double *)p; p += al(out_b);
    double *d_coll = (double *)p; p += al(coll_b);
    unsigned *beg = (unsigned *)p; p += al(seg_b);
    unsigned *end = beg + ncell;
    void *d_cub = p; p += al(cub_b);
    int *d_bad = (int *)p;
    cudaStream_t s = c->stream;
    if (G > 0) {
        if ((rc = cuda_check(c, cudaMemcpyAsync(d_rp, randpar, rp_b, cudaMemcpyHostToDevice, s), "upload randpar")))
            return rc;
        if ((rc = cuda_check(c, cudaMemcpyAsync(d_dt, data, dt_b, cudaMemcpyHostToDevice, s), "upload records")))
            return rc;
    }
    cudaMemsetAsync(d_bad, 0, sizeof(int), s);
    cudaMemsetAsync(beg, 0, seg_b, s);
    if (G > 0) {
        cell_kernel<<<(unsigned)((G + 255) / 256), 256, 0, s>>>(d_rp, npar, G, nu_chan0, dU, Umax, NN, ncell, k0, v0,
                                                                d_bad);
        int bits = 1;
        while (bits < 32 && ((long)1 << bits) <= ncell) ++bits;
        cub::DeviceRadixSort::SortPairs(d_cub, cub_b, k0, k1, v0, v1, (int)G, 0, bits, s);
        segment_kernel<<<(unsigned)((G + 255) / 256), 256, 0, s>>>(k1, G, ncell, beg, end);
    }
    dim3 g2((unsigned)ncell, (unsigned)((nc + 127) / 128));
    sum_kernel<<<g2, 128, 0, s>>>(beg, end, v1, d_rp, npar, d_dt, nc, nstokes, flag_key, ncell, d_out,
                                  d_out + 2 * ncell * nc);
    const double *res = d_out;
    if (n_collapse > 1) {
        const long total_c = ncell * ncoll;
        const unsigned blocks = (unsigned)std::min<long>((total_c + 255) / 256, (long)c->num_sms * 16);
        collapse_kernel<<<blocks, 256, 0, s>>>(d_out, d_out + 2 * ncell * nc, ncell, nc, n_collapse, ncoll, d_coll,
                                               d_coll + 2 * ncell * ncoll);
        res = d_coll;
    }
    if ((rc = cuda_check(c, cudaGetLastError(), "gridding kernels"))) return rc;
    int bad = 0;
    cudaMemcpyAsync(&bad, d_bad, sizeof(int), cudaMemcpyDeviceToHost, s);
    if ((rc = cuda_check(c, cudaMemcpyAsync(re_im_out, res, sizeof(double) * 2 * ncell * ncoll,
                                            cudaMemcpyDeviceToHost, s),
                         "download grid")))
        return rc;
    if ((rc = cuda_check(c, cudaMemcpyAsync(ntig_out, res + 2 * ncell * ncoll, sizeof(double) * ncell * ncoll,
                                            cudaMemcpyDeviceToHost, s),
                         "download counts")))
        return rc;
    if ((rc = cuda_check(c, cudaStreamSynchronize(s), "gridding"))) return rc;
    if (bad) return fail(c, AMBER_ERR_ARG, "a record inside Umax maps outside the %ld x %ld grid", NN, H);
    return AMBER_OK;
}

extern "C" int amber_cuda_grid_vis(amber_cuda_ctx *c, long NN, long nc, double dU, double Umax, float nu_chan0,
                                   int flag_key, long ngroups, long npar, long nstokes, const float *randpar,
                                   const float *data, double *re_im_out, double *ntig_out)
{
    return amber_cuda_grid_vis_collapsed(c, NN, nc, dU, Umax, nu_chan0, flag_key, ngroups, npar, nstokes, randpar,
                                         data, 1, re_im_out, ntig_out);
}
